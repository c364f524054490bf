// Internal entry points shared by the commitment code.
#pragma once
#include "common.cuh"

// Builds nodes 1 .. sz-1 of a heap-ordered tree (digest words, 4 uint64 per
// node) whose sz = n_leaves_padded leaves are already stored at [sz, 2 sz).
int vg_merkle_build(vg_ctx *c, uint64_t *tree, long n_leaves_padded);
// Leaf hash chains of a slice-major codeword set (see vg_leaf_chain).
int vg_leaf_chain_dev(vg_ctx *c, const fe *cw, int n_slices, long n, uint64_t *leaves);

// Batched leaf chains (65 slices each) and Merkle trees of one proof.
constexpr int MAX_HASH_JOBS = 16;
constexpr int MERKLE_TOP = 256;   // parents per tree left to the one-CTA top pass
struct ChainJob {
    const fe *cw;       // slice-major codeword set, 65 slices of n
    long n;
    uint64_t *leaves;   // n / 2 digests
    long begin;         // first thread of this job
};
struct ChainJobs {
    ChainJob j[MAX_HASH_JOBS];
    int count;
    long total;   // threads = sum of n / 2
};
struct TreeJob {
    uint64_t *tree;   // heap-ordered, leaves at [nleaves, 2 nleaves)
    long nleaves;     // power of two
};
struct TreeJobs {
    TreeJob t[MAX_HASH_JOBS];
    int count;
};
int vg_leaf_chains(vg_ctx *c, const ChainJobs &jobs);
// Builds every tree; roots_dev receives 4 words per tree, in job order.
int vg_merkle_trees(vg_ctx *c, const TreeJobs &jobs, uint64_t *roots_dev);
