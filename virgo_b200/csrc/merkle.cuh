// Internal entry points shared by the commitment code.
#pragma once
#include "common.cuh"

// Builds nodes 1 .. sz-1 of a heap-ordered tree (digest words, 4 uint64 per
// node) whose sz = n_leaves_padded leaves are already stored at [sz, 2 sz).
int vg_merkle_build(vg_ctx *c, uint64_t *tree, long n_leaves_padded);
// Leaf hash chains of a slice-major codeword set (see vg_leaf_chain).
int vg_leaf_chain_dev(vg_ctx *c, const fe *cw, int n_slices, long n, uint64_t *leaves);
