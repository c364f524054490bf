// Hash kernels: batched 64-byte hashing, Merkle trees and the FRI leaf hash
// chains.  All are integer-ALU bound (Keccak-f[1600]: 24 rounds of 64-bit
// xor/and-not/rotate; SHA-256: 2 x 64 rounds of 32-bit ops).
#include "common.cuh"
#include "hash.cuh"
#include "merkle.cuh"

namespace {

constexpr int HASH_THREADS = 128;

__device__ __forceinline__ void load_digest2(const uint64_t *p, uint64_t w[8])
{
    const ulonglong2 *q = (const ulonglong2 *)p;
    ulonglong2 a = q[0], b = q[1], c = q[2], d = q[3];
    w[0] = a.x; w[1] = a.y; w[2] = b.x; w[3] = b.y; w[4] = c.x; w[5] = c.y; w[6] = d.x; w[7] = d.y;
}
__device__ __forceinline__ void store_digest(uint64_t *p, const uint64_t d[4])
{
    ulonglong2 *q = (ulonglong2 *)p;
    q[0] = make_ulonglong2(d[0], d[1]);
    q[1] = make_ulonglong2(d[2], d[3]);
}

template <int KIND>
__global__ void k_hash64(const uint64_t *__restrict__ msgs, uint64_t *__restrict__ out, long n)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t w[8], d[4];
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = msgs[i * 8 + k];
    vg::hash64<KIND>(w, d);
#pragma unroll
    for (int k = 0; k < 4; ++k) out[i * 4 + k] = d[k];
}

}  // namespace

// ---- Merkle levels ----
template <int KIND>
__global__ void k_merkle_level(uint64_t *__restrict__ tree, long first, long count)
{
    // parents tree[first .. first+count) from children tree[2 first ..)
    long j = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (j >= count) return;
    long p = first + j;
    uint64_t w[8], d[4];
    load_digest2(tree + 8 * p, w);   // children 2p, 2p+1 are contiguous
    vg::hash64<KIND>(w, d);
    store_digest(tree + 4 * p, d);
}

// The top levels of a tree (at most 2 * MERKLE_TOP nodes below node 1) in one
// CTA: each level waits for the one below with __syncthreads.
template <int KIND>
__global__ void k_merkle_top(uint64_t *__restrict__ tree, long width)
{
    for (long cnt = width; cnt >= 1; cnt >>= 1) {
        for (long j = threadIdx.x; j < cnt; j += blockDim.x) {
            long p = cnt + j;
            uint64_t w[8], d[4];
            load_digest2(tree + 8 * p, w);
            vg::hash64<KIND>(w, d);
            store_digest(tree + 4 * p, d);
        }
        __threadfence_block();
        __syncthreads();
    }
}

template <int KIND>
__global__ void k_fill_pad(uint64_t *__restrict__ tree, long from, long to)
{
    long i = from + blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= to) return;
    uint64_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0}, d[4];
    vg::hash64<KIND>(w, d);
    store_digest(tree + 4 * i, d);
}

// ---- leaf hash chains ----
// Leaf k of a codeword set with per-slice length n: h = 0; for s:
// h = H(c[s][k] || c[s][k + n/2] || h).  One thread per leaf; a warp reads
// 32 consecutive k of one slice, i.e. 512 contiguous bytes per load.
template <int KIND>
__global__ void __launch_bounds__(HASH_THREADS) k_leaf_chain(const fe *__restrict__ c, int n_slices, long n,
                                                            uint64_t *__restrict__ leaves)
{
    const long half = n >> 1;
    long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (k >= half) return;
    uint64_t h[4] = {0, 0, 0, 0};
    for (int s = 0; s < n_slices; ++s) {
        fe a = c[(long)s * n + k], b = c[(long)s * n + k + half];
        uint64_t w[8] = {a.img, a.real, b.img, b.real, h[0], h[1], h[2], h[3]};
        vg::hash64<KIND>(w, h);
    }
    store_digest(leaves + 4 * k, h);
}

// ------------------------------------------------------------------ host
int vg_merkle_build(vg_ctx *c, uint64_t *tree, long n_leaves_padded)
{
    // leaves already in tree[sz .. 2 sz); builds nodes 1 .. sz-1
    const long TOP = 1024;
    long cnt = n_leaves_padded >> 1;
    while (cnt > TOP) {
        ProfScope ps(c, KF_MERKLE, 96.0 * (double)cnt);
        if (c->hash_kind == VG_HASH_SHA256)
            k_merkle_level<VG_HASH_SHA256><<<grid_for(cnt, HASH_THREADS), HASH_THREADS, 0, c->stream>>>(tree, cnt, cnt);
        else
            k_merkle_level<VG_HASH_SHA3_256><<<grid_for(cnt, HASH_THREADS), HASH_THREADS, 0, c->stream>>>(tree, cnt, cnt);
        VG_LAUNCHED(c);
        cnt >>= 1;
    }
    if (cnt >= 1) {
        ProfScope ps(c, KF_MERKLE, 96.0 * (double)(2 * cnt));
        if (c->hash_kind == VG_HASH_SHA256)
            k_merkle_top<VG_HASH_SHA256><<<1, 512, 0, c->stream>>>(tree, cnt);
        else
            k_merkle_top<VG_HASH_SHA3_256><<<1, 512, 0, c->stream>>>(tree, cnt);
        VG_LAUNCHED(c);
    }
    return VG_OK;
}

int vg_leaf_chain_dev(vg_ctx *c, const fe *cw, int n_slices, long n, uint64_t *leaves)
{
    long half = n >> 1;
    if (half < 1) return VG_OK;
    ProfScope ps(c, KF_LEAF_CHAIN, 16.0 * (double)n_slices * (double)n + 32.0 * (double)half);
    if (c->hash_kind == VG_HASH_SHA256)
        k_leaf_chain<VG_HASH_SHA256><<<grid_for(half, HASH_THREADS), HASH_THREADS, 0, c->stream>>>(cw, n_slices, n, leaves);
    else
        k_leaf_chain<VG_HASH_SHA3_256><<<grid_for(half, HASH_THREADS), HASH_THREADS, 0, c->stream>>>(cw, n_slices, n, leaves);
    VG_LAUNCHED(c);
    return VG_OK;
}

extern "C" int vg_hash64(vg_ctx *c, const void *msgs, void *digests, long n)
{
    if (!c || !msgs || !digests || n < 0) return vg_fail(VG_ERR_ARG, "vg_hash64: bad argument");
    if (n == 0) return VG_OK;
    if (c->hash_kind == VG_HASH_SHA256)
        k_hash64<VG_HASH_SHA256><<<grid_for(n, HASH_THREADS), HASH_THREADS, 0, c->stream>>>((const uint64_t *)msgs, (uint64_t *)digests, n);
    else
        k_hash64<VG_HASH_SHA3_256><<<grid_for(n, HASH_THREADS), HASH_THREADS, 0, c->stream>>>((const uint64_t *)msgs, (uint64_t *)digests, n);
    VG_LAUNCHED(c);
    return VG_OK;
}

extern "C" int vg_merkle_tree(vg_ctx *c, const vg_digest *leaves, long n, vg_digest *tree)
{
    if (!c || !leaves || !tree || n < 1) return vg_fail(VG_ERR_ARG, "vg_merkle_tree: bad argument");
    long sz = 1;
    while (sz < n) sz <<= 1;
    VG_CHECK_CUDA(cudaMemsetAsync(tree, 0, 2 * sz * sizeof(vg_digest), c->stream));
    VG_CHECK_CUDA(cudaMemcpyAsync(tree + sz, leaves, n * sizeof(vg_digest), cudaMemcpyDeviceToDevice, c->stream));
    if (n < sz) {
        if (c->hash_kind == VG_HASH_SHA256)
            k_fill_pad<VG_HASH_SHA256><<<grid_for(sz - n, HASH_THREADS), HASH_THREADS, 0, c->stream>>>((uint64_t *)tree, sz + n, 2 * sz);
        else
            k_fill_pad<VG_HASH_SHA3_256><<<grid_for(sz - n, HASH_THREADS), HASH_THREADS, 0, c->stream>>>((uint64_t *)tree, sz + n, 2 * sz);
        VG_LAUNCHED(c);
    }
    return vg_merkle_build(c, (uint64_t *)tree, sz);
}

extern "C" int vg_leaf_chain(vg_ctx *c, const vg_fe *cw, int n_slices, long n, vg_digest *leaves)
{
    if (!c || !cw || !leaves || n_slices < 1 || n < 2 || (n & (n - 1)))
        return vg_fail(VG_ERR_ARG, "vg_leaf_chain: bad argument");
    return vg_leaf_chain_dev(c, (const fe *)cw, n_slices, n, (uint64_t *)leaves);
}
