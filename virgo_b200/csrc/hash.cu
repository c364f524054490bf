// Hash kernels: batched 64-byte hashing, Merkle trees and the FRI leaf hash
// chains.  All are integer-ALU bound (Keccak-f[1600]: 24 rounds of 64-bit
// xor/and-not/rotate; SHA-256: 2 x 64 rounds of 32-bit ops).
#include <mutex>
#include "common.cuh"
// 2^n, n < 32, for the multiply-pipe rotations (VG_MROT_*); filled per device
// at first use (pow2_table)
#define VG_HASH_MULROT 1
static __constant__ uint32_t vg_pow2c[32];
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
template <int KIND, int T>
__global__ void __launch_bounds__(T) k_leaf_chain(const fe *__restrict__ c, int n_slices, long n,
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

// ---- batched forms: every leaf chain and every Merkle tree of a proof ----
// Leaf chains of several codeword sets in one launch: thread t serves leaf
// t - begin of the job whose range holds t.  The next slice's pair is loaded
// before the current hash so the loads overlap the permutation.
template <int KIND, int T, int ROT>
__global__ void __launch_bounds__(T) k_leaf_chains(ChainJobs jobs)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= jobs.total) return;
    int q = 0;
    while (q + 1 < jobs.count && t >= jobs.j[q + 1].begin) ++q;
    const fe *__restrict__ c = jobs.j[q].cw;
    const long n = jobs.j[q].n, half = n >> 1, k = t - jobs.j[q].begin;
    uint64_t h[4] = {0, 0, 0, 0};
    fe a = c[k], b = c[k + half];
    for (int s = 0; s < 65; ++s) {
        fe na = a, nb = b;
        if (s + 1 < 65) {
            na = c[(long)(s + 1) * n + k];
            nb = c[(long)(s + 1) * n + k + half];
        }
        uint64_t w[8] = {a.img, a.real, b.img, b.real, h[0], h[1], h[2], h[3]};
        vg::hash64_rot<KIND, ROT>(w, h);
        a = na;
        b = nb;
    }
    store_digest(jobs.j[q].leaves + 4 * k, h);
}

// ---- leaf chains, one warp per chain (SHA3-256 only) ----
// Lanes 0..3 load the chain's next pair (a.img, a.real, b.img, b.real) as the
// first four message words; lanes 4..7 take the running digest, which the
// previous permutation left in lanes 0..3; lanes 8 and 16 hold the padding.
__device__ __forceinline__ uint64_t chain_word(const fe *__restrict__ c, long off, long half, int l)
{
    const uint64_t *p = (const uint64_t *)(c + off + (l < 2 ? 0 : half));
    return p[l & 1];
}

__device__ __forceinline__ void warp_chain(const fe *__restrict__ c, int n_slices, long n, long k,
                                           uint64_t *__restrict__ out)
{
    const unsigned FULL = 0xffffffffu;
    const int l = threadIdx.x & 31;
    const long half = n >> 1;
    const vg::KeccakLanes K = vg::keccak_lanes(l);
    uint32_t lo = 0, hi = 0;
    uint64_t word = l < 4 ? chain_word(c, k, half, l) : 0;
    for (int s = 0; s < n_slices; ++s) {
        const uint64_t next = (l < 4 && s + 1 < n_slices) ? chain_word(c, (long)(s + 1) * n + k, half, l) : 0;
        const uint32_t dl = __shfl_sync(FULL, lo, (l - 4) & 31), dh = __shfl_sync(FULL, hi, (l - 4) & 31);
        if (l < 4) {
            lo = (uint32_t)word;
            hi = (uint32_t)(word >> 32);
        } else if (l < 8) {
            lo = dl;
            hi = dh;
        } else {
            lo = l == 8 ? 0x06u : 0u;
            hi = l == 16 ? 0x80000000u : 0u;
        }
        vg::keccak_f_warp(lo, hi, K);
        word = next;
    }
    if (l < 4) out[l] = lo | ((uint64_t)hi << 32);
}

constexpr int WARP_CHAIN_THREADS = 128;

__global__ void __launch_bounds__(WARP_CHAIN_THREADS) k_leaf_chains_warp(ChainJobs jobs)
{
    const long w = ((long)blockIdx.x * WARP_CHAIN_THREADS + threadIdx.x) >> 5;
    if (w >= jobs.total) return;   // whole warps
    int q = 0;
    while (q + 1 < jobs.count && w >= jobs.j[q + 1].begin) ++q;
    const long k = w - jobs.j[q].begin;
    warp_chain(jobs.j[q].cw, 65, jobs.j[q].n, k, jobs.j[q].leaves + 4 * k);
}

__global__ void __launch_bounds__(WARP_CHAIN_THREADS) k_leaf_chain_warp(const fe *__restrict__ c, int n_slices, long n,
                                                                       uint64_t *__restrict__ leaves)
{
    const long k = ((long)blockIdx.x * WARP_CHAIN_THREADS + threadIdx.x) >> 5;
    if (k >= (n >> 1)) return;   // whole warps
    warp_chain(c, n_slices, n, k, leaves + 4 * k);
}

static unsigned warp_chain_grid(long chains)
{
    return (unsigned)((chains * 32 + WARP_CHAIN_THREADS - 1) / WARP_CHAIN_THREADS);
}

// leaf hashing form for a launch of `chains` chains: one warp per chain when
// SHA3 and at most VG_TUNE_LEAF_WARP_MAX chains
static bool use_warp_chains(vg_ctx *c, long chains)
{
    return c->hash_kind == VG_HASH_SHA3_256 && chains <= vg_tune_value(c->device, VG_TUNE_LEAF_WARP_MAX);
}

// One Merkle level (parents of height `height`) of every tree that still has
// more than MERKLE_TOP parents there.
template <int KIND>
__global__ void __launch_bounds__(HASH_THREADS) k_merkle_levels(TreeJobs jobs, int height, long total)
{
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    int q = 0;
    for (; q < jobs.count; ++q) {
        const long cnt = jobs.t[q].nleaves >> height;
        if (cnt <= MERKLE_TOP) continue;
        if (t < cnt) break;
        t -= cnt;
    }
    if (q >= jobs.count) return;
    const long p = (jobs.t[q].nleaves >> height) + t;
    uint64_t w[8], d[4];
    load_digest2(jobs.t[q].tree + 8 * p, w);
    vg::hash64<KIND>(w, d);
    store_digest(jobs.t[q].tree + 4 * p, d);
}

// The top MERKLE_TOP parents and above of every tree, one CTA per tree; the
// root is also copied to roots[tree].
template <int KIND>
__global__ void __launch_bounds__(MERKLE_TOP) k_merkle_tops(TreeJobs jobs, uint64_t *__restrict__ roots)
{
    const TreeJob J = jobs.t[blockIdx.x];
    uint64_t *tree = J.tree;
    for (long cnt = J.nleaves >> 1 < MERKLE_TOP ? J.nleaves >> 1 : MERKLE_TOP; cnt >= 1; cnt >>= 1) {
        for (long j = threadIdx.x; j < cnt; j += blockDim.x) {
            const long p = cnt + j;
            uint64_t w[8], d[4];
            load_digest2(tree + 8 * p, w);
            vg::hash64<KIND>(w, d);
            store_digest(tree + 4 * p, d);
        }
        __threadfence_block();
        __syncthreads();
    }
    if (threadIdx.x < 4) roots[4 * blockIdx.x + threadIdx.x] = tree[4 + threadIdx.x];
}

// fills vg_pow2c on the current device, once per device
static int pow2_table(int dev)
{
    static std::mutex mu;
    static std::vector<bool> done;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= (int)done.size()) done.resize(dev + 1, false);
    if (!done[dev]) {
        uint32_t p[32];
        for (int i = 0; i < 32; ++i) p[i] = 1u << i;
        VG_CHECK_CUDA(cudaMemcpyToSymbol(vg_pow2c, p, sizeof p));
        done[dev] = true;
    }
    return VG_OK;
}

int vg_leaf_chains(vg_ctx *c, const ChainJobs &jobs)
{
    if (jobs.total < 1) return VG_OK;
    double bytes = 0;
    for (int q = 0; q < jobs.count; ++q) bytes += 16.0 * 65.0 * (double)jobs.j[q].n + 32.0 * (double)(jobs.j[q].n >> 1);
    ProfScope ps(c, KF_LEAF_CHAIN, bytes);
    if (use_warp_chains(c, jobs.total)) {
        k_leaf_chains_warp<<<warp_chain_grid(jobs.total), WARP_CHAIN_THREADS, 0, c->stream>>>(jobs);
    } else {
        const int T = (int)vg_tune_value(c->device, VG_TUNE_LEAF_THREADS);
        const int rot = c->hash_kind == VG_HASH_SHA3_256 ? (int)vg_tune_value(c->device, VG_TUNE_LEAF_ROT) : 0;
        if (rot == 1 || rot == 2) VG_TRY(pow2_table(c->device));
#define VG_CHAINS_LAUNCH(TT)                                                                                    \
    if (c->hash_kind == VG_HASH_SHA256)                                                                          \
        k_leaf_chains<VG_HASH_SHA256, TT, 0><<<grid_for(jobs.total, TT), TT, 0, c->stream>>>(jobs);             \
    else if (rot == 1)                                                                                           \
        k_leaf_chains<VG_HASH_SHA3_256, TT, 1><<<grid_for(jobs.total, TT), TT, 0, c->stream>>>(jobs);          \
    else if (rot == 2)                                                                                           \
        k_leaf_chains<VG_HASH_SHA3_256, TT, 2><<<grid_for(jobs.total, TT), TT, 0, c->stream>>>(jobs);          \
    else if (rot == 3)                                                                                           \
        k_leaf_chains<VG_HASH_SHA3_256, TT, 3><<<grid_for(jobs.total, TT), TT, 0, c->stream>>>(jobs);          \
    else                                                                                                         \
        k_leaf_chains<VG_HASH_SHA3_256, TT, 0><<<grid_for(jobs.total, TT), TT, 0, c->stream>>>(jobs)
        if (T == 64) VG_CHAINS_LAUNCH(64);
        else if (T == 256) VG_CHAINS_LAUNCH(256);
        else VG_CHAINS_LAUNCH(128);
#undef VG_CHAINS_LAUNCH
    }
    VG_LAUNCHED(c);
    return VG_OK;
}

int vg_merkle_trees(vg_ctx *c, const TreeJobs &jobs, uint64_t *roots_dev)
{
    if (jobs.count < 1) return VG_OK;
    for (int height = 1;; ++height) {
        long total = 0;
        for (int q = 0; q < jobs.count; ++q) {
            const long cnt = jobs.t[q].nleaves >> height;
            if (cnt > MERKLE_TOP) total += cnt;
        }
        if (total == 0) break;
        ProfScope ps(c, KF_MERKLE, 96.0 * (double)total);
        if (c->hash_kind == VG_HASH_SHA256)
            k_merkle_levels<VG_HASH_SHA256><<<grid_for(total, HASH_THREADS), HASH_THREADS, 0, c->stream>>>(jobs, height, total);
        else
            k_merkle_levels<VG_HASH_SHA3_256><<<grid_for(total, HASH_THREADS), HASH_THREADS, 0, c->stream>>>(jobs, height, total);
        VG_LAUNCHED(c);
    }
    ProfScope ps(c, KF_MERKLE, 96.0 * 2.0 * MERKLE_TOP * jobs.count);
    if (c->hash_kind == VG_HASH_SHA256)
        k_merkle_tops<VG_HASH_SHA256><<<jobs.count, MERKLE_TOP, 0, c->stream>>>(jobs, roots_dev);
    else
        k_merkle_tops<VG_HASH_SHA3_256><<<jobs.count, MERKLE_TOP, 0, c->stream>>>(jobs, roots_dev);
    VG_LAUNCHED(c);
    return VG_OK;
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
    if (use_warp_chains(c, half)) {
        k_leaf_chain_warp<<<warp_chain_grid(half), WARP_CHAIN_THREADS, 0, c->stream>>>(cw, n_slices, n, leaves);
    } else {
        const int T = (int)vg_tune_value(c->device, VG_TUNE_LEAF_THREADS);
#define VG_CHAIN_LAUNCH(TT)                                                                                           \
    if (c->hash_kind == VG_HASH_SHA256)                                                                                \
        k_leaf_chain<VG_HASH_SHA256, TT><<<grid_for(half, TT), TT, 0, c->stream>>>(cw, n_slices, n, leaves);          \
    else                                                                                                               \
        k_leaf_chain<VG_HASH_SHA3_256, TT><<<grid_for(half, TT), TT, 0, c->stream>>>(cw, n_slices, n, leaves)
        if (T == 64) VG_CHAIN_LAUNCH(64);
        else if (T == 256) VG_CHAIN_LAUNCH(256);
        else VG_CHAIN_LAUNCH(128);
#undef VG_CHAIN_LAUNCH
    }
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
