// Shared definitions for the virgo_b200 CUDA library: the context object,
// error reporting and launch bookkeeping, and block reductions over F_{p^2}.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string>
#include <vector>
#include "fp2.cuh"
#include "virgo_b200.h"

using vg::fe;

struct TwEntry {
    uint64_t key_real, key_img;  // the root
    int logn;
    fe *lo;   // w^i, i < 4096
    fe *hi;   // w^(4096 j), j < max(1, n / 4096)
    fe *full = nullptr;   // w^e, e < n, for the NTT's column twiddles (small n only), or null
};

// Kernel families timed by the optional per-launch profiler (vg_ctx_profile).
enum KernelFamily {
    KF_NTT = 0, KF_LEAF_CHAIN, KF_MERKLE, KF_FRI_FOLD, KF_VIRTUAL_ORACLE, KF_EVAL, KF_SCATTER1, KF_SCATTER2,
    KF_FINALIZE, KF_ROUND, KF_REDUCE, KF_OTHER, KF_GATHER_ROUND, KF_COUNT
};
struct ProfRec {
    int fam;
    cudaEvent_t a, b;
    double bytes;
    bool shared_a;   // a is the previous record's b (back-to-back launches)
};
struct TraceRec {
    int fam;
    double ms, bytes;
};

struct vg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int hash_kind = VG_HASH_SHA3_256;
    long long launches = 0;
    std::vector<TwEntry> tw_cache;
    // reusable device scratch (grown on demand, freed with the context)
    void *scratch = nullptr;
    size_t scratch_cap = 0;
    void *scratch2 = nullptr;
    size_t scratch2_cap = 0;
    fe *partials = nullptr;  // block partial sums of reductions
    size_t partials_cap = 0;
    fe *pinned = nullptr;    // pinned host staging for small results
    size_t pinned_cap = 0;
    // pinned ring for uploads from pageable host memory (vg_h2d_staged)
    char *ring[2] = {nullptr, nullptr};
    std::vector<void *> retired_pinned;   // outgrown pinned blocks, freed with the context
    cudaEvent_t ring_ev[2] = {nullptr, nullptr};
    // per-launch profiler: event pairs around launches of each kernel family
    bool profiling = false;
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> event_pool;
    std::vector<TraceRec> trace;   // every profiled launch in order
    long long prof_launches[KF_COUNT] = {0};
    double prof_ms[KF_COUNT] = {0}, prof_bytes[KF_COUNT] = {0};
    // back-to-back profiled launches share one event (the end of one is the
    // start of the next), so the profiler adds one event per launch
    bool prof_chain = false;
    cudaEvent_t prof_prev_end = nullptr;
    long long prof_prev_launches = -1;
};

// Profiler hooks around one launch: no-ops unless profiling is on.  Events are
// recorded on the context stream without synchronising; vg_ctx_profile_read
// resolves them.
void vg_prof_begin(vg_ctx *c, int fam, ProfRec *r);
void vg_prof_end(vg_ctx *c, ProfRec *r, double bytes);
struct ProfScope {
    vg_ctx *c;
    ProfRec r;
    double bytes;
    bool on;
    ProfScope(vg_ctx *ctx, int fam, double b) : c(ctx), bytes(b), on(ctx->profiling)
    {
        if (on) vg_prof_begin(c, fam, &r);
    }
    ~ProfScope()
    {
        if (on) vg_prof_end(c, &r, bytes);
    }
};

// ---- errors ----
int vg_fail(int code, const char *fmt, ...);
#define VG_CHECK_CUDA(call)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return vg_fail(VG_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,        \
                           cudaGetErrorString(e_));                                      \
    } while (0)
#define VG_TRY(expr)                   \
    do {                               \
        int rc_ = (expr);              \
        if (rc_ != VG_OK) return rc_;  \
    } while (0)
#define VG_LAUNCHED(ctx)                                                                   \
    do {                                                                                   \
        (ctx)->launches++;                                                                 \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess)                                                             \
            return vg_fail(VG_ERR_CUDA, "%s:%d launch: %s", __FILE__, __LINE__,             \
                           cudaGetErrorString(e_));                                        \
    } while (0)

// Host-to-device copy on the context stream.  Pageable sources go through the
// context's two pinned chunks (host memcpy of one chunk overlaps the DMA of
// the other), so concurrent sessions do not serialise on the driver's
// staging.  A pageable source may be reused on return; a pinned or device
// source is copied directly and must stay valid until the stream reaches the
// copy.
int vg_h2d_staged(vg_ctx *c, void *dst, const void *src, size_t bytes);

// Grows a pinned host buffer geometrically without synchronising: the
// outgrown block is retired (freed when the context is destroyed), since
// cudaFreeHost would wait for the whole device.
int vg_pinned_grow(vg_ctx *c, void **p, size_t *cap, size_t bytes);

// stream-ordered device memory from the device pool (see ctx.cu)
int vg_alloc(vg_ctx *c, void **p, size_t bytes);
void vg_release(vg_ctx *c, void *p);

// scratch buffers owned by the context; contents do not survive other calls
int vg_scratch(vg_ctx *ctx, size_t bytes, void **p);
int vg_scratch2(vg_ctx *ctx, size_t bytes, void **p);
int vg_partials(vg_ctx *ctx, size_t n, fe **p);
int vg_pinned(vg_ctx *ctx, size_t n, fe **p);
int vg_twiddles(vg_ctx *ctx, fe root, int logn, const fe **lo, const fe **hi);
bool vg_is_device_ptr(const void *p);

static inline unsigned grid_for(long n, int threads)
{
    long g = (n + threads - 1) / threads;
    return (unsigned)(g < 1 ? 1 : g);
}

// ---- reductions ----
__device__ __forceinline__ fe shfl_down_fe(fe x, int off)
{
    fe r;
    r.real = __shfl_down_sync(0xffffffffu, x.real, off);
    r.img = __shfl_down_sync(0xffffffffu, x.img, off);
    return r;
}
__device__ __forceinline__ fe warp_sum(fe x)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x = x + shfl_down_fe(x, off);
    return x;
}
// Sum of K values over the block; result valid in thread 0.  sm holds
// K * 32 elements.  Field addition is exact and commutative, so the result is
// independent of the reduction order.
template <int K>
__device__ __forceinline__ void block_sum(fe (&v)[K], fe *sm)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) sm[k * 32 + wid] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            fe x = lane < nw ? sm[k * 32 + lane] : vg::fe_zero();
            v[k] = warp_sum(x);
        }
    }
}

// sum of `nparts` groups of K partials (layout [part][K]) into out[K]
int vg_reduce_partials(vg_ctx *ctx, const fe *parts, int nparts, int K, fe *out_dev);

// Exclusive prefix sum of d[0 .. n) in place, d[n] (zero on entry) receives
// the total; tmp holds vg_scan_tmp_words(n) words.
long vg_scan_tmp_words(long n);
int vg_scan_u32(vg_ctx *c, uint32_t *d, long n, uint32_t *tmp);

// The device's launch-shape parameter `key` (VG_TUNE_*; tune.cu).
long vg_tune_value(int device, int key);
