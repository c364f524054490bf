#include <cstdlib>
#include <cstring>
#include <algorithm>
// Context, device memory, error reporting, elementwise field ops and the
// generic partial-sum reduction.
#include "common.cuh"
#include <mutex>

static thread_local std::string g_err;

int vg_fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

extern "C" const char *vg_last_error(void) { return g_err.c_str(); }

// Concurrent sessions run three streams each (sumcheck, commitment, side
// proof); with CUDA's default of 8 hardware work queues per device, streams
// beyond the eighth share a queue and their kernels wait on each other's.
// The variable is read when the process creates its CUDA context, so it takes
// effect only when this library makes the process's first CUDA call, and a
// value the caller set is kept.
static void default_connections()
{
    static std::once_flag once;
    std::call_once(once, [] { setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0); });
}

extern "C" int vg_ctx_create(int device, vg_ctx **out)
{
    if (!out) return vg_fail(VG_ERR_ARG, "vg_ctx_create: null out");
    default_connections();
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return vg_fail(VG_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= n) return vg_fail(VG_ERR_ARG, "device %d out of range (%d)", device, n);
    VG_CHECK_CUDA(cudaSetDevice(device));
    vg_ctx *c = new vg_ctx();
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return vg_fail(VG_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    *out = c;
    return VG_OK;
}

// Gives the context's stream the device's highest scheduling priority (a new
// stream; the old one is drained and destroyed).  For a stream that carries
// a proof's critical path, so that concurrent work on other streams fills
// the SMs it leaves idle instead of delaying it.
int vg_ctx_raise_priority(vg_ctx *c)
{
    if (!c) return vg_fail(VG_ERR_ARG, "vg_ctx_raise_priority: null context");
    VG_CHECK_CUDA(cudaSetDevice(c->device));
    int least = 0, greatest = 0;
    VG_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    if (greatest == least) return VG_OK;
    cudaStream_t s;
    VG_CHECK_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    cudaStreamDestroy(c->stream);
    c->stream = s;
    return VG_OK;
}

static cudaEvent_t get_event(vg_ctx *c)
{
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// A launch that directly follows the previous profiled one on the stream
// (exactly one launch since that one began) starts at its end event; an
// event pair around every launch would add several microseconds to each.
void vg_prof_begin(vg_ctx *c, int fam, ProfRec *r)
{
    r->fam = fam;
    r->shared_a = c->prof_chain && c->launches == c->prof_prev_launches + 1;
    if (r->shared_a) {
        r->a = c->prof_prev_end;
    } else {
        r->a = get_event(c);
        cudaEventRecord(r->a, c->stream);
    }
    r->b = get_event(c);
    c->prof_prev_launches = c->launches;
}

void vg_prof_end(vg_ctx *c, ProfRec *r, double bytes)
{
    cudaEventRecord(r->b, c->stream);
    c->prof_prev_end = r->b;
    c->prof_chain = true;
    r->bytes = bytes;
    c->prof.push_back(*r);
    if (c->prof.size() > 4096) {   // resolve in batches to bound the event count
        cudaStreamSynchronize(c->stream);
        for (auto &p : c->prof) {
            float ms = 0;
            cudaEventElapsedTime(&ms, p.a, p.b);
            if (c->trace.size() < 1000000) c->trace.push_back({p.fam, ms, p.bytes});
            c->prof_launches[p.fam]++;
            c->prof_ms[p.fam] += ms;
            c->prof_bytes[p.fam] += p.bytes;
            if (!p.shared_a) c->event_pool.push_back(p.a);
            c->event_pool.push_back(p.b);
        }
        c->prof.clear();
        c->prof_chain = false;   // the last end event went back to the pool
    }
}

extern "C" int vg_ctx_profile(vg_ctx *c, int enable)
{
    if (!c) return vg_fail(VG_ERR_ARG, "null ctx");
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    c->profiling = enable != 0;
    c->prof_chain = false;
    for (auto &p : c->prof) {
        if (!p.shared_a) c->event_pool.push_back(p.a);
        c->event_pool.push_back(p.b);
    }
    c->prof.clear();
    c->trace.clear();
    for (int k = 0; k < KF_COUNT; ++k) {
        c->prof_launches[k] = 0;
        c->prof_ms[k] = c->prof_bytes[k] = 0;
    }
    return VG_OK;
}

extern "C" int vg_ctx_profile_read(vg_ctx *c, int family, long long *launches, double *ms, double *bytes)
{
    if (!c || family < 0 || family >= KF_COUNT) return vg_fail(VG_ERR_ARG, "vg_ctx_profile_read: bad family");
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    for (auto &p : c->prof) {
        float t = 0;
        cudaEventElapsedTime(&t, p.a, p.b);
        if (c->trace.size() < 1000000) c->trace.push_back({p.fam, t, p.bytes});
        c->prof_launches[p.fam]++;
        c->prof_ms[p.fam] += t;
        c->prof_bytes[p.fam] += p.bytes;
        if (!p.shared_a) c->event_pool.push_back(p.a);
        c->event_pool.push_back(p.b);
    }
    c->prof.clear();
    c->prof_chain = false;
    if (launches) *launches = c->prof_launches[family];
    if (ms) *ms = c->prof_ms[family];
    if (bytes) *bytes = c->prof_bytes[family];
    return VG_OK;
}

extern "C" int vg_ctx_profile_trace(vg_ctx *c, int *family, double *ms, double *bytes, long max, long *n)
{
    if (!c || !n) return vg_fail(VG_ERR_ARG, "vg_ctx_profile_trace: null argument");
    VG_TRY(vg_ctx_profile_read(c, 0, nullptr, nullptr, nullptr));   // resolves pending events
    const long k = std::min<long>(max, (long)c->trace.size());
    for (long i = 0; i < k; ++i) {
        if (family) family[i] = c->trace[i].fam;
        if (ms) ms[i] = c->trace[i].ms;
        if (bytes) bytes[i] = c->trace[i].bytes;
    }
    *n = (long)c->trace.size();
    return VG_OK;
}

extern "C" int vg_timer_start(vg_ctx *c, void **timer)
{
    if (!c || !timer) return vg_fail(VG_ERR_ARG, "null argument");
    cudaEvent_t *ev = new cudaEvent_t[2];
    VG_CHECK_CUDA(cudaEventCreate(&ev[0]));
    VG_CHECK_CUDA(cudaEventCreate(&ev[1]));
    VG_CHECK_CUDA(cudaEventRecord(ev[0], c->stream));
    *timer = ev;
    return VG_OK;
}

extern "C" int vg_timer_stop(vg_ctx *c, void *timer, double *ms)
{
    if (!c || !timer || !ms) return vg_fail(VG_ERR_ARG, "null argument");
    cudaEvent_t *ev = (cudaEvent_t *)timer;
    VG_CHECK_CUDA(cudaEventRecord(ev[1], c->stream));
    VG_CHECK_CUDA(cudaEventSynchronize(ev[1]));
    float t = 0;
    VG_CHECK_CUDA(cudaEventElapsedTime(&t, ev[0], ev[1]));
    *ms = t;
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    delete[] ev;
    return VG_OK;
}

extern "C" int vg_timer_stop_multi(vg_ctx *const *ctxs, int n, void *timer, double *ms)
{
    if (!ctxs || n < 1 || !timer || !ms) return vg_fail(VG_ERR_ARG, "null argument");
    cudaEvent_t *ev = (cudaEvent_t *)timer;
    double worst = 0;
    for (int i = 0; i < n; ++i) {
        cudaEvent_t e;
        VG_CHECK_CUDA(cudaEventCreate(&e));
        VG_CHECK_CUDA(cudaEventRecord(e, ctxs[i]->stream));
        VG_CHECK_CUDA(cudaEventSynchronize(e));
        float t = 0;
        VG_CHECK_CUDA(cudaEventElapsedTime(&t, ev[0], e));
        if (t > worst) worst = t;
        cudaEventDestroy(e);
    }
    *ms = worst;
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    delete[] ev;
    return VG_OK;
}

extern "C" int vg_ctx_destroy(vg_ctx *c)
{
    if (!c) return VG_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto &p : c->prof) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : c->event_pool) cudaEventDestroy(e);
    for (auto &t : c->tw_cache) {
        cudaFree(t.lo);
        cudaFree(t.hi);
        if (t.full) cudaFree(t.full);
    }
    if (c->scratch) cudaFree(c->scratch);
    if (c->scratch2) cudaFree(c->scratch2);
    if (c->partials) cudaFree(c->partials);
    if (c->pinned) cudaFreeHost(c->pinned);
    for (void *q : c->retired_pinned) cudaFreeHost(q);
    for (int k = 0; k < 2; ++k) {
        if (c->ring[k]) cudaFreeHost(c->ring[k]);
        if (c->ring_ev[k]) cudaEventDestroy(c->ring_ev[k]);
    }
    cudaStreamDestroy(c->stream);
    delete c;
    return VG_OK;
}

extern "C" int vg_ctx_set_hash(vg_ctx *c, int kind)
{
    if (!c) return vg_fail(VG_ERR_ARG, "null ctx");
    if (kind != VG_HASH_SHA3_256 && kind != VG_HASH_SHA256) return vg_fail(VG_ERR_ARG, "unknown hash kind %d", kind);
    c->hash_kind = kind;
    return VG_OK;
}
extern "C" int vg_ctx_get_hash(vg_ctx *c, int *kind)
{
    if (!c || !kind) return vg_fail(VG_ERR_ARG, "null argument");
    *kind = c->hash_kind;
    return VG_OK;
}

extern "C" int vg_ctx_device(vg_ctx *c, int *device)
{
    if (!c || !device) return vg_fail(VG_ERR_ARG, "null argument");
    *device = c->device;
    return VG_OK;
}

extern "C" int vg_ctx_sync(vg_ctx *c)
{
    if (!c) return vg_fail(VG_ERR_ARG, "null ctx");
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return VG_OK;
}

extern "C" int vg_ctx_launch_count(vg_ctx *c, long long *count)
{
    if (!c || !count) return vg_fail(VG_ERR_ARG, "null argument");
    *count = c->launches;
    return VG_OK;
}

// Stream-ordered allocations from the device's default memory pool.  The
// pool keeps freed blocks (its release threshold is raised once per device),
// so growing a buffer neither synchronises the device, as cudaFree does, nor
// returns memory to the driver between proofs.
static int pool_setup(int dev)
{
    static std::mutex mu;
    static std::vector<bool> done;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= (int)done.size()) done.resize(dev + 1, false);
    if (done[dev]) return VG_OK;
    cudaMemPool_t pool;
    VG_CHECK_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = ~0ull;
    VG_CHECK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    done[dev] = true;
    return VG_OK;
}

int vg_alloc(vg_ctx *c, void **p, size_t bytes)
{
    VG_TRY(pool_setup(c->device));
    cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return vg_fail(VG_ERR_OOM, "device allocation of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    return VG_OK;
}

void vg_release(vg_ctx *c, void *p)
{
    if (p) cudaFreeAsync(p, c->stream);
}

constexpr size_t RING_CHUNK = 8u << 20;

int vg_h2d_staged(vg_ctx *c, void *dst, const void *src, size_t bytes)
{
    if (!bytes) return VG_OK;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, src) == cudaSuccess && a.type != cudaMemoryTypeUnregistered) {
        VG_CHECK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));
        return VG_OK;   // pinned or device source: in flight until the stream gets there
    }
    cudaGetLastError();
    if (!c->ring[0]) {
        for (int k = 0; k < 2; ++k) {
            VG_CHECK_CUDA(cudaMallocHost((void **)&c->ring[k], RING_CHUNK));
            VG_CHECK_CUDA(cudaEventCreateWithFlags(&c->ring_ev[k], cudaEventDisableTiming));
            VG_CHECK_CUDA(cudaEventRecord(c->ring_ev[k], c->stream));
        }
    }
    int k = 0;
    for (size_t off = 0; off < bytes; off += RING_CHUNK, k ^= 1) {
        const size_t len = std::min(RING_CHUNK, bytes - off);
        VG_CHECK_CUDA(cudaEventSynchronize(c->ring_ev[k]));   // the chunk's previous copy is done
        memcpy(c->ring[k], (const char *)src + off, len);
        VG_CHECK_CUDA(cudaMemcpyAsync((char *)dst + off, c->ring[k], len, cudaMemcpyHostToDevice, c->stream));
        VG_CHECK_CUDA(cudaEventRecord(c->ring_ev[k], c->stream));
    }
    return VG_OK;
}

static int grow(vg_ctx *c, void **p, size_t *cap, size_t bytes)
{
    if (bytes <= *cap) return VG_OK;
    vg_release(c, *p);
    *p = nullptr;
    *cap = 0;
    VG_TRY(vg_alloc(c, p, bytes));
    *cap = bytes;
    return VG_OK;
}

int vg_scratch(vg_ctx *c, size_t bytes, void **p)
{
    VG_TRY(grow(c, &c->scratch, &c->scratch_cap, bytes));
    *p = c->scratch;
    return VG_OK;
}
int vg_scratch2(vg_ctx *c, size_t bytes, void **p)
{
    VG_TRY(grow(c, &c->scratch2, &c->scratch2_cap, bytes));
    *p = c->scratch2;
    return VG_OK;
}
int vg_partials(vg_ctx *c, size_t n, fe **p)
{
    void *q = c->partials;
    VG_TRY(grow(c, &q, &c->partials_cap, n * sizeof(fe)));
    c->partials = (fe *)q;
    *p = c->partials;
    return VG_OK;
}
int vg_pinned_grow(vg_ctx *c, void **p, size_t *cap, size_t bytes)
{
    if (bytes <= *cap) return VG_OK;
    size_t ncap = std::max(bytes, std::max(2 * *cap, (size_t)1 << 20));
    void *q = nullptr;
    VG_CHECK_CUDA(cudaMallocHost(&q, ncap));
    if (*p) c->retired_pinned.push_back(*p);
    *p = q;
    *cap = ncap;
    return VG_OK;
}

int vg_pinned(vg_ctx *c, size_t n, fe **p)
{
    void *q = c->pinned;
    VG_TRY(vg_pinned_grow(c, &q, &c->pinned_cap, n * sizeof(fe)));
    c->pinned = (fe *)q;
    *p = c->pinned;
    return VG_OK;
}

int vg_ctx_grow_dev(vg_ctx *c, void **p, size_t *cap, size_t bytes) { return grow(c, p, cap, bytes); }

int vg_ctx_wait_for(vg_ctx *waiter, vg_ctx *signaler)
{
    if (!waiter || !signaler) return vg_fail(VG_ERR_ARG, "vg_ctx_wait_for: null context");
    cudaEvent_t e;
    VG_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t rc = cudaEventRecord(e, signaler->stream);
    if (rc == cudaSuccess) rc = cudaStreamWaitEvent(waiter->stream, e, 0);
    cudaEventDestroy(e);   // released once the wait is resolved
    VG_CHECK_CUDA(rc);
    return VG_OK;
}

bool vg_is_device_ptr(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

extern "C" int vg_dev_alloc(vg_ctx *c, size_t bytes, void **dev)
{
    if (!c || !dev) return vg_fail(VG_ERR_ARG, "null argument");
    cudaError_t e = cudaMalloc(dev, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *dev = nullptr;
        return vg_fail(VG_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    return VG_OK;
}
extern "C" int vg_dev_free(vg_ctx *c, void *dev)
{
    if (!c) return vg_fail(VG_ERR_ARG, "null ctx");
    if (dev) {
        VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
        VG_CHECK_CUDA(cudaFree(dev));
    }
    return VG_OK;
}
extern "C" int vg_h2d(vg_ctx *c, void *dev, const void *host, size_t bytes)
{
    if (!c) return vg_fail(VG_ERR_ARG, "null ctx");
    VG_CHECK_CUDA(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyDefault, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return VG_OK;
}
extern "C" int vg_d2h(vg_ctx *c, void *host, const void *dev, size_t bytes)
{
    if (!c) return vg_fail(VG_ERR_ARG, "null ctx");
    VG_CHECK_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDefault, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return VG_OK;
}

// ------------------------------------------------------------ field binop
__global__ void k_binop(int op, const fe *__restrict__ a, const fe *__restrict__ b, fe *__restrict__ c, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        fe x = a[i], y = b[i];
        c[i] = op == 0 ? x + y : (op == 1 ? x - y : x * y);
    }
}

extern "C" int vg_fe_binop(vg_ctx *c, int op, const vg_fe *a, const vg_fe *b, vg_fe *out, long n)
{
    if (!c || !a || !b || !out || n < 0 || op < 0 || op > 2) return vg_fail(VG_ERR_ARG, "vg_fe_binop: bad argument");
    if (n == 0) return VG_OK;
    unsigned g = grid_for(n, 256);
    if (g > 148 * 32) g = 148 * 32;
    k_binop<<<g, 256, 0, c->stream>>>(op, (const fe *)a, (const fe *)b, (fe *)out, n);
    VG_LAUNCHED(c);
    return VG_OK;
}

// ------------------------------------------------------- partial reductions
template <int K>
__global__ void k_reduce_parts(const fe *__restrict__ parts, int nparts, fe *__restrict__ out)
{
    __shared__ fe sm[K * 32];
    fe v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = vg::fe_zero();
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = v[k] + parts[(long)i * K + k];
    }
    block_sum<K>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = v[k];
    }
}

int vg_reduce_partials(vg_ctx *c, const fe *parts, int nparts, int K, fe *out_dev)
{
    ProfScope ps(c, KF_REDUCE, 16.0 * (double)nparts * K);
    switch (K) {
    case 1: k_reduce_parts<1><<<1, 1024, 0, c->stream>>>(parts, nparts, out_dev); break;
    case 3: k_reduce_parts<3><<<1, 1024, 0, c->stream>>>(parts, nparts, out_dev); break;
    case 14: k_reduce_parts<14><<<1, 256, 0, c->stream>>>(parts, nparts, out_dev); break;
    default: return vg_fail(VG_ERR_ARG, "vg_reduce_partials: K=%d unsupported", K);
    }
    VG_LAUNCHED(c);
    return VG_OK;
}

// ------------------------------------------------------------ prefix sums
namespace {
constexpr int SCAN_THREADS = 1024, SCAN_TILE = 2 * SCAN_THREADS;

// exclusive scan of each tile of SCAN_TILE entries in place; tile totals to sums
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(uint32_t *__restrict__ d, long n, uint32_t *__restrict__ sums)
{
    __shared__ uint32_t s[SCAN_TILE];
    const long base = (long)blockIdx.x * SCAN_TILE;
    const int t = threadIdx.x;
    s[2 * t] = base + 2 * t < n ? d[base + 2 * t] : 0;
    s[2 * t + 1] = base + 2 * t + 1 < n ? d[base + 2 * t + 1] : 0;
    // work-efficient (up-sweep / down-sweep) scan
    int off = 1;
    for (int w = SCAN_TILE >> 1; w > 0; w >>= 1) {
        __syncthreads();
        if (t < w) {
            const int a = off * (2 * t + 1) - 1, b = off * (2 * t + 2) - 1;
            s[b] += s[a];
        }
        off <<= 1;
    }
    if (t == 0) {
        sums[blockIdx.x] = s[SCAN_TILE - 1];
        s[SCAN_TILE - 1] = 0;
    }
    for (int w = 1; w < SCAN_TILE; w <<= 1) {
        off >>= 1;
        __syncthreads();
        if (t < w) {
            const int a = off * (2 * t + 1) - 1, b = off * (2 * t + 2) - 1;
            const uint32_t x = s[a];
            s[a] = s[b];
            s[b] += x;
        }
    }
    __syncthreads();
    if (base + 2 * t < n) d[base + 2 * t] = s[2 * t];
    if (base + 2 * t + 1 < n) d[base + 2 * t + 1] = s[2 * t + 1];
}

__global__ void k_scan_add(uint32_t *__restrict__ d, long n, const uint32_t *__restrict__ offs)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) d[i] += offs[i / SCAN_TILE];
}
}  // namespace

// Exclusive prefix sum of d[0 .. n) in place; d[n] receives the total.  tmp
// needs vg_scan_tmp_words(n) words.
long vg_scan_tmp_words(long n)
{
    long w = 0;
    for (long m = n + 1; m > 1; m = (m + SCAN_TILE - 1) / SCAN_TILE) w += (m + SCAN_TILE - 1) / SCAN_TILE + 1;
    return w + 1;
}

int vg_scan_u32(vg_ctx *c, uint32_t *d, long n, uint32_t *tmp)
{
    // scan n + 1 entries (d[n] = 0 on entry after the caller's counts) so the
    // last entry becomes the total
    const long m = n + 1;
    const long tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, c->stream>>>(d, m, tmp);
    VG_LAUNCHED(c);
    if (tiles > 1) {
        VG_TRY(vg_scan_u32(c, tmp, tiles - 1, tmp + tiles + 1));   // tmp[0 .. tiles) exclusive
        k_scan_add<<<grid_for(m, 256), 256, 0, c->stream>>>(d, m, tmp);
        VG_LAUNCHED(c);
    }
    return VG_OK;
}
