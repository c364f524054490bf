// vg_mle_eval_noalloc: the multilinear evaluation of vg_mle_eval for callers
// that must not allocate device memory.
//
// Who needs it: a host whose memory pool has already reserved the whole GPU
// (cudaMalloc would fail), code that must not take the device-wide
// synchronisation of cudaFree on a latency-critical path, and embedders with a
// fixed device-memory budget.  The call works entirely in one file-scope
// device array of 16,760 field elements (268,160 bytes); every GPU that loads
// this library holds its own copy of the array until the process exits.
//
// Contract (also in include/virgo_b200.h):
//   - vals is device memory (n >= 2^log_n entries), r and out host memory;
//   - log_n <= NOALLOC_MAX_LOG (26); larger sizes are rejected with
//     VG_ERR_ARG and a message before anything touches the GPU;
//   - the kernels run on the legacy default stream, which does not wait for
//     work on non-blocking streams (this library's context streams are
//     non-blocking): a caller whose vals come from such a stream must
//     synchronise it first (vg_ctx_sync for a library context);
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it, so make
//     that first call before any stream capture.  The cache is per device and
//     per process: after cudaDeviceReset of a device the cached address is
//     no longer valid, so do not call this entry point on that device again
//     in the same process;
//   - every call on a device reuses that device's array and it keeps the
//     previous call's contents; each call writes every region before reading
//     it, so nothing has to start at zero.  Calls on the same device that
//     overlap on the GPU (two host threads, two streams) race: serialise them;
//   - the call returns after the result is copied to out.
#include "common.cuh"
#include <mutex>

namespace {

constexpr int NOALLOC_MAX_LOG = 26;
constexpr int NOALLOC_BLOCKS = 296;
constexpr long NOALLOC_HALF = 1L << (NOALLOC_MAX_LOG - NOALLOC_MAX_LOG / 2);   // 8192
// r (64) | lo table (8192) | hi table (8192) | block partials (296) | result (1)
constexpr long OFF_R = 0, OFF_LO = 64, OFF_HI = OFF_LO + NOALLOC_HALF, OFF_PART = OFF_HI + NOALLOC_HALF,
               OFF_RES = OFF_PART + NOALLOC_BLOCKS, SCRATCH_ELEMS = OFF_RES + 16;

static __device__ __align__(256) fe g_noalloc_scratch[SCRATCH_ELEMS];

// out[i] = prod_{b < nbits} (bit b of i ? r[b] : 1 - r[b])
__global__ void k_na_eq_half(const fe *__restrict__ r, int nbits, fe *__restrict__ out)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (1L << nbits)) return;
    fe x = vg::fe_one();
    for (int b = 0; b < nbits; ++b) x = x * (((i >> b) & 1) ? r[b] : vg::fe_one() - r[b]);
    out[i] = x;
}

// per-block partial sums of vals[x] * lo[x & mask] * hi[x >> fh]
__global__ void k_na_dot(const fe *__restrict__ vals, const fe *__restrict__ lo, const fe *__restrict__ hi, int fh,
                         long n, fe *__restrict__ parts)
{
    __shared__ fe sm[32];
    const long mask = (1L << fh) - 1;
    fe acc[1] = {vg::fe_zero()};
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < n; x += (long)gridDim.x * blockDim.x)
        acc[0] = acc[0] + vals[x] * (lo[x & mask] * hi[x >> fh]);
    block_sum<1>(acc, sm);
    if (threadIdx.x == 0) parts[blockIdx.x] = acc[0];
}

__global__ void k_na_sum(const fe *__restrict__ parts, int nparts, fe *__restrict__ out)
{
    __shared__ fe sm[32];
    fe acc[1] = {vg::fe_zero()};
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc[0] = acc[0] + parts[i];
    block_sum<1>(acc, sm);
    if (threadIdx.x == 0) out[0] = acc[0];
}

std::mutex g_na_mutex;
fe *g_na_addr[64] = {nullptr};   // per device, looked up on first use

}  // namespace

extern "C" int vg_mle_eval_noalloc(const vg_fe *vals, long n, const vg_fe *r, int log_n, vg_fe *out)
{
    if (log_n < 0 || log_n > NOALLOC_MAX_LOG)   // checked before any shift by log_n
        return vg_fail(VG_ERR_ARG, "vg_mle_eval_noalloc: log_n %d outside the fixed scratch limit [0, %d]", log_n,
                       NOALLOC_MAX_LOG);
    if (!vals || !r || !out || n < (1L << log_n))
        return vg_fail(VG_ERR_ARG, "vg_mle_eval_noalloc: bad argument (n=%ld log_n=%d)", n, log_n);
    {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, vals) != cudaSuccess || a.type != cudaMemoryTypeDevice) {
            cudaGetLastError();
            return vg_fail(VG_ERR_ARG, "vg_mle_eval_noalloc: vals must be device memory");
        }
    }
    int dev = 0;
    VG_CHECK_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return vg_fail(VG_ERR_ARG, "vg_mle_eval_noalloc: device %d", dev);
    fe *scratch;
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!g_na_addr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return vg_fail(VG_ERR_CUDA, "vg_mle_eval_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            g_na_addr[dev] = (fe *)p;
        }
        scratch = g_na_addr[dev];
    }
    const int f = log_n >> 1, s = log_n - f;
    fe *rd = scratch + OFF_R, *lo = scratch + OFF_LO, *hi = scratch + OFF_HI, *parts = scratch + OFF_PART,
       *res = scratch + OFF_RES;
    if (log_n) VG_CHECK_CUDA(cudaMemcpy(rd, r, log_n * sizeof(fe), cudaMemcpyHostToDevice));
    k_na_eq_half<<<grid_for(1L << f, 256), 256>>>(rd, f, lo);
    VG_CHECK_CUDA(cudaGetLastError());
    k_na_eq_half<<<grid_for(1L << s, 256), 256>>>(rd + f, s, hi);
    VG_CHECK_CUDA(cudaGetLastError());
    k_na_dot<<<NOALLOC_BLOCKS, 256>>>((const fe *)vals, lo, hi, f, 1L << log_n, parts);
    VG_CHECK_CUDA(cudaGetLastError());
    k_na_sum<<<1, 512>>>(parts, NOALLOC_BLOCKS, res);
    VG_CHECK_CUDA(cudaGetLastError());
    VG_CHECK_CUDA(cudaMemcpy(out, res, sizeof(fe), cudaMemcpyDeviceToHost));
    return VG_OK;
}
