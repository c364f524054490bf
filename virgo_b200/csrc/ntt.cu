// Batched number-theoretic transform over F_{p^2}, natural order in and out.
//
// n = 2^logn is split into factors F_1 .. F_P (each <= 2^10).  Passes 1..P-1
// are "column passes": inside every block of the current size A, DFTs of size
// F_q run down the columns (stride A / F_q) and output k of column c is scaled
// by w_A^(c k), in place.  Pass P is a "row pass": each contiguous block of
// F_P elements is transformed and written to its natural-order position
// k_1 + F_1 (k_2 + F_2 (... + F_{P-1} k_P)).  This is the four-step
// decomposition applied recursively, so no separate bit-reversal pass is
// needed and every pass reads and writes runs of >= G contiguous elements.
//
// Inside a CTA each sub-DFT is a decimation-in-time transform in shared
// memory (bit-reversed load, natural-order result) with radix-4 butterflies
// (two radix-2 stages each, three twiddle products per four entries).
//
// Twiddles: w^e for e < n comes from two small tables, lo[e & 4095] *
// hi[e >> 12], built once per root and cached in the context; for n up to
// 2^TW_FULL_MAX_LOG the column passes read w^e from a full table instead
// (one load in place of two loads and a product per element).
#include "common.cuh"
#include <algorithm>
#include <mutex>
#include <vector>

namespace {

constexpr int NTT_THREADS = 256;
constexpr int MAX_LM = 10, MAX_TILE_LOG = 13;

struct PassArgs {
    const fe *in;
    fe *out;
    long in_len;        // valid input elements per batch item (first pass), zero beyond
    long in_bstride, out_bstride;
    int logn, lm, logG;
    int kind;           // 0 column pass, 1 row pass, 2 single pass
    int logA;           // column pass: block size
    int nfac;           // row pass: number of previous factors
    int fac[6];         // row pass: their logs, F_1 first
    const fe *tw_lo, *tw_hi;
    const fe *tw_full;  // w^e for every e < n, or null
    int scale;
    fe inv_n;
};

__device__ __forceinline__ fe tw_pow(const fe *__restrict__ lo, const fe *__restrict__ hi, uint64_t e)
{
    fe a = lo[e & 4095];
    uint64_t h = e >> 12;
    if (h) a = a * hi[h];
    return a;
}

__device__ __forceinline__ int bitrev(int x, int bits) { return bits ? (int)(__brev((unsigned)x) >> (32 - bits)) : 0; }

__global__ void __launch_bounds__(NTT_THREADS) k_ntt_pass(PassArgs a)
{
    extern __shared__ fe smem[];
    const int m = 1 << a.lm, G = 1 << a.logG, mg = m << a.logG;
    fe *S = smem;            // [m][G]
    fe *T = smem + mg;       // w_m^e, e < m/2
    const long n = 1L << a.logn;
    const long item = blockIdx.y;
    const fe *in = a.in + item * a.in_bstride;
    fe *out = a.out + item * a.out_bstride;

    for (int e = threadIdx.x; e < (m >> 1); e += blockDim.x)
        T[e] = tw_pow(a.tw_lo, a.tw_hi, (uint64_t)e << (a.logn - a.lm));

    // ---- transform geometry ----
    long col_base = 0, C = 1;    // column pass: element (g, r) at col_base + g + r*C
    long row_base = 0;           // row pass: element (g, r) at row_base + g*rowW*m + r
    long rowW = 0, pos_rest = 0;
    if (a.kind == 0) {
        const long A = 1L << a.logA;
        C = A >> a.lm;
        const long cpb = C >> a.logG;                  // CTAs per block
        const long blk = blockIdx.x / cpb;
        const long c0 = (blockIdx.x % cpb) << a.logG;
        col_base = blk * A + c0;
    } else if (a.kind == 1) {
        const long T_all = n >> a.lm;
        rowW = T_all >> a.fac[0];                       // transforms per k_1 value
        const long t_rest = blockIdx.x % rowW;
        const long k10 = (blockIdx.x / rowW) << a.logG;
        row_base = (k10 * rowW + t_rest) << a.lm;
        // natural position of the digits k_2..k_{P-1} held by t_rest
        long tmp = t_rest, acc = 0;
        int shift_lo = 0;
        for (int q = 0; q < a.nfac; ++q) shift_lo += a.fac[q];
        for (int q = a.nfac - 1; q >= 1; --q) {
            shift_lo -= a.fac[q];
            long kq = tmp & ((1L << a.fac[q]) - 1);
            tmp >>= a.fac[q];
            acc += kq << shift_lo;
        }
        pos_rest = acc + k10;
    } else {
        // single pass: G whole batch items per CTA (item index folded into blockIdx.x)
    }

    // ---- load (bit-reversed rows) ----
    for (int idx = threadIdx.x; idx < mg; idx += blockDim.x) {
        int r, g;
        long gi;
        const fe *src = in;
        if (a.kind == 0) {
            g = idx & (G - 1);
            r = idx >> a.logG;
            gi = col_base + g + (long)r * C;
        } else if (a.kind == 1) {
            r = idx & (m - 1);
            g = idx >> a.lm;
            gi = row_base + (long)g * rowW * m + r;
        } else {
            r = idx & (m - 1);
            g = idx >> a.lm;
            src = a.in + ((long)blockIdx.x * G + g) * a.in_bstride;
            gi = r;
        }
        fe x = gi < a.in_len ? src[gi] : vg::fe_zero();
        S[(bitrev(r, a.lm) << a.logG) + g] = x;
    }
    __syncthreads();

    // ---- DIT stages, two radix-2 stages at a time (radix 4) ----
    // For the stage pair (s, s+1), position pos < 2^s inside a group of
    // 2^(s+2) entries and u = w_m^e, e = pos 2^(lm-2-s), the two radix-2
    // butterfly layers equal
    //   t1 = x1 u^2, t2 = x2 u, t3 = x3 u^3,
    //   y0 = (x0 + t1) + (t2 + t3), y2 = (x0 + t1) - (t2 + t3),
    //   y1 = (x0 - t1) + J (t2 - t3), y3 = (x0 - t1) - J (t2 - t3),
    // with J = w_m^(m/4), a square root of -1 in F_p2, i.e. +-i, whose
    // product is a swap and a negation: three products per four entries
    // instead of four, and one shared-memory round trip and barrier per two
    // stages.  The first pair (s = 0) has u = 1 and no products.  u^3 = w^(3e)
    // with 3e >= m/2 is -T[3e - m/2].  An odd lm ends with one radix-2 stage.
    const bool j_plus = a.lm >= 2 && T[m >> 2].img == 1;
    int s = 0;
    for (; s + 1 < a.lm; s += 2) {
        const int quarter = 1 << s;
        for (int b = threadIdx.x; b < (mg >> 2); b += blockDim.x) {
            const int g = b & (G - 1), q = b >> a.logG;
            const int pos = q & (quarter - 1), grp = q >> s;
            const int i0 = (grp << (s + 2)) + pos;
            fe *p0 = &S[(i0 << a.logG) + g];
            const int st = quarter << a.logG;
            fe x0 = p0[0], t1 = p0[st], t2 = p0[2 * st], t3 = p0[3 * st];
            bool neg3 = false;
            if (s) {
                const int e = pos << (a.lm - 2 - s), e3 = 3 * e, h = m >> 1;
                t1 = t1 * T[2 * e];
                t2 = t2 * T[e];
                neg3 = e3 >= h;
                t3 = t3 * T[neg3 ? e3 - h : e3];
            }
            const fe E = x0 + t1, O = x0 - t1;
            const fe F = neg3 ? t2 - t3 : t2 + t3;
            const fe Dm = neg3 ? t2 + t3 : t2 - t3;
            const fe D = j_plus ? vg::fe_make(vg::negp(Dm.img), Dm.real) : vg::fe_make(Dm.img, vg::negp(Dm.real));
            p0[0] = E + F;
            p0[2 * st] = E - F;
            p0[st] = O + D;
            p0[3 * st] = O - D;
        }
        __syncthreads();
    }
    if (s < a.lm) {
        const int half = 1 << s;
        for (int b = threadIdx.x; b < (mg >> 1); b += blockDim.x) {
            const int g = b & (G - 1), q = b >> a.logG;
            const int pos = q & (half - 1), grp = q >> s;
            const int i0 = (grp << (s + 1)) + pos, i1 = i0 + half;
            fe x0 = S[(i0 << a.logG) + g];
            fe x1 = S[(i1 << a.logG) + g];
            if (pos) x1 = x1 * T[pos << (a.lm - 1 - s)];
            S[(i0 << a.logG) + g] = x0 + x1;
            S[(i1 << a.logG) + g] = x0 - x1;
        }
        __syncthreads();
    }

    // ---- store ----
    for (int idx = threadIdx.x; idx < mg; idx += blockDim.x) {
        int k, g;
        long gi;
        fe *dst = out;
        if (a.kind == 0) {
            g = idx & (G - 1);
            k = idx >> a.logG;
            gi = col_base + g + (long)k * C;
        } else if (a.kind == 1) {
            g = idx & (G - 1);
            k = idx >> a.logG;
            gi = pos_rest + g + ((long)k << (a.logn - a.lm));
        } else {
            k = idx & (m - 1);
            g = idx >> a.lm;
            dst = a.out + ((long)blockIdx.x * G + g) * a.out_bstride;
            gi = k;
        }
        fe y = S[(k << a.logG) + g];
        if (a.kind == 0) {
            const long A = 1L << a.logA;
            const long c = (col_base % A) + g;
            uint64_t e = ((uint64_t)c * (uint64_t)k) << (a.logn - a.logA);   // c k < A, so e < n
            if (e) y = y * (a.tw_full ? a.tw_full[e] : tw_pow(a.tw_lo, a.tw_hi, e));
        }
        if (a.scale) y = y * a.inv_n;
        dst[gi] = y;
    }
}

// w^e for every e < n, from the two small tables
__global__ void k_tw_full(const fe *__restrict__ lo, const fe *__restrict__ hi, long n, fe *__restrict__ full)
{
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        full[e] = tw_pow(lo, hi, (uint64_t)e);
}

__global__ void k_tw_build(fe w, fe w4096, fe *lo, fe *hi, int nhi)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 4096) lo[i] = vg::fe_pow(w, (uint64_t)i);
    if (i < nhi) hi[i] = vg::fe_pow(w4096, (uint64_t)i);
}

// n = 2^logn as ceil(logn / max_lm) factors of nearly equal size (the
// radix: VG_TUNE_NTT_MAX_LOG, at most MAX_LM)
void plan_factors(int logn, int max_lm, std::vector<int> &f)
{
    f.clear();
    if (logn <= max_lm) {
        f.push_back(logn);
        return;
    }
    int P = (logn + max_lm - 1) / max_lm;
    int base = logn / P, extra = logn % P;
    for (int q = 0; q < P; ++q) f.push_back(base + (q < extra ? 1 : 0));
}

// columns (or whole items) per CTA: m * G ~ 2^tile_log elements
// (VG_TUNE_NTT_TILE_LOG, at most MAX_TILE_LOG)
int pick_logG(int lm, long avail_log, int tile_log)
{
    int lg = tile_log - lm;
    if (lg < 0) lg = 0;
    if (lg > avail_log) lg = (int)avail_log;
    return lg;
}

}  // namespace

int vg_twiddles(vg_ctx *c, fe root, int logn, const fe **lo, const fe **hi)
{
    for (auto &t : c->tw_cache)
        if (t.key_real == root.real && t.key_img == root.img && t.logn == logn) {
            *lo = t.lo;
            *hi = t.hi;
            return VG_OK;
        }
    TwEntry t;
    t.key_real = root.real;
    t.key_img = root.img;
    t.logn = logn;
    int nhi = logn > 12 ? (1 << (logn - 12)) : 1;
    VG_TRY(vg_alloc(c, (void **)&t.lo, 4096 * sizeof(fe)));
    VG_TRY(vg_alloc(c, (void **)&t.hi, nhi * sizeof(fe)));
    fe w4096 = vg::fe_pow(root, 4096);
    k_tw_build<<<grid_for(std::max(4096, nhi), 256), 256, 0, c->stream>>>(root, w4096, t.lo, t.hi, nhi);
    VG_LAUNCHED(c);
    if (c->tw_cache.size() >= 64) {
        vg_release(c, c->tw_cache.front().lo);
        vg_release(c, c->tw_cache.front().hi);
        if (c->tw_cache.front().full) vg_release(c, c->tw_cache.front().full);
        c->tw_cache.erase(c->tw_cache.begin());
    }
    c->tw_cache.push_back(t);
    *lo = t.lo;
    *hi = t.hi;
    return VG_OK;
}

// The full table w^e, e < 2^logn, of a cached root (built on first use), or
// null when n is above 2^TW_FULL_MAX_LOG or the context's full tables would
// pass TW_FULL_BUDGET bytes: the column passes then form w^e from lo and hi.
constexpr int TW_FULL_MAX_LOG = 20;
constexpr size_t TW_FULL_BUDGET = 64u << 20;

static int twiddles_full(vg_ctx *c, fe root, int logn, const fe **full)
{
    *full = nullptr;
    if (logn > TW_FULL_MAX_LOG) return VG_OK;
    const fe *lo, *hi;
    VG_TRY(vg_twiddles(c, root, logn, &lo, &hi));
    size_t used = 0;
    TwEntry *mine = nullptr;
    for (auto &t : c->tw_cache) {
        if (t.full) used += ((size_t)1 << t.logn) * sizeof(fe);
        if (t.key_real == root.real && t.key_img == root.img && t.logn == logn) mine = &t;
    }
    if (!mine) return VG_OK;
    if (!mine->full) {
        const size_t bytes = ((size_t)1 << logn) * sizeof(fe);
        if (used + bytes > TW_FULL_BUDGET) return VG_OK;
        // never allocate inside a stream capture (the table would belong to the graph)
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        VG_CHECK_CUDA(cudaStreamIsCapturing(c->stream, &cs));
        if (cs != cudaStreamCaptureStatusNone) return VG_OK;
        VG_TRY(vg_alloc(c, (void **)&mine->full, bytes));
        k_tw_full<<<std::min<unsigned>(grid_for(1L << logn, 256), 148u * 8u), 256, 0, c->stream>>>(mine->lo, mine->hi,
                                                                                                   1L << logn, mine->full);
        VG_LAUNCHED(c);
    }
    *full = mine->full;
    return VG_OK;
}

// Largest dynamic shared memory of a pass: m * G <= 2^MAX_TILE_LOG items
// (pick_logG) plus m / 2 <= 512 twiddles.  The kernel attribute is
// process-wide per device, so it is raised once to this bound: setting it per
// launch to the launch's own size races with other threads' launches of other
// sizes.
constexpr size_t NTT_MAX_SMEM = ((1 << MAX_TILE_LOG) + (1 << (MAX_LM - 1))) * sizeof(fe);

static int ntt_smem_attribute(int dev)
{
    static std::mutex mu;
    static std::vector<bool> done;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= (int)done.size()) done.resize(dev + 1, false);
    if (!done[dev]) {
        VG_CHECK_CUDA(cudaFuncSetAttribute(k_ntt_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)NTT_MAX_SMEM));
        done[dev] = true;
    }
    return VG_OK;
}

static int launch_pass(vg_ctx *c, PassArgs &a, long nblocks, int batch)
{
    const int m = 1 << a.lm, G = 1 << a.logG;
    size_t sm = ((size_t)m * G + (m >> 1)) * sizeof(fe);
    if (sm > NTT_MAX_SMEM) return vg_fail(VG_ERR_ARG, "ntt pass: %zu bytes of shared memory", sm);
    if (sm > 48 * 1024) VG_TRY(ntt_smem_attribute(c->device));
    dim3 grid((unsigned)nblocks, (unsigned)batch);
    {
        ProfScope ps(c, KF_NTT, 2.0 * 16.0 * (double)batch * (double)(1L << a.logn));
        k_ntt_pass<<<grid, NTT_THREADS, sm, c->stream>>>(a);
    }
    VG_LAUNCHED(c);
    return VG_OK;
}

extern "C" int vg_ntt(vg_ctx *c, const vg_fe *in_, long in_len, long in_bstride, vg_fe *out_, int logn,
                      long out_bstride, int batch, vg_fe root_, int scale_inv_n)
{
    if (!c || !in_ || !out_ || logn < 0 || logn > 30 || batch < 1 || in_len < 0 || in_len > (1L << logn))
        return vg_fail(VG_ERR_ARG, "vg_ntt: bad argument (logn=%d in_len=%ld batch=%d)", logn, in_len, batch);
    if (batch > 65535) return vg_fail(VG_ERR_ARG, "vg_ntt: batch %d > 65535", batch);
    const fe *in = (const fe *)in_;
    fe *out = (fe *)out_;
    fe root;
    root.real = root_.real;
    root.img = root_.img;
    const long n = 1L << logn;
    const fe *lo, *hi, *full;
    VG_TRY(vg_twiddles(c, root, logn, &lo, &hi));
    VG_TRY(twiddles_full(c, root, logn, &full));
    fe inv_n = vg::fe_inv(vg::fe_make((uint64_t)n % vg::P, 0));

    std::vector<int> f;
    const int max_lm = std::min(MAX_LM, (int)vg_tune_value(c->device, VG_TUNE_NTT_MAX_LOG));
    const int tile_log = std::min(MAX_TILE_LOG, (int)vg_tune_value(c->device, VG_TUNE_NTT_TILE_LOG));
    plan_factors(logn, max_lm, f);
    const int P = (int)f.size();

    if (P == 1) {
        PassArgs a{};
        a.in = in; a.out = out; a.in_len = in_len; a.in_bstride = in_bstride; a.out_bstride = out_bstride;
        a.logn = logn; a.lm = logn; a.kind = 2; a.tw_lo = lo; a.tw_hi = hi; a.scale = scale_inv_n; a.inv_n = inv_n;
        // G whole items per CTA, G must divide batch
        int lg = pick_logG(logn, 30, std::max(tile_log, logn));
        while (lg > 0 && (batch % (1 << lg)) != 0) --lg;
        a.logG = lg;
        VG_TRY(launch_pass(c, a, batch >> lg, 1));
        return VG_OK;
    }

    // intermediate buffer: passes 1..P-1 write tmp in place; the last pass writes out
    fe *tmp = out;
    bool in_place_ok = (in == out) ? (in_len == n && in_bstride == out_bstride) : false;
    const bool overlap = (in != out) && !((const char *)in + (size_t)batch * in_bstride * sizeof(fe) <= (const char *)out ||
                                          (const char *)out + (size_t)batch * out_bstride * sizeof(fe) <= (const char *)in);
    if (overlap && !in_place_ok) return vg_fail(VG_ERR_ARG, "vg_ntt: in and out overlap");
    // the row pass reads tmp and writes out in a permuted order, so tmp != out
    void *s;
    VG_TRY(vg_scratch(c, (size_t)batch * n * sizeof(fe), &s));
    tmp = (fe *)s;

    int logA = logn;
    for (int q = 0; q < P - 1; ++q) {
        PassArgs a{};
        a.in = q == 0 ? in : tmp;
        a.out = tmp;
        a.in_len = q == 0 ? in_len : n;
        a.in_bstride = q == 0 ? in_bstride : n;
        a.out_bstride = n;
        a.logn = logn; a.lm = f[q]; a.kind = 0; a.logA = logA;
        a.tw_lo = lo; a.tw_hi = hi; a.tw_full = full; a.scale = 0;
        long logC = logA - f[q];
        a.logG = pick_logG(f[q], logC, tile_log);
        long nblocks = (n >> logA) * ((1L << logC) >> a.logG);
        VG_TRY(launch_pass(c, a, nblocks, batch));
        logA -= f[q];
    }
    {
        PassArgs a{};
        a.in = tmp; a.out = out; a.in_len = n; a.in_bstride = n; a.out_bstride = out_bstride;
        a.logn = logn; a.lm = f[P - 1]; a.kind = 1;
        a.nfac = P - 1;
        for (int q = 0; q < P - 1; ++q) a.fac[q] = f[q];
        a.tw_lo = lo; a.tw_hi = hi; a.scale = scale_inv_n; a.inv_n = inv_n;
        a.logG = pick_logG(f[P - 1], f[0], tile_log);
        long T_all = n >> f[P - 1];
        long nblocks = T_all >> a.logG;
        VG_TRY(launch_pass(c, a, nblocks, batch));
    }
    return VG_OK;
}
