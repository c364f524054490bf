// The fft_gkr side prover on the GPU (src/VPD/fft_circuit_GKR.cpp, which the
// reference verifier runs as its own process, vpd_verifier.cpp:89-99, and whose
// prover time counts in the reference's Prove Time).
//
// The program proves, for lg = L - 6, that 64 evaluations of the inverse FFT
// of an eq-expansion of lg random points are right, with a GKR over a fixed
// circuit: an addition layer (64 x 2^lg products summed per block), a
// multiplication layer (each coefficient times its powers of the 64 points),
// a scaling layer, and one butterfly layer per inverse-FFT level (two
// sumcheck phases each).  Its challenges come from rand() in that process
// (never seeded: the stream of seed 1) and do not depend on the messages, so
// every challenge is drawn on the host up front and the whole prover is one
// stream of launches with one synchronisation:
//
//   circuit values  k_fg_expand, k_fg_butterfly x lg, k_fg_products (with the
//                   64 output sums)
//   phase tables    k_fg_halves (every eq half table of every layer, one
//                   launch), k_fg_add_tables, k_fg_mult_part + _reduce,
//                   k_fg_ifft_p1 / k_fg_ifft_p2 per level (phase 2 reads v_u
//                   from the device record of phase 1's last round)
//   rounds          the GKR prover's round kernels (vg_gkr_round over
//                   caller-built tables), records on the device
//
// then the host reads the records once and replays the reference's
// in-process verifier over them (every message against the running claim and
// each layer's closed-form predicate, fft_circuit_GKR.cpp:323-354, :438-489,
// :681-760).
#include "common.cuh"
#include "internal.h"
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace
{
vg_fe tovg(fe x)
{
    vg_fe r;
    r.real = x.real;
    r.img = x.img;
    return r;
}

constexpr int FG_THREADS = 256;
constexpr int FG_MAX_LG = 22;
constexpr int PROD_STEPS = 16;   // products per thread in k_fg_products (stride FG_THREADS)
constexpr int MULT_STEPS = 8;    // table entries per thread in k_fg_mult_part (large tables)

__device__ __forceinline__ fe fg_one_minus(fe r) { return vg::fe_one() - r; }

// eq-expansion of r (build_circuit :24-34): entry x multiplies, for each bit
// p of x, 1 - r[lg-1-p] when the bit is set and r[lg-1-p] when not.
__global__ void k_fg_expand(const fe *__restrict__ r, int lg, fe *__restrict__ out)
{
    const long x = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (x >= (1L << lg)) return;
    fe v = vg::fe_one();
    for (int p = 0; p < lg; ++p) v = v * (((x >> p) & 1) ? fg_one_minus(r[lg - 1 - p]) : r[lg - 1 - p]);
    out[x] = v;
}

// T[m] = w^m for m < n, 32 consecutive powers per thread from one fe_pow
__global__ void k_fg_powers(fe w, long n, fe *__restrict__ T)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long i0 = t * 32;
    if (i0 >= n) return;
    fe x = vg::fe_pow(w, (uint64_t)i0);
    for (long i = i0; i < i0 + 32 && i < n; ++i) {
        T[i] = x;
        x = x * w;
    }
}

// One inverse-FFT level (build_circuit :47-70) with parameter dep: for
// k < 2^(lg-dep-1), j < 2^dep, t = k 2^dep + j: l = pre[2k 2^dep + j],
// r = inv_rou^(k 2^dep) pre[(2k+1) 2^dep + j]; cur[t] = l + r,
// cur[t + 2^(lg-1)] = l - r.
__global__ void k_fg_butterfly(const fe *__restrict__ pre, fe *__restrict__ cur, const fe *__restrict__ T, int lg, int dep)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long half_n = 1L << (lg - 1);
    if (t >= half_n) return;
    const long k = t >> dep, j = t & ((1L << dep) - 1);
    const long li = (k << (dep + 1)) | j;
    const fe l = pre[li], rr = T[k << dep] * pre[li | (1L << dep)];
    cur[t] = l + rr;
    cur[t + half_n] = l - rr;
}

// Scaling and product layers (build_circuit :71-101): S[i] = X[i] inv_n and
// P[j 2^lg + i] = S[i] ep_j^i, with the per-block partial sums of P for the
// 64 outputs (:102-111).  Block (bx, j) covers FG_THREADS x PROD_STEPS
// entries of row j, thread stride FG_THREADS, ep_j^i stepped by
// ep_step[j] = ep_j^FG_THREADS.
__global__ void __launch_bounds__(FG_THREADS) k_fg_products(const fe *__restrict__ X, fe inv_n, const fe *__restrict__ ep,
                                                            const fe *__restrict__ ep_step, int lg, fe *__restrict__ S,
                                                            fe *__restrict__ P, fe *__restrict__ parts)
{
    __shared__ fe sm[32];
    const long N = 1L << lg;
    const int j = blockIdx.y;
    const long i0 = (long)blockIdx.x * FG_THREADS * PROD_STEPS + threadIdx.x;
    fe acc[1] = {vg::fe_zero()};
    if (i0 < N) {
        fe x = vg::fe_pow(ep[j], (uint64_t)i0);
        const fe step = ep_step[j];
        for (int m = 0; m < PROD_STEPS; ++m) {
            const long i = i0 + (long)m * FG_THREADS;
            if (i >= N) break;
            const fe s = X[i] * inv_n;
            if (j == 0) S[i] = s;
            const fe p = s * x;
            P[(long)j * N + i] = p;
            acc[0] = acc[0] + p;
            x = x * step;
        }
    }
    block_sum<1>(acc, sm);
    if (threadIdx.x == 0) parts[(long)j * gridDim.x + blockIdx.x] = acc[0];
}

// Every eq half table of the proof in one launch: job q writes
// out[q][i] = scale[q] * prod_b (bit b of i ? r[b] : 1 - r[b]) over nbits[q]
// bits of the challenge block r[q], for i < 2^nbits[q].
struct HalfJob {
    int r_off, nbits;
    long out_off, begin;   // begin: first thread of the job (prefix over the jobs)
    fe scale;
};
__global__ void k_fg_halves(const HalfJob *__restrict__ jobs, int njobs, long total, const fe *__restrict__ R,
                            fe *__restrict__ out)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    int lo = 0, hi = njobs - 1;   // last job with begin <= t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].begin <= t) lo = mid;
        else hi = mid - 1;
    }
    const HalfJob J = jobs[lo];
    const long i = t - J.begin;
    const fe *r = R + J.r_off;
    fe x = J.scale;
    for (int b = 0; b < J.nbits; ++b) x = x * (((i >> b) & 1) ? r[b] : fg_one_minus(r[b]));
    out[J.out_off + i] = x;
}

// alpha eq(r0, g) + beta eq(r1, g) from the four half tables (alpha and beta
// folded into the low halves): lo0, hi0, lo1, hi1 at h, h + sh, ...
struct BetaHalves {
    const fe *lo0, *hi0, *lo1, *hi1;
    int fb;
    long mask;
    __device__ __forceinline__ fe at(long g) const
    {
        return lo0[g & mask] * hi0[g >> fb] + lo1[g & mask] * hi1[g >> fb];
    }
};
struct EqHalves {
    const fe *lo, *hi;
    int fb;
    long mask;
    __device__ __forceinline__ fe at(long u) const { return lo[u & mask] * hi[u >> fb]; }
};

// addition layer (:238-290): add_mult_sum[j] = beta_g(j >> lg) over 6 bits,
// addV = 0
__global__ void k_fg_add_tables(const fe *__restrict__ bg6, int lg, long n, fe *__restrict__ AV, fe *__restrict__ AM)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        AV[i] = vg::fe_zero();
        AM[i] = bg6[i >> lg];
    }
}

// multiplication layer (:398-430): add_mult_sum[i] = sum_j beta_g(j 2^lg + i) ep_j^i
// over lg + 6 bits, addV = 0.  Block (bx, q) sums the points q jper ..
// (q + 1) jper - 1 for the entries i0 + m FG_THREADS (m < STEPS) into
// parts[q N + i]; k_fg_mult_reduce adds the 64 / jper partials.  Small tables
// take one point and one entry per thread, so the 64 N terms spread over the
// whole GPU instead of a few blocks.
template <int STEPS>
__global__ void __launch_bounds__(FG_THREADS) k_fg_mult_part(BetaHalves bg, const fe *__restrict__ ep,
                                                             const fe *__restrict__ ep_step, int lg, int jper,
                                                             fe *__restrict__ parts)
{
    const long N = 1L << lg;
    const long i0 = (long)blockIdx.x * FG_THREADS * STEPS + threadIdx.x;
    if (i0 >= N) return;
    fe acc[STEPS];
#pragma unroll
    for (int m = 0; m < STEPS; ++m) acc[m] = vg::fe_zero();
    for (int j = blockIdx.y * jper; j < (int)(blockIdx.y + 1) * jper; ++j) {
        fe x = vg::fe_pow(ep[j], (uint64_t)i0);
        const fe step = ep_step[j];
#pragma unroll
        for (int m = 0; m < STEPS; ++m) {
            const long i = i0 + (long)m * FG_THREADS;
            if (i < N) acc[m] = acc[m] + bg.at((long)j * N + i) * x;
            x = x * step;
        }
    }
#pragma unroll
    for (int m = 0; m < STEPS; ++m) {
        const long i = i0 + (long)m * FG_THREADS;
        if (i < N) parts[(long)blockIdx.y * N + i] = acc[m];
    }
}

// AM[i] = sum of the partials; AV[i] = 0 (parts may be AV itself: thread i
// reads its own entry of group 0 before clearing it)
__global__ void k_fg_mult_reduce(const fe *parts, int groups, long N, fe *AV, fe *__restrict__ AM)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= N) return;
    fe s = vg::fe_zero();
    for (int q = 0; q < groups; ++q) s = s + parts[(long)q * N + i];
    AM[i] = s;
    AV[i] = vg::fe_zero();
}

// inverse-FFT level dep, phase 1 (:536-566): for the pair of gates
// g1 = k 2^dep + j, g2 = g1 + 2^(lg-1) reading u = 2k 2^dep + j and
// v = u + 2^dep with twiddle x = inv_rou^(k 2^dep):
// add_mult_sum[u] = bg(g1) + bg(g2), addV[u] = x V[v] (bg(g1) - bg(g2));
// the entries at v are zero.
__global__ void k_fg_ifft_p1(const fe *__restrict__ pre, const fe *__restrict__ T, BetaHalves bg, int lg, int dep,
                             fe *__restrict__ AV, fe *__restrict__ AM)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long half_n = 1L << (lg - 1);
    if (t >= half_n) return;
    const long k = t >> dep, j = t & ((1L << dep) - 1);
    const long u = (k << (dep + 1)) | j, v = u | (1L << dep);
    const fe b1 = bg.at(t), b2 = bg.at(t + half_n), x = T[k << dep];
    AM[u] = b1 + b2;
    AV[u] = (x * pre[v]) * (b1 - b2);
    AM[v] = vg::fe_zero();
    AV[v] = vg::fe_zero();
}

// phase 2 (:587-640): with t_i = bg(g_i) beta_u(u):
// add_mult_sum[v] = x (t1 - t2), addV[v] = v_u (t1 + t2); entries at u zero.
// v_u = V(r_u) is the folded V pair of phase 1's last round (its record,
// values 3 and 4) at the last challenge.
__global__ void k_fg_ifft_p2(const fe *__restrict__ T, BetaHalves bg, EqHalves bu, const fe *__restrict__ rec_last,
                             fe r_last, int lg, int dep, fe *__restrict__ AV, fe *__restrict__ AM)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long half_n = 1L << (lg - 1);
    if (t >= half_n) return;
    const fe l0 = rec_last[3], l1 = rec_last[4];
    const fe vu = l0 + r_last * (l1 - l0);
    const long k = t >> dep, j = t & ((1L << dep) - 1);
    const long u = (k << (dep + 1)) | j, v = u | (1L << dep);
    const fe beu = bu.at(u);
    const fe t1 = bg.at(t) * beu, t2 = bg.at(t + half_n) * beu, x = T[k << dep];
    AM[v] = x * (t1 - t2);
    AV[v] = vu * (t1 + t2);
    AM[u] = vg::fe_zero();
    AV[u] = vg::fe_zero();
}

// prime_field::random (prime_field.cpp:35-41) over a private rand() stream:
// real part first, then imaginary, each rand() % p (rand() < 2^31 < p)
struct Rng {
    random_data d;
    char st[128];
    explicit Rng(unsigned seed)
    {
        memset(&d, 0, sizeof d);
        memset(st, 0, sizeof st);
        initstate_r(seed, st, sizeof st, &d);
    }
    fe next()
    {
        int32_t a = 0, b = 0;
        random_r(&d, &a);
        random_r(&d, &b);
        return vg::fe_make((uint64_t)a, (uint64_t)b);
    }
    void fill(std::vector<fe> &v, size_t at, int n)
    {
        for (int i = 0; i < n; ++i) v[at + i] = next();
    }
};

fe eq_host(const fe *r, int len, long i)
{
    fe x = vg::fe_one();
    for (int b = 0; b < len; ++b) x = x * (((i >> b) & 1) ? r[b] : vg::fe_one() - r[b]);
    return x;
}
fe qeval(const fe *m, fe x) { return (m[0] * x + m[1]) * x + m[2]; }
bool feq(fe a, fe b) { return a.real == b.real && a.img == b.img; }

// The challenge block (field-element offsets): every rand() draw of one run
// in the reference's order (main :827-845, build_circuit :22-112,
// engage_gkr :786-825, each layer's refreshes), then the addition layer's
// beta_g values and the 64 points' power steps.
struct Layout {
    int lg, R;
    size_t o_r, o_ep, o_r0, o_r1, o_au, o_av, o_mu, o_mv, o_lv, o_ab, o_bg6, o_step, n_chal;
    explicit Layout(int lg_) : lg(lg_), R(lg_ + 10)
    {
        o_r = 0;
        o_ep = o_r + lg;
        o_r0 = o_ep + 64;
        o_r1 = o_r0 + R;
        o_au = o_r1 + R;
        o_av = o_au + lg + 6;
        o_mu = o_av + lg + 6;
        o_mv = o_mu + lg;
        o_lv = o_mv + lg;                      // per level: r_u (lg), r_v (lg)
        o_ab = o_lv + 2 * (size_t)lg * lg;     // per level: alpha, beta drawn at its end
        o_bg6 = o_ab + 2 * (size_t)lg;
        o_step = o_bg6 + 64;
        n_chal = o_step + 64;
    }
    size_t lv_u(int d) const { return o_lv + 2 * (size_t)d * lg; }
    size_t lv_v(int d) const { return lv_u(d) + lg; }
    // r_0, r_1 of level d: the previous layer's r_u, r_v
    size_t prev_u(int d) const { return d == 0 ? o_mu : lv_u(d - 1); }
    size_t prev_v(int d) const { return d == 0 ? o_mv : lv_v(d - 1); }
};
}  // namespace

struct vg_fft_gkr {
    vg_ctx *ctx = nullptr;
    int max_lg = 0;
    vg_gkr *tables = nullptr;
    // device: challenges + per-proof constants (one upload), circuit layers,
    // twiddles, products, eq half tables, output partials
    fe *dev = nullptr;
    size_t dev_cap = 0;
    void *host = nullptr;   // pinned upload block
    size_t host_cap = 0;
    fe *parts_host = nullptr;   // pinned: output partial sums
    size_t parts_host_cap = 0;
    // the run in flight between launch and finish
    bool pending = false;
    int lg = 0;
    std::vector<fe> H;          // challenge block
    long prod_blocks = 0;
    std::chrono::steady_clock::time_point t0;
    long long launched = 0;
    const vg_fe *recs = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};   // around the run's device steps
    // The device steps as a CUDA graph.  A run with the size, seed and
    // buffers of the previous one enqueues exactly the same steps (every
    // challenge comes from the seed), so the second such run is captured
    // and later ones replay the graph: every kernel still runs, from one
    // launch instead of one per kernel.
    cudaGraphExec_t gexec = nullptr;
    int g_lg = 0;
    unsigned g_seed = 0;
    const void *g_key[3] = {nullptr, nullptr, nullptr};   // dev, host, parts_host at capture
    long long g_launched = 0;   // kernels in the graph
    bool g_seen = false;        // the last plain run had the current key
    bool g_off = false;         // a capture failed: plain launches from then on
};

// VIRGO_GRAPHS=0 turns the side proof's graph off (plain launches)
static bool fg_graphs_enabled()
{
    static const bool on = [] {
        const char *e = getenv("VIRGO_GRAPHS");
        return !(e && e[0] == '0');
    }();
    return on;
}

static void fg_drop_graph(vg_fft_gkr *f)
{
    if (f->gexec) cudaGraphExecDestroy(f->gexec);
    f->gexec = nullptr;
    f->g_seen = false;
}

// Ends a stream capture left open by an early error return.
struct CaptureGuard {
    cudaStream_t s = nullptr;
    bool active = false;
    ~CaptureGuard()
    {
        if (!active) return;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
    }
};

extern "C" int vg_fft_gkr_rounds(int lg) { return (lg + 6) + lg + 2 * lg * lg; }

extern "C" size_t vg_fft_gkr_footprint(int lg)
{
    if (lg < 1) return 0;
    const size_t N = (size_t)1 << lg, NE = N << 6;
    size_t fe_count = 3 * NE + 3 * (NE / 2 + 1);                     // ping-pong tables
    fe_count += (NE / 1024 + 1) * 36 + 9 * (size_t)vg_fft_gkr_rounds(lg);   // group partials, records
    fe_count += (size_t)(lg + 1) * N + N / 2 + 1 + N + NE;          // layers, twiddles, scaled, products
    fe_count += 64 * ((N + 4095) / 4096) + 16 * ((size_t)1 << ((lg + 7) / 2)) * (lg + 1);   // partials, halves
    return fe_count * sizeof(fe) + ((size_t)1 << 20);
}

extern "C" int vg_fft_gkr_create(vg_ctx *ctx, int max_lg, vg_fft_gkr **out)
{
    if (!ctx || !out || max_lg < 1 || max_lg > FG_MAX_LG)
        return vg_fail(VG_ERR_ARG, "vg_fft_gkr_create: max_lg %d outside 1..%d", max_lg, FG_MAX_LG);
    vg_fft_gkr *f = new vg_fft_gkr();
    f->ctx = ctx;
    f->max_lg = max_lg;
    int rc = vg_gkr_tables_create(ctx, 64L << max_lg, vg_fft_gkr_rounds(max_lg), &f->tables);
    if (rc == VG_OK && (cudaEventCreate(&f->ev[0]) != cudaSuccess || cudaEventCreate(&f->ev[1]) != cudaSuccess))
        rc = vg_fail(VG_ERR_CUDA, "vg_fft_gkr_create: event creation failed");
    if (rc != VG_OK) {
        vg_fft_gkr_destroy(f);
        return rc;
    }
    *out = f;
    return VG_OK;
}

int vg_fft_gkr_reserve(vg_fft_gkr *f, int max_lg)
{
    if (!f || max_lg < 1 || max_lg > FG_MAX_LG)
        return vg_fail(VG_ERR_ARG, "vg_fft_gkr_reserve: max_lg %d outside 1..%d", max_lg, FG_MAX_LG);
    if (max_lg <= f->max_lg) return VG_OK;
    if (f->pending) return vg_fail(VG_ERR_STATE, "vg_fft_gkr_reserve: a run is in flight");
    fg_drop_graph(f);   // the tables move
    VG_TRY(vg_gkr_tables_reserve(f->tables, 64L << max_lg, vg_fft_gkr_rounds(max_lg)));
    f->max_lg = max_lg;
    return VG_OK;
}

extern "C" int vg_fft_gkr_destroy(vg_fft_gkr *f)
{
    if (!f) return VG_OK;
    cudaStreamSynchronize(f->ctx->stream);
    fg_drop_graph(f);
    vg_gkr_destroy(f->tables);
    vg_release(f->ctx, f->dev);
    for (cudaEvent_t e : f->ev)
        if (e) cudaEventDestroy(e);
    if (f->host) cudaFreeHost(f->host);
    if (f->parts_host) cudaFreeHost(f->parts_host);
    delete f;
    return VG_OK;
}

int vg_fft_gkr_launch(vg_fft_gkr *f, int lg, unsigned seed)
{
    if (!f) return vg_fail(VG_ERR_ARG, "vg_fft_gkr_launch: null argument");
    if (lg < 1 || lg > f->max_lg) return vg_fail(VG_ERR_ARG, "vg_fft_gkr: lg %d outside 1..%d", lg, f->max_lg);
    if (f->pending) return vg_fail(VG_ERR_STATE, "vg_fft_gkr_launch: the previous run was not finished");
    vg_ctx *c = f->ctx;
    f->t0 = std::chrono::steady_clock::now();
    const bool graphs = fg_graphs_enabled() && !f->g_off && !c->profiling;
    if (graphs && f->gexec && f->g_lg == lg && f->g_seed == seed && f->g_key[0] == f->dev && f->g_key[1] == f->host &&
        f->g_key[2] == f->parts_host) {
        // H, prod_blocks and the host record pointer are those of the captured run
        VG_CHECK_CUDA(cudaEventRecord(f->ev[0], c->stream));
        VG_CHECK_CUDA(cudaGraphLaunch(f->gexec, c->stream));
        VG_CHECK_CUDA(cudaEventRecord(f->ev[1], c->stream));
        c->launches += f->g_launched;
        f->launched = f->g_launched;
        f->lg = lg;
        f->pending = true;
        return VG_OK;
    }
    const long long launches0 = c->launches;
    const long N = 1L << lg, NE = 64L << lg;
    const int nrounds = vg_fft_gkr_rounds(lg);

    // ---- every challenge, drawn up front ----
    Rng rng(seed);
    const Layout Lo(lg);
    const int R = Lo.R;
    const size_t o_r = Lo.o_r, o_ep = Lo.o_ep, o_r0 = Lo.o_r0, o_r1 = Lo.o_r1, o_au = Lo.o_au, o_av = Lo.o_av;
    const size_t o_mu = Lo.o_mu, o_mv = Lo.o_mv, o_ab = Lo.o_ab, o_bg6 = Lo.o_bg6, o_step = Lo.o_step;
    const size_t n_chal = Lo.n_chal;
    std::vector<fe> &H = f->H;
    H.assign(n_chal, vg::fe_zero());
    rng.fill(H, o_r, lg);
    rng.fill(H, o_ep, 64);
    rng.fill(H, o_r0, R);
    rng.fill(H, o_r1, R);
    rng.fill(H, o_au, lg + 6);
    rng.fill(H, o_av, lg + 6);
    rng.fill(H, o_mu, lg);
    rng.fill(H, o_mv, lg);
    for (int d = 0; d < lg; ++d) {
        rng.fill(H, Lo.lv_u(d), lg);
        rng.fill(H, Lo.lv_v(d), lg);
        rng.fill(H, o_ab + 2 * d, 2);
    }
    // alpha, beta of each level's beta_g: 1, 0 until the first level ends
    auto alpha_at = [&](int d) { return d == 0 ? vg::fe_one() : H[o_ab + 2 * (d - 1)]; };
    auto beta_at = [&](int d) { return d == 0 ? vg::fe_zero() : H[o_ab + 2 * (d - 1) + 1]; };
    for (int i = 0; i < 64; ++i) {
        H[o_bg6 + i] = eq_host(&H[o_r0], 6, i);   // alpha = 1, beta = 0 on the addition layer
        H[o_step + i] = vg::fe_pow(H[o_ep + i], FG_THREADS);
    }
    // eq half tables: the multiplication layer's beta_g (lg + 6 bits; r0 = the
    // addition layer's r_u, r1 = its r_v), then per level beta_g (lg bits) and
    // beta_u (lg bits)
    std::vector<HalfJob> jobs;
    long half_total = 0;
    auto add_job = [&](size_t r_off, int nbits, fe scale) {
        HalfJob J;
        J.r_off = (int)r_off;
        J.nbits = nbits;
        J.scale = scale;
        J.out_off = half_total;
        J.begin = half_total;
        half_total += 1L << nbits;
        jobs.push_back(J);
        return J.out_off;
    };
    struct Beta4 {
        long lo0, hi0, lo1, hi1;
        int fb;
    };
    auto add_beta = [&](size_t r0, size_t r1, int len, fe a, fe b) {
        const int fb = len >> 1;
        Beta4 q;
        q.lo0 = add_job(r0, fb, a);
        q.hi0 = add_job(r0 + fb, len - fb, vg::fe_one());
        q.lo1 = add_job(r1, fb, b);
        q.hi1 = add_job(r1 + fb, len - fb, vg::fe_one());
        q.fb = fb;
        return q;
    };
    const Beta4 mult_bg = add_beta(o_au, o_av, lg + 6, vg::fe_one(), vg::fe_zero());
    std::vector<Beta4> lvl_bg(lg);
    std::vector<long> lvl_ulo(lg), lvl_uhi(lg);
    for (int d = 0; d < lg; ++d) {
        lvl_bg[d] = add_beta(Lo.prev_u(d), Lo.prev_v(d), lg, alpha_at(d), beta_at(d));
        const size_t ru = Lo.lv_u(d);
        lvl_ulo[d] = add_job(ru, lg >> 1, vg::fe_one());
        lvl_uhi[d] = add_job(ru + (lg >> 1), lg - (lg >> 1), vg::fe_one());
    }

    // ---- device layout ----
    const long prod_blocks = (N + FG_THREADS * PROD_STEPS - 1) / (FG_THREADS * PROD_STEPS);
    f->prod_blocks = prod_blocks;
    const size_t jobs_fe = (jobs.size() * sizeof(HalfJob) + sizeof(fe) - 1) / sizeof(fe);
    const size_t d_chal = 0, d_jobs = d_chal + n_chal, d_layers = d_jobs + jobs_fe;
    const size_t d_T = d_layers + (size_t)(lg + 1) * N, d_S = d_T + N / 2 + 1, d_P = d_S + N;
    const size_t d_half = d_P + NE, d_parts = d_half + half_total, d_end = d_parts + 64 * prod_blocks;
    VG_TRY(vg_ctx_grow_dev(c, (void **)&f->dev, &f->dev_cap, d_end * sizeof(fe)));
    const size_t up_bytes = (n_chal + jobs_fe) * sizeof(fe);
    VG_TRY(vg_pinned_grow(c, &f->host, &f->host_cap, up_bytes));
    {
        size_t cap = f->parts_host_cap * sizeof(fe);
        void *p = f->parts_host;
        VG_TRY(vg_pinned_grow(c, &p, &cap, 64 * prod_blocks * sizeof(fe)));
        f->parts_host = (fe *)p;
        f->parts_host_cap = cap / sizeof(fe);
    }
    memcpy(f->host, H.data(), n_chal * sizeof(fe));
    memcpy((fe *)f->host + n_chal, jobs.data(), jobs.size() * sizeof(HalfJob));
    fe *D = f->dev;
    const fe *Rd = D + d_chal;
    fe *layer0 = D + d_layers, *T = D + d_T, *S = D + d_S, *P = D + d_P, *half = D + d_half, *parts = D + d_parts;
    auto layer = [&](int s) { return layer0 + (size_t)s * N; };
    auto beta = [&](const Beta4 &q) {
        BetaHalves b;
        b.lo0 = half + q.lo0;
        b.hi0 = half + q.hi0;
        b.lo1 = half + q.lo1;
        b.hi1 = half + q.hi1;
        b.fb = q.fb;
        b.mask = (1L << q.fb) - 1;
        return b;
    };
    VG_CHECK_CUDA(cudaEventRecord(f->ev[0], c->stream));
    // capture when the previous plain run had the same size, seed and buffers
    const bool same_key = f->g_lg == lg && f->g_seed == seed && f->g_key[0] == f->dev && f->g_key[1] == f->host &&
                          f->g_key[2] == f->parts_host;
    const bool capture = graphs && f->g_seen && same_key;
    CaptureGuard guard;
    if (capture) {
        fg_drop_graph(f);
        VG_CHECK_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
        guard.s = c->stream;
        guard.active = true;
    }
    VG_CHECK_CUDA(cudaMemcpyAsync(D, f->host, up_bytes, cudaMemcpyHostToDevice, c->stream));

    // ---- circuit values ----
    const fe inv_rou = vg::fe_inv(vg::fe_root_of_unity(lg));
    const fe inv_n = vg::fe_inv(vg::fe_make((uint64_t)N, 0));
    k_fg_expand<<<grid_for(N, FG_THREADS), FG_THREADS, 0, c->stream>>>(Rd + o_r, lg, layer(0));
    VG_LAUNCHED(c);
    k_fg_powers<<<grid_for((N / 2 + 31) / 32, FG_THREADS), FG_THREADS, 0, c->stream>>>(inv_rou, std::max(N / 2, 1L), T);
    VG_LAUNCHED(c);
    k_fg_halves<<<grid_for(half_total, FG_THREADS), FG_THREADS, 0, c->stream>>>(
        (const HalfJob *)(D + d_jobs), (int)jobs.size(), half_total, Rd, half);
    VG_LAUNCHED(c);
    for (int s = 1; s <= lg; ++s) {
        k_fg_butterfly<<<grid_for(N / 2, FG_THREADS), FG_THREADS, 0, c->stream>>>(layer(s - 1), layer(s), T, lg, lg - s);
        VG_LAUNCHED(c);
    }
    k_fg_products<<<dim3((unsigned)prod_blocks, 64), FG_THREADS, 0, c->stream>>>(layer(lg), inv_n, Rd + o_ep,
                                                                                 Rd + o_step, lg, S, P, parts);
    VG_LAUNCHED(c);
    VG_CHECK_CUDA(cudaMemcpyAsync(f->parts_host, parts, 64 * prod_blocks * sizeof(fe), cudaMemcpyDeviceToHost,
                                  c->stream));

    // ---- GKR: every layer's tables and rounds ----
    vg_gkr *g = f->tables;
    VG_TRY(vg_gkr_tables_rewind(g));
    auto rounds = [&](size_t r_off, int nv) -> int {
        for (int i = 0; i < nv; ++i)
            VG_TRY(vg_gkr_round(g, i == 0 ? vg_fe{0, 0} : tovg(H[r_off + i - 1]), i, nullptr, nullptr));
        return VG_OK;
    };
    vg_fe *AV, *AM;
    // addition layer
    VG_TRY(vg_gkr_tables_begin(g, (const vg_fe *)P, NE, &AV, &AM));
    k_fg_add_tables<<<std::min<unsigned>(grid_for(NE, FG_THREADS), 148u * 16u), FG_THREADS, 0, c->stream>>>(
        Rd + o_bg6, lg, NE, (fe *)AV, (fe *)AM);
    VG_LAUNCHED(c);
    VG_TRY(rounds(o_au, lg + 6));
    // multiplication layer
    VG_TRY(vg_gkr_tables_begin(g, (const vg_fe *)S, N, &AV, &AM));
    {
        // the partial sums live in AV (64 N entries), cleared by the reduction
        const bool small = N <= (1L << 14);
        const int jper = small ? 1 : 4, groups = 64 / jper, per_block = FG_THREADS * (small ? 1 : MULT_STEPS);
        const dim3 grid((unsigned)((N + per_block - 1) / per_block), (unsigned)groups);
        if (small)
            k_fg_mult_part<1><<<grid, FG_THREADS, 0, c->stream>>>(beta(mult_bg), Rd + o_ep, Rd + o_step, lg, jper,
                                                                (fe *)AV);
        else
            k_fg_mult_part<MULT_STEPS><<<grid, FG_THREADS, 0, c->stream>>>(beta(mult_bg), Rd + o_ep, Rd + o_step, lg,
                                                                         jper, (fe *)AV);
        VG_LAUNCHED(c);
        k_fg_mult_reduce<<<grid_for(N, FG_THREADS), FG_THREADS, 0, c->stream>>>((const fe *)AV, groups, N, (fe *)AV,
                                                                                (fe *)AM);
        VG_LAUNCHED(c);
    }
    VG_TRY(rounds(o_mu, lg));
    // inverse-FFT levels
    for (int d = 0; d < lg; ++d) {
        const fe *pre = layer(lg - d - 1);
        const size_t ru = Lo.lv_u(d), rv = Lo.lv_v(d);
        const int slot_p1_last = (2 * lg + 6) + 2 * lg * d + lg - 1;
        VG_TRY(vg_gkr_tables_begin(g, (const vg_fe *)pre, N, &AV, &AM));
        k_fg_ifft_p1<<<grid_for(N / 2, FG_THREADS), FG_THREADS, 0, c->stream>>>(pre, T, beta(lvl_bg[d]), lg, d,
                                                                                (fe *)AV, (fe *)AM);
        VG_LAUNCHED(c);
        VG_TRY(rounds(ru, lg));
        VG_TRY(vg_gkr_tables_begin(g, (const vg_fe *)pre, N, &AV, &AM));   // flushes phase 1: its record is written
        EqHalves bu;
        bu.lo = half + lvl_ulo[d];
        bu.hi = half + lvl_uhi[d];
        bu.fb = lg >> 1;
        bu.mask = (1L << bu.fb) - 1;
        k_fg_ifft_p2<<<grid_for(N / 2, FG_THREADS), FG_THREADS, 0, c->stream>>>(
            T, beta(lvl_bg[d]), bu, (const fe *)vg_gkr_records_dev(g) + 9 * (size_t)slot_p1_last, H[ru + lg - 1], lg, d,
            (fe *)AV, (fe *)AM);
        VG_LAUNCHED(c);
        VG_TRY(rounds(rv, lg));
    }
    int nrec;
    VG_TRY(vg_gkr_records(g, &f->recs, &nrec));
    if (nrec != nrounds) return vg_fail(VG_ERR_STATE, "fft_gkr: %d records for %d rounds", nrec, nrounds);
    if (capture) {
        guard.active = false;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
        if (e == cudaSuccess) e = cudaGraphInstantiate(&f->gexec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            // nothing of this run executed: launch it plainly, and from now on
            cudaGetLastError();
            f->gexec = nullptr;
            f->g_off = true;
            c->launches = launches0;
            return vg_fft_gkr_launch(f, lg, seed);
        }
        f->g_launched = c->launches - launches0;
        VG_CHECK_CUDA(cudaGraphLaunch(f->gexec, c->stream));
    } else if (graphs) {
        if (!same_key) fg_drop_graph(f);   // a graph of another key must not be replayed for this one
        f->g_seen = true;                  // the next run with this key is captured
        f->g_lg = lg;
        f->g_seed = seed;
        f->g_key[0] = f->dev;
        f->g_key[1] = f->host;
        f->g_key[2] = f->parts_host;
    }
    VG_CHECK_CUDA(cudaEventRecord(f->ev[1], c->stream));
    f->launched = c->launches - launches0;
    f->lg = lg;
    f->pending = true;
    return VG_OK;
}

int vg_fft_gkr_finish(vg_fft_gkr *f, vg_fft_gkr_stats *st, vg_fe *msgs, vg_fe *vals)
{
    using clk = std::chrono::steady_clock;
    if (!f || !st) return vg_fail(VG_ERR_ARG, "vg_fft_gkr_finish: null argument");
    if (!f->pending) return vg_fail(VG_ERR_STATE, "vg_fft_gkr_finish: nothing launched");
    f->pending = false;
    VG_CHECK_CUDA(cudaStreamSynchronize(f->ctx->stream));

    // ---- replay: the reference's in-process verifier over the messages ----
    const auto tv0 = clk::now();
    const int lg = f->lg;
    const long N = 1L << lg;
    const int nrounds = vg_fft_gkr_rounds(lg);
    const long prod_blocks = f->prod_blocks;
    const std::vector<fe> &H = f->H;
    const Layout Lo(lg);
    const size_t o_r0 = Lo.o_r0, o_ep = Lo.o_ep, o_au = Lo.o_au, o_av = Lo.o_av, o_mu = Lo.o_mu, o_ab = Lo.o_ab;
    const size_t o_bg6 = Lo.o_bg6;
    auto alpha_at = [&](int d) { return d == 0 ? vg::fe_one() : H[o_ab + 2 * (d - 1)]; };
    auto beta_at = [&](int d) { return d == 0 ? vg::fe_zero() : H[o_ab + 2 * (d - 1) + 1]; };
    const fe inv_rou = vg::fe_inv(vg::fe_root_of_unity(lg));
    const fe *rec = (const fe *)f->recs;
    const fe *r0 = &H[o_r0];
    bool ok = true;
    int m = 0, nv_out = 0;
    fe claim;
    {
        fe out[64];
        for (int j = 0; j < 64; ++j) {
            fe s = vg::fe_zero();
            for (long b = 0; b < prod_blocks; ++b) s = s + f->parts_host[j * prod_blocks + b];
            out[j] = s;
        }
        // V_output (:134-150): the multilinear extension of the 64 outputs at r_0
        for (int i = 0, n = 64; i < 6; ++i, n >>= 1)
            for (int k = 0; k < n / 2; ++k) out[k] = out[2 * k] * (vg::fe_one() - r0[i]) + out[2 * k + 1] * r0[i];
        claim = out[0];
    }
    auto phase = [&](size_t r_off, int nv) {
        for (int i = 0; i < nv; ++i, ++m) {
            const fe *q = rec + 9 * (size_t)m;
            if (msgs)
                for (int k = 0; k < 3; ++k) msgs[3 * m + k] = tovg(q[k]);
            if (!feq(qeval(q, vg::fe_zero()) + qeval(q, vg::fe_one()), claim)) ok = false;
            claim = qeval(q, H[r_off + i]);
        }
        const fe *last = rec + 9 * (size_t)(m - 1) + 3;
        const fe v = last[0] + H[r_off + nv - 1] * (last[1] - last[0]);
        if (vals) vals[nv_out] = tovg(v);
        ++nv_out;
        return v;
    };
    const fe one = vg::fe_one();
    // addition layer (:336-354)
    fe vu = phase(o_au, lg + 6);
    {
        fe sum = vg::fe_zero();
        for (int i = 0; i < 64; ++i) sum = sum + H[o_bg6 + i] * eq_host(&H[o_au + lg], 6, i);
        if (!feq(claim, sum * vu)) ok = false;
        claim = vu;   // alpha = 1
    }
    // multiplication layer (:438-489); r_0, r_1 are the addition layer's r_u, r_v
    vu = phase(o_mu, lg);
    {
        const fe *a0 = &H[o_au], *a1 = &H[o_av], *ru = &H[o_mu];
        fe sum = vg::fe_zero();
        for (int i = 0; i < 64; ++i) {
            fe t0 = one, t1 = vg::fe_zero(), u0 = one, u1 = one, x = H[o_ep + i];
            for (int j = 0; j < 6; ++j) {
                t0 = t0 * (((i >> j) & 1) ? a0[lg + j] : one - a0[lg + j]);
                t1 = t1 * (((i >> j) & 1) ? a1[lg + j] : one - a1[lg + j]);
            }
            for (int j = 0; j < lg; ++j) {
                u0 = u0 * (a0[j] * ru[j] * x + (one - a0[j]) * (one - ru[j]));
                u1 = u1 * (a1[j] * ru[j] * x + (one - a1[j]) * (one - ru[j]));
                x = x * x;
            }
            sum = sum + t0 * u0 + t1 * u1;
        }
        if (!feq(claim, sum * vu)) ok = false;
        claim = vu * vg::fe_make((uint64_t)N, 0);   // alpha = 1, then the scaling layer (:491-496)
    }
    // inverse-FFT levels (:681-760)
    fe rot[62];
    rot[0] = inv_rou;
    for (int i = 1; i < 62; ++i) rot[i] = rot[i - 1] * rot[i - 1];
    for (int d = 0; d < lg; ++d) {
        const size_t ru_o = Lo.lv_u(d), rv_o = Lo.lv_v(d);
        const fe *p0 = &H[Lo.prev_u(d)], *p1 = &H[Lo.prev_v(d)];
        const fe al = alpha_at(d), be = beta_at(d);
        const fe vu_d = phase(ru_o, lg);
        const fe vv_d = phase(rv_o, lg);
        const fe *ru = &H[ru_o], *rv = &H[rv_o];
        const int lk = lg - d - 1, lj = d;
        fe w = rot[d];
        const fe c0 = (one - ru[lj]) * rv[lj];
        fe uA0 = (one - p0[lg - 1]) * c0 * al, uA1 = (one - p1[lg - 1]) * c0 * be;
        fe vA0 = uA0, vA1 = uA1;
        fe uB0 = p0[lg - 1] * c0 * al, uB1 = p1[lg - 1] * c0 * be;
        fe vB0 = uB0, vB1 = uB1;
        for (int i = 0; i < lk; ++i) {
            const fe su = ru[lj + 1 + i], sv = rv[lj + 1 + i];
            const fe e0 = p0[lj + i] * su * sv, n0 = (one - p0[lj + i]) * (one - su) * (one - sv);
            const fe e1 = p1[lj + i] * su * sv, n1 = (one - p1[lj + i]) * (one - su) * (one - sv);
            uA0 = uA0 * (e0 + n0);
            uA1 = uA1 * (e1 + n1);
            vA0 = vA0 * (e0 * w + n0);
            vA1 = vA1 * (e1 * w + n1);
            uB0 = uB0 * (e0 + n0);
            uB1 = uB1 * (e1 + n1);
            vB0 = vB0 * (n0 + e0 * w);
            vB1 = vB1 * (n1 + e1 * w);
            w = w * w;
        }
        for (int i = 0; i < lj; ++i) {
            const fe t0 = p0[i] * ru[i] * rv[i] + (one - p0[i]) * (one - ru[i]) * (one - rv[i]);
            const fe t1 = p1[i] * ru[i] * rv[i] + (one - p1[i]) * (one - ru[i]) * (one - rv[i]);
            uA0 = uA0 * t0;
            uA1 = uA1 * t1;
            vA0 = vA0 * t0;
            vA1 = vA1 * t1;
            uB0 = uB0 * t0;
            uB1 = uB1 * t1;
            vB0 = vB0 * t0;
            vB1 = vB1 * t1;
        }
        if (!feq(claim, (uA0 + uA1 + uB0 + uB1) * vu_d + ((vA0 + vA1) - (vB0 + vB1)) * vv_d)) ok = false;
        claim = H[o_ab + 2 * d] * vu_d + H[o_ab + 2 * d + 1] * vv_d;
    }
    const auto t1 = clk::now();
    st->rounds = nrounds;
    st->pass = ok ? 1 : 0;
    st->proof_size = 48 * (nrounds + lg * (lg + 1) / 2);   // extension_gkr (:770-779) counts messages it never sends
    st->v_time = std::chrono::duration<double>(t1 - tv0).count();
    st->p_time = std::chrono::duration<double>(t1 - f->t0).count();
    float ms = 0;
    VG_CHECK_CUDA(cudaEventElapsedTime(&ms, f->ev[0], f->ev[1]));
    st->gpu_s = ms / 1000.0;
    st->launches = f->launched;
    return VG_OK;
}

extern "C" int vg_fft_gkr_prove(vg_fft_gkr *f, int lg, unsigned seed, vg_fft_gkr_stats *st, vg_fe *msgs, vg_fe *vals)
{
    if (!f || !st) return vg_fail(VG_ERR_ARG, "vg_fft_gkr_prove: null argument");
    const int rc = vg_fft_gkr_launch(f, lg, seed);
    if (rc != VG_OK) {
        cudaStreamSynchronize(f->ctx->stream);   // drain what was enqueued before the error
        return rc;
    }
    return vg_fft_gkr_finish(f, st, msgs, vals);
}

extern "C" int vg_fft_gkr_run(vg_ctx *ctx, int lg, unsigned seed, vg_fft_gkr_stats *st, vg_fe *msgs, vg_fe *vals)
{
    vg_fft_gkr *f;
    VG_TRY(vg_fft_gkr_create(ctx, lg, &f));
    const int rc = vg_fft_gkr_prove(f, lg, seed, st, msgs, vals);
    vg_fft_gkr_destroy(f);
    return rc;
}
