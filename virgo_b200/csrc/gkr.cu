// GKR prover kernels: layered-circuit evaluation, V_res, the phase-1/phase-2
// bookkeeping scatters and the per-round sumcheck fold + reduction.
//
// Gate records live on the device as three arrays per layer (ty: uint8,
// u, v: uint32 bit patterns; 9 bytes per gate instead of the reference's
// 24-byte AoS `gate`).
//
// Bookkeeping tables.  The reference keeps linear polynomials {a, b} (32 B per
// entry) and, at each round, evaluates the previous round's polynomial at the
// verifier's challenge (zk_prover.cpp:616-626).  Here each table is the list of
// values W (16 B per entry): at round t the entries are folded with the
// previous challenge, W'[k] = W[2k] + r (W[2k+1] - W[2k]), which is exactly
// V_mult_add[k].eval(r) of the reference, and the round sums read the pair
// (W'[2i], W'[2i+1]) as b = W'[2i], a = W'[2i+1] - W'[2i].  One fused kernel
// per round reads 4 entries of each table per thread, writes the 2 folded
// ones, and reduces the three round sums per block (exact field addition, so
// the sum does not depend on the order).
//
// Scatters.  phase*_init add gate contributions into table entries chosen by
// the gate's u (phase 1) or v (phase 2).  Field additions are done exactly with
// 64-bit integer atomics: a canonical value x < 2^61 is split into
// x mod 2^32 and x >> 32, each accumulated in its own uint64 (at most 2^30
// contributions per entry keeps both below 2^64), and a finalise pass folds
// lo + hi * 2^32 back into a canonical element.
#include "common.cuh"
#include "internal.h"
#include <algorithm>
#include <mutex>
#include <cstring>

namespace {

constexpr int GKR_THREADS = 256;

// The wiring of one layer grouped by the table entry each gate feeds in one
// sumcheck phase (phase 1: u, phase 2: v; summation gates expanded to one
// edge per summed wire).  Built once per circuit, it turns the phase inits
// into gathers: every table entry is summed by one thread (or one warp for
// long lists) and written once, without atomics.
struct EdgeSet {
    bool launched = false;        // offsets and edges enqueued by launch_edges
    bool ok = false;
    long N = 0;                   // table entries (keys)
    long E = 0;                   // edges
    uint32_t *off = nullptr;      // N + 1 offsets
    uint32_t *g = nullptr;        // gate index (the relay's u in phase 1)
    uint32_t *o = nullptr;        // the other wire (phase 1: v, phase 2: u or the summed wire)
    uint16_t *tk = nullptr;       // gate type | doubling count << 8
    uint32_t *medium = nullptr;   // keys with LIGHT_MAX < edges <= HEAVY_MIN
    long n_medium = 0;
    uint32_t *heavy = nullptr;    // (key, first edge, end edge) of keys with more than HEAVY_MIN edges
    long cap_H = 0;
    std::vector<uint32_t> heavy_host;   // the same triples on the host
    long cap_N = 0, cap_E = 0, cap_M = 0;
};

struct DevLayer {
    int bl = 0;
    long n = 0;
    uint8_t *ty = nullptr;
    uint32_t *u = nullptr, *v = nullptr;
    EdgeSet ph[2];
};

constexpr int LIGHT_MAX = 64;   // edges a single thread sums; longer lists get a warp
constexpr long HEAVY_MIN = 32768;   // longer lists are split over many CTAs
constexpr int EDGE_STATS = 4;       // per edge set: total, long keys, overflow, heavy keys
constexpr int MAX_HEAVY = 16;       // heavy keys per launch
constexpr int HEAVY_PARTS = 296;    // CTAs per heavy key

__device__ __forceinline__ fe from_int32(int32_t x)
{
    uint64_t val = (uint64_t)(int64_t)x;   // zk_prover.cpp:60-65 (int) then field_element(unsigned long long)
    uint64_t r = (val & vg::P) + (val >> 61);
    return vg::fe_make(r >= vg::P ? r - vg::P : r, 0);
}

// --------------------------------------------------------------- evaluate
__global__ void k_eval_input(const int64_t *__restrict__ u, long n, fe *__restrict__ out)
{
    long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (g < n) out[g] = from_int32((int32_t)u[g]);
}

// zk_prover::evaluate, one layer (zk_prover.cpp:68-150)
__global__ void k_eval_layer(const uint8_t *__restrict__ ty, const uint32_t *__restrict__ uu,
                             const uint32_t *__restrict__ vv, long n, const fe *__restrict__ prev,
                             fe *__restrict__ out)
{
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < n; g += (long)gridDim.x * blockDim.x) {
        const uint32_t u = uu[g], v = vv[g];
        fe r = vg::fe_zero();
        switch (ty[g]) {
        case 0: r = prev[u] + prev[v]; break;
        case 1: r = prev[u] * prev[v]; break;
        case 3: r = from_int32((int32_t)u); break;
        case 4:
        case 10: r = prev[u]; break;
        case 5:
            for (uint32_t k = u; k < v; ++k) r = r + prev[k];
            break;
        case 6: r = vg::fe_one() - prev[u]; break;
        case 7: r = prev[u] - prev[v]; break;
        case 8: {
            fe x = prev[u], y = prev[v], xy = x * y;
            r = (x + y) - (xy + xy);
        } break;
        case 9: {
            fe x = prev[u], y = prev[v];
            r = y - x * y;
        } break;
        case 12:   // sum_k prev[k] 2^(k-u), Horner from the top
            for (long k = (long)v; k >= (long)u; --k) r = (r + r) + prev[k];
            break;
        case 13: r = prev[u] * (vg::fe_one() - prev[v]); break;
        default: break;   // 2 (dummy) and unknown types evaluate to 0
        }
        out[g] = r;
    }
}

// ------------------------------------------------------------ eq tables
// out[i] = scale * prod_{b < nbits} (bit b of i ? r[b] : 1 - r[b])
__global__ void k_eq_half(const fe *__restrict__ r, int nbits, fe scale, fe *__restrict__ out)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= (1L << nbits)) return;
    fe x = scale;
    for (int b = 0; b < nbits; ++b) x = x * (((i >> b) & 1) ? r[b] : vg::fe_one() - r[b]);
    out[i] = x;
}

// Several half tables in one launch (the tables of a phase init are built
// together): table q covers threads [begin[q], begin[q + 1]).
struct EqJobs {
    const fe *r[4];
    fe *out[4];
    fe scale[4];
    int nbits[4];
    long begin[5];
    int count;
};
__global__ void k_eq_halves(EqJobs J)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= J.begin[J.count]) return;
    int q = 0;
    while (t >= J.begin[q + 1]) ++q;
    const long i = t - J.begin[q];
    const fe *r = J.r[q];
    fe x = J.scale[q];
    for (int b = 0; b < J.nbits[q]; ++b) x = x * (((i >> b) & 1) ? r[b] : vg::fe_one() - r[b]);
    J.out[q][i] = x;
}

// out[x] = lo[x & mask] * hi[x >> fh]
__global__ void k_eq_combine(const fe *__restrict__ lo, const fe *__restrict__ hi, int fh, long n, fe *__restrict__ out)
{
    const long mask = (1L << fh) - 1;
    for (long x = blockIdx.x * (long)blockDim.x + threadIdx.x; x < n; x += (long)gridDim.x * blockDim.x)
        out[x] = lo[x & mask] * hi[x >> fh];
}

// sum_x vals[x] * lo[x & mask] * hi[x >> fh]  (V_res as an inner product with eq)
__global__ void k_eq_dot(const fe *__restrict__ vals, const fe *__restrict__ lo, const fe *__restrict__ hi, int fh,
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

// ---------------------------------------------------------- accumulators
struct BetaG {
    const fe *f0, *s0, *f1, *s1;   // alpha*eq(r0 low half), eq(r0 high half), beta*..., eq(r1 high)
    int fh;
    long mask;
    // the layer's values by gate: phase 1's gathers store each gate's value
    // there (save), phase 2's read it (tab) instead of forming it again
    fe *save = nullptr;
    const fe *tab = nullptr;
    __device__ __forceinline__ fe at(long i) const
    {
        if (tab) return tab[i];
        return vg::fe_fma(f0[i & mask] * s0[i >> fh], f1[i & mask], s1[i >> fh]);
    }
};
struct BetaU {
    const fe *f, *s;
    int fh;
    long mask;
    __device__ __forceinline__ fe at(long i) const { return f[i & mask] * s[i >> fh]; }
};

__device__ __forceinline__ void acc_add(unsigned long long *acc, long j, fe x)
{
    unsigned long long *p = acc + 4 * j;
    atomicAdd(p + 0, (unsigned long long)(x.real & 0xffffffffull));
    atomicAdd(p + 1, (unsigned long long)(x.real >> 32));
    atomicAdd(p + 2, (unsigned long long)(x.img & 0xffffffffull));
    atomicAdd(p + 3, (unsigned long long)(x.img >> 32));
}
__device__ __forceinline__ void acc_sub(unsigned long long *acc, long j, fe x) { acc_add(acc, j, -x); }

__device__ __forceinline__ uint64_t fold_split(uint64_t lo, uint64_t hi)
{
    uint64_t a = (lo & vg::P) + (lo >> 61);
    a = a >= vg::P ? a - vg::P : a;
    uint64_t b = (hi & vg::P) + (hi >> 61);
    b = b >= vg::P ? b - vg::P : b;
    return vg::addp(a, vg::mulp(b, 1ull << 32));
}

__global__ void k_acc_finalize(const unsigned long long *__restrict__ acc, long n, fe *__restrict__ out)
{
    for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n; j += (long)gridDim.x * blockDim.x) {
        const unsigned long long *p = acc + 4 * j;
        out[j] = vg::fe_make(fold_split(p[0], p[1]), fold_split(p[2], p[3]));
    }
}

// add a block's sum of `x` into acc entry j with 4 atomics from thread 0
__device__ __forceinline__ void block_acc_add(unsigned long long *acc, long j, fe x, fe *sm)
{
    fe v[1] = {x};
    block_sum<1>(v, sm);
    if (threadIdx.x == 0 && !vg::fe_is_zero(v[0])) acc_add(acc, j, v[0]);
}

// sumcheck_phase1_init gate scatter (zk_prover.cpp:422-587).  am/av are the
// accumulators of add_mult_sum[.].b and addV_array[.].b.
__global__ void __launch_bounds__(GKR_THREADS) k_phase1_scatter(const uint8_t *__restrict__ ty, const uint32_t *__restrict__ uu,
                                                                const uint32_t *__restrict__ vv, long ng, BetaG bg,
                                                                const fe *__restrict__ prev, unsigned long long *am,
                                                                unsigned long long *av)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ng; i += (long)gridDim.x * blockDim.x) {
        const int t = ty[i];
        if (t == 2 || t == 3 || t == 11 || t > 13) continue;
        const uint32_t u = uu[i], v = vv[i];
        if (t == 4) {   // direct relay: beta taken at u (zk_prover.cpp:496-497)
            acc_add(am, u, bg.at(u));
            continue;
        }
        fe tmp = bg.at(i);
        switch (t) {
        case 0: acc_add(av, u, prev[v] * tmp); acc_add(am, u, tmp); break;
        case 1: acc_add(am, u, prev[v] * tmp); break;
        case 5:
            for (uint32_t j = u; j < v; ++j) acc_add(am, j, tmp);
            break;
        case 12:
            for (uint32_t j = u; j <= v; ++j) {
                acc_add(am, j, tmp);
                tmp = tmp + tmp;
            }
            break;
        case 6: acc_sub(am, u, tmp); acc_add(av, u, tmp); break;
        case 7: acc_sub(av, u, prev[v] * tmp); acc_add(am, u, tmp); break;
        case 8: {
            fe tv = tmp * prev[v];
            acc_add(av, u, tv);
            acc_add(am, u, tmp - (tv + tv));
        } break;
        case 13: {
            fe tv = tmp * prev[v];
            acc_add(am, u, tmp - tv);
        } break;
        case 9: {
            fe tv = tmp * prev[v];
            acc_add(av, u, tv);
            acc_sub(am, u, tv);
        } break;
        case 10: acc_add(am, u, tmp); break;
        default: break;
        }
    }
}

// sumcheck_phase2_init gate scatter (zk_prover.cpp:845-972).  Summation gates
// (5, 12) all add into addV_array[0]: those contributions are summed per block
// first and added with one set of atomics per block.
__global__ void __launch_bounds__(GKR_THREADS) k_phase2_scatter(const uint8_t *__restrict__ ty, const uint32_t *__restrict__ uu,
                                                                const uint32_t *__restrict__ vv, long ng, BetaG bg, BetaU bu,
                                                                const fe *__restrict__ vu_ptr, unsigned long long *am,
                                                                unsigned long long *av)
{
    __shared__ fe sm[32];
    const fe vu = *vu_ptr;
    fe zero_acc = vg::fe_zero();
    const long stride = (long)gridDim.x * blockDim.x;
    const long start = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long iters = (ng + stride - 1) / stride;
    for (long it = 0; it < iters; ++it) {
        long i = start + it * stride;
        if (i >= ng) continue;
        const int t = ty[i];
        if (t == 2 || t == 3 || t == 4 || t == 11 || t > 13) continue;
        const uint32_t u = uu[i], v = vv[i];
        fe tg = bg.at(i);
        switch (t) {
        case 1: acc_add(am, v, (tg * bu.at(u)) * vu); break;
        case 0: {
            fe tgu = tg * bu.at(u);
            acc_add(am, v, tgu);
            acc_add(av, v, tgu * vu);
        } break;
        case 5: {
            fe tvu = tg * vu;
            for (uint32_t j = u; j < v; ++j) zero_acc = zero_acc + tvu * bu.at(j);
        } break;
        case 12: {
            fe tvu = tg * vu;
            for (uint32_t j = u; j <= v; ++j) {
                zero_acc = zero_acc + tvu * bu.at(j);
                tvu = tvu + tvu;
            }
        } break;
        case 6: {
            fe tgu = tg * bu.at(u);
            acc_add(av, v, tgu - tgu * vu);
        } break;
        case 7: {
            fe tgu = tg * bu.at(u);
            acc_sub(am, v, tgu);
            acc_add(av, v, tgu * vu);
        } break;
        case 8: {
            fe tgu = tg * bu.at(u), tv = tgu * vu;
            acc_add(am, v, tgu - (tv + tv));
            acc_add(av, v, tv);
        } break;
        case 13: {
            fe tv = (tg * bu.at(u)) * vu;
            acc_sub(am, v, tv);
            acc_add(av, v, tv);
        } break;
        case 9: {
            fe tgu = tg * bu.at(u);
            acc_add(am, v, tgu - vu * tgu);
        } break;
        case 10: acc_add(av, v, (tg * bu.at(u)) * vu); break;
        default: break;
        }
    }
    block_acc_add(av, 0, zero_acc, sm);
}

// ------------------------------------------------------- wiring transpose
// Calls emit(key, gate, other, type | doublings << 8) for every edge of gate
// g in phase PH (0: keyed by u as in k_phase1_scatter, 1: keyed by v as in
// k_phase2_scatter, summation gates at key 0).
template <int PH, typename Emit>
__device__ __forceinline__ void gate_edges(int t, uint32_t g, uint32_t u, uint32_t v, Emit emit)
{
    if (t == 2 || t == 3 || t == 11 || t > 13) return;
    if (PH == 0) {
        if (t == 4) emit(u, u, 0u, (uint16_t)4);
        else if (t == 5)
            for (uint32_t j = u; j < v; ++j) emit(j, g, 0u, (uint16_t)5);
        else if (t == 12)
            for (uint32_t j = u; j <= v; ++j) emit(j, g, 0u, (uint16_t)(12 | ((j - u) << 8)));
        else emit(u, g, v, (uint16_t)t);
    } else {
        if (t == 4) return;
        if (t == 5)
            for (uint32_t j = u; j < v; ++j) emit(0u, g, j, (uint16_t)5);
        else if (t == 12)
            for (uint32_t j = u; j <= v; ++j) emit(0u, g, j, (uint16_t)(12 | ((j - u) << 8)));
        else emit(v, g, u, (uint16_t)t);
    }
}

// FILL == false: count edges per key; FILL == true: place them (cursor holds
// the offsets on entry) unless the total exceeds cap, which sets stats[2].
// The order inside a key is not fixed, which does not matter: the gathers sum
// exactly in F_p2.
template <int PH, bool FILL>
__global__ void k_edges(const uint8_t *__restrict__ ty, const uint32_t *__restrict__ uu, const uint32_t *__restrict__ vv,
                        long ng, uint32_t *__restrict__ cnt, uint32_t *__restrict__ eg, uint32_t *__restrict__ eo,
                        uint16_t *__restrict__ etk, const uint32_t *__restrict__ total, long cap,
                        unsigned long long *__restrict__ stats)
{
    if (FILL && (long)*total > cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) stats[2] = 1;
        return;
    }
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ng; i += (long)gridDim.x * blockDim.x) {
        gate_edges<PH>(ty[i], (uint32_t)i, uu[i], vv[i], [&](uint32_t key, uint32_t gv, uint32_t o, uint16_t tk) {
            const uint32_t p = atomicAdd(&cnt[key], 1u);
            if (FILL) {
                eg[p] = gv;
                eo[p] = o;
                etk[p] = tk;
            }
        });
    }
}

// keys with more than LIGHT_MAX edges into list (room for cap_list), those
// with more than HEAVY_MIN as (key, first, end) triples into heavy;
// stats[0] = edge total, stats[1] = listed keys, stats[3] = heavy keys
__global__ void k_medium_keys(const uint32_t *__restrict__ off, long N, uint32_t *__restrict__ list, long cap_list,
                              uint32_t *__restrict__ heavy, long cap_heavy, unsigned long long *__restrict__ stats)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) stats[0] = off[N];
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < N; k += (long)gridDim.x * blockDim.x) {
        const uint32_t len = off[k + 1] - off[k];
        if (len > (uint32_t)HEAVY_MIN) {
            const unsigned long long i = atomicAdd(&stats[3], 1ull);
            if ((long)i < cap_heavy) {
                heavy[3 * i] = (uint32_t)k;
                heavy[3 * i + 1] = off[k];
                heavy[3 * i + 2] = off[k + 1];
            }
        } else if (len > (uint32_t)LIGHT_MAX) {
            const unsigned long long i = atomicAdd(&stats[1], 1ull);
            if ((long)i < cap_list) list[i] = (uint32_t)k;
        }
    }
}

// contribution of one edge to the phase-1 tables (k_phase1_scatter's cases)
__device__ __forceinline__ void edge1(int tk, uint32_t gv, uint32_t o, const BetaG &bg, const fe *__restrict__ prev, fe &am,
                                      fe &av)
{
    const int t = tk & 255;
    const fe b = bg.at(gv);
    if (bg.save) bg.save[gv] = b;   // every edge of a gate stores the same value
    switch (t) {
    case 0: av = vg::fe_fma(av, prev[o], b); am = am + b; break;
    case 1: am = vg::fe_fma(am, prev[o], b); break;
    case 4:
    case 5:
    case 10: am = am + b; break;
    case 12: am = am + vg::fe_mul_pow2(b, tk >> 8); break;
    case 6: am = am - b; av = av + b; break;
    case 7: av = av - prev[o] * b; am = am + b; break;
    case 8: {
        const fe x = b * prev[o];
        av = av + x;
        am = am + (b - (x + x));
    } break;
    case 13: am = am + (b - b * prev[o]); break;
    case 9: {
        const fe x = b * prev[o];
        av = av + x;
        am = am - x;
    } break;
    default: break;
    }
}

// contribution to the phase-2 tables, split into the parts with and without
// the factor v_u (applied once per key): am = am1 + amv v_u, av = av1 + avv v_u.
// `used` collects which parts an edge touched (bit q for a[q]): a part no
// edge touched is zero, so its product with v_u can be skipped.
__device__ __forceinline__ void edge2(int tk, uint32_t gv, uint32_t o, const BetaG &bg, const BetaU &bu, fe (&a)[4],
                                      unsigned &used)
{
    const int t = tk & 255;
    const fe x = bg.at(gv) * bu.at(o);
    switch (t) {
    case 1: a[1] = a[1] + x; used |= 2; break;
    case 0: a[0] = a[0] + x; a[3] = a[3] + x; used |= 9; break;
    case 5:
    case 10: a[3] = a[3] + x; used |= 8; break;
    case 12: a[3] = a[3] + vg::fe_mul_pow2(x, tk >> 8); used |= 8; break;
    case 6: a[2] = a[2] + x; a[3] = a[3] - x; used |= 12; break;
    case 7: a[0] = a[0] - x; a[3] = a[3] + x; used |= 9; break;
    case 8: a[0] = a[0] + x; a[1] = a[1] - (x + x); a[3] = a[3] + x; used |= 11; break;
    case 13: a[1] = a[1] - x; a[3] = a[3] + x; used |= 10; break;
    case 9: a[0] = a[0] + x; a[1] = a[1] - x; used |= 3; break;
    default: break;
    }
}

// the phase-2 entries from the parts: am1 + amv v_u and av1 + avv v_u, the
// product skipped for a part no edge touched (it is zero)
__device__ __forceinline__ void phase2_out(const fe (&a)[4], unsigned used, fe vu, fe &m, fe &v)
{
    m = (used & 2) ? vg::fe_fma(a[0], a[1], vu) : a[0];
    v = (used & 8) ? vg::fe_fma(a[2], a[3], vu) : a[2];
}

struct EdgeView {
    const uint32_t *off, *g, *o;
    const uint16_t *tk;
};

// One thread per key with at most LIGHT_MAX edges; out_m / out_v are the
// add_mult_sum and addV_array tables.
template <int PH>
__global__ void __launch_bounds__(GKR_THREADS) k_gather_keys(EdgeView e, long N, BetaG bg, BetaU bu,
                                                             const fe *__restrict__ prev, const fe *__restrict__ vu_ptr,
                                                             fe *__restrict__ out_m, fe *__restrict__ out_v)
{
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < N; k += (long)gridDim.x * blockDim.x) {
        const uint32_t s = e.off[k], t = e.off[k + 1];
        if (t - s > (uint32_t)LIGHT_MAX) continue;
        if (PH == 0) {
            fe am = vg::fe_zero(), av = vg::fe_zero();
            for (uint32_t p = s; p < t; ++p) edge1(e.tk[p], e.g[p], e.o[p], bg, prev, am, av);
            out_m[k] = am;
            out_v[k] = av;
        } else if (t == s) {   // no edges: both entries are zero
            out_m[k] = vg::fe_zero();
            out_v[k] = vg::fe_zero();
        } else {
            fe a[4] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
            unsigned used = 0;
            for (uint32_t p = s; p < t; ++p) edge2(e.tk[p], e.g[p], e.o[p], bg, bu, a, used);
            phase2_out(a, used, *vu_ptr, out_m[k], out_v[k]);
        }
    }
}

// One warp per listed key (more than LIGHT_MAX edges)
template <int PH>
__global__ void __launch_bounds__(GKR_THREADS) k_gather_long(EdgeView e, const uint32_t *__restrict__ keys, long nkeys,
                                                             BetaG bg, BetaU bu, const fe *__restrict__ prev,
                                                             const fe *__restrict__ vu_ptr, fe *__restrict__ out_m,
                                                             fe *__restrict__ out_v)
{
    const int lane = threadIdx.x & 31;
    const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
    for (long w = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5; w < nkeys; w += nwarps) {
        const uint32_t k = keys[w], s = e.off[k], t = e.off[k + 1];
        if (PH == 0) {
            fe am = vg::fe_zero(), av = vg::fe_zero();
            for (uint32_t p = s + lane; p < t; p += 32) edge1(e.tk[p], e.g[p], e.o[p], bg, prev, am, av);
            am = warp_sum(am);
            av = warp_sum(av);
            if (lane == 0) {
                out_m[k] = am;
                out_v[k] = av;
            }
        } else {
            fe a[4] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
            unsigned used = 0;
            for (uint32_t p = s + lane; p < t; p += 32) edge2(e.tk[p], e.g[p], e.o[p], bg, bu, a, used);
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] = warp_sum(a[q]);
            used = __reduce_or_sync(0xffffffffu, used);
            if (lane == 0) phase2_out(a, used, *vu_ptr, out_m[k], out_v[k]);
        }
    }
}

// Keys with more than HEAVY_MIN edges (in phase 2 every summation gate's
// edges land on entry 0): CTA (x, q) sums a strided share of heavy key q's
// edges into parts[q][x], then k_heavy_finish adds the shares of each key.
struct HeavyKeys {
    uint32_t key[MAX_HEAVY], s[MAX_HEAVY], e[MAX_HEAVY];
    int count;
};

template <int PH>
__global__ void __launch_bounds__(GKR_THREADS) k_gather_heavy(EdgeView e, HeavyKeys H, BetaG bg, BetaU bu,
                                                              const fe *__restrict__ prev, fe *__restrict__ parts)
{
    __shared__ fe sm[4 * 32];
    const int q = blockIdx.y;
    fe a[4] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
    for (long p = H.s[q] + blockIdx.x * (long)blockDim.x + threadIdx.x; p < (long)H.e[q];
         p += (long)gridDim.x * blockDim.x) {
        unsigned used = 0;
        if (PH == 0) edge1(e.tk[p], e.g[p], e.o[p], bg, prev, a[0], a[1]);
        else edge2(e.tk[p], e.g[p], e.o[p], bg, bu, a, used);
    }
    block_sum<4>(a, sm);
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) parts[((long)q * gridDim.x + blockIdx.x) * 4 + k] = a[k];
}

template <int PH>
__global__ void __launch_bounds__(GKR_THREADS) k_heavy_finish(HeavyKeys H, const fe *__restrict__ parts, int nparts,
                                                              const fe *__restrict__ vu_ptr, fe *__restrict__ out_m,
                                                              fe *__restrict__ out_v)
{
    __shared__ fe sm[4 * 32];
    const int q = blockIdx.x;
    fe a[4] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x)
        for (int k = 0; k < 4; ++k) a[k] = a[k] + parts[((long)q * nparts + b) * 4 + k];
    block_sum<4>(a, sm);
    if (threadIdx.x == 0) {
        const uint32_t k = H.key[q];
        if (PH == 0) {
            out_m[k] = a[0];
            out_v[k] = a[1];
        } else {
            const fe vu = *vu_ptr;
            out_m[k] = a[0] + a[1] * vu;
            out_v[k] = a[2] + a[3] * vu;
        }
    }
}

// --------------------------------------------------- chunked round groups
// Round folds only combine neighbouring entries, so a CTA that owns a
// contiguous chunk of the three tables can run several consecutive rounds on
// it without any other CTA: a chunk of 2 RG_CHUNK entries folds into shared
// memory (RG_CHUNK entries) and keeps folding there until two entries are
// left, i.e. up to 10 rounds.  The challenges of all those rounds are known
// in advance (they come from the verifier's rand() stream), so one launch
// replaces up to 10 round launches and each table is read from HBM once per
// group instead of once per round.  Per-round partial sums are reduced by
// the last CTA to finish, which then runs the group's tail: the entries the
// chunks left (at most 2 RG_CHUNK, written out by every CTA) fold on in its
// shared memory for up to 10 more rounds, so the rounds of a phase below the
// group start take one launch.  Every round's sums go to its record.
constexpr int RG_LOG = 10, RG_CHUNK = 1 << RG_LOG, RG_THREADS = 256;
// rounds of the chunks (RG_MAX) and of a whole launch with its tail (RG_STEPS)
constexpr int RG_MAX = 12, RG_STEPS = 20;
// Per-round partial sums of a group's CTAs ([round][CTA][3]): a group on
// tables of up to N entries has at most N / RG_CHUNK CTAs, and a group split
// into small chunks (at most 2 RG_CHUNK entries) at most 2 RG_CHUNK.
static inline size_t rg_parts_len(long N) { return ((size_t)N / RG_CHUNK + 1 + 2 * RG_CHUNK) * RG_MAX * 3; }

// shared-memory index of table entry i: one pad entry per 8 keeps the
// stride-4 reads (entries 4k .. 4k+3 of a pair) and the stride-2 writes free
// of bank conflicts
__device__ __forceinline__ int rg_ix(long i) { return (int)(i + (i >> 3)); }
constexpr int RG_TABLE = RG_CHUNK + RG_CHUNK / 8;
// dynamic shared memory of a group CTA (elements): three tables, per-warp
// round sums, each round's totals and challenge, the folded pairs of the
// three-thread steps
constexpr int RG_SMEM_FE = 3 * RG_TABLE + RG_STEPS * (RG_THREADS / 32) * 3 + RG_STEPS * 4 + 6 * (RG_THREADS / 3);
struct RoundGroup {
    int chunk_log;      // log2 of a CTA's entries after its first step (at most RG_LOG)
    int nsteps;         // rounds in this launch, the tail's included (at most RG_STEPS)
    int tail;           // of those, the rounds the last CTA runs on the chunks' remaining entries
    int first_nofold;   // the first round has no fold (the round right after a phase init)
    int slot0;          // record of the first round; the others follow
    int last6;          // write the final pair (the table ends at 2 entries) into the last record
    int split3;         // steps with at most RG_THREADS / 3 pairs run three threads per pair
    const fe *r;        // fold challenge of each round (device memory, nsteps values)
};

// x0 + r (x1 - x0); LAZY: the unreduced difference and the four-product
// form (vg::fold_lazy), the same canonical value
template <bool LAZY>
__device__ __forceinline__ fe rg_fold(fe x0, fe x1, fe r)
{
    if (LAZY) return vg::fold_lazy(x0, x1, r);
    return vg::fe_fma(x0, r, x1 - x0);
}

// A round's sums over one pair: (m0 + ma x)(v0 + va x) + a0 + aa x has x^2
// term ma va, x term ma v0 + m0 va + aa = m1 v1 - m0 v0 - ma va + aa (three
// products, not four) and constant m0 v0 + a0.  FULL = false leaves out the
// x term (the group's epilogue forms it from the round's claim): two products.
template <bool FULL = true>
__device__ __forceinline__ void rg_sums(fe v0, fe v1, fe a0, fe a1, fe m0, fe m1, fe (&acc)[3])
{
    const fe va = v1 - v0, ma = m1 - m0;
    if (FULL) {
        const fe p2 = ma * va, p0 = m0 * v0;
        acc[0] = acc[0] + p2;
        acc[1] = acc[1] + ((m1 * v1 - p0 - p2) + (a1 - a0));
        acc[2] = acc[2] + p0 + a0;
    } else {   // each product added inside its last fold (vg::fe_fma)
        acc[0] = vg::fe_fma(acc[0], ma, va);
        acc[2] = vg::fe_fma(acc[2] + a0, m0, v0);
    }
}

// The x term of a round that follows another round of its phase, from the
// others: the round's polynomial s(x) = a x^2 + b x + c sums to the claim
// s(0) + s(1) = 2c + a + b, and the claim is the previous round's
// polynomial at this round's fold challenge r (the tables folded with r sum
// to exactly that), so b = prev(r) - 2c - a, the same field element as the
// sum of the pairs' x terms (zk_prover.cpp:596-787 sums them).
__device__ __forceinline__ void rg_derive(fe (&rec)[3], const fe (&prev)[3], fe r)
{
    const fe claim = (prev[0] * r + prev[1]) * r + prev[2];
    rec[1] = claim - (rec[2] + rec[2]) - rec[0];
}

// a field element read at L2 (written by other CTAs of this launch, or by an
// earlier launch)
__device__ __forceinline__ fe ld_fe_cg(const fe *p)
{
    const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2 *>(p));
    fe x;
    x.img = v.x;
    x.real = v.y;
    return x;
}

// a record's three sums, read at L2
__device__ __forceinline__ void ld_rec3(fe (&x)[3], const fe *p)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) x[k] = ld_fe_cg(p + k);
}

// warp sums of acc added into sm[step][warp][3] (a CTA's chunks accumulate
// there); warps without an active lane (first thread >= active) add nothing
__device__ __forceinline__ void rg_warp_add(fe (&acc)[3], fe *sm, int step, long active)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if ((long)(threadIdx.x & ~31) >= active) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = warp_sum(acc[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            fe *o = &sm[(step * (RG_THREADS / 32) + wid) * 3 + k];
            *o = *o + acc[k];
        }
    }
}

// The x terms of a group's rounds after its first (rg_derive), in shared
// memory:
//   b_st = a_{st-1} r^2 + b_{st-1} r + c_{st-1} - 2 c_st - a_st.
// The terms without b_{st-1} are formed
// by one thread per round, then one thread runs the chain b_st = r b_{st-1}
// + d_st.  tot: [round][3]; sr: the challenges; d: scratch [round].
__device__ __forceinline__ void rg_derive_smem(fe *tot, const fe *sr, fe *d, int nsteps)
{
    const int t = threadIdx.x;
    if (t >= 1 && t < nsteps) {
        const fe r = sr[t];
        const fe *p = tot + 3 * (t - 1), *o = tot + 3 * t;
        d[t] = ((p[0] * (r * r) + p[2]) - (o[2] + o[2])) - o[0];
    }
    __syncthreads();
    if (t == 0) {
        fe b = tot[1];
        for (int st = 1; st < nsteps; ++st) {
            b = sr[st] * b + d[st];
            tot[3 * st + 1] = b;
        }
    }
    __syncthreads();
}

// CTAs loop over the chunks (chunk q at q * cin of the input), so the grid
// stays within what is resident at once and the last CTA's reduction reads
// at most gridDim.x partials per round.  Each CTA runs its chunks as jobs,
// and the last one then runs the tail as one more job through the same step
// code (one copy of it: the default kernel stays small enough for the
// instruction cache).  The tail reads the chunks' remaining entries at L2,
// after the fence and counter that order every CTA's writes before it.
// SPLIT: the three-thread steps (VG_TUNE_GROUP_SPLIT) are compiled in only
// when asked for, for the same reason
template <bool LAZY, bool SPLIT>
__global__ void __launch_bounds__(RG_THREADS) k_round_group(const fe *__restrict__ xV, const fe *__restrict__ xA,
                                                            const fe *__restrict__ xM, long n_in, RoundGroup G,
                                                            fe *yV, fe *yA, fe *yM, fe *__restrict__ parts,
                                                            unsigned *__restrict__ counter, fe *__restrict__ rec)
{
    extern __shared__ fe smem[];
    constexpr int NW = RG_THREADS / 32;
    fe *sV = smem, *sA = smem + RG_TABLE, *sM = smem + 2 * RG_TABLE;
    fe *wsum = smem + 3 * RG_TABLE;        // [RG_STEPS][warps][3]
    fe *tot = wsum + RG_STEPS * NW * 3;    // [RG_STEPS][3]: each round's sums over the whole table
    fe *sr = tot + RG_STEPS * 3;           // [RG_STEPS]: the rounds' challenges
    fe *stage = sr + RG_STEPS;             // [pair][6] of the three-thread steps; the epilogue's scratch
    __shared__ bool last;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    for (int i = t; i < RG_STEPS * NW * 3; i += RG_THREADS) wsum[i] = vg::fe_zero();
    if (t < G.nsteps) sr[t] = ld_fe_cg(G.r + t);
    const int k1 = G.nsteps - G.tail;      // rounds of the chunks
    const long chunk = 1L << G.chunk_log;
    const long cin = G.first_nofold ? min(n_in, chunk) : min(n_in, 2L * chunk);
    const long nchunks = n_in / cin;
    const long mfin = (G.first_nofold ? cin : cin / 2) >> (k1 - 1);   // entries a chunk leaves
    const bool alone = gridDim.x == 1;
    long m = 0;          // entries in shared memory
    bool tail = false;   // the job is the tail (after every chunk)
    for (long q = blockIdx.x;;) {
        if (!tail && q >= nchunks) {
            // every chunk of this CTA is done: its round sums
            __syncthreads();
            if (alone) {   // a single CTA: its sums are the totals
                if (t < 3 * k1) {
                    fe x = vg::fe_zero();
                    for (int w = 0; w < NW; ++w) x = x + wsum[((t / 3) * NW + w) * 3 + t % 3];
                    tot[t] = x;
                }
            } else {
                if (t < 3 * k1) {
                    fe x = vg::fe_zero();
                    for (int w = 0; w < NW; ++w) x = x + wsum[((t / 3) * NW + w) * 3 + t % 3];
                    parts[((long)(t / 3) * gridDim.x + blockIdx.x) * 3 + t % 3] = x;
                }
                __threadfence();
                __syncthreads();
                if (t == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
                __syncthreads();
                if (!last) return;
                __threadfence();
                // warp st sums round st over all CTAs, four partials in flight per lane
                for (int st = wid; st < k1; st += NW) {
                    fe s3[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
                    for (long b0 = lane; b0 < gridDim.x; b0 += 4 * 32) {
                        fe x[4][3];
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const long b = b0 + 32 * j;
#pragma unroll
                            for (int k = 0; k < 3; ++k)
                                x[j][k] = b < gridDim.x ? ld_fe_cg(&parts[((long)st * gridDim.x + b) * 3 + k])
                                                        : vg::fe_zero();
                        }
#pragma unroll
                        for (int j = 0; j < 4; ++j)
#pragma unroll
                            for (int k = 0; k < 3; ++k) s3[k] = s3[k] + x[j][k];
                    }
#pragma unroll
                    for (int k = 0; k < 3; ++k) s3[k] = warp_sum(s3[k]);
                    if (lane == 0) {
                        tot[3 * st] = s3[0];
                        tot[3 * st + 1] = s3[1];
                        tot[3 * st + 2] = s3[2];
                    }
                }
            }
            if (!G.tail) break;
            tail = true;
        }
        // one job: chunk q (rounds 0 .. k1-1), or the tail (rounds k1 .. nsteps-1)
        const fe *X0 = tail ? yV : xV, *X1 = tail ? yA : xA, *X2 = tail ? yM : xM;
        const long base = tail ? 0 : q * cin, nin = tail ? nchunks * mfin : cin;
        const bool nofold = !tail && G.first_nofold;
        const int st0 = tail ? k1 : 0, st1 = tail ? G.nsteps : k1;
        m = nofold ? nin : nin / 2;   // entries in shared memory after the first step
        __syncthreads();   // wsum zeroed, sr loaded; the previous job's tables written out
        // first step: from global into shared
        {
            fe acc[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
            const fe r = sr[st0];
            for (long k = t; k < m / 2; k += RG_THREADS) {
                fe v0, v1, a0, a1, m0v, m1v;
                if (nofold) {
                    const long b = base + 2 * k;
                    v0 = ld_fe_cg(X0 + b); v1 = ld_fe_cg(X0 + b + 1);
                    a0 = ld_fe_cg(X1 + b); a1 = ld_fe_cg(X1 + b + 1);
                    m0v = ld_fe_cg(X2 + b); m1v = ld_fe_cg(X2 + b + 1);
                } else {
                    const long b = base + 4 * k;
                    v0 = rg_fold<LAZY>(ld_fe_cg(X0 + b), ld_fe_cg(X0 + b + 1), r);
                    v1 = rg_fold<LAZY>(ld_fe_cg(X0 + b + 2), ld_fe_cg(X0 + b + 3), r);
                    a0 = rg_fold<LAZY>(ld_fe_cg(X1 + b), ld_fe_cg(X1 + b + 1), r);
                    a1 = rg_fold<LAZY>(ld_fe_cg(X1 + b + 2), ld_fe_cg(X1 + b + 3), r);
                    m0v = rg_fold<LAZY>(ld_fe_cg(X2 + b), ld_fe_cg(X2 + b + 1), r);
                    m1v = rg_fold<LAZY>(ld_fe_cg(X2 + b + 2), ld_fe_cg(X2 + b + 3), r);
                }
                const int i0 = rg_ix(2 * k), i1 = rg_ix(2 * k + 1);
                sV[i0] = v0; sV[i1] = v1;
                sA[i0] = a0; sA[i1] = a1;
                sM[i0] = m0v; sM[i1] = m1v;
                rg_sums(v0, v1, a0, a1, m0v, m1v, acc);
            }
            rg_warp_add(acc, wsum, st0, m / 2);
        }
        // further steps in shared memory: fold m -> m/2, sums over m/4 pairs
        for (int st = st0 + 1; st < st1; ++st) {
            const fe r = sr[st];
            const long npairs = m / 4;
            if (SPLIT && 3 * npairs <= RG_THREADS) {
                // few pairs: three threads per pair, one per table, each
                // folding its table's two entries; the folded pairs meet in
                // `stage`, and the V and add_mult threads add the x^0 and x^2
                // sums (p0 = m0 v0 plus a0, p2 = (m1 - m0)(v1 - v0)); the x
                // term follows from the claim (rg_derive_smem)
                const int pp = t / 3, role = t - 3 * pp;
                const bool act = pp < npairs;
                fe *tab = role == 0 ? sV : (role == 1 ? sA : sM);
                fe f0 = vg::fe_zero(), f1 = vg::fe_zero();
                __syncthreads();
                if (act) {
                    f0 = rg_fold<LAZY>(tab[rg_ix(4 * pp)], tab[rg_ix(4 * pp + 1)], r);
                    f1 = rg_fold<LAZY>(tab[rg_ix(4 * pp + 2)], tab[rg_ix(4 * pp + 3)], r);
                    stage[6 * pp + 2 * role] = f0;
                    stage[6 * pp + 2 * role + 1] = f1;
                }
                __syncthreads();   // every read of this step's tables is done
                fe acc[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
                if (act) {
                    tab[rg_ix(2 * pp)] = f0;
                    tab[rg_ix(2 * pp + 1)] = f1;
                    const fe *s6 = stage + 6 * pp;   // v0 v1 a0 a1 m0 m1
                    if (role == 0) acc[2] = s6[4] * s6[0] + s6[2];
                    else if (role == 2) acc[0] = (s6[5] - s6[4]) * (s6[1] - s6[0]);
                }
                m >>= 1;
                rg_warp_add(acc, wsum, st, 3 * npairs);
                continue;
            }
            fe acc[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
            fe v0, v1, a0, a1, m0v, m1v;
            __syncthreads();
            const bool act = t < npairs;   // m / 4 <= RG_CHUNK / 4 = RG_THREADS: at most one pair per thread
            if (act) {
                const int b0 = rg_ix(4 * t), b1 = rg_ix(4 * t + 1), b2 = rg_ix(4 * t + 2), b3 = rg_ix(4 * t + 3);
                v0 = rg_fold<LAZY>(sV[b0], sV[b1], r); v1 = rg_fold<LAZY>(sV[b2], sV[b3], r);
                a0 = rg_fold<LAZY>(sA[b0], sA[b1], r); a1 = rg_fold<LAZY>(sA[b2], sA[b3], r);
                m0v = rg_fold<LAZY>(sM[b0], sM[b1], r); m1v = rg_fold<LAZY>(sM[b2], sM[b3], r);
                rg_sums<false>(v0, v1, a0, a1, m0v, m1v, acc);
            }
            __syncthreads();
            if (act) {
                const int i0 = rg_ix(2 * t), i1 = rg_ix(2 * t + 1);
                sV[i0] = v0; sV[i1] = v1;
                sA[i0] = a0; sA[i1] = a1;
                sM[i0] = m0v; sM[i1] = m1v;
            }
            m >>= 1;
            rg_warp_add(acc, wsum, st, npairs);
        }
        __syncthreads();
        // the job's remaining m entries (none when the group folded nothing);
        // the tail's go to the start of the same tables, every read of them done
        const long yo = tail ? 0 : q * m;
        for (long k = t; yV && k < m; k += RG_THREADS) {
            yV[yo + k] = sV[rg_ix(k)];
            yA[yo + k] = sA[rg_ix(k)];
            yM[yo + k] = sM[rg_ix(k)];
        }
        if (tail) break;
        q += gridDim.x;
    }
    // a single CTA or the last one: the tail's sums (its own warps'), the
    // final pair, the x terms, the records
    __syncthreads();
    if (tail && t < 3 * G.tail) {
        fe x = vg::fe_zero();
        for (int w = 0; w < NW; ++w) x = x + wsum[((k1 + t / 3) * NW + w) * 3 + t % 3];
        tot[3 * k1 + t] = x;
    }
    if (G.last6 && m == 2 && t == 0) {
        fe *l6 = rec + 9 * (G.slot0 + G.nsteps - 1) + 3;
        l6[0] = sV[0]; l6[1] = sV[1]; l6[2] = sA[0]; l6[3] = sA[1]; l6[4] = sM[0]; l6[5] = sM[1];   // rg_ix(0, 1) = 0, 1
    }
    __syncthreads();
    rg_derive_smem(tot, sr, stage, G.nsteps);
    for (int i = t; i < 3 * G.nsteps; i += RG_THREADS) rec[9 * (G.slot0 + i / 3) + i % 3] = tot[i];
    if (!alone && t == 0) *counter = 0;
}

// ------------------------------------------------ verifier's wiring predicates
// zk_verifier::predicates (zk_verifier.cpp:219-606) for a layer that is not
// data-parallel: per gate type t, the sum over the layer's gates of type t of
// beta_g(g) * beta_u(u) * beta_v(v), with the reference's special forms for
// summation (5: over u <= j < v, times beta_v(0)), exp-sum (12: over
// u <= j <= v, times 2^(j-u) beta_v(0)) and relay (10: times beta_v(0) once at
// the end); beta_g = alpha eq(r_0, g) + beta eq(r_1, g).  One partial of 14
// values per CTA.
constexpr int PRED_THREADS = 256;
__global__ void __launch_bounds__(PRED_THREADS) k_predicates(const uint8_t *__restrict__ ty, const uint32_t *__restrict__ uu,
                                                            const uint32_t *__restrict__ vv, long ng, BetaG bg, BetaU bu,
                                                            BetaU bv, uint32_t vmask, fe *__restrict__ parts)
{
    __shared__ fe sm[14 * 32];
    fe acc[14];
#pragma unroll
    for (int k = 0; k < 14; ++k) acc[k] = vg::fe_zero();
    const fe bv0 = bv.at(0);
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < ng; g += (long)gridDim.x * blockDim.x) {
        const int t = ty[g];
        if (t == 2 || t == 3 || t == 4 || t == 11 || t > 13) continue;
        const uint32_t u = uu[g], v = vv[g];
        const fe b = bg.at(g);
        switch (t) {
        case 5: {
            fe s = vg::fe_zero();
            for (uint32_t j = u; j < v; ++j) s = s + bu.at(j);
            acc[5] = acc[5] + (b * bv0) * s;
        } break;
        case 12: {
            fe s = vg::fe_zero();
            for (uint32_t j = u; j <= v; ++j) s = s + vg::fe_mul_pow2(bu.at(j), (int)(j - u));
            acc[12] = acc[12] + (b * bv0) * s;
        } break;
        case 10: acc[10] = acc[10] + b * bu.at(u); break;
        // v of a type-6 gate is not checked at upload (the gate reads u only);
        // masking keeps the read in bounds and leaves valid wires unchanged
        default: acc[t] = acc[t] + (b * bu.at(u)) * bv.at(v & vmask); break;
        }
    }
    block_sum<14>(acc, sm);
    if (threadIdx.x == 0)
        for (int k = 0; k < 14; ++k) parts[(long)blockIdx.x * 14 + k] = acc[k];
}

// ret[10] *= beta_v(0), the product of the two half tables' first entries
// (zk_verifier.cpp:600)
__global__ void k_predicates_relay(fe *__restrict__ out, const fe *__restrict__ bv_lo, const fe *__restrict__ bv_hi)
{
    out[10] = out[10] * (bv_lo[0] * bv_hi[0]);
}

// v_u = V(r_u) + mask term: the folded V pair of the last phase-1 round at r
// (zk_prover.cpp:796-797), computed where the pair is, so phase 2 can start
// without the host reading it first
__global__ void k_vu(const fe *__restrict__ last6, fe r, fe addend, fe *__restrict__ vu)
{
    *vu = (last6[0] + r * (last6[1] - last6[0])) + addend;
}

// ------------------------------------------------------------ round kernel
template <bool LAZY>
__device__ __forceinline__ fe fold(fe x0, fe x1, fe r)
{
    if (LAZY) return vg::fold_lazy(x0, x1, r);
    return vg::fe_fma(x0, r, x1 - x0);
}

// The block partials are reduced by the last block to finish (a counter in
// device memory decides which one), so one launch returns the round sums.
// The fold challenge comes from device memory (rp), so a captured launch
// sequence can be replayed with the next proof's challenges.
// A folding round's x term follows from the claim (rg_derive): prev3 holds
// the previous round's sums (the record before it, or on a synchronous
// object the sums buffer out3 itself, read before it is written).
template <bool FOLD, int THREADS, bool LAZY>
__global__ void __launch_bounds__(THREADS) k_round(const fe *__restrict__ xV, const fe *__restrict__ xAV,
                                                       const fe *__restrict__ xAM, long npairs,
                                                       const fe *__restrict__ rp,
                                                       fe *__restrict__ yV, fe *__restrict__ yAV, fe *__restrict__ yAM,
                                                       fe *__restrict__ parts, unsigned *__restrict__ counter,
                                                       fe *out3, fe *__restrict__ last6, const fe *prev3)
{
    __shared__ fe sm[3 * 32];
    __shared__ bool last;
    const fe r = FOLD ? *rp : vg::fe_zero();
    fe acc[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < npairs; i += (long)gridDim.x * blockDim.x) {
        fe v0, v1, a0, a1, m0, m1;
        if (FOLD) {
            const long b = 4 * i;
            v0 = fold<LAZY>(xV[b], xV[b + 1], r);
            v1 = fold<LAZY>(xV[b + 2], xV[b + 3], r);
            a0 = fold<LAZY>(xAV[b], xAV[b + 1], r);
            a1 = fold<LAZY>(xAV[b + 2], xAV[b + 3], r);
            m0 = fold<LAZY>(xAM[b], xAM[b + 1], r);
            m1 = fold<LAZY>(xAM[b + 2], xAM[b + 3], r);
            yV[2 * i] = v0; yV[2 * i + 1] = v1;
            yAV[2 * i] = a0; yAV[2 * i + 1] = a1;
            yAM[2 * i] = m0; yAM[2 * i + 1] = m1;
        } else {
            v0 = xV[2 * i]; v1 = xV[2 * i + 1];
            a0 = xAV[2 * i]; a1 = xAV[2 * i + 1];
            m0 = xAM[2 * i]; m1 = xAM[2 * i + 1];
        }
        if (last6 && npairs == 1) {   // the folded pairs the last round of a phase needs
            last6[0] = v0; last6[1] = v1; last6[2] = a0; last6[3] = a1; last6[4] = m0; last6[5] = m1;
        }
        rg_sums<!FOLD>(v0, v1, a0, a1, m0, m1, acc);
    }
    block_sum<3>(acc, sm);
    if (threadIdx.x == 0) {
        parts[3 * blockIdx.x + 0] = acc[0];
        parts[3 * blockIdx.x + 1] = acc[1];
        parts[3 * blockIdx.x + 2] = acc[2];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    fe tot[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            fe x;
            x.img = __ldcg(&parts[3 * b + k].img);
            x.real = __ldcg(&parts[3 * b + k].real);
            tot[k] = tot[k] + x;
        }
    }
    __syncthreads();
    block_sum<3>(tot, sm);
    if (threadIdx.x == 0) {
        if (FOLD) {
            fe prev[3];
            ld_rec3(prev, prev3);
            rg_derive(tot, prev, r);
        }
        out3[0] = tot[0];
        out3[1] = tot[1];
        out3[2] = tot[2];
        *counter = 0;
    }
}

// The two rounds' sums of a paired pass: one block reduction of the six
// values, a CTA's partials into parts, and the last CTA to finish (a counter
// in device memory decides which) adds every CTA's into the two records.
// The second round's x term, and the first's when it folds (derive_a), follow
// from the claims (rg_derive): the first round's claim is the record before
// out_a at ra, the second's the first round's polynomial at rb.
__device__ __forceinline__ void round2_finish(const fe (&sa)[3], const fe (&sb)[3], fe *sm, bool &last,
                                              fe *__restrict__ parts, unsigned *__restrict__ counter,
                                              fe *out_a, fe *__restrict__ out_b, bool derive_a, fe ra, fe rb)
{
    fe acc[6] = {sa[0], sa[1], sa[2], sb[0], sb[1], sb[2]};
    block_sum<6>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) parts[6 * blockIdx.x + k] = acc[k];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    fe tot[6] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            fe x;
            x.img = __ldcg(&parts[6 * b + k].img);
            x.real = __ldcg(&parts[6 * b + k].real);
            tot[k] = tot[k] + x;
        }
    }
    __syncthreads();
    block_sum<6>(tot, sm);
    if (threadIdx.x == 0) {
        fe A[3] = {tot[0], tot[1], tot[2]}, B[3] = {tot[3], tot[4], tot[5]};
        if (derive_a) {
            fe prev[3];
            ld_rec3(prev, out_a - 9);
            rg_derive(A, prev, ra);
        }
        rg_derive(B, A, rb);
        out_a[0] = A[0]; out_a[1] = A[1]; out_a[2] = A[2];
        out_b[0] = B[0]; out_b[1] = B[1]; out_b[2] = B[2];
        *counter = 0;
    }
}

// Two consecutive rounds in one pass over tables above the group start
// (deferred mode): rounds only combine neighbouring entries and both
// challenges are known, so a thread takes 8 consecutive entries of each table
// (4 when the first round is the unfolded one after a phase init), folds them
// with ra into 4, adds the first round's sums over those two pairs, folds
// with rb into 2, adds the second round's sums over that pair and writes the
// 2 entries: one read of the tables for two rounds, a quarter of them
// written.  Both rounds' sums go through one block reduction and the
// last-block pass (6 values per CTA).
// (both challenges from device memory: rp[0] for the first fold, rp[1] for
// the second)
template <bool FOLD, int THREADS, bool LAZY>
__global__ void __launch_bounds__(THREADS) k_round2(const fe *__restrict__ xV, const fe *__restrict__ xAV,
                                                    const fe *__restrict__ xAM, long nquads,
                                                    const fe *__restrict__ rp,
                                                    fe *__restrict__ yV, fe *__restrict__ yAV, fe *__restrict__ yAM,
                                                    fe *__restrict__ parts, unsigned *__restrict__ counter,
                                                    fe *__restrict__ out_a, fe *__restrict__ out_b)
{
    __shared__ fe sm[6 * 32];
    __shared__ bool last;
    const fe ra = FOLD ? rp[0] : vg::fe_zero(), rb = rp[1];
    fe sa[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()}, sb[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nquads; i += (long)gridDim.x * blockDim.x) {
        fe v[4], a[4], m[4];
        if (FOLD) {
            const long b = 8 * i;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v[k] = fold<LAZY>(xV[b + 2 * k], xV[b + 2 * k + 1], ra);
                a[k] = fold<LAZY>(xAV[b + 2 * k], xAV[b + 2 * k + 1], ra);
                m[k] = fold<LAZY>(xAM[b + 2 * k], xAM[b + 2 * k + 1], ra);
            }
        } else {
            const long b = 4 * i;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v[k] = xV[b + k];
                a[k] = xAV[b + k];
                m[k] = xAM[b + k];
            }
        }
        rg_sums<!FOLD>(v[0], v[1], a[0], a[1], m[0], m[1], sa);
        rg_sums<!FOLD>(v[2], v[3], a[2], a[3], m[2], m[3], sa);
        const fe v0 = fold<LAZY>(v[0], v[1], rb), v1 = fold<LAZY>(v[2], v[3], rb);
        const fe a0 = fold<LAZY>(a[0], a[1], rb), a1 = fold<LAZY>(a[2], a[3], rb);
        const fe m0 = fold<LAZY>(m[0], m[1], rb), m1 = fold<LAZY>(m[2], m[3], rb);
        rg_sums<false>(v0, v1, a0, a1, m0, m1, sb);
        yV[2 * i] = v0; yV[2 * i + 1] = v1;
        yAV[2 * i] = a0; yAV[2 * i + 1] = a1;
        yAM[2 * i] = m0; yAM[2 * i + 1] = m1;
    }
    round2_finish(sa, sb, sm, last, parts, counter, out_a, out_b, FOLD, ra, rb);
}

// The phase's table build fused with its first two rounds (deferred mode,
// paired rounds, tables above the group start).  A thread takes a quad of
// consecutive keys, sums each key's edges as k_gather_keys does (a key with
// more than LIGHT_MAX edges was summed beforehand by k_gather_long or
// k_gather_heavy into tm / tv, read here), reads the quad's V entries and
// runs k_round2's unfolded body on them: the addV and add_mult tables are
// never written in full, and the pass after it starts from the folded
// quarter.
struct GatherArgs {
    EdgeView e;
    BetaG bg;
    BetaU bu;
    const fe *prev;   // phase 1: the layer below's values, the edges' other operand
    const fe *vu;     // phase 2: v_u (device scalar)
    fe *tm, *tv;      // the add_mult and addV tables: here only the long and heavy keys' entries are read
};

template <int PH, int THREADS>
__global__ void __launch_bounds__(THREADS) k_gather_round2(GatherArgs ga, const fe *__restrict__ xV, long nquads,
                                                           const fe *__restrict__ rp, fe *__restrict__ yV,
                                                           fe *__restrict__ yAV, fe *__restrict__ yAM,
                                                           fe *__restrict__ parts, unsigned *__restrict__ counter,
                                                           fe *__restrict__ out_a, fe *__restrict__ out_b)
{
    __shared__ fe sm[6 * 32];
    __shared__ bool last;
    const fe rb = rp[1];
    const fe vu = PH == 1 ? *ga.vu : vg::fe_zero();
    fe sa[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()}, sb[3] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nquads; i += (long)gridDim.x * blockDim.x) {
        const long b = 4 * i;
        fe v[4], a[4], m[4];
        uint32_t off[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) off[k] = ga.e.off[b + k];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = xV[b + k];
            const uint32_t s = off[k], t = off[k + 1];
            if (t - s > (uint32_t)LIGHT_MAX) {
                m[k] = ga.tm[b + k];
                a[k] = ga.tv[b + k];
            } else if (PH == 0) {
                fe am = vg::fe_zero(), av = vg::fe_zero();
                for (uint32_t p = s; p < t; ++p) edge1(ga.e.tk[p], ga.e.g[p], ga.e.o[p], ga.bg, ga.prev, am, av);
                m[k] = am;
                a[k] = av;
            } else {
                fe q[4] = {vg::fe_zero(), vg::fe_zero(), vg::fe_zero(), vg::fe_zero()};
                unsigned used = 0;
                for (uint32_t p = s; p < t; ++p) edge2(ga.e.tk[p], ga.e.g[p], ga.e.o[p], ga.bg, ga.bu, q, used);
                phase2_out(q, used, vu, m[k], a[k]);
            }
        }
        rg_sums(v[0], v[1], a[0], a[1], m[0], m[1], sa);
        rg_sums(v[2], v[3], a[2], a[3], m[2], m[3], sa);
        const fe v0 = fold<false>(v[0], v[1], rb), v1 = fold<false>(v[2], v[3], rb);
        const fe a0 = fold<false>(a[0], a[1], rb), a1 = fold<false>(a[2], a[3], rb);
        const fe m0 = fold<false>(m[0], m[1], rb), m1 = fold<false>(m[2], m[3], rb);
        rg_sums<false>(v0, v1, a0, a1, m0, m1, sb);
        yV[2 * i] = v0; yV[2 * i + 1] = v1;
        yAV[2 * i] = a0; yAV[2 * i + 1] = a1;
        yAM[2 * i] = m0; yAM[2 * i + 1] = m1;
    }
    round2_finish(sa, sb, sm, last, parts, counter, out_a, out_b, false, vg::fe_zero(), rb);
}

vg::fe tofe(vg_fe x) { return vg::fe_make(x.real, x.img); }
vg_fe tovg(vg::fe x) { vg_fe r; r.real = x.real; r.img = x.img; return r; }

// ---------------------------------------------------- device circuit build
// Input layer: values from the file's u (read through int, zk_prover.cpp:60-65)
// and the padding gates (3, 0, 0), i.e. value 0, up to 2^bl; types must be 2 or 3.
__global__ void k_build_input(const uint8_t *__restrict__ ty, const int64_t *__restrict__ u, long n, long width,
                              fe *__restrict__ vals, unsigned long long *__restrict__ err)
{
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < width; g += (long)gridDim.x * blockDim.x) {
        if (g < n) {
            const int t = ty[g];
            if (t != 2 && t != 3) atomicMin(err, (0ull << 40) | (unsigned long long)g);
            vals[g] = from_int32((int32_t)u[g]);
        } else {
            vals[g] = vg::fe_zero();
        }
    }
}

// the relay layer the reader inserts above the input (zk_verifier.cpp:114, 123):
// relay gates (4, g, 0) over the padded input, dummies (2, 0, 0) above it
__global__ void k_build_relay(long padded, long width, uint8_t *__restrict__ ty, uint32_t *__restrict__ u,
                              uint32_t *__restrict__ v)
{
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < width; g += (long)gridDim.x * blockDim.x) {
        ty[g] = g < padded ? 4 : 2;
        u[g] = g < padded ? (uint32_t)g : 0u;
        v[g] = 0;
    }
}

// One file layer into prover layer `li`: wires narrowed to uint32, checked
// against the previous layer's width (the reader's asserts,
// zk_verifier.cpp:70-102), v cleared for NOT and relay gates, dummy (2, 0, 0)
// gates above n.  The first bad gate is reported as (li << 40) | g.
template <typename IDX>
__global__ void k_build_layer(const uint8_t *__restrict__ ty_in, const IDX *__restrict__ u_in, const IDX *__restrict__ v_in,
                              long n, long width, long prev_width, int li, uint8_t *__restrict__ ty, uint32_t *__restrict__ u,
                              uint32_t *__restrict__ v, unsigned long long *__restrict__ err)
{
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < width; g += (long)gridDim.x * blockDim.x) {
        if (g >= n) {
            ty[g] = 2;
            u[g] = 0;
            v[g] = 0;
            continue;
        }
        const int t = ty_in[g];
        const long long a = (long long)u_in[g], b = (long long)v_in[g];
        bool ok;
        if (t == 2 || t == 3) ok = true;
        else if (t == 5) ok = a >= 0 && a < prev_width && b > a && b <= prev_width;
        else if (t == 12) ok = a >= 0 && a <= b && b < prev_width && b - a + 1 <= 60;
        else if (t == 6 || t == 10) ok = a >= 0 && a < prev_width;
        else if (t > 13 || t == 11) ok = false;
        else ok = a >= 0 && a < prev_width && b >= 0 && b < prev_width && (t != 13 || a == b) && (t != 4 || a < width);
        if (!ok) atomicMin(err, ((unsigned long long)li << 40) | (unsigned long long)g);
        ty[g] = ok ? (uint8_t)t : (uint8_t)2;
        u[g] = ok ? (uint32_t)a : 0u;
        v[g] = ok && t != 6 && t != 10 ? (uint32_t)b : 0u;
    }
}

}  // namespace

struct vg_circuit {
    vg_ctx *ctx = nullptr;     // the context it was built on (may be gone when forks outlive it)
    int device = 0;
    int depth = 0;
    int max_bl = 0;
    std::vector<DevLayer> L;
    fe *input = nullptr;   // layer 0 values
    // capacities (entries) of the arrays above, for reuse by vg_circuit_build
    std::vector<long> cap;
    long input_cap = 0;
    void *staging = nullptr;   // upload staging for one layer
    size_t staging_cap = 0;
    unsigned long long *err = nullptr;
    uint32_t *work = nullptr;   // edge build: cursors and scan temporaries
    size_t work_cap = 0;        // words
    unsigned long long *edge_stats = nullptr;   // 3 per edge set: total, long keys, overflow
    int edge_stats_cap = 0;
    std::vector<unsigned long long> edge_stats_host;
};

// One deferred round launch (k_round, k_round2 or k_round_group), held until
// the next flush so that a phase's rounds are issued together: after one H2D
// copy of their challenges, plainly or as a captured CUDA graph.
struct RoundLaunch {
    int kind = 0;               // 0 k_round, 1 k_round2, 2 k_round_group, 3 k_gather_round2
    bool fold = false;
    bool lazy = false;          // folds in the unreduced four-product form (VG_TUNE_LAZY_FOLD)
    int threads = 0;
    unsigned grid = 0;
    long count = 0;             // pairs (k_round), quads (k_round2), input entries (group)
    const fe *x[3] = {nullptr, nullptr, nullptr};
    fe *y[3] = {nullptr, nullptr, nullptr};
    int slot = 0;               // challenge slot of the (first) round
    fe *oa = nullptr, *ob = nullptr;   // k_round: sums, folded pair; k_round2: the two rounds' sums
    const fe *prev = nullptr;   // k_round that folds: the previous round's sums
    RoundGroup G{};             // k_round_group (G.r set when issued)
    GatherArgs ga{};            // k_gather_round2: the table build's operands
    int ph = 0;                 // k_gather_round2: the phase
    double prof_bytes = 0;
};

// A phase's round launches captured once and replayed: the key lists every
// pointer, size and shape the graph's nodes use, so a replay does exactly
// what issuing the same launches would.
struct PhaseGraph {
    std::vector<uint64_t> key;
    uint64_t hash = 0;
    cudaGraphExec_t exec = nullptr;
    long launches = 0;
};

struct vg_gkr {
    vg_ctx *ctx = nullptr;
    const vg_circuit *C = nullptr;
    std::vector<fe *> vals;              // per layer, into vals_slab (layer 0: the circuit's input)
    fe *vals_slab = nullptr;
    long vals_cap = 0, N_cap = 0, acc_cap = 0;
    fe *buf[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};   // ping-pong V, AV, AM
    unsigned long long *acc = nullptr;   // 2 tables x 4 words x 2^max_bl
    fe *eq = nullptr;                    // half tables
    fe *rbuf = nullptr;                  // challenges (device copy)
    fe *round_parts = nullptr;           // block partials of the round kernels (6 x 148 x 8 values)
    fe *round_out = nullptr;             // round sums (3) written by the last block
    unsigned *round_counter = nullptr;   // blocks finished, reset by the last one
    long eq_half = 0;
    int layer = -1, length_g = 0;
    long n = 0;                          // current table length
    const fe *cur[3] = {nullptr, nullptr, nullptr};
    int next_buf = 1;
    bool round0_pending = false;
    BetaG bg{};
    BetaU bu{};                          // eq(r_u) halves of phase 2
    fe *vu = nullptr;                    // v_u of phase 2 (device scalar)
    // deferred mode: results stay on the device as records of 9 values
    // (round: 3 sums + the 6 folded values when one pair remained;
    // v_res: the value), read back once with vg_gkr_records
    bool deferred = false;
    fe *rec = nullptr;
    int rec_cap = 0, rec_n = 0;
    fe *rec_host = nullptr;              // pinned
    int rec_host_cap = 0;
    // deferred rounds not yet launched: they run as one k_round_group
    std::vector<fe> pend_r;
    int pend_slot0 = 0;
    long pend_n0 = 0;                    // table length before the group's first round
    long pend_chunk = 0;                 // a CTA's entries after its first step
    bool pend_nofold = false;
    fe *rg_parts = nullptr;              // per-CTA, per-round partial sums of a group
    // deferred round above the group start held back to run together with
    // the next round in one k_round2 pass (VG_TUNE_ROUND_FUSE = 2)
    bool held = false;
    bool held_fold = false;
    int held_slot = 0;
    long held_n = 0;                     // table length before the held round
    fe *heavy_parts = nullptr;           // per-CTA partial sums of heavy keys
    fe *bgt = nullptr;                   // beta_g by gate of the current layer (2^max_bl entries)
    int bgt_layer = -1;                  // the layer whose phase-1 gathers filled bgt, -1 none
    // a deferred phase's table build left to run inside its first paired
    // pass (k_gather_round2, VG_TUNE_GATHER_FUSE): the build's operands until
    // that pass is queued, or until another launch needs the tables whole
    bool gather_pending = false;
    int gather_ph = 0;
    long gather_n = 0;                   // table length
    double gather_bytes = 0;             // the build's algorithmic bytes
    GatherArgs gather{};
    // fold challenges of the deferred rounds: record slot k's at rhost[k]
    // (pinned, written when the round is queued) and rdev[k] (copied once per
    // flush); a synchronous round's at rsync_host / rsync_dev
    fe *rdev = nullptr, *rhost = nullptr;
    size_t rhost_cap = 0;                // bytes
    int r_cap = 0;                       // slots of rdev
    fe *rsync_dev = nullptr, *rsync_host = nullptr;
    // deferred round launches not issued yet, and the challenge slots they read
    std::vector<RoundLaunch> pend_launch;
    int pend_lo = 0, pend_hi = 0;
    // captured phase graphs; keys seen once (a key is captured the second
    // time it comes, replayed from then on)
    std::vector<PhaseGraph> graphs;
    std::vector<uint64_t> seen;
    bool graphs_off = false;
    long long graph_replays = 0, graph_captures = 0;
};

static int flush_rounds(vg_gkr *g);
static void destroy_graphs(vg_gkr *g);

// ------------------------------------------------------------------ circuit
static int grow_u32(vg_ctx *c, uint32_t **p, long *cap, long n)
{
    if (n <= *cap) return VG_OK;
    vg_release(c, *p);
    *p = nullptr;
    *cap = 0;
    VG_TRY(vg_alloc(c, (void **)p, (size_t)std::max(n, 1L) * 4));
    *cap = n;
    return VG_OK;
}

static int alloc_edges(vg_ctx *c, EdgeSet &E, long n)
{
    vg_release(c, E.g);
    vg_release(c, E.o);
    vg_release(c, E.tk);
    E.g = E.o = nullptr;
    E.tk = nullptr;
    E.cap_E = 0;
    n = std::max(n, 1L);
    VG_TRY(vg_alloc(c, (void **)&E.g, (size_t)n * 4));
    VG_TRY(vg_alloc(c, (void **)&E.o, (size_t)n * 4));
    VG_TRY(vg_alloc(c, (void **)&E.tk, (size_t)n * 2));
    E.cap_E = n;
    return VG_OK;
}

// Enqueues the fill of edge set ph of layer li (offsets already scanned) and
// the list of its long keys.
static int fill_edges(vg_circuit *c, int li, int ph)
{
    vg_ctx *ctx = c->ctx;
    DevLayer &D = c->L[li];
    EdgeSet &E = D.ph[ph];
    const long N = E.N;
    unsigned long long *st = c->edge_stats + EDGE_STATS * (2 * li + ph);
    const unsigned grid = std::min<unsigned>(grid_for(D.n, 256), 148u * 32u);
    VG_CHECK_CUDA(cudaMemsetAsync(st, 0, EDGE_STATS * 8, ctx->stream));
    VG_CHECK_CUDA(cudaMemcpyAsync(c->work, E.off, N * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    if (ph == 0)
        k_edges<0, true><<<grid, 256, 0, ctx->stream>>>(D.ty, D.u, D.v, D.n, c->work, E.g, E.o, E.tk, E.off + N, E.cap_E, st);
    else
        k_edges<1, true><<<grid, 256, 0, ctx->stream>>>(D.ty, D.u, D.v, D.n, c->work, E.g, E.o, E.tk, E.off + N, E.cap_E, st);
    VG_LAUNCHED(ctx);
    // a key with more than LIGHT_MAX edges: at most cap_E / (LIGHT_MAX + 1) of them
    VG_TRY(grow_u32(ctx, &E.medium, &E.cap_M, E.cap_E / (LIGHT_MAX + 1) + 1));
    VG_TRY(grow_u32(ctx, &E.heavy, &E.cap_H, 3 * (E.cap_E / HEAVY_MIN + 1)));
    k_medium_keys<<<std::min<unsigned>(grid_for(N, 256), 148u * 32u), 256, 0, ctx->stream>>>(
        E.off, N, E.medium, E.cap_M, E.heavy, E.cap_H / 3, st);
    VG_LAUNCHED(ctx);
    return VG_OK;
}

// Enqueues the phase-1 and phase-2 edge sets of prover layer li (see
// EdgeSet), without synchronising: the edge arrays are sized for one edge per
// gate, and a set that needs more is rebuilt by finish_edges.
static int launch_edges(vg_circuit *c, int li)
{
    vg_ctx *ctx = c->ctx;
    DevLayer &D = c->L[li];
    D.ph[0].ok = D.ph[1].ok = false;
    D.ph[0].launched = D.ph[1].launched = false;
    const char *mode = getenv("VIRGO_PHASE_TABLES");   // "atomic": keep the scatter path (tests compare both)
    if (mode && !strcmp(mode, "atomic")) return VG_OK;
    const long N = c->L[li - 1].n;
    const unsigned grid = std::min<unsigned>(grid_for(D.n, 256), 148u * 32u);
    const size_t work = (size_t)N + (size_t)vg_scan_tmp_words(N);
    if (work > c->work_cap) {
        vg_release(ctx, c->work);
        c->work = nullptr;
        c->work_cap = 0;
        VG_TRY(vg_alloc(ctx, (void **)&c->work, work * 4));
        c->work_cap = work;
    }
    for (int ph = 0; ph < 2; ++ph) {
        EdgeSet &E = D.ph[ph];
        E.N = N;
        VG_TRY(grow_u32(ctx, &E.off, &E.cap_N, N + 1));
        if (E.cap_E < D.n) VG_TRY(alloc_edges(ctx, E, D.n));
        VG_CHECK_CUDA(cudaMemsetAsync(E.off, 0, (N + 1) * 4, ctx->stream));
        if (ph == 0)
            k_edges<0, false><<<grid, 256, 0, ctx->stream>>>(D.ty, D.u, D.v, D.n, E.off, nullptr, nullptr, nullptr, nullptr, 0,
                                                            nullptr);
        else
            k_edges<1, false><<<grid, 256, 0, ctx->stream>>>(D.ty, D.u, D.v, D.n, E.off, nullptr, nullptr, nullptr, nullptr, 0,
                                                            nullptr);
        VG_LAUNCHED(ctx);
        VG_TRY(vg_scan_u32(ctx, E.off, N, c->work + N));
        VG_TRY(fill_edges(c, li, ph));
        E.launched = true;
    }
    return VG_OK;
}

// Enqueues the edge sets of every layer and the copy of their counts to
// c->edge_stats_host (valid after the stream is synchronised).
static int launch_all_edges(vg_circuit *c)
{
    const int need = EDGE_STATS * 2 * c->depth;
    if (need > c->edge_stats_cap) {
        vg_release(c->ctx, c->edge_stats);
        c->edge_stats = nullptr;
        c->edge_stats_cap = 0;
        VG_TRY(vg_alloc(c->ctx, (void **)&c->edge_stats, need * 8));
        c->edge_stats_cap = need;
    }
    c->edge_stats_host.assign(need, 0);
    VG_CHECK_CUDA(cudaMemsetAsync(c->edge_stats, 0, need * 8, c->ctx->stream));
    for (int li = 1; li < c->depth; ++li) VG_TRY(launch_edges(c, li));
    VG_CHECK_CUDA(cudaMemcpyAsync(c->edge_stats_host.data(), c->edge_stats, need * 8, cudaMemcpyDeviceToHost, c->ctx->stream));
    return VG_OK;
}

// The heavy keys' (key, first, end) triples to the host (circuits that have
// any: one more synchronisation at build time).
static int read_heavy(vg_circuit *c, EdgeSet &E, long n_heavy)
{
    E.heavy_host.assign(3 * (size_t)n_heavy, 0);
    if (!n_heavy) return VG_OK;
    if (3 * n_heavy > E.cap_H) return vg_fail(VG_ERR_STATE, "heavy key list overflow");
    VG_CHECK_CUDA(cudaMemcpyAsync(E.heavy_host.data(), E.heavy, 3 * n_heavy * 4, cudaMemcpyDeviceToHost, c->ctx->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->ctx->stream));
    return VG_OK;
}

// Reads the edge counts of every layer (the caller synchronised the stream
// after stats_host was copied) and rebuilds the sets whose edges did not fit.
static int finish_edges(vg_circuit *c, const unsigned long long *stats_host)
{
    bool refill = false;
    for (int li = 1; li < c->depth; ++li)
        for (int ph = 0; ph < 2; ++ph) {
            EdgeSet &E = c->L[li].ph[ph];
            const unsigned long long *st = stats_host + EDGE_STATS * (2 * li + ph);
            if (!E.launched) continue;
            if (st[0] >= (1ull << 31)) {   // too many edges: atomic path
                E.launched = false;
                continue;
            }
            E.E = (long)st[0];
            if (st[2]) {   // overflowed: exact size now known (rare: summation gates)
                VG_TRY(alloc_edges(c->ctx, E, E.E));
                refill = true;
                E.ok = false;
                continue;
            }
            E.n_medium = (long)st[1];
            VG_TRY(read_heavy(c, E, (long)st[3]));
            E.ok = true;
        }
    if (!refill) return VG_OK;
    // the offsets are intact (the fill works on a copy): fill again with room
    vg_ctx *ctx = c->ctx;
    for (int li = 1; li < c->depth; ++li)
        for (int ph = 0; ph < 2; ++ph) {
            EdgeSet &E = c->L[li].ph[ph];
            if (!E.launched || E.ok || E.cap_E < E.E || E.E >= (1L << 31)) continue;
            VG_TRY(fill_edges(c, li, ph));
            unsigned long long st[EDGE_STATS];
            VG_CHECK_CUDA(cudaMemcpyAsync(st, c->edge_stats + EDGE_STATS * (2 * li + ph), EDGE_STATS * 8,
                                          cudaMemcpyDeviceToHost, ctx->stream));
            VG_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
            if (st[2]) continue;   // still does not fit: atomic path
            E.n_medium = (long)st[1];
            VG_TRY(read_heavy(c, E, (long)st[3]));
            E.ok = true;
        }
    return VG_OK;
}

extern "C" int vg_circuit_upload(vg_ctx *ctx, int depth, const int *bit_length, const uint8_t *const *ty,
                                 const int64_t *const *u, const int64_t *const *v, vg_circuit **out)
{
    if (!ctx || !out || depth < 2 || !bit_length || !ty || !u || !v)
        return vg_fail(VG_ERR_ARG, "vg_circuit_upload: bad argument (depth %d)", depth);
    for (int i = 0; i < depth; ++i)
        if (bit_length[i] < 0 || bit_length[i] > 30) return vg_fail(VG_ERR_ARG, "layer %d: bit length %d", i, bit_length[i]);
    // validate every gate against the previous layer (zk_verifier.cpp:70-102)
    for (int i = 1; i < depth; ++i) {
        const long n = 1L << bit_length[i], np = 1L << bit_length[i - 1];
        for (long g = 0; g < n; ++g) {
            const int t = ty[i][g];
            const int64_t a = u[i][g], b = v[i][g];
            bool ok = true;
            if (t > 13 || t == 11) ok = false;
            else if (t == 3 || t == 2) ok = true;
            else if (t == 5) ok = a >= 0 && a < np && b > a && b <= np;
            else if (t == 12) ok = a >= 0 && b >= a && b < np && b - a + 1 <= 60;
            else if (t == 6 || t == 10 || t == 4) ok = a >= 0 && a < np;
            else ok = a >= 0 && a < np && b >= 0 && b < np && (t != 13 || a == b);
            if (t == 4 && a >= n) ok = false;   // relay reads beta at u over this layer's bits
            if (!ok)
                return vg_fail(VG_ERR_ARG, "layer %d gate %ld: type %d u %lld v %lld invalid for previous width %ld",
                               i, g, t, (long long)a, (long long)b, np);
        }
    }
    vg_circuit *c = new vg_circuit();
    c->ctx = ctx;
    c->device = ctx->device;
    c->depth = depth;
    c->L.resize(depth);
    auto fail = [&](int rc) { vg_circuit_destroy(c); return rc; };
    for (int i = 0; i < depth; ++i) {
        DevLayer &D = c->L[i];
        D.bl = bit_length[i];
        D.n = 1L << D.bl;
        c->max_bl = std::max(c->max_bl, D.bl);
        if (i == 0) {
            int64_t *tmp;
            if (cudaMalloc(&c->input, D.n * sizeof(fe)) != cudaSuccess || cudaMalloc(&tmp, D.n * 8) != cudaSuccess) {
                cudaGetLastError();
                return fail(vg_fail(VG_ERR_OOM, "circuit input allocation"));
            }
            cudaMemcpyAsync(tmp, u[0], D.n * 8, cudaMemcpyHostToDevice, ctx->stream);
            k_eval_input<<<grid_for(D.n, 256), 256, 0, ctx->stream>>>(tmp, D.n, c->input);
            ctx->launches++;
            cudaStreamSynchronize(ctx->stream);
            cudaFree(tmp);
            continue;
        }
        std::vector<uint32_t> hu(D.n), hv(D.n);
        for (long g = 0; g < D.n; ++g) {
            hu[g] = (uint32_t)u[i][g];
            hv[g] = (ty[i][g] == 6 || ty[i][g] == 10) ? 0u : (uint32_t)v[i][g];   // zk_verifier.cpp:87-98
        }
        if (cudaMalloc(&D.ty, D.n) != cudaSuccess || cudaMalloc(&D.u, D.n * 4) != cudaSuccess ||
            cudaMalloc(&D.v, D.n * 4) != cudaSuccess) {
            cudaGetLastError();
            return fail(vg_fail(VG_ERR_OOM, "circuit layer %d allocation", i));
        }
        cudaMemcpyAsync(D.ty, ty[i], D.n, cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(D.u, hu.data(), D.n * 4, cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(D.v, hv.data(), D.n * 4, cudaMemcpyHostToDevice, ctx->stream);
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return fail(vg_fail(VG_ERR_CUDA, "circuit upload: %s", cudaGetErrorString(e)));
    }
    int rc = launch_all_edges(c);
    if (rc == VG_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return fail(vg_fail(VG_ERR_CUDA, "circuit upload: %s", cudaGetErrorString(e)));
        rc = finish_edges(c, c->edge_stats_host.data());
    }
    if (rc != VG_OK) return fail(rc);
    *out = c;
    return VG_OK;
}

extern "C" int vg_circuit_destroy(vg_circuit *c)
{
    if (!c) return VG_OK;
    // not through c->ctx: forked sessions may release the circuit after the
    // context that built it is gone
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    for (auto &D : c->L) {
        cudaFree(D.ty);
        cudaFree(D.u);
        cudaFree(D.v);
        for (auto &E : D.ph) {
            cudaFree(E.off);
            cudaFree(E.g);
            cudaFree(E.o);
            cudaFree(E.tk);
            cudaFree(E.medium);
            cudaFree(E.heavy);
        }
    }
    cudaFree(c->input);
    cudaFree(c->staging);
    cudaFree(c->err);
    cudaFree(c->work);
    cudaFree(c->edge_stats);
    cudaSetDevice(cur);
    delete c;
    return VG_OK;
}

static int grow_dev(vg_ctx *c, void **p, size_t *cap, size_t bytes)
{
    if (bytes <= *cap) return VG_OK;
    vg_release(c, *p);
    *p = nullptr;
    *cap = 0;
    VG_TRY(vg_alloc(c, p, bytes));
    *cap = bytes;
    return VG_OK;
}

// log2 of the layer width the reader gives n gates (zk_verifier.cpp:129-169)
static int width_log(long n)
{
    int bl = 0;
    while ((1L << bl) < n) ++bl;
    return n == 1 ? 1 : bl;
}

extern "C" int vg_circuit_build(vg_ctx *ctx, int d, const long *n, const uint8_t *const *ty, const void *const *u,
                                const void *const *v, int index_bytes, vg_circuit **inout, int *bit_lengths)
{
    if (!ctx || d < 1 || !n || !ty || !u || !v || !inout || (index_bytes != 4 && index_bytes != 8))
        return vg_fail(VG_ERR_ARG, "vg_circuit_build: bad argument");
    for (int i = 0; i < d; ++i)
        if (n[i] < 1 || n[i] > (1L << 30)) return vg_fail(VG_ERR_ARG, "layer %d: %ld gates", i, n[i]);
    // prover layers: 0 input values, 1 relay, 1 + i for file layer i >= 1
    const int depth = d + 1;
    std::vector<int> bl(depth);
    const long pad = 1L << (d > 3 ? 17 : 15);   // zk_verifier.cpp:32-41
    bl[0] = bl[1] = width_log(std::max(n[0], pad));
    for (int i = 1; i < d; ++i) bl[i + 1] = width_log(n[i]);
    vg_circuit *c = *inout;
    if (!c) {
        c = new vg_circuit();
        c->ctx = ctx;
    }
    c->ctx = ctx;
    c->device = ctx->device;
    c->depth = depth;
    c->max_bl = 0;
    // layer slots only grow: a shallower circuit leaves the deeper slots'
    // buffers allocated for the next deep one (dropping them would leak them)
    if ((int)c->L.size() < depth) {
        c->L.resize(depth);
        c->cap.resize(depth, 0);
    }
    auto fail = [&](int rc) {
        if (!*inout) vg_circuit_destroy(c);
        return rc;
    };
    if (!c->err && cudaMalloc(&c->err, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        return fail(vg_fail(VG_ERR_OOM, "circuit error flag"));
    }
    VG_CHECK_CUDA(cudaMemsetAsync(c->err, 0xff, sizeof(unsigned long long), ctx->stream));
    for (int i = 0; i < depth; ++i) {
        DevLayer &D = c->L[i];
        D.bl = bl[i];
        D.n = 1L << bl[i];
        c->max_bl = std::max(c->max_bl, D.bl);
        if (i == 0) {
            size_t capb = c->input_cap * sizeof(fe);
            int rc = grow_dev(ctx, (void **)&c->input, &capb, D.n * sizeof(fe));
            if (rc != VG_OK) return fail(rc);
            c->input_cap = (long)(capb / sizeof(fe));
            continue;
        }
        if (c->cap[i] < D.n) {
            vg_release(ctx, D.ty);
            vg_release(ctx, D.u);
            vg_release(ctx, D.v);
            D.ty = nullptr;
            D.u = D.v = nullptr;
            c->cap[i] = 0;
            int rc = vg_alloc(ctx, (void **)&D.ty, D.n);
            if (rc == VG_OK) rc = vg_alloc(ctx, (void **)&D.u, D.n * 4);
            if (rc == VG_OK) rc = vg_alloc(ctx, (void **)&D.v, D.n * 4);
            if (rc != VG_OK) return fail(rc);
            c->cap[i] = D.n;
        }
    }
    // staging for the largest file layer: types, then u and v
    long nmax = 0;
    for (int i = 0; i < d; ++i) nmax = std::max(nmax, n[i]);
    const size_t stage_b = ((size_t)nmax + 255) / 256 * 256 + 2 * (size_t)nmax * 8;
    int rc = grow_dev(ctx, &c->staging, &c->staging_cap, stage_b);
    if (rc != VG_OK) return fail(rc);
    const unsigned grid_cap = 148u * 32u;
    for (int fi = 0; fi < d; ++fi) {
        const long cnt = n[fi];
        const size_t wb = fi == 0 ? 8 : (size_t)index_bytes;   // the input layer's u are values (int64)
        uint8_t *sty = (uint8_t *)c->staging;
        char *su = (char *)c->staging + ((size_t)nmax + 255) / 256 * 256;
        char *sv = su + (size_t)nmax * 8;
        VG_TRY(vg_h2d_staged(ctx, sty, ty[fi], cnt));
        VG_TRY(vg_h2d_staged(ctx, su, u[fi], cnt * wb));
        if (fi > 0) VG_TRY(vg_h2d_staged(ctx, sv, v[fi], cnt * wb));
        if (fi == 0) {
            const long width = c->L[0].n;
            k_build_input<<<std::min<unsigned>(grid_for(width, 256), grid_cap), 256, 0, ctx->stream>>>(
                sty, (const int64_t *)su, cnt, width, c->input, c->err);
            VG_LAUNCHED(ctx);
            DevLayer &R = c->L[1];
            k_build_relay<<<std::min<unsigned>(grid_for(R.n, 256), grid_cap), 256, 0, ctx->stream>>>(
                std::max(cnt, pad), R.n, R.ty, R.u, R.v);
            VG_LAUNCHED(ctx);
        } else {
            const int li = fi + 1;
            DevLayer &D = c->L[li];
            const long prev = c->L[li - 1].n;
            const unsigned grid = std::min<unsigned>(grid_for(D.n, 256), grid_cap);
            if (index_bytes == 8)
                k_build_layer<int64_t><<<grid, 256, 0, ctx->stream>>>(sty, (const int64_t *)su, (const int64_t *)sv, cnt, D.n,
                                                                      prev, li, D.ty, D.u, D.v, c->err);
            else
                k_build_layer<uint32_t><<<grid, 256, 0, ctx->stream>>>(sty, (const uint32_t *)su, (const uint32_t *)sv, cnt,
                                                                       D.n, prev, li, D.ty, D.u, D.v, c->err);
            VG_LAUNCHED(ctx);
        }
    }
    // edge sets from the checked wires (invalid gates became dummies), then one
    // synchronisation for the error flag and the edge counts
    rc = launch_all_edges(c);
    if (rc != VG_OK) return fail(rc);
    unsigned long long e = 0;
    VG_CHECK_CUDA(cudaMemcpyAsync(&e, c->err, sizeof e, cudaMemcpyDeviceToHost, ctx->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    if (e != ~0ull) {
        const int li = (int)(e >> 40);
        const long gi = (long)(e & ((1ull << 40) - 1));
        return fail(vg_fail(VG_ERR_ARG, "file layer %d gate %ld: invalid type or wire", li == 0 ? 0 : li - 1, gi));
    }
    rc = finish_edges(c, c->edge_stats_host.data());
    if (rc != VG_OK) return fail(rc);
    if (bit_lengths)
        for (int i = 0; i < depth; ++i) bit_lengths[i] = bl[i];
    *inout = c;
    return VG_OK;
}

extern "C" int vg_circuit_depth(const vg_circuit *c, int *depth)
{
    if (!c || !depth) return vg_fail(VG_ERR_ARG, "null argument");
    *depth = c->depth;
    return VG_OK;
}

// ---------------------------------------------------------------------- GKR
// Points g at circuit c, reusing every buffer that is large enough (a server
// proving circuits of changing shapes then allocates only when one grows,
// and cudaFree's device-wide synchronisation stays out of the proofs).
static int gkr_bind(vg_gkr *g, const vg_circuit *c)
{
    auto oom = [&](const char *what) {
        cudaGetLastError();
        return vg_fail(VG_ERR_OOM, "vg_gkr: %s allocation failed", what);
    };
    long total = 0;
    for (int i = 1; i < c->depth; ++i) total += c->L[i].n;
    vg_ctx *x = g->ctx;
    if (total > g->vals_cap) {
        vg_release(x, g->vals_slab);
        g->vals_slab = nullptr;
        g->vals_cap = 0;
        if (vg_alloc(x, (void **)&g->vals_slab, total * sizeof(fe)) != VG_OK) return oom("layer values");
        g->vals_cap = total;
    }
    g->vals.assign(c->depth, nullptr);
    g->vals[0] = c->input;
    long off = 0;
    for (int i = 1; i < c->depth; ++i) {
        g->vals[i] = g->vals_slab + off;
        off += c->L[i].n;
    }
    const long N = 1L << c->max_bl;
    if (N > g->N_cap) {
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 3; ++k) {
                vg_release(x, g->buf[b][k]);
                g->buf[b][k] = nullptr;
            }
        vg_release(x, g->eq);
        vg_release(x, g->rg_parts);
        vg_release(x, g->bgt);
        g->eq = g->rg_parts = g->bgt = nullptr;
        g->N_cap = 0;
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 3; ++k)
                if (vg_alloc(x, (void **)&g->buf[b][k], (b == 0 ? N : N / 2 + 1) * sizeof(fe)) != VG_OK) return oom("tables");
        if (vg_alloc(x, (void **)&g->eq, 6 * (1L << (c->max_bl / 2 + 1)) * sizeof(fe)) != VG_OK) return oom("eq tables");
        if (vg_alloc(x, (void **)&g->rg_parts, rg_parts_len(N) * sizeof(fe)) != VG_OK)
            return oom("group partials");
        if (vg_alloc(x, (void **)&g->bgt, N * sizeof(fe)) != VG_OK) return oom("beta_g table");
        g->N_cap = N;
    }
    g->C = c;
    g->bgt_layer = -1;
    g->held = false;
    g->eq_half = 1L << (c->max_bl / 2 + 1);
    g->layer = -1;
    g->n = 0;
    g->round0_pending = false;
    g->pend_r.clear();
    return VG_OK;
}

// the 2 x 4 x N accumulators of the atomic scatter path, on first use
static int ensure_acc(vg_gkr *g, long N)
{
    if (N <= g->acc_cap) return VG_OK;
    vg_release(g->ctx, g->acc);
    g->acc = nullptr;
    g->acc_cap = 0;
    VG_TRY(vg_alloc(g->ctx, (void **)&g->acc, 2 * 4 * N * sizeof(unsigned long long)));
    g->acc_cap = N;
    return VG_OK;
}

extern "C" int vg_gkr_create(vg_ctx *ctx, const vg_circuit *c, vg_gkr **out)
{
    if (!ctx || !c || !out) return vg_fail(VG_ERR_ARG, "vg_gkr_create: null argument");
    vg_gkr *g = new vg_gkr();
    g->ctx = ctx;
    auto fail = [&](const char *what) {
        cudaGetLastError();
        vg_gkr_destroy(g);
        return vg_fail(VG_ERR_OOM, "vg_gkr_create: %s allocation failed", what);
    };
    if (cudaMalloc(&g->rbuf, 3 * 64 * sizeof(fe)) != cudaSuccess) return fail("challenges");
    if (cudaMalloc(&g->round_parts, 6 * 148 * 8 * sizeof(fe)) != cudaSuccess) return fail("round partials");
    if (cudaMalloc(&g->round_out, 16 * sizeof(fe)) != cudaSuccess) return fail("round sums");
    if (cudaMalloc(&g->round_counter, sizeof(unsigned)) != cudaSuccess) return fail("round counter");
    if (cudaMalloc(&g->vu, sizeof(fe)) != cudaSuccess) return fail("v_u");
    if (cudaMalloc(&g->rsync_dev, sizeof(fe)) != cudaSuccess) return fail("round challenge");
    if (cudaMallocHost(&g->rsync_host, sizeof(fe)) != cudaSuccess) return fail("round challenge (pinned)");
    if (cudaMalloc(&g->heavy_parts, (size_t)MAX_HEAVY * HEAVY_PARTS * 4 * sizeof(fe)) != cudaSuccess)
        return fail("heavy partials");
    // on the context's stream: the streams are non-blocking, so a memset on
    // the legacy stream would not be ordered before the first round kernel
    if (cudaMemsetAsync(g->round_counter, 0, sizeof(unsigned), ctx->stream) != cudaSuccess) return fail("round counter");
    int rc = gkr_bind(g, c);
    if (rc != VG_OK) {
        vg_gkr_destroy(g);
        return rc;
    }
    *out = g;
    return VG_OK;
}

extern "C" int vg_gkr_rebind(vg_gkr *g, const vg_circuit *c)
{
    if (!g || !c) return vg_fail(VG_ERR_ARG, "vg_gkr_rebind: null argument");
    VG_TRY(flush_rounds(g));
    return gkr_bind(g, c);
}

extern "C" int vg_gkr_destroy(vg_gkr *g)
{
    if (!g) return VG_OK;
    cudaStreamSynchronize(g->ctx->stream);
    cudaFree(g->vals_slab);
    for (int b = 0; b < 2; ++b)
        for (int k = 0; k < 3; ++k) cudaFree(g->buf[b][k]);
    cudaFree(g->acc);
    cudaFree(g->eq);
    cudaFree(g->rbuf);
    cudaFree(g->round_parts);
    cudaFree(g->round_out);
    cudaFree(g->round_counter);
    cudaFree(g->vu);
    cudaFree(g->heavy_parts);
    cudaFree(g->rg_parts);
    cudaFree(g->bgt);
    cudaFree(g->rec);
    if (g->rec_host) cudaFreeHost(g->rec_host);
    destroy_graphs(g);
    cudaFree(g->rdev);
    if (g->rhost) cudaFreeHost(g->rhost);
    cudaFree(g->rsync_dev);
    if (g->rsync_host) cudaFreeHost(g->rsync_host);
    delete g;
    return VG_OK;
}

extern "C" int vg_gkr_evaluate(vg_gkr *g)
{
    if (!g) return vg_fail(VG_ERR_ARG, "null gkr");
    VG_TRY(flush_rounds(g));
    vg_ctx *c = g->ctx;
    for (int i = 1; i < g->C->depth; ++i) {
        const DevLayer &D = g->C->L[i];
        unsigned grid = std::min<unsigned>(grid_for(D.n, GKR_THREADS), 148u * 64u);
        {
            ProfScope ps(c, KF_EVAL, 57.0 * (double)D.n);   // gate record, two operands, one result
            k_eval_layer<<<grid, GKR_THREADS, 0, c->stream>>>(D.ty, D.u, D.v, D.n, g->vals[i - 1], g->vals[i]);
        }
        VG_LAUNCHED(c);
    }
    if (!g->deferred) VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return VG_OK;
}

int vg_gkr_set_input(vg_gkr *g, const vg_fe *input)
{
    if (!g || !g->C || g->vals.empty()) return vg_fail(VG_ERR_STATE, "vg_gkr_set_input: no circuit bound");
    g->vals[0] = input ? (fe *)input : g->C->input;
    return VG_OK;
}

// layer-0 values from input-gate u values: read through int32 as the
// circuit build does (zk_prover.cpp:60-65), zero from n up to width
__global__ void k_input_values(const int64_t *__restrict__ u, long n, long width, fe *__restrict__ out)
{
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < width; g += (long)gridDim.x * blockDim.x)
        out[g] = g < n ? from_int32((int32_t)u[g]) : vg::fe_zero();
}

int vg_input_values(vg_ctx *c, const int64_t *dev_u, long n, long width, vg_fe *out)
{
    if (!c || !dev_u || !out || n < 1 || n > width) return vg_fail(VG_ERR_ARG, "vg_input_values: bad argument");
    k_input_values<<<std::min<unsigned>(grid_for(width, 256), 148u * 16u), 256, 0, c->stream>>>(dev_u, n, width,
                                                                                            (fe *)out);
    VG_LAUNCHED(c);
    return VG_OK;
}

extern "C" int vg_gkr_layer_values(vg_gkr *g, int layer, const vg_fe **dev_values)
{
    if (!g || !dev_values || layer < 0 || layer >= g->C->depth) return vg_fail(VG_ERR_ARG, "vg_gkr_layer_values: bad layer");
    *dev_values = (const vg_fe *)g->vals[layer];
    return VG_OK;
}

// eq half tables for bits r[0..len): low half (len >> 1 bits, scaled) and high half
// Adds the low half (len >> 1 bits, scaled) and the high half of the eq table
// of r to J; *fh = the low half's bit count.
static void add_halves(EqJobs &J, const fe *r_dev, int len, fe scale, fe *lo, fe *hi, int *fh)
{
    const int f = len >> 1, s = len - f;
    const int bits[2] = {f, s};
    const fe *rs[2] = {r_dev, r_dev + f};
    fe *outs[2] = {lo, hi};
    for (int k = 0; k < 2; ++k) {
        const int q = J.count++;
        J.r[q] = rs[k];
        J.out[q] = outs[k];
        J.scale[q] = k == 0 ? scale : vg::fe_one();
        J.nbits[q] = bits[k];
        J.begin[q + 1] = J.begin[q] + (1L << bits[k]);
    }
    *fh = f;
}

static int launch_halves(vg_gkr *g, const EqJobs &J)
{
    k_eq_halves<<<grid_for(J.begin[J.count], 256), 256, 0, g->ctx->stream>>>(J);
    VG_LAUNCHED(g->ctx);
    return VG_OK;
}

static int build_halves(vg_gkr *g, const fe *r_dev, int len, fe scale, fe *lo, fe *hi, int *fh)
{
    EqJobs J{};
    add_halves(J, r_dev, len, scale, lo, hi, fh);
    return launch_halves(g, J);
}

static int upload_r(vg_gkr *g, int slot, const vg_fe *r, int len)
{
    if (len > 64) return vg_fail(VG_ERR_ARG, "challenge vector longer than 64");
    if (len == 0) return VG_OK;
    VG_CHECK_CUDA(cudaMemcpyAsync(g->rbuf + 64 * slot, r, len * sizeof(fe), cudaMemcpyHostToDevice, g->ctx->stream));
    return VG_OK;
}

extern "C" int vg_gkr_v_res(vg_gkr *g, const vg_fe *r, int r_len, vg_fe *out)
{
    if (!g || !r || !out) return vg_fail(VG_ERR_ARG, "vg_gkr_v_res: null argument");
    const int last = g->C->depth - 1;
    if (r_len != g->C->L[last].bl) return vg_fail(VG_ERR_ARG, "r_len %d != output bit length %d", r_len, g->C->L[last].bl);
    vg_ctx *c = g->ctx;
    VG_TRY(flush_rounds(g));
    VG_TRY(upload_r(g, 0, r, r_len));
    fe *lo = g->eq, *hi = g->eq + g->eq_half;
    int fh;
    VG_TRY(build_halves(g, g->rbuf, r_len, vg::fe_one(), lo, hi, &fh));
    fe *parts;
    const int nb = 148 * 2;
    VG_TRY(vg_partials(c, nb + 1, &parts));
    const long n = 1L << r_len;
    k_eq_dot<<<nb, 256, 0, c->stream>>>(g->vals[last], lo, hi, fh, n, parts);
    VG_LAUNCHED(c);
    if (g->deferred) {
        if (g->rec_n >= g->rec_cap) return vg_fail(VG_ERR_STATE, "deferred record buffer full");
        VG_TRY(vg_reduce_partials(c, parts, nb, 1, g->rec + 9 * g->rec_n++));
        return VG_OK;
    }
    VG_TRY(vg_reduce_partials(c, parts, nb, 1, parts + nb));
    VG_CHECK_CUDA(cudaMemcpyAsync(out, parts + nb, sizeof(fe), cudaMemcpyDeviceToHost, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return VG_OK;
}

extern "C" int vg_mle_eval(vg_ctx *c, const vg_fe *vals, long n, const vg_fe *r, int log_n, vg_fe *out)
{
    if (!c || !vals || !r || !out || log_n < 0 || log_n > 30 || n < (1L << log_n))
        return vg_fail(VG_ERR_ARG, "vg_mle_eval: bad argument (n=%ld log_n=%d)", n, log_n);
    const long m = 1L << log_n;
    int f = log_n >> 1, s = log_n - f;
    fe *tmp;
    VG_CHECK_CUDA(cudaMalloc(&tmp, ((1L << f) + (1L << s) + 64 + (vg_is_device_ptr(vals) ? 0 : m)) * sizeof(fe)));
    fe *lo = tmp, *hi = tmp + (1L << f), *rd = hi + (1L << s);
    const fe *v = (const fe *)vals;
    if (!vg_is_device_ptr(vals)) {
        fe *vd = rd + 64;
        cudaMemcpyAsync(vd, vals, m * sizeof(fe), cudaMemcpyHostToDevice, c->stream);
        v = vd;
    }
    if (log_n) cudaMemcpyAsync(rd, r, log_n * sizeof(fe), cudaMemcpyHostToDevice, c->stream);
    k_eq_half<<<grid_for(1L << f, 256), 256, 0, c->stream>>>(rd, f, vg::fe_one(), lo);
    c->launches++;
    k_eq_half<<<grid_for(1L << s, 256), 256, 0, c->stream>>>(rd + f, s, vg::fe_one(), hi);
    c->launches++;
    fe *parts;
    const int nb = 148 * 2;
    int rc = vg_partials(c, nb + 1, &parts);
    if (rc != VG_OK) {
        cudaFree(tmp);
        return rc;
    }
    k_eq_dot<<<nb, 256, 0, c->stream>>>(v, lo, hi, f, m, parts);
    c->launches++;
    rc = vg_reduce_partials(c, parts, nb, 1, parts + nb);
    if (rc == VG_OK) {
        cudaMemcpyAsync(out, parts + nb, sizeof(fe), cudaMemcpyDeviceToHost, c->stream);
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) rc = vg_fail(VG_ERR_CUDA, "vg_mle_eval: %s", cudaGetErrorString(e));
    }
    cudaFree(tmp);
    return rc;
}

static int eq_table(vg_ctx *c, const vg_fe *r, int log_len, vg_fe *pub)
{
    if (!c || !r || !pub || log_len < 1 || log_len > 30) return vg_fail(VG_ERR_ARG, "vg_eq_table: bad argument");
    fe *tmp;
    int f = log_len >> 1, s = log_len - f;
    VG_TRY(vg_scratch2(c, ((1L << f) + (1L << s) + 64) * sizeof(fe), (void **)&tmp));
    fe *lo = tmp, *hi = tmp + (1L << f), *rd = hi + (1L << s);
    VG_CHECK_CUDA(cudaMemcpyAsync(rd, r, log_len * sizeof(fe), cudaMemcpyHostToDevice, c->stream));   // staged copy
    k_eq_half<<<grid_for(1L << f, 256), 256, 0, c->stream>>>(rd, f, vg::fe_one(), lo);
    c->launches++;
    k_eq_half<<<grid_for(1L << s, 256), 256, 0, c->stream>>>(rd + f, s, vg::fe_one(), hi);
    c->launches++;
    long n = 1L << log_len;
    k_eq_combine<<<std::min<unsigned>(grid_for(n, 256), 148u * 32u), 256, 0, c->stream>>>(lo, hi, f, n, (fe *)pub);
    VG_LAUNCHED(c);
    return VG_OK;
}

extern "C" int vg_eq_table(vg_ctx *c, const vg_fe *r, int log_len, vg_fe *pub)
{
    VG_TRY(eq_table(c, r, log_len, pub));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return VG_OK;
}

int vg_eq_table_async(vg_ctx *c, const vg_fe *r, int log_len, vg_fe *pub) { return eq_table(c, r, log_len, pub); }

extern "C" int vg_circuit_predicates(vg_ctx *c, const vg_circuit *C, int layer, const vg_fe *r_0, const vg_fe *r_1,
                                     const vg_fe *r_u, const vg_fe *r_v, vg_fe alpha, vg_fe beta, vg_fe *out)
{
    if (!c || !C || !r_0 || !r_1 || !r_u || !r_v || !out) return vg_fail(VG_ERR_ARG, "vg_circuit_predicates: null argument");
    if (layer < 1 || layer >= C->depth) return vg_fail(VG_ERR_ARG, "vg_circuit_predicates: layer %d out of range", layer);
    if (layer == 1) {   // the reader's relay layer: the reference returns zeros (zk_verifier.cpp:231-234)
        for (int t = 0; t < 14; ++t) out[t] = vg_fe{0, 0};
        return VG_OK;
    }
    const DevLayer &D = C->L[layer];
    const int lg = D.bl, luv = C->L[layer - 1].bl;   // at most 30 (checked at upload)
    const int fg = lg >> 1, sg = lg - fg, fuv = luv >> 1, suv = luv - fuv;
    const long hg = 1L << std::max(fg, sg), huv = 1L << std::max(fuv, suv);
    const int nb = 148 * 4;
    // scratch: r values, 4 g halves, 4 u/v halves, partials, result
    const size_t n_fe = 4 * 64 + 4 * hg + 4 * huv + (size_t)nb * 14 + 16;
    fe *w;
    VG_TRY(vg_scratch(c, n_fe * sizeof(fe), (void **)&w));
    fe *rr = w, *tg = rr + 4 * 64, *tuv = tg + 4 * hg, *parts = tuv + 4 * huv, *res = parts + (size_t)nb * 14;
    VG_CHECK_CUDA(cudaMemcpyAsync(rr, r_0, lg * sizeof(fe), cudaMemcpyHostToDevice, c->stream));
    VG_CHECK_CUDA(cudaMemcpyAsync(rr + 64, r_1, lg * sizeof(fe), cudaMemcpyHostToDevice, c->stream));
    VG_CHECK_CUDA(cudaMemcpyAsync(rr + 128, r_u, luv * sizeof(fe), cudaMemcpyHostToDevice, c->stream));
    VG_CHECK_CUDA(cudaMemcpyAsync(rr + 192, r_v, luv * sizeof(fe), cudaMemcpyHostToDevice, c->stream));
    int fh;
    EqJobs J1{}, J2{};
    add_halves(J1, rr, lg, tofe(alpha), tg, tg + hg, &fh);
    add_halves(J1, rr + 64, lg, tofe(beta), tg + 2 * hg, tg + 3 * hg, &fh);
    add_halves(J2, rr + 128, luv, vg::fe_one(), tuv, tuv + huv, &fh);
    add_halves(J2, rr + 192, luv, vg::fe_one(), tuv + 2 * huv, tuv + 3 * huv, &fh);
    for (const EqJobs *J : {&J1, &J2}) {
        k_eq_halves<<<grid_for(J->begin[J->count], 256), 256, 0, c->stream>>>(*J);
        VG_LAUNCHED(c);
    }
    BetaG bg{tg, tg + hg, tg + 2 * hg, tg + 3 * hg, fg, (1L << fg) - 1};
    BetaU bu{tuv, tuv + huv, fuv, (1L << fuv) - 1};
    BetaU bv{tuv + 2 * huv, tuv + 3 * huv, fuv, (1L << fuv) - 1};
    k_predicates<<<nb, PRED_THREADS, 0, c->stream>>>(D.ty, D.u, D.v, D.n, bg, bu, bv, (uint32_t)((1L << luv) - 1), parts);
    VG_LAUNCHED(c);
    VG_TRY(vg_reduce_partials(c, parts, nb, 14, res));
    k_predicates_relay<<<1, 1, 0, c->stream>>>(res, tuv + 2 * huv, tuv + 3 * huv);
    VG_LAUNCHED(c);
    fe host[14];
    VG_CHECK_CUDA(cudaMemcpyAsync(host, res, 14 * sizeof(fe), cudaMemcpyDeviceToHost, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    for (int t = 0; t < 14; ++t) out[t] = tovg(host[t]);
    return VG_OK;
}

// the phase's tables (add_mult_sum in buf[0][2], addV_array in buf[0][1]) are
// in place: the rounds start from them
static int tables_ready(vg_gkr *g, long N)
{
    g->n = N;
    g->cur[1] = g->buf[0][1];
    g->cur[2] = g->buf[0][2];
    g->next_buf = 1;
    g->round0_pending = true;
    return VG_OK;
}

static bool fuse_gather(vg_gkr *g, long N);

// The pending table build (gather_tables) as a plain k_gather_keys launch,
// for a launch that reads the tables whole.
static int gather_now(vg_gkr *g)
{
    if (!g->gather_pending) return VG_OK;
    g->gather_pending = false;
    vg_ctx *c = g->ctx;
    const GatherArgs &a = g->gather;
    const long N = g->gather_n;
    const unsigned grid = std::min<unsigned>(grid_for(N, GKR_THREADS), 148u * 64u);
    {
        ProfScope ps(c, g->gather_ph == 0 ? KF_SCATTER1 : KF_SCATTER2, g->gather_bytes + 32.0 * (double)N);
        if (g->gather_ph == 0)
            k_gather_keys<0><<<grid, GKR_THREADS, 0, c->stream>>>(a.e, N, a.bg, a.bu, a.prev, a.vu, a.tm, a.tv);
        else
            k_gather_keys<1><<<grid, GKR_THREADS, 0, c->stream>>>(a.e, N, a.bg, a.bu, a.prev, a.vu, a.tm, a.tv);
    }
    VG_LAUNCHED(c);
    return VG_OK;
}

// phase tables by gathering over the layer's edge set (no atomics, no
// finalize).  The keys with more than LIGHT_MAX edges are summed now; the
// others by k_gather_keys now, or, when the phase's first two rounds will
// run as one pass (fuse_gather), inside that pass (k_gather_round2).
template <int PH>
static int gather_tables(vg_gkr *g, const EdgeSet &E, long N, const fe *prev, const BetaG &bg)
{
    vg_ctx *c = g->ctx;
    const EdgeView ev{E.off, E.g, E.o, E.tk};
    fe *out_m = g->buf[0][2], *out_v = g->buf[0][1];
    VG_TRY(gather_now(g));
    g->gather_pending = true;
    g->gather_ph = PH;
    g->gather_n = N;
    g->gather_bytes = 10.0 * (double)E.E + 4.0 * (double)N;   // edge records and key offsets
    g->gather = GatherArgs{ev, bg, g->bu, prev, g->vu, out_m, out_v};
    if (!fuse_gather(g, N)) VG_TRY(gather_now(g));
    const int nheavy = (int)(E.heavy_host.size() / 3);
    for (int h0 = 0; h0 < nheavy; h0 += MAX_HEAVY) {   // heavy keys, split over many CTAs
        HeavyKeys H{};
        for (int q = h0; q < nheavy && H.count < MAX_HEAVY; ++q) {
            H.key[H.count] = E.heavy_host[3 * q];
            H.s[H.count] = E.heavy_host[3 * q + 1];
            H.e[H.count] = E.heavy_host[3 * q + 2];
            ++H.count;
        }
        const int nparts = HEAVY_PARTS;
        ProfScope ps(c, PH == 0 ? KF_SCATTER1 : KF_SCATTER2, 0.0);
        k_gather_heavy<PH><<<dim3(nparts, H.count), GKR_THREADS, 0, c->stream>>>(ev, H, bg, g->bu, prev, g->heavy_parts);
        VG_LAUNCHED(c);
        k_heavy_finish<PH><<<H.count, GKR_THREADS, 0, c->stream>>>(H, g->heavy_parts, nparts, g->vu, out_m, out_v);
        VG_LAUNCHED(c);
    }
    if (E.n_medium) {
        ProfScope ps(c, PH == 0 ? KF_SCATTER1 : KF_SCATTER2, 0.0);
        k_gather_long<PH><<<std::min<unsigned>(grid_for(E.n_medium * 32, GKR_THREADS), 148u * 64u), GKR_THREADS, 0,
                            c->stream>>>(ev, E.medium, E.n_medium, bg, g->bu, prev, g->vu, out_m, out_v);
        VG_LAUNCHED(c);
    }
    return VG_OK;
}

static int finalize_tables(vg_gkr *g, long N)
{
    vg_ctx *c = g->ctx;
    const long maxN = 1L << g->C->max_bl;
    unsigned grid = std::min<unsigned>(grid_for(N, 256), 148u * 32u);
    {
        ProfScope ps(c, KF_FINALIZE, 48.0 * (double)N);
        k_acc_finalize<<<grid, 256, 0, c->stream>>>(g->acc, N, g->buf[0][2]);   // add_mult_sum
    }
    VG_LAUNCHED(c);
    {
        ProfScope ps(c, KF_FINALIZE, 48.0 * (double)N);
        k_acc_finalize<<<grid, 256, 0, c->stream>>>(g->acc + 4 * maxN, N, g->buf[0][1]);   // addV_array
    }
    VG_LAUNCHED(c);
    return tables_ready(g, N);
}

extern "C" int vg_gkr_phase1_init(vg_gkr *g, int layer, const vg_fe *r0, const vg_fe *r1, int length_g, vg_fe alpha,
                                  vg_fe beta)
{
    if (!g || !r0 || !r1) return vg_fail(VG_ERR_ARG, "vg_gkr_phase1_init: null argument");
    VG_TRY(flush_rounds(g));
    if (layer < 1 || layer >= g->C->depth) return vg_fail(VG_ERR_ARG, "layer %d out of range", layer);
    if (length_g != g->C->L[layer].bl) return vg_fail(VG_ERR_ARG, "length_g %d != layer bit length %d", length_g, g->C->L[layer].bl);
    vg_ctx *c = g->ctx;
    const DevLayer &D = g->C->L[layer];
    const long N = g->C->L[layer - 1].n, maxN = 1L << g->C->max_bl;
    g->layer = layer;
    g->length_g = length_g;
    VG_TRY(upload_r(g, 0, r0, length_g));
    VG_TRY(upload_r(g, 1, r1, length_g));
    fe *e = g->eq;
    const long H = g->eq_half;
    int fh;
    {   // the alpha- and beta-weighted tables of r0 and r1 in one launch
        EqJobs J{};
        add_halves(J, g->rbuf, length_g, tofe(alpha), e, e + H, &fh);
        add_halves(J, g->rbuf + 64, length_g, tofe(beta), e + 2 * H, e + 3 * H, &fh);
        VG_TRY(launch_halves(g, J));
    }
    g->bg.f0 = e;
    g->bg.s0 = e + H;
    g->bg.f1 = e + 2 * H;
    g->bg.s1 = e + 3 * H;
    g->bg.fh = fh;
    g->bg.mask = (1L << fh) - 1;
    g->bg.save = nullptr;
    g->bg.tab = nullptr;
    g->bgt_layer = -1;
    if (D.ph[0].ok) {
        // the gathers store every gate's beta_g for phase 2 (a gate with a
        // phase-2 edge has a phase-1 edge: both need its u); every store of
        // entry x holds beta_g(x), whichever edge made it
        const bool table = vg_tune_value(c->device, VG_TUNE_BETA_TABLE) != 0;
        BetaG b1 = g->bg;
        b1.save = table ? g->bgt : nullptr;
        VG_TRY(gather_tables<0>(g, D.ph[0], N, g->vals[layer - 1], b1));
        g->bgt_layer = table ? layer : -1;
        g->cur[0] = g->vals[layer - 1];
        return tables_ready(g, N);
    }
    VG_TRY(ensure_acc(g, maxN));
    VG_CHECK_CUDA(cudaMemsetAsync(g->acc, 0, N * 4 * sizeof(unsigned long long), c->stream));
    VG_CHECK_CUDA(cudaMemsetAsync(g->acc + 4 * maxN, 0, N * 4 * sizeof(unsigned long long), c->stream));
    unsigned grid = std::min<unsigned>(grid_for(D.n, GKR_THREADS), 148u * 32u);
    {
        // gate record, one operand gather, two 32-byte accumulator updates
        ProfScope ps(c, KF_SCATTER1, 89.0 * (double)D.n);
        k_phase1_scatter<<<grid, GKR_THREADS, 0, c->stream>>>(D.ty, D.u, D.v, D.n, g->bg, g->vals[layer - 1], g->acc,
                                                             g->acc + 4 * maxN);
    }
    VG_LAUNCHED(c);
    g->cur[0] = g->vals[layer - 1];
    return finalize_tables(g, N);
}

// Table length at which a phase's remaining rounds become round groups: the
// device's VG_TUNE_GROUP_START (at least 2 RG_CHUNK).  A group on a longer
// table runs one CTA per chunk of 2 RG_CHUNK entries (RG_CHUNK for a group
// whose first round does not fold), each folding its chunk in shared memory
// for up to 10 rounds; groups follow one another until the phase ends.
static long group_start(int device) { return vg_tune_value(device, VG_TUNE_GROUP_START); }

// Whether a deferred phase's table build of N entries runs inside its first
// paired pass: builds fused (VG_TUNE_GATHER_FUSE = 1), paired rounds
// (VG_TUNE_ROUND_FUSE = 2) and a table above the group start, so that the
// phase's unfolded first round is held and pairs with the second
// (vg_gkr_round).  Should the rounds go otherwise, the first launch that
// reads the tables builds them plainly before it (add_launch).
static bool fuse_gather(vg_gkr *g, long N)
{
    const int d = g->ctx->device;
    const long S = std::max(2L * RG_CHUNK, group_start(d));
    return g->deferred && vg_tune_value(d, VG_TUNE_GATHER_FUSE) != 0 && vg_tune_value(d, VG_TUNE_ROUND_FUSE) >= 2 &&
           N > S && N >= 8;
}

// Rounds the chunks of a group starting at table length n0 with chunks of
// `chunk` can hold (see k_round_group).
static int group_capacity(long n0, bool nofold, long chunk)
{
    const long m0 = nofold ? std::min(n0, chunk) : std::min(n0, 2 * chunk) / 2;
    int k = 0;
    while ((1L << (k + 1)) <= m0) ++k;
    return std::min(k, RG_MAX);
}

// Shape of a group of nsteps rounds from table length n0: the chunks' rounds
// (k1), the last CTA's tail rounds on the entries the chunks leave, and the
// table length at the end.
struct GroupShape {
    long cin = 0, nchunks = 0;
    int k1 = 0, tail = 0;
    long final_n = 0;
};
static GroupShape group_shape(long n0, bool nofold, long chunk, int nsteps)
{
    GroupShape s;
    s.cin = nofold ? std::min(n0, chunk) : std::min(n0, 2 * chunk);
    s.nchunks = n0 / s.cin;
    s.k1 = std::min(nsteps, group_capacity(n0, nofold, chunk));
    const long mfin = (nofold ? s.cin : s.cin / 2) >> (s.k1 - 1);
    s.tail = nsteps - s.k1;
    const long rem = s.nchunks * mfin;   // entries the chunks leave
    s.final_n = s.tail ? (rem / 2) >> (s.tail - 1) : rem;
    return s;
}

// Rounds a whole group launch can hold: the chunks' rounds, then, when the
// chunks leave between 4 and 2 RG_CHUNK entries in all, the rounds the last
// CTA runs on them (a fold-first group of one chunk).
static int group_total_capacity(long n0, bool nofold, long chunk)
{
    const int k1 = group_capacity(n0, nofold, chunk);
    const GroupShape s = group_shape(n0, nofold, chunk, k1);
    if (s.nchunks < 2 || s.final_n < 4 || s.final_n > 2L * RG_CHUNK) return k1;
    return std::min(RG_STEPS, k1 + group_capacity(s.final_n, false, RG_CHUNK));
}

static int rg_smem_attribute(int dev)
{
    static std::mutex mu;
    static std::vector<bool> done;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= (int)done.size()) done.resize(dev + 1, false);
    if (!done[dev]) {
        const int bytes = (int)(RG_SMEM_FE * sizeof(fe));
        VG_CHECK_CUDA(cudaFuncSetAttribute(k_round_group<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        VG_CHECK_CUDA(cudaFuncSetAttribute(k_round_group<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        VG_CHECK_CUDA(cudaFuncSetAttribute(k_round_group<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        VG_CHECK_CUDA(cudaFuncSetAttribute(k_round_group<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        done[dev] = true;
    }
    return VG_OK;
}

// Issues one round launch on the context stream (rp: its challenge(s) in
// device memory).
static int issue_launch(vg_gkr *g, const RoundLaunch &L, const fe *rp)
{
    vg_ctx *c = g->ctx;
    {
        ProfScope ps(c, L.kind == 3 ? KF_GATHER_ROUND : KF_ROUND, L.prof_bytes);
        fe *pr = g->round_parts;
        unsigned *cnt = g->round_counter;
        if (L.kind == 0) {
#define VG_ROUND_LAUNCH(TT, LZ)                                                                                      \
    if (L.fold)                                                                                                       \
        k_round<true, TT, LZ><<<L.grid, TT, 0, c->stream>>>(L.x[0], L.x[1], L.x[2], L.count, rp, L.y[0], L.y[1],     \
                                                            L.y[2], pr, cnt, L.oa, L.ob, L.prev);                     \
    else                                                                                                              \
        k_round<false, TT, LZ><<<L.grid, TT, 0, c->stream>>>(L.x[0], L.x[1], L.x[2], L.count, rp, nullptr, nullptr,  \
                                                             nullptr, pr, cnt, L.oa, L.ob, nullptr)
#define VG_ROUND_LAUNCH_T(LZ)                     \
    if (L.threads == 128) VG_ROUND_LAUNCH(128, LZ); \
    else if (L.threads == 512) VG_ROUND_LAUNCH(512, LZ); \
    else VG_ROUND_LAUNCH(256, LZ)
            if (L.lazy) { VG_ROUND_LAUNCH_T(true); }
            else { VG_ROUND_LAUNCH_T(false); }
#undef VG_ROUND_LAUNCH_T
#undef VG_ROUND_LAUNCH
        } else if (L.kind == 1) {
#define VG_ROUND2_LAUNCH(TT, LZ)                                                                                     \
    if (L.fold)                                                                                                       \
        k_round2<true, TT, LZ><<<L.grid, TT, 0, c->stream>>>(L.x[0], L.x[1], L.x[2], L.count, rp, L.y[0], L.y[1],    \
                                                             L.y[2], pr, cnt, L.oa, L.ob);                            \
    else                                                                                                              \
        k_round2<false, TT, LZ><<<L.grid, TT, 0, c->stream>>>(L.x[0], L.x[1], L.x[2], L.count, rp, L.y[0], L.y[1],   \
                                                              L.y[2], pr, cnt, L.oa, L.ob)
#define VG_ROUND2_LAUNCH_T(LZ)                     \
    if (L.threads == 128) VG_ROUND2_LAUNCH(128, LZ); \
    else if (L.threads == 512) VG_ROUND2_LAUNCH(512, LZ); \
    else VG_ROUND2_LAUNCH(256, LZ)
            if (L.lazy) { VG_ROUND2_LAUNCH_T(true); }
            else { VG_ROUND2_LAUNCH_T(false); }
#undef VG_ROUND2_LAUNCH_T
#undef VG_ROUND2_LAUNCH
        } else if (L.kind == 3) {
#define VG_GR2_LAUNCH(TT, PH)                                                                                       \
    k_gather_round2<PH, TT><<<L.grid, TT, 0, c->stream>>>(L.ga, L.x[0], L.count, rp, L.y[0], L.y[1], L.y[2], pr, cnt, \
                                                          L.oa, L.ob)
#define VG_GR2_LAUNCH_T(PH)                     \
    if (L.threads == 128) VG_GR2_LAUNCH(128, PH); \
    else if (L.threads == 512) VG_GR2_LAUNCH(512, PH); \
    else VG_GR2_LAUNCH(256, PH)
            if (L.ph == 0) { VG_GR2_LAUNCH_T(0); }
            else { VG_GR2_LAUNCH_T(1); }
#undef VG_GR2_LAUNCH_T
#undef VG_GR2_LAUNCH
        } else {
            RoundGroup G = L.G;
            G.r = rp;
#define VG_GROUP_LAUNCH(LZ, SP)                                                                                      \
    k_round_group<LZ, SP><<<L.grid, RG_THREADS, RG_SMEM_FE * sizeof(fe), c->stream>>>(                               \
        L.x[0], L.x[1], L.x[2], L.count, G, L.y[0], L.y[1], L.y[2], g->rg_parts, g->round_counter, g->rec)
            if (L.lazy && G.split3) VG_GROUP_LAUNCH(true, true);
            else if (L.lazy) VG_GROUP_LAUNCH(true, false);
            else if (G.split3) VG_GROUP_LAUNCH(false, true);
            else VG_GROUP_LAUNCH(false, false);
#undef VG_GROUP_LAUNCH
        }
    }
    VG_LAUNCHED(c);
    return VG_OK;
}

// A round launch: issued now on a synchronous object (its challenge staged
// through rsync), queued until the next flush on a deferred one (challenges
// from the record slots).
static int add_launch(vg_gkr *g, RoundLaunch &L, int nslots, fe r_sync)
{
    if (L.kind != 3) VG_TRY(gather_now(g));   // this launch reads the tables whole
    if (!g->deferred) {
        if (!g->rsync_host) return vg_fail(VG_ERR_STATE, "synchronous round on a tables object");
        *g->rsync_host = r_sync;
        VG_CHECK_CUDA(cudaMemcpyAsync(g->rsync_dev, g->rsync_host, sizeof(fe), cudaMemcpyHostToDevice, g->ctx->stream));
        return issue_launch(g, L, g->rsync_dev);
    }
    if (g->pend_launch.empty()) {
        g->pend_lo = L.slot;
        g->pend_hi = L.slot + nslots;
    } else {
        g->pend_lo = std::min(g->pend_lo, L.slot);
        g->pend_hi = std::max(g->pend_hi, L.slot + nslots);
    }
    g->pend_launch.push_back(L);
    return VG_OK;
}

// VIRGO_GRAPHS=0 issues every deferred round launch plainly
static bool rg_graphs_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("VIRGO_GRAPHS");
        on = (e && e[0] == '0') ? 0 : 1;
    }
    return on != 0;
}

static void destroy_graphs(vg_gkr *g)
{
    for (auto &pg : g->graphs)
        if (pg.exec) cudaGraphExecDestroy(pg.exec);
    g->graphs.clear();
    g->seen.clear();
}

// Issues the queued round launches: one H2D copy of the challenge slots they
// read, then the launches.  A sequence seen before (same pointers, sizes,
// shapes and slots: the same phase of the same circuit in a later proof) is
// captured as a graph the second time and replayed from then on; a stream
// already being captured (the fft_gkr side proof's graph) or the per-launch
// profiler gets plain launches.
static int exec_pending(vg_gkr *g)
{
    if (g->pend_launch.empty()) return VG_OK;
    vg_ctx *c = g->ctx;
    const int lo = g->pend_lo, hi = g->pend_hi;
    std::vector<RoundLaunch> launches;
    launches.swap(g->pend_launch);
    auto issue = [&]() -> int {
        if (hi > lo)
            VG_CHECK_CUDA(cudaMemcpyAsync(g->rdev + lo, g->rhost + lo, (size_t)(hi - lo) * sizeof(fe),
                                          cudaMemcpyHostToDevice, c->stream));
        for (const RoundLaunch &L : launches) VG_TRY(issue_launch(g, L, g->rdev + L.slot));
        return VG_OK;
    };
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    VG_CHECK_CUDA(cudaStreamIsCapturing(c->stream, &cs));
    if (!rg_graphs_enabled() || g->graphs_off || c->profiling || cs != cudaStreamCaptureStatusNone) return issue();

    std::vector<uint64_t> key;
    key.reserve(4 + 24 * launches.size());
    key.push_back((uint64_t)(uintptr_t)g->rdev);
    key.push_back((uint64_t)(uintptr_t)g->rhost);
    key.push_back((uint64_t)lo);
    key.push_back((uint64_t)hi);
    for (const RoundLaunch &L : launches) {
        key.push_back((uint64_t)L.kind | ((uint64_t)L.fold << 4) | ((uint64_t)L.lazy << 5) | ((uint64_t)L.threads << 16) |
                      ((uint64_t)L.grid << 32));
        key.push_back((uint64_t)L.count);
        for (int k = 0; k < 3; ++k) key.push_back((uint64_t)(uintptr_t)L.x[k]);
        for (int k = 0; k < 3; ++k) key.push_back((uint64_t)(uintptr_t)L.y[k]);
        key.push_back((uint64_t)L.slot);
        key.push_back((uint64_t)(uintptr_t)L.oa);
        key.push_back((uint64_t)(uintptr_t)L.ob);
        key.push_back((uint64_t)(uintptr_t)L.prev);
        key.push_back(((uint64_t)L.G.chunk_log) | ((uint64_t)L.G.nsteps << 8) | ((uint64_t)L.G.first_nofold << 16) |
                      ((uint64_t)L.G.last6 << 24) | ((uint64_t)L.G.split3 << 32) |
                      ((uint64_t)L.G.tail << 40));
        key.push_back((uint64_t)L.G.slot0);
        if (L.kind == 3) {
            const GatherArgs &a = L.ga;
            const void *ptrs[] = {a.e.off, a.e.g, a.e.o, a.e.tk, a.bg.f0, a.bg.s0, a.bg.f1, a.bg.s1, a.bg.save,
                                  a.bg.tab, a.bu.f, a.bu.s, a.prev, a.vu, a.tm, a.tv};
            for (const void *q : ptrs) key.push_back((uint64_t)(uintptr_t)q);
            key.push_back((uint64_t)(uint32_t)a.bg.fh | ((uint64_t)(uint32_t)a.bu.fh << 16) | ((uint64_t)L.ph << 32));
            key.push_back((uint64_t)a.bg.mask);
            key.push_back((uint64_t)a.bu.mask);
        }
    }
    key.push_back((uint64_t)(uintptr_t)g->round_parts);
    key.push_back((uint64_t)(uintptr_t)g->round_counter);
    key.push_back((uint64_t)(uintptr_t)g->rg_parts);
    key.push_back((uint64_t)(uintptr_t)g->rec);
    uint64_t h = 1469598103934665603ull;   // FNV-1a over the key words
    for (uint64_t w : key) {
        h ^= w;
        h *= 1099511628211ull;
    }
    for (PhaseGraph &pg : g->graphs)
        if (pg.hash == h && pg.key == key) {
            VG_CHECK_CUDA(cudaGraphLaunch(pg.exec, c->stream));
            c->launches += pg.launches;
            ++g->graph_replays;
            return VG_OK;
        }
    if (std::find(g->seen.begin(), g->seen.end(), h) == g->seen.end()) {
        if (g->seen.size() >= 1024) g->seen.clear();
        g->seen.push_back(h);   // first sight: plain launches
        return issue();
    }
    // second sight: capture, instantiate, launch
    if (g->graphs.size() >= 256) destroy_graphs(g);
    const long launches0 = c->launches;
    VG_CHECK_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    const int rc = issue();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (rc == VG_OK && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (rc != VG_OK || e != cudaSuccess) {
        // nothing of the capture ran: issue plainly, and no graphs from now on
        cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        g->graphs_off = true;
        c->launches = launches0;
        return issue();
    }
    PhaseGraph pg;
    pg.key.swap(key);
    pg.hash = h;
    pg.exec = exec;
    pg.launches = c->launches - launches0;
    g->graphs.push_back(std::move(pg));
    ++g->graph_captures;
    VG_CHECK_CUDA(cudaGraphLaunch(exec, c->stream));
    return VG_OK;
}

// One round on the current tables of length n_in (before the round's fold):
// k_round with its sums (and, when one pair remains, the folded pair) at o3
// (and o6); its challenge is record slot `slot`'s (deferred) or r.
static int launch_round(vg_gkr *g, long n_in, bool fold, fe r, int slot, fe *o3, fe *o6)
{
    vg_ctx *c = g->ctx;
    const long n_out = fold ? n_in / 2 : n_in;   // table length the sums are taken over
    const long npairs = n_out / 2;
    // threads per CTA from the device's tuning; the grid covers at most
    // 148 x 2048 threads and at most 148 x 16 CTAs (the partials buffer holds
    // 3 sums for each), looping beyond
    RoundLaunch L;
    L.kind = 0;
    L.fold = fold;
    L.lazy = vg_tune_value(c->device, VG_TUNE_LAZY_FOLD) != 0;
    L.threads = (int)vg_tune_value(c->device, VG_TUNE_ROUND_THREADS);
    L.grid = std::min<unsigned>(grid_for(npairs, L.threads), std::min(148u * 16u, 148u * 2048u / (unsigned)L.threads));
    L.count = npairs;
    for (int k = 0; k < 3; ++k) {
        L.x[k] = g->cur[k];
        L.y[k] = fold ? g->buf[g->next_buf][k] : nullptr;
    }
    L.slot = slot;
    L.oa = o3;
    L.ob = o6;
    // the previous round's sums: its record, or (synchronous object) the sums buffer itself
    L.prev = fold ? (g->deferred ? o3 - 9 : o3) : nullptr;
    L.prof_bytes = (fold ? 288.0 : 96.0) * (double)npairs;   // fold: read 3 tables x 4 entries, write 3 x 2 per pair
    VG_TRY(add_launch(g, L, 1, r));
    if (fold) {
        for (int k = 0; k < 3; ++k) g->cur[k] = L.y[k];
        g->next_buf ^= 1;
    }
    return VG_OK;
}

// Two rounds in one k_round2 pass on the current tables of length n_in: the
// first (record slot `slot`) folds when `fold` (else it is a phase's unfolded
// first round), the second (slot + 1) folds; sums to their records.
static int launch_round2(vg_gkr *g, long n_in, bool fold, int slot)
{
    vg_ctx *c = g->ctx;
    const long nquads = fold ? n_in / 8 : n_in / 4;
    // at most 148 x 2048 threads and 148 x 8 CTAs (6 sums each in the partials buffer)
    // the phase's pending table build runs inside its unfolded first pass
    const bool fused = g->gather_pending && !fold && n_in == g->gather_n;
    RoundLaunch L;
    L.kind = fused ? 3 : 1;
    L.fold = fold;
    L.lazy = !fused && vg_tune_value(c->device, VG_TUNE_LAZY_FOLD) != 0;
    L.threads = (int)vg_tune_value(c->device, VG_TUNE_ROUND_THREADS);
    L.grid = std::min<unsigned>(grid_for(nquads, L.threads), std::min(148u * 8u, 148u * 2048u / (unsigned)L.threads));
    L.count = nquads;
    for (int k = 0; k < 3; ++k) {
        L.x[k] = g->cur[k];
        L.y[k] = g->buf[g->next_buf][k];
    }
    L.slot = slot;
    L.oa = g->rec + 9 * slot;
    L.ob = g->rec + 9 * (slot + 1);
    L.prof_bytes = (fold ? 480.0 : 288.0) * (double)nquads;   // per quad: read 3 x 8 (or 4) entries, write 3 x 2
    if (fused) {
        L.ga = g->gather;
        L.ph = g->gather_ph;
        g->gather_pending = false;
        // the build's edge records and offsets, then per quad: V read (4 entries), 3 x 2 entries written
        L.prof_bytes = g->gather_bytes + 160.0 * (double)nquads;
    }
    VG_TRY(add_launch(g, L, 2, vg::fe_zero()));
    for (int k = 0; k < 3; ++k) g->cur[k] = L.y[k];
    g->next_buf ^= 1;
    return VG_OK;
}

// A held round with no partner (the next round starts a group, or the phase
// ends): it runs alone.
static int flush_held(vg_gkr *g)
{
    if (!g->held) return VG_OK;
    g->held = false;
    fe *o3 = g->rec + 9 * g->held_slot;
    return launch_round(g, g->held_n, g->held_fold, vg::fe_zero(), g->held_slot, o3, o3 + 3);
}

// Queues the pending deferred rounds as one group: one chunk per CTA when
// the table fits the grid, CTAs looping over chunks beyond.
static int group_rounds(vg_gkr *g)
{
    VG_TRY(flush_held(g));
    if (g->pend_r.empty()) return VG_OK;
    vg_ctx *c = g->ctx;
    RoundLaunch L;
    L.kind = 2;
    L.lazy = vg_tune_value(c->device, VG_TUNE_LAZY_FOLD) != 0;
    RoundGroup &G = L.G;
    int cl = 0;
    while ((1L << cl) < g->pend_chunk) ++cl;
    G.chunk_log = cl;
    G.nsteps = (int)g->pend_r.size();
    G.first_nofold = g->pend_nofold ? 1 : 0;
    G.slot0 = g->pend_slot0;
    G.r = nullptr;
    const long n_in = g->pend_n0;
    const GroupShape gs = group_shape(n_in, g->pend_nofold, g->pend_chunk, G.nsteps);
    if (G.nsteps > RG_STEPS || (gs.tail && (gs.nchunks < 2 || gs.final_n < 2)))
        return vg_fail(VG_ERR_STATE, "round group of %d rounds on %ld entries", G.nsteps, n_in);
    G.tail = gs.tail;
    const long nchunks = gs.nchunks;
    // CTAs loop over chunks: at most 3 resident per SM (72 KB of shared memory each)
    L.grid = (unsigned)std::min(nchunks, 148L * 3L);
    G.last6 = (gs.final_n == 2 && (gs.tail || nchunks == 1)) ? 1 : 0;
    G.split3 = vg_tune_value(c->device, VG_TUNE_GROUP_SPLIT) != 0 ? 1 : 0;
    const bool folds = !(G.first_nofold && G.nsteps == 1);
    L.threads = RG_THREADS;
    L.count = n_in;
    for (int k = 0; k < 3; ++k) {
        L.x[k] = g->cur[k];
        L.y[k] = folds ? g->buf[g->next_buf][k] : nullptr;
    }
    L.slot = G.slot0;
    // every round of the group: the first reads 3 tables of n_in, writes nothing more than the chunk tails
    L.prof_bytes = 48.0 * (double)n_in + (folds ? 48.0 * (double)gs.final_n : 0.0);
    VG_TRY(rg_smem_attribute(c->device));   // before any capture
    VG_TRY(add_launch(g, L, G.nsteps, vg::fe_zero()));
    if (folds) {
        for (int k = 0; k < 3; ++k) g->cur[k] = L.y[k];
        g->next_buf ^= 1;
    }
    g->pend_r.clear();
    return VG_OK;
}

// Every queued round: held and grouped rounds into launches, then issued.
static int flush_rounds(vg_gkr *g)
{
    VG_TRY(group_rounds(g));
    VG_TRY(gather_now(g));   // a build no round took in
    return exec_pending(g);
}

// phase-2 tables for the current layer once g->vu holds v_u
static int phase2_tables(vg_gkr *g, const vg_fe *r_u, int length_u)
{
    const int layer = g->layer;
    vg_ctx *c = g->ctx;
    const DevLayer &D = g->C->L[layer];
    const long N = g->C->L[layer - 1].n, maxN = 1L << g->C->max_bl;
    VG_TRY(upload_r(g, 2, r_u, length_u));
    fe *e = g->eq + 4 * g->eq_half;
    int fh;
    VG_TRY(build_halves(g, g->rbuf + 128, length_u, vg::fe_one(), e, e + g->eq_half, &fh));
    BetaU bu;
    bu.f = e;
    bu.s = e + g->eq_half;
    bu.fh = fh;
    bu.mask = (1L << fh) - 1;
    g->bu = bu;
    if (D.ph[1].ok) {
        BetaG b2 = g->bg;
        if (g->bgt_layer == layer) b2.tab = g->bgt;
        VG_TRY(gather_tables<1>(g, D.ph[1], N, nullptr, b2));
        g->cur[0] = g->vals[layer - 1];
        return tables_ready(g, N);
    }
    VG_TRY(ensure_acc(g, maxN));
    VG_CHECK_CUDA(cudaMemsetAsync(g->acc, 0, N * 4 * sizeof(unsigned long long), c->stream));
    VG_CHECK_CUDA(cudaMemsetAsync(g->acc + 4 * maxN, 0, N * 4 * sizeof(unsigned long long), c->stream));
    unsigned grid = std::min<unsigned>(grid_for(D.n, GKR_THREADS), 148u * 32u);
    {
        ProfScope ps(c, KF_SCATTER2, 73.0 * (double)D.n);   // gate record, two accumulator updates
        k_phase2_scatter<<<grid, GKR_THREADS, 0, c->stream>>>(D.ty, D.u, D.v, D.n, g->bg, bu, g->vu, g->acc,
                                                             g->acc + 4 * maxN);
    }
    VG_LAUNCHED(c);
    g->cur[0] = g->vals[layer - 1];
    return finalize_tables(g, N);
}

static int phase2_check(vg_gkr *g, const vg_fe *r_u, int length_u)
{
    if (!g || !r_u) return vg_fail(VG_ERR_ARG, "vg_gkr_phase2_init: null argument");
    VG_TRY(flush_rounds(g));
    if (g->layer < 1) return vg_fail(VG_ERR_STATE, "phase2_init before phase1_init");
    if (length_u != g->C->L[g->layer - 1].bl)
        return vg_fail(VG_ERR_ARG, "length_u %d != previous layer bit length %d", length_u, g->C->L[g->layer - 1].bl);
    return VG_OK;
}

extern "C" int vg_gkr_phase2_init(vg_gkr *g, const vg_fe *r_u, int length_u, vg_fe v_u)
{
    VG_TRY(phase2_check(g, r_u, length_u));
    fe vu = tofe(v_u);
    VG_CHECK_CUDA(cudaMemcpyAsync(g->vu, &vu, sizeof(fe), cudaMemcpyHostToDevice, g->ctx->stream));   // staged copy
    return phase2_tables(g, r_u, length_u);
}

int vg_gkr_phase2_init_deferred(vg_gkr *g, const vg_fe *r_u, int length_u, vg_fe r_last, vg_fe addend)
{
    VG_TRY(phase2_check(g, r_u, length_u));
    if (!g->deferred || g->rec_n < 1 || g->n != 2)
        return vg_fail(VG_ERR_STATE, "deferred phase2_init must follow the last deferred phase-1 round");
    k_vu<<<1, 1, 0, g->ctx->stream>>>(g->rec + 9 * (g->rec_n - 1) + 3, tofe(r_last), tofe(addend), g->vu);
    VG_LAUNCHED(g->ctx);
    return phase2_tables(g, r_u, length_u);
}

// challenge slots for n records: device copy from the pool, pinned host side
static int grow_challenges(vg_gkr *g, int n)
{
    if (n <= g->r_cap) return VG_OK;
    vg_release(g->ctx, g->rdev);
    g->rdev = nullptr;
    g->r_cap = 0;
    VG_TRY(vg_alloc(g->ctx, (void **)&g->rdev, (size_t)n * sizeof(fe)));
    void *h = g->rhost;
    VG_TRY(vg_pinned_grow(g->ctx, &h, &g->rhost_cap, (size_t)n * sizeof(fe)));
    g->rhost = (fe *)h;
    g->r_cap = n;
    return VG_OK;
}

int vg_gkr_defer(vg_gkr *g, int on)
{
    if (!g) return vg_fail(VG_ERR_ARG, "null gkr");
    VG_TRY(flush_rounds(g));
    g->pend_r.clear();
    g->deferred = on != 0;
    g->rec_n = 0;
    if (!on) return VG_OK;
    // one record per round (at most 2 x 32 per layer) plus v_res
    const int need = 64 * g->C->depth + 16;
    if (need > g->rec_cap) {
        vg_release(g->ctx, g->rec);
        g->rec = nullptr;
        g->rec_cap = 0;
        VG_TRY(vg_alloc(g->ctx, (void **)&g->rec, (size_t)need * 9 * sizeof(fe)));
        g->rec_cap = need;
    }
    VG_TRY(grow_challenges(g, g->rec_cap));
    return VG_OK;
}

int vg_gkr_records(vg_gkr *g, const vg_fe **host, int *n)
{
    if (!g || !host || !n) return vg_fail(VG_ERR_ARG, "vg_gkr_records: null argument");
    VG_TRY(flush_rounds(g));
    if (g->rec_n > g->rec_host_cap) {
        void *p = g->rec_host;
        size_t cap = (size_t)g->rec_host_cap * 9 * sizeof(fe);
        VG_TRY(vg_pinned_grow(g->ctx, &p, &cap, (size_t)g->rec_cap * 9 * sizeof(fe)));
        g->rec_host = (fe *)p;
        g->rec_host_cap = (int)(cap / (9 * sizeof(fe)));
    }
    if (g->rec_n)
        VG_CHECK_CUDA(cudaMemcpyAsync(g->rec_host, g->rec, (size_t)g->rec_n * 9 * sizeof(fe), cudaMemcpyDeviceToHost,
                                      g->ctx->stream));
    *host = (const vg_fe *)g->rec_host;
    *n = g->rec_n;
    return VG_OK;
}

extern "C" int vg_gkr_round(vg_gkr *g, vg_fe previous_random, int current_bit, vg_fe *out3, vg_fe *last6)
{
    if (!g || (!out3 && !(g && g->deferred))) return vg_fail(VG_ERR_ARG, "vg_gkr_round: null argument");
    if (g->deferred && g->rec_n >= g->rec_cap) return vg_fail(VG_ERR_STATE, "deferred record buffer full");
    if (g->layer < 1 || g->n < 2) return vg_fail(VG_ERR_STATE, "sumcheck round without tables (n=%ld)", g->n);
    const bool fold = current_bit != 0;
    if (!fold && !g->round0_pending) return vg_fail(VG_ERR_STATE, "current_bit 0 only directly after an init");
    if (fold && g->round0_pending) return vg_fail(VG_ERR_STATE, "first round after an init must have current_bit 0");
    if (fold && g->n < 4) return vg_fail(VG_ERR_STATE, "no variables left to fold");
    // deferred: once the table is at most the group start, the remaining
    // rounds of the phase are queued and run as round groups (one CTA per
    // chunk, the last group a single CTA); larger tables run one round per
    // launch (their rounds are throughput bound, the group kernel's serial
    // in-CTA steps are not).  A first round that does not fold reads its
    // chunk unfolded, so it starts at half the length.
    const long S = std::max(2L * RG_CHUNK, group_start(g->ctx->device));
    const long lim = fold ? S : S / 2;
    if (g->deferred) {
        if (g->rec_n >= g->r_cap) return vg_fail(VG_ERR_STATE, "challenge slots full");
        g->rhost[g->rec_n] = tofe(previous_random);   // this round's record slot; copied at the next flush
    }
    if (g->deferred && (!g->pend_r.empty() || g->n <= lim)) {
        VG_TRY(flush_held(g));   // the round before this one ran alone
        if (g->pend_r.empty()) {
            g->pend_n0 = g->n;
            g->pend_nofold = !fold;
            g->pend_slot0 = g->rec_n;
            g->pend_chunk = RG_CHUNK;
        }
        g->pend_r.push_back(tofe(previous_random));
        ++g->rec_n;
        if (fold) g->n /= 2;
        g->round0_pending = false;
        if ((int)g->pend_r.size() >= group_total_capacity(g->pend_n0, g->pend_nofold, g->pend_chunk))
            VG_TRY(group_rounds(g));
        return VG_OK;
    }
    vg_ctx *c = g->ctx;
    const fe r = tofe(previous_random);
    if (g->deferred) {
        if (g->held) {
            // this round pairs with the held one: one pass for both
            g->held = false;
            if (g->rec_n != g->held_slot + 1) return vg_fail(VG_ERR_STATE, "paired rounds in non-adjacent records");
            VG_TRY(launch_round2(g, g->held_n, g->held_fold, g->held_slot));
            ++g->rec_n;
            g->n /= 2;   // a round after another always folds
            g->round0_pending = false;
            return VG_OK;
        }
        if (vg_tune_value(c->device, VG_TUNE_ROUND_FUSE) >= 2) {
            g->held = true;
            g->held_fold = fold;
            g->held_slot = g->rec_n;
            g->held_n = g->n;
            ++g->rec_n;
            if (fold) g->n /= 2;
            g->round0_pending = false;
            return VG_OK;
        }
    }
    fe *o3 = g->deferred ? g->rec + 9 * g->rec_n : g->round_out;
    VG_TRY(launch_round(g, g->n, fold, r, g->deferred ? g->rec_n : 0, o3, g->deferred ? o3 + 3 : nullptr));
    if (fold) g->n /= 2;
    g->round0_pending = false;
    if (g->deferred) {
        ++g->rec_n;
        return VG_OK;
    }
    fe *host;
    VG_TRY(vg_pinned(c, 9, &host));
    VG_CHECK_CUDA(cudaMemcpyAsync(host, g->round_out, 3 * sizeof(fe), cudaMemcpyDeviceToHost, c->stream));
    const bool want_last = last6 && g->n == 2;
    if (want_last) {
        for (int k = 0; k < 3; ++k)
            VG_CHECK_CUDA(cudaMemcpyAsync(host + 3 + 2 * k, g->cur[k], 2 * sizeof(fe), cudaMemcpyDeviceToHost, c->stream));
    }
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 3; ++k) out3[k] = tovg(host[k]);
    if (want_last)
        for (int k = 0; k < 6; ++k) last6[k] = tovg(host[3 + k]);
    return VG_OK;
}

// ------------------------------------------- sumcheck tables without a circuit
// The rounds of vg_gkr_round (deferred, records on the device) over tables
// that the caller builds, for provers whose layers are not a gate list (the
// FFT side prover).  The object owns ping-pong tables for up to max_n entries
// and max_records records.
int vg_gkr_tables_create(vg_ctx *ctx, long max_n, int max_records, vg_gkr **out)
{
    if (!ctx || !out || max_n < 2 || (max_n & (max_n - 1)) || max_records < 1)
        return vg_fail(VG_ERR_ARG, "vg_gkr_tables_create: bad argument (max_n %ld, records %d)", max_n, max_records);
    vg_gkr *g = new vg_gkr();
    g->ctx = ctx;
    auto fail = [&](const char *what) {
        cudaGetLastError();
        vg_gkr_destroy(g);
        return vg_fail(VG_ERR_OOM, "vg_gkr_tables_create: %s allocation failed", what);
    };
    if (cudaMalloc(&g->round_parts, 6 * 148 * 8 * sizeof(fe)) != cudaSuccess) return fail("round partials");
    if (cudaMalloc(&g->round_out, 16 * sizeof(fe)) != cudaSuccess) return fail("round sums");
    if (cudaMalloc(&g->round_counter, sizeof(unsigned)) != cudaSuccess) return fail("round counter");
    // ordered on the context's (non-blocking) stream before the first round
    if (cudaMemsetAsync(g->round_counter, 0, sizeof(unsigned), ctx->stream) != cudaSuccess) return fail("round counter");
    g->deferred = true;
    const int rc = vg_gkr_tables_reserve(g, max_n, max_records);
    if (rc != VG_OK) {
        vg_gkr_destroy(g);
        return rc;
    }
    *out = g;
    return VG_OK;
}

// Grows the tables, group partials and records from the stream-ordered pool
// (no device-wide synchronisation, so a server slot can grow while the
// others prove); never shrinks.
int vg_gkr_tables_reserve(vg_gkr *g, long max_n, int max_records)
{
    if (!g || g->C || max_n < 2 || (max_n & (max_n - 1)) || max_records < 1)
        return vg_fail(VG_ERR_ARG, "vg_gkr_tables_reserve: bad argument (max_n %ld, records %d)", max_n, max_records);
    vg_ctx *x = g->ctx;
    VG_TRY(flush_rounds(g));
    if (max_n > g->N_cap) {
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 3; ++k) {
                vg_release(x, g->buf[b][k]);
                g->buf[b][k] = nullptr;
            }
        vg_release(x, g->rg_parts);
        g->rg_parts = nullptr;
        g->N_cap = 0;
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 3; ++k)
                VG_TRY(vg_alloc(x, (void **)&g->buf[b][k], (b == 0 ? max_n : max_n / 2 + 1) * sizeof(fe)));
        VG_TRY(vg_alloc(x, (void **)&g->rg_parts, rg_parts_len(max_n) * sizeof(fe)));
        g->N_cap = max_n;
    }
    if (max_records > g->rec_cap) {
        vg_release(x, g->rec);
        g->rec = nullptr;
        g->rec_cap = 0;
        VG_TRY(vg_alloc(x, (void **)&g->rec, (size_t)max_records * 9 * sizeof(fe)));
        g->rec_cap = max_records;
    }
    VG_TRY(grow_challenges(g, g->rec_cap));
    return VG_OK;
}

int vg_gkr_tables_rewind(vg_gkr *g)
{
    if (!g || g->C) return vg_fail(VG_ERR_ARG, "vg_gkr_tables_rewind: not a tables object");
    VG_TRY(flush_rounds(g));
    g->rec_n = 0;
    g->layer = -1;
    g->n = 0;
    g->round0_pending = false;
    return VG_OK;
}

int vg_gkr_tables_begin(vg_gkr *g, const vg_fe *V, long n, vg_fe **AV, vg_fe **AM)
{
    if (!g || g->C || !V || !AV || !AM) return vg_fail(VG_ERR_ARG, "vg_gkr_tables_begin: bad argument");
    if (n < 2 || n > g->N_cap || (n & (n - 1))) return vg_fail(VG_ERR_ARG, "vg_gkr_tables_begin: %ld entries", n);
    VG_TRY(flush_rounds(g));   // pending rounds of the previous phase read the tables handed out now
    *AV = (vg_fe *)g->buf[0][1];
    *AM = (vg_fe *)g->buf[0][2];
    g->cur[0] = (const fe *)V;
    g->layer = 1;
    return tables_ready(g, n);
}

const vg_fe *vg_gkr_records_dev(const vg_gkr *g) { return (const vg_fe *)g->rec; }
void vg_gkr_graph_counts(const vg_gkr *g, long long *replays, long long *captures)
{
    *replays = g ? g->graph_replays : 0;
    *captures = g ? g->graph_captures : 0;
}
int vg_gkr_record_count(const vg_gkr *g) { return g->rec_n; }
