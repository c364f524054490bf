// Polynomial commitment and FRI commit phase on the device.
//
// Data layout in HBM: every codeword set is slice-major, 65 slices (64 data +
// 1 mask) of the per-slice length n, slice s at base + s * n.  The reference
// stores the same values interleaved ((j << 7) | (s << 1) | b, fri.cpp:86-96,
// 345-362); slice-major keeps every kernel's loads coalesced (a warp reads 32
// consecutive positions of one slice) and the interleaved form is produced
// only for the small final level the verifier reads.
//
// Per commitment of an input of 2^L elements (S = 2^(L-1), R = S/32):
//   l_eval, h_eval       65 x S      kept for query answers
//   q_eval, virtual oracle 65 x S    temporaries (freed after use)
//   FRI level t          65 x S/2^(t+1) codewords + Merkle tree
#include "common.cuh"
#include "merkle.cuh"
#include "hash.cuh"
#include "internal.h"
#include <algorithm>
#include <cstring>

namespace {

__device__ __forceinline__ uint64_t halfp(uint64_t x) { return (x & 1) ? ((x + vg::P) >> 1) : (x >> 1); }
__device__ __forceinline__ fe half_fe(fe x) { return vg::fe_make(halfp(x.real), halfp(x.img)); }

__device__ __forceinline__ fe tw_pow(const fe *__restrict__ lo, const fe *__restrict__ hi, uint64_t e)
{
    fe a = lo[e & 4095];
    uint64_t h = e >> 12;
    if (h) a = a * hi[h];
    return a;
}

// lq[s][j] = l[s][j * stride] * q[s][j * stride], j < 2m (poly_commit.h:211-218, 271-278)
__global__ void k_lq_sample(const fe *__restrict__ l, const fe *__restrict__ q, long S, long m, long stride,
                            int nslices, fe *__restrict__ lq)
{
    long total = (long)nslices * 2 * m;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        long s = i / (2 * m), j = i % (2 * m);
        long src = s * S + j * stride;
        lq[i] = l[src] * q[src];
    }
}

// Virtual oracle (poly_commit.h:241-263 mask slice, 298-322 data slices):
// vo[s][j] = (l q - (x^m - 1) h - c0_s) * m * x^-1 at x = w_S^j, where
// c0_s = lq_coef[s][0] + lq_coef[s][m] is the constant term of g + h.
// tw_f/tw_i are the twiddle tables of w_S and w_S^-1.
__global__ void k_virtual_oracle(const fe *__restrict__ l, const fe *__restrict__ q, const fe *__restrict__ h,
                                 const fe *__restrict__ lq_coef, long S, long m, int logS, int slice0, int nslices,
                                 const fe *__restrict__ twf_lo, const fe *__restrict__ twf_hi,
                                 const fe *__restrict__ twi_lo, const fe *__restrict__ twi_hi, fe *__restrict__ vo)
{
    const uint64_t mask = (uint64_t)S - 1;
    const fe mm = vg::fe_make((uint64_t)m % vg::P, 0);
    long total = (long)nslices * S;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        long s = i >> logS, j = i & mask;
        long off = (long)(slice0 + s) * S + j;
        fe c0 = lq_coef[s * 2 * m] + lq_coef[s * 2 * m + m];
        fe xm = tw_pow(twf_lo, twf_hi, ((uint64_t)j * (uint64_t)m) & mask);
        fe g = vg::fe_fma(l[off] * q[off], vg::fe_one() - xm, h[off]);   // l q - (x^m - 1) h
        fe xinv = tw_pow(twi_lo, twi_hi, (uint64_t)j);
        vo[off] = ((g - c0) * mm) * xinv;
    }
}

// all_sum[s] = (lq_coef[s][0] + lq_coef[s][m]) * m  (poly_commit.h:264, 326)
__global__ void k_all_sum(const fe *__restrict__ lq_coef, long m, int slice0, int nslices, fe *__restrict__ out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslices) return;
    fe c0 = lq_coef[(long)s * 2 * m] + lq_coef[(long)s * 2 * m + m];
    out[slice0 + s] = c0 * vg::fe_make((uint64_t)m % vg::P, 0);
}

// sum over data positions (stride 32 in every data slice) and mask positions
// (stride gap in the mask slice) of l * q  (poly_commit.h:179-193)
__global__ void k_inner_product(const fe *__restrict__ l, const fe *__restrict__ q, long S, long gap,
                                fe *__restrict__ parts)
{
    __shared__ fe sm[32];
    const long R = S >> 5;
    const long n_data = 64 * R, n_mask = S / gap;
    fe acc[1] = {vg::fe_zero()};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n_data + n_mask; i += (long)gridDim.x * blockDim.x) {
        long pos = i < n_data ? (i << 5) : (64 * S + (i - n_data) * gap);
        acc[0] = vg::fe_fma(acc[0], l[pos], q[pos]);
    }
    block_sum<1>(acc, sm);
    if (threadIdx.x == 0) parts[blockIdx.x] = acc[0];
}

// One FRI fold fused with the next level's leaf hash chains.
// Input codeword set (per-slice length n, domain <w>, w = w_S^(2^t)):
//   out[s][i] = ((a + b) + r w^-i (a - b)) / 2,  a = c[s][i], b = c[s][i + n/2]
// (fri.cpp:321-340 data, 367-379 mask).  Thread k < n/4 produces out[s][k] and
// out[s][k + n/4], which are exactly the pair hashed into leaf k of the new
// level (fri.cpp:394-420), so the fold output is never re-read.
template <int KIND>
__global__ void __launch_bounds__(128) k_fri_fold_leaf(const fe *__restrict__ c, long n, int t, fe r,
                                                       const fe *__restrict__ twi_lo, const fe *__restrict__ twi_hi,
                                                       fe *__restrict__ out, uint64_t *__restrict__ leaves)
{
    const long q4 = n >> 2, half = n >> 1, nh = n >> 1;
    long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (k >= q4) return;
    fe t0 = r * tw_pow(twi_lo, twi_hi, (uint64_t)k << t);
    fe t1 = r * tw_pow(twi_lo, twi_hi, (uint64_t)(k + q4) << t);
    uint64_t h[4] = {0, 0, 0, 0};
    for (int s = 0; s < 65; ++s) {
        const fe *cs = c + (long)s * n;
        fe a0 = cs[k], b0 = cs[k + half], a1 = cs[k + q4], b1 = cs[k + q4 + half];
        fe y0 = half_fe(vg::fe_fma(a0 + b0, t0, a0 - b0));
        fe y1 = half_fe(vg::fe_fma(a1 + b1, t1, a1 - b1));
        out[(long)s * nh + k] = y0;
        out[(long)s * nh + k + q4] = y1;
        uint64_t w[8] = {y0.img, y0.real, y1.img, y1.real, h[0], h[1], h[2], h[3]};
        vg::hash64<KIND>(w, h);
    }
    ulonglong2 *o = (ulonglong2 *)(leaves + 4 * k);
    o[0] = make_ulonglong2(h[0], h[1]);
    o[1] = make_ulonglong2(h[2], h[3]);
}

// One FRI fold without hashing (the leaf chains of all levels are batched):
// out[s][i] = ((a + b) + r w^-(i 2^t) (a - b)) / 2, a = c[s][i], b = c[s][i + n/2].
__global__ void k_fri_fold(const fe *__restrict__ c, long n, int t, fe r, const fe *__restrict__ twi_lo,
                           const fe *__restrict__ twi_hi, fe *__restrict__ out)
{
    const long h = n >> 1, total = 65 * h;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long s = i / h, k = i - s * h;
        const fe a = c[s * n + k], b = c[s * n + k + h];
        const fe w = r * tw_pow(twi_lo, twi_hi, (uint64_t)k << t);
        out[i] = half_fe(vg::fe_fma(a + b, w, a - b));
    }
}

// Query answers for a batch: block q answers query q from codeword set
// desc[which[q]] at position pos[q] (taken modulo n/2): 65 value pairs and the
// authentication path (siblings bottom-up, then the leaf).
struct QueryDesc {
    const fe *cw;
    const uint64_t *tree;
    long n;
    int depth;
};
__global__ void k_gather_batch(const QueryDesc *__restrict__ desc, const int *__restrict__ which,
                               const long *__restrict__ pos, fe *__restrict__ vals, uint64_t *__restrict__ paths)
{
    const int q = blockIdx.x, i = threadIdx.x;
    const QueryDesc d = desc[which[q]];
    const long h = d.n >> 1, p = pos[q] % h;
    if (i < 65) {
        vals[(long)q * 130 + 2 * i] = d.cw[(long)i * d.n + p];
        vals[(long)q * 130 + 2 * i + 1] = d.cw[(long)i * d.n + p + h];
    }
    if (i <= d.depth) {
        const long leaf = p + h;
        const long src = i < d.depth ? ((leaf >> i) ^ 1) : leaf;
        for (int w = 0; w < 4; ++w) paths[((long)q * 32 + i) * 4 + w] = d.tree[4 * src + w];
    }
}

long mask_gap(long S, long n_mask)
{
    long gap = S / n_mask, g = 1;
    while (g * 2 <= gap) g *= 2;
    return g;
}

int ilog2l(long x)
{
    int k = 0;
    while ((1L << k) < x) ++k;
    return k;
}

}  // namespace

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

// grows a persistent buffer; buffers are kept across commitments so a proof
// does not pay cudaMalloc/cudaFree (and cudaFree's device synchronisation)
static int ensure(vg_ctx *c, DevBuf &b, size_t bytes)
{
    if (bytes <= b.cap) return VG_OK;
    vg_release(c, b.p);   // stream ordered: no device-wide synchronisation
    b.p = nullptr;
    b.cap = 0;
    VG_TRY(vg_alloc(c, &b.p, bytes));
    b.cap = bytes;
    return VG_OK;
}

struct PcLevel {
    DevBuf cw, tree;   // 65 x n codewords, n digests (n/2 leaves)
    long n = 0;
};

struct vg_pc {
    vg_ctx *ctx = nullptr;
    int log_len = 0;
    long S = 0, R = 0, gap = 0, M = 0;
    DevBuf l_eval, h_eval, q_eval, vo, lq, lqc, mask, staging, tree_l, tree_h, qdesc, qio;
    DevBuf mask2, res, roots;   // deferred proof: public mask, <l,q> + all_sum, roots
    fe *hpin = nullptr;         // deferred proof: pinned staging and results
    size_t hpin_cap = 0;        // in elements
    std::vector<PcLevel> levels;
    int nlevels = 0;
    bool have_private = false, have_public = false;
    fe *F(DevBuf &b) { return (fe *)b.p; }
    uint64_t *U(DevBuf &b) { return (uint64_t *)b.p; }
};

static void pc_free(vg_pc *pc)
{
    DevBuf *all[] = {&pc->l_eval, &pc->h_eval, &pc->q_eval, &pc->vo, &pc->lq, &pc->lqc, &pc->mask, &pc->staging,
                     &pc->tree_l, &pc->tree_h, &pc->qdesc, &pc->qio, &pc->mask2, &pc->res, &pc->roots};
    for (DevBuf *b : all) {
        cudaFree(b->p);
        b->p = nullptr;
        b->cap = 0;
    }
    for (auto &L : pc->levels) {
        cudaFree(L.cw.p);
        cudaFree(L.tree.p);
    }
    pc->levels.clear();
    pc->nlevels = 0;
    pc->have_private = pc->have_public = false;
    if (pc->hpin) cudaFreeHost(pc->hpin);
    pc->hpin = nullptr;
    pc->hpin_cap = 0;
}

static fe root_of(int log_order) { return vg::fe_root_of_unity(log_order); }
static vg_fe to_vg(fe x) { vg_fe r; r.img = x.img; r.real = x.real; return r; }

// RS encoding of `batch` slices of m values (stride m) into length S (stride S):
// interpolate on <w_m>, evaluate on <w_S>  (poly_commit.h:107-108, 152-153)
static int rs_encode(vg_ctx *c, const fe *vals, long m, int batch, fe *out, long S, fe *coef_tmp)
{
    int lm = ilog2l(m), lS = ilog2l(S);
    VG_TRY(vg_ntt(c, (const vg_fe *)vals, m, m, (vg_fe *)coef_tmp, lm, m, batch, to_vg(vg::fe_inv(root_of(lm))), 1));
    VG_TRY(vg_ntt(c, (const vg_fe *)coef_tmp, m, m, (vg_fe *)out, lS, S, batch, to_vg(root_of(lS)), 0));
    return VG_OK;
}

static int commit_tree(vg_ctx *c, const fe *cw, long S, uint64_t *tree, vg_digest *root)
{
    long nleaves = S >> 1;
    VG_TRY(vg_leaf_chain_dev(c, cw, 65, S, tree + 4 * nleaves));
    VG_TRY(vg_merkle_build(c, tree, nleaves));
    if (root) {
        fe *host;
        VG_TRY(vg_pinned(c, 2, &host));
        VG_CHECK_CUDA(cudaMemcpyAsync(host, tree + 4, 32, cudaMemcpyDeviceToHost, c->stream));
        VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
        memcpy(root, host, 32);
    }
    return VG_OK;
}

extern "C" int vg_pc_create(vg_ctx *ctx, vg_pc **out)
{
    if (!ctx || !out) return vg_fail(VG_ERR_ARG, "vg_pc_create: null argument");
    vg_pc *pc = new vg_pc();
    pc->ctx = ctx;
    *out = pc;
    return VG_OK;
}

extern "C" int vg_pc_destroy(vg_pc *pc)
{
    if (!pc) return VG_OK;
    cudaStreamSynchronize(pc->ctx->stream);
    pc_free(pc);
    delete pc;
    return VG_OK;
}

extern "C" int vg_pc_info(vg_pc *pc, int *log_len, long *slice_size, int *levels)
{
    if (!pc) return vg_fail(VG_ERR_ARG, "null pc");
    if (log_len) *log_len = pc->log_len;
    if (slice_size) *slice_size = pc->S;
    if (levels) *levels = pc->nlevels;
    return VG_OK;
}

// the private/public input on the device (a host array is staged)
static int device_input(vg_pc *pc, const vg_fe *x, long N, const fe **out)
{
    if (vg_is_device_ptr(x)) {
        *out = (const fe *)x;
        return VG_OK;
    }
    VG_TRY(ensure(pc->ctx, pc->staging, N * sizeof(fe)));
    VG_CHECK_CUDA(cudaMemcpyAsync(pc->staging.p, x, N * sizeof(fe), cudaMemcpyHostToDevice, pc->ctx->stream));
    *out = (const fe *)pc->staging.p;
    return VG_OK;
}

// zero-padded mask of M entries on the device (poly_commit.h:66-70, 138-139);
// with staging == nullptr through the context's pinned buffer (synchronised,
// it is reused), else through the caller's pinned staging (not synchronised)
static int device_mask(vg_pc *pc, DevBuf &dst, const vg_fe *mask, long n_mask, long M, fe *staging = nullptr)
{
    vg_ctx *c = pc->ctx;
    VG_TRY(ensure(c, dst, M * sizeof(fe)));
    fe *host = staging;
    if (!host) VG_TRY(vg_pinned(c, M, &host));
    for (long i = 0; i < M; ++i) host[i] = i < n_mask ? vg::fe_make(mask[i].real, mask[i].img) : vg::fe_zero();
    VG_CHECK_CUDA(cudaMemcpyAsync(dst.p, host, M * sizeof(fe), cudaMemcpyHostToDevice, c->stream));
    if (!staging) VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    return VG_OK;
}

static int encode_private(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *mask, long n_mask, long *mask_len,
                          fe *staging)
{
    if (!pc || !priv || !mask || n_mask < 1 || log_len < 7 || log_len > 28)
        return vg_fail(VG_ERR_ARG, "vg_pc_encode_private: bad argument (log_len=%d n_mask=%ld)", log_len, n_mask);
    vg_ctx *c = pc->ctx;
    pc->have_private = pc->have_public = false;
    pc->nlevels = 0;
    pc->log_len = log_len;
    pc->S = 1L << (log_len - 1);
    pc->R = pc->S >> 5;
    if (n_mask > pc->S) return vg_fail(VG_ERR_ARG, "mask longer than a slice (%ld > %ld)", n_mask, pc->S);
    pc->gap = mask_gap(pc->S, n_mask);
    pc->M = pc->S / pc->gap;
    const long S = pc->S, R = pc->R, M = pc->M, N = 1L << log_len;
    VG_TRY(ensure(c, pc->l_eval, 65 * S * sizeof(fe)));
    const fe *priv_d;
    VG_TRY(device_input(pc, priv, N, &priv_d));
    fe *coef;
    VG_TRY(vg_scratch2(c, 64 * R * sizeof(fe), (void **)&coef));
    VG_TRY(rs_encode(c, priv_d, R, 64, pc->F(pc->l_eval), S, coef));
    VG_TRY(device_mask(pc, pc->mask, mask, n_mask, M, staging));
    VG_TRY(rs_encode(c, pc->F(pc->mask), M, 1, pc->F(pc->l_eval) + 64 * S, S, coef));
    if (mask_len) *mask_len = M;
    pc->have_private = true;
    return VG_OK;
}

extern "C" int vg_pc_encode_private(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *mask, long n_mask,
                                    long *mask_len)
{
    return encode_private(pc, priv, log_len, mask, n_mask, mask_len, nullptr);
}

long vg_pc_mask_len(int log_len, long n_pri_mask)
{
    const long S = 1L << (log_len - 1);
    return S / mask_gap(S, n_pri_mask);
}

// <l, q> to res_dev[0] and all_sum to res_dev[1 .. 65]
static int encode_public(vg_pc *pc, const vg_fe *pub, const vg_fe *pub_mask, long n_mask, fe *res_dev, fe *staging)
{
    if (!pc || !pub || !pub_mask) return vg_fail(VG_ERR_ARG, "vg_pc_encode_public: null argument");
    if (!pc->have_private) return vg_fail(VG_ERR_STATE, "commit_public before commit_private");
    if (n_mask > pc->M) return vg_fail(VG_ERR_ARG, "public mask longer than the padded private mask (%ld > %ld)", n_mask, pc->M);
    if (pc->gap == 1) return vg_fail(VG_ERR_ARG, "mask fills the whole slice (mask_position_gap == 1)");
    vg_ctx *c = pc->ctx;
    const long S = pc->S, R = pc->R, M = pc->M, N = 1L << pc->log_len;
    const int logS = ilog2l(S);
    const long lq_len = 64 * 2 * R + 2 * M;
    VG_TRY(ensure(c, pc->q_eval, 65 * S * sizeof(fe)));
    VG_TRY(ensure(c, pc->h_eval, 65 * S * sizeof(fe)));
    VG_TRY(ensure(c, pc->vo, 65 * S * sizeof(fe)));
    VG_TRY(ensure(c, pc->lq, lq_len * sizeof(fe)));
    VG_TRY(ensure(c, pc->lqc, lq_len * sizeof(fe)));
    fe *l_eval = pc->F(pc->l_eval), *q_eval = pc->F(pc->q_eval), *h_eval = pc->F(pc->h_eval);
    fe *lq = pc->F(pc->lq), *lqc = pc->F(pc->lqc);

    const fe *pub_d;
    VG_TRY(device_input(pc, pub, N, &pub_d));
    fe *coef;
    VG_TRY(vg_scratch2(c, 64 * R * sizeof(fe), (void **)&coef));
    VG_TRY(rs_encode(c, pub_d, R, 64, q_eval, S, coef));
    DevBuf &mbuf = staging ? pc->mask2 : pc->mask;   // the deferred proof keeps the private mask
    VG_TRY(device_mask(pc, mbuf, pub_mask, n_mask, M, staging));
    VG_TRY(rs_encode(c, pc->F(mbuf), M, 1, q_eval + 64 * S, S, coef));

    // inner product check value
    fe *parts;
    const int nb = 148 * 4;
    VG_TRY(vg_partials(c, nb, &parts));
    k_inner_product<<<nb, 256, 0, c->stream>>>(l_eval, q_eval, S, pc->gap, parts);
    VG_LAUNCHED(c);
    VG_TRY(vg_reduce_partials(c, parts, nb, 1, res_dev));

    // lq samples, their interpolation and the quotient h
    fe *lq_m = lq + 64 * 2 * R, *lqc_m = lqc + 64 * 2 * R;
    k_lq_sample<<<148 * 8, 256, 0, c->stream>>>(l_eval, q_eval, S, R, S / (2 * R), 64, lq);
    VG_LAUNCHED(c);
    k_lq_sample<<<grid_for(2 * M, 256), 256, 0, c->stream>>>(l_eval + 64 * S, q_eval + 64 * S, S, M, S / (2 * M), 1, lq_m);
    VG_LAUNCHED(c);
    int l2R = ilog2l(2 * R), l2M = ilog2l(2 * M);
    VG_TRY(vg_ntt(c, (const vg_fe *)lq, 2 * R, 2 * R, (vg_fe *)lqc, l2R, 2 * R, 64, to_vg(vg::fe_inv(root_of(l2R))), 1));
    VG_TRY(vg_ntt(c, (const vg_fe *)lq_m, 2 * M, 2 * M, (vg_fe *)lqc_m, l2M, 2 * M, 1, to_vg(vg::fe_inv(root_of(l2M))), 1));
    VG_TRY(vg_ntt(c, (const vg_fe *)(lqc + R), R, 2 * R, (vg_fe *)h_eval, logS, S, 64, to_vg(root_of(logS)), 0));
    VG_TRY(vg_ntt(c, (const vg_fe *)(lqc_m + M), M, 2 * M, (vg_fe *)(h_eval + 64 * S), logS, S, 1, to_vg(root_of(logS)), 0));

    // virtual oracle and all_sum
    const fe *tf_lo, *tf_hi, *ti_lo, *ti_hi;
    VG_TRY(vg_twiddles(c, root_of(logS), logS, &tf_lo, &tf_hi));
    VG_TRY(vg_twiddles(c, vg::fe_inv(root_of(logS)), logS, &ti_lo, &ti_hi));
    {
        ProfScope ps(c, KF_VIRTUAL_ORACLE, 64.0 * 64.0 * (double)S);
        k_virtual_oracle<<<148 * 16, 256, 0, c->stream>>>(l_eval, q_eval, h_eval, lqc, S, R, logS, 0, 64,
                                                          tf_lo, tf_hi, ti_lo, ti_hi, pc->F(pc->vo));
    }
    VG_LAUNCHED(c);
    k_virtual_oracle<<<grid_for(S, 256), 256, 0, c->stream>>>(l_eval, q_eval, h_eval, lqc_m, S, M, logS, 64, 1,
                                                             tf_lo, tf_hi, ti_lo, ti_hi, pc->F(pc->vo));
    VG_LAUNCHED(c);
    fe *sums_d = res_dev + 1;
    k_all_sum<<<1, 64, 0, c->stream>>>(lqc, R, 0, 64, sums_d);
    VG_LAUNCHED(c);
    k_all_sum<<<1, 1, 0, c->stream>>>(lqc_m, M, 64, 1, sums_d);
    VG_LAUNCHED(c);
    pc->have_public = true;
    return VG_OK;
}

extern "C" int vg_pc_encode_public(vg_pc *pc, const vg_fe *pub, const vg_fe *pub_mask, long n_mask, vg_fe *all_sum,
                                   vg_fe *inner_product)
{
    if (!pc || !all_sum) return vg_fail(VG_ERR_ARG, "vg_pc_encode_public: null argument");
    vg_ctx *c = pc->ctx;
    VG_TRY(ensure(c, pc->res, 66 * sizeof(fe)));
    VG_TRY(encode_public(pc, pub, pub_mask, n_mask, pc->F(pc->res), nullptr));
    fe *host;
    VG_TRY(vg_pinned(c, 66, &host));
    VG_CHECK_CUDA(cudaMemcpyAsync(host, pc->res.p, 66 * sizeof(fe), cudaMemcpyDeviceToHost, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < 65; ++i) all_sum[i] = to_vg(host[1 + i]);
    if (inner_product) *inner_product = to_vg(host[0]);
    return VG_OK;
}

extern "C" int vg_pc_init_commit(vg_pc *pc, int oracle, vg_digest *root)
{
    if (!pc || !root || (oracle != 0 && oracle != 1)) return vg_fail(VG_ERR_ARG, "vg_pc_init_commit: bad argument");
    if (oracle == 0 && !pc->have_private) return vg_fail(VG_ERR_STATE, "init_commit(0) before encode_private");
    if (oracle == 1 && !pc->have_public) return vg_fail(VG_ERR_STATE, "init_commit(1) before encode_public");
    if (oracle == 0) pc->nlevels = 0;   // a new private commitment restarts the FRI levels
    DevBuf &t = oracle == 0 ? pc->tree_l : pc->tree_h;
    VG_TRY(ensure(pc->ctx, t, (size_t)pc->S * 32));
    return commit_tree(pc->ctx, pc->F(oracle == 0 ? pc->l_eval : pc->h_eval), pc->S, pc->U(t), root);
}

extern "C" int vg_eq_table(vg_ctx *c, const vg_fe *r, int log_len, vg_fe *pub);

extern "C" int vg_pc_fri_step(vg_pc *pc, vg_fe r_, vg_digest *root)
{
    if (!pc || !root) return vg_fail(VG_ERR_ARG, "vg_pc_fri_step: null argument");
    if (!pc->have_public) return vg_fail(VG_ERR_STATE, "fri step before commit_public");
    vg_ctx *c = pc->ctx;
    const int t = pc->nlevels;
    const long n = pc->S >> t;
    if (n < 8) return vg_fail(VG_ERR_STATE, "FRI folded below 8 elements per slice");
    const fe *in = t == 0 ? pc->F(pc->vo) : pc->F(pc->levels[t - 1].cw);
    if ((int)pc->levels.size() <= t) pc->levels.resize(t + 1);
    PcLevel &L = pc->levels[t];
    L.n = n >> 1;
    VG_TRY(ensure(c, L.cw, 65 * L.n * sizeof(fe)));
    VG_TRY(ensure(c, L.tree, L.n * 32));
    const int logS = ilog2l(pc->S);
    const fe *ti_lo, *ti_hi;
    VG_TRY(vg_twiddles(c, vg::fe_inv(root_of(logS)), logS, &ti_lo, &ti_hi));
    fe r = vg::fe_make(r_.real, r_.img);
    long q4 = n >> 2;
    long nleaves = L.n >> 1;
    uint64_t *tree = pc->U(L.tree);
    {
        ProfScope ps(c, KF_FRI_FOLD, 16.0 * 65.0 * (double)n * 1.5 + 32.0 * (double)q4);
        if (c->hash_kind == VG_HASH_SHA256)
            k_fri_fold_leaf<VG_HASH_SHA256><<<grid_for(q4, 128), 128, 0, c->stream>>>(in, n, t, r, ti_lo, ti_hi, pc->F(L.cw), tree + 4 * nleaves);
        else
            k_fri_fold_leaf<VG_HASH_SHA3_256><<<grid_for(q4, 128), 128, 0, c->stream>>>(in, n, t, r, ti_lo, ti_hi, pc->F(L.cw), tree + 4 * nleaves);
    }
    VG_LAUNCHED(c);
    VG_TRY(vg_merkle_build(c, tree, nleaves));
    pc->nlevels = t + 1;
    fe *host;
    VG_TRY(vg_pinned(c, 2, &host));
    VG_CHECK_CUDA(cudaMemcpyAsync(host, tree + 4, 32, cudaMemcpyDeviceToHost, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    memcpy(root, host, 32);
    return VG_OK;
}

extern "C" int vg_pc_fri_final(vg_pc *pc, vg_fe *data, vg_fe *mask, long *n_out)
{
    if (!pc || pc->nlevels == 0) return vg_fail(VG_ERR_STATE, "vg_pc_fri_final: no FRI level");
    PcLevel &L = pc->levels[pc->nlevels - 1];
    const long n = L.n, h = n >> 1;
    if (n_out) *n_out = n;
    if (!data && !mask) return VG_OK;
    fe *buf;
    VG_TRY(vg_pinned(pc->ctx, 65 * n, &buf));
    VG_CHECK_CUDA(cudaMemcpyAsync(buf, L.cw.p, 65 * n * sizeof(fe), cudaMemcpyDeviceToHost, pc->ctx->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(pc->ctx->stream));
    // interleaved layout of fri.cpp:348-363 and 382-388
    for (long j = 0; j < h; ++j) {
        for (int s = 0; s < 64; ++s) {
            if (data) {
                data[(j << 7) | (s << 1) | 0] = to_vg(buf[s * n + j]);
                data[(j << 7) | (s << 1) | 1] = to_vg(buf[s * n + j + h]);
            }
        }
        if (mask) {
            mask[2 * j] = to_vg(buf[64 * n + j]);
            mask[2 * j + 1] = to_vg(buf[64 * n + j + h]);
        }
    }
    return VG_OK;
}

// one descriptor per codeword set: 0 = l, 1 = h, 2 + t = FRI level t
static int query_descs(vg_pc *pc, std::vector<QueryDesc> &d)
{
    d.clear();
    const int depth0 = ilog2l(pc->S / 2);
    d.push_back({pc->F(pc->l_eval), pc->U(pc->tree_l), pc->S, depth0});
    d.push_back({pc->F(pc->h_eval), pc->U(pc->tree_h), pc->S, depth0});
    for (int t = 0; t < pc->nlevels; ++t)
        d.push_back({pc->F(pc->levels[t].cw), pc->U(pc->levels[t].tree), pc->levels[t].n, ilog2l(pc->levels[t].n / 2)});
    return VG_OK;
}

extern "C" int vg_pc_query_batch(vg_pc *pc, int nq, const int *which, const long *pos, vg_fe *values, vg_digest *paths,
                                 int *path_len)
{
    if (!pc || nq < 0 || (nq && (!which || !pos || !values || !paths)))
        return vg_fail(VG_ERR_ARG, "vg_pc_query_batch: bad argument");
    if (nq == 0) return VG_OK;
    std::vector<QueryDesc> d;
    query_descs(pc, d);
    for (int q = 0; q < nq; ++q) {
        if (which[q] < 0 || which[q] >= (int)d.size()) return vg_fail(VG_ERR_ARG, "query %d: no codeword set %d", q, which[q]);
        if (which[q] == 0 && !pc->have_private) return vg_fail(VG_ERR_STATE, "no private commitment");
        if (which[q] == 1 && !pc->have_public) return vg_fail(VG_ERR_STATE, "no public commitment");
        if (pos[q] < 0) return vg_fail(VG_ERR_ARG, "query %d: negative position", q);
        if (which[q] < 2 && pos[q] >= pc->S / 2) return vg_fail(VG_ERR_ARG, "query %d: position out of range", q);
        if (path_len) path_len[q] = d[which[q]].depth + 1;
    }
    vg_ctx *c = pc->ctx;
    // sections of the upload, each starting on a 16-byte boundary:
    // descriptors (8-byte members), positions (long), codeword-set indices (int)
    auto up16 = [](size_t x) { return (x + 15) / 16 * 16; };
    const size_t desc_b = d.size() * sizeof(QueryDesc), pos_b = nq * sizeof(long), which_b = nq * sizeof(int);
    const size_t off_pos = up16(desc_b), off_which = off_pos + up16(pos_b), in_b = off_which + up16(which_b);
    const size_t vals_b = (size_t)nq * 130 * sizeof(fe), paths_b = (size_t)nq * 32 * 32;
    VG_TRY(ensure(c, pc->qdesc, in_b));
    VG_TRY(ensure(c, pc->qio, vals_b + paths_b));
    fe *host;
    const size_t pinned_elems = (std::max(in_b, vals_b + paths_b) + 15) / 16;
    VG_TRY(vg_pinned(c, pinned_elems, &host));
    char *hb = (char *)host;
    memcpy(hb, d.data(), desc_b);
    memcpy(hb + off_pos, pos, pos_b);
    memcpy(hb + off_which, which, which_b);
    char *db = (char *)pc->qdesc.p;
    VG_CHECK_CUDA(cudaMemcpyAsync(db, hb, in_b, cudaMemcpyHostToDevice, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    fe *vals_d = (fe *)pc->qio.p;
    uint64_t *paths_d = (uint64_t *)((char *)pc->qio.p + vals_b);
    k_gather_batch<<<nq, 96, 0, c->stream>>>((const QueryDesc *)db, (const int *)(db + off_which),
                                             (const long *)(db + off_pos), vals_d, paths_d);
    VG_LAUNCHED(c);
    VG_CHECK_CUDA(cudaMemcpyAsync(host, pc->qio.p, vals_b + paths_b, cudaMemcpyDeviceToHost, c->stream));
    VG_CHECK_CUDA(cudaStreamSynchronize(c->stream));
    memcpy(values, host, vals_b);
    memcpy(paths, (char *)host + vals_b, paths_b);
    return VG_OK;
}

extern "C" int vg_pc_query_init(vg_pc *pc, long pow0, int oracle, vg_fe *values, vg_digest *path)
{
    if (!pc || !values || !path || (oracle != 0 && oracle != 1)) return vg_fail(VG_ERR_ARG, "vg_pc_query_init: bad argument");
    std::vector<vg_digest> p(32);
    int plen = 0;
    long pos = pow0;
    VG_TRY(vg_pc_query_batch(pc, 1, &oracle, &pos, values, p.data(), &plen));
    memcpy(path, p.data(), plen * sizeof(vg_digest));
    return VG_OK;
}

extern "C" int vg_pc_query_step(vg_pc *pc, int lvl, long pow, vg_fe *values, vg_digest *path, int *path_len)
{
    if (!pc || !values || !path || lvl < 0 || lvl >= pc->nlevels)
        return vg_fail(VG_ERR_ARG, "vg_pc_query_step: bad argument (lvl %d)", lvl);
    std::vector<vg_digest> p(32);
    int plen = 0, which = 2 + lvl;
    VG_TRY(vg_pc_query_batch(pc, 1, &which, &pow, values, p.data(), &plen));
    memcpy(path, p.data(), plen * sizeof(vg_digest));
    if (path_len) *path_len = plen;
    return VG_OK;
}

// ------------------------------------------------ one-sync proof commitment
static int ensure_pinned(vg_pc *pc, size_t elems)
{
    if (elems <= pc->hpin_cap) return VG_OK;
    void *p = pc->hpin;
    size_t cap = pc->hpin_cap * sizeof(fe);
    VG_TRY(vg_pinned_grow(pc->ctx, &p, &cap, elems * sizeof(fe)));
    pc->hpin = (fe *)p;
    pc->hpin_cap = cap / sizeof(fe);
    return VG_OK;
}

int vg_pc_prove_deferred(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *pri_mask, long n_pri_mask,
                         const vg_fe *pub, const vg_fe *pub_mask, long n_pub_mask, const vg_fe *fri_r, int nlevels,
                         int nq, const int *which, const long *pos, vg_pc_results *out)
{
    if (!pc || !priv || !pri_mask || !pub || !pub_mask || (nlevels && !fri_r) || nq < 0 || (nq && (!which || !pos)) || !out)
        return vg_fail(VG_ERR_ARG, "vg_pc_prove_deferred: bad argument");
    if (log_len < 7 || log_len > 28 || n_pri_mask < 1) return vg_fail(VG_ERR_ARG, "vg_pc_prove_deferred: log_len %d", log_len);
    vg_ctx *c = pc->ctx;
    const long S = 1L << (log_len - 1);
    if (nlevels < 0 || (S >> nlevels) < 8) return vg_fail(VG_ERR_ARG, "%d FRI levels fold below 8 elements", nlevels);
    const long M = vg_pc_mask_len(log_len, n_pri_mask);
    const long n_final = nlevels ? (S >> nlevels) : S;

    // pinned layout (16-byte elements): masks | query upload | results
    const size_t ndesc = 2 + nlevels;
    auto up16 = [](size_t x) { return (x + 15) / 16 * 16; };
    const size_t desc_b = ndesc * sizeof(QueryDesc), pos_b = (size_t)nq * sizeof(long), which_b = (size_t)nq * sizeof(int);
    const size_t off_pos = up16(desc_b), off_which = off_pos + up16(pos_b), in_b = off_which + up16(which_b);
    const size_t e_masks = 2 * (size_t)M, e_in = in_b / 16;
    const size_t e_res = 66, e_roots = 2 * ndesc, e_final = 65 * (size_t)n_final, e_qv = (size_t)nq * 130,
                 e_qp = (size_t)nq * 32 * 2;
    VG_TRY(ensure_pinned(pc, e_masks + e_in + e_res + e_roots + e_final + e_qv + e_qp));
    fe *h_mask = pc->hpin, *h_in = h_mask + e_masks, *h_res = h_in + e_in, *h_roots = h_res + e_res,
       *h_final = h_roots + e_roots, *h_qv = h_final + e_final, *h_qp = h_qv + e_qv;

    // commitment of the private and public inputs, virtual oracle
    long Mp = 0;
    VG_TRY(encode_private(pc, priv, log_len, pri_mask, n_pri_mask, &Mp, h_mask));
    if (Mp != M) return vg_fail(VG_ERR_STATE, "mask length %ld != %ld", Mp, M);
    if (n_pub_mask > M) return vg_fail(VG_ERR_ARG, "public mask longer than the padded private mask (%ld > %ld)", n_pub_mask, M);
    VG_TRY(ensure(c, pc->res, 66 * sizeof(fe)));
    VG_TRY(encode_public(pc, pub, pub_mask, n_pub_mask, pc->F(pc->res), h_mask + M));

    // FRI folds, level by level (fri.cpp:321-340, 367-379)
    const int logS = ilog2l(S);
    const fe *ti_lo, *ti_hi;
    VG_TRY(vg_twiddles(c, vg::fe_inv(root_of(logS)), logS, &ti_lo, &ti_hi));
    if ((int)pc->levels.size() < nlevels) pc->levels.resize(nlevels);
    for (int t = 0; t < nlevels; ++t) {
        const long n = S >> t;
        PcLevel &L = pc->levels[t];
        L.n = n >> 1;
        VG_TRY(ensure(c, L.cw, 65 * L.n * sizeof(fe)));
        VG_TRY(ensure(c, L.tree, L.n * 32));
        const fe *in = t == 0 ? pc->F(pc->vo) : pc->F(pc->levels[t - 1].cw);
        const long total = 65 * L.n;
        {
            ProfScope ps(c, KF_FRI_FOLD, 16.0 * 65.0 * (double)n * 1.5);
            k_fri_fold<<<std::min<unsigned>(grid_for(total, 256), 148u * 16u), 256, 0, c->stream>>>(
                in, n, t, vg::fe_make(fri_r[t].real, fri_r[t].img), ti_lo, ti_hi, pc->F(L.cw));
        }
        VG_LAUNCHED(c);
    }
    pc->nlevels = nlevels;

    // every leaf chain, then every Merkle tree, batched (fri.cpp:394-420, merkle_tree.cpp)
    VG_TRY(ensure(c, pc->tree_l, (size_t)S * 32));
    VG_TRY(ensure(c, pc->tree_h, (size_t)S * 32));
    VG_TRY(ensure(c, pc->roots, ndesc * 32));
    struct Set { const fe *cw; long n; uint64_t *tree; };
    std::vector<Set> sets;
    sets.push_back({pc->F(pc->l_eval), S, pc->U(pc->tree_l)});
    sets.push_back({pc->F(pc->h_eval), S, pc->U(pc->tree_h)});
    for (int t = 0; t < nlevels; ++t) sets.push_back({pc->F(pc->levels[t].cw), pc->levels[t].n, pc->U(pc->levels[t].tree)});
    for (size_t b = 0; b < sets.size(); b += MAX_HASH_JOBS) {
        ChainJobs cj{};
        long total = 0;
        for (size_t k = b; k < sets.size() && k < b + MAX_HASH_JOBS; ++k) {
            const long nleaves = sets[k].n >> 1;
            cj.j[cj.count++] = {sets[k].cw, sets[k].n, sets[k].tree + 4 * nleaves, total};
            total += nleaves;
        }
        cj.total = total;
        VG_TRY(vg_leaf_chains(c, cj));
    }
    for (size_t b = 0; b < sets.size(); b += MAX_HASH_JOBS) {
        TreeJobs tj{};
        for (size_t k = b; k < sets.size() && k < b + MAX_HASH_JOBS; ++k) tj.t[tj.count++] = {sets[k].tree, sets[k].n >> 1};
        VG_TRY(vg_merkle_trees(c, tj, pc->U(pc->roots) + 4 * b));
    }

    // query answers (fri.cpp:148-289), positions checked as in vg_pc_query_batch
    std::vector<QueryDesc> dsc;
    query_descs(pc, dsc);
    for (int q = 0; q < nq; ++q) {
        if (which[q] < 0 || which[q] >= (int)dsc.size()) return vg_fail(VG_ERR_ARG, "query %d: no codeword set %d", q, which[q]);
        if (pos[q] < 0) return vg_fail(VG_ERR_ARG, "query %d: negative position", q);
        if (which[q] < 2 && pos[q] >= S / 2) return vg_fail(VG_ERR_ARG, "query %d: position out of range", q);
    }
    const size_t vals_b = (size_t)nq * 130 * sizeof(fe), paths_b = (size_t)nq * 32 * 32;
    if (nq) {
        VG_TRY(ensure(c, pc->qdesc, in_b));
        VG_TRY(ensure(c, pc->qio, vals_b + paths_b));
        char *hb = (char *)h_in;
        memcpy(hb, dsc.data(), desc_b);
        memcpy(hb + off_pos, pos, pos_b);
        memcpy(hb + off_which, which, which_b);
        char *db = (char *)pc->qdesc.p;
        VG_CHECK_CUDA(cudaMemcpyAsync(db, hb, in_b, cudaMemcpyHostToDevice, c->stream));
        k_gather_batch<<<nq, 96, 0, c->stream>>>((const QueryDesc *)db, (const int *)(db + off_which),
                                                 (const long *)(db + off_pos), (fe *)pc->qio.p,
                                                 (uint64_t *)((char *)pc->qio.p + vals_b));
        VG_LAUNCHED(c);
    }

    // results to pinned memory
    VG_CHECK_CUDA(cudaMemcpyAsync(h_res, pc->res.p, 66 * sizeof(fe), cudaMemcpyDeviceToHost, c->stream));
    VG_CHECK_CUDA(cudaMemcpyAsync(h_roots, pc->roots.p, ndesc * 32, cudaMemcpyDeviceToHost, c->stream));
    const fe *fin = nlevels ? pc->F(pc->levels[nlevels - 1].cw) : pc->F(pc->vo);
    VG_CHECK_CUDA(cudaMemcpyAsync(h_final, fin, e_final * sizeof(fe), cudaMemcpyDeviceToHost, c->stream));
    if (nq) VG_CHECK_CUDA(cudaMemcpyAsync(h_qv, pc->qio.p, vals_b + paths_b, cudaMemcpyDeviceToHost, c->stream));
    out->inner = (const vg_fe *)h_res;
    out->all_sum = (const vg_fe *)(h_res + 1);
    out->roots = (const vg_digest *)h_roots;
    out->final_cw = (const vg_fe *)h_final;
    out->n_final = n_final;
    out->qvals = (const vg_fe *)h_qv;
    out->qpaths = (const vg_digest *)h_qp;
    return VG_OK;
}

extern "C" int vg_pc_commit_all(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *pri_mask, long n_pri_mask,
                                const vg_fe *pub, const vg_fe *pub_mask, long n_pub_mask, const vg_fe *fri_r,
                                int nlevels, int nq, const int *which, const long *pos, vg_digest *roots,
                                vg_fe *all_sum, vg_fe *inner, vg_fe *final_cw, vg_fe *qvals, vg_digest *qpaths)
{
    if (!roots || !all_sum || !inner || !final_cw || (nq && (!qvals || !qpaths)))
        return vg_fail(VG_ERR_ARG, "vg_pc_commit_all: null output");
    vg_pc_results r{};
    VG_TRY(vg_pc_prove_deferred(pc, priv, log_len, pri_mask, n_pri_mask, pub, pub_mask, n_pub_mask, fri_r, nlevels, nq,
                                which, pos, &r));
    VG_CHECK_CUDA(cudaStreamSynchronize(pc->ctx->stream));
    memcpy(roots, r.roots, (size_t)(2 + nlevels) * sizeof(vg_digest));
    memcpy(all_sum, r.all_sum, 65 * sizeof(vg_fe));
    *inner = *r.inner;
    memcpy(final_cw, r.final_cw, (size_t)65 * r.n_final * sizeof(vg_fe));
    if (nq) {
        memcpy(qvals, r.qvals, (size_t)nq * 130 * sizeof(vg_fe));
        memcpy(qpaths, r.qpaths, (size_t)nq * 32 * sizeof(vg_digest));
    }
    return VG_OK;
}
