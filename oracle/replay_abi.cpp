// The subset of the C ABI (include/virgo_b200.h) that the drop-in prover
// classes call, answered from a proof file written by vg_session_write_proof
// instead of a GPU.  TEST INFRASTRUCTURE ONLY: linked with the drop-in host
// sources (virgo_b200/host/src) into libvirgo_replay.so, it lets the
// reference verifier, compiled unchanged, check a serialized GPU proof in a
// process of its own with no GPU (oracle/verify_file_main.cpp).
//
// Every device result comes from the file in the order the prover consumes
// it: V_res and the sumcheck rounds from the GKR records, the commitment
// roots, all_sum, <l, q>, the FRI level roots (each FRI challenge the
// verifier draws must equal the one the proof was folded with), the final
// codeword and the query answers (each query's oracle and position must
// equal the proof's).  Everything the verifier computes itself stays on the
// host: the reference's own checks decide Pass or Fail.  A record or query
// requested beyond the file, or a mismatch of the circuit's shape, the FRI
// challenges or the query plan, is an error (the drop-in aborts with it).
#include "virgo_b200.h"
#include "infrastructure/my_hhash.h"
#include "../virgo_b200/host/src/device.h"
#include "../virgo_b200/host/include/infrastructure/constants.h"
#include "virgo_oracle.h"
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>

namespace {

struct ProofFile {
    bool open = false;
    unsigned seed = 0;
    std::vector<int> bl;
    int nrec = 0, levels = 0, nq = 0, proof_size = 0;
    long n_final = 0;
    std::vector<vg_fe> rec, all_sum, fri_r, final_cw, qvals;
    vg_fe inner{};
    std::vector<vg_digest> roots, qpaths;
    std::vector<int> which;
    std::vector<long> pos;
    // consumption
    int rec_i = 0, fri_i = 0, q_i = 0;
    int log_len = 0;
};

ProofFile g_pf;
std::string g_err;
std::set<const void *> g_dev;   // "device" buffers handed out by vg_dev_alloc
vg_fe g_layer_dummy[2];          // stands in for the layer values the verifier only passes back

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

template <class T>
bool rd(FILE *f, T *p, size_t n)
{
    return n == 0 || fread(p, sizeof(T), n, f) == n;
}

}  // namespace

extern "C" {

// Opens the proof file; *seed receives the seed the proof was made with.
int vg_replay_open(const char *path, unsigned *seed)
{
    FILE *f = fopen(path, "rb");
    if (!f) return fail(VG_ERR_ARG, "cannot open %s", path);
    ProofFile &p = g_pf;
    p = ProofFile();
    char magic[4];
    uint32_t version = 0, sd = 0;
    int32_t depth = 0;
    bool ok = rd(f, magic, 4) && memcmp(magic, "VGPF", 4) == 0 && rd(f, &version, 1) && version == 1 &&
              rd(f, &sd, 1) && rd(f, &depth, 1) && depth > 0 && depth < 1000000;
    if (ok) {
        std::vector<int32_t> bl(depth);
        ok = rd(f, bl.data(), depth);
        p.bl.assign(bl.begin(), bl.end());
    }
    int64_t n_final = 0;
    ok = ok && rd(f, &p.nrec, 1) && rd(f, &p.levels, 1) && rd(f, &p.nq, 1) && rd(f, &n_final, 1) &&
         rd(f, &p.proof_size, 1) && p.nrec >= 0 && p.levels >= 0 && p.nq >= 0 && n_final > 0 && n_final < (1L << 30);
    if (ok) {
        p.n_final = n_final;
        p.rec.resize((size_t)p.nrec * 9);
        p.roots.resize(2 + p.levels);
        p.all_sum.resize(slice_number + 1);
        p.fri_r.resize(p.levels);
        p.final_cw.resize((size_t)(slice_number + 1) * p.n_final);
        p.which.resize(p.nq);
        p.pos.resize(p.nq);
        p.qvals.resize((size_t)p.nq * 130);
        p.qpaths.resize((size_t)p.nq * 32);
        std::vector<int32_t> w(p.nq);
        std::vector<int64_t> ps(p.nq);
        ok = rd(f, p.rec.data(), p.rec.size()) && rd(f, p.roots.data(), p.roots.size()) &&
             rd(f, p.all_sum.data(), p.all_sum.size()) && rd(f, &p.inner, 1) && rd(f, p.fri_r.data(), p.fri_r.size()) &&
             rd(f, p.final_cw.data(), p.final_cw.size()) && rd(f, w.data(), p.nq) && rd(f, ps.data(), p.nq) &&
             rd(f, p.qvals.data(), p.qvals.size()) && rd(f, p.qpaths.data(), p.qpaths.size());
        for (int q = 0; q < p.nq; ++q) {
            p.which[q] = w[q];
            p.pos[q] = (long)ps[q];
        }
        char extra;
        ok = ok && fread(&extra, 1, 1, f) == 0;   // nothing after the last section
    }
    fclose(f);
    if (!ok) return fail(VG_ERR_ARG, "%s is not a complete VGPF version 1 proof file", path);
    p.seed = sd;
    p.open = true;
    if (seed) *seed = sd;
    return VG_OK;
}

// After the verifier: every record and query of the file must have been consumed.
int vg_replay_close(void)
{
    ProofFile &p = g_pf;
    if (!p.open) return fail(VG_ERR_STATE, "no proof file open");
    p.open = false;
    if (p.rec_i != p.nrec || p.q_i != p.nq || p.fri_i != p.levels)
        return fail(VG_ERR_STATE, "the verifier used %d of %d records, %d of %d queries, %d of %d FRI levels", p.rec_i,
                    p.nrec, p.q_i, p.nq, p.fri_i, p.levels);
    return VG_OK;
}

int vg_replay_proof_size(void) { return g_pf.proof_size; }

const char *vg_last_error(void) { return g_err.c_str(); }

// ---- contexts and memory: host stand-ins ----
int vg_ctx_create(int device, vg_ctx **out)
{
    (void)device;
    static char dummy;
    *out = (vg_ctx *)&dummy;
    return VG_OK;
}
int vg_ctx_set_hash(vg_ctx *ctx, int kind)
{
    (void)ctx;
    return kind == 0 ? VG_OK : fail(VG_ERR_ARG, "the replay answers SHA3-256 proofs only");
}
int vg_ctx_sync(vg_ctx *ctx)
{
    (void)ctx;
    return VG_OK;
}
int vg_dev_alloc(vg_ctx *ctx, size_t bytes, void **dev)
{
    (void)ctx;
    *dev = malloc(bytes ? bytes : 1);
    if (!*dev) return fail(VG_ERR_OOM, "host allocation of %zu bytes", bytes);
    g_dev.insert(*dev);
    return VG_OK;
}
int vg_dev_free(vg_ctx *ctx, void *dev)
{
    (void)ctx;
    g_dev.erase(dev);
    free(dev);
    return VG_OK;
}
int vg_h2d(vg_ctx *ctx, void *dev, const void *host, size_t bytes)
{
    (void)ctx;
    memcpy(dev, host, bytes);
    return VG_OK;
}
int vg_d2h(vg_ctx *ctx, void *host, const void *dev, size_t bytes)
{
    (void)ctx;
    memcpy(host, dev, bytes);
    return VG_OK;
}

// The verifier's own transforms (the public mask's and the public array's
// inverse FFTs), through the oracle's FFT: n = 2^log_n, one batch item.
int vg_ntt(vg_ctx *ctx, const vg_fe *in, long in_len, long in_batch_stride, vg_fe *out, int log_n, long out_batch_stride,
           int batch, vg_fe root, int scale_inv_n)
{
    (void)ctx;
    (void)in_batch_stride;
    (void)out_batch_stride;
    if (batch != 1) return fail(VG_ERR_ARG, "vg_ntt: one transform at a time in the replay");
    const long n = 1L << log_n;
    std::vector<vo_fe> co(n), res(n);
    memcpy(co.data(), in, (size_t)in_len * sizeof(vg_fe));
    vo_fe r;
    memcpy(&r, &root, sizeof r);
    vo_fft(co.data(), in_len, n, &r, res.data());
    if (scale_inv_n) {
        vo_fe nn = {0, (uint64_t)n}, inv;   // {img, real}
        vo_fe_inv(&nn, &inv);
        vo_fe_mul_arr(res.data(), std::vector<vo_fe>(n, inv).data(), res.data(), n);
    }
    memcpy(out, res.data(), (size_t)n * sizeof(vg_fe));
    return VG_OK;
}

int vg_merkle_tree(vg_ctx *ctx, const vg_digest *leaves, long n, vg_digest *tree)
{
    (void)ctx;
    (void)leaves;
    (void)n;
    (void)tree;
    return fail(VG_ERR_STATE, "vg_merkle_tree: the verifier builds no tree");
}
int vg_mle_eval(vg_ctx *ctx, const vg_fe *vals, long n, const vg_fe *r, int log_n, vg_fe *out)
{
    (void)ctx;
    (void)vals;
    (void)n;
    (void)r;
    (void)log_n;
    (void)out;
    return fail(VG_ERR_STATE, "vg_mle_eval: not part of the recorded proof");
}

// ---- GKR: the recorded device results ----
int vg_circuit_upload(vg_ctx *ctx, int depth, const int *bit_length, const uint8_t *const *ty, const int64_t *const *u,
                      const int64_t *const *v, vg_circuit **out)
{
    (void)ctx;
    (void)ty;
    (void)u;
    (void)v;
    const ProofFile &p = g_pf;
    if (!p.open) return fail(VG_ERR_STATE, "no proof file open");
    if (depth != (int)p.bl.size()) return fail(VG_ERR_ARG, "circuit depth %d, proof made for %zu", depth, p.bl.size());
    for (int i = 0; i < depth; ++i)
        if (bit_length[i] != p.bl[i])
            return fail(VG_ERR_ARG, "layer %d has 2^%d gates, the proof's 2^%d", i, bit_length[i], p.bl[i]);
    static char dummy;
    *out = (vg_circuit *)&dummy;
    return VG_OK;
}
int vg_circuit_destroy(vg_circuit *c)
{
    (void)c;
    return VG_OK;
}
int vg_gkr_create(vg_ctx *ctx, const vg_circuit *c, vg_gkr **out)
{
    (void)ctx;
    (void)c;
    static char dummy;
    *out = (vg_gkr *)&dummy;
    return VG_OK;
}
int vg_gkr_destroy(vg_gkr *g)
{
    (void)g;
    return VG_OK;
}
int vg_gkr_rebind(vg_gkr *g, const vg_circuit *c)
{
    (void)g;
    (void)c;
    return VG_OK;
}
int vg_gkr_evaluate(vg_gkr *g)
{
    (void)g;
    return VG_OK;
}
int vg_gkr_layer_values(vg_gkr *g, int layer, const vg_fe **dev_values)
{
    (void)g;
    (void)layer;
    *dev_values = g_layer_dummy;
    return VG_OK;
}
int vg_gkr_v_res(vg_gkr *g, const vg_fe *r, int r_len, vg_fe *out)
{
    (void)g;
    (void)r;
    (void)r_len;
    ProofFile &p = g_pf;
    if (p.rec_i >= p.nrec) return fail(VG_ERR_STATE, "V_res: the proof has no record left");
    *out = p.rec[9 * (size_t)p.rec_i++];
    return VG_OK;
}
int vg_gkr_phase1_init(vg_gkr *g, int layer, const vg_fe *r0, const vg_fe *r1, int length_g, vg_fe alpha, vg_fe beta)
{
    (void)g;
    (void)layer;
    (void)r0;
    (void)r1;
    (void)length_g;
    (void)alpha;
    (void)beta;
    return VG_OK;
}
int vg_gkr_phase2_init(vg_gkr *g, const vg_fe *r_u, int length_u, vg_fe v_u)
{
    (void)g;
    (void)r_u;
    (void)length_u;
    (void)v_u;
    return VG_OK;
}
int vg_gkr_round(vg_gkr *g, vg_fe previous_random, int current_bit, vg_fe *out3, vg_fe *last6)
{
    (void)g;
    (void)previous_random;
    (void)current_bit;
    ProofFile &p = g_pf;
    if (p.rec_i >= p.nrec) return fail(VG_ERR_STATE, "sumcheck round: the proof has no record left");
    const vg_fe *r = &p.rec[9 * (size_t)p.rec_i++];
    for (int k = 0; k < 3; ++k) out3[k] = r[k];
    if (last6)
        for (int k = 0; k < 6; ++k) last6[k] = r[3 + k];
    return VG_OK;
}

// ---- commitment: the recorded roots, sums, codeword and answers ----
int vg_pc_create(vg_ctx *ctx, vg_pc **out)
{
    (void)ctx;
    static char dummy;
    *out = (vg_pc *)&dummy;
    return VG_OK;
}
int vg_pc_encode_private(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *mask, long n_mask, long *mask_len)
{
    (void)pc;
    (void)priv;
    (void)mask;
    const long S = 1L << (log_len - 1);
    long gap = 1;
    while (gap * 2 <= S / n_mask) gap *= 2;   // mask_position_gap, poly_commit.h:56-64
    *mask_len = S / gap;
    g_pf.log_len = log_len;
    return VG_OK;
}
int vg_pc_init_commit(vg_pc *pc, int oracle, vg_digest *root)
{
    (void)pc;
    if (oracle < 0 || oracle > 1) return fail(VG_ERR_ARG, "oracle %d", oracle);
    *root = g_pf.roots[oracle];
    return VG_OK;
}
int vg_pc_encode_public(vg_pc *pc, const vg_fe *pub, const vg_fe *pub_mask, long n_mask, vg_fe *all_sum, vg_fe *inner)
{
    (void)pc;
    (void)pub;
    (void)pub_mask;
    (void)n_mask;
    for (int i = 0; i <= slice_number; ++i) all_sum[i] = g_pf.all_sum[i];
    *inner = g_pf.inner;
    return VG_OK;
}
int vg_pc_fri_step(vg_pc *pc, vg_fe r, vg_digest *root)
{
    (void)pc;
    ProofFile &p = g_pf;
    if (p.fri_i >= p.levels) return fail(VG_ERR_STATE, "FRI: the proof has %d levels", p.levels);
    const vg_fe &want = p.fri_r[p.fri_i];
    if (want.real != r.real || want.img != r.img)
        return fail(VG_ERR_STATE, "FRI level %d: the verifier's challenge differs from the proof's", p.fri_i);
    *root = p.roots[2 + p.fri_i++];
    return VG_OK;
}
int vg_pc_fri_final(vg_pc *pc, vg_fe *data, vg_fe *mask, long *n)
{
    (void)pc;
    const ProofFile &p = g_pf;
    const long nf = p.n_final, h = nf / 2;
    *n = nf;
    if (!data || !mask) return VG_OK;
    const vg_fe *b = p.final_cw.data();
    for (long j = 0; j < h; ++j) {   // slice-major to the interleaved layout
        for (int s = 0; s < slice_number; ++s) {
            data[(j << 7) | (s << 1) | 0] = b[s * nf + j];
            data[(j << 7) | (s << 1) | 1] = b[s * nf + j + h];
        }
        mask[2 * j] = b[slice_number * nf + j];
        mask[2 * j + 1] = b[slice_number * nf + j + h];
    }
    return VG_OK;
}
int vg_pc_query_init(vg_pc *pc, long pow0, int oracle, vg_fe *values, vg_digest *path)
{
    (void)pc;
    ProofFile &p = g_pf;
    if (p.q_i >= p.nq) return fail(VG_ERR_STATE, "query: the proof has %d answers", p.nq);
    const int q = p.q_i++;
    if (p.which[q] != oracle || p.pos[q] != pow0)
        return fail(VG_ERR_STATE, "query %d: the verifier asks oracle %d at %ld, the proof answers %d at %ld", q, oracle,
                    pow0, p.which[q], p.pos[q]);
    memcpy(values, &p.qvals[(size_t)q * 130], 130 * sizeof(vg_fe));
    const int depth = p.log_len - 2;
    memcpy(path, &p.qpaths[(size_t)q * 32], (size_t)(depth + 1) * sizeof(vg_digest));
    return VG_OK;
}
int vg_pc_query_step(vg_pc *pc, int lvl, long pow, vg_fe *values, vg_digest *path, int *path_len)
{
    (void)pc;
    ProofFile &p = g_pf;
    if (p.q_i >= p.nq) return fail(VG_ERR_STATE, "query: the proof has %d answers", p.nq);
    const int q = p.q_i++;
    const int depth = p.log_len - lvl - 3;   // log2 of the level's leaf count
    const long half = 1L << depth;
    if (p.which[q] != 2 + lvl || (p.pos[q] % half) != (pow % half))
        return fail(VG_ERR_STATE, "query %d: the verifier asks level %d at %ld, the proof answers set %d at %ld", q, lvl,
                    pow, p.which[q], p.pos[q]);
    memcpy(values, &p.qvals[(size_t)q * 130], 130 * sizeof(vg_fe));
    memcpy(path, &p.qpaths[(size_t)q * 32], (size_t)(depth + 1) * sizeof(vg_digest));
    *path_len = depth + 1;
    return VG_OK;
}

}  // extern "C"

// (an internal entry point of the library, C++ linkage; the drop-in classes
// call it only in their deferred launch mode, never in the replay)
int vg_gkr_phase2_init_deferred(vg_gkr *g, const vg_fe *r_u, int length_u, vg_fe r_last, vg_fe addend)
{
    (void)g;
    (void)r_u;
    (void)length_u;
    (void)r_last;
    (void)addend;
    return fail(VG_ERR_STATE, "deferred phase 2 init in the replay");
}

// the drop-in classes' process context (virgo_b200/host/src/device.h)
namespace virgo
{
vg_ctx *ctx()
{
    vg_ctx *c;
    vg_ctx_create(0, &c);
    return c;
}
vg_pc *pc()
{
    vg_pc *p;
    vg_pc_create(nullptr, &p);
    return p;
}
void check(int rc, const char *what)
{
    if (rc != VG_OK) {
        fprintf(stderr, "virgo_b200 replay: %s failed (%d): %s\n", what, rc, vg_last_error());
        abort();
    }
}
bool is_device_ptr(const void *p) { return g_dev.count(p) != 0; }
}  // namespace virgo
