/* virgo_b200: B200 (sm_100a) kernels for the Virgo prover hot path, behind a
 * plain C ABI.
 *
 * The drop-in C++ classes (zk_prover, poly_commit::poly_commit_prover, the
 * fri:: functions, fast_fourier_transform, create_tree, my_hhash; headers under
 * virgo_b200/host/include) are thin wrappers over these entry points; a caller
 * in any language can bind them directly (ctypes, cgo, JNI, a C++ link).
 *
 * Conventions
 *  - Every entry point returns VG_OK (0) or a VG_ERR_* code; vg_last_error()
 *    gives a message for the calling thread.
 *  - vg_fe is the reference's prime_field::field_element layout: {img, real},
 *    two uint64 in [0, 2^61 - 1).  vg_digest is __hhash_digest (32 bytes).
 *  - "dev" pointers are device memory (vg_dev_alloc); "host" pointers are
 *    ordinary host memory; "any" pointers may be either (detected per call).
 *  - All work of one context is ordered on that context's CUDA stream.
 *    Entry points that return values to host memory synchronise it.
 */
#ifndef VIRGO_B200_H
#define VIRGO_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { uint64_t img, real; } vg_fe;
typedef struct { uint8_t bytes[32]; } vg_digest;

enum {
    VG_OK = 0,
    VG_ERR_CUDA = 1,      /* a CUDA call failed (message has the CUDA error) */
    VG_ERR_ARG = 2,       /* invalid argument (sizes, null pointers, ranges)  */
    VG_ERR_OOM = 3,       /* device allocation failed                         */
    VG_ERR_NO_DEVICE = 4, /* no CUDA device / extension not usable            */
    VG_ERR_STATE = 5      /* call out of protocol order                        */
};

enum { VG_HASH_SHA3_256 = 0, VG_HASH_SHA256 = 1 };

typedef struct vg_ctx vg_ctx;          /* device, stream, scratch, twiddle cache */
typedef struct vg_circuit vg_circuit;  /* device-resident layered circuit        */
typedef struct vg_gkr vg_gkr;          /* GKR prover state for one circuit       */
typedef struct vg_pc vg_pc;            /* polynomial commitment + FRI state      */

/* ---------------------------------------------------------------- context */
const char *vg_last_error(void);
/* Creates a context on `device` with its own stream.  Replaces the implicit
 * global state of the reference (prime_field::init, prime_field.cpp:19-24;
 * init_scratch_pad, RS_polynomial.cpp:8-16). */
int vg_ctx_create(int device, vg_ctx **out);
int vg_ctx_destroy(vg_ctx *ctx);
/* Hash used for every Merkle commitment of this context.  The reference
 * chooses it at build time (#define USESHA3, my_hhash.h:10); default SHA3-256. */
int vg_ctx_set_hash(vg_ctx *ctx, int kind);
int vg_ctx_get_hash(vg_ctx *ctx, int *kind);
int vg_ctx_sync(vg_ctx *ctx);
int vg_ctx_device(vg_ctx *ctx, int *device);
/* Number of kernels this context has launched since creation. */
int vg_ctx_launch_count(vg_ctx *ctx, long long *count);

/* Per-launch profiler.  While enabled, every kernel launch of the context is
 * bracketed by CUDA events on its stream (no extra synchronisation);
 * vg_ctx_profile_read returns, for one kernel family, the launches, their
 * summed device time and their summed algorithmic bytes (bytes the kernel
 * must move by its definition, not measured traffic).  Families: 0 NTT pass,
 * 1 leaf hash chain, 2 Merkle level, 3 FRI fold + leaf chain, 4 virtual
 * oracle, 5 layer evaluation, 6 phase-1 scatter, 7 phase-2 scatter,
 * 8 accumulator finalise, 9 sumcheck round, 10 partial-sum reduction,
 * 11 other.  Enabling resets the counters. */
int vg_ctx_profile(vg_ctx *ctx, int enable);
int vg_ctx_profile_read(vg_ctx *ctx, int family, long long *launches, double *ms, double *bytes);
/* The profiled launches in launch order (family, device ms, algorithmic
 * bytes), at most max of them; *n receives how many were recorded. */
int vg_ctx_profile_trace(vg_ctx *ctx, int *family, double *ms, double *bytes, long max, long *n);
/* Device time between two points of the context's stream. */
int vg_timer_start(vg_ctx *ctx, void **timer);
int vg_timer_stop(vg_ctx *ctx, void *timer, double *ms);
/* Device time from the start point to the end of the work queued so far on
 * every listed context (the latest of them); consumes the timer. */
int vg_timer_stop_multi(vg_ctx *const *ctxs, int n, void *timer, double *ms);

/* ----------------------------------------------------------- device memory */
int vg_dev_alloc(vg_ctx *ctx, size_t bytes, void **dev);
int vg_dev_free(vg_ctx *ctx, void *dev);
int vg_h2d(vg_ctx *ctx, void *dev, const void *host, size_t bytes);
int vg_d2h(vg_ctx *ctx, void *host, const void *dev, size_t bytes);

/* ------------------------------------------------------------------- field */
/* Elementwise c = a op b on n elements, op 0 = add, 1 = sub, 2 = mul
 * (prime_field::field_element operators, prime_field.h:114-165). dev. */
int vg_fe_binop(vg_ctx *ctx, int op, const vg_fe *a, const vg_fe *b, vg_fe *c, long n);

/* --------------------------------------------------------------------- NTT */
/* Batched transform: for each of `batch` arrays, out = the evaluations of the
 * polynomial with coefficients in[0..in_len) (zero beyond) at root^0 ..
 * root^(n-1), n = 2^log_n, natural order; root must have order n.  With
 * scale_inv_n != 0 the outputs are multiplied by n^-1.  in_len <= n.
 * Replaces fast_fourier_transform (RS_polynomial.h:10, RS_polynomial.cpp:27)
 * and, with the inverse root and scale_inv_n, inverse_fast_fourier_transform
 * (RS_polynomial.h:16, RS_polynomial.cpp:169) for coef_len == order.
 * in/out dev; in and out may not overlap unless in == out and in_len == n. */
int vg_ntt(vg_ctx *ctx, const vg_fe *in, long in_len, long in_batch_stride,
           vg_fe *out, int log_n, long out_batch_stride, int batch,
           vg_fe root, int scale_inv_n);

/* ------------------------------------------------------------------- hash */
/* n independent hashes of 64-byte messages (my_hhash, my_hhash.h:28). dev. */
int vg_hash64(vg_ctx *ctx, const void *msgs, void *digests, long n);
/* Merkle tree over n leaves, tree = 2 * next_pow2(n) digests, tree[1] = root,
 * leaves stored raw, padding leaves H(0^64), nodes H(left || right)
 * (merkle_tree::merkle_tree_prover::create_tree, merkle_tree.h:12,
 * merkle_tree.cpp:4-57). dev. */
int vg_merkle_tree(vg_ctx *ctx, const vg_digest *leaves, long n, vg_digest *tree);
/* Leaf hash chains of a slice-major codeword set (n_slices slices of length
 * n): leaf k < n/2 is h = H((c[s][k], c[s][k+n/2]) || h) over s from h = 0
 * (the leaf loops of fri::request_init_commit, fri.cpp:97-126, and
 * fri::commit_phase_step, fri.cpp:394-420). dev. */
int vg_leaf_chain(vg_ctx *ctx, const vg_fe *codewords, int n_slices, long n, vg_digest *leaves);

/* --------------------------------------------------------------- circuits */
/* Uploads a layered circuit: layer i has 2^bit_length[i] gates given as
 * ty[i][g] (gate type 0..13), u[i][g], v[i][g] (host arrays, the fields of
 * `gate`, circuit_fast_track.h:6-14).  Layer 0 is the input layer (its u is
 * the input value, read through int as zk_prover::evaluate does,
 * zk_prover.cpp:57-66).  Mirrors layered_circuit after
 * zk_verifier::read_circuit (zk_verifier.cpp:15-217). */
int vg_circuit_upload(vg_ctx *ctx, int depth, const int *bit_length,
                      const uint8_t *const *ty, const int64_t *const *u, const int64_t *const *v,
                      vg_circuit **out);
/* Builds the prover's circuit on the device from file-level layers, as
 * zk_verifier::read_circuit does on the host (zk_verifier.cpp:24-191): the
 * input layer (u = values, int64) becomes layer 0 padded to 2^17 gates (2^15
 * for at most three file layers) plus a relay layer, wires are checked
 * against the previous layer and narrowed to 32 bits, gates above a layer's
 * count become dummies.  index_bytes is the width of u and v of the other
 * layers in host memory: 8 (int64, as in the text format) or 4 (uint32).
 * *inout is reused (its buffers grown as needed) when non-NULL.
 * bit_lengths (host, d + 1 entries, may be NULL) receives the layer widths. */
int vg_circuit_build(vg_ctx *ctx, int d, const long *n, const uint8_t *const *ty, const void *const *u,
                     const void *const *v, int index_bytes, vg_circuit **inout, int *bit_lengths);
int vg_circuit_destroy(vg_circuit *c);
int vg_circuit_depth(const vg_circuit *c, int *depth);
/* The verifier's wiring predicates of prover layer `layer` (>= 1) at
 * (r_0, r_1; r_u, r_v): zk_verifier::predicates, zk_verifier.cpp:219-606,
 * with the beta tables of zk_verifier::beta_init (alpha- and beta-weighted
 * eq(r_0, g), eq(r_1, g); eq(r_u, .), eq(r_v, .)).  out[t], t < 14, is the
 * sum over the layer's gates of type t; layer 1 (the reader's relay layer)
 * gives zeros as in the reference.  r_0/r_1 have bl(layer) entries, r_u/r_v
 * bl(layer - 1); all host.  Layers are taken as not data-parallel. */
int vg_circuit_predicates(vg_ctx *ctx, const vg_circuit *c, int layer, const vg_fe *r_0, const vg_fe *r_1,
                          const vg_fe *r_u, const vg_fe *r_v, vg_fe alpha, vg_fe beta, vg_fe *out);

/* ------------------------------------------------------------------- GKR */
/* State for proving one circuit; buffers are sized for its widest layer
 * (zk_prover::init_array, zk_prover.cpp:337-350). */
int vg_gkr_create(vg_ctx *ctx, const vg_circuit *c, vg_gkr **out);
int vg_gkr_destroy(vg_gkr *g);
/* Points an existing GKR state at another circuit on the same context; its
 * device tables are reused and only grow when the circuit needs more (no
 * reference counterpart: the reference allocates per zk_prover). */
int vg_gkr_rebind(vg_gkr *g, const vg_circuit *c);
/* All layer values (zk_prover::evaluate, zk_prover.cpp:54-157). */
int vg_gkr_evaluate(vg_gkr *g);
/* Device pointer to the 2^bit_length values of a layer (after evaluate). */
int vg_gkr_layer_values(vg_gkr *g, int layer, const vg_fe **dev_values);
/* Multilinear extension of the output layer at r (r_len = its bit length)
 * (zk_prover::V_res, zk_prover.cpp:30-52).  r host, out host. */
int vg_gkr_v_res(vg_gkr *g, const vg_fe *r, int r_len, vg_fe *out);
/* Multilinear extension of vals (any, 2^log_n entries) at r (host, log_n
 * entries; bit b of the index pairs with r[b]), the fold of V_res
 * (zk_prover.cpp:37-44).  out host. */
int vg_mle_eval(vg_ctx *ctx, const vg_fe *vals, long n, const vg_fe *r, int log_n, vg_fe *out);
/* vg_mle_eval for callers that cannot allocate device memory (a host whose
 * pool already holds the GPU, a latency-critical path that must not take
 * cudaFree's device-wide synchronisation, a fixed memory budget).  No
 * counterpart in the reference.  It allocates nothing: its scratch (eq tables,
 * block partials) is one file-scope device array of 268,160 bytes that every
 * GPU loading this library keeps until exit.  vals device (n >= 2^log_n), r and
 * out host; log_n in [0, 26], anything else is rejected with VG_ERR_ARG.  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress,
 * that device current) and caches it: make it before any stream capture, and
 * do not use the entry point on a device again after cudaDeviceReset of it.
 * All calls on a device share that device's array, which keeps the last
 * call's contents (each call writes what it reads); calls on one device that
 * overlap on the GPU race.  Runs on the legacy default stream, which does NOT
 * wait for non-blocking streams such as this library's context streams:
 * synchronise the stream that produced vals first (vg_ctx_sync).  Returns
 * after *out is written. */
int vg_mle_eval_noalloc(const vg_fe *vals, long n, const vg_fe *r, int log_n, vg_fe *out);
/* Phase-1 bookkeeping of layer `layer` (zk_prover::sumcheck_phase1_init,
 * zk_prover.cpp:375-592): beta_g = alpha*eq(r0,g) + beta*eq(r1,g) over
 * length_g bits, then the gate scatter into add_mult_sum / addV_array by u.
 * r0, r1 host (length_g entries). */
int vg_gkr_phase1_init(vg_gkr *g, int layer, const vg_fe *r0, const vg_fe *r1, int length_g,
                       vg_fe alpha, vg_fe beta);
/* Phase-2 bookkeeping (zk_prover::sumcheck_phase2_init, zk_prover.cpp:789-972):
 * scatter by v with beta_g * eq(r_u, u) and the claimed value v_u.
 * r_u host (length_u entries). */
int vg_gkr_phase2_init(vg_gkr *g, const vg_fe *r_u, int length_u, vg_fe v_u);
/* One sumcheck round over the three bookkeeping tables (the array loop of
 * sumcheck_phase{1,2}_update[lastbit], zk_prover.cpp:600-633, 684-717,
 * 992-1025, 1075-1108): folds the tables with previous_random (unless
 * current_bit == 0), returns the round sums (a, b, c) before the mask terms
 * in out3, and, when two entries remain, the folded tables in last6 as
 * {V[0], V[1], addV[0], addV[1], add_mult[0], add_mult[1]} (may be NULL).
 * out3, last6 host. */
int vg_gkr_round(vg_gkr *g, vg_fe previous_random, int current_bit, vg_fe *out3, vg_fe *last6);

/* ------------------------------------------------ polynomial commitment */
int vg_pc_create(vg_ctx *ctx, vg_pc **out);
int vg_pc_destroy(vg_pc *pc);
/* poly_commit_prover::commit_private_array (poly_commit.h:42-116): RS-encodes
 * 64 slices of the private array (any, 2^log_len entries) and the mask (host,
 * n_mask entries, zero-padded to the next power of two M that divides the
 * slice evenly) at rate 1/32 into l_eval (65 slices of S = 2^(log_len-1)).
 * *mask_len (host, may be NULL) receives M. */
int vg_pc_encode_private(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *mask, long n_mask, long *mask_len);
/* poly_commit_prover::commit_public_array (poly_commit.h:125-342): RS-encodes
 * the public array (any, 2^log_len) and the public mask (host, n_mask <= M,
 * zero-padded to M), forms l*q, divides out the vanishing polynomial (h) and
 * builds the virtual oracle.  all_sum (host, 65 entries) is written;
 * *inner_product (host, may be NULL) receives <l, q> + <mask_l, mask_q> over
 * the committed points, the value the reference asserts equal to target_sum
 * (poly_commit.h:179-193). */
int vg_pc_encode_public(vg_pc *pc, const vg_fe *pub, const vg_fe *pub_mask, long n_mask, vg_fe *all_sum,
                        vg_fe *inner_product);
/* fri::request_init_commit (fri.cpp:36-139): leaf hash chains and Merkle tree
 * of oracle 0 (l_eval) or 1 (h_eval); *root host. */
int vg_pc_init_commit(vg_pc *pc, int oracle, vg_digest *root);
/* Public array eq(r, .) over log_len bits: pub[x] = prod_b (x_b ? r_b : 1 - r_b),
 * the table the reference verifier builds with dfs_for_public_eval
 * (zk_verifier.cpp:838-847).  r host, pub dev (2^log_len entries). */
int vg_eq_table(vg_ctx *ctx, const vg_fe *r, int log_len, vg_fe *pub);
/* fri::commit_phase_step (fri.cpp:291-430): folds the current codeword set
 * with r, hashes the new leaf chains and Merkle tree; root host. */
int vg_pc_fri_step(vg_pc *pc, vg_fe r, vg_digest *root);
/* fri::commit_phase_final (fri.cpp:432-438): the last folded codeword set in
 * the reference's interleaved layout, data[(j << 7) | (s << 1) | b] and
 * mask[2j + b] for j < n/2 (n = final per-slice length), host.  n host. */
int vg_pc_fri_final(vg_pc *pc, vg_fe *data, vg_fe *mask, long *n);
/* fri::request_init_value_with_merkle (fri.cpp:148-201) without the proof-size
 * bookkeeping: the 65 value pairs at (pow0, pow0 + S/2) of oracle 0 (l) or 1 (h)
 * and the authentication path (path[0..depth-1] siblings bottom-up,
 * path[depth] the leaf; depth = log_len - 2).  values (130 entries) and path
 * (depth + 1 entries) host. */
int vg_pc_query_init(vg_pc *pc, long pow0, int oracle, vg_fe *values, vg_digest *path);
/* fri::request_step_commit (fri.cpp:227-289) without the proof-size
 * bookkeeping: the 65 value pairs of FRI level lvl at position pow and its
 * authentication path (siblings bottom-up, then the leaf). host. */
int vg_pc_query_step(vg_pc *pc, int lvl, long pow, vg_fe *values, vg_digest *path, int *path_len);
/* Many query answers in one gather: query q reads codeword set which[q]
 * (0 = l, 1 = h, 2 + t = FRI level t) at position pos[q] (taken modulo half
 * the per-slice length) and returns 130 values (values[q*130 ..]) and its
 * authentication path (paths[q*32 ..], path_len[q] digests: siblings
 * bottom-up, then the leaf).  All arrays host. */
int vg_pc_query_batch(vg_pc *pc, int nq, const int *which, const long *pos, vg_fe *values, vg_digest *paths,
                      int *path_len);
/* The whole commitment of one proof in one call and one synchronisation
 * (poly_commit.h:42-351 commit_private_array / commit_public_array,
 * vpd_verifier.cpp:46-78 commit_phase, fri.cpp:36-139 and 291-430 with the
 * query answers of fri.cpp:148-289): RS encodings of priv and pub with their
 * masks, the virtual oracle, nlevels FRI folds with challenges fri_r, every
 * leaf chain and Merkle tree batched, and the nq query answers of
 * vg_pc_query_batch.  Outputs (host): roots[2 + nlevels] (l, h, FRI level
 * t), all_sum[65], *inner (the sampled <l, q>), final_cw[65 * n] (the last
 * level, slice-major, n = 2^(log_len - 1 - nlevels)), qvals[nq * 130],
 * qpaths[nq * 32].  The private mask is padded to vg_pc_info's mask length;
 * n_pub_mask may not exceed it. */
int vg_pc_commit_all(vg_pc *pc, const vg_fe *priv, int log_len, const vg_fe *pri_mask, long n_pri_mask,
                     const vg_fe *pub, const vg_fe *pub_mask, long n_pub_mask, const vg_fe *fri_r, int nlevels,
                     int nq, const int *which, const long *pos, vg_digest *roots, vg_fe *all_sum, vg_fe *inner,
                     vg_fe *final_cw, vg_fe *qvals, vg_digest *qpaths);
/* Sizes of the current commitment: log_len, slice size S, FRI levels so far. */
int vg_pc_info(vg_pc *pc, int *log_len, long *slice_size, int *levels);

/* ------------------------------------------------------------ whole proofs */
/* A session holds one circuit on the device and proves it on request.  Each
 * proof replays the reference verifier's challenge draws (glibc rand() after
 * srand(seed), zk_verifier.cpp:910-1253, vpd_verifier.cpp:80-312) and calls
 * the prover in the verifier's order, so the messages, roots and query
 * answers equal those of the reference prover run by the reference verifier
 * with that seed (the fft_gkr side proof is not part of it). */
typedef struct vg_session vg_session;
/* A proof runs the protocol twice from the same rand() state: the launch pass
 * enqueues every device step of the proof on the session's stream without
 * reading anything back, one synchronisation follows, and the replay pass
 * forms the messages, checks and transcript from the device results. */
typedef struct {
    double launch_s;        /* host time of the launch pass */
    double wait_s;          /* then the wait for the device */
    double replay_s;        /* host time of the replay pass */
    double total_s;         /* wall time of the call */
    double prove_time;      /* launch_s + wait_s: every prover message is on the host */
    long long proof_size;   /* bytes by the reference's accounting, without fft_gkr */
    long long launches;     /* kernels launched for this proof, the side proof's included */
    double fft_gkr_s;       /* the fft_gkr side proof: device time of its stream (0 when not run) */
    int fft_gkr_lg;         /* its size L - 6, 0 when not run */
    int fft_gkr_proof_size; /* its bytes as the reference counts them (the verifier adds them) */
    int graph_replays;      /* sumcheck phases whose round launches were replayed from a captured CUDA graph */
    int graph_captures;     /* sumcheck phases captured as a graph during this proof */
} vg_proof_stats;
/* From file-level layers as in the circuit text format (src/linear_gkr/README.md):
 * d layers, the input layer first (types 2/3, u = value), layer i has n[i]
 * gates ty[i][g], u[i][g], v[i][g] (host).  The input layer is padded and a
 * relay layer inserted as zk_verifier::read_circuit does
 * (zk_verifier.cpp:24-191). */
int vg_session_create(int d, const long *n, const uint8_t *const *ty, const int64_t *const *u,
                      const int64_t *const *v, vg_session **out);
/* A session proving the same circuit with its own stream, commitment state and
 * tables; the device circuit is shared (kept until every session using it is
 * destroyed).  Sessions of one circuit prove concurrently. */
int vg_session_fork(vg_session *base, vg_session **out);
/* Replaces a session's circuit, reusing its device buffers when the new
 * circuit fits them (the file-level layers as for vg_session_create;
 * index_bytes as for vg_circuit_build).  Forks keep the old circuit. */
int vg_session_load(vg_session *s, int d, const long *n, const uint8_t *const *ty, const void *const *u,
                    const void *const *v, int index_bytes);
/* Reads the circuit text format. */
int vg_session_from_file(const char *circuit_path, vg_session **out);
int vg_session_destroy(vg_session *s);
/* The context the drop-in classes and sessions run on (created on first use,
 * device $VIRGO_DEVICE, default 0). */
int vg_default_ctx(vg_ctx **out);
/* Writes file-level layers (as for vg_session_create) in the circuit text
 * format, and a meta file with one "0 0 1 0 0" line per layer.  Host only. */
int vg_circuit_write_text(int d, const long *n, const uint8_t *const *ty, const int64_t *const *u,
                          const int64_t *const *v, const char *circuit_path, const char *meta_path);
/* Binary circuit files (no reference counterpart; the reference parses text
 * with fscanf, zk_verifier.cpp:15-217): the file-level layers in the
 * vg_session_load layout (8-byte sections: "VGC1", version, d, index_bytes,
 * n[d], then per layer types, u, v; the input layer's u/v are int64), so a
 * load maps the file and builds the circuit on the device without parsing.
 * vg_session_from_file accepts either format. */
int vg_circuit_write_binary(const char *path, int d, const long *n, const uint8_t *const *ty, const void *const *u,
                            const void *const *v, int index_bytes);
/* 1 if path starts with the binary circuit magic, else 0.  Host only. */
int vg_circuit_is_binary(const char *path);
/* Header of a binary circuit file (validated against the file size): layer
 * count, wire width, and up to n_cap layer sizes.  Host only. */
int vg_circuit_binary_info(const char *path, int *d, int *index_bytes, long *n, int n_cap);
/* vg_session_load from a binary circuit file. */
int vg_session_load_file(vg_session *s, const char *path);
/* depth of the prover's circuit (file layers + 1) and log2 of the padded input */
int vg_session_depth(vg_session *s, int *depth, int *input_log);
/* One proof.  With want_transcript, *transcript (free with vg_free) receives
 * the records: tag byte, uint32 count of 16-byte units, the units. */
int vg_session_prove(vg_session *s, unsigned seed, int want_transcript, vg_proof_stats *stats,
                     uint8_t **transcript, size_t *transcript_len);
/* Every proof also runs the fft_gkr side proof for lg = L - 6 (2^L inputs,
 * L > 6) on the GPU beside it, as the reference verifier runs ./fft_gkr next
 * to every proof (vpd_verifier.cpp:89-99); on by default, off with on = 0.
 * A side proof that fails its checks fails the proof. */
int vg_session_set_fft_gkr(vg_session *s, int on);
/* New input values for the loaded circuit: the u of the n input gates of the
 * file-level input layer (as in vg_session_load: values read through int32,
 * the rest of the padded layer zero), host memory (pinned or pageable).  The
 * wiring stays on the device, so a circuit proven for many witnesses uploads
 * only these values (8 bytes each) per proof.  Forks keep their own values;
 * loading a circuit returns to that circuit's. */
int vg_session_set_inputs(vg_session *s, const int64_t *values, long n);
/* n proofs at once, session i with seed i, each on its own host thread and
 * CUDA stream (the sessions must be distinct objects, e.g. forks of one).
 * stats, transcripts and transcript_lens have n entries (or are NULL). */
int vg_session_prove_batch(vg_session *const *ss, int n, const unsigned *seeds, int want_transcript,
                           vg_proof_stats *stats, uint8_t **transcripts, size_t *transcript_lens);
/* The session's last proof as a file, for a verifier in another process
 * (no counterpart in the reference, whose prover and verifier share one
 * process and talk through method calls, zk_verifier.cpp:910-1253 and
 * vpd_verifier.cpp:80-335).  The file holds every device result the prover's
 * host replay consumes; with the circuit file and the seed (in the file), a
 * process running the reference verifier and the drop-in prover classes over
 * these results, no GPU, reproduces the proof: the verifier draws the same
 * rand() values and receives the same messages.  Valid after vg_session_prove
 * until the next proof or load.  Format (little-endian):
 *   char "VGPF"; uint32 version (1); uint32 seed; int32 depth;
 *   int32 bit_length[depth]  (the padded circuit's layers, input first);
 *   int32 nrec; int32 levels; int32 nq; int64 n_final; int32 proof_size;
 *   vg_fe records[9 * nrec]  (V_res, then every sumcheck round in call order:
 *                             its 3 sums, then the folded V, addV, add_mult
 *                             pairs when one pair remained);
 *   vg_digest roots[2 + levels] (l, h, FRI level t); vg_fe all_sum[65];
 *   vg_fe inner; vg_fe fri_r[levels]; vg_fe final_cw[65 * n_final]
 *   (slice-major); int32 which[nq]; int64 pos[nq] (as for vg_pc_query_batch);
 *   vg_fe qvals[130 * nq]; vg_digest qpaths[32 * nq]. */
int vg_session_write_proof(vg_session *s, const char *path);
/* A session with a context and no circuit yet (vg_session_load gives it one). */
int vg_session_new(vg_session **out);

/* ---- proof server (no reference counterpart: the reference proves one
 * circuit per process).  Continuous batching on one GPU: `slots` worker
 * sessions, each on its own stream, take queued jobs in arrival order as
 * they become free and as the job's device footprint fits hbm_budget bytes
 * (0: 90% of the free memory) next to what the other workers hold.  A job is
 * a circuit in the vg_session_load layout plus a seed; the arrays must stay
 * valid until vg_server_wait returns for that job.  Its transcript equals
 * the one vg_session_prove gives for the same circuit and seed. */
typedef struct vg_server vg_server;
typedef struct {
    int status;             /* VG_OK or the job's error code */
    double queued_s;        /* submit -> a worker took it */
    double run_s;           /* load + prove */
    double latency_s;       /* submit -> done */
    size_t footprint;       /* device bytes the admission reserved */
    vg_proof_stats stats;
} vg_job_info;
/* Device bytes a session needs for a circuit with file-layer widths n. */
size_t vg_job_footprint(int d, const long *n);
int vg_server_create(int device, int slots, size_t hbm_budget, vg_server **out);
int vg_server_submit(vg_server *s, int d, const long *n, const uint8_t *const *ty, const void *const *u,
                     const void *const *v, int index_bytes, unsigned seed, int want_transcript, long long *job_id);
/* Blocks until the job is done; *transcript (free with vg_free) as for
 * vg_session_prove.  Returns the job's status. */
int vg_server_wait(vg_server *s, long long job_id, vg_job_info *info, uint8_t **transcript, size_t *transcript_len);
int vg_server_destroy(vg_server *s);
/* The context (stream) a session runs on. */
int vg_session_ctx(vg_session *s, vg_ctx **out);
/* The context of the session's commitment work (its second stream; the
 * commitment overlaps the sumcheck rounds).  Profile both contexts to see a
 * whole proof. */
int vg_session_commit_ctx(vg_session *s, vg_ctx **out);
void vg_free(void *p);

/* ---- launch-shape tuning (no reference counterpart: the reference's loops
 * have no launch shapes).  One set of parameters per device, process-wide,
 * read by every launch on that device.  Every value gives bit-identical
 * results; only speed changes.  Defaults are the shapes measured best on the
 * 256x256 matmul proof. */
enum {
    VG_TUNE_GROUP_START = 0,   /* sumcheck tile: table length (power of two, 2^11 .. 2^22) at
                                  which a phase's remaining rounds run as round groups (chunks of
                                  2048 entries folded up to 10 rounds in shared memory, one CTA
                                  per chunk) instead of one launch per round */
    VG_TUNE_ROUND_THREADS = 1, /* threads per CTA of the one-round kernel (128, 256, 512) */
    VG_TUNE_NTT_MAX_LOG = 2,   /* NTT radix: log2 of the largest sub-DFT one pass runs in shared
                                  memory (6 .. 10); a 2^n transform takes ceil(n / this) passes */
    VG_TUNE_NTT_TILE_LOG = 3,  /* NTT stage fusion width: log2 of the elements one CTA holds in a
                                  pass (10 .. 13; sub-DFTs of several columns share a CTA) */
    VG_TUNE_LEAF_THREADS = 4,  /* threads per CTA of the per-thread leaf-chain kernels (64, 128, 256) */
    VG_TUNE_LEAF_WARP_MAX = 5, /* Merkle leaf hashing: launches of at most this many SHA3 leaf
                                  chains hash each chain with a whole warp (25 lanes of the
                                  Keccak state, one per thread) instead of one thread per chain;
                                  0 = never (0 .. 2^24) */
    VG_TUNE_ROUND_FUSE = 6,    /* sumcheck rounds per launch above the group start (1, 2): with 2,
                                  consecutive rounds pair into one pass that reads the tables
                                  once and writes a quarter of them */
    VG_TUNE_LEAF_ROT = 7,      /* SHA3 leaf chains (per-thread form): 0 = every 64-bit rotation as
                                  two funnel shifts (ALU pipe), the 24 rounds fully unrolled;
                                  1 = every other rho rotation, 2 =
                                  every rho rotation as multiplies by 2^n (integer-multiply pipe);
                                  3 (default) = funnel shifts with the 24 rounds in a loop
                                  unrolled four times (a sixth of the code: the fully unrolled
                                  permutation stalled on instruction fetch) */
    VG_TUNE_BETA_TABLE = 8,    /* phase-2 table builds read each gate's beta_g from a table the
                                  phase-1 builds of the same layer wrote (1), or form it again
                                  from the eq half tables (0) */
    VG_TUNE_GROUP_SPLIT = 9,   /* round groups: steps with few pairs left spread each pair over three
                                  threads, one per table (1), or keep one thread per pair (0) */
    VG_TUNE_LAZY_FOLD = 10,    /* sumcheck folds x0 + r (x1 - x0): 0 = canonical difference and the
                                  three-product (Karatsuba) F_p2 product; 1 = the difference left
                                  unreduced (x1 + 2p - x0) and a four-product (schoolbook) one,
                                  fewer integer-ALU steps for more multiply-pipe work */
    VG_TUNE_GATHER_FUSE = 11,  /* deferred proofs with paired rounds: a phase's table build over
                                  the layer's edges runs inside the pass of its first two rounds
                                  when the table is above the group start (1: the two tables it
                                  builds are never written in full), or as a launch of its own (0) */
    VG_TUNE_COUNT = 12
};
int vg_tune_get(int device, int key, long *value);
/* VG_ERR_ARG for a value outside the key's range. */
int vg_tune_set(int device, int key, long value);
int vg_tune_reset(int device);
int vg_tune_range(int key, long *lo, long *hi, long *def);

/* Autotuner: for each parameter in turn (the others fixed at their best so
 * far) times every candidate value by proving with the given sessions
 * (vg_session_prove_batch over all n at once: n = 1 tunes one proof's
 * latency, n > 1 the throughput of n proofs in flight), `reps` timed batches
 * after one warm-up batch per candidate, the best of them counting; keeps a
 * candidate only if it beats the value in force by more than 3%, and leaves
 * the winners set for the sessions' device.  trials (optional, up to
 * max_trials) receives every timing.  Do not prove on the same device from
 * other threads meanwhile. */
typedef struct {
    int key;
    long value;
    double ms;      /* best wall time of one batch */
    int chosen;     /* 1 for the value the tuner kept */
} vg_tune_trial;
int vg_autotune(vg_session *const *ss, int n, unsigned seed, int reps, vg_tune_trial *trials, int max_trials,
                int *n_trials);

/* ---- the fft_gkr side prover (src/VPD/fft_circuit_GKR.cpp) ----
 * The reference verifier runs it as a process, `fft_gkr <L-6> <file>`
 * (vpd_verifier.cpp:89-99), and adds its prover time to Prove Time; main
 * (fft_circuit_GKR.cpp:827-845) builds the circuit for lg and runs
 * engage_gkr (:786-825) with the prover's messages checked in process.
 * vg_fft_gkr_prove does the same on the GPU with the challenge stream of
 * rand() after srand(seed) (the reference process never seeds: seed 1).
 * msgs (optional, vg_fft_gkr_rounds(lg) x 3 values) receives every sumcheck
 * message (a, b, c) in order: addition layer (lg + 6 rounds), multiplication
 * layer (lg), then per inverse-FFT level phase 1 and phase 2 (lg each); vals
 * (optional, 2 + 2 lg) the value each phase ends on.  st->pass is 1 when every
 * check of the reference's in-process verifier holds. */
typedef struct vg_fft_gkr vg_fft_gkr;
typedef struct {
    double p_time;        /* seconds: first launch to the last message checked */
    double v_time;        /* seconds: the in-process verifier's checks */
    double gpu_s;         /* seconds of its stream: first to last of its device steps */
    int proof_size;       /* bytes, counted as fft_circuit_GKR.cpp counts them */
    int pass;
    int rounds;           /* sumcheck messages */
    long long launches;   /* kernels launched */
} vg_fft_gkr_stats;
int vg_fft_gkr_rounds(int lg_size);
int vg_fft_gkr_create(vg_ctx *ctx, int max_lg, vg_fft_gkr **out);   /* max_lg <= 22 */
int vg_fft_gkr_prove(vg_fft_gkr *f, int lg_size, unsigned seed, vg_fft_gkr_stats *st, vg_fe *msgs, vg_fe *vals);
int vg_fft_gkr_destroy(vg_fft_gkr *f);
/* device bytes a vg_fft_gkr object of max_lg holds */
size_t vg_fft_gkr_footprint(int max_lg);
/* create + prove + destroy */
int vg_fft_gkr_run(vg_ctx *ctx, int lg_size, unsigned seed, vg_fft_gkr_stats *st, vg_fe *msgs, vg_fe *vals);

#ifdef __cplusplus
}
#endif
#endif
