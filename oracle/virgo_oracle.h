/* CPU restatement of the Virgo prover hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as the checker (or the timed CPU baseline);
 * nothing in the product calls it.  Every routine names the reference
 * file:line it restates.  It is pinned against the reference itself: the
 * tests compare it with routines of the reference compiled from source
 * (oracle/ref_kernels.cpp) and with the committed golden vectors under
 * tests/golden/, which come from whole reference runs.
 *
 * Layouts: a field element is {img, real} (16 bytes), a digest 32 bytes.
 * "Codeword sets" are slice-major: slice s of length n at c[s * n].
 */
#ifndef VIRGO_ORACLE_H
#define VIRGO_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { uint64_t img, real; } vo_fe;
typedef struct { uint8_t b[32]; } vo_digest;

/* field (include/linear_gkr/prime_field.h:114-172, src/linear_gkr/prime_field.cpp:60-92) */
void vo_fe_mul_arr(const vo_fe *a, const vo_fe *b, vo_fe *c, long n);
void vo_fe_add_arr(const vo_fe *a, const vo_fe *b, vo_fe *c, long n);
void vo_fe_sub_arr(const vo_fe *a, const vo_fe *b, vo_fe *c, long n);
void vo_fe_inv(const vo_fe *a, vo_fe *out);
void vo_root_of_unity(int log_order, vo_fe *out);

/* FFT (src/infrastructure/RS_polynomial.cpp:27-240) */
void vo_fft(const vo_fe *coef, long coef_len, long order, const vo_fe *root, vo_fe *out);
void vo_ifft(const vo_fe *evals, long coef_len, long order, const vo_fe *root, vo_fe *out);

/* hashes of exactly 64 bytes (include/infrastructure/my_hhash.h:28-35) */
void vo_sha3_256_64(const uint8_t *in64, uint8_t *out32);
void vo_sha256_64(const uint8_t *in64, uint8_t *out32);
void vo_hash64_batch(int kind, const uint8_t *in, uint8_t *out, long n);

/* Merkle tree (src/infrastructure/merkle_tree.cpp:4-57): tree holds
 * 2 * next_pow2(n) digests, tree[1] is the root. */
void vo_merkle_tree(int kind, const vo_digest *leaves, long n, vo_digest *tree);

/* Leaf hash chains of a codeword set of n_slices slices of length n
 * (src/VPD/fri.cpp:97-126 and :394-420): leaf k (k < n/2) chains
 * h = H((c[s][k], c[s][k + n/2]) || h) over s = 0..n_slices-1 from h = 0. */
void vo_leaf_chain(int kind, const vo_fe *c, int n_slices, long n, vo_digest *leaves);

/* One FRI fold (src/VPD/fri.cpp:321-340, :367-379) of a codeword set of
 * per-slice length n whose evaluation domain is <w>, w of order n:
 * out[s][i] = ((a + b) + w^-i * r * (a - b)) / 2, a = c[s][i], b = c[s][i+n/2]. */
void vo_fri_fold(const vo_fe *c, int n_slices, long n, const vo_fe *w, const vo_fe *r, vo_fe *out);

/* RS encoding of one slice (include/poly_commitment/poly_commit.h:107-108):
 * interpolate m values on <w_m>, evaluate on <w_s>. */
void vo_rs_encode(const vo_fe *vals, long m, long s, vo_fe *out);

/* commit_private_array (poly_commit.h:42-124): l_eval gets 65 slices of S;
 * returns the padded mask length. */
long vo_commit_private(const vo_fe *priv, int log_len, const vo_fe *mask, long n_mask, vo_fe *l_eval);

/* commit_public_array (poly_commit.h:125-351): given l_eval from
 * vo_commit_private, the public array (2^log_len) and the padded public mask
 * (n_mask entries, a power of two) fills q_eval, h_eval (65 slices of S),
 * the virtual oracle (65 slices of S, slice-major, mask slice last) and
 * all_sum[65]. */
void vo_commit_public(const vo_fe *l_eval, const vo_fe *pub, int log_len, const vo_fe *pub_mask, long n_mask,
                      vo_fe *q_eval, vo_fe *h_eval, vo_fe *vo, vo_fe *all_sum);

/* GKR pieces (src/linear_gkr/zk_prover.cpp) over one layer's gates (ty, u, v) */
void vo_eval_input(const int64_t *u, long n, vo_fe *out);                         /* :57-66 */
void vo_eval_layer(const uint8_t *ty, const int64_t *u, const int64_t *v, long n,
                   const vo_fe *prev, vo_fe *out);                                /* :68-150 */
void vo_v_res(const vo_fe *vals, int log_n, const vo_fe *r, vo_fe *out);         /* :30-52 */
/* beta_g(i) = alpha*eq(r0, i) + beta*eq(r1, i) over length_g bits (:391-418) */
void vo_beta_g(int length_g, const vo_fe *r0, const vo_fe *r1, const vo_fe *alpha, const vo_fe *beta, vo_fe *out);
void vo_phase1_init(const uint8_t *ty, const int64_t *u, const int64_t *v, long n_g, const vo_fe *beta_g,
                    const vo_fe *prev, long n_uv, vo_fe *add_mult_b, vo_fe *addv_b);  /* :375-592 */
void vo_phase2_init(const uint8_t *ty, const int64_t *u, const int64_t *v, long n_g, const vo_fe *beta_g,
                    const vo_fe *beta_u, const vo_fe *v_u, long n_uv, vo_fe *add_mult_b, vo_fe *addv_b); /* :789-972 */
/* The verifier's wiring predicates of one layer (src/linear_gkr/zk_verifier.cpp
 * :219-606, the layer not data-parallel): out[t] sums, over the layer's gates
 * of type t, beta_g(g) beta_u(u) beta_v(v) with beta_g as vo_beta_g,
 * beta_u = eq(r_u, .), beta_v = eq(r_v, .) over bl_uv bits; summation (5,
 * u <= j < v) and exp-sum (12, u <= j <= v, weight 2^(j-u)) sum beta_u over
 * the range times beta_v(0); relays (10) take beta_u(u), the total times
 * beta_v(0).  Types 2, 3, 4 contribute nothing. */
void vo_predicates(const uint8_t *ty, const int64_t *u, const int64_t *v, int bl_g, int bl_uv, const vo_fe *r0,
                   const vo_fe *r1, const vo_fe *ru, const vo_fe *rv, const vo_fe *alpha, const vo_fe *beta,
                   vo_fe out[14]);
/* One round of sumcheck_phase{1,2}_update (:596-633, :988-1025) on the
 * linear-polynomial tables V_mult_add, addV_array, add_mult_sum ({a, b} pairs,
 * total_uv entries), in place exactly as the reference loop; returns the
 * round polynomial (a, b, c) before the mask terms are added. */
typedef struct { vo_fe a, b; } vo_lp;
void vo_sumcheck_round(vo_lp *V, vo_lp *addv, vo_lp *am, long total_uv, const vo_fe *r, int current_bit, vo_fe out3[3]);

/* The fft_gkr side prover (src/VPD/fft_circuit_GKR.cpp, run by the
 * verifier as its own process, vpd_verifier.cpp:89-99) for lg_size:
 * build_circuit (:22-112) and engage_gkr (:786-825) with the random stream of
 * rand() after srand(seed) (the reference process never seeds: seed 1).
 * msgs receives every sumcheck message (a, b, c) in order: the addition
 * layer (lg+6 rounds), the multiplication layer (lg), then per inverse-FFT
 * level phase 1 and phase 2 (lg each); vals the final value of each phase
 * (addition v_u, multiplication v_u, then v_u, v_v per level).  Returns 1
 * when every check of the reference's in-process verifier passes;
 * *proof_size as the reference counts it. */
int vo_fft_gkr_rounds(int lg_size);
int vo_fft_gkr(int lg_size, unsigned seed, vo_fe *msgs, vo_fe *vals, int *proof_size);

#ifdef __cplusplus
}
#endif
#endif
