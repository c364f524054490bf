// GKR prover with the reference's interface (include/linear_gkr/zk_prover.h:16-122):
// the verifier calls these methods in protocol order and reads the public
// scalar members directly, so their names and types are kept.  The layer
// values, the bookkeeping tables and the circuit live on the GPU:
// circuit_value[i] holds device pointers (valid after evaluate()), and the
// reference's host tables (addV_array, V_mult_add, add_mult_sum, beta_*)
// are replaced by device state behind the C ABI of include/virgo_b200.h.
// The scalar mask and claim bookkeeping runs on the host exactly as in the
// reference (it consumes rand() in the same order).
#ifndef __zk_prover
#define __zk_prover

#include "linear_gkr/circuit_fast_track.h"
#include "linear_gkr/prime_field.h"
#include "linear_gkr/polynomial.h"
#include <cstring>
#include <utility>
#include <vector>
#include <chrono>
#include "VPD/vpd_prover.h"
#include "infrastructure/my_hhash.h"
#include "VPD/fri.h"
#include "poly_commitment/poly_commit.h"

struct vg_circuit;
struct vg_gkr;

class zk_prover
{
public:
    poly_commit::poly_commit_prover poly_prover;
    prime_field::field_element v_u, v_v;
    int total_uv;
    layered_circuit C;
    prime_field::field_element *circuit_value[1000000];

    int sumcheck_layer_id, length_g, length_u, length_v;

    prime_field::field_element alpha, beta;
    const prime_field::field_element *r_0, *r_1;
    prime_field::field_element *one_minus_r_0, *one_minus_r_1;

    double total_time;
    void init_array(int);
    // Copies the circuit to the GPU (once per circuit).
    void get_circuit(const layered_circuit &from_verifier);
    // Evaluates all layers on the GPU; returns the device pointer of the output layer.
    prime_field::field_element *evaluate();
    void proof_init();

    void sumcheck_init(int layer_id, int bit_length_g, int bit_length_u, int bit_length_v, const prime_field::field_element &,
                       const prime_field::field_element &, const prime_field::field_element *, const prime_field::field_element *,
                       prime_field::field_element *, prime_field::field_element *);
    void sumcheck_phase1_init();
    void sumcheck_phase2_init(prime_field::field_element, const prime_field::field_element *, const prime_field::field_element *);
    quadratic_poly sumcheck_phase1_update(prime_field::field_element, int);
    quintuple_poly sumcheck_phase1_updatelastbit(prime_field::field_element, int);
    quadratic_poly sumcheck_phase2_update(prime_field::field_element, int);
    quintuple_poly sumcheck_phase2_updatelastbit(prime_field::field_element, int);
    quadratic_poly sumcheck_finalround(prime_field::field_element, int, prime_field::field_element);
    // Multilinear extension of output_raw (the output layer from evaluate(), or
    // any host/device array of output_size values) at r_0.
    prime_field::field_element V_res(const prime_field::field_element *, const prime_field::field_element *,
                                     const prime_field::field_element *, int, int);
    std::pair<prime_field::field_element, prime_field::field_element> sumcheck_finalize(prime_field::field_element);
    void delete_self();
    zk_prover();
    ~zk_prover();

    void generate_maskR(int layer_id);
    std::vector<prime_field::field_element> all_pri_mask;
    prime_field::field_element *maskpoly;
    prime_field::field_element maskpoly_sumc;
    prime_field::field_element maskpoly_sumr;
    prime_field::field_element rho;
    void generate_maskpoly_pre_rho(int, int);
    void generate_maskpoly_after_rho(int, int);
    prime_field::field_element maskR[6], preR[6];

    prime_field::field_element maskR_sumcu, maskR_sumcv, preZu, preZv, Zu, Zv, preu1, prev1, Iuv, prepreu1, preprev1;
    quadratic_poly Rg1, Rg2, sumRc;

    prime_field::field_element query(prime_field::field_element *, prime_field::field_element *, prime_field::field_element);
    prime_field::field_element queryRg1(prime_field::field_element);
    prime_field::field_element queryRg2(prime_field::field_element);

    std::vector<prime_field::field_element> maskr;

    // ---- device state (not part of the reference interface) ----
    struct vg_ctx *dev_ctx;   // context (stream) of this prover; the process default when null
    vg_circuit *dev_circuit;
    vg_gkr *dev_gkr;
    bool owns_circuit;
    bool quiet;               // no timing line on stderr from evaluate()
    prime_field::field_element tables_last[6];   // folded V, addV, add_mult pairs after a phase's last round
    // Reuses an uploaded circuit (e.g. many proofs of one circuit); the
    // prover then does not free it.
    void attach_circuit(const layered_circuit &c, vg_circuit *dev, struct vg_ctx *ctx = nullptr);
    // Clears the per-proof state so the same object can prove again.
    void reset_proof();
    // One-sync proofs (vg_session_prove) run the protocol twice from the same
    // rand() state: DEFER_LAUNCH only enqueues the device work (round sums and
    // the other device results stay on the device as records), DEFER_REPLAY
    // does no device work and takes the device results from `replay`, in call
    // order.  DEFER_OFF (default) is the reference's synchronous behaviour.
    enum { DEFER_OFF = 0, DEFER_LAUNCH = 1, DEFER_REPLAY = 2 };
    int defer_mode;
    const prime_field::field_element *replay;   // 9 values per record
    int replay_n, replay_i;
};

#endif
