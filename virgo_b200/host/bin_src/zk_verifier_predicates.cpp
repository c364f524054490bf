// zk_verifier::predicates on the GPU, for a drop-in build of the reference
// verifier.
//
// The reference verifier spends most of its time in the wiring predicates
// of each layer (zk_verifier.cpp:219-606): per gate type, the sum over the
// layer's gates of beta_g(g) beta_u(u) beta_v(v), one pass over every gate on
// one core (about 1.5 s of the 1.54 s verification of the 2^24-gate matmul
// circuit).  This file gives the verifier's class a definition of that member
// which sums on the GPU over the circuit the drop-in prover already holds
// there (vg_circuit_predicates): main_zk.cpp:22 hands the verifier's circuit
// to zk_prover::get_circuit, which uploads it with the same layer numbering
// (the reader's relay layer included).
//
// The reference returns the plain form's sums for every layer: for a
// data-parallel layer it also forms the block form, only to assert that both
// agree (zk_verifier.cpp:601-605), so the plain form serves every layer.
// Layer 1, the relay layer, returns zeros as there (its term comes from
// direct_relay).
//
// Build: the reference's zk_verifier.cpp calls predicates from its own
// translation unit, so a linker wrap does not reach the call.  Instead its
// definition is made weak in the compiled object and this strong one is
// linked beside it (the calls then resolve here):
//   g++ ... -c zk_verifier.cpp -o zk_verifier.o
//   objcopy --weaken-symbol=_ZN11zk_verifier10predicatesEiPN11prime_field13field_elementES2_S2_S2_S1_S1_ \
//       zk_verifier.o
//   g++ ... -c zk_verifier_predicates.cpp      (same include path as zk_verifier.cpp)
//   g++ -o zk_proof main_zk.o zk_verifier.o zk_verifier_predicates.o vpd_verifier.o ... -lvirgo_b200
// VIRGO_LOG_PREDICATES=1 prints one line per layer answered here (stderr).
#include "linear_gkr/zk_verifier.h"

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "virgo_b200.h"

static_assert(sizeof(prime_field::field_element) == sizeof(vg_fe), "field element layout");

static vg_fe to_vg(const prime_field::field_element &x)
{
    vg_fe r;
    r.img = x.img;
    r.real = x.real;
    return r;
}

std::vector<prime_field::field_element> zk_verifier::predicates(int depth, prime_field::field_element *r_0,
                                                                prime_field::field_element *r_1,
                                                                prime_field::field_element *r_u,
                                                                prime_field::field_element *r_v,
                                                                prime_field::field_element alpha,
                                                                prime_field::field_element beta)
{
    const int gate_type_count = 14;
    std::vector<prime_field::field_element> ret(gate_type_count, prime_field::field_element(0));
    if (depth == 1) return ret;
    if (!p || !p->dev_circuit) {
        fprintf(stderr, "zk_verifier::predicates: the prover holds no device circuit (get_circuit not called)\n");
        abort();
    }
    vg_ctx *ctx = p->dev_ctx;
    if (!ctx && vg_default_ctx(&ctx) != VG_OK) {
        fprintf(stderr, "zk_verifier::predicates: %s\n", vg_last_error());
        abort();
    }
    vg_fe out[gate_type_count];
    if (vg_circuit_predicates(ctx, p->dev_circuit, depth, reinterpret_cast<const vg_fe *>(r_0),
                              reinterpret_cast<const vg_fe *>(r_1), reinterpret_cast<const vg_fe *>(r_u),
                              reinterpret_cast<const vg_fe *>(r_v), to_vg(alpha), to_vg(beta), out) != VG_OK) {
        fprintf(stderr, "zk_verifier::predicates: %s\n", vg_last_error());
        abort();
    }
    for (int t = 0; t < gate_type_count; ++t) {
        ret[t].img = out[t].img;
        ret[t].real = out[t].real;
    }
    if (getenv("VIRGO_LOG_PREDICATES")) fprintf(stderr, "virgo predicates: layer %d on the GPU\n", depth);
    return ret;
}
