// C shim over the reference verifier's wiring predicates, compiled with the
// reference's own objects (oracle/Makefile, target "ref").  TEST
// INFRASTRUCTURE ONLY: it pins vg_circuit_predicates against
//   zk_verifier::beta_init  src/linear_gkr/zk_verifier.cpp:620-720
//   zk_verifier::predicates src/linear_gkr/zk_verifier.cpp:219-606
// on a circuit given as prover-level layers (layer 0 the input values, every
// layer a power of two wide).
#include "linear_gkr/zk_verifier.h"
#include <vector>

typedef prime_field::field_element fe;

extern "C" int ref_predicates(int depth, const int *bit_length, const unsigned char *const *ty, const long long *const *u,
                              const long long *const *v, int which, const fe *r_0, const fe *r_1, const fe *r_u,
                              const fe *r_v, const fe *alpha, const fe *beta, fe *out)
{
    prime_field::init();
    zk_verifier V;
    V.C.total_depth = depth;
    V.C.circuit = new layer[depth];
    int max_bl = 0;
    for (int i = 0; i < depth; ++i) {
        const long n = 1L << bit_length[i];
        V.C.circuit[i].bit_length = bit_length[i];
        V.C.circuit[i].is_parallel = false;
        V.C.circuit[i].gates = new gate[n];
        for (long g = 0; g < n; ++g) V.C.circuit[i].gates[g] = gate(ty[i][g], u[i][g], v[i][g]);
        if (bit_length[i] > max_bl) max_bl = bit_length[i];
    }
    const int f = max_bl / 2, s = max_bl - f;
    fe **halves[8] = {&V.beta_g_r0_first_half, &V.beta_g_r0_second_half, &V.beta_g_r1_first_half,
                      &V.beta_g_r1_second_half, &V.beta_u_first_half,   &V.beta_u_second_half,
                      &V.beta_v_first_half,    &V.beta_v_second_half};
    for (int k = 0; k < 8; ++k) *halves[k] = new fe[1 << ((k & 1) ? s : f)];
    const int lg = bit_length[which], luv = bit_length[which - 1];
    std::vector<fe> r0(r_0, r_0 + lg), r1(r_1, r_1 + lg), ru(r_u, r_u + luv), rv(r_v, r_v + luv);
    std::vector<fe> o0(lg), o1(lg), ou(luv), ov(luv);
    for (int i = 0; i < lg; ++i) {
        o0[i] = fe(1) - r0[i];
        o1[i] = fe(1) - r1[i];
    }
    for (int i = 0; i < luv; ++i) {
        ou[i] = fe(1) - ru[i];
        ov[i] = fe(1) - rv[i];
    }
    V.beta_init(which, *alpha, *beta, r0.data(), r1.data(), ru.data(), rv.data(), o0.data(), o1.data(), ou.data(),
                ov.data());
    std::vector<fe> ret = V.predicates(which, r0.data(), r1.data(), ru.data(), rv.data(), *alpha, *beta);
    for (int t = 0; t < 14; ++t) out[t] = ret[t];
    return 0;
}
