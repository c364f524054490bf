// C shim over single routines of the reference, compiled from the reference's
// own sources (oracle/Makefile, target "ref").  TEST INFRASTRUCTURE ONLY: it
// lets the tests pin the C restatement (virgo_oracle.c) routine by routine
// against the reference itself.
//   ref_fft / ref_ifft   -> src/infrastructure/RS_polynomial.cpp:27,169
//   ref_create_tree      -> src/infrastructure/merkle_tree.cpp:4
//   ref_hash64           -> include/infrastructure/my_hhash.h:28 (XKCP SHA3-256)
//   ref_fe_mul / ref_root_of_unity / ref_inv -> include/linear_gkr/prime_field.h,
//                           src/linear_gkr/prime_field.cpp:60-92
#include "linear_gkr/prime_field.h"
#include "infrastructure/RS_polynomial.h"
#include "infrastructure/merkle_tree.h"
#include "infrastructure/my_hhash.h"
#include <cstdlib>
#include <cstring>

typedef prime_field::field_element fe;
static int g_pad = 0;
static void ensure_pad(int order)
{
    if (order > g_pad) {
        init_scratch_pad(order);
        g_pad = order;
    }
}

extern "C" {
void ref_init() { prime_field::init(); }

void ref_fft(const fe *coef, int coef_len, int order, int log_root, fe *out)
{
    ensure_pad(order);
    fast_fourier_transform(coef, coef_len, order, prime_field::get_root_of_unity(log_root), out);
}

void ref_ifft(fe *evals, int coef_len, int order, int log_root, fe *out)
{
    ensure_pad(order);
    inverse_fast_fourier_transform(evals, coef_len, order, prime_field::get_root_of_unity(log_root), out);
}

// out must hold 2 * next_pow2(n) digests; out[1] is the root.
void ref_create_tree(const __hhash_digest *leaves, int n, __hhash_digest *out)
{
    __hhash_digest *dst = out;
    merkle_tree::merkle_tree_prover::create_tree((void *)leaves, n, dst, sizeof(__hhash_digest), false);
}

void ref_hash64(const unsigned char *src, unsigned char *dst) { my_hhash(src, dst); }

void ref_fe_mul(const fe *a, const fe *b, fe *c, long n)
{
    for (long i = 0; i < n; ++i) c[i] = a[i] * b[i];
}
void ref_fe_add(const fe *a, const fe *b, fe *c, long n)
{
    for (long i = 0; i < n; ++i) c[i] = a[i] + b[i];
}
void ref_fe_sub(const fe *a, const fe *b, fe *c, long n)
{
    for (long i = 0; i < n; ++i) c[i] = a[i] - b[i];
}
void ref_root_of_unity(int log_order, fe *out) { *out = prime_field::get_root_of_unity(log_order); }
void ref_inv(const fe *a, fe *out) { *out = prime_field::inv(*a); }
}
