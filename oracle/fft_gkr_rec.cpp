// Message recorder around the reference fft_gkr side prover.  TEST
// INFRASTRUCTURE ONLY: linked into oracle/_ref/fft_gkr_rec, never into the
// product library.
//
// src/VPD/fft_circuit_GKR.cpp is compiled unchanged with its main renamed to
// ref_fft_gkr_main.  Its prover checks every sumcheck message in place
// (poly.eval(0) + poly.eval(1), then poly.eval(r), :323-333) and reads every
// phase's final value with V_mult_add[0].eval(r) (:335, :581, :680); both eval
// methods live in src/linear_gkr/polynomial.cpp, another object, so GNU ld's
// --wrap routes each call here.  Every call is appended to the file named by
// the third argument:
//   'Q' a b c x   quadratic_poly::eval  (4 field elements)
//   'L' a b x     linear_poly::eval     (3 field elements)
// field elements as {img, real}, 16 bytes.  Usage: fft_gkr_rec <lg> <out> <rec>
#include "linear_gkr/polynomial.h"
#include <cstdio>

typedef prime_field::field_element fe;

int ref_fft_gkr_main(int argc, char *argv[]);

static FILE *g_rec = nullptr;

static void put(char tag, const fe *v, int n)
{
    if (!g_rec) return;
    fputc(tag, g_rec);
    for (int i = 0; i < n; ++i) {
        fwrite(&v[i].img, 8, 1, g_rec);
        fwrite(&v[i].real, 8, 1, g_rec);
    }
}

extern "C" fe __real__ZNK14quadratic_poly4evalERKN11prime_field13field_elementE(const quadratic_poly *p, const fe &x);
extern "C" fe __wrap__ZNK14quadratic_poly4evalERKN11prime_field13field_elementE(const quadratic_poly *p, const fe &x)
{
    const fe v[4] = {p->a, p->b, p->c, x};
    put('Q', v, 4);
    return __real__ZNK14quadratic_poly4evalERKN11prime_field13field_elementE(p, x);
}

extern "C" fe __real__ZNK11linear_poly4evalERKN11prime_field13field_elementE(const linear_poly *p, const fe &x);
extern "C" fe __wrap__ZNK11linear_poly4evalERKN11prime_field13field_elementE(const linear_poly *p, const fe &x)
{
    const fe v[3] = {p->a, p->b, x};
    put('L', v, 3);
    return __real__ZNK11linear_poly4evalERKN11prime_field13field_elementE(p, x);
}

int main(int argc, char *argv[])
{
    if (argc < 4) {
        fprintf(stderr, "usage: %s <lg> <out> <rec>\n", argv[0]);
        return 2;
    }
    g_rec = fopen(argv[3], "wb");
    if (!g_rec) return 2;
    const int rc = ref_fft_gkr_main(3, argv);
    fclose(g_rec);
    return rc;
}
