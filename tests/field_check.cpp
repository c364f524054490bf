// The F_{p^2} arithmetic of virgo_b200/csrc/fp2.cuh (host build of the same
// code the kernels run) against an independent restatement: schoolbook
// products with unsigned 128-bit integers reduced by %, p = 2^61 - 1,
// i^2 = -1.  Checks the product, x + a*b (fe_fma), sums and differences,
// canonical results, on every combination of edge values and on random
// inputs.  Exit status 0 when everything agrees; the first mismatch is
// printed.  Built and run by tests/test_host.py.
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <random>

#include "fp2.cuh"

using u128 = unsigned __int128;
static const uint64_t P = vg::P;

static uint64_t mod(u128 x) { return (uint64_t)(x % P); }
static uint64_t sub(uint64_t a, uint64_t b) { return mod((u128)a + P - b); }

// (ar + i ai)(br + i bi) = (ar br - ai bi) + i (ar bi + ai br)
static vg::fe ref_mul(vg::fe a, vg::fe b)
{
    const uint64_t re = sub(mod((u128)a.real * b.real), mod((u128)a.img * b.img));
    const uint64_t im = mod((u128)mod((u128)a.real * b.img) + mod((u128)a.img * b.real));
    return vg::fe_make(re, im);
}
static vg::fe ref_add(vg::fe a, vg::fe b)
{
    return vg::fe_make(mod((u128)a.real + b.real), mod((u128)a.img + b.img));
}

static long n_checked = 0;
static bool check(vg::fe x, vg::fe a, vg::fe b)
{
    const vg::fe m = ref_mul(a, b);
    const vg::fe want_fma = ref_add(x, m);
    const vg::fe want_sub = vg::fe_make(sub(a.real, b.real), sub(a.img, b.img));
    const vg::fe got = a * b, got_fma = vg::fe_fma(x, a, b), got_add = a + b, got_sub = a - b;
    ++n_checked;
    if (vg::fe_eq(got, m) && vg::fe_eq(got_fma, want_fma) && vg::fe_eq(got_add, ref_add(a, b)) &&
        vg::fe_eq(got_sub, want_sub))
        return true;
    printf("mismatch: a = (%llu, %llu) b = (%llu, %llu) x = (%llu, %llu)\n", (unsigned long long)a.real,
           (unsigned long long)a.img, (unsigned long long)b.real, (unsigned long long)b.img,
           (unsigned long long)x.real, (unsigned long long)x.img);
    return false;
}

int main(int argc, char **argv)
{
    const long n_random = argc > 1 ? atol(argv[1]) : 2000000;
    const uint64_t edge[] = {0, 1, 2, 7, 8, P - 1, P - 2, P - 8, P >> 1, (P >> 1) + 1, 1ull << 60, (1ull << 60) - 1,
                             (1ull << 32) - 1, 1ull << 32, (1ull << 32) + 1, 0x1FFFFFFF00000000ull, 0xFFFFFFFFull};
    const int ne = sizeof edge / sizeof edge[0];
    for (int i = 0; i < ne; ++i)
        for (int j = 0; j < ne; ++j)
            for (int k = 0; k < ne; ++k)
                for (int l = 0; l < ne; ++l) {
                    const vg::fe a = vg::fe_make(edge[i], edge[j]), b = vg::fe_make(edge[k], edge[l]);
                    if (!check(vg::fe_make(edge[(i + k) % ne], edge[(j + l) % ne]), a, b)) return 1;
                    if (!check(vg::fe_make(P - 1, P - 1), a, b)) return 1;
                }
    std::mt19937_64 rng(20261204);
    for (long it = 0; it < n_random; ++it) {
        vg::fe a = vg::fe_make(rng() % P, rng() % P), b = vg::fe_make(rng() % P, rng() % P);
        vg::fe x = vg::fe_make(rng() % P, rng() % P);
        if (it & 1) {   // operands near p, where the bounds of the folds are tightest
            a.real = P - 1 - (rng() & 0xFFFF);
            b.img = P - 1 - (rng() & 0xFF);
            x.img = P - 1 - (rng() & 0xF);
        }
        if (!check(x, a, b)) return 1;
    }
    printf("field check: %ld cases agree\n", n_checked);
    return 0;
}
