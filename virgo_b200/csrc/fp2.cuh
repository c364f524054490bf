// F_{p^2} arithmetic, p = 2^61 - 1, i^2 = -1, shared by device kernels and
// host code.
//
// Element layout is {img, real} (two uint64, img first), the in-memory layout
// of prime_field::field_element (reference include/linear_gkr/prime_field.h:93),
// so buffers cross the C ABI unchanged.  Every operation returns a canonical
// value in [0, p) for canonical inputs; the reference's operators do the same
// (prime_field.h:114-172), so results agree bit for bit whatever the order of
// evaluation.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define VG_HD __host__ __device__ __forceinline__
#else
#define VG_HD inline
#endif

namespace vg {

constexpr uint64_t P = 0x1FFFFFFFFFFFFFFFull;  // 2^61 - 1

struct alignas(16) fe {
    uint64_t img, real;
};

VG_HD fe fe_make(uint64_t real, uint64_t img) { fe r; r.real = real; r.img = img; return r; }
VG_HD fe fe_zero() { return fe_make(0, 0); }
VG_HD fe fe_one() { return fe_make(1, 0); }
VG_HD bool fe_eq(fe a, fe b) { return a.real == b.real && a.img == b.img; }
VG_HD bool fe_is_zero(fe a) { return (a.real | a.img) == 0; }

// ---- F_p ----
// For canonical a, b: a + b - p is negative (as a signed 64-bit value)
// exactly when a + b < p, and a - b exactly when a < b; the sign picks the
// result without a 64-bit comparison.
VG_HD uint64_t addp(uint64_t a, uint64_t b)
{
    const uint64_t s = a + b, t = s - P;
    return (int64_t)t < 0 ? s : t;
}
VG_HD uint64_t subp(uint64_t a, uint64_t b)
{
    const uint64_t d = a - b;
    return (int64_t)d < 0 ? d + P : d;
}
VG_HD uint64_t negp(uint64_t a) { return a ? P - a : 0; }

VG_HD void mul64wide(uint64_t a, uint64_t b, uint64_t &lo, uint64_t &hi)
{
#if defined(__CUDA_ARCH__)
    lo = a * b;
    hi = __umul64hi(a, b);
#else
    unsigned __int128 x = (unsigned __int128)a * b;
    lo = (uint64_t)x;
    hi = (uint64_t)(x >> 64);
#endif
}

// x mod p for x < 2^64, partly reduced: the result is below 2^61 + 8.
VG_HD uint64_t foldp(uint64_t x) { return (x & P) + (x >> 61); }
// x mod p, canonical, for x < 2p: x + 1 reaches 2^61 exactly when x >= p.
VG_HD uint64_t canonp(uint64_t x) { return (x + ((x + 1) >> 61)) & P; }

// a*b mod p for a, b < 2^61 (canonical).  x = hi*2^64 + lo <= (p-1)^2, and
// x = (x >> 61) * 2^61 + (x & p) == (x >> 61) + (x & p) (mod p); both terms are
// at most p and not both p (x < p 2^61 + p), so the sum is below 2p.
VG_HD uint64_t mulp(uint64_t a, uint64_t b)
{
    uint64_t lo, hi;
    mul64wide(a, b, lo, hi);
    return canonp((lo & P) + ((hi << 3) | (lo >> 61)));
}
// a*b mod p, partly reduced (below 2^61 + 8), for a*b < 2^124.
VG_HD uint64_t mulp_partial(uint64_t a, uint64_t b)
{
    uint64_t lo, hi;
    mul64wide(a, b, lo, hi);
    return foldp((lo & P) + ((hi << 3) | (lo >> 61)));
}
// x = a*b mod p as (x & p) + (x >> 61), not folded further, for a*b < 2^124:
// below 2^62 when a, b < 2^61 (x >> 61 < 2^61), below 2^61 + 2^63 when
// a, b < 2^62.
VG_HD uint64_t mulp_fold1(uint64_t a, uint64_t b)
{
    uint64_t lo, hi;
    mul64wide(a, b, lo, hi);
    return (lo & P) + ((hi << 3) | (lo >> 61));
}

// ---- F_{p^2} ----
VG_HD fe operator+(fe a, fe b) { return fe_make(addp(a.real, b.real), addp(a.img, b.img)); }
VG_HD fe operator-(fe a, fe b) { return fe_make(subp(a.real, b.real), subp(a.img, b.img)); }
VG_HD fe operator-(fe a) { return fe_make(negp(a.real), negp(a.img)); }

// (ar + i ai)(br + i bi) = (ar br - ai bi) + i((ar + ai)(br + bi) - ar br - ai bi)
// For canonical inputs ac = ar br and bd = ai bi are taken once folded
// (mulp_fold1: below 2^62), t = (ar + ai)(br + bi) (operands below 2^62, the
// product below 2^124) folded twice (below 2^61 + 5), and the differences as
// ac + 3p - bd (3p > 2^62 > bd; the sum below 5 2^61) and t + 5p - ac - bd
// (5p > 2^63 > ac + bd; the sum below 6 2^61), each folded once (below
// 2^61 + 5) before the final canonical step: the canonical product with two
// folds fewer than folding every partial product.
VG_HD fe operator*(fe a, fe b)
{
    const uint64_t ac = mulp_fold1(a.real, b.real);
    const uint64_t bd = mulp_fold1(a.img, b.img);
    const uint64_t t = foldp(mulp_fold1(a.real + a.img, b.real + b.img));
    const uint64_t re = foldp(ac + (3 * P - bd));
    const uint64_t im = foldp(t + (5 * P - ac - bd));
    return fe_make(canonp(re), canonp(im));
}

// x + a*b for canonical x, a, b: x joins the product's two sums before their
// last fold (ac + 3p - bd + x.real below 6 2^61, t + 5p - ac - bd + x.img
// below 7 2^61 + 5), so an integer add replaces a canonical one; the same
// canonical result as x + a * b.
VG_HD fe fe_fma(fe x, fe a, fe b)
{
    const uint64_t ac = mulp_fold1(a.real, b.real);
    const uint64_t bd = mulp_fold1(a.img, b.img);
    const uint64_t t = foldp(mulp_fold1(a.real + a.img, b.real + b.img));
    const uint64_t re = foldp(ac + (3 * P - bd) + x.real);
    const uint64_t im = foldp(t + (5 * P - ac - bd) + x.img);
    return fe_make(canonp(re), canonp(im));
}

VG_HD fe fe_double(fe a) { return a + a; }

// x0 + r (x1 - x0) for canonical x0, x1, r with the difference left
// unreduced: x1 + 2p - x0 < 3p < 2^63 per component, multiplied by r with
// four partial products (no sums of operands), each below 3p * p < 2^124,
// mulp_partial's range.  Fewer integer-ALU steps than the canonical
// subtraction and three-product form; the same canonical result.
VG_HD fe fold_lazy(fe x0, fe x1, fe r)
{
    const uint64_t dr = x1.real + 2 * P - x0.real, di = x1.img + 2 * P - x0.img;
    const uint64_t ac = mulp_partial(dr, r.real), bd = mulp_partial(di, r.img);
    const uint64_t ad = mulp_partial(dr, r.img), bc = mulp_partial(di, r.real);
    const uint64_t re = foldp(ac + (4 * P - bd));
    const uint64_t im = foldp(ad + bc);
    return x0 + fe_make(canonp(re), canonp(im));
}

// a * 2^k for canonical a and 0 <= k <= 60: since 2^61 = 1 (mod p), this is a
// left rotation of each 61-bit component
VG_HD uint64_t rotp(uint64_t x, int k) { return ((x << k) | (x >> (61 - k))) & P; }
VG_HD fe fe_mul_pow2(fe a, int k) { return fe_make(rotp(a.real, k), rotp(a.img, k)); }

// multiplication by an element of F_p (img = 0)
VG_HD fe fe_scale(fe a, uint64_t s) { return fe_make(mulp(a.real, s), mulp(a.img, s)); }

VG_HD fe fe_pow(fe x, uint64_t e)
{
    fe r = fe_one();
    while (e) {
        if (e & 1) r = r * x;
        x = x * x;
        e >>= 1;
    }
    return r;
}

// x^(p^2 - 2) = x^-1; p^2 - 2 does not fit 64 bits, so exponentiate by the
// 128-bit value with two 64-bit words.
VG_HD fe fe_inv(fe x)
{
    // p^2 - 2 = (2^61-1)^2 - 2 = 2^122 - 2^62 - 1
    const uint64_t e_hi = (1ull << 58) - 1;            // bits 64..121 of 2^122 - 2^62 - 1
    const uint64_t e_lo = 0xBFFFFFFFFFFFFFFFull;       // low 64 bits
    fe r = fe_one();
    fe b = x;
    for (int i = 0; i < 64; ++i) {
        if ((e_lo >> i) & 1) r = r * b;
        b = b * b;
    }
    for (int i = 0; i < 58; ++i) {
        if ((e_hi >> i) & 1) r = r * b;
        b = b * b;
    }
    return r;
}

// Root of unity of order 2^log_order: the generator of the 2-adic subgroup of
// order 2^62 (real 2^31, img 1033321771269002680), squared 62 - log_order times.
// Same construction as the reference (src/linear_gkr/prime_field.cpp:60-73).
VG_HD fe fe_root_of_unity(int log_order)
{
    fe r = fe_make(2147483648ull, 1033321771269002680ull);
    for (int i = 0; i < 62 - log_order; ++i) r = r * r;
    return r;
}

}  // namespace vg
