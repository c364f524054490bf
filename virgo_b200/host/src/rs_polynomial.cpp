// fast_fourier_transform / inverse_fast_fourier_transform with the reference's
// interface (src/infrastructure/RS_polynomial.cpp:27-240), computed by vg_ntt.
#include "infrastructure/RS_polynomial.h"
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "device.h"

typedef prime_field::field_element F;

void init_scratch_pad(int order) { (void)order; }

static vg_fe V(const F &x)
{
    vg_fe r;
    r.real = x.real;
    r.img = x.img;
    return r;
}

static int lg(long long x)
{
    int k = 0;
    while ((1LL << k) < x) ++k;
    return (1LL << k) == x ? k : -1;
}

// out[i] = sum_k in[k] root^(ik), i < order, on the device; in/out host or device
static void run_ntt(const F *in, int in_len, int order, F root, F *out, bool scale)
{
    const int lo = lg(order);
    if (lo < 0 || lg(in_len) < 0 || in_len > order) {
        fprintf(stderr, "fast_fourier_transform: sizes %d, %d must be powers of two with coef_len <= order\n", in_len, order);
        abort();
    }
    vg_ctx *c = virgo::ctx();
    const bool din = virgo::is_device_ptr(in), dout = virgo::is_device_ptr(out);
    void *bi = nullptr, *bo = nullptr;
    const vg_fe *src = (const vg_fe *)in;
    vg_fe *dst = (vg_fe *)out;
    if (!din) {
        virgo::check(vg_dev_alloc(c, (size_t)in_len * sizeof(F), &bi), "vg_dev_alloc");
        virgo::check(vg_h2d(c, bi, in, (size_t)in_len * sizeof(F)), "vg_h2d");
        src = (const vg_fe *)bi;
    }
    if (!dout) {
        virgo::check(vg_dev_alloc(c, (size_t)order * sizeof(F), &bo), "vg_dev_alloc");
        dst = (vg_fe *)bo;
    }
    virgo::check(vg_ntt(c, src, in_len, in_len, dst, lo, order, 1, V(root), scale ? 1 : 0), "vg_ntt");
    if (!dout) virgo::check(vg_d2h(c, out, bo, (size_t)order * sizeof(F)), "vg_d2h");
    else virgo::check(vg_ctx_sync(c), "vg_ctx_sync");
    if (bi) vg_dev_free(c, bi);
    if (bo) vg_dev_free(c, bo);
}

void fast_fourier_transform(const F *coefficients, int coef_len, int order, F root_of_unity, F *result)
{
    run_ntt(coefficients, coef_len, order, root_of_unity, result, false);
}

void inverse_fast_fourier_transform(F *evaluations, int coef_len, int order, F root_of_unity, F *dst)
{
    if (coef_len > order) {
        fprintf(stderr, "Warning, Request do inverse fft with inefficient number of evaluations.");
        fprintf(stderr, "Will construct a polynomial with less order than required.");
        coef_len = order;
    }
    const int step = order / coef_len;
    // root of order coef_len and its inverse as the reference forms them
    // (RS_polynomial.cpp:209-236): new_rou = root^step, inverse = new_rou^(coef_len - 1)
    F new_rou(1);
    for (int i = 0; i < step; ++i) new_rou = new_rou * root_of_unity;
    F inv_rou(1), t = new_rou;
    for (int i = 0; i < lg(coef_len); ++i) {
        inv_rou = inv_rou * t;
        t = t * t;
    }
    if (step == 1) {
        run_ntt(evaluations, coef_len, coef_len, inv_rou, dst, true);
        return;
    }
    std::vector<F> sub(coef_len);
    if (virgo::is_device_ptr(evaluations)) {
        std::vector<F> all(order);
        virgo::check(vg_d2h(virgo::ctx(), all.data(), evaluations, (size_t)order * sizeof(F)), "vg_d2h");
        for (int i = 0; i < coef_len; ++i) sub[i] = all[(long)i * step];
    } else {
        for (int i = 0; i < coef_len; ++i) sub[i] = evaluations[(long)i * step];
    }
    run_ntt(sub.data(), coef_len, coef_len, inv_rou, dst, true);
}
