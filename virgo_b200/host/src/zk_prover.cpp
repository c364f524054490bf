// zk_prover on the GPU.  Follows src/linear_gkr/zk_prover.cpp of the
// reference method by method: the gate-level work (evaluate, the phase-1 and
// phase-2 scatters, the per-round fold and sums, V_res) goes through the C ABI
// to the device; the O(bit length) mask and claim bookkeeping stays on the
// host, in the same order, drawing randomness in the same order.
#include "linear_gkr/zk_prover.h"
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include "device.h"
#include "internal.h"
#include "infrastructure/utility.h"

typedef prime_field::field_element F;
using clk = std::chrono::high_resolution_clock;

// 1/2 in F_p (the reference's global inv_2, zk_prover.cpp:23-28)
static const F inv_2 = prime_field::inv(F(2));

static inline vg_fe to_vg(const F &x)
{
    vg_fe r;
    r.img = x.img;
    r.real = x.real;
    return r;
}
static inline F from_vg(const vg_fe &x)
{
    F r;
    r.img = x.img;
    r.real = x.real;
    return r;
}
static inline double since(clk::time_point t0)
{
    return std::chrono::duration_cast<std::chrono::duration<double>>(clk::now() - t0).count();
}
// x doubled k times
static inline F dbl(F x, int k)
{
    for (int i = 0; i < k; ++i) x = x + x;
    return x;
}

zk_prover::zk_prover()
{
    memset(circuit_value, 0, sizeof circuit_value);
    maskpoly = nullptr;
    dev_ctx = nullptr;
    dev_circuit = nullptr;
    dev_gkr = nullptr;
    owns_circuit = false;
    quiet = false;
    total_time = 0;
    r_0 = r_1 = nullptr;
    one_minus_r_0 = one_minus_r_1 = nullptr;
    defer_mode = DEFER_OFF;
    replay = nullptr;
    replay_n = replay_i = 0;
}

zk_prover::~zk_prover() {}

void zk_prover::init_array(int max_bit_length)
{
    // device tables are sized from the circuit in get_circuit()
    (void)max_bit_length;
}

static void upload(const layered_circuit &C, vg_circuit **out)
{
    const int depth = C.total_depth;
    std::vector<int> bl(depth);
    std::vector<std::vector<uint8_t> > ty(depth);
    std::vector<std::vector<int64_t> > u(depth), v(depth);
    std::vector<const uint8_t *> pty(depth);
    std::vector<const int64_t *> pu(depth), pv(depth);
    for (int i = 0; i < depth; ++i) {
        bl[i] = C.circuit[i].bit_length;
        const long n = 1L << bl[i];
        ty[i].resize(n);
        u[i].resize(n);
        v[i].resize(n);
        const gate *g = C.circuit[i].gates;
        for (long k = 0; k < n; ++k) {
            ty[i][k] = (uint8_t)g[k].ty;
            u[i][k] = g[k].u;
            v[i][k] = g[k].v;
        }
        pty[i] = ty[i].data();
        pu[i] = u[i].data();
        pv[i] = v[i].data();
    }
    virgo::check(vg_circuit_upload(virgo::ctx(), depth, bl.data(), pty.data(), pu.data(), pv.data(), out), "vg_circuit_upload");
}

static vg_ctx *ctx_of(const zk_prover *p) { return p->dev_ctx ? p->dev_ctx : virgo::ctx(); }

void zk_prover::get_circuit(const layered_circuit &from_verifier)
{
    C = from_verifier;
    if (dev_gkr) vg_gkr_destroy(dev_gkr);
    if (dev_circuit && owns_circuit) vg_circuit_destroy(dev_circuit);
    dev_gkr = nullptr;
    upload(C, &dev_circuit);
    owns_circuit = true;
    virgo::check(vg_gkr_create(ctx_of(this), dev_circuit, &dev_gkr), "vg_gkr_create");
}

void zk_prover::attach_circuit(const layered_circuit &c, vg_circuit *dev, vg_ctx *ctx)
{
    C = c;
    const bool same_ctx = !ctx || ctx == dev_ctx;
    if (ctx) dev_ctx = ctx;
    if (dev_circuit && owns_circuit && dev_circuit != dev) vg_circuit_destroy(dev_circuit);
    dev_circuit = dev;
    owns_circuit = false;
    if (dev_gkr && same_ctx) {   // keep the device tables, grown if the circuit needs more
        virgo::check(vg_gkr_rebind(dev_gkr, dev_circuit), "vg_gkr_rebind");
        return;
    }
    if (dev_gkr) vg_gkr_destroy(dev_gkr);
    virgo::check(vg_gkr_create(ctx_of(this), dev_circuit, &dev_gkr), "vg_gkr_create");
}

void zk_prover::reset_proof()
{
    all_pri_mask.clear();
    maskr.clear();
    delete[] maskpoly;
    maskpoly = nullptr;
    total_time = 0;
    poly_prover.total_time = 0;
    for (int i = 0; i < 6; ++i) maskR[i] = preR[i] = F(0);
    maskR_sumcu = maskR_sumcv = preZu = preZv = Zu = Zv = preu1 = prev1 = Iuv = prepreu1 = preprev1 = F(0);
    Rg1 = Rg2 = sumRc = quadratic_poly(F(0), F(0), F(0));
    maskpoly_sumc = maskpoly_sumr = rho = v_u = v_v = alpha = beta = F(0);
}

void zk_prover::proof_init() {}

// zk_prover.cpp:54-157: all layers on the device
F *zk_prover::evaluate()
{
    auto t0 = clk::now();
    if (defer_mode != DEFER_REPLAY) virgo::check(vg_gkr_evaluate(dev_gkr), "vg_gkr_evaluate");
    for (int i = 0; i < C.total_depth; ++i) {
        const vg_fe *p;
        virgo::check(vg_gkr_layer_values(dev_gkr, i, &p), "vg_gkr_layer_values");
        circuit_value[i] = (F *)p;
    }
    if (!quiet) std::cerr << "total evaluation time: " << since(t0) << " seconds." << std::endl;
    return circuit_value[C.total_depth - 1];
}

// zk_prover.cpp:30-52: MLE of the outputs at r_0 (one_minus_r_0 is 1 - r_0)
F zk_prover::V_res(const F *one_minus_r_0, const F *r_0, const F *output_raw, int r_0_size, int output_size)
{
    (void)one_minus_r_0;
    auto t0 = clk::now();
    F res;
    std::vector<vg_fe> r(r_0_size);
    for (int i = 0; i < r_0_size; ++i) r[i] = to_vg(r_0[i]);
    vg_fe out{0, 0};
    if (defer_mode == DEFER_REPLAY) {
        if (replay_i >= replay_n) virgo::check(VG_ERR_STATE, "V_res: no recorded result");
        res = replay[9 * replay_i++];
        total_time += since(t0);
        return res;
    }
    if (output_raw == circuit_value[C.total_depth - 1] && output_size == (1 << C.circuit[C.total_depth - 1].bit_length)) {
        virgo::check(vg_gkr_v_res(dev_gkr, r.data(), r_0_size, &out), "vg_gkr_v_res");
    } else {
        virgo::check(vg_mle_eval(ctx_of(this), (const vg_fe *)output_raw, output_size, r.data(), r_0_size, &out), "vg_mle_eval");
    }
    res = from_vg(out);
    total_time += since(t0);
    return res;
}

// zk_prover.cpp:162-172
void zk_prover::generate_maskpoly_pre_rho(int length, int degree)
{
    delete[] maskpoly;
    const int n = length * degree + 1 + 6;   // the last 6 are the u_n, v_n terms of degree 3..5
    maskpoly = new F[n];
    for (int i = 0; i < n; ++i) {
        maskpoly[i] = prime_field::random();
        all_pri_mask.push_back(maskpoly[i]);
    }
}

// zk_prover.cpp:174-188: scale by rho; the sum of the mask polynomial over
// the hypercube (constant term counted 2^length times)
void zk_prover::generate_maskpoly_after_rho(int length, int degree)
{
    const int n = length * degree + 1 + 6;
    for (int i = 0; i < n; ++i) maskpoly[i] = maskpoly[i] * rho;
    maskpoly_sumc = maskpoly[length * degree];
    for (int i = length * degree; i >= 0; --i) maskpoly_sumc = maskpoly_sumc + maskpoly[i];
    for (int i = 1; i <= 6; ++i) maskpoly_sumc = maskpoly_sumc + maskpoly[length * degree + i];
    maskpoly_sumc = dbl(maskpoly_sumc, length - 1);
    maskpoly_sumr = F(0);
}

// zk_prover.cpp:192-255: R(z, c) = a0 + a1 z + a2 z^2 + a3 c + a4 c^2 + a5 z c
void zk_prover::generate_maskR(int layer_id)
{
    for (int i = 0; i < 6; ++i) all_pri_mask.push_back(maskR[i]);
    prepreu1 = preu1;
    preprev1 = prev1;
    for (int i = 0; i < 6; ++i) preR[i] = maskR[i];
    Rg1.a = maskR[4];
    Rg1.b = maskR[3] + maskR[5] * preu1;
    Rg1.c = maskR[0] + maskR[1] * preu1 + maskR[2] * preu1 * preu1;
    Rg2.a = maskR[4];
    Rg2.b = maskR[3] + maskR[5] * prev1;
    Rg2.c = maskR[0] + maskR[1] * prev1 + maskR[2] * prev1 * prev1;
    F sumRu = Rg1.a + Rg1.b + Rg1.c + Rg1.c;
    F sumRv = Rg2.a + Rg2.b + Rg2.c + Rg2.c;
    maskR_sumcu = alpha * Zu * sumRu;
    maskR_sumcv = beta * Zv * sumRv;
    preZu = Zu;
    preZv = Zv;
    Zu = F(1);
    Zv = F(1);
    Iuv = F(1);
    if (layer_id > 1) {
        for (int i = 0; i < 6; ++i) maskR[i] = prime_field::random();
        sumRc.a = maskR[2] + maskR[2];
        sumRc.b = maskR[1] + maskR[1] + maskR[5];
        sumRc.c = maskR[0] + maskR[0] + maskR[3] + maskR[4];
    }
    maskr.resize(2);
    maskr[0] = prime_field::random();
    maskr[1] = prime_field::random();
    if (layer_id == 1) {   // input layer: R is the linear a + b x
        maskR[0] = maskr[0];
        maskR[1] = maskr[1];
        maskR[2] = maskR[3] = maskR[4] = maskR[5] = F(0);
        sumRc.a = F(0);
        sumRc.b = maskR[1];
        sumRc.c = maskR[0];
    }
}

// zk_prover.cpp:284-306
F zk_prover::query(F *u, F *v, F r_c)
{
    const int m = 2 * (length_u + length_v + 1);
    F result(0);
    for (int i = 0; i < length_u; ++i) {
        result = result + maskpoly[2 * i] * u[i] * u[i] + maskpoly[2 * i + 1] * u[i];
        if (i == length_u - 1) {
            F x = u[i], x3 = x * x * x;
            result = result + maskpoly[m + 1] * x3 * x * x;
            result = result + maskpoly[m + 2] * x3 * x;
            result = result + maskpoly[m + 3] * x3;
        }
    }
    for (int i = 0; i < length_v; ++i) {
        result = result + maskpoly[2 * (i + length_u)] * v[i] * v[i] + maskpoly[2 * (i + length_u) + 1] * v[i];
        if (i == length_v - 1) {
            F x = v[i], x3 = x * x * x;
            result = result + maskpoly[m + 4] * x3 * x * x;
            result = result + maskpoly[m + 5] * x3 * x;
            result = result + maskpoly[m + 6] * x3;
        }
    }
    result = result + maskpoly[2 * (length_u + length_v)] * r_c * r_c + maskpoly[2 * (length_u + length_v) + 1] * r_c;
    result = result + maskpoly[m];
    return result;
}

F zk_prover::queryRg1(F r_c) { return Rg1.eval(r_c); }
F zk_prover::queryRg2(F r_c) { return Rg2.eval(r_c); }

// zk_prover.cpp:317-333
void zk_prover::sumcheck_init(int layer_id, int bit_length_g, int bit_length_u, int bit_length_v, const F &a, const F &b,
                              const F *R_0, const F *R_1, F *o_r_0, F *o_r_1)
{
    r_0 = R_0;
    r_1 = R_1;
    alpha = a;
    beta = b;
    sumcheck_layer_id = layer_id;
    length_g = bit_length_g;
    length_u = bit_length_u;
    length_v = bit_length_v;
    one_minus_r_0 = o_r_0;
    one_minus_r_1 = o_r_1;
    generate_maskR(layer_id);
}

// zk_prover.cpp:375-592 on the device
void zk_prover::sumcheck_phase1_init()
{
    auto t0 = clk::now();
    total_uv = 1 << C.circuit[sumcheck_layer_id - 1].bit_length;
    if (defer_mode == DEFER_REPLAY) return;
    std::vector<vg_fe> a(length_g), b(length_g);
    for (int i = 0; i < length_g; ++i) {
        a[i] = to_vg(r_0[i]);
        b[i] = to_vg(r_1[i]);
    }
    virgo::check(vg_gkr_phase1_init(dev_gkr, sumcheck_layer_id, a.data(), b.data(), length_g, to_vg(alpha), to_vg(beta)),
                 "vg_gkr_phase1_init");
    total_time += since(t0);
}

// one device round: the three sums of the array loop, and the folded tables
// when two entries remain (deferred modes: enqueue only, or the recorded result)
static quadratic_poly device_round(zk_prover *p, const F &r, int bit, F *last6)
{
    if (p->defer_mode == zk_prover::DEFER_LAUNCH) {
        virgo::check(vg_gkr_round(p->dev_gkr, to_vg(r), bit, nullptr, nullptr), "vg_gkr_round");
        if (last6)
            for (int k = 0; k < 6; ++k) last6[k] = F(0);
        return quadratic_poly(F(0), F(0), F(0));
    }
    if (p->defer_mode == zk_prover::DEFER_REPLAY) {
        if (p->replay_i >= p->replay_n) virgo::check(VG_ERR_STATE, "sumcheck round: no recorded result");
        const F *rec = p->replay + 9 * p->replay_i++;
        if (last6)
            for (int k = 0; k < 6; ++k) last6[k] = rec[3 + k];
        return quadratic_poly(rec[0], rec[1], rec[2]);
    }
    vg_gkr *g = p->dev_gkr;
    vg_fe s[3], l6[6];
    virgo::check(vg_gkr_round(g, to_vg(r), bit, s, last6 ? l6 : nullptr), "vg_gkr_round");
    if (last6)
        for (int k = 0; k < 6; ++k) last6[k] = from_vg(l6[k]);
    return quadratic_poly(from_vg(s[0]), from_vg(s[1]), from_vg(s[2]));
}

// zk_prover.cpp:596-678
quadratic_poly zk_prover::sumcheck_phase1_update(F previous_random, int current_bit)
{
    auto t0 = clk::now();
    quadratic_poly ret = device_round(this, previous_random, current_bit, nullptr);
    total_uv >>= 1;
    const F one(1), omr = one - previous_random;
    Iuv = Iuv * omr;
    if (current_bit > 0) {
        maskR_sumcu = maskR_sumcu * omr;
        maskR_sumcv = maskR_sumcv * omr;
        Zu = Zu * omr * previous_random;
    }
    ret.b = ret.b - maskR_sumcu - maskR_sumcv;
    ret.c = ret.c + maskR_sumcu + maskR_sumcv;

    const int k = length_u + length_v - current_bit;
    F tmp1 = dbl(maskpoly[current_bit << 1], k);
    F tmp2 = dbl(maskpoly[(current_bit << 1) + 1], k);
    maskpoly_sumc = (maskpoly_sumc - tmp1 - tmp2) * inv_2;
    F tmp3;
    if (current_bit > 0) {
        maskpoly_sumr = maskpoly_sumr + maskpoly[(current_bit << 1) - 2] * previous_random * previous_random +
                        maskpoly[(current_bit << 1) - 1] * previous_random;
        tmp3 = dbl(maskpoly_sumr, k);
    }
    ret.a = ret.a + tmp1;
    ret.b = ret.b + tmp2;
    ret.c = ret.c + maskpoly_sumc + tmp3;
    total_time += since(t0);
    return ret;
}

// the extra terms of the last round: Z(x) (a x^2 + b x + c) ((d - e) x + e)
// with d, e the folded add_mult_sum pair (zk_prover.cpp:736-747, 1122-1133)
static void last_bit_terms(quadratic_poly &ret, F &rd, F &re, F &rf, const quadratic_poly &sumRc, const F &am0,
                           const F &am1, const F &Z)
{
    const F a = sumRc.a, b = sumRc.b, c = sumRc.c;
    const F d = am1 - am0, e = am0;   // add_mult_sum[0].a, .b
    rd = (F(0) - a) * d * Z;
    re = (a * (d - e) - b * d) * Z;
    rf = (a * e + b * (d - e) - c * d) * Z;
    ret.a = ret.a + (c * (d - e) + b * e) * Z;
    ret.b = ret.b + c * e * Z;
}

// zk_prover.cpp:680-787
quintuple_poly zk_prover::sumcheck_phase1_updatelastbit(F previous_random, int current_bit)
{
    auto t0 = clk::now();
    quadratic_poly ret = device_round(this, previous_random, current_bit, tables_last);
    total_uv >>= 1;
    const F one(1), omr = one - previous_random;
    Iuv = Iuv * omr;
    if (current_bit > 0) {
        maskR_sumcv = maskR_sumcv * omr;
        maskR_sumcu = maskR_sumcu * omr;
        Zu = Zu * omr * previous_random;
    }
    ret.b = ret.b - maskR_sumcu - maskR_sumcv;
    ret.c = ret.c + maskR_sumcu + maskR_sumcv;
    F rd(0), re(0), rf(0);
    if (current_bit == length_u - 1) last_bit_terms(ret, rd, re, rf, sumRc, tables_last[4], tables_last[5], Zu);

    const int m = (length_u + length_v + 1) << 1;
    const int k = length_u + length_v - current_bit;
    F tmp1 = dbl(maskpoly[current_bit << 1], k);
    F tmp2 = dbl(maskpoly[(current_bit << 1) + 1], k);
    F tmp4 = dbl(maskpoly[m + 1], k);
    F tmp5 = dbl(maskpoly[m + 2], k);
    F tmp6 = dbl(maskpoly[m + 3], k);
    maskpoly_sumc = (maskpoly_sumc - tmp1 - tmp2 - tmp4 - tmp5 - tmp6) * inv_2;
    F tmp3;
    if (current_bit > 0) {
        maskpoly_sumr = maskpoly_sumr + maskpoly[(current_bit << 1) - 2] * previous_random * previous_random +
                        maskpoly[(current_bit << 1) - 1] * previous_random;
        tmp3 = dbl(maskpoly_sumr, k);
    }
    ret.a = ret.a + tmp1;
    ret.b = ret.b + tmp2;
    ret.c = ret.c + maskpoly_sumc + tmp3;
    rd = rd + tmp4;
    re = re + tmp5;
    rf = rf + tmp6;
    total_time += since(t0);
    return quintuple_poly(rd, re, rf, ret.a, ret.b, ret.c);
}

// zk_prover.cpp:789-983
void zk_prover::sumcheck_phase2_init(F previous_random, const F *r_u, const F *one_minus_r_u)
{
    (void)one_minus_r_u;
    auto t0 = clk::now();
    const F one(1), omr = one - previous_random;
    preu1 = previous_random;
    maskR_sumcu = maskR_sumcu * omr;
    maskR_sumcv = maskR_sumcv * omr;
    Iuv = Iuv * omr;
    // V_mult_add[0].eval(r): the folded pair of the last phase-1 round
    Zu = Zu * omr * previous_random;
    const F addend = Zu * sumRc.eval(previous_random);
    v_u = tables_last[0] + previous_random * (tables_last[1] - tables_last[0]) + addend;

    std::vector<vg_fe> ru(length_u);
    for (int i = 0; i < length_u; ++i) ru[i] = to_vg(r_u[i]);
    if (defer_mode == DEFER_LAUNCH)   // v_u is formed on the device from the recorded pair
        virgo::check(vg_gkr_phase2_init_deferred(dev_gkr, ru.data(), length_u, to_vg(previous_random), to_vg(addend)),
                     "vg_gkr_phase2_init");
    else if (defer_mode == DEFER_OFF)
        virgo::check(vg_gkr_phase2_init(dev_gkr, ru.data(), length_u, to_vg(v_u)), "vg_gkr_phase2_init");
    total_uv = 1 << C.circuit[sumcheck_layer_id - 1].bit_length;

    const int m = (length_u + length_v + 1) * 2;
    const F r = previous_random, r2 = r * r, r3 = r2 * r;
    maskpoly_sumr = maskpoly_sumr + maskpoly[length_u * 2 - 2] * r2 + maskpoly[length_u * 2 - 1] * r;
    maskpoly_sumr = maskpoly_sumr + maskpoly[m + 1] * r3 * r2;
    maskpoly_sumr = maskpoly_sumr + maskpoly[m + 2] * r3 * r;
    maskpoly_sumr = maskpoly_sumr + maskpoly[m + 3] * r3;
    total_time += since(t0);
}

// zk_prover.cpp:988-1069
quadratic_poly zk_prover::sumcheck_phase2_update(F previous_random, int current_bit)
{
    auto t0 = clk::now();
    quadratic_poly ret = device_round(this, previous_random, current_bit, nullptr);
    total_uv >>= 1;
    const F one(1), omr = one - previous_random;
    if (current_bit > 0) {
        Iuv = Iuv * omr;
        maskR_sumcu = maskR_sumcu * omr;
        maskR_sumcv = maskR_sumcv * omr;
        Zv = Zv * omr * previous_random;
    }
    ret.b = ret.b - maskR_sumcu - maskR_sumcv;
    ret.c = ret.c + maskR_sumcu + maskR_sumcv;

    const int current = current_bit + length_u;
    const int k = length_u + length_v - current;
    F tmp1 = dbl(maskpoly[current << 1], k);
    F tmp2 = dbl(maskpoly[(current << 1) + 1], k);
    maskpoly_sumc = (maskpoly_sumc - tmp1 - tmp2) * inv_2;
    maskpoly_sumr = maskpoly_sumr + maskpoly[(current << 1) - 2] * previous_random * previous_random +
                    maskpoly[(current << 1) - 1] * previous_random;
    F tmp3 = dbl(maskpoly_sumr, k);
    ret.a = ret.a + tmp1;
    ret.b = ret.b + tmp2;
    ret.c = ret.c + maskpoly_sumc + tmp3;
    total_time += since(t0);
    return ret;
}

// zk_prover.cpp:1071-1171
quintuple_poly zk_prover::sumcheck_phase2_updatelastbit(F previous_random, int current_bit)
{
    auto t0 = clk::now();
    quadratic_poly ret = device_round(this, previous_random, current_bit, tables_last);
    total_uv >>= 1;
    const F one(1), omr = one - previous_random;
    Iuv = Iuv * omr;
    if (current_bit > 0) {
        maskR_sumcu = maskR_sumcu * omr;
        maskR_sumcv = maskR_sumcv * omr;
        Zv = Zv * omr * previous_random;
    }
    ret.b = ret.b - maskR_sumcu - maskR_sumcv;
    ret.c = ret.c + maskR_sumcu + maskR_sumcv;
    F rd(0), re(0), rf(0);
    if (current_bit == length_v - 1) last_bit_terms(ret, rd, re, rf, sumRc, tables_last[4], tables_last[5], Zv);

    const int current = current_bit + length_u;
    const int m = (length_u + length_v + 1) * 2;
    const int k = length_u + length_v - current;
    F tmp1 = dbl(maskpoly[current << 1], k);
    F tmp2 = dbl(maskpoly[(current << 1) + 1], k);
    F tmp4 = dbl(maskpoly[m + 4], k);
    F tmp5 = dbl(maskpoly[m + 5], k);
    F tmp6 = dbl(maskpoly[m + 6], k);
    maskpoly_sumc = (maskpoly_sumc - tmp1 - tmp2 - tmp4 - tmp5 - tmp6) * inv_2;
    maskpoly_sumr = maskpoly_sumr + maskpoly[(current << 1) - 2] * previous_random * previous_random +
                    maskpoly[(current << 1) - 1] * previous_random;
    F tmp3 = dbl(maskpoly_sumr, k);
    rd = rd + tmp4;
    re = re + tmp5;
    rf = rf + tmp6;
    ret.a = ret.a + tmp1;
    ret.b = ret.b + tmp2;
    ret.c = ret.c + maskpoly_sumc + tmp3;
    total_time += since(t0);
    return quintuple_poly(rd, re, rf, ret.a, ret.b, ret.c);
}

// zk_prover.cpp:1173-1203 (host only)
quadratic_poly zk_prover::sumcheck_finalround(F previous_random, int current, F general_value)
{
    quadratic_poly ret(F(0), F(0), F(0));
    ret.a = Iuv * preZu * Rg1.a * alpha + Iuv * preZv * Rg2.a * beta;
    ret.b = Iuv * preZu * Rg1.b * alpha + Iuv * preZv * Rg2.b * beta + general_value;
    ret.c = Iuv * preZu * Rg1.c * alpha + Iuv * preZv * Rg2.c * beta;
    const int k = length_u + length_v - current;
    F tmp1 = dbl(maskpoly[current << 1], k);
    F tmp2 = dbl(maskpoly[(current << 1) + 1], k);
    maskpoly_sumc = (maskpoly_sumc - tmp1 - tmp2) * inv_2;
    const F r = previous_random, r2 = r * r, r3 = r2 * r;
    const int m = (length_u + length_v + 1) * 2;
    maskpoly_sumr = maskpoly_sumr + maskpoly[(current << 1) - 2] * r2 + maskpoly[(current << 1) - 1] * r;
    maskpoly_sumr = maskpoly_sumr + maskpoly[m + 4] * r3 * r2;
    maskpoly_sumr = maskpoly_sumr + maskpoly[m + 5] * r3 * r;
    maskpoly_sumr = maskpoly_sumr + maskpoly[m + 6] * r3;
    F tmp3 = dbl(maskpoly_sumr, k);
    ret.a = ret.a + tmp1;
    ret.b = ret.b + tmp2;
    ret.c = ret.c + maskpoly_sumc + tmp3;
    return ret;
}

// zk_prover.cpp:1206-1215
std::pair<F, F> zk_prover::sumcheck_finalize(F previous_random)
{
    const F one(1), omr = one - previous_random;
    prev1 = previous_random;
    Iuv = Iuv * omr;
    v_v = tables_last[0] + previous_random * (tables_last[1] - tables_last[0]);
    Zv = Zv * omr * previous_random;
    v_v = v_v + Zv * sumRc.eval(previous_random);
    return std::make_pair(v_u, v_v);
}

void zk_prover::delete_self()
{
    if (dev_gkr) vg_gkr_destroy(dev_gkr);
    dev_gkr = nullptr;
    if (dev_circuit && owns_circuit) vg_circuit_destroy(dev_circuit);
    dev_circuit = nullptr;
    for (int i = 0; i < C.total_depth && i < 1000000; ++i) circuit_value[i] = nullptr;
    delete[] maskpoly;
    maskpoly = nullptr;
}
