// poly_commit::poly_commit_prover on the GPU (reference
// include/poly_commitment/poly_commit.h:42-351 and the prover half of
// src/VPD/vpd_verifier.cpp:46-78).
#include "poly_commitment/poly_commit.h"
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include "device.h"

typedef prime_field::field_element F;
using clk = std::chrono::high_resolution_clock;

namespace poly_commit
{
F *all_pri_msk_arr = nullptr, *all_pub_msk_arr = nullptr, *inner_prod_evals = nullptr;
F *l_coef = nullptr, *l_eval = nullptr, *q_coef = nullptr, *q_eval = nullptr;
F *lq_eval = nullptr, *h_coef = nullptr, *lq_coef = nullptr, *h_eval = nullptr;
F *h_eval_arr = nullptr;
int l_coef_len = 0, l_eval_len = 0, q_coef_len = 0, q_eval_len = 0;
int slice_size = 0, slice_count = 0, slice_real_ele_cnt = 0;
int mask_position_gap = 0;
bool pre_prepare_executed = false;
}  // namespace poly_commit

static double since(clk::time_point t0)
{
    return std::chrono::duration_cast<std::chrono::duration<double>>(clk::now() - t0).count();
}

__hhash_digest poly_commit::poly_commit_prover::commit_private_array(F *private_array, int log_array_length,
                                                                     std::vector<F> private_mask_array)
{
    total_time = 0;
    auto t0 = clk::now();
    if (private_mask_array.empty()) {
        // the reference divides by the mask count here (poly_commit.h:56)
        fprintf(stderr, "commit_private_array: the mask vector must not be empty\n");
        abort();
    }
    pre_prepare_executed = true;
    slice_count = (1 << log_slice_number) + 1;   // 64 data slices and one mask slice
    slice_size = 1 << (log_array_length + rs_code_rate - log_slice_number);
    slice_real_ele_cnt = slice_size >> rs_code_rate;
    l_eval_len = slice_count * slice_size;
    // masks sit every mask_position_gap positions, a power of two
    long gap = slice_size / (long)private_mask_array.size(), g = 1;
    while (g * 2 <= gap) g *= 2;
    mask_position_gap = (int)g;
    const long padded = slice_size / mask_position_gap;
    while ((long)private_mask_array.size() < padded) private_mask_array.push_back(F(0));
    all_pri_mask = private_mask_array;

    long M = 0;
    virgo::check(vg_pc_encode_private(virgo::pc(), (const vg_fe *)private_array, log_array_length,
                                      (const vg_fe *)private_mask_array.data(), (long)private_mask_array.size(), &M),
                 "vg_pc_encode_private");
    auto ret = vpd_prover_init(l_eval, l_coef, log_array_length, slice_size, slice_count);
    total_time += since(t0);
    return ret;
}

__hhash_digest poly_commit::poly_commit_prover::commit_public_array(std::vector<F> &all_pub_msk, F *public_array, int r_0_len,
                                                                    F target_sum, F *all_sum)
{
    auto t0 = clk::now();
    if (!pre_prepare_executed) {
        fprintf(stderr, "commit_public_array called before commit_private_array\n");
        abort();
    }
    if ((slice_count - 1) * slice_real_ele_cnt != (1 << r_0_len)) {
        fprintf(stderr, "commit_public_array: public array length 2^%d does not match the private commitment\n", r_0_len);
        abort();
    }
    const long padded = slice_size / mask_position_gap;
    if ((long)all_pri_mask.size() > padded || (long)all_pub_msk.size() > padded) {
        fprintf(stderr, "commit_public_array: more public masks (%zu) than committed mask positions (%ld)\n",
                all_pub_msk.size(), padded);
        abort();
    }
    while ((long)all_pub_msk.size() < padded) all_pub_msk.push_back(F(0));   // the caller sees the padding
    vg_fe sums[slice_number + 1], inner;
    virgo::check(vg_pc_encode_public(virgo::pc(), (const vg_fe *)public_array, (const vg_fe *)all_pub_msk.data(),
                                     (long)all_pub_msk.size(), sums, &inner),
                 "vg_pc_encode_public");
    for (int i = 0; i <= slice_number; ++i) {
        all_sum[i].real = sums[i].real;
        all_sum[i].img = sums[i].img;
    }
    if (inner.real != target_sum.real || inner.img != target_sum.img) {
        // poly_commit.h:193 asserts the claimed inner product
        fprintf(stderr, "commit_public_array: inner product does not match the target sum\n");
        abort();
    }
    total_time += since(t0);
    t0 = clk::now();
    auto ret = fri::request_init_commit(r_0_len, 1);
    total_time += since(t0);
    return ret;
}

// FRI folding with verifier randomness until the codeword of a slice has
// 2^rs_code_rate entries (vpd_verifier.cpp:46-78)
poly_commit::ldt_commitment poly_commit::poly_commit_prover::commit_phase(int log_length)
{
    auto t0 = clk::now();
    const int saved = fri::log_current_witness_size_per_slice;
    int codeword_size = 1 << (log_length + rs_code_rate - log_slice_number);
    __hhash_digest *roots = new __hhash_digest[log_length + rs_code_rate - log_slice_number];
    F *randomness = new F[log_length + rs_code_rate];
    int depth = 0;
    while (codeword_size > (1 << rs_code_rate)) {
        randomness[depth] = prime_field::random();
        roots[depth] = fri::commit_phase_step(randomness[depth]);
        codeword_size /= 2;
        ++depth;
    }
    ldt_commitment com;
    com.commitment_hhash = roots;
    com.final_rs_code = fri::commit_phase_final();
    com.randomness = randomness;
    com.mx_depth = depth;
    com.repeat_no = 0;
    fri::log_current_witness_size_per_slice = saved;
    const double dt = since(t0);
    total_time += dt;
    printf("Commit time %lf\n", dt);
    return com;
}
