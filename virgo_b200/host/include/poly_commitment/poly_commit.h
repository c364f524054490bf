// Polynomial (vector) commitment with the reference's interface
// (include/poly_commitment/poly_commit.h, include/poly_commitment/README.md).
// The reference defines the prover methods inline in this header; here they
// are ordinary declarations implemented on the GPU, so the reference verifier
// sources compile unchanged against this header.
//
// The namespace-scope sizes keep the reference's names and meaning.  The
// evaluation arrays themselves live on the device; l_eval and h_eval_arr
// here are host pointers that stay NULL (the FRI query functions read the
// device copies).
#pragma once
#ifndef __poly_commit
#define __poly_commit
#include <algorithm>
#include <chrono>
#include <vector>
#include "infrastructure/RS_polynomial.h"
#include "infrastructure/utility.h"
#include "VPD/fri.h"
#include "VPD/vpd_prover.h"

namespace poly_commit
{
extern prime_field::field_element *all_pri_msk_arr;
extern prime_field::field_element *all_pub_msk_arr;
extern prime_field::field_element *inner_prod_evals;
extern prime_field::field_element *l_coef, *l_eval, *q_coef, *q_eval;
extern prime_field::field_element *lq_eval, *h_coef, *lq_coef, *h_eval;
extern prime_field::field_element *h_eval_arr;
extern int l_coef_len, l_eval_len, q_coef_len, q_eval_len;
extern int slice_size, slice_count, slice_real_ele_cnt;
extern int mask_position_gap;
extern bool pre_prepare_executed;

class ldt_commitment
{
public:
    __hhash_digest *commitment_hhash;
    prime_field::field_element *randomness;
    prime_field::field_element *final_rs_code;
    int mx_depth;
    int repeat_no;
};

class poly_commit_prover
{
public:
    double total_time;
    std::vector<prime_field::field_element> all_pri_mask;
    // RS-encodes 64 slices of private_array (2^log_array_length elements, host
    // or device memory) and the zero-padded mask at rate 1/32, then commits
    // (poly_commit.h:42-124 of the reference).  Returns the Merkle root.
    __hhash_digest commit_private_array(prime_field::field_element *private_array, int log_array_length,
                                        std::vector<prime_field::field_element> private_mask_array);
    // Commits the public side: RS codes of the public array and public mask,
    // the quotient h and the virtual oracle; pads all_pub_msk with zeros to
    // the private mask length, writes all_sum[0..slice_number] and asserts the
    // inner product equals target_sum (poly_commit.h:125-351).  Returns h's root.
    __hhash_digest commit_public_array(std::vector<prime_field::field_element> &all_pub_msk,
                                       prime_field::field_element *public_array, int r_0_len,
                                       prime_field::field_element target_sum, prime_field::field_element *all_sum);
    // The FRI folding rounds with verifier randomness (src/VPD/vpd_verifier.cpp:46-78).
    ldt_commitment commit_phase(int log_length);
};

class poly_commit_verifier
{
public:
    poly_commit_prover *p;
    bool verify_poly_commitment(prime_field::field_element *all_sum, int log_length, prime_field::field_element *public_array,
                                std::vector<prime_field::field_element> &all_pub_mask, double &v_time, int &proof_size,
                                double &p_time, __hhash_digest merkle_tree_l, __hhash_digest merkle_tree_h);
};
}  // namespace poly_commit
#endif
