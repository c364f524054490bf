// FRI commit phase and query answers with the reference's interface
// (include/VPD/fri.h:9-101).  Codewords and Merkle trees stay on the GPU.
// What the reference verifier reads directly is mirrored on the host:
//   cpd.rs_codeword[t] / cpd.rs_codeword_msk[t] for the final level t (in the
//   reference's interleaved layout, filled by commit_phase_final),
//   witness_merkle[k][1] and cpd.merkle[t][1] (the roots; other entries of
//   these two-entry host arrays are unused).
#ifndef __fri
#define __fri
#include "infrastructure/merkle_tree.h"
#include <utility>
#include "linear_gkr/prime_field.h"
#include "infrastructure/constants.h"
#include <vector>

namespace fri
{
class commit_phase_data
{
public:
    __hhash_digest *merkle[max_fri_depth];
    int merkle_size[max_fri_depth];
    prime_field::field_element *rs_codeword[max_fri_depth], *poly_coef[max_fri_depth];
    prime_field::field_element *rs_codeword_msk[max_fri_depth];
    int *rs_codeword_mapping[max_fri_depth], *rs_codeword_msk_mapping[max_fri_depth];
    commit_phase_data()
    {
        for (int i = 0; i < max_fri_depth; ++i) {
            merkle[i] = NULL;
            rs_codeword[i] = NULL;
            poly_coef[i] = NULL;
            rs_codeword_msk[i] = NULL;
            rs_codeword_mapping[i] = NULL;
            rs_codeword_msk_mapping[i] = NULL;
            merkle_size[i] = 0;
        }
    }
    void delete_self()
    {
        for (int i = 0; i < max_fri_depth; ++i) {
            delete[] merkle[i];
            delete[] rs_codeword[i];
            delete[] poly_coef[i];
            delete[] rs_codeword_msk[i];
            delete[] rs_codeword_mapping[i];
            delete[] rs_codeword_msk_mapping[i];
            merkle[i] = NULL;
            rs_codeword[i] = NULL;
            poly_coef[i] = NULL;
            rs_codeword_msk[i] = NULL;
            rs_codeword_mapping[i] = NULL;
            rs_codeword_msk_mapping[i] = NULL;
            merkle_size[i] = 0;
        }
    }
    ~commit_phase_data() { delete_self(); }
};
extern int log_current_witness_size_per_slice, current_step_no, witness_bit_length_per_slice;
extern commit_phase_data cpd;
extern double __fri_timer;
extern __hhash_digest *witness_merkle[2];

// Merkle root of the initial codeword of oracle 0 (private, from
// poly_commit::l_eval) or 1 (public quotient h, from poly_commit::h_eval_arr).
__hhash_digest request_init_commit(const int bit_len, const int oracle_indicator);
// The 65 value pairs at w^pow_0, w^pow_1 (pow_1 = pow_0 + S/2) and the Merkle
// path; adds the newly revealed bytes to new_size (reference accounting).
std::pair<std::vector<std::pair<prime_field::field_element, prime_field::field_element> >, std::vector<__hhash_digest> >
request_init_value_with_merkle(long long pow_0, long long pow_1, int &new_size, const int oracle_indicator);
// The 65 value pairs of FRI level lvl at position pow (and its conjugate) with
// the Merkle path; adds the newly revealed bytes to new_size.
std::pair<std::vector<std::pair<prime_field::field_element, prime_field::field_element> >, std::vector<__hhash_digest> >
request_step_commit(int lvl, long long pow, int &new_size);
// Folds the current codeword with r and commits the result; returns its root.
__hhash_digest commit_phase_step(prime_field::field_element r);
// The final (constant-size) codeword, host memory, reference layout.
prime_field::field_element *commit_phase_final();
void delete_self();
}  // namespace fri

#endif
