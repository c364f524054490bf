// reference src/VPD/vpd_prover.cpp: the private oracle's initial commitment.
#include "VPD/vpd_prover.h"
#include "VPD/fri.h"

__hhash_digest merkle_root;

__hhash_digest vpd_prover_init(prime_field::field_element *l_eval, prime_field::field_element *&l_coef, int log_input_length,
                               int slice_size, int slice_count)
{
    (void)l_eval;
    (void)l_coef;
    (void)slice_size;
    (void)slice_count;
    merkle_root = fri::request_init_commit(log_input_length, 0);
    return merkle_root;
}
