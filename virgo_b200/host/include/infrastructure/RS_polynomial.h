// Reed-Solomon / FFT interface of the reference (include/infrastructure/RS_polynomial.h),
// computed on the GPU (vg_ntt).  Arrays are host memory, or device memory
// obtained from this library.
#ifndef __RS_polynomial
#define __RS_polynomial

#include "my_hhash.h"
#include "merkle_tree.h"
#include "linear_gkr/prime_field.h"
#include <cassert>
#include "infrastructure/constants.h"

// Kept for interface compatibility: device scratch is managed by the library.
void init_scratch_pad(int order);

// result[i] = sum_k coefficients[k] * root^(i k), i < order (natural order);
// root must have order `order`, coef_len <= order.
void fast_fourier_transform(const prime_field::field_element *coefficients, int coef_len, int order,
                            prime_field::field_element root_of_unity, prime_field::field_element *result);

// Interpolation: the coef_len coefficients of the polynomial through the
// evaluations at root^(i * order / coef_len).
void inverse_fast_fourier_transform(prime_field::field_element *evaluations, int coef_len, int order,
                                    prime_field::field_element root_of_unity, prime_field::field_element *result);

#endif
