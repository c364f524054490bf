// Protocol constants of the Virgo commitment, identical to the reference's
// include/infrastructure/constants.h:2-11 (they fix the proof format).
#pragma once
const int max_fri_depth = 30;
const int ldt_repeat_num = 33;
// 2^log_slice_number slices; each slice holds pairs of evaluations (x, -x)
const int log_slice_number = 6;
const int slice_number = 1 << log_slice_number;
const int rs_code_rate = 5;          // Reed-Solomon blowup 2^5
const int max_bit_length = 30;
const int packed_size = 4;
