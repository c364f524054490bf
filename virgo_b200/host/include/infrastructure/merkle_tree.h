// Merkle tree with the reference's interface (include/infrastructure/merkle_tree.h).
// create_tree runs on the GPU: heap layout, dst[1] = root, leaves stored raw
// at [size, 2 size), padding leaves H(0^64), internal nodes H(left || right).
#ifndef __merkle_tree
#define __merkle_tree
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <immintrin.h>
#include "my_hhash.h"

namespace merkle_tree
{
extern int size_after_padding;
namespace merkle_tree_prover
{
// data: ele_num 32-byte leaves in host memory; dst receives 2 * size_after_padding
// digests (allocated with malloc when alloc_required)
void create_tree(void *data, int ele_num, __hhash_digest *&dst, const int element_size, bool alloc_required);
}  // namespace merkle_tree_prover

namespace merkle_tree_verifier
{
bool verify_claim(__m128i root_hhash, const void *tree, __m128i hhash_element, int pos_element);
}
}  // namespace merkle_tree

#endif
