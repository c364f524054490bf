// merkle_tree:: functions with the reference's interface
// (src/infrastructure/merkle_tree.cpp): the tree is built by vg_merkle_tree.
#include "infrastructure/merkle_tree.h"
#include <cstdio>
#include <cstdlib>
#include "device.h"

int merkle_tree::size_after_padding;

void merkle_tree::merkle_tree_prover::create_tree(void *src_data, int ele_num, __hhash_digest *&dst, const int element_size,
                                                  bool alloc_required)
{
    if (element_size != 32 || ele_num < 1) {
        fprintf(stderr, "create_tree: %d leaves of %d bytes (32-byte leaves required)\n", ele_num, element_size);
        abort();
    }
    size_after_padding = 1;
    while (size_after_padding < ele_num) size_after_padding *= 2;
    const size_t bytes = (size_t)size_after_padding * 2 * element_size;
    if (alloc_required) {
        dst = (__hhash_digest *)malloc(bytes);
        if (!dst) {
            printf("Merkle Tree Bad Alloc\n");
            abort();
        }
    }
    vg_ctx *c = virgo::ctx();
    virgo::check(vg_ctx_set_hash(c, virgo_hash_kind()), "vg_ctx_set_hash");
    void *leaves = nullptr, *tree = nullptr;
    virgo::check(vg_dev_alloc(c, (size_t)ele_num * 32, &leaves), "vg_dev_alloc");
    virgo::check(vg_dev_alloc(c, bytes, &tree), "vg_dev_alloc");
    virgo::check(vg_h2d(c, leaves, src_data, (size_t)ele_num * 32), "vg_h2d");
    virgo::check(vg_merkle_tree(c, (const vg_digest *)leaves, ele_num, (vg_digest *)tree), "vg_merkle_tree");
    virgo::check(vg_d2h(c, dst, tree, bytes), "vg_d2h");
    vg_dev_free(c, leaves);
    vg_dev_free(c, tree);
}

// walks from a leaf to the root (merkle_tree.cpp:59-73); host-side verifier helper
bool merkle_tree::merkle_tree_verifier::verify_claim(__m128i root_hhash, const void *tree, __m128i hhash_element, int pos_element_arr)
{
    int pos = pos_element_arr + size_after_padding;
    __m128i data[2];
    while (pos != 1) {
        data[pos & 1] = hhash_element;
        data[(pos & 1) ^ 1] = ((const __m128i *)tree)[pos ^ 1];
        my_hhash(data, &hhash_element);
        pos /= 2;
    }
    const long long *a = (const long long *)&root_hhash, *b = (const long long *)&hhash_element;
    return a[0] == b[0] && a[1] == b[1];
}
