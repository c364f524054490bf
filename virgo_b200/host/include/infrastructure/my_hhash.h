// 64-byte-message hash used by every Merkle commitment, with the reference's
// names (include/infrastructure/my_hhash.h): __hhash_digest is two 128-bit
// words, my_hhash(src, dst) hashes exactly 64 bytes into 32.
//
// The reference fixes the hash at build time (#define USESHA3 -> SHA3-256,
// else SHA-256).  Here it is chosen at run time for the host and device
// together: SHA3-256 unless VIRGO_HASH=sha256 is set before first use, or
// virgo_set_hash() is called.  The host implementation is this project's own
// (FIPS 202 / FIPS 180-4); the device kernels use the same definitions.
#ifndef __hhash
#define __hhash

#include <immintrin.h>
#include <cassert>

class __hhash_digest
{
public:
    __m128i h0, h1;
};

inline bool equals(const __hhash_digest &a, const __hhash_digest &b)
{
    __m128i v0 = _mm_xor_si128(a.h0, b.h0);
    __m128i v1 = _mm_xor_si128(a.h1, b.h1);
    return _mm_test_all_zeros(v0, v0) && _mm_test_all_zeros(v1, v1);
}

// 0 = SHA3-256 (default), 1 = SHA-256
int virgo_hash_kind();
void virgo_set_hash(int kind);
void virgo_hash64(const void *src, void *dst);

inline void my_hhash(const void *src, void *dst) { virgo_hash64(src, dst); }

#endif
