// Device hash functions for 64-byte messages, the only message length the
// prover hashes (reference include/infrastructure/my_hhash.h:28-35).
//
// Messages and digests are handled as little-endian 64-bit words of their
// in-memory bytes: a message is w[0..7] (bytes 0..63), a digest d[0..3].
// SHA3-256 (default, the reference's USESHA3 build) is one Keccak-f[1600]
// permutation with the pad10*1 bits and the 0x06 domain byte folded into lanes
// 8 and 16.  SHA-256 (the alternative build) is two compression calls, the
// second over the constant padding block.
#pragma once
#include <stdint.h>
#include "hash_code.inc"

namespace vg {

enum HashKind { HASH_SHA3_256 = 0, HASH_SHA256 = 1 };

#define VG_ROTL(x, n) (((x) << (n)) | ((x) >> (64 - (n))))

__device__ __forceinline__ void sha3_256_64(const uint64_t w[8], uint64_t d[4])
{
    const uint64_t RC[24] = VG_KECCAK_ROUND_CONSTANTS;
    uint64_t a0 = w[0], a1 = w[1], a2 = w[2], a3 = w[3], a4 = w[4], a5 = w[5], a6 = w[6], a7 = w[7];
    uint64_t a8 = 0x06ull, a9 = 0, a10 = 0, a11 = 0, a12 = 0, a13 = 0, a14 = 0, a15 = 0;
    uint64_t a16 = 0x8000000000000000ull, a17 = 0, a18 = 0, a19 = 0, a20 = 0, a21 = 0, a22 = 0, a23 = 0, a24 = 0;
#pragma unroll
    for (int r = 0; r < 24; ++r) VG_KECCAK_ROUND(RC[r]);
    d[0] = a0; d[1] = a1; d[2] = a2; d[3] = a3;
}

__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }
__device__ __forceinline__ uint32_t ror32(uint32_t x, int n) { return __funnelshift_r(x, x, n); }

__device__ __forceinline__ void sha256_compress(uint32_t H[8], const uint32_t blk[16])
{
    const uint32_t K[64] = VG_SHA256_K;
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = blk[i];
    uint32_t a = H[0], b = H[1], c = H[2], d = H[3], e = H[4], f = H[5], g = H[6], h = H[7];
#pragma unroll
    for (int i = 0; i < 64; ++i) {
        uint32_t wi;
        if (i < 16) {
            wi = w[i];
        } else {
            uint32_t w15 = w[(i + 1) & 15], w2 = w[(i + 14) & 15];
            uint32_t s0 = ror32(w15, 7) ^ ror32(w15, 18) ^ (w15 >> 3);
            uint32_t s1 = ror32(w2, 17) ^ ror32(w2, 19) ^ (w2 >> 10);
            wi = w[i & 15] + s0 + w[(i + 9) & 15] + s1;
            w[i & 15] = wi;
        }
        uint32_t S1 = ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25);
        uint32_t ch = (e & f) ^ (~e & g);
        uint32_t t1 = h + S1 + ch + K[i] + wi;
        uint32_t S0 = ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22);
        uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + S0 + mj;
    }
    H[0] += a; H[1] += b; H[2] += c; H[3] += d; H[4] += e; H[5] += f; H[6] += g; H[7] += h;
}

__device__ __forceinline__ void sha256_64(const uint64_t w[8], uint64_t d[4])
{
    const uint32_t H0[8] = VG_SHA256_H0;
    uint32_t H[8], blk[16];
#pragma unroll
    for (int i = 0; i < 8; ++i) H[i] = H0[i];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        blk[2 * i] = bswap32((uint32_t)w[i]);
        blk[2 * i + 1] = bswap32((uint32_t)(w[i] >> 32));
    }
    sha256_compress(H, blk);
#pragma unroll
    for (int i = 0; i < 16; ++i) blk[i] = 0;
    blk[0] = 0x80000000u;
    blk[15] = 512;
    sha256_compress(H, blk);
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = (uint64_t)bswap32(H[2 * i]) | ((uint64_t)bswap32(H[2 * i + 1]) << 32);
}

template <int KIND>
__device__ __forceinline__ void hash64(const uint64_t w[8], uint64_t d[4])
{
    if (KIND == HASH_SHA256) sha256_64(w, d);
    else sha3_256_64(w, d);
}

}  // namespace vg
