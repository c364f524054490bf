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

// a ^ b ^ c and a ^ (~b & c) as one lop3 each (truth tables 0x96, 0xD2)
__device__ __forceinline__ uint32_t vg_xor3(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ uint32_t vg_chi(uint32_t a, uint32_t b, uint32_t c)
{
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0xD2;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// The lanes as 32-bit halves: 64-bit rotations become two funnel shifts and
// the xors of theta and the chi step one lop3 per half, 180 instructions a
// round (the 64-bit formulation compiled to about a fifth more).
__device__ __forceinline__ void sha3_256_64(const uint64_t w[8], uint64_t d[4])
{
    const uint32_t RCL[24] = VG_KECCAK_RC_LO, RCH[24] = VG_KECCAK_RC_HI;
    uint32_t aL0 = (uint32_t)w[0], aH0 = (uint32_t)(w[0] >> 32), aL1 = (uint32_t)w[1], aH1 = (uint32_t)(w[1] >> 32);
    uint32_t aL2 = (uint32_t)w[2], aH2 = (uint32_t)(w[2] >> 32), aL3 = (uint32_t)w[3], aH3 = (uint32_t)(w[3] >> 32);
    uint32_t aL4 = (uint32_t)w[4], aH4 = (uint32_t)(w[4] >> 32), aL5 = (uint32_t)w[5], aH5 = (uint32_t)(w[5] >> 32);
    uint32_t aL6 = (uint32_t)w[6], aH6 = (uint32_t)(w[6] >> 32), aL7 = (uint32_t)w[7], aH7 = (uint32_t)(w[7] >> 32);
    // pad10*1 with the SHA-3 domain bits: 0x06 after the 64 message bytes
    // (lane 8), the final bit at the end of the 136-byte rate (lane 16)
    uint32_t aL8 = 0x06u, aH8 = 0, aL9 = 0, aH9 = 0, aL10 = 0, aH10 = 0, aL11 = 0, aH11 = 0, aL12 = 0, aH12 = 0;
    uint32_t aL13 = 0, aH13 = 0, aL14 = 0, aH14 = 0, aL15 = 0, aH15 = 0, aL16 = 0, aH16 = 0x80000000u;
    uint32_t aL17 = 0, aH17 = 0, aL18 = 0, aH18 = 0, aL19 = 0, aH19 = 0, aL20 = 0, aH20 = 0, aL21 = 0, aH21 = 0;
    uint32_t aL22 = 0, aH22 = 0, aL23 = 0, aH23 = 0, aL24 = 0, aH24 = 0;
#pragma unroll
    for (int r = 0; r < 24; ++r) VG_KECCAK_ROUND32(RCL[r], RCH[r]);
    d[0] = aL0 | ((uint64_t)aH0 << 32);
    d[1] = aL1 | ((uint64_t)aH1 << 32);
    d[2] = aL2 | ((uint64_t)aH2 << 32);
    d[3] = aL3 | ((uint64_t)aH3 << 32);
}

// sha3_256_64 with the first 20 rounds in a loop unrolled four times (round
// constants from constant memory) and the last four written out, so that the
// last round forms only the lanes the 256-bit digest reads (row 0: theta's
// five column sums, five lanes through rho and pi, four chi outputs, about a
// third of a round): under half of the fully unrolled code, for kernels whose
// permutation body would not stay in the instruction cache
__constant__ uint32_t vg_keccak_rcl[24] = VG_KECCAK_RC_LO, vg_keccak_rch[24] = VG_KECCAK_RC_HI;
__device__ __forceinline__ void sha3_256_64_compact(const uint64_t w[8], uint64_t d[4])
{
    uint32_t aL0 = (uint32_t)w[0], aH0 = (uint32_t)(w[0] >> 32), aL1 = (uint32_t)w[1], aH1 = (uint32_t)(w[1] >> 32);
    uint32_t aL2 = (uint32_t)w[2], aH2 = (uint32_t)(w[2] >> 32), aL3 = (uint32_t)w[3], aH3 = (uint32_t)(w[3] >> 32);
    uint32_t aL4 = (uint32_t)w[4], aH4 = (uint32_t)(w[4] >> 32), aL5 = (uint32_t)w[5], aH5 = (uint32_t)(w[5] >> 32);
    uint32_t aL6 = (uint32_t)w[6], aH6 = (uint32_t)(w[6] >> 32), aL7 = (uint32_t)w[7], aH7 = (uint32_t)(w[7] >> 32);
    uint32_t aL8 = 0x06u, aH8 = 0, aL9 = 0, aH9 = 0, aL10 = 0, aH10 = 0, aL11 = 0, aH11 = 0, aL12 = 0, aH12 = 0;
    uint32_t aL13 = 0, aH13 = 0, aL14 = 0, aH14 = 0, aL15 = 0, aH15 = 0, aL16 = 0, aH16 = 0x80000000u;
    uint32_t aL17 = 0, aH17 = 0, aL18 = 0, aH18 = 0, aL19 = 0, aH19 = 0, aL20 = 0, aH20 = 0, aL21 = 0, aH21 = 0;
    uint32_t aL22 = 0, aH22 = 0, aL23 = 0, aH23 = 0, aL24 = 0, aH24 = 0;
#pragma unroll 4
    for (int r = 0; r < 20; ++r) VG_KECCAK_ROUND32(vg_keccak_rcl[r], vg_keccak_rch[r]);
#pragma unroll
    for (int r = 20; r < 24; ++r) VG_KECCAK_ROUND32(vg_keccak_rcl[r], vg_keccak_rch[r]);
    d[0] = aL0 | ((uint64_t)aH0 << 32);
    d[1] = aL1 | ((uint64_t)aH1 << 32);
    d[2] = aL2 | ((uint64_t)aH2 << 32);
    d[3] = aL3 | ((uint64_t)aH3 << 32);
}

#ifdef VG_HASH_MULROT
// 64-bit rotation left by n (0..31) of (hi:lo) on the integer-multiply pipe:
// lo * 2^n keeps the bits that stay in the low word and umulhi(hi, 2^n)
// brings in those crossing from the high word; they share no bit, so the
// sum is their union.  The funnel-shift form runs on the ALU pipe, which the
// permutation saturates while the multiply pipe idles.  2^n is read from
// vg_pow2c (constant memory, filled at run time by the including file) so
// that the compiler cannot turn the multiplies back into shifts.
#define VG_MROT_LO(lo, hi, n) ((lo) * vg_pow2c[n] + __umulhi((hi), vg_pow2c[n]))
#define VG_MROT_HI(lo, hi, n) ((hi) * vg_pow2c[n] + __umulhi((lo), vg_pow2c[n]))

// sha3_256_64 with every other (MODE 1) or every (MODE 2) rho rotation on
// the multiply pipe; the same digest
template <int MODE>
__device__ __forceinline__ void sha3_256_64_mrot(const uint64_t w[8], uint64_t d[4])
{
    const uint32_t RCL[24] = VG_KECCAK_RC_LO, RCH[24] = VG_KECCAK_RC_HI;
    uint32_t aL0 = (uint32_t)w[0], aH0 = (uint32_t)(w[0] >> 32), aL1 = (uint32_t)w[1], aH1 = (uint32_t)(w[1] >> 32);
    uint32_t aL2 = (uint32_t)w[2], aH2 = (uint32_t)(w[2] >> 32), aL3 = (uint32_t)w[3], aH3 = (uint32_t)(w[3] >> 32);
    uint32_t aL4 = (uint32_t)w[4], aH4 = (uint32_t)(w[4] >> 32), aL5 = (uint32_t)w[5], aH5 = (uint32_t)(w[5] >> 32);
    uint32_t aL6 = (uint32_t)w[6], aH6 = (uint32_t)(w[6] >> 32), aL7 = (uint32_t)w[7], aH7 = (uint32_t)(w[7] >> 32);
    uint32_t aL8 = 0x06u, aH8 = 0, aL9 = 0, aH9 = 0, aL10 = 0, aH10 = 0, aL11 = 0, aH11 = 0, aL12 = 0, aH12 = 0;
    uint32_t aL13 = 0, aH13 = 0, aL14 = 0, aH14 = 0, aL15 = 0, aH15 = 0, aL16 = 0, aH16 = 0x80000000u;
    uint32_t aL17 = 0, aH17 = 0, aL18 = 0, aH18 = 0, aL19 = 0, aH19 = 0, aL20 = 0, aH20 = 0, aL21 = 0, aH21 = 0;
    uint32_t aL22 = 0, aH22 = 0, aL23 = 0, aH23 = 0, aL24 = 0, aH24 = 0;
    if (MODE == 1) {
#pragma unroll
        for (int r = 0; r < 24; ++r) VG_KECCAK_ROUND32_M1(RCL[r], RCH[r]);
    } else {
#pragma unroll
        for (int r = 0; r < 24; ++r) VG_KECCAK_ROUND32_M2(RCL[r], RCH[r]);
    }
    d[0] = aL0 | ((uint64_t)aH0 << 32);
    d[1] = aL1 | ((uint64_t)aH1 << 32);
    d[2] = aL2 | ((uint64_t)aH2 << 32);
    d[3] = aL3 | ((uint64_t)aH3 << 32);
}
#endif

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

// ---- Keccak-f[1600] on a whole warp ----
// Lane l = x + 5y (l < 25) holds state word A[x, y] as two 32-bit halves;
// lanes 25..31 take part in the shuffles and hold nothing used.  A round is
// ten 64-bit shuffles: five for the column parity C[x], two for C[x-1] and
// C[x+1], one for pi (each lane rotates its own word by its rho offset
// first), two for the chi neighbours.  About a fifth of the per-thread
// permutation's instructions per lane, at 32 lanes per permutation: it pays
// only when too few chains exist to fill the GPU one thread each.
struct KeccakLanes {
    int col[5];      // lanes of column x: x + 5 y', y' < 5
    int xm, xp, xp2; // lanes (x - 1, y), (x + 1, y), (x + 2, y)
    int pi;          // lane whose rotated word pi moves here
    int rn;          // rho rotation modulo 32
    bool rswap;      // rho rotation >= 32: halves swap first
    bool iota;       // lane 0
};

__device__ __forceinline__ KeccakLanes keccak_lanes(int l)
{
    const uint8_t RHO[25] = VG_KECCAK_RHO, PI[25] = VG_KECCAK_PI_SRC;
    KeccakLanes K;
    const bool in = l < 25;
    const int x = l % 5, y = l / 5;
#pragma unroll
    for (int j = 0; j < 5; ++j) K.col[j] = in ? x + 5 * j : l;
    K.xm = in ? (x + 4) % 5 + 5 * y : l;
    K.xp = in ? (x + 1) % 5 + 5 * y : l;
    K.xp2 = in ? (x + 2) % 5 + 5 * y : l;
    K.pi = in ? PI[l] : l;
    const int rho = in ? RHO[l] : 0;
    K.rn = rho & 31;
    K.rswap = rho >= 32;
    K.iota = l == 0;
    return K;
}

__device__ __forceinline__ void keccak_f_warp(uint32_t &lo, uint32_t &hi, const KeccakLanes &K)
{
    const uint32_t RCL[24] = VG_KECCAK_RC_LO, RCH[24] = VG_KECCAK_RC_HI;
    const unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int r = 0; r < 24; ++r) {
        // theta
        uint32_t s0l = __shfl_sync(FULL, lo, K.col[0]), s0h = __shfl_sync(FULL, hi, K.col[0]);
        uint32_t s1l = __shfl_sync(FULL, lo, K.col[1]), s1h = __shfl_sync(FULL, hi, K.col[1]);
        uint32_t s2l = __shfl_sync(FULL, lo, K.col[2]), s2h = __shfl_sync(FULL, hi, K.col[2]);
        uint32_t s3l = __shfl_sync(FULL, lo, K.col[3]), s3h = __shfl_sync(FULL, hi, K.col[3]);
        uint32_t s4l = __shfl_sync(FULL, lo, K.col[4]), s4h = __shfl_sync(FULL, hi, K.col[4]);
        const uint32_t cl = vg_xor3(vg_xor3(s0l, s1l, s2l), s3l, s4l);
        const uint32_t ch = vg_xor3(vg_xor3(s0h, s1h, s2h), s3h, s4h);
        const uint32_t ml = __shfl_sync(FULL, cl, K.xm), mh = __shfl_sync(FULL, ch, K.xm);
        const uint32_t pl = __shfl_sync(FULL, cl, K.xp), ph = __shfl_sync(FULL, ch, K.xp);
        // D = C[x-1] ^ rotl(C[x+1], 1)
        lo = vg_xor3(lo, ml, __funnelshift_l(ph, pl, 1));
        hi = vg_xor3(hi, mh, __funnelshift_l(pl, ph, 1));
        // rho (own word), then pi
        uint32_t a = K.rswap ? hi : lo, b = K.rswap ? lo : hi;
        const uint32_t rl = __funnelshift_l(b, a, K.rn), rh = __funnelshift_l(a, b, K.rn);
        const uint32_t bl = __shfl_sync(FULL, rl, K.pi), bh = __shfl_sync(FULL, rh, K.pi);
        // chi
        const uint32_t b1l = __shfl_sync(FULL, bl, K.xp), b1h = __shfl_sync(FULL, bh, K.xp);
        const uint32_t b2l = __shfl_sync(FULL, bl, K.xp2), b2h = __shfl_sync(FULL, bh, K.xp2);
        lo = vg_chi(bl, b1l, b2l);
        hi = vg_chi(bh, b1h, b2h);
        // iota
        if (K.iota) {
            lo ^= RCL[r];
            hi ^= RCH[r];
        }
    }
}

// The digest of 64 bytes; SHA3-256 in the compact form (the rounds in a
// loop: the fully unrolled permutation stalls on instruction fetch)
template <int KIND>
__device__ __forceinline__ void hash64(const uint64_t w[8], uint64_t d[4])
{
    if (KIND == HASH_SHA256) sha256_64(w, d);
    else sha3_256_64_compact(w, d);
}

#ifdef VG_HASH_MULROT
// hash64 with the SHA3 rotations in form ROT (0: funnel shifts; 1, 2: see
// sha3_256_64_mrot; 3: funnel shifts, rounds in a loop unrolled four times)
template <int KIND, int ROT>
__device__ __forceinline__ void hash64_rot(const uint64_t w[8], uint64_t d[4])
{
    if (KIND == HASH_SHA256 || ROT == 3) hash64<KIND>(w, d);
    else if (ROT == 0) sha3_256_64(w, d);
    else sha3_256_64_mrot<ROT>(w, d);
}
#endif

}  // namespace vg
