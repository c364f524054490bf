// Host side of the 64-byte hash (my_hhash): SHA3-256 and SHA-256 from the
// same generated FIPS 202 / FIPS 180-4 definitions as the device kernels
// (csrc/hash_code.inc).  Used by the verifier-side calls and by the few
// hashes the prover does on the host.
#include "infrastructure/my_hhash.h"
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include "../../csrc/hash_code.inc"

#define VG_ROTL(x, n) (((x) << (n)) | ((x) >> (64 - (n))))

static std::atomic<int> g_kind{-1};

int virgo_hash_kind()
{
    int k = g_kind.load();
    if (k < 0) {
        const char *s = getenv("VIRGO_HASH");
        k = (s && (!strcmp(s, "sha256") || !strcmp(s, "SHA256") || !strcmp(s, "1"))) ? 1 : 0;
        g_kind.store(k);
    }
    return k;
}

void virgo_set_hash(int kind) { g_kind.store(kind == 1 ? 1 : 0); }

static void sha3_256_64(const uint64_t w[8], uint64_t d[4])
{
    static const uint64_t RC[24] = VG_KECCAK_ROUND_CONSTANTS;
    uint64_t a0 = w[0], a1 = w[1], a2 = w[2], a3 = w[3], a4 = w[4], a5 = w[5], a6 = w[6], a7 = w[7];
    uint64_t a8 = 0x06ull, a9 = 0, a10 = 0, a11 = 0, a12 = 0, a13 = 0, a14 = 0, a15 = 0;
    uint64_t a16 = 0x8000000000000000ull, a17 = 0, a18 = 0, a19 = 0, a20 = 0, a21 = 0, a22 = 0, a23 = 0, a24 = 0;
    for (int r = 0; r < 24; ++r) VG_KECCAK_ROUND(RC[r]);
    d[0] = a0; d[1] = a1; d[2] = a2; d[3] = a3;
}

static inline uint32_t ror32(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

static void sha256_compress(uint32_t H[8], const uint32_t blk[16])
{
    static const uint32_t K[64] = VG_SHA256_K;
    uint32_t w[64];
    for (int i = 0; i < 16; ++i) w[i] = blk[i];
    for (int i = 16; i < 64; ++i) {
        uint32_t s0 = ror32(w[i - 15], 7) ^ ror32(w[i - 15], 18) ^ (w[i - 15] >> 3);
        uint32_t s1 = ror32(w[i - 2], 17) ^ ror32(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = H[0], b = H[1], c = H[2], d = H[3], e = H[4], f = H[5], g = H[6], h = H[7];
    for (int i = 0; i < 64; ++i) {
        uint32_t t1 = h + (ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25)) + ((e & f) ^ (~e & g)) + K[i] + w[i];
        uint32_t t2 = (ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    H[0] += a; H[1] += b; H[2] += c; H[3] += d; H[4] += e; H[5] += f; H[6] += g; H[7] += h;
}

static void sha256_64(const uint8_t *in, uint8_t *out)
{
    static const uint32_t H0[8] = VG_SHA256_H0;
    uint32_t H[8], blk[16];
    memcpy(H, H0, sizeof H);
    for (int i = 0; i < 16; ++i)
        blk[i] = (uint32_t)in[4 * i] << 24 | (uint32_t)in[4 * i + 1] << 16 | (uint32_t)in[4 * i + 2] << 8 | in[4 * i + 3];
    sha256_compress(H, blk);
    memset(blk, 0, sizeof blk);
    blk[0] = 0x80000000u;
    blk[15] = 512;
    sha256_compress(H, blk);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(H[i] >> 24);
        out[4 * i + 1] = (uint8_t)(H[i] >> 16);
        out[4 * i + 2] = (uint8_t)(H[i] >> 8);
        out[4 * i + 3] = (uint8_t)H[i];
    }
}

void virgo_hash64(const void *src, void *dst)
{
    if (virgo_hash_kind() == 1) {
        sha256_64((const uint8_t *)src, (uint8_t *)dst);
        return;
    }
    uint64_t w[8], d[4];
    memcpy(w, src, 64);   // little-endian lanes
    sha3_256_64(w, d);
    memcpy(dst, d, 32);
}
