"""Generates hash_code.inc: the unrolled Keccak-f[1600] round on 64-bit lanes
(host) and on 32-bit lane halves (device), and the SHA-256 constants.

All constants are derived from their FIPS definitions rather than typed in:
Keccak round constants from the rc(t) LFSR and rotation offsets from the
(x, y) -> (y, 2x + 3y) walk (FIPS 202, 3.2.2 and 3.2.5); SHA-256 round
constants and initial hash value from the cube and square roots of the first
primes (FIPS 180-4, 4.2.2 and 5.3.3), taken exactly with integer roots.

Run:  python gen_hash_code.py > hash_code.inc
"""


def keccak_round_constants():
    out, r = [], 1
    for _ in range(24):
        rc = 0
        for j in range(7):
            if r & 1:
                rc ^= 1 << ((1 << j) - 1)
            r = ((r << 1) ^ 0x71) & 0xFF if r & 0x80 else (r << 1) & 0xFF
        out.append(rc)
    return out


def keccak_rotations():
    rot = [[0] * 5 for _ in range(5)]
    x, y = 1, 0
    for t in range(24):
        rot[x][y] = ((t + 1) * (t + 2) // 2) % 64
        x, y = y, (2 * x + 3 * y) % 5
    return rot


def round32(rot, mode):
    """One Keccak-f round on 32-bit lane halves as macro lines.  mode 0: every
    rotation a pair of funnel shifts; 1 / 2: every other / every rho rotation
    as multiplies by 2^n (VG_MROT_LO / VG_MROT_HI)."""
    body = []
    for h in "LH":
        for x in range(5):
            body.append("    uint32_t c%s%d = vg_xor3(vg_xor3(a%s%d, a%s%d, a%s%d), a%s%d, a%s%d); \\"
                        % (h, x, h, x, h, x + 5, h, x + 10, h, x + 15, h, x + 20))
    for x in range(5):   # rot1 of each column parity
        body.append("    uint32_t rL%d = __funnelshift_l(cH%d, cL%d, 1), rH%d = __funnelshift_l(cL%d, cH%d, 1); \\"
                    % (x, x, x, x, x, x))
    for i in range(25):
        x = i % 5
        for h in "LH":
            body.append("    a%s%d = vg_xor3(a%s%d, c%s%d, r%s%d); \\" % (h, i, h, i, h, (x + 4) % 5, h, (x + 1) % 5))
    # rho + pi: b[y, 2x+3y] = rot(a[x, y], r[x][y])
    k = 0
    for x in range(5):
        for y in range(5):
            dst = y + 5 * ((2 * x + 3 * y) % 5)
            src = x + 5 * y
            n = rot[x][y]
            if n == 0:
                body.append("    uint32_t bL%d = aL%d, bH%d = aH%d; \\" % (dst, src, dst, src))
                continue
            mul = mode == 2 or (mode == 1 and k % 2 == 0)
            k += 1
            lo, hi = ("aL%d" % src, "aH%d" % src) if n < 32 else ("aH%d" % src, "aL%d" % src)   # >= 32: halves swap
            m = n % 32
            if mul:
                body.append("    uint32_t bL%d = VG_MROT_LO(%s, %s, %d), bH%d = VG_MROT_HI(%s, %s, %d); \\"
                            % (dst, lo, hi, m, dst, lo, hi, m))
            else:
                body.append("    uint32_t bL%d = __funnelshift_l(%s, %s, %d), bH%d = __funnelshift_l(%s, %s, %d); \\"
                            % (dst, hi, lo, m, dst, lo, hi, m))
    # chi
    for y in range(5):
        for x in range(5):
            i = x + 5 * y
            j, kk = (x + 1) % 5 + 5 * y, (x + 2) % 5 + 5 * y
            for h in "LH":
                body.append("    a%s%d = vg_chi(b%s%d, b%s%d, b%s%d); \\" % (h, i, h, i, h, j, h, kk))
    body.append("    aL0 ^= (RCL); aH0 ^= (RCH); }")
    return body


def primes(n):
    ps, c = [], 2
    while len(ps) < n:
        if all(c % d for d in range(2, int(c ** 0.5) + 1)):
            ps.append(c)
        c += 1
    return ps


def iroot(x, k):
    lo, hi = 0, 1 << (x.bit_length() // k + 2)
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if mid ** k <= x:
            lo = mid
        else:
            hi = mid - 1
    return lo


def main():
    rc = keccak_round_constants()
    rot = keccak_rotations()
    L = []
    L.append("// Generated by gen_hash_code.py from the FIPS 202 / FIPS 180-4 definitions. Do not edit.")
    # 64-bit lanes a0..a24 (the host implementation)
    L.append("#define VG_KECCAK_ROUND_CONSTANTS { \\")
    L.append("    " + ", ".join("0x%016xull" % v for v in rc) + " }")
    L.append("")
    # one round as a macro over named lanes; RC is the round constant expression
    body = []
    body.append("    { uint64_t c0 = a0 ^ a5 ^ a10 ^ a15 ^ a20, c1 = a1 ^ a6 ^ a11 ^ a16 ^ a21, \\")
    body.append("               c2 = a2 ^ a7 ^ a12 ^ a17 ^ a22, c3 = a3 ^ a8 ^ a13 ^ a18 ^ a23, \\")
    body.append("               c4 = a4 ^ a9 ^ a14 ^ a19 ^ a24; \\")
    for x in range(5):
        body.append("      uint64_t d%d = c%d ^ VG_ROTL(c%d, 1); \\" % (x, (x + 4) % 5, (x + 1) % 5))
    for i in range(25):
        body.append("      a%d ^= d%d; \\" % (i, i % 5))
    # rho + pi: b[y, 2x+3y] = rot(a[x, y], r[x][y])
    for x in range(5):
        for y in range(5):
            dst = y + 5 * ((2 * x + 3 * y) % 5)
            src = x + 5 * y
            if rot[x][y]:
                body.append("      uint64_t b%d = VG_ROTL(a%d, %d); \\" % (dst, src, rot[x][y]))
            else:
                body.append("      uint64_t b%d = a%d; \\" % (dst, src))
    # chi
    for y in range(5):
        for x in range(5):
            i = x + 5 * y
            body.append("      a%d = b%d ^ (~b%d & b%d); \\" % (i, i, (x + 1) % 5 + 5 * y, (x + 2) % 5 + 5 * y))
    body.append("      a0 ^= (RC); }")
    L.append("#define VG_KECCAK_ROUND(RC) \\")
    L.extend(body)
    L.append("")
    # Lanes are held as 32-bit halves aL<i> (bits 0..31) and aH<i> (bits
    # 32..63) of a[x + 5y]: a 64-bit rotation is two funnel shifts, the
    # 3-input xors of theta and the chi step are one lop3 each (vg_xor3,
    # vg_chi in hash.cuh), and theta's D[x] is folded into the lane update.
    L.append("// Lanes a[x + 5*y] are held as 32-bit halves aL<i>, aH<i>.")
    L.append("#define VG_KECCAK_RC_LO { " + ", ".join("0x%08xu" % (v & 0xFFFFFFFF) for v in rc) + " }")
    L.append("#define VG_KECCAK_RC_HI { " + ", ".join("0x%08xu" % (v >> 32) for v in rc) + " }")
    # per-lane tables of the warp formulation (lane x + 5y holds A[x, y]):
    # its rho rotation, and the lane pi takes its value from, since
    # B[y, 2x + 3y] = A[x, y] puts A[(X + 3Y) % 5, X] at lane X + 5Y
    L.append("#define VG_KECCAK_RHO { " + ", ".join(str(rot[i % 5][i // 5]) for i in range(25)) + " }")
    L.append("#define VG_KECCAK_PI_SRC { " + ", ".join(str(((i % 5) + 3 * (i // 5)) % 5 + 5 * (i % 5)) for i in range(25)) + " }")
    L.append("")
    L.append("#define VG_KECCAK_ROUND32(RCL, RCH) { \\")
    L.extend(round32(rot, 0))
    L.append("")
    # the same round with rho's rotations partly (1: every other one) or
    # wholly (2) on the integer-multiply pipe (VG_MROT_*, hash.cuh), which
    # the funnel-shift form leaves idle while the ALU pipe saturates
    for mode in (1, 2):
        L.append("#define VG_KECCAK_ROUND32_M%d(RCL, RCH) { \\" % mode)
        L.extend(round32(rot, mode))
        L.append("")
    ps = primes(64)
    k = [iroot(p << 96, 3) & 0xFFFFFFFF for p in ps]
    h0 = [iroot(p << 64, 2) & 0xFFFFFFFF for p in ps[:8]]
    L.append("#define VG_SHA256_K { \\")
    for i in range(0, 64, 8):
        L.append("    " + ", ".join("0x%08xu" % v for v in k[i:i + 8]) + (", \\" if i < 56 else " }"))
    L.append("#define VG_SHA256_H0 { " + ", ".join("0x%08xu" % v for v in h0) + " }")
    print("\n".join(L))


if __name__ == "__main__":
    main()
