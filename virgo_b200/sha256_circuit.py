"""SHA-256 compression circuits (FIPS 180-4, section 6.2.2) in the
reference's layered-circuit gate set, for the served benchmark mix.

Each circuit proves the compression of `blocks` independent seeded 512-bit
blocks from the standard initial hash value.  It takes the form of a
witness checker: the input layer holds every word that the compression
computes as bits (message schedule, the new a and e of each round, the
output hash value) together with the carry bits of each addition modulo
2^32; the circuit recomputes the bitwise functions (Sigma/sigma as xor (8)
of rotated and shifted bits, Ch with multiply (1) and not-a-and-b (9), Maj
with multiply and xor), packs 32-bit words with the exp-sum gate (12), adds
packed words in the field (0) and outputs, per addition, packed result plus
2^32 x carry minus the sum of its terms (7), and per word the sum (5) of its
bit tests (13).  With a correct witness every output is zero.  Constants
(the round constants K and the initial hash value) come from their
definition (fractional parts of cube and square roots of the first primes),
and enter as input bits.
"""
from __future__ import annotations

import numpy as np

from .layered import Builder

MASK = 0xFFFFFFFF


def _primes(n):
    out, k = [], 2
    while len(out) < n:
        if all(k % p for p in out if p * p <= k):
            out.append(k)
        k += 1
    return out


def _iroot(x, k):
    """floor(x^(1/k)) for integers"""
    r = int(round(x ** (1.0 / k)))
    while r ** k > x:
        r -= 1
    while (r + 1) ** k <= x:
        r += 1
    return r


K = [_iroot(p << 96, 3) & MASK for p in _primes(64)]
H0 = [_iroot(p << 64, 2) & MASK for p in _primes(8)]


def _rotr(x, n):
    return ((x >> n) | (x << (32 - n))) & MASK


def compress(state, block_words):
    """One compression (FIPS 180-4 6.2.2) and its witness: the message
    schedule, the new a and e of every round, the carries of every addition
    and the output hash value."""
    W = list(block_words)
    cw = [0] * 64
    for t in range(16, 64):
        s0 = _rotr(W[t - 15], 7) ^ _rotr(W[t - 15], 18) ^ (W[t - 15] >> 3)
        s1 = _rotr(W[t - 2], 17) ^ _rotr(W[t - 2], 19) ^ (W[t - 2] >> 10)
        tot = s1 + W[t - 7] + s0 + W[t - 16]
        W.append(tot & MASK)
        cw[t] = tot >> 32
    a, b, c, d, e, f, g, h = state
    A, E, ca, ce = [], [], [], []
    for t in range(64):
        S1 = _rotr(e, 6) ^ _rotr(e, 11) ^ _rotr(e, 25)
        ch = (e & f) ^ (~e & g & MASK)
        t1 = h + S1 + ch + K[t] + W[t]
        S0 = _rotr(a, 2) ^ _rotr(a, 13) ^ _rotr(a, 22)
        mj = (a & b) ^ (a & c) ^ (b & c)
        t2 = S0 + mj
        ne, na = d + t1, t1 + t2
        ce.append(ne >> 32)
        ca.append(na >> 32)
        h, g, f, e, d, c, b, a = g, f, e, ne & MASK, c, b, a, na & MASK
        A.append(a)
        E.append(e)
    fin = [a, b, c, d, e, f, g, h]
    out = [(s + x) for s, x in zip(state, fin)]
    return {"W": W, "cw": cw, "A": A, "E": E, "ca": ca, "ce": ce,
            "out": [x & MASK for x in out], "co": [x >> 32 for x in out]}


def _bits(x, n=32):
    return [(x >> j) & 1 for j in range(n)]


def sha256_blocks(blocks: int, seed: int) -> list:
    """File-level layers of a circuit checking `blocks` compressions of seeded
    random 512-bit blocks from the initial hash value."""
    rng = np.random.default_rng(seed)
    B = Builder()
    zero = B.input(0)
    k_bits = [[B.input(x) for x in _bits(K[t])] for t in range(64)]
    k_pack = [None] * 64

    def word_in(x):
        return [B.input(b) for b in _bits(x)]

    def rot(bits, n):
        return [bits[(j + n) % 32] for j in range(32)]

    def shr(bits, n):
        return [bits[j + n] if j + n < 32 else zero for j in range(32)]

    def xor3(x, y, z):
        return [B.xor(B.xor(p, q), r) for p, q, r in zip(x, y, z)]

    def checked(bits):
        B.output(B.total([B.bitcheck(b) for b in bits]))

    for blk in range(blocks):
        words = [int(x) for x in rng.integers(0, 1 << 32, size=16, dtype=np.uint64)]
        wit = compress(H0, words)
        h_in = [word_in(x) for x in H0]
        W = [word_in(x) for x in wit["W"]]
        A = [word_in(x) for x in wit["A"]]
        E = [word_in(x) for x in wit["E"]]
        cw = {t: [B.input(b) for b in _bits(wit["cw"][t], 2)] for t in range(16, 64)}
        ca = [[B.input(b) for b in _bits(x, 3)] for x in wit["ca"]]
        ce = [[B.input(b) for b in _bits(x, 3)] for x in wit["ce"]]
        out = [word_in(x) for x in wit["out"]]
        co = [[B.input(b) for b in _bits(x, 1)] for x in wit["co"]]
        for grp in [W[16:], A, E, out]:
            for w in grp:
                checked(w)
        checked([b for t in range(16, 64) for b in cw[t]] + [b for c in ca + ce + co for b in c])
        P = {}

        def pk(bits):
            key = tuple(bits)
            if key not in P:
                P[key] = B.pack(list(bits))
            return P[key]

        # message schedule
        for t in range(16, 64):
            s0 = xor3(rot(W[t - 15], 7), rot(W[t - 15], 18), shr(W[t - 15], 3))
            s1 = xor3(rot(W[t - 2], 17), rot(W[t - 2], 19), shr(W[t - 2], 10))
            rhs = B.add_tree([pk(s1), pk(W[t - 7]), pk(s0), pk(W[t - 16])])
            B.output(B.sub(B.pack(W[t] + cw[t]), rhs))
        # rounds: state words at round t
        Aw = [h_in[3], h_in[2], h_in[1], h_in[0]] + A   # Aw[t + 3] = a at round t
        Ew = [h_in[7], h_in[6], h_in[5], h_in[4]] + E
        for t in range(64):
            a, b, c, d = Aw[t + 3], Aw[t + 2], Aw[t + 1], Aw[t]
            e, f, g, h = Ew[t + 3], Ew[t + 2], Ew[t + 1], Ew[t]
            S1 = xor3(rot(e, 6), rot(e, 11), rot(e, 25))
            ch = [B.xor(B.mul(x, y), B.naab(x, z)) for x, y, z in zip(e, f, g)]
            S0 = xor3(rot(a, 2), rot(a, 13), rot(a, 22))
            mj = [B.xor(B.xor(B.mul(x, y), B.mul(x, z)), B.mul(y, z)) for x, y, z in zip(a, b, c)]
            if k_pack[t] is None:
                k_pack[t] = B.pack(k_bits[t])
            t1 = B.add_tree([pk(h), pk(S1), pk(ch), k_pack[t], pk(W[t])])
            t2 = B.add(pk(S0), pk(mj))
            B.output(B.sub(B.pack(E[t] + ce[t]), B.add(pk(d), t1)))
            B.output(B.sub(B.pack(A[t] + ca[t]), B.add(t1, t2)))
        fin = [Aw[67], Aw[66], Aw[65], Aw[64], Ew[67], Ew[66], Ew[65], Ew[64]]
        for i in range(8):
            B.output(B.sub(B.pack(out[i] + co[i]), B.add(pk(h_in[i]), pk(fin[i]))))
    return B.layers()
