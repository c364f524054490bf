/* CPU restatement of the Virgo prover hot path.  TEST INFRASTRUCTURE ONLY:
 * the checker and the timed CPU baseline, never the product.  See
 * virgo_oracle.h for the contract and the reference line each routine
 * restates.  Plain C11 (with the GCC 128-bit integer extension). */
#define _GNU_SOURCE   /* random_r: a private rand() stream */
#include "virgo_oracle.h"
#include <stdlib.h>
#include <string.h>

#define P61 0x1FFFFFFFFFFFFFFFull
typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ field */
/* prime_field.h:114-172: canonical add, sub and Karatsuba multiply over
 * F_p[i]/(i^2+1).  Any exact implementation with canonical results agrees. */
static uint64_t addp(uint64_t a, uint64_t b) { uint64_t s = a + b; return s >= P61 ? s - P61 : s; }
static uint64_t subp(uint64_t a, uint64_t b) { return a >= b ? a - b : a + P61 - b; }
static uint64_t redp(u128 x)
{
    uint64_t r = (uint64_t)(x & P61) + (uint64_t)(x >> 61);
    r = (r & P61) + (r >> 61);
    return r >= P61 ? r - P61 : r;
}
static uint64_t mulp(uint64_t a, uint64_t b) { return redp((u128)a * b); }

static vo_fe fe(uint64_t real, uint64_t img) { vo_fe r; r.real = real; r.img = img; return r; }
static vo_fe fadd(vo_fe a, vo_fe b) { return fe(addp(a.real, b.real), addp(a.img, b.img)); }
static vo_fe fsub(vo_fe a, vo_fe b) { return fe(subp(a.real, b.real), subp(a.img, b.img)); }
static vo_fe fmul(vo_fe a, vo_fe b)
{
    /* schoolbook: (ar br - ai bi) + i (ar bi + ai br) */
    uint64_t re = subp(mulp(a.real, b.real), mulp(a.img, b.img));
    uint64_t im = addp(mulp(a.real, b.img), mulp(a.img, b.real));
    return fe(re, im);
}
static vo_fe fconst(uint64_t x) { return fe(x % P61, 0); }
static int fzero(vo_fe a) { return a.real == 0 && a.img == 0; }

static vo_fe fpow(vo_fe x, u128 e)
{
    vo_fe r = fe(1, 0);
    while (e) {
        if (e & 1) r = fmul(r, x);
        x = fmul(x, x);
        e >>= 1;
    }
    return r;
}
static vo_fe finv(vo_fe x) { u128 p = P61; return fpow(x, p * p - 2); }   /* prime_field.cpp:88-92 */

/* prime_field.cpp:60-73: the order-2^62 generator squared 62-k times */
static vo_fe froot(int log_order)
{
    vo_fe r = fe(2147483648ull, 1033321771269002680ull);
    for (int i = 0; i < 62 - log_order; ++i) r = fmul(r, r);
    return r;
}

void vo_fe_mul_arr(const vo_fe *a, const vo_fe *b, vo_fe *c, long n) { for (long i = 0; i < n; ++i) c[i] = fmul(a[i], b[i]); }
void vo_fe_add_arr(const vo_fe *a, const vo_fe *b, vo_fe *c, long n) { for (long i = 0; i < n; ++i) c[i] = fadd(a[i], b[i]); }
void vo_fe_sub_arr(const vo_fe *a, const vo_fe *b, vo_fe *c, long n) { for (long i = 0; i < n; ++i) c[i] = fsub(a[i], b[i]); }
void vo_fe_inv(const vo_fe *a, vo_fe *out) { *out = finv(*a); }
void vo_root_of_unity(int log_order, vo_fe *out) { *out = froot(log_order); }

static int ilog2(long x) { int k = 0; while ((1L << k) < x) ++k; return k; }

/* -------------------------------------------------------------------- FFT */
/* RS_polynomial.cpp:27-167 evaluates the polynomial with coef_len
 * coefficients at root^0..root^(order-1) in natural order (its leaf
 * replication equals zero padding).  Restated as a radix-2 DIT transform of
 * the zero-padded coefficient vector. */
static void dft_inplace(vo_fe *a, long n, vo_fe w)
{
    int lg = ilog2(n);
    for (long i = 0; i < n; ++i) {
        long j = 0;
        for (int b = 0; b < lg; ++b) if (i >> b & 1) j |= 1L << (lg - 1 - b);
        if (i < j) { vo_fe t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (long len = 2; len <= n; len <<= 1) {
        vo_fe wl = fpow(w, (u128)(n / len));
        for (long i = 0; i < n; i += len) {
            vo_fe x = fe(1, 0);
            for (long j = 0; j < len / 2; ++j) {
                vo_fe u = a[i + j], v = fmul(a[i + j + len / 2], x);
                a[i + j] = fadd(u, v);
                a[i + j + len / 2] = fsub(u, v);
                x = fmul(x, wl);
            }
        }
    }
}

void vo_fft(const vo_fe *coef, long coef_len, long order, const vo_fe *root, vo_fe *out)
{
    vo_fe *a = (vo_fe *)calloc(order, sizeof(vo_fe));
    memcpy(a, coef, coef_len * sizeof(vo_fe));
    dft_inplace(a, order, *root);
    memcpy(out, a, order * sizeof(vo_fe));
    free(a);
}

/* RS_polynomial.cpp:169-240: subsample every order/coef_len-th evaluation,
 * transform with the inverse of root^(order/coef_len), scale by 1/coef_len. */
void vo_ifft(const vo_fe *evals, long coef_len, long order, const vo_fe *root, vo_fe *out)
{
    if (coef_len > order) coef_len = order;
    long step = order / coef_len;
    vo_fe *a = (vo_fe *)malloc(coef_len * sizeof(vo_fe));
    for (long i = 0; i < coef_len; ++i) a[i] = evals[i * step];
    vo_fe w = finv(fpow(*root, (u128)step));
    dft_inplace(a, coef_len, w);
    vo_fe inv_n = finv(fconst((uint64_t)coef_len));
    for (long i = 0; i < coef_len; ++i) out[i] = fmul(a[i], inv_n);
    free(a);
}

/* ----------------------------------------------------------------- hashes */
/* SHA3-256 (FIPS 202) of a 64-byte message: one Keccak-f[1600] call, since
 * the rate is 136 bytes.  Round constants and rotation offsets are derived
 * here from their FIPS 202 definitions (LFSR rc(t), the (x,y) -> (y,2x+3y)
 * walk) rather than tabulated. */
static uint64_t kc_rc[24];
static int kc_rot[25];
static int kc_ready = 0;
static void keccak_init(void)
{
    if (kc_ready) return;
    uint8_t R = 1;
    for (int ir = 0; ir < 24; ++ir) {
        uint64_t rc = 0;
        for (int j = 0; j < 7; ++j) {
            if (R & 1) rc ^= 1ull << ((1 << j) - 1);
            R = (R & 0x80) ? (uint8_t)((R << 1) ^ 0x71) : (uint8_t)(R << 1);
        }
        kc_rc[ir] = rc;
    }
    memset(kc_rot, 0, sizeof kc_rot);
    int x = 1, y = 0;
    for (int t = 0; t < 24; ++t) {
        kc_rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
        int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx; y = ny;
    }
    kc_ready = 1;
}
static uint64_t rotl(uint64_t v, int n) { return n ? (v << n) | (v >> (64 - n)) : v; }
static void keccak_f(uint64_t A[25])
{
    for (int ir = 0; ir < 24; ++ir) {
        uint64_t C[5], D[5], B[25];
        for (int x = 0; x < 5; ++x) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
        for (int x = 0; x < 5; ++x) D[x] = C[(x + 4) % 5] ^ rotl(C[(x + 1) % 5], 1);
        for (int i = 0; i < 25; ++i) A[i] ^= D[i % 5];
        /* rho + pi: B[y, 2x+3y] = rot(A[x,y]) */
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y)
                B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(A[x + 5 * y], kc_rot[x + 5 * y]);
        for (int x = 0; x < 5; ++x)
            for (int y = 0; y < 5; ++y)
                A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
        A[0] ^= kc_rc[ir];
    }
}
static uint64_t ld64le(const uint8_t *p) { uint64_t v = 0; for (int i = 7; i >= 0; --i) v = v << 8 | p[i]; return v; }
static void st64le(uint8_t *p, uint64_t v) { for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i)); }

void vo_sha3_256_64(const uint8_t *in64, uint8_t *out32)
{
    keccak_init();
    uint64_t A[25];
    memset(A, 0, sizeof A);
    for (int i = 0; i < 8; ++i) A[i] = ld64le(in64 + 8 * i);
    A[8] ^= 0x06;                  /* domain bits 01 + first pad bit, byte 64 */
    A[16] ^= 0x80ull << 56;        /* last pad bit, byte 135 */
    keccak_f(A);
    for (int i = 0; i < 4; ++i) st64le(out32 + 8 * i, A[i]);
}

/* SHA-256 (FIPS 180-4) of a 64-byte message: two compressions (the message
 * block, then the padding block).  Constants are the fractional parts of
 * square and cube roots of the first primes, computed here exactly with
 * integer roots. */
static uint32_t sh_k[64], sh_h0[8];
static int sh_ready = 0;
static u128 icbrt(u128 x) { u128 r = 0; for (int b = 42; b >= 0; --b) { u128 t = r | ((u128)1 << b); if (t * t * t <= x) r = t; } return r; }
static u128 isqrt(u128 x) { u128 r = 0; for (int b = 63; b >= 0; --b) { u128 t = r | ((u128)1 << b); if (t * t <= x) r = t; } return r; }
static void sha256_init(void)
{
    if (sh_ready) return;
    int primes[64], np = 0;
    for (int c = 2; np < 64; ++c) {
        int ok = 1;
        for (int d = 2; d * d <= c; ++d) if (c % d == 0) { ok = 0; break; }
        if (ok) primes[np++] = c;
    }
    for (int i = 0; i < 64; ++i) sh_k[i] = (uint32_t)icbrt((u128)primes[i] << 96);
    for (int i = 0; i < 8; ++i) sh_h0[i] = (uint32_t)isqrt((u128)primes[i] << 64);
    sh_ready = 1;
}
static uint32_t ror32(uint32_t v, int n) { return (v >> n) | (v << (32 - n)); }
static void sha256_block(uint32_t H[8], const uint8_t blk[64])
{
    uint32_t w[64];
    for (int i = 0; i < 16; ++i)
        w[i] = (uint32_t)blk[4 * i] << 24 | (uint32_t)blk[4 * i + 1] << 16 | (uint32_t)blk[4 * i + 2] << 8 | blk[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
        uint32_t s0 = ror32(w[i - 15], 7) ^ ror32(w[i - 15], 18) ^ (w[i - 15] >> 3);
        uint32_t s1 = ror32(w[i - 2], 17) ^ ror32(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = H[0], b = H[1], c = H[2], d = H[3], e = H[4], f = H[5], g = H[6], h = H[7];
    for (int i = 0; i < 64; ++i) {
        uint32_t S1 = ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25);
        uint32_t ch = (e & f) ^ (~e & g);
        uint32_t t1 = h + S1 + ch + sh_k[i] + w[i];
        uint32_t S0 = ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22);
        uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        uint32_t t2 = S0 + mj;
        h = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    H[0] += a; H[1] += b; H[2] += c; H[3] += d; H[4] += e; H[5] += f; H[6] += g; H[7] += h;
}
void vo_sha256_64(const uint8_t *in64, uint8_t *out32)
{
    sha256_init();
    uint32_t H[8];
    memcpy(H, sh_h0, sizeof H);
    sha256_block(H, in64);
    uint8_t pad[64];
    memset(pad, 0, 64);
    pad[0] = 0x80;
    pad[62] = 0x02;                /* message length 512 bits, big endian */
    sha256_block(H, pad);
    for (int i = 0; i < 8; ++i) {
        out32[4 * i] = (uint8_t)(H[i] >> 24); out32[4 * i + 1] = (uint8_t)(H[i] >> 16);
        out32[4 * i + 2] = (uint8_t)(H[i] >> 8); out32[4 * i + 3] = (uint8_t)H[i];
    }
}
static void hash64(int kind, const uint8_t *in, uint8_t *out)
{
    if (kind == 1) vo_sha256_64(in, out);
    else vo_sha3_256_64(in, out);
}
void vo_hash64_batch(int kind, const uint8_t *in, uint8_t *out, long n)
{
    for (long i = 0; i < n; ++i) hash64(kind, in + 64 * i, out + 32 * i);
}

/* ------------------------------------------------------------ Merkle tree */
void vo_merkle_tree(int kind, const vo_digest *leaves, long n, vo_digest *tree)
{
    long sz = 1;
    while (sz < n) sz *= 2;
    memset(tree, 0, 2 * sz * sizeof(vo_digest));
    uint8_t zero[64];
    memset(zero, 0, 64);
    for (long i = 0; i < sz; ++i) {
        if (i < n) tree[sz + i] = leaves[i];
        else hash64(kind, zero, tree[sz + i].b);
    }
    for (long j = sz - 1; j >= 1; --j) {
        uint8_t buf[64];
        memcpy(buf, tree[2 * j].b, 32);
        memcpy(buf + 32, tree[2 * j + 1].b, 32);
        hash64(kind, buf, tree[j].b);
    }
}

void vo_leaf_chain(int kind, const vo_fe *c, int n_slices, long n, vo_digest *leaves)
{
    long half = n / 2;
    for (long k = 0; k < half; ++k) {
        uint8_t buf[64], h[32];
        memset(h, 0, 32);
        for (int s = 0; s < n_slices; ++s) {
            memcpy(buf, &c[s * n + k], 16);
            memcpy(buf + 16, &c[s * n + k + half], 16);
            memcpy(buf + 32, h, 32);
            hash64(kind, buf, h);
        }
        memcpy(leaves[k].b, h, 32);
    }
}

/* ------------------------------------------------------------------ FRI */
void vo_fri_fold(const vo_fe *c, int n_slices, long n, const vo_fe *w, const vo_fe *r, vo_fe *out)
{
    vo_fe inv2 = finv(fconst(2));
    vo_fe winv = finv(*w);
    long half = n / 2;
    vo_fe mu = fe(1, 0);                      /* w^-i */
    for (long i = 0; i < half; ++i) {
        vo_fe t = fmul(mu, *r);
        for (int s = 0; s < n_slices; ++s) {
            vo_fe a = c[s * n + i], b = c[s * n + i + half];
            out[s * half + i] = fmul(inv2, fadd(fadd(a, b), fmul(t, fsub(a, b))));
        }
        mu = fmul(mu, winv);
    }
}

/* ---------------------------------------------------------- commitments */
void vo_rs_encode(const vo_fe *vals, long m, long s, vo_fe *out)
{
    vo_fe rm = froot(ilog2(m)), rs = froot(ilog2(s));
    vo_fe *coef = (vo_fe *)malloc(m * sizeof(vo_fe));
    vo_ifft(vals, m, m, &rm, coef);
    vo_fft(coef, m, s, &rs, out);
    free(coef);
}

static long mask_gap(long S, long n_mask)
{
    long gap = S / n_mask, g = 1;
    while (g * 2 <= gap) g *= 2;
    return g;
}

long vo_commit_private(const vo_fe *priv, int log_len, const vo_fe *mask, long n_mask, vo_fe *l_eval)
{
    long S = 1L << (log_len - 1), R = S >> 5;
    long M = S / mask_gap(S, n_mask);
    for (int i = 0; i < 64; ++i) vo_rs_encode(priv + i * R, R, S, l_eval + i * S);
    vo_fe *pm = (vo_fe *)calloc(M, sizeof(vo_fe));
    memcpy(pm, mask, n_mask * sizeof(vo_fe));
    vo_rs_encode(pm, M, S, l_eval + 64 * S);
    free(pm);
    return M;
}

/* lq sampled at 2m points -> quotient h = high half of its coefficients ->
 * h evaluated on <w_S>; the virtual oracle of poly_commit.h:241-263,298-322:
 * vo[j] = (l q - (x^m - 1) h - (lq_0 + h_0)) * m * x^-1 at x = w_S^j. */
static void public_slice(const vo_fe *l, const vo_fe *q, long S, long m, vo_fe *h_eval, vo_fe *vo, vo_fe *sum)
{
    long stride = S / (2 * m);
    vo_fe *lq = (vo_fe *)malloc(2 * m * sizeof(vo_fe));
    vo_fe *lqc = (vo_fe *)malloc(2 * m * sizeof(vo_fe));
    for (long j = 0; j < 2 * m; ++j) lq[j] = fmul(l[j * stride], q[j * stride]);
    vo_fe r2m = froot(ilog2(2 * m)), rs = froot(ilog2(S));
    vo_ifft(lq, 2 * m, 2 * m, &r2m, lqc);
    vo_fft(lqc + m, m, S, &rs, h_eval);
    vo_fe c0 = fadd(lqc[0], lqc[m]);
    vo_fe mm = fconst((uint64_t)m);
    vo_fe inv_rs = finv(rs), rs_m = fpow(rs, (u128)m);
    vo_fe xn = fe(1, 0), ix = mm;
    for (long j = 0; j < S; ++j) {
        vo_fe g = fsub(fmul(l[j], q[j]), fmul(fsub(xn, fe(1, 0)), h_eval[j]));
        vo[j] = fmul(fsub(g, c0), ix);
        ix = fmul(ix, inv_rs);
        xn = fmul(xn, rs_m);
    }
    *sum = fmul(c0, mm);
    free(lq);
    free(lqc);
}

void vo_commit_public(const vo_fe *l_eval, const vo_fe *pub, int log_len, const vo_fe *pub_mask, long n_mask,
                      vo_fe *q_eval, vo_fe *h_eval, vo_fe *vo, vo_fe *all_sum)
{
    long S = 1L << (log_len - 1), R = S >> 5;
    for (int i = 0; i < 64; ++i) vo_rs_encode(pub + i * R, R, S, q_eval + i * S);
    vo_rs_encode(pub_mask, n_mask, S, q_eval + 64 * S);
    for (int i = 0; i < 65; ++i) {
        long m = i < 64 ? R : n_mask;
        public_slice(l_eval + i * S, q_eval + i * S, S, m, h_eval + i * S, vo + i * S, &all_sum[i]);
    }
}

/* -------------------------------------------------------------------- GKR */
void vo_eval_input(const int64_t *u, long n, vo_fe *out)
{
    for (long g = 0; g < n; ++g) {
        int x = (int)u[g];                       /* zk_prover.cpp:60-65 reads through int */
        out[g] = fconst((uint64_t)(long long)x);
    }
}

void vo_eval_layer(const uint8_t *ty, const int64_t *u64, const int64_t *v64, long n, const vo_fe *prev, vo_fe *out)
{
    vo_fe one = fe(1, 0), two = fe(2, 0);
    for (long g = 0; g < n; ++g) {
        int u = (int)u64[g], v = (int)v64[g];
        vo_fe r = fe(0, 0);
        switch (ty[g]) {
        case 0: r = fadd(prev[u], prev[v]); break;
        case 1: r = fmul(prev[u], prev[v]); break;
        case 2: break;
        case 3: r = fconst((uint64_t)(long long)u); break;
        case 4: case 10: r = prev[u]; break;
        case 5: for (int k = u; k < v; ++k) r = fadd(r, prev[k]); break;
        case 6: r = fsub(one, prev[u]); break;
        case 7: r = fsub(prev[u], prev[v]); break;
        case 8: r = fsub(fadd(prev[u], prev[v]), fmul(fmul(two, prev[u]), prev[v])); break;
        case 9: r = fsub(prev[v], fmul(prev[u], prev[v])); break;
        case 12: for (int k = u; k <= v; ++k) r = fadd(r, fmul(prev[k], fconst(1ull << (k - u)))); break;
        case 13: r = fmul(prev[u], fsub(one, prev[v])); break;
        default: break;
        }
        out[g] = r;
    }
}

void vo_v_res(const vo_fe *vals, int log_n, const vo_fe *r, vo_fe *out)
{
    long n = 1L << log_n;
    vo_fe *t = (vo_fe *)malloc(n * sizeof(vo_fe));
    memcpy(t, vals, n * sizeof(vo_fe));
    for (int i = 0; i < log_n; ++i) {
        vo_fe om = fsub(fe(1, 0), r[i]);
        for (long j = 0; j < (n >> 1); ++j) t[j] = fadd(fmul(t[2 * j], om), fmul(t[2 * j + 1], r[i]));
        n >>= 1;
    }
    *out = t[0];
    free(t);
}

static vo_fe eq_at(const vo_fe *r, int len, long i)
{
    vo_fe x = fe(1, 0);
    for (int b = 0; b < len; ++b) x = fmul(x, (i >> b & 1) ? r[b] : fsub(fe(1, 0), r[b]));
    return x;
}

void vo_beta_g(int length_g, const vo_fe *r0, const vo_fe *r1, const vo_fe *alpha, const vo_fe *beta, vo_fe *out)
{
    for (long i = 0; i < (1L << length_g); ++i)
        out[i] = fadd(fmul(*alpha, eq_at(r0, length_g, i)), fmul(*beta, eq_at(r1, length_g, i)));
}

void vo_phase1_init(const uint8_t *ty, const int64_t *u64, const int64_t *v64, long n_g, const vo_fe *bg,
                    const vo_fe *prev, long n_uv, vo_fe *am, vo_fe *av)
{
    memset(am, 0, n_uv * sizeof(vo_fe));
    memset(av, 0, n_uv * sizeof(vo_fe));
    for (long i = 0; i < n_g; ++i) {
        int u = (int)u64[i], v = (int)v64[i];
        vo_fe t = bg[i];
        switch (ty[i]) {
        case 0: av[u] = fadd(av[u], fmul(prev[v], t)); am[u] = fadd(am[u], t); break;
        case 1: am[u] = fadd(am[u], fmul(prev[v], t)); break;
        case 5: for (int j = u; j < v; ++j) am[j] = fadd(am[j], t); break;
        case 12: for (int j = u; j <= v; ++j) { am[j] = fadd(am[j], t); t = fadd(t, t); } break;
        case 4: am[u] = fadd(am[u], bg[u]); break;
        case 6: am[u] = fsub(am[u], t); av[u] = fadd(av[u], t); break;
        case 7: av[u] = fsub(av[u], fmul(prev[v], t)); am[u] = fadd(am[u], t); break;
        case 8: { vo_fe tv = fmul(t, prev[v]); av[u] = fadd(av[u], tv); am[u] = fsub(fadd(am[u], t), fadd(tv, tv)); } break;
        case 13: { vo_fe tv = fmul(t, prev[v]); am[u] = fadd(fsub(am[u], tv), t); } break;
        case 9: { vo_fe tv = fmul(t, prev[v]); av[u] = fadd(av[u], tv); am[u] = fsub(am[u], tv); } break;
        case 10: am[u] = fadd(am[u], t); break;
        default: break;
        }
    }
}

void vo_phase2_init(const uint8_t *ty, const int64_t *u64, const int64_t *v64, long n_g, const vo_fe *bg,
                    const vo_fe *bu, const vo_fe *vu_p, long n_uv, vo_fe *am, vo_fe *av)
{
    vo_fe vu = *vu_p;
    memset(am, 0, n_uv * sizeof(vo_fe));
    memset(av, 0, n_uv * sizeof(vo_fe));
    for (long i = 0; i < n_g; ++i) {
        int u = (int)u64[i], v = (int)v64[i];
        vo_fe tg = bg[i];
        switch (ty[i]) {
        case 1: am[v] = fadd(am[v], fmul(fmul(tg, bu[u]), vu)); break;
        case 0: { vo_fe t = fmul(tg, bu[u]); am[v] = fadd(am[v], t); av[v] = fadd(av[v], fmul(t, vu)); } break;
        case 5: { vo_fe t = fmul(tg, vu); for (int j = u; j < v; ++j) av[0] = fadd(av[0], fmul(t, bu[j])); } break;
        case 12: { vo_fe t = fmul(tg, vu); for (int j = u; j <= v; ++j) { av[0] = fadd(av[0], fmul(t, bu[j])); t = fadd(t, t); } } break;
        case 6: { vo_fe t = fmul(tg, bu[u]); av[v] = fsub(fadd(av[v], t), fmul(t, vu)); } break;
        case 7: { vo_fe t = fmul(tg, bu[u]); am[v] = fsub(am[v], t); av[v] = fadd(av[v], fmul(t, vu)); } break;
        case 8: { vo_fe t = fmul(tg, bu[u]); vo_fe tv = fmul(t, vu); am[v] = fsub(fsub(fadd(am[v], t), tv), tv); av[v] = fadd(av[v], tv); } break;
        case 13: { vo_fe t = fmul(tg, bu[u]); vo_fe tv = fmul(t, vu); am[v] = fsub(am[v], tv); av[v] = fadd(av[v], tv); } break;
        case 9: { vo_fe t = fmul(tg, bu[u]); am[v] = fsub(fadd(am[v], t), fmul(vu, t)); } break;
        case 10: { vo_fe t = fmul(tg, bu[u]); av[v] = fadd(av[v], fmul(t, vu)); } break;
        default: break;
        }
    }
}

void vo_predicates(const uint8_t *ty, const int64_t *u64, const int64_t *v64, int bl_g, int bl_uv, const vo_fe *r0,
                   const vo_fe *r1, const vo_fe *ru, const vo_fe *rv, const vo_fe *alpha, const vo_fe *beta,
                   vo_fe out[14])
{
    const long n_g = 1L << bl_g, n_uv = 1L << bl_uv;
    vo_fe *bg = malloc(n_g * sizeof(vo_fe)), *bu = malloc(n_uv * sizeof(vo_fe)), *bv = malloc(n_uv * sizeof(vo_fe));
    vo_beta_g(bl_g, r0, r1, alpha, beta, bg);
    for (long i = 0; i < n_uv; ++i) {
        bu[i] = eq_at(ru, bl_uv, i);
        bv[i] = eq_at(rv, bl_uv, i);
    }
    for (int t = 0; t < 14; ++t) out[t] = fe(0, 0);
    for (long g = 0; g < n_g; ++g) {
        const long u = u64[g], v = v64[g];
        const int t = ty[g];
        switch (t) {
        case 0: case 1: case 6: case 7: case 8: case 9: case 13:
            out[t] = fadd(out[t], fmul(fmul(bg[g], bu[u]), bv[v]));
            break;
        case 5:
            for (long j = u; j < v; ++j) out[5] = fadd(out[5], fmul(fmul(bg[g], bv[0]), bu[j]));
            break;
        case 12: {
            vo_fe w = fmul(bg[g], bv[0]);
            for (long j = u; j <= v; ++j) {
                out[12] = fadd(out[12], fmul(w, bu[j]));
                w = fadd(w, w);
            }
        } break;
        case 10: out[10] = fadd(out[10], fmul(bg[g], bu[u])); break;
        default: break;
        }
    }
    out[10] = fmul(out[10], bv[0]);
    free(bg);
    free(bu);
    free(bv);
}

void vo_sumcheck_round(vo_lp *V, vo_lp *addv, vo_lp *am, long total_uv, const vo_fe *r, int current_bit, vo_fe out3[3])
{
    vo_fe ra = fe(0, 0), rb = fe(0, 0), rc = fe(0, 0);
    for (long i = 0; i < (total_uv >> 1); ++i) {
        long g0 = i << 1, g1 = i << 1 | 1;
        if (current_bit == 0) {
            V[i].b = V[g0].b; V[i].a = fsub(V[g1].b, V[i].b);
            addv[i].b = addv[g0].b; addv[i].a = fsub(addv[g1].b, addv[i].b);
            am[i].b = am[g0].b; am[i].a = fsub(am[g1].b, am[i].b);
        } else {
            V[i].b = fadd(fmul(V[g0].a, *r), V[g0].b);
            V[i].a = fsub(fadd(fmul(V[g1].a, *r), V[g1].b), V[i].b);
            addv[i].b = fadd(fmul(addv[g0].a, *r), addv[g0].b);
            addv[i].a = fsub(fadd(fmul(addv[g1].a, *r), addv[g1].b), addv[i].b);
            am[i].b = fadd(fmul(am[g0].a, *r), am[g0].b);
            am[i].a = fsub(fadd(fmul(am[g1].a, *r), am[g1].b), am[i].b);
        }
        ra = fadd(ra, fmul(am[i].a, V[i].a));
        rb = fadd(rb, fadd(fadd(fmul(am[i].a, V[i].b), fmul(am[i].b, V[i].a)), addv[i].a));
        rc = fadd(rc, fadd(fmul(am[i].b, V[i].b), addv[i].b));
    }
    out3[0] = ra; out3[1] = rb; out3[2] = rc;
}

int vo_is_zero(const vo_fe *a) { return fzero(*a); }

/* ------------------------------------------------------------ fft_gkr */
/* prime_field::random (prime_field.cpp:35-41): real, then img, each rand() */
typedef struct { struct random_data d; char st[128]; } vo_rng;
static void rng_init(vo_rng *g, unsigned seed) { memset(g, 0, sizeof *g); initstate_r(seed, g->st, sizeof g->st, &g->d); }
static vo_fe rng_fe(vo_rng *g)
{
    int32_t a, b;
    random_r(&g->d, &a);
    random_r(&g->d, &b);
    return fe((uint64_t)a % P61, (uint64_t)b % P61);
}
static void rng_fill(vo_rng *g, vo_fe *r, int n) { for (int i = 0; i < n; ++i) r[i] = rng_fe(g); }
static vo_fe fone(void) { return fe(1, 0); }
static int feq(vo_fe a, vo_fe b) { return a.real == b.real && a.img == b.img; }
static vo_fe fomr(vo_fe r) { return fsub(fone(), r); }
static vo_fe qeval(const vo_fe m[3], vo_fe x) { return fadd(fmul(fadd(fmul(m[0], x), m[1]), x), m[2]); }
/* alpha eq(r0, g) + beta eq(r1, g) over len bits */
static vo_fe bgat(const vo_fe *r0, const vo_fe *r1, int len, vo_fe al, vo_fe be, long g)
{
    return fadd(fmul(al, eq_at(r0, len, g)), fmul(be, eq_at(r1, len, g)));
}

int vo_fft_gkr_rounds(int lg) { return (lg + 6) + lg + 2 * lg * lg; }

/* one phase: rounds over (V, addv, am) of 2^nv entries with challenges r;
 * checks each message against *claim as fft_circuit_GKR.cpp:323-333 does */
static int fg_phase(vo_lp *V, vo_lp *addv, vo_lp *am, int nv, const vo_fe *r, vo_fe *claim, vo_fe **msgs, vo_fe *vfinal)
{
    int ok = 1;
    vo_fe prev = fe(0, 0);
    for (int i = 0; i < nv; ++i) {
        vo_fe m[3];
        vo_sumcheck_round(V, addv, am, 1L << (nv - i), &prev, i, m);
        memcpy(*msgs, m, sizeof m);
        *msgs += 3;
        prev = r[i];
        if (!feq(fadd(qeval(m, fe(0, 0)), qeval(m, fone())), *claim)) ok = 0;
        *claim = qeval(m, r[i]);
    }
    *vfinal = fadd(fmul(V[0].a, prev), V[0].b);
    return ok;
}

int vo_fft_gkr(int lg, unsigned seed, vo_fe *msgs, vo_fe *vals, int *proof_size)
{
    const long N = 1L << lg, NE = 64L << lg;
    vo_rng g;
    rng_init(&g, seed);
    /* ---- build_circuit (:22-112) ---- */
    vo_fe *r = malloc(lg * sizeof(vo_fe)), ep[64];
    rng_fill(&g, r, lg);
    int nl = 2 * lg + 4;   /* layers 0..lg expansion, lg+1..2lg ifft, scaled, products, sums */
    vo_fe **L = calloc(nl, sizeof(vo_fe *));
    L[0] = malloc(sizeof(vo_fe));
    L[0][0] = fone();
    for (int i = 0; i < lg; ++i) {
        L[i + 1] = malloc((2L << i) * sizeof(vo_fe));
        for (long j = 0; j < (1L << i); ++j) {
            L[i + 1][j << 1] = fmul(L[i][j], r[i]);
            L[i + 1][j << 1 | 1] = fmul(L[i][j], fomr(r[i]));
        }
    }
    const vo_fe rou = froot(lg), inv_rou = finv(rou), inv_n = finv(fconst((uint64_t)N));
    vo_fe rot[62];
    rot[0] = inv_rou;
    for (int i = 1; i < 62; ++i) rot[i] = fmul(rot[i - 1], rot[i - 1]);
    vo_fe *xa = malloc(N * sizeof(vo_fe));
    for (int dep = lg - 1; dep >= 0; --dep) {
        const long blk = 1L << (lg - dep), half = blk >> 1;
        const int cur = lg + (lg - dep), pre = cur - 1;
        L[cur] = malloc(N * sizeof(vo_fe));
        xa[0] = fone();
        for (long j = 1; j < blk; ++j) xa[j] = fmul(xa[j - 1], rot[dep]);
        for (long k = 0; k < half; ++k)
            for (long j = 0; j < (1L << dep); ++j) {
                vo_fe l = L[pre][k << (dep + 1) | j], rr = fmul(xa[k], L[pre][k << (dep + 1) | (1L << dep) | j]);
                L[cur][k << dep | j] = fadd(l, rr);
                L[cur][(k + half) << dep | j] = fsub(l, rr);
            }
    }
    const int Ls = 2 * lg + 1, Lp = 2 * lg + 2, Lo = 2 * lg + 3;
    L[Ls] = malloc(N * sizeof(vo_fe));
    for (long i = 0; i < N; ++i) L[Ls][i] = fmul(L[Ls - 1][i], inv_n);
    L[Lp] = malloc(NE * sizeof(vo_fe));
    for (int i = 0; i < 64; ++i) {
        ep[i] = rng_fe(&g);
        vo_fe x = fone();
        for (long j = 0; j < N; ++j) {
            L[Lp][j + ((long)i << lg)] = fmul(L[Ls][j], x);
            x = fmul(x, ep[i]);
        }
    }
    L[Lo] = malloc(64 * sizeof(vo_fe));
    for (int i = 0; i < 64; ++i) {
        L[Lo][i] = fe(0, 0);
        for (long j = 0; j < N; ++j) L[Lo][i] = fadd(L[Lo][i], L[Lp][j + i * N]);
    }
    /* ---- engage_gkr (:786-825) ---- */
    const int R = lg + 10;
    vo_fe *r0 = malloc(R * sizeof(vo_fe)), *r1 = malloc(R * sizeof(vo_fe));
    vo_fe *ru = malloc(R * sizeof(vo_fe)), *rv = malloc(R * sizeof(vo_fe));
    rng_fill(&g, r0, R);
    rng_fill(&g, r1, R);
    vo_fe al = fone(), be = fe(0, 0), claim;
    vo_v_res(L[Lo], 6, r0, &claim);   /* V_output (:134-150) */
    vo_lp *V = malloc(NE * sizeof(vo_lp)), *AV = malloc(NE * sizeof(vo_lp)), *AM = malloc(NE * sizeof(vo_lp));
    int ok = 1, nm = 0;
    vo_fe *mp = msgs, vu, vv;
    /* addition layer (:238-354): add_mult_sum[j] = beta_g(j / N) over 6 bits */
    for (long j = 0; j < NE; ++j) {
        V[j].a = fe(0, 0); V[j].b = L[Lp][j];
        AV[j].a = AV[j].b = fe(0, 0);
        AM[j].a = fe(0, 0); AM[j].b = bgat(r0, r1, 6, al, be, j >> lg);
    }
    rng_fill(&g, ru, lg + 6);
    rng_fill(&g, rv, lg + 6);
    ok &= fg_phase(V, AV, AM, lg + 6, ru, &claim, &mp, &vu);
    {
        vo_fe sum = fe(0, 0);
        for (int i = 0; i < 64; ++i) sum = fadd(sum, fmul(bgat(r0, r1, 6, al, be, i), eq_at(ru + lg, 6, i)));
        if (!feq(claim, fmul(sum, vu))) ok = 0;
    }
    vals[nm++] = vu;
    memcpy(r0, ru, (lg + 6) * sizeof(vo_fe));
    memcpy(r1, rv, (lg + 6) * sizeof(vo_fe));
    claim = fmul(al, vu);
    /* multiplication layer (:356-489): add_mult_sum[i] = sum_j beta_g(jN + i) ep_j^i */
    for (long i = 0; i < N; ++i) {
        V[i].a = fe(0, 0); V[i].b = L[Ls][i];
        AV[i].a = AV[i].b = fe(0, 0);
        AM[i].a = AM[i].b = fe(0, 0);
    }
    for (int j = 0; j < 64; ++j) {
        vo_fe x = fone();
        for (long i = 0; i < N; ++i) {
            AM[i].b = fadd(AM[i].b, fmul(bgat(r0, r1, lg + 6, al, be, (long)j * N + i), x));
            x = fmul(x, ep[j]);
        }
    }
    rng_fill(&g, ru, lg);
    rng_fill(&g, rv, lg);
    ok &= fg_phase(V, AV, AM, lg, ru, &claim, &mp, &vu);
    {
        vo_fe sum = fe(0, 0);
        for (int i = 0; i < 64; ++i) {
            vo_fe t0 = al, t1 = be, u0 = fone(), u1 = fone(), x = ep[i];
            for (int j = 0; j < 6; ++j) {
                t0 = fmul(t0, ((i >> j) & 1) ? r0[lg + j] : fomr(r0[lg + j]));
                t1 = fmul(t1, ((i >> j) & 1) ? r1[lg + j] : fomr(r1[lg + j]));
            }
            for (int j = 0; j < lg; ++j) {
                u0 = fmul(u0, fadd(fmul(fmul(r0[j], ru[j]), x), fmul(fomr(r0[j]), fomr(ru[j]))));
                u1 = fmul(u1, fadd(fmul(fmul(r1[j], ru[j]), x), fmul(fomr(r1[j]), fomr(ru[j]))));
                x = fmul(x, x);
            }
            sum = fadd(sum, fadd(fmul(t0, u0), fmul(t1, u1)));
        }
        if (!feq(claim, fmul(sum, vu))) ok = 0;
    }
    vals[nm++] = vu;
    memcpy(r0, ru, lg * sizeof(vo_fe));
    memcpy(r1, rv, lg * sizeof(vo_fe));
    claim = fmul(al, vu);
    /* intermediate layer (:491-496) */
    claim = fmul(claim, fconst((uint64_t)N));
    /* inverse FFT levels (:498-768) */
    for (int dep = 0; dep < lg; ++dep) {
        const long half = 1L << (lg - dep - 1);
        const int pre = lg + (lg - dep) - 1;
        const vo_fe *pv = L[pre];
        for (long i = 0; i < N; ++i) {
            V[i].a = fe(0, 0); V[i].b = pv[i];
            AV[i].a = AV[i].b = AM[i].a = AM[i].b = fe(0, 0);
        }
        vo_fe x = fone();
        for (long k = 0; k < half; ++k) {
            for (long j = 0; j < (1L << dep); ++j) {
                const long u = k << (dep + 1) | j, v = u | (1L << dep);
                const vo_fe b1 = bgat(r0, r1, lg, al, be, k << dep | j), b2 = bgat(r0, r1, lg, al, be, (k + half) << dep | j);
                AM[u].b = fadd(AM[u].b, fadd(b1, b2));
                AV[u].b = fadd(AV[u].b, fmul(fmul(x, pv[v]), fsub(b1, b2)));
            }
            x = fmul(x, rot[dep]);
        }
        rng_fill(&g, ru, lg);
        rng_fill(&g, rv, lg);
        ok &= fg_phase(V, AV, AM, lg, ru, &claim, &mp, &vu);
        for (long i = 0; i < N; ++i) {
            V[i].a = fe(0, 0); V[i].b = pv[i];
            AV[i].a = AV[i].b = AM[i].a = AM[i].b = fe(0, 0);
        }
        x = fone();
        for (long k = 0; k < half; ++k) {
            for (long j = 0; j < (1L << dep); ++j) {
                const long u = k << (dep + 1) | j, v = u | (1L << dep);
                const vo_fe bu = eq_at(ru, lg, u);
                const vo_fe t1 = fmul(bgat(r0, r1, lg, al, be, k << dep | j), bu);
                const vo_fe t2 = fmul(bgat(r0, r1, lg, al, be, (k + half) << dep | j), bu);
                AM[v].b = fadd(AM[v].b, fmul(x, fsub(t1, t2)));
                AV[v].b = fadd(AV[v].b, fmul(vu, fadd(t1, t2)));
            }
            x = fmul(x, rot[dep]);
        }
        ok &= fg_phase(V, AV, AM, lg, rv, &claim, &mp, &vv);
        /* the verifier's closed form (:681-750) */
        {
            const int lk = lg - dep - 1, lj = dep;
            vo_fe w = rot[dep];
            const vo_fe c0 = fmul(fomr(ru[lj]), rv[lj]);
            vo_fe uA0 = fmul(fmul(fomr(r0[lg - 1]), c0), al), uA1 = fmul(fmul(fomr(r1[lg - 1]), c0), be);
            vo_fe vA0 = uA0, vA1 = uA1;
            vo_fe uB0 = fmul(fmul(r0[lg - 1], c0), al), uB1 = fmul(fmul(r1[lg - 1], c0), be);
            vo_fe vB0 = uB0, vB1 = uB1;
            for (int i = 0; i < lk; ++i) {
                const vo_fe su = ru[lj + 1 + i], sv = rv[lj + 1 + i];
                const vo_fe e0 = fmul(fmul(r0[lj + i], su), sv), n0 = fmul(fmul(fomr(r0[lj + i]), fomr(su)), fomr(sv));
                const vo_fe e1 = fmul(fmul(r1[lj + i], su), sv), n1 = fmul(fmul(fomr(r1[lj + i]), fomr(su)), fomr(sv));
                uA0 = fmul(uA0, fadd(e0, n0)); uA1 = fmul(uA1, fadd(e1, n1));
                vA0 = fmul(vA0, fadd(fmul(e0, w), n0)); vA1 = fmul(vA1, fadd(fmul(e1, w), n1));
                uB0 = fmul(uB0, fadd(e0, n0)); uB1 = fmul(uB1, fadd(e1, n1));
                vB0 = fmul(vB0, fadd(n0, fmul(e0, w))); vB1 = fmul(vB1, fadd(n1, fmul(e1, w)));
                w = fmul(w, w);
            }
            for (int i = 0; i < lj; ++i) {
                const vo_fe t0 = fadd(fmul(fmul(r0[i], ru[i]), rv[i]), fmul(fmul(fomr(r0[i]), fomr(ru[i])), fomr(rv[i])));
                const vo_fe t1 = fadd(fmul(fmul(r1[i], ru[i]), rv[i]), fmul(fmul(fomr(r1[i]), fomr(ru[i])), fomr(rv[i])));
                uA0 = fmul(uA0, t0); uA1 = fmul(uA1, t1); vA0 = fmul(vA0, t0); vA1 = fmul(vA1, t1);
                uB0 = fmul(uB0, t0); uB1 = fmul(uB1, t1); vB0 = fmul(vB0, t0); vB1 = fmul(vB1, t1);
            }
            const vo_fe want = fadd(fmul(fadd(fadd(uA0, uA1), fadd(uB0, uB1)), vu),
                                    fmul(fsub(fadd(vA0, vA1), fadd(vB0, vB1)), vv));
            if (!feq(claim, want)) ok = 0;
        }
        vals[nm++] = vu;
        vals[nm++] = vv;
        memcpy(r0, ru, lg * sizeof(vo_fe));
        memcpy(r1, rv, lg * sizeof(vo_fe));
        al = rng_fe(&g);
        be = rng_fe(&g);
        claim = fadd(fmul(al, vu), fmul(be, vv));
    }
    /* proof size (:323-324 per message; extension_gkr :770-779) */
    *proof_size = 48 * (vo_fft_gkr_rounds(lg) + lg * (lg + 1) / 2);
    for (int i = 0; i < nl; ++i) free(L[i]);
    free(L); free(r); free(xa); free(r0); free(r1); free(ru); free(rv); free(V); free(AV); free(AM);
    return ok;
}
