// The kernel-level commit path run by the reference itself, through its
// poly_commit API (include/poly_commitment/README.md:1-86).  TEST
// INFRASTRUCTURE ONLY: it produces the golden roots, sums, final codeword and
// query answers that vg_pc_commit_all is checked against, and times the
// reference on that path.
//
//   commit_ref <in.bin> <out.bin>
//
// in.bin, little-endian: int32 log_len, n_pri_mask, n_pub_mask; uint32 seed;
// int32 nq; nq x (int32 which, int64 pos); then the field elements
// (16 bytes each, {img, real}): private[2^log_len], public[2^log_len],
// private mask[n_pri_mask], public mask[n_pub_mask].
//
// Steps, as a user of the API takes them:
//   poly_commit_prover::commit_private_array   (poly_commit.h:42-124)
//   poly_commit_prover::commit_public_array    (poly_commit.h:125-351) with
//       target_sum = <private, public> + <padded private mask, public mask>
//       (the claim the function asserts, poly_commit.h:179-193)
//   srand(seed); poly_commit_prover::commit_phase (vpd_verifier.cpp:46-78),
//       which draws one prime_field::random() per FRI level
//   fri::request_init_value_with_merkle (fri.cpp:148-201) for which 0 / 1 at
//       (pos, pos + S/2), fri::request_step_commit (fri.cpp:227-289) for
//       which 2 + t at pos.
//
// out.bin: int32 nlevels; roots (2 + nlevels) x 32 bytes (l, h, FRI level t);
// all_sum[65]; randomness[nlevels]; int32 n (final per-slice length); the
// final level cpd.rs_codeword[nlevels - 1] (64 * n elements, the reference's
// interleaved layout (j << 7) | (s << 1) | b of the 64 data slices) and
// cpd.rs_codeword_msk[nlevels - 1] (n elements); per query 130 values,
// int32 path length, the path digests; three doubles: the seconds of
// commit_private_array, commit_public_array and commit_phase.
#include "poly_commitment/poly_commit.h"
#include "VPD/fri.h"
#include "linear_gkr/prime_field.h"
#include "infrastructure/constants.h"
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

typedef prime_field::field_element fe;

static void rd(FILE *f, void *p, size_t n)
{
    if (fread(p, 1, n, f) != n) {
        fprintf(stderr, "commit_ref: short input\n");
        exit(2);
    }
}

static void wr(FILE *f, const void *p, size_t n)
{
    if (fwrite(p, 1, n, f) != n) {
        fprintf(stderr, "commit_ref: short write\n");
        exit(2);
    }
}

static double since(std::chrono::high_resolution_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
}

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE *in = fopen(argv[1], "rb");
    if (!in) return 2;
    int32_t log_len, n_pri, n_pub, nq;
    uint32_t seed;
    rd(in, &log_len, 4);
    rd(in, &n_pri, 4);
    rd(in, &n_pub, 4);
    rd(in, &seed, 4);
    rd(in, &nq, 4);
    std::vector<int32_t> which(nq);
    std::vector<int64_t> pos(nq);
    for (int q = 0; q < nq; ++q) {
        rd(in, &which[q], 4);
        rd(in, &pos[q], 8);
    }
    const long n = 1L << log_len;
    fe *priv = new fe[n], *pub = new fe[n];
    std::vector<fe> pri_mask(n_pri), pub_mask(n_pub);
    rd(in, priv, n * sizeof(fe));
    rd(in, pub, n * sizeof(fe));
    rd(in, pri_mask.data(), n_pri * sizeof(fe));
    rd(in, pub_mask.data(), n_pub * sizeof(fe));
    fclose(in);

    prime_field::init();
    poly_commit::poly_commit_prover prover;
    double secs[3];

    auto t0 = std::chrono::high_resolution_clock::now();
    __hhash_digest root_l = prover.commit_private_array(priv, log_len, pri_mask);
    secs[0] = since(t0);

    // the claim commit_public_array asserts: the sampled inner product plus
    // the masks' (the private mask as padded by commit_private_array)
    fe target(0);
    for (long i = 0; i < n; ++i) target = target + priv[i] * pub[i];
    for (int k = 0; k < n_pub && k < (int)prover.all_pri_mask.size(); ++k)
        target = target + prover.all_pri_mask[k] * pub_mask[k];
    fe *all_sum = new fe[slice_number + 1];
    t0 = std::chrono::high_resolution_clock::now();
    __hhash_digest root_h = prover.commit_public_array(pub_mask, pub, log_len, target, all_sum);
    secs[1] = since(t0);

    srand(seed);
    t0 = std::chrono::high_resolution_clock::now();
    poly_commit::ldt_commitment com = prover.commit_phase(log_len);
    secs[2] = since(t0);
    const int nlevels = com.mx_depth;

    FILE *out = fopen(argv[2], "wb");
    if (!out) return 2;
    wr(out, &nlevels, 4);
    wr(out, &root_l, 32);
    wr(out, &root_h, 32);
    for (int t = 0; t < nlevels; ++t) wr(out, &com.commitment_hhash[t], 32);
    wr(out, all_sum, (slice_number + 1) * sizeof(fe));
    wr(out, com.randomness, nlevels * sizeof(fe));
    const int S = 1 << (log_len + rs_code_rate - log_slice_number);
    const int32_t fin_n = S >> nlevels;
    wr(out, &fin_n, 4);
    wr(out, fri::cpd.rs_codeword[nlevels - 1], (size_t)fin_n * slice_number * sizeof(fe));
    wr(out, fri::cpd.rs_codeword_msk[nlevels - 1], (size_t)fin_n * sizeof(fe));
    for (int q = 0; q < nq; ++q) {
        int new_size = 0;
        std::pair<std::vector<std::pair<fe, fe>>, std::vector<__hhash_digest>> ans;
        if (which[q] < 2)
            ans = fri::request_init_value_with_merkle(pos[q], pos[q] + S / 2, new_size, which[q]);
        else
            ans = fri::request_step_commit(which[q] - 2, pos[q], new_size);
        if (ans.first.size() != slice_number + 1) {
            fprintf(stderr, "commit_ref: query %d returned %zu pairs\n", q, ans.first.size());
            return 3;
        }
        for (auto &pr : ans.first) {
            wr(out, &pr.first, sizeof(fe));
            wr(out, &pr.second, sizeof(fe));
        }
        int32_t plen = (int32_t)ans.second.size();
        wr(out, &plen, 4);
        wr(out, ans.second.data(), plen * sizeof(__hhash_digest));
    }
    wr(out, secs, sizeof(secs));
    fclose(out);
    printf("commit_ref: log_len %d, commit_private %.3f s, commit_public %.3f s, commit_phase %.3f s\n", log_len,
           secs[0], secs[1], secs[2]);
    return 0;
}
