// Transcript recorder for prover binaries that are driven by the reference
// verifier.  TEST INFRASTRUCTURE ONLY: linked into the oracle binaries under
// oracle/_ref/, never into the product library.
//
// The recorder interposes on every prover entry point that the reference
// verifier calls (src/linear_gkr/zk_verifier.cpp:910-1253 and
// src/VPD/vpd_verifier.cpp:80-335) with GNU ld's --wrap option: a call from the
// verifier's object file to symbol S is routed to __wrap_S, which calls
// __real_S and appends the returned message to the transcript.  The same source
// is compiled once against the reference headers (pure CPU reference prover) and
// once against this repository's drop-in headers (GPU prover under the
// unchanged reference verifier), so the two transcripts are byte-comparable.
//
// Record layout: 1 byte tag, uint32 count of 16-byte units, then the units.
// Field elements are written as {img, real} (16 bytes, the in-memory layout of
// prime_field::field_element); a 32-byte digest counts as two units.

#include "linear_gkr/zk_prover.h"
#include "linear_gkr/polynomial.h"
#include "VPD/fri.h"
#include "poly_commitment/poly_commit.h"
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <vector>
#include <utility>

typedef prime_field::field_element fe;
typedef std::pair<std::vector<std::pair<fe, fe> >, std::vector<__hhash_digest> > query_answer;

static FILE *g_tr = nullptr;

extern "C" void virgo_transcript_open(const char *path)
{
    g_tr = path ? fopen(path, "wb") : nullptr;
}
extern "C" void virgo_transcript_close()
{
    if (g_tr) fclose(g_tr);
    g_tr = nullptr;
}

static void put(char tag, const void *units, uint32_t n16)
{
    if (!g_tr) return;
    fputc(tag, g_tr);
    fwrite(&n16, 4, 1, g_tr);
    if (n16) fwrite(units, 16, n16, g_tr);
}
static void put_fe(char tag, const fe &x) { put(tag, &x, 1); }

static void put_answer(char tag, const query_answer &a, int new_size)
{
    std::vector<unsigned char> buf;
    buf.resize(16 + a.first.size() * 32 + a.second.size() * 32);
    int64_t hdr[2] = {(int64_t)new_size, (int64_t)((a.first.size() << 16) | a.second.size())};
    memcpy(buf.data(), hdr, 16);
    size_t off = 16;
    for (auto &pv : a.first) {
        memcpy(&buf[off], &pv.first, 16);
        memcpy(&buf[off + 16], &pv.second, 16);
        off += 32;
    }
    for (auto &h : a.second) {
        memcpy(&buf[off], &h, 32);
        off += 32;
    }
    put(tag, buf.data(), (uint32_t)(buf.size() / 16));
}

#define REAL(sym) __real_##sym
#define WRAP(sym) __wrap_##sym

extern "C" {

// zk_prover::V_res  (src/linear_gkr/zk_prover.cpp:30)
fe REAL(_ZN9zk_prover5V_resEPKN11prime_field13field_elementES3_S3_ii)(zk_prover *, const fe *, const fe *, const fe *, int, int);
fe WRAP(_ZN9zk_prover5V_resEPKN11prime_field13field_elementES3_S3_ii)(zk_prover *p, const fe *a, const fe *b, const fe *c, int n, int m)
{
    fe r = REAL(_ZN9zk_prover5V_resEPKN11prime_field13field_elementES3_S3_ii)(p, a, b, c, n, m);
    put_fe('R', r);
    return r;
}

// zk_prover::generate_maskpoly_after_rho  (zk_prover.cpp:174)
void REAL(_ZN9zk_prover27generate_maskpoly_after_rhoEii)(zk_prover *, int, int);
void WRAP(_ZN9zk_prover27generate_maskpoly_after_rhoEii)(zk_prover *p, int a, int b)
{
    REAL(_ZN9zk_prover27generate_maskpoly_after_rhoEii)(p, a, b);
    put_fe('S', p->maskpoly_sumc);
}

// zk_prover::sumcheck_phase1_update  (zk_prover.cpp:596)
quadratic_poly REAL(_ZN9zk_prover22sumcheck_phase1_updateEN11prime_field13field_elementEi)(zk_prover *, fe, int);
quadratic_poly WRAP(_ZN9zk_prover22sumcheck_phase1_updateEN11prime_field13field_elementEi)(zk_prover *p, fe r, int bit)
{
    quadratic_poly q = REAL(_ZN9zk_prover22sumcheck_phase1_updateEN11prime_field13field_elementEi)(p, r, bit);
    fe u[3] = {q.a, q.b, q.c};
    put('q', u, 3);
    return q;
}

// zk_prover::sumcheck_phase1_updatelastbit  (zk_prover.cpp:680)
quintuple_poly REAL(_ZN9zk_prover29sumcheck_phase1_updatelastbitEN11prime_field13field_elementEi)(zk_prover *, fe, int);
quintuple_poly WRAP(_ZN9zk_prover29sumcheck_phase1_updatelastbitEN11prime_field13field_elementEi)(zk_prover *p, fe r, int bit)
{
    quintuple_poly q = REAL(_ZN9zk_prover29sumcheck_phase1_updatelastbitEN11prime_field13field_elementEi)(p, r, bit);
    fe u[6] = {q.a, q.b, q.c, q.d, q.e, q.f};
    put('p', u, 6);
    return q;
}

// zk_prover::sumcheck_phase2_init  (zk_prover.cpp:789); records v_u
void REAL(_ZN9zk_prover20sumcheck_phase2_initEN11prime_field13field_elementEPKS1_S3_)(zk_prover *, fe, const fe *, const fe *);
void WRAP(_ZN9zk_prover20sumcheck_phase2_initEN11prime_field13field_elementEPKS1_S3_)(zk_prover *p, fe r, const fe *ru, const fe *omru)
{
    REAL(_ZN9zk_prover20sumcheck_phase2_initEN11prime_field13field_elementEPKS1_S3_)(p, r, ru, omru);
    put_fe('u', p->v_u);
}

// zk_prover::sumcheck_phase2_update  (zk_prover.cpp:988)
quadratic_poly REAL(_ZN9zk_prover22sumcheck_phase2_updateEN11prime_field13field_elementEi)(zk_prover *, fe, int);
quadratic_poly WRAP(_ZN9zk_prover22sumcheck_phase2_updateEN11prime_field13field_elementEi)(zk_prover *p, fe r, int bit)
{
    quadratic_poly q = REAL(_ZN9zk_prover22sumcheck_phase2_updateEN11prime_field13field_elementEi)(p, r, bit);
    fe u[3] = {q.a, q.b, q.c};
    put('Q', u, 3);
    return q;
}

// zk_prover::sumcheck_phase2_updatelastbit  (zk_prover.cpp:1071)
quintuple_poly REAL(_ZN9zk_prover29sumcheck_phase2_updatelastbitEN11prime_field13field_elementEi)(zk_prover *, fe, int);
quintuple_poly WRAP(_ZN9zk_prover29sumcheck_phase2_updatelastbitEN11prime_field13field_elementEi)(zk_prover *p, fe r, int bit)
{
    quintuple_poly q = REAL(_ZN9zk_prover29sumcheck_phase2_updatelastbitEN11prime_field13field_elementEi)(p, r, bit);
    fe u[6] = {q.a, q.b, q.c, q.d, q.e, q.f};
    put('P', u, 6);
    return q;
}

// zk_prover::sumcheck_finalize  (zk_prover.cpp:1206)
std::pair<fe, fe> REAL(_ZN9zk_prover17sumcheck_finalizeEN11prime_field13field_elementE)(zk_prover *, fe);
std::pair<fe, fe> WRAP(_ZN9zk_prover17sumcheck_finalizeEN11prime_field13field_elementE)(zk_prover *p, fe r)
{
    std::pair<fe, fe> v = REAL(_ZN9zk_prover17sumcheck_finalizeEN11prime_field13field_elementE)(p, r);
    fe u[2] = {v.first, v.second};
    put('z', u, 2);
    return v;
}

// zk_prover::sumcheck_finalround  (zk_prover.cpp:1173)
quadratic_poly REAL(_ZN9zk_prover19sumcheck_finalroundEN11prime_field13field_elementEiS1_)(zk_prover *, fe, int, fe);
quadratic_poly WRAP(_ZN9zk_prover19sumcheck_finalroundEN11prime_field13field_elementEiS1_)(zk_prover *p, fe r, int c, fe g)
{
    quadratic_poly q = REAL(_ZN9zk_prover19sumcheck_finalroundEN11prime_field13field_elementEiS1_)(p, r, c, g);
    fe u[3] = {q.a, q.b, q.c};
    put('f', u, 3);
    return q;
}

// zk_prover::query / queryRg1 / queryRg2  (zk_prover.cpp:284-314)
fe REAL(_ZN9zk_prover5queryEPN11prime_field13field_elementES2_S1_)(zk_prover *, fe *, fe *, fe);
fe WRAP(_ZN9zk_prover5queryEPN11prime_field13field_elementES2_S1_)(zk_prover *p, fe *u, fe *v, fe c)
{
    fe r = REAL(_ZN9zk_prover5queryEPN11prime_field13field_elementES2_S1_)(p, u, v, c);
    put_fe('y', r);
    return r;
}
fe REAL(_ZN9zk_prover8queryRg1EN11prime_field13field_elementE)(zk_prover *, fe);
fe WRAP(_ZN9zk_prover8queryRg1EN11prime_field13field_elementE)(zk_prover *p, fe c)
{
    fe r = REAL(_ZN9zk_prover8queryRg1EN11prime_field13field_elementE)(p, c);
    put_fe('g', r);
    return r;
}
fe REAL(_ZN9zk_prover8queryRg2EN11prime_field13field_elementE)(zk_prover *, fe);
fe WRAP(_ZN9zk_prover8queryRg2EN11prime_field13field_elementE)(zk_prover *p, fe c)
{
    fe r = REAL(_ZN9zk_prover8queryRg2EN11prime_field13field_elementE)(p, c);
    put_fe('h', r);
    return r;
}

// fri::request_init_commit  (src/VPD/fri.cpp:36): the witness Merkle roots
__hhash_digest REAL(_ZN3fri19request_init_commitEii)(int, int);
__hhash_digest WRAP(_ZN3fri19request_init_commitEii)(int bl, int oi)
{
    __hhash_digest h = REAL(_ZN3fri19request_init_commitEii)(bl, oi);
    put('C', &h, 2);
    return h;
}

// fri::commit_phase_step  (fri.cpp:291): one FRI level root
__hhash_digest REAL(_ZN3fri17commit_phase_stepEN11prime_field13field_elementE)(fe);
__hhash_digest WRAP(_ZN3fri17commit_phase_stepEN11prime_field13field_elementE)(fe r)
{
    __hhash_digest h = REAL(_ZN3fri17commit_phase_stepEN11prime_field13field_elementE)(r);
    put('T', &h, 2);
    return h;
}

// fri::commit_phase_final  (fri.cpp:432): the last folded codeword, data and mask
fe *REAL(_ZN3fri18commit_phase_finalEv)();
fe *WRAP(_ZN3fri18commit_phase_finalEv)()
{
    fe *r = REAL(_ZN3fri18commit_phase_finalEv)();
    int n = 1 << fri::log_current_witness_size_per_slice;
    put('X', r, (uint32_t)(n * slice_number));
    put('x', fri::cpd.rs_codeword_msk[fri::current_step_no - 1], (uint32_t)n);
    return r;
}

// fri::request_init_value_with_merkle  (fri.cpp:148)
query_answer REAL(_ZN3fri30request_init_value_with_merkleExxRii)(long long, long long, int &, int);
query_answer WRAP(_ZN3fri30request_init_value_with_merkleExxRii)(long long a, long long b, int &ns, int oi)
{
    query_answer q = REAL(_ZN3fri30request_init_value_with_merkleExxRii)(a, b, ns, oi);
    put_answer('I', q, ns);
    return q;
}

// fri::request_step_commit  (fri.cpp:227)
query_answer REAL(_ZN3fri19request_step_commitEixRi)(int, long long, int &);
query_answer WRAP(_ZN3fri19request_step_commitEixRi)(int lvl, long long pw, int &ns)
{
    query_answer q = REAL(_ZN3fri19request_step_commitEixRi)(lvl, pw, ns);
    put_answer('J', q, ns);
    return q;
}

// poly_commit_verifier::verify_poly_commitment  (src/VPD/vpd_verifier.cpp:80):
// records all_sum[0..slice_number] and both witness roots as handed over.
bool REAL(_ZN11poly_commit20poly_commit_verifier22verify_poly_commitmentEPN11prime_field13field_elementEiS3_RSt6vectorIS2_SaIS2_EERdRiS8_14__hhash_digestSA_)(
    poly_commit::poly_commit_verifier *, fe *, int, fe *, std::vector<fe> &, double &, int &, double &, __hhash_digest, __hhash_digest);
bool WRAP(_ZN11poly_commit20poly_commit_verifier22verify_poly_commitmentEPN11prime_field13field_elementEiS3_RSt6vectorIS2_SaIS2_EERdRiS8_14__hhash_digestSA_)(
    poly_commit::poly_commit_verifier *v, fe *all_sum, int ll, fe *pub, std::vector<fe> &msk, double &vt, int &ps, double &pt, __hhash_digest l, __hhash_digest h)
{
    put('A', all_sum, slice_number + 1);
    __hhash_digest lh[2] = {l, h};
    put('B', lh, 4);
    bool ok = REAL(_ZN11poly_commit20poly_commit_verifier22verify_poly_commitmentEPN11prime_field13field_elementEiS3_RSt6vectorIS2_SaIS2_EERdRiS8_14__hhash_digestSA_)(
        v, all_sum, ll, pub, msk, vt, ps, pt, l, h);
    uint64_t res[2] = {(uint64_t)ok, (uint64_t)(int64_t)ps};
    put('V', res, 1);
    return ok;
}

}  // extern "C"

// The list of symbols above, for the link line (kept in one place).
extern "C" const char *virgo_transcript_wrapped_symbols =
    "_ZN9zk_prover5V_resEPKN11prime_field13field_elementES3_S3_ii "
    "_ZN9zk_prover27generate_maskpoly_after_rhoEii "
    "_ZN9zk_prover22sumcheck_phase1_updateEN11prime_field13field_elementEi "
    "_ZN9zk_prover29sumcheck_phase1_updatelastbitEN11prime_field13field_elementEi "
    "_ZN9zk_prover20sumcheck_phase2_initEN11prime_field13field_elementEPKS1_S3_ "
    "_ZN9zk_prover22sumcheck_phase2_updateEN11prime_field13field_elementEi "
    "_ZN9zk_prover29sumcheck_phase2_updatelastbitEN11prime_field13field_elementEi "
    "_ZN9zk_prover17sumcheck_finalizeEN11prime_field13field_elementE "
    "_ZN9zk_prover19sumcheck_finalroundEN11prime_field13field_elementEiS1_ "
    "_ZN9zk_prover5queryEPN11prime_field13field_elementES2_S1_ "
    "_ZN9zk_prover8queryRg1EN11prime_field13field_elementE "
    "_ZN9zk_prover8queryRg2EN11prime_field13field_elementE "
    "_ZN3fri19request_init_commitEii "
    "_ZN3fri17commit_phase_stepEN11prime_field13field_elementE "
    "_ZN3fri18commit_phase_finalEv "
    "_ZN3fri30request_init_value_with_merkleExxRii "
    "_ZN3fri19request_step_commitEixRi "
    "_ZN11poly_commit20poly_commit_verifier22verify_poly_commitmentEPN11prime_field13field_elementEiS3_RSt6vectorIS2_SaIS2_EERdRiS8_14__hhash_digestSA_";
