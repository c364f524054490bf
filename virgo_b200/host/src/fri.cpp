// fri:: functions (reference src/VPD/fri.cpp) over the device commitment state.
// The proof-size bookkeeping of the query functions (which revealed values
// and tree nodes are new) follows the reference's rules exactly; the visited
// sets are sparse here instead of dense arrays sized by the codeword.
#include "VPD/fri.h"
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <unordered_set>
#include "device.h"
#include "poly_commitment/poly_commit.h"

typedef prime_field::field_element F;
typedef std::pair<std::vector<std::pair<F, F> >, std::vector<__hhash_digest> > answer;
using clk = std::chrono::high_resolution_clock;

namespace fri
{
int log_current_witness_size_per_slice = 0, current_step_no = 0, witness_bit_length_per_slice = 0;
commit_phase_data cpd;
double __fri_timer = 0;
__hhash_digest *witness_merkle[2] = {nullptr, nullptr};
}  // namespace fri

static std::unordered_set<long long> g_visited_witness[2], g_visited_init[2];
static std::vector<std::unordered_set<long long> > g_visited_level;

static void sync_hash() { virgo::check(vg_ctx_set_hash(virgo::ctx(), virgo_hash_kind()), "vg_ctx_set_hash"); }

static __hhash_digest to_digest(const vg_digest &d)
{
    __hhash_digest h;
    memcpy(&h, d.bytes, 32);
    return h;
}

__hhash_digest fri::request_init_commit(const int bit_len, const int oracle_indicator)
{
    if (poly_commit::slice_size * poly_commit::slice_count !=
        (1 << (bit_len + rs_code_rate - log_slice_number)) * (1 + (1 << log_slice_number))) {
        fprintf(stderr, "request_init_commit: bit length %d does not match the encoded slices\n", bit_len);
        abort();
    }
    __fri_timer = 0;
    current_step_no = 0;
    log_current_witness_size_per_slice = bit_len + rs_code_rate - log_slice_number;
    witness_bit_length_per_slice = bit_len - log_slice_number;
    auto t0 = clk::now();
    sync_hash();
    vg_digest root;
    virgo::check(vg_pc_init_commit(virgo::pc(), oracle_indicator, &root), "vg_pc_init_commit");
    delete[] witness_merkle[oracle_indicator];
    witness_merkle[oracle_indicator] = new __hhash_digest[2];
    memset(witness_merkle[oracle_indicator], 0, 2 * sizeof(__hhash_digest));
    witness_merkle[oracle_indicator][1] = to_digest(root);
    g_visited_witness[oracle_indicator].clear();
    g_visited_init[oracle_indicator].clear();
    if (oracle_indicator == 0) {
        cpd.delete_self();
        g_visited_level.clear();
    }
    __fri_timer = std::chrono::duration_cast<std::chrono::duration<double>>(clk::now() - t0).count();
    return witness_merkle[oracle_indicator][1];
}

__hhash_digest fri::commit_phase_step(F r)
{
    auto t0 = clk::now();
    const int nxt = (1 << log_current_witness_size_per_slice) / 2;
    sync_hash();
    vg_digest root;
    vg_fe rv;
    rv.real = r.real;
    rv.img = r.img;
    virgo::check(vg_pc_fri_step(virgo::pc(), rv, &root), "vg_pc_fri_step");
    if (!cpd.merkle[current_step_no]) cpd.merkle[current_step_no] = new __hhash_digest[2];
    memset(cpd.merkle[current_step_no], 0, 2 * sizeof(__hhash_digest));
    cpd.merkle[current_step_no][1] = to_digest(root);
    cpd.merkle_size[current_step_no] = nxt / 2;
    if ((int)g_visited_level.size() <= current_step_no) g_visited_level.resize(current_step_no + 1);
    g_visited_level[current_step_no].clear();
    __fri_timer += std::chrono::duration_cast<std::chrono::duration<double>>(clk::now() - t0).count();
    log_current_witness_size_per_slice--;
    return cpd.merkle[current_step_no++][1];
}

F *fri::commit_phase_final()
{
    if (current_step_no == 0) {
        fprintf(stderr, "commit_phase_final before any commit_phase_step\n");
        abort();
    }
    const int t = current_step_no - 1;
    long n = 0;
    virgo::check(vg_pc_fri_final(virgo::pc(), nullptr, nullptr, &n), "vg_pc_fri_final");
    delete[] cpd.rs_codeword[t];
    delete[] cpd.rs_codeword_msk[t];
    cpd.rs_codeword[t] = new F[n * poly_commit::slice_count];
    cpd.rs_codeword_msk[t] = new F[n];
    virgo::check(vg_pc_fri_final(virgo::pc(), (vg_fe *)cpd.rs_codeword[t], (vg_fe *)cpd.rs_codeword_msk[t], &n),
                 "vg_pc_fri_final");
    return cpd.rs_codeword[t];
}

answer fri::request_init_value_with_merkle(long long pow_0, long long pow_1, int &new_size, const int oracle_indicator)
{
    if (pow_0 > pow_1) std::swap(pow_0, pow_1);
    if (pow_0 + (1LL << log_current_witness_size_per_slice) / 2 != pow_1) {
        fprintf(stderr, "request_init_value_with_merkle: %lld and %lld are not a conjugate pair\n", pow_0, pow_1);
        abort();
    }
    const int depth = log_current_witness_size_per_slice - 1;
    vg_fe vals[2 * (slice_number + 1)];
    std::vector<vg_digest> path(depth + 1);
    virgo::check(vg_pc_query_init(virgo::pc(), (long)pow_0, oracle_indicator, vals, path.data()), "vg_pc_query_init");
    new_size = 0;
    answer out;
    auto &seen = g_visited_witness[oracle_indicator];
    for (int i = 0; i < slice_number; ++i) {
        F a, b;
        a.real = vals[2 * i].real; a.img = vals[2 * i].img;
        b.real = vals[2 * i + 1].real; b.img = vals[2 * i + 1].img;
        out.first.push_back(std::make_pair(a, b));
        for (int k = 0; k < 2; ++k)
            if (seen.insert((pow_0 << (log_slice_number + 1)) | (i << 1) | k).second) new_size += sizeof(F);
    }
    F ma, mb;
    ma.real = vals[2 * slice_number].real; ma.img = vals[2 * slice_number].img;
    mb.real = vals[2 * slice_number + 1].real; mb.img = vals[2 * slice_number + 1].img;
    out.first.push_back(std::make_pair(ma, mb));
    out.second.resize(depth + 1);
    long long pos = pow_0 + (1LL << (log_current_witness_size_per_slice - 1));
    out.second[depth] = to_digest(path[depth]);
    auto &nodes = g_visited_init[oracle_indicator];
    for (int i = 0; i < depth; ++i) {
        if (!nodes.count(pos ^ 1)) new_size += sizeof(__hhash_digest);
        nodes.insert(pos);
        nodes.insert(pos ^ 1);
        out.second[i] = to_digest(path[i]);
        pos /= 2;
    }
    return out;
}

answer fri::request_step_commit(int lvl, long long pow, int &new_size)
{
    new_size = 0;
    if (lvl < 0 || lvl >= current_step_no + 64 || lvl >= (int)g_visited_level.size()) {
        fprintf(stderr, "request_step_commit: no FRI level %d\n", lvl);
        abort();
    }
    vg_fe vals[2 * (slice_number + 1)];
    std::vector<vg_digest> path(64);
    int plen = 0;
    virgo::check(vg_pc_query_step(virgo::pc(), lvl, (long)pow, vals, path.data(), &plen), "vg_pc_query_step");
    const long long h = cpd.merkle_size[lvl];
    const long long p = pow % h;
    auto &seen = g_visited_level[lvl];
    bool visited_element = false;
    answer out;
    for (int i = 0; i < slice_number; ++i) {
        if (seen.count((p << (log_slice_number + 1)) | (i << 1))) visited_element = true;
        F a, b;
        a.real = vals[2 * i].real; a.img = vals[2 * i].img;
        b.real = vals[2 * i + 1].real; b.img = vals[2 * i + 1].img;
        out.first.push_back(std::make_pair(a, b));
    }
    if (!visited_element) new_size += sizeof(F);
    F ma, mb;
    ma.real = vals[2 * slice_number].real; ma.img = vals[2 * slice_number].img;
    mb.real = vals[2 * slice_number + 1].real; mb.img = vals[2 * slice_number + 1].img;
    out.first.push_back(std::make_pair(ma, mb));
    long long node = p + h;
    int k = 0;
    while (node != 1) {
        if (!seen.count(node ^ 1)) {
            new_size += sizeof(__hhash_digest);
            seen.insert(node ^ 1);
            seen.insert(node);
        }
        out.second.push_back(to_digest(path[k++]));
        node /= 2;
    }
    out.second.push_back(to_digest(path[plen - 1]));
    return out;
}

void fri::delete_self()
{
    cpd.delete_self();
    for (int k = 0; k < 2; ++k) {
        delete[] witness_merkle[k];
        witness_merkle[k] = nullptr;
    }
}
