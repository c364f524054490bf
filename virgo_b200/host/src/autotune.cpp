// Autotuner over the device's launch-shape parameters (VG_TUNE_*).
//
// Coordinate search: each parameter in turn is swept over its candidates
// with the others fixed at the best found so far, timing whole proofs of the
// caller's sessions (all of them at once through vg_session_prove_batch, so
// n > 1 tunes the throughput of n proofs in flight and n = 1 one proof's
// latency).  Whole proofs are the objective because the parameters interact
// with the overlap of the sumcheck, commitment and side-proof streams: a
// faster NTT on the commitment stream, for instance, buys nothing when the
// commitment is not on the proof's critical path.  Every candidate gets one
// warm-up batch, then `reps` timed batches of which the fastest counts; a
// candidate replaces the value in force only when it is faster by more than
// 3% (repeated batches of one setting vary by up to 2.5% on one box), so
// timing noise leaves the defaults alone.
//
// Every parameter value gives bit-identical proofs (the tests prove each one
// against the same transcripts), so the tuner never changes a result.
#include <chrono>
#include <limits>
#include <vector>
#include "virgo_b200.h"

int vg_fail(int code, const char *fmt, ...);

namespace {

struct Knob {
    int key;
    std::vector<long> cands;
};

// candidates per parameter; the defaults are among them
const std::vector<Knob> &knobs()
{
    static const std::vector<Knob> k = {
        {VG_TUNE_GROUP_START, {1L << 11, 1L << 13, 1L << 15, 1L << 17, 1L << 19}},
        {VG_TUNE_ROUND_FUSE, {1, 2}},
        {VG_TUNE_ROUND_THREADS, {128, 256, 512}},
        {VG_TUNE_BETA_TABLE, {0, 1}},
        {VG_TUNE_GROUP_SPLIT, {0, 1}},
        {VG_TUNE_LAZY_FOLD, {0, 1}},
        {VG_TUNE_GATHER_FUSE, {0, 1}},
        {VG_TUNE_NTT_MAX_LOG, {8, 9, 10}},
        {VG_TUNE_NTT_TILE_LOG, {11, 12, 13}},
        {VG_TUNE_LEAF_THREADS, {64, 128, 256}},
        {VG_TUNE_LEAF_ROT, {0, 1, 2, 3}},
        {VG_TUNE_LEAF_WARP_MAX, {0, 1024, 8192}},
    };
    return k;
}

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" int vg_autotune(vg_session *const *ss, int n, unsigned seed, int reps, vg_tune_trial *trials, int max_trials,
                           int *n_trials)
{
    if (!ss || n < 1 || reps < 1 || (max_trials > 0 && !trials) || max_trials < 0)
        return vg_fail(VG_ERR_ARG, "vg_autotune: bad argument (n=%d reps=%d max_trials=%d)", n, reps, max_trials);
    for (int i = 0; i < n; ++i)
        if (!ss[i]) return vg_fail(VG_ERR_ARG, "vg_autotune: session %d is null", i);
    vg_ctx *ctx = nullptr;
    int dev = 0, rc = vg_session_ctx(ss[0], &ctx);
    if (rc != VG_OK) return rc;
    if ((rc = vg_ctx_device(ctx, &dev)) != VG_OK) return rc;
    std::vector<unsigned> seeds(n);
    for (int i = 0; i < n; ++i) seeds[i] = seed + (unsigned)i;

    auto time_batch = [&](double *best) -> int {
        int r = vg_session_prove_batch(ss, n, seeds.data(), 0, nullptr, nullptr, nullptr);   // warm-up
        if (r != VG_OK) return r;
        *best = std::numeric_limits<double>::infinity();
        for (int k = 0; k < reps; ++k) {
            const double t0 = now_ms();
            r = vg_session_prove_batch(ss, n, seeds.data(), 0, nullptr, nullptr, nullptr);
            if (r != VG_OK) return r;
            const double dt = now_ms() - t0;
            if (dt < *best) *best = dt;
        }
        return VG_OK;
    };

    int nt = 0;
    auto record = [&](int key, long value, double ms) -> int {
        if (nt < max_trials) {
            trials[nt].key = key;
            trials[nt].value = value;
            trials[nt].ms = ms;
            trials[nt].chosen = 0;
        }
        return nt++;
    };

    for (const Knob &kb : knobs()) {
        long cur = 0;
        if ((rc = vg_tune_get(dev, kb.key, &cur)) != VG_OK) return rc;
        double cur_ms = 0;
        if ((rc = time_batch(&cur_ms)) != VG_OK) return rc;
        int best_trial = record(kb.key, cur, cur_ms);
        long best = cur;
        double best_ms = cur_ms;
        for (long v : kb.cands) {
            if (v == cur) continue;
            if ((rc = vg_tune_set(dev, kb.key, v)) != VG_OK) return rc;
            double ms = 0;
            rc = time_batch(&ms);
            if (rc != VG_OK) {
                vg_tune_set(dev, kb.key, cur);
                return rc;
            }
            const int t = record(kb.key, v, ms);
            if (ms < best_ms && ms < 0.97 * cur_ms) {
                best = v;
                best_ms = ms;
                best_trial = t;
            }
        }
        if ((rc = vg_tune_set(dev, kb.key, best)) != VG_OK) return rc;
        if (best_trial < max_trials) trials[best_trial].chosen = 1;
    }
    if (n_trials) *n_trials = nt < max_trials ? nt : max_trials;
    return VG_OK;
}
