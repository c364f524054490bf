// Launch-shape parameters, one set per device, read by the kernels' host
// wrappers at every launch (vg_tune_value).  Every value of every parameter
// computes the same results bit for bit; the parameters only move work
// between launches, CTAs and threads.  vg_autotune (host/src/session.cpp)
// chooses them by timing proofs; vg_tune_set sets them by hand.
#include "common.cuh"
#include <atomic>

namespace {

constexpr int MAX_DEVICES = 64;

struct Range {
    long lo, hi, def;
    bool pow2;
};

// VG_TUNE_* order.  The defaults are the fastest shapes measured for one
// 256x256-matmul proof on a B200; with eight such proofs in flight the
// autotuner finds no candidate more than 2% faster than them.
const Range RANGES[VG_TUNE_COUNT] = {
    {1L << 11, 1L << 22, 1L << 17, true},   // GROUP_START: table length at which round groups take over
    {128, 512, 256, true},                  // ROUND_THREADS
    {6, 10, 10, false},                     // NTT_MAX_LOG
    {10, 13, 12, false},                    // NTT_TILE_LOG
    {64, 256, 256, true},                   // LEAF_THREADS
    {0, 1L << 24, 0, false},                // LEAF_WARP_MAX
    {1, 2, 2, false},                       // ROUND_FUSE
    {0, 3, 3, false},                       // LEAF_ROT
    {0, 1, 1, false},                       // BETA_TABLE
    {0, 1, 0, false},                       // GROUP_SPLIT
    {0, 1, 0, false},                       // LAZY_FOLD
    {0, 1, 1, false},                       // GATHER_FUSE
};

std::atomic<long> g_tune[MAX_DEVICES][VG_TUNE_COUNT];

// defaults for every device when the library loads
struct Init {
    Init()
    {
        for (int d = 0; d < MAX_DEVICES; ++d)
            for (int k = 0; k < VG_TUNE_COUNT; ++k) g_tune[d][k].store(RANGES[k].def, std::memory_order_relaxed);
    }
} g_init_defaults;

bool valid(int key, long v)
{
    const Range &r = RANGES[key];
    if (v < r.lo || v > r.hi) return false;
    if (r.pow2 && (v & (v - 1))) return false;
    return true;
}

}  // namespace

long vg_tune_value(int device, int key)
{
    if (key < 0 || key >= VG_TUNE_COUNT) return 0;
    if (device < 0 || device >= MAX_DEVICES) return RANGES[key].def;
    return g_tune[device][key].load(std::memory_order_relaxed);
}

extern "C" int vg_tune_get(int device, int key, long *value)
{
    if (!value) return vg_fail(VG_ERR_ARG, "vg_tune_get: null value");
    if (device < 0 || device >= MAX_DEVICES) return vg_fail(VG_ERR_ARG, "vg_tune_get: device %d", device);
    if (key < 0 || key >= VG_TUNE_COUNT) return vg_fail(VG_ERR_ARG, "vg_tune_get: unknown key %d", key);
    *value = vg_tune_value(device, key);
    return VG_OK;
}

extern "C" int vg_tune_set(int device, int key, long value)
{
    if (device < 0 || device >= MAX_DEVICES) return vg_fail(VG_ERR_ARG, "vg_tune_set: device %d", device);
    if (key < 0 || key >= VG_TUNE_COUNT) return vg_fail(VG_ERR_ARG, "vg_tune_set: unknown key %d", key);
    if (!valid(key, value))
        return vg_fail(VG_ERR_ARG, "vg_tune_set: value %ld for key %d outside [%ld, %ld]%s", value, key, RANGES[key].lo,
                       RANGES[key].hi, RANGES[key].pow2 ? " or not a power of two" : "");
    g_tune[device][key].store(value, std::memory_order_relaxed);
    return VG_OK;
}

extern "C" int vg_tune_reset(int device)
{
    if (device < 0 || device >= MAX_DEVICES) return vg_fail(VG_ERR_ARG, "vg_tune_reset: device %d", device);
    for (int k = 0; k < VG_TUNE_COUNT; ++k) g_tune[device][k].store(RANGES[k].def, std::memory_order_relaxed);
    return VG_OK;
}

extern "C" int vg_tune_range(int key, long *lo, long *hi, long *def)
{
    if (key < 0 || key >= VG_TUNE_COUNT) return vg_fail(VG_ERR_ARG, "vg_tune_range: unknown key %d", key);
    if (lo) *lo = RANGES[key].lo;
    if (hi) *hi = RANGES[key].hi;
    if (def) *def = RANGES[key].def;
    return VG_OK;
}
