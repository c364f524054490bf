#include "device.h"
#include "infrastructure/my_hhash.h"
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace virgo
{
static vg_ctx *g_ctx = nullptr;
static vg_pc *g_pc = nullptr;
static std::once_flag g_once;

static void create()
{
    int dev = 0;
    if (const char *s = getenv("VIRGO_DEVICE")) dev = atoi(s);
    int rc = vg_ctx_create(dev, &g_ctx);
    if (rc != VG_OK) {
        fprintf(stderr, "virgo_b200: cannot create a CUDA context on device %d: %s\n", dev, vg_last_error());
        abort();
    }
    check(vg_ctx_set_hash(g_ctx, virgo_hash_kind()), "vg_ctx_set_hash");
    check(vg_pc_create(g_ctx, &g_pc), "vg_pc_create");
}

vg_ctx *ctx()
{
    std::call_once(g_once, create);
    return g_ctx;
}

vg_pc *pc()
{
    std::call_once(g_once, create);
    return g_pc;
}

void check(int rc, const char *what)
{
    if (rc != VG_OK) {
        fprintf(stderr, "virgo_b200: %s failed (%d): %s\n", what, rc, vg_last_error());
        abort();
    }
}

bool is_device_ptr(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}
}  // namespace virgo
