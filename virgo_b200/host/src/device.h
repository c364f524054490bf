// Process-wide default device context used by the drop-in classes, which,
// like the reference, have no context argument.
#pragma once
#include "virgo_b200.h"

namespace virgo
{
// The default context (created on first use on device $VIRGO_DEVICE, default
// 0).  Aborts with a message when no usable GPU or CUDA library is present:
// there is no CPU fallback.
vg_ctx *ctx();
// The default polynomial-commitment state shared by poly_commit:: and fri::.
vg_pc *pc();
// Aborts with the library's error message when rc != VG_OK.
void check(int rc, const char *what);
// True when p is device memory.
bool is_device_ptr(const void *p);
}  // namespace virgo
