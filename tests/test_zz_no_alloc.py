"""vg_mle_eval_noalloc: the allocation-free entry point for callers that
cannot allocate device memory (their pool already holds the GPU, or they must
avoid cudaFree's device-wide synchronisation).  Checked through the C ABI
against vg_mle_eval, the entry point it mirrors, bit for bit, on two calls in
a row (the shared static scratch keeps the first call's contents), and
against the oracle.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import _oracle as O
import virgo_b200 as vb

pytestmark = pytest.mark.gpu


def test_noalloc_matches_mle_eval_twice():
    L = vb.lib()
    L.vg_mle_eval_noalloc.restype = ctypes.c_int
    L.vg_mle_eval_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    ctx = vb.Context(0)
    try:
        for log_n, seed in [(20, 1), (13, 2)]:
            n = 1 << log_n
            vals = O.fe_random(seed, n)
            r = O.fe_random(seed + 100, log_n)
            dv = ctx.buffer(vals)
            a = np.zeros(2, np.uint64)
            b = np.zeros(2, np.uint64)
            vb.check(L.vg_mle_eval(ctx.h, dv.p, n, vb.ptr(r), log_n, vb.ptr(a)), "vg_mle_eval")
            vb.check(L.vg_mle_eval_noalloc(dv.p, n, vb.ptr(r), log_n, vb.ptr(b)), "vg_mle_eval_noalloc")
            assert (a == b).all()                 # integer arithmetic: exact
            assert (b == O.v_res(vals, r)).all()
            dv.free()
        # beyond the fixed scratch: a clear error, nothing launched
        big = ctx.buffer(16)
        out = np.zeros(2, np.uint64)
        rr = O.fe_random(3, 27)
        rc = L.vg_mle_eval_noalloc(big.p, 1 << 27, vb.ptr(rr), 27, vb.ptr(out))
        assert rc == 2 and b"scratch" in L.vg_last_error()
        # sizes far beyond any shift width are rejected before anything is
        # computed from them
        for log_n in (64, 100, -1):
            rc = L.vg_mle_eval_noalloc(big.p, 16, vb.ptr(rr), log_n, vb.ptr(out))
            assert rc == 2 and b"scratch" in L.vg_last_error()
    finally:
        ctx.close()


def test_noalloc_after_library_stream_producer():
    """vals written by a kernel on a library context's (non-blocking) stream
    right before the call: the caller synchronises that stream, as the
    contract asks, and the result equals the oracle's."""
    L = vb.lib()
    L.vg_mle_eval_noalloc.restype = ctypes.c_int
    L.vg_mle_eval_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    ctx = vb.Context(0)
    try:
        log_n = 18
        n = 1 << log_n
        co = O.fe_random(7, 1 << 12)
        w = O.root_of_unity(log_n)
        src, dst = ctx.buffer(co), ctx.buffer(n * 16)
        r = O.fe_random(8, log_n)
        want = O.v_res(O.fft(co, n, w), r)
        for _ in range(2):
            vb.check(L.vg_ntt(ctx.h, src.p, 1 << 12, 1 << 12, dst.p, log_n, n, 1, vb.to_fe(w), 0), "vg_ntt")
            vb.check(L.vg_ctx_sync(ctx.h), "vg_ctx_sync")
            out = np.zeros(2, np.uint64)
            vb.check(L.vg_mle_eval_noalloc(dst.p, n, vb.ptr(r), log_n, vb.ptr(out)), "vg_mle_eval_noalloc")
            assert (out == want).all()
    finally:
        ctx.close()
