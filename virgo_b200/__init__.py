"""virgo_b200: B200-native Virgo prover hot path.

The product is the shared library lib/libvirgo_b200.so (CUDA kernels for
sm_100a behind the C ABI of include/virgo_b200.h, plus the drop-in C++ prover
classes).  This module binds the C ABI with ctypes for tests, benchmarks and
Python callers.  There is no CPU fallback: if the library or a CUDA device is
missing, every call raises.

Field elements are numpy uint64 arrays of shape (n, 2) holding (img, real),
the memory layout of the reference's prime_field::field_element.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

# Concurrent sessions run three streams each; CUDA's default of 8 hardware
# work queues per device makes streams beyond the eighth share a queue (and
# wait on each other's kernels).  Read when the process creates its CUDA
# context; a value set by the caller is kept.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libvirgo_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "virgo_b200.h")
P = (1 << 61) - 1

_lib = None


class VirgoError(RuntimeError):
    pass


class vg_fe(ctypes.Structure):
    _fields_ = [("img", ctypes.c_uint64), ("real", ctypes.c_uint64)]


class vg_proof_stats(ctypes.Structure):
    _fields_ = [
        ("launch_s", ctypes.c_double), ("wait_s", ctypes.c_double), ("replay_s", ctypes.c_double),
        ("total_s", ctypes.c_double), ("prove_time", ctypes.c_double), ("proof_size", ctypes.c_longlong), ("launches", ctypes.c_longlong),
        ("fft_gkr_s", ctypes.c_double), ("fft_gkr_lg", ctypes.c_int), ("fft_gkr_proof_size", ctypes.c_int),
        ("graph_replays", ctypes.c_int), ("graph_captures", ctypes.c_int),
    ]


class vg_fft_gkr_stats(ctypes.Structure):
    _fields_ = [("p_time", ctypes.c_double), ("v_time", ctypes.c_double), ("gpu_s", ctypes.c_double),
                ("proof_size", ctypes.c_int),
                ("pass_", ctypes.c_int), ("rounds", ctypes.c_int), ("launches", ctypes.c_longlong)]


class vg_job_info(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("queued_s", ctypes.c_double), ("run_s", ctypes.c_double),
                ("latency_s", ctypes.c_double), ("footprint", ctypes.c_size_t), ("stats", vg_proof_stats)]


class vg_tune_trial(ctypes.Structure):
    _fields_ = [("key", ctypes.c_int), ("value", ctypes.c_long), ("ms", ctypes.c_double), ("chosen", ctypes.c_int)]


# launch-shape parameters (VG_TUNE_* in include/virgo_b200.h)
TUNE_KEYS = {"group_start": 0, "round_threads": 1, "ntt_max_log": 2, "ntt_tile_log": 3, "leaf_threads": 4,
             "leaf_warp_max": 5, "round_fuse": 6,
             "leaf_rot": 7, "beta_table": 8,
             "group_split": 9, "lazy_fold": 10, "gather_fuse": 11}


def lib():
    """Loads the library (raises VirgoError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise VirgoError("libvirgo_b200.so not built: run `make -C virgo_b200` (or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        c_p, c_i, c_l, c_sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_size_t
        sig = {
            "vg_last_error": (ctypes.c_char_p, []),
            "vg_ctx_create": (c_i, [c_i, ctypes.POINTER(c_p)]),
            "vg_ctx_destroy": (c_i, [c_p]),
            "vg_ctx_set_hash": (c_i, [c_p, c_i]),
            "vg_ctx_sync": (c_i, [c_p]),
            "vg_ctx_launch_count": (c_i, [c_p, ctypes.POINTER(ctypes.c_longlong)]),
            "vg_dev_alloc": (c_i, [c_p, c_sz, ctypes.POINTER(c_p)]),
            "vg_dev_free": (c_i, [c_p, c_p]),
            "vg_h2d": (c_i, [c_p, c_p, c_p, c_sz]),
            "vg_d2h": (c_i, [c_p, c_p, c_p, c_sz]),
            "vg_fe_binop": (c_i, [c_p, c_i, c_p, c_p, c_p, c_l]),
            "vg_ntt": (c_i, [c_p, c_p, c_l, c_l, c_p, c_i, c_l, c_i, vg_fe, c_i]),
            "vg_hash64": (c_i, [c_p, c_p, c_p, c_l]),
            "vg_merkle_tree": (c_i, [c_p, c_p, c_l, c_p]),
            "vg_leaf_chain": (c_i, [c_p, c_p, c_i, c_l, c_p]),
            "vg_circuit_upload": (c_i, [c_p, c_i, c_p, c_p, c_p, c_p, ctypes.POINTER(c_p)]),
            "vg_circuit_destroy": (c_i, [c_p]),
            "vg_circuit_predicates": (c_i, [c_p, c_p, c_i, c_p, c_p, c_p, c_p, vg_fe, vg_fe, c_p]),
            "vg_fft_gkr_rounds": (c_i, [c_i]),
            "vg_fft_gkr_footprint": (c_sz, [c_i]),
            "vg_session_set_fft_gkr": (c_i, [c_p, c_i]),
            "vg_session_set_inputs": (c_i, [c_p, c_p, c_l]),
            "vg_fft_gkr_create": (c_i, [c_p, c_i, ctypes.POINTER(c_p)]),
            "vg_fft_gkr_prove": (c_i, [c_p, c_i, ctypes.c_uint, ctypes.POINTER(vg_fft_gkr_stats), c_p, c_p]),
            "vg_fft_gkr_destroy": (c_i, [c_p]),
            "vg_fft_gkr_run": (c_i, [c_p, c_i, ctypes.c_uint, ctypes.POINTER(vg_fft_gkr_stats), c_p, c_p]),
            "vg_gkr_create": (c_i, [c_p, c_p, ctypes.POINTER(c_p)]),
            "vg_gkr_destroy": (c_i, [c_p]),
            "vg_gkr_evaluate": (c_i, [c_p]),
            "vg_gkr_layer_values": (c_i, [c_p, c_i, ctypes.POINTER(c_p)]),
            "vg_gkr_v_res": (c_i, [c_p, c_p, c_i, c_p]),
            "vg_mle_eval": (c_i, [c_p, c_p, c_l, c_p, c_i, c_p]),
            "vg_gkr_phase1_init": (c_i, [c_p, c_i, c_p, c_p, c_i, vg_fe, vg_fe]),
            "vg_gkr_phase2_init": (c_i, [c_p, c_p, c_i, vg_fe]),
            "vg_gkr_round": (c_i, [c_p, vg_fe, c_i, c_p, c_p]),
            "vg_pc_create": (c_i, [c_p, ctypes.POINTER(c_p)]),
            "vg_pc_destroy": (c_i, [c_p]),
            "vg_pc_encode_private": (c_i, [c_p, c_p, c_i, c_p, c_l, ctypes.POINTER(c_l)]),
            "vg_pc_encode_public": (c_i, [c_p, c_p, c_p, c_l, c_p, c_p]),
            "vg_pc_init_commit": (c_i, [c_p, c_i, c_p]),
            "vg_eq_table": (c_i, [c_p, c_p, c_i, c_p]),
            "vg_pc_fri_step": (c_i, [c_p, vg_fe, c_p]),
            "vg_pc_fri_final": (c_i, [c_p, c_p, c_p, ctypes.POINTER(c_l)]),
            "vg_pc_query_init": (c_i, [c_p, c_l, c_i, c_p, c_p]),
            "vg_pc_query_step": (c_i, [c_p, c_i, c_l, c_p, c_p, ctypes.POINTER(c_i)]),
            "vg_pc_info": (c_i, [c_p, ctypes.POINTER(c_i), ctypes.POINTER(c_l), ctypes.POINTER(c_i)]),
            "vg_session_create": (c_i, [c_i, c_p, c_p, c_p, c_p, ctypes.POINTER(c_p)]),
            "vg_session_from_file": (c_i, [ctypes.c_char_p, ctypes.POINTER(c_p)]),
            "vg_session_destroy": (c_i, [c_p]),
            "vg_session_depth": (c_i, [c_p, ctypes.POINTER(c_i), ctypes.POINTER(c_i)]),
            "vg_session_write_proof": (c_i, [c_p, ctypes.c_char_p]),
            "vg_session_prove": (c_i, [c_p, ctypes.c_uint, c_i, ctypes.POINTER(vg_proof_stats),
                                       ctypes.POINTER(c_p), ctypes.POINTER(c_sz)]),
            "vg_session_fork": (c_i, [c_p, ctypes.POINTER(c_p)]),
            "vg_session_prove_batch": (c_i, [c_p, c_i, c_p, c_i, c_p, c_p, c_p]),
            "vg_session_new": (c_i, [ctypes.POINTER(c_p)]),
            "vg_session_commit_ctx": (c_i, [c_p, ctypes.POINTER(c_p)]),
            "vg_circuit_write_binary": (c_i, [ctypes.c_char_p, c_i, c_p, c_p, c_p, c_p, c_i]),
            "vg_circuit_is_binary": (c_i, [ctypes.c_char_p]),
            "vg_circuit_binary_info": (c_i, [ctypes.c_char_p, ctypes.POINTER(c_i), ctypes.POINTER(c_i), c_p, c_i]),
            "vg_session_load_file": (c_i, [c_p, ctypes.c_char_p]),
            "vg_pc_commit_all": (c_i, [c_p, c_p, c_i, c_p, c_l, c_p, c_p, c_l, c_p, c_i, c_i, c_p, c_p, c_p, c_p, c_p,
                                       c_p, c_p, c_p]),
            "vg_gkr_rebind": (c_i, [c_p, c_p]),
            "vg_job_footprint": (c_sz, [c_i, c_p]),
            "vg_server_create": (c_i, [c_i, c_i, c_sz, ctypes.POINTER(c_p)]),
            "vg_server_submit": (c_i, [c_p, c_i, c_p, c_p, c_p, c_p, c_i, ctypes.c_uint, c_i,
                                       ctypes.POINTER(ctypes.c_longlong)]),
            "vg_server_wait": (c_i, [c_p, ctypes.c_longlong, ctypes.POINTER(vg_job_info), ctypes.POINTER(c_p),
                                     ctypes.POINTER(c_sz)]),
            "vg_server_destroy": (c_i, [c_p]),
            "vg_session_ctx": (c_i, [c_p, ctypes.POINTER(c_p)]),
            "vg_pc_query_batch": (c_i, [c_p, c_i, c_p, c_p, c_p, c_p, c_p]),
            "vg_ctx_profile": (c_i, [c_p, c_i]),
            "vg_ctx_profile_trace": (c_i, [c_p, c_p, c_p, c_p, c_l, ctypes.POINTER(c_l)]),
            "vg_ctx_profile_read": (c_i, [c_p, c_i, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double)]),
            "vg_timer_start": (c_i, [c_p, ctypes.POINTER(c_p)]),
            "vg_timer_stop": (c_i, [c_p, c_p, ctypes.POINTER(ctypes.c_double)]),
            "vg_timer_stop_multi": (c_i, [c_p, c_i, c_p, ctypes.POINTER(ctypes.c_double)]),
            "vg_default_ctx": (c_i, [ctypes.POINTER(c_p)]),
            "vg_ctx_device": (c_i, [c_p, ctypes.POINTER(c_i)]),
            "vg_circuit_write_text": (c_i, [c_i, c_p, c_p, c_p, c_p, ctypes.c_char_p, ctypes.c_char_p]),
            "vg_mle_eval_noalloc": (c_i, [c_p, c_l, c_p, c_i, c_p]),
            "vg_session_load": (c_i, [c_p, c_i, c_p, c_p, c_p, c_p, c_i]),
            "vg_circuit_build": (c_i, [c_p, c_i, c_p, c_p, c_p, c_p, c_i, ctypes.POINTER(c_p), c_p]),
            "vg_free": (None, [c_p]),
            "vg_tune_get": (c_i, [c_i, c_i, ctypes.POINTER(c_l)]),
            "vg_tune_set": (c_i, [c_i, c_i, c_l]),
            "vg_tune_reset": (c_i, [c_i]),
            "vg_tune_range": (c_i, [c_i, ctypes.POINTER(c_l), ctypes.POINTER(c_l), ctypes.POINTER(c_l)]),
            "vg_autotune": (c_i, [c_p, c_i, ctypes.c_uint, c_i, ctypes.POINTER(vg_tune_trial), c_i,
                                  ctypes.POINTER(c_i)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = ""):
    if rc != 0:
        msg = lib().vg_last_error().decode(errors="replace")
        raise VirgoError("%s failed (%d): %s" % (what, rc, msg))


def fe_array(n: int) -> np.ndarray:
    return np.zeros((n, 2), dtype=np.uint64)


def to_fe(x) -> vg_fe:
    """(img, real) pair or numpy row -> vg_fe"""
    return vg_fe(int(x[0]), int(x[1]))


def ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


class DeviceBuffer:
    def __init__(self, ctx: "Context", nbytes: int):
        self.ctx = ctx
        self.nbytes = nbytes
        p = ctypes.c_void_p()
        check(lib().vg_dev_alloc(ctx.h, nbytes, ctypes.byref(p)), "vg_dev_alloc")
        self.p = p

    def upload(self, arr: np.ndarray):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        check(lib().vg_h2d(self.ctx.h, self.p, ptr(arr), arr.nbytes), "vg_h2d")

    def download(self, arr: np.ndarray):
        check(lib().vg_d2h(self.ctx.h, ptr(arr), self.p, arr.nbytes), "vg_d2h")
        return arr

    def free(self):
        if self.p:
            lib().vg_dev_free(self.ctx.h, self.p)
            self.p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """A device context (vg_ctx): one CUDA stream plus caches."""

    def __init__(self, device: int = 0, hash_kind: int = 0):
        h = ctypes.c_void_p()
        check(lib().vg_ctx_create(device, ctypes.byref(h)), "vg_ctx_create")
        self.h = h
        check(lib().vg_ctx_set_hash(h, hash_kind), "vg_ctx_set_hash")

    def close(self):
        if self.h:
            lib().vg_ctx_destroy(self.h)
            self.h = None

    def buffer(self, arr_or_nbytes) -> DeviceBuffer:
        if isinstance(arr_or_nbytes, np.ndarray):
            b = DeviceBuffer(self, max(16, arr_or_nbytes.nbytes))
            b.upload(arr_or_nbytes)
            return b
        return DeviceBuffer(self, max(16, int(arr_or_nbytes)))

    def sync(self):
        check(lib().vg_ctx_sync(self.h), "vg_ctx_sync")

    def launches(self) -> int:
        c = ctypes.c_longlong()
        check(lib().vg_ctx_launch_count(self.h, ctypes.byref(c)), "vg_ctx_launch_count")
        return c.value


class Session:
    """One circuit resident on the GPU (default context of the drop-in
    classes); prove() runs a whole proof for a seed."""

    def __init__(self, layers=None, circuit_path: str | None = None):
        h = ctypes.c_void_p()
        if circuit_path is not None:
            check(lib().vg_session_from_file(circuit_path.encode(), ctypes.byref(h)), "vg_session_from_file")
        else:
            d = len(layers)
            ns = np.array([len(t) for t, _, _ in layers], dtype=np.int64)
            self._keep = []
            tys = (ctypes.c_void_p * d)()
            us = (ctypes.c_void_p * d)()
            vs = (ctypes.c_void_p * d)()
            for i, (t, u, v) in enumerate(layers):
                t = np.ascontiguousarray(t, dtype=np.uint8)
                u = np.ascontiguousarray(u, dtype=np.int64)
                v = np.ascontiguousarray(v, dtype=np.int64)
                self._keep += [t, u, v]
                tys[i], us[i], vs[i] = t.ctypes.data, u.ctypes.data, v.ctypes.data
            self._keep.append(ns)
            check(lib().vg_session_create(d, ptr(ns), tys, us, vs, ctypes.byref(h)), "vg_session_create")
        self.h = h

    def depth(self):
        d, li = ctypes.c_int(), ctypes.c_int()
        check(lib().vg_session_depth(self.h, ctypes.byref(d), ctypes.byref(li)), "vg_session_depth")
        return d.value, li.value

    def prove(self, seed: int, transcript: bool = True):
        st = vg_proof_stats()
        buf = ctypes.c_void_p()
        n = ctypes.c_size_t()
        check(lib().vg_session_prove(self.h, seed, 1 if transcript else 0, ctypes.byref(st), ctypes.byref(buf),
                                     ctypes.byref(n)), "vg_session_prove")
        data = ctypes.string_at(buf, n.value) if (transcript and n.value) else b""
        lib().vg_free(buf)
        return st, data

    def set_inputs(self, values):
        """New witness for the loaded circuit: the u of its input gates
        (int64 array, host; pinned memory is copied without staging)."""
        if isinstance(values, np.ndarray):
            v = np.ascontiguousarray(values, dtype=np.int64)
            check(lib().vg_session_set_inputs(self.h, v.ctypes.data, len(v)), "vg_session_set_inputs")
        else:   # a pinned torch tensor
            check(lib().vg_session_set_inputs(self.h, values.data_ptr(), values.numel()), "vg_session_set_inputs")

    def write_proof(self, path: str):
        """The last proof as a file (vg_session_write_proof)."""
        check(lib().vg_session_write_proof(self.h, path.encode()), "vg_session_write_proof")

    def set_fft_gkr(self, on: bool):
        """Run the fft_gkr side proof beside every proof (default on)."""
        check(lib().vg_session_set_fft_gkr(self.h, 1 if on else 0), "vg_session_set_fft_gkr")

    def load(self, layers, index_bytes: int = 8):
        """Replaces the circuit (device buffers reused when it fits).  layers
        are (ty, u, v) arrays; with index_bytes=4 the wires of layers >= 1 are
        passed as uint32 (the input layer's u, its values, stay int64)."""
        ns, tys, us, vs, keep = _layer_arrays(layers, index_bytes)
        check(lib().vg_session_load(self.h, len(layers), ptr(ns), tys, us, vs, index_bytes), "vg_session_load")

    def fork(self) -> "Session":
        """A session on the same (shared) device circuit with its own stream."""
        h = ctypes.c_void_p()
        check(lib().vg_session_fork(self.h, ctypes.byref(h)), "vg_session_fork")
        s = Session.__new__(Session)
        s.h = h
        return s

    def ctx(self):
        c = ctypes.c_void_p()
        check(lib().vg_session_ctx(self.h, ctypes.byref(c)), "vg_session_ctx")
        return c

    def commit_ctx(self):
        """the context (second stream) of the commitment work"""
        c = ctypes.c_void_p()
        check(lib().vg_session_commit_ctx(self.h, ctypes.byref(c)), "vg_session_commit_ctx")
        return c

    def close(self):
        if self.h:
            lib().vg_session_destroy(self.h)
            self.h = None


def prove_batch(sessions, seeds, transcript: bool = True):
    """One proof per session, all at once (each session on its own stream)."""
    n = len(sessions)
    hs = (ctypes.c_void_p * n)(*[s.h.value for s in sessions])
    sd = (ctypes.c_uint * n)(*seeds)
    st = (vg_proof_stats * n)()
    bufs = (ctypes.c_void_p * n)()
    lens = (ctypes.c_size_t * n)()
    check(lib().vg_session_prove_batch(hs, n, sd, 1 if transcript else 0, st, bufs, lens), "vg_session_prove_batch")
    out = []
    for i in range(n):
        data = ctypes.string_at(bufs[i], lens[i]) if (transcript and lens[i]) else b""
        lib().vg_free(bufs[i])
        out.append((st[i], data))
    return out


def tune_get(device: int = 0) -> dict:
    """The device's launch-shape parameters by name."""
    out = {}
    for name, k in TUNE_KEYS.items():
        v = ctypes.c_long()
        check(lib().vg_tune_get(device, k, ctypes.byref(v)), "vg_tune_get")
        out[name] = v.value
    return out


def tune_set(device: int = 0, **values):
    for name, v in values.items():
        check(lib().vg_tune_set(device, TUNE_KEYS[name], int(v)), "vg_tune_set %s" % name)


def tune_reset(device: int = 0):
    check(lib().vg_tune_reset(device), "vg_tune_reset")


def autotune(sessions, seed: int = 1, reps: int = 2):
    """Runs vg_autotune over the sessions (all proving at once).  Returns the
    chosen parameters by name and every trial as (name, value, ms, chosen)."""
    n = len(sessions)
    hs = (ctypes.c_void_p * n)(*[s.h.value for s in sessions])
    cap = 64
    tr = (vg_tune_trial * cap)()
    nt = ctypes.c_int()
    check(lib().vg_autotune(hs, n, seed, reps, tr, cap, ctypes.byref(nt)), "vg_autotune")
    names = {k: name for name, k in TUNE_KEYS.items()}
    trials = [(names[tr[i].key], tr[i].value, tr[i].ms, bool(tr[i].chosen)) for i in range(nt.value)]
    dev = ctypes.c_int()
    ctx = ctypes.c_void_p()
    check(lib().vg_session_ctx(sessions[0].h, ctypes.byref(ctx)), "vg_session_ctx")
    check(lib().vg_ctx_device(ctx, ctypes.byref(dev)), "vg_ctx_device")
    return tune_get(dev.value), trials


def _layer_arrays(layers, index_bytes):
    """(n, ty*, u*, v*, keep) for the vg_session_load layout"""
    d = len(layers)
    ns = np.array([len(t) for t, _, _ in layers], dtype=np.int64)
    keep = [ns]
    tys, us, vs = (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)()
    for i, (t, u, v) in enumerate(layers):
        dt = np.int64 if (i == 0 or index_bytes == 8) else np.uint32
        t = t if isinstance(t, np.ndarray) and t.dtype == np.uint8 and t.flags.c_contiguous else np.ascontiguousarray(t, np.uint8)
        u = u if getattr(u, "dtype", None) == dt and u.flags.c_contiguous else np.ascontiguousarray(u, dt)
        v = v if getattr(v, "dtype", None) == dt and v.flags.c_contiguous else np.ascontiguousarray(v, dt)
        keep += [t, u, v]
        tys[i], us[i], vs[i] = t.ctypes.data, u.ctypes.data, v.ctypes.data
    keep += [tys, us, vs]
    return ns, tys, us, vs, keep


def write_circuit_binary(layers, path: str, index_bytes: int = 4):
    """Writes file-level layers (input layer first) as a binary circuit file."""
    ns, tys, us, vs, keep = _layer_arrays(layers, index_bytes)
    check(lib().vg_circuit_write_binary(path.encode(), len(layers), ns.ctypes.data, tys, us, vs, index_bytes),
          "vg_circuit_write_binary")


def circuit_binary_info(path: str):
    """(layer sizes, index_bytes) of a binary circuit file."""
    d, ib = ctypes.c_int(), ctypes.c_int()
    check(lib().vg_circuit_binary_info(path.encode(), ctypes.byref(d), ctypes.byref(ib), None, 0))
    n = np.zeros(d.value, np.int64)
    check(lib().vg_circuit_binary_info(path.encode(), ctypes.byref(d), ctypes.byref(ib), n.ctypes.data, d.value))
    return [int(x) for x in n], ib.value


class FftGkr:
    """The fft_gkr side prover on the GPU (vg_fft_gkr_*): the reference runs
    it as `fft_gkr <L-6> <file>` next to every proof of input size 2^L."""

    def __init__(self, ctx: Context, max_lg: int):
        self.ctx = ctx
        self.h = ctypes.c_void_p()
        check(lib().vg_fft_gkr_create(ctx.h, max_lg, ctypes.byref(self.h)), "vg_fft_gkr_create")

    def prove(self, lg: int, seed: int = 1, messages: bool = True):
        """-> (stats, messages (rounds, 3, 2) or None, phase values (2 + 2 lg, 2))"""
        st = vg_fft_gkr_stats()
        msgs = np.zeros((lib().vg_fft_gkr_rounds(lg), 3, 2), np.uint64) if messages else None
        vals = np.zeros((2 + 2 * lg, 2), np.uint64)
        check(lib().vg_fft_gkr_prove(self.h, lg, seed, ctypes.byref(st), ptr(msgs) if messages else None, ptr(vals)),
              "vg_fft_gkr_prove")
        return st, msgs, vals

    def close(self):
        if self.h:
            lib().vg_fft_gkr_destroy(self.h)
            self.h = None


def job_footprint(widths) -> int:
    """Device bytes a proof of a circuit with these file-layer widths needs."""
    ns = np.ascontiguousarray(widths, dtype=np.int64)
    return int(lib().vg_job_footprint(len(ns), ns.ctypes.data))


class Server:
    """Continuous-batching proof server on one GPU (vg_server_*): jobs are
    taken in arrival order by `slots` worker sessions as they free up and as
    their device footprint fits the HBM budget."""

    def __init__(self, slots: int = 8, device: int = 0, hbm_budget: int = 0):
        self.h = ctypes.c_void_p()
        check(lib().vg_server_create(device, slots, hbm_budget, ctypes.byref(self.h)), "vg_server_create")
        self._keep = {}

    def submit(self, layers, seed: int, transcript: bool = True, index_bytes: int = 4) -> int:
        ns, tys, us, vs, keep = _layer_arrays(layers, index_bytes)
        jid = ctypes.c_longlong()
        check(lib().vg_server_submit(self.h, len(layers), ns.ctypes.data, tys, us, vs, index_bytes, seed,
                                     1 if transcript else 0, ctypes.byref(jid)), "vg_server_submit")
        self._keep[jid.value] = keep   # the arrays must live until the job is done
        return jid.value

    def wait(self, job: int):
        info = vg_job_info()
        buf, n = ctypes.c_void_p(), ctypes.c_size_t()
        rc = lib().vg_server_wait(self.h, job, ctypes.byref(info), ctypes.byref(buf), ctypes.byref(n))
        data = ctypes.string_at(buf, n.value) if n.value else b""
        lib().vg_free(buf)
        self._keep.pop(job, None)
        check(rc, "vg_server_wait")
        return info, data

    def close(self):
        if self.h:
            lib().vg_server_destroy(self.h)
            self.h = None
            self._keep.clear()


def header_functions(path: str = HEADER) -> list:
    """Names of the functions declared in include/virgo_b200.h."""
    import re
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vg_[a-z0-9_]+)\s*\(", src)))
