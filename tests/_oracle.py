"""ctypes binding of the C restatement (oracle/virgo_oracle.c), the checker
the tests compare the CUDA path against.  Test infrastructure only."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "libvirgo_oracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
P = (1 << 61) - 1

_o = None


def oracle():
    global _o
    if _o is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", ORACLE_DIR, "restatement"], check=True, capture_output=True)
        _o = ctypes.CDLL(LIB)
        for name in ["vo_fft", "vo_ifft", "vo_merkle_tree", "vo_leaf_chain", "vo_fri_fold", "vo_rs_encode",
                     "vo_commit_private", "vo_commit_public", "vo_eval_input", "vo_eval_layer", "vo_v_res",
                     "vo_beta_g", "vo_phase1_init", "vo_phase2_init", "vo_hash64_batch", "vo_predicates"]:
            getattr(_o, name).restype = ctypes.c_long if name == "vo_commit_private" else None
    return _o


def vp(a):
    return ctypes.c_void_p(a.ctypes.data)


def L(x):
    return ctypes.c_long(int(x))


def fe_random(seed, n):
    rng = np.random.default_rng(seed)
    a = np.empty((n, 2), dtype=np.uint64)
    a[:, 0] = rng.integers(0, P, n, dtype=np.uint64)
    a[:, 1] = rng.integers(0, P, n, dtype=np.uint64)
    return a


def root_of_unity(log_order):
    r = np.zeros(2, np.uint64)
    oracle().vo_root_of_unity(log_order, vp(r))
    return r


def inv(x):
    x = np.ascontiguousarray(x, dtype=np.uint64)
    r = np.zeros(2, np.uint64)
    oracle().vo_fe_inv(vp(x), vp(r))
    return r


def fft(coef, order, root):
    out = np.zeros((order, 2), np.uint64)
    coef = np.ascontiguousarray(coef)
    oracle().vo_fft(vp(coef), L(len(coef)), L(order), vp(np.ascontiguousarray(root)), vp(out))
    return out


def ifft(evals, coef_len, root):
    out = np.zeros((coef_len, 2), np.uint64)
    evals = np.ascontiguousarray(evals)
    oracle().vo_ifft(vp(evals), L(coef_len), L(len(evals)), vp(np.ascontiguousarray(root)), vp(out))
    return out


def hash64(kind, msgs):
    msgs = np.ascontiguousarray(msgs, dtype=np.uint8)
    n = msgs.size // 64
    out = np.zeros((n, 32), np.uint8)
    oracle().vo_hash64_batch(kind, vp(msgs), vp(out), L(n))
    return out


def merkle_tree(kind, leaves):
    leaves = np.ascontiguousarray(leaves, dtype=np.uint8)
    n = len(leaves)
    sz = 1
    while sz < n:
        sz *= 2
    t = np.zeros((2 * sz, 32), np.uint8)
    oracle().vo_merkle_tree(kind, vp(leaves), L(n), vp(t))
    return t


def leaf_chain(kind, cw, n_slices, n):
    out = np.zeros((n // 2, 32), np.uint8)
    oracle().vo_leaf_chain(kind, vp(np.ascontiguousarray(cw)), n_slices, L(n), vp(out))
    return out


def fri_fold(cw, n_slices, n, w, r):
    out = np.zeros((n_slices * (n // 2), 2), np.uint64)
    oracle().vo_fri_fold(vp(np.ascontiguousarray(cw)), n_slices, L(n), vp(np.ascontiguousarray(w)),
                         vp(np.ascontiguousarray(r)), vp(out))
    return out


def commit_private(priv, log_len, mask):
    S = 1 << (log_len - 1)
    l_eval = np.zeros((65 * S, 2), np.uint64)
    m = oracle().vo_commit_private(vp(np.ascontiguousarray(priv)), log_len, vp(np.ascontiguousarray(mask)),
                                   L(len(mask)), vp(l_eval))
    return l_eval, m


def commit_public(l_eval, pub, log_len, pub_mask):
    S = 1 << (log_len - 1)
    q = np.zeros((65 * S, 2), np.uint64)
    h = np.zeros((65 * S, 2), np.uint64)
    vo = np.zeros((65 * S, 2), np.uint64)
    sums = np.zeros((65, 2), np.uint64)
    oracle().vo_commit_public(vp(l_eval), vp(np.ascontiguousarray(pub)), log_len, vp(np.ascontiguousarray(pub_mask)),
                              L(len(pub_mask)), vp(q), vp(h), vp(vo), vp(sums))
    return q, h, vo, sums


def eval_input(u):
    u = np.ascontiguousarray(u, dtype=np.int64)
    out = np.zeros((len(u), 2), np.uint64)
    oracle().vo_eval_input(vp(u), L(len(u)), vp(out))
    return out


def eval_layer(ty, u, v, prev):
    ty = np.ascontiguousarray(ty, dtype=np.uint8)
    u = np.ascontiguousarray(u, dtype=np.int64)
    v = np.ascontiguousarray(v, dtype=np.int64)
    out = np.zeros((len(ty), 2), np.uint64)
    oracle().vo_eval_layer(vp(ty), vp(u), vp(v), L(len(ty)), vp(np.ascontiguousarray(prev)), vp(out))
    return out


def v_res(vals, r):
    out = np.zeros(2, np.uint64)
    oracle().vo_v_res(vp(np.ascontiguousarray(vals)), len(r), vp(np.ascontiguousarray(r)), vp(out))
    return out


def beta_g(length_g, r0, r1, alpha, beta):
    out = np.zeros((1 << length_g, 2), np.uint64)
    oracle().vo_beta_g(length_g, vp(np.ascontiguousarray(r0)), vp(np.ascontiguousarray(r1)),
                       vp(np.ascontiguousarray(alpha)), vp(np.ascontiguousarray(beta)), vp(out))
    return out


def phase1_init(ty, u, v, bg, prev):
    n_uv = len(prev)
    am = np.zeros((n_uv, 2), np.uint64)
    av = np.zeros((n_uv, 2), np.uint64)
    oracle().vo_phase1_init(vp(np.ascontiguousarray(ty, dtype=np.uint8)), vp(np.ascontiguousarray(u, dtype=np.int64)),
                            vp(np.ascontiguousarray(v, dtype=np.int64)), L(len(ty)), vp(bg), vp(np.ascontiguousarray(prev)),
                            L(n_uv), vp(am), vp(av))
    return am, av


def phase2_init(ty, u, v, bg, bu, vu, n_uv):
    am = np.zeros((n_uv, 2), np.uint64)
    av = np.zeros((n_uv, 2), np.uint64)
    oracle().vo_phase2_init(vp(np.ascontiguousarray(ty, dtype=np.uint8)), vp(np.ascontiguousarray(u, dtype=np.int64)),
                            vp(np.ascontiguousarray(v, dtype=np.int64)), L(len(ty)), vp(bg), vp(bu),
                            vp(np.ascontiguousarray(vu)), L(n_uv), vp(am), vp(av))
    return am, av


def predicates(layers, which, r0, r1, ru, rv, alpha, beta):
    """the wiring predicates of layer `which` (>= 2) of prover-level layers"""
    t, u, v = layers[which]
    bl_g = len(t).bit_length() - 1
    bl_uv = len(layers[which - 1][0]).bit_length() - 1
    out = np.zeros((14, 2), np.uint64)
    oracle().vo_predicates(vp(np.ascontiguousarray(t, dtype=np.uint8)), vp(np.ascontiguousarray(u, dtype=np.int64)),
                           vp(np.ascontiguousarray(v, dtype=np.int64)), bl_g, bl_uv,
                           *[vp(np.ascontiguousarray(x)) for x in (r0, r1, ru, rv, alpha, beta)], vp(out))
    return out


def ref_predicates(layers, which, r0, r1, ru, rv, alpha, beta):
    """the same through the reference's own zk_verifier::predicates (the C
    shim oracle/_ref/libvirgo_refverifier.so); None when it is not built"""
    path = os.path.join(REF_DIR, "libvirgo_refverifier.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    d = len(layers)
    bl = np.array([len(t).bit_length() - 1 for t, _, _ in layers], np.int32)
    keep = [[np.ascontiguousarray(t, np.uint8), np.ascontiguousarray(u, np.int64), np.ascontiguousarray(v, np.int64)]
            for t, u, v in layers]
    ptrs = [(ctypes.c_void_p * d)(*[k[j].ctypes.data for k in keep]) for j in range(3)]
    out = np.zeros((14, 2), np.uint64)
    lib.ref_predicates(d, vp(bl), *ptrs, which, *[vp(np.ascontiguousarray(x)) for x in (r0, r1, ru, rv, alpha, beta)],
                       vp(out))
    return out


def fft_gkr(lg, seed=1):
    """the fft_gkr side prover restated: (pass, messages (rounds, 3, 2),
    final value of each phase, proof size)"""
    o = oracle()
    n = o.vo_fft_gkr_rounds(lg)
    msgs = np.zeros((n, 3, 2), np.uint64)
    vals = np.zeros((2 + 2 * lg, 2), np.uint64)
    ps = ctypes.c_int()
    ok = o.vo_fft_gkr(lg, ctypes.c_uint(seed), vp(msgs), vp(vals), ctypes.byref(ps))
    return bool(ok), msgs, vals, ps.value


class RoundTables:
    """The reference's linear-polynomial tables ({a, b} per entry) for the
    round-by-round oracle."""

    def __init__(self, V, AV, AM):
        n = len(V)
        self.n = n
        self.t = [np.zeros((n, 4), np.uint64) for _ in range(3)]
        for tab, vals in zip(self.t, (V, AV, AM)):
            tab[:, 2:] = vals   # .b = value, .a = 0

    def round(self, r, bit):
        out = np.zeros((3, 2), np.uint64)
        oracle().vo_sumcheck_round(vp(self.t[0]), vp(self.t[1]), vp(self.t[2]), L(self.n),
                                   vp(np.ascontiguousarray(r)), bit, vp(out))
        self.n //= 2
        return out
