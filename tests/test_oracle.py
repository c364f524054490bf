"""The C restatement (the oracle) pinned against the reference: known-answer
hashes from hashlib, golden vectors produced by the reference's own routines
(tests/golden/kernels.json), and, where the reference was compiled here, the
routines themselves.  CPU only."""
import hashlib
import json
import os

import numpy as np
import pytest

import _oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kernels():
    with open(os.path.join(GOLD, "kernels.json")) as f:
        return json.load(f)


def _same(arr, stored):
    if stored.startswith("sha256:"):
        return hashlib.sha256(arr.tobytes()).hexdigest() == stored[7:]
    return arr.tobytes().hex() == stored


@pytest.mark.parametrize("kind,fn", [(0, hashlib.sha3_256), (1, hashlib.sha256)])
def test_hash_known_answers(kind, fn):
    rng = np.random.default_rng(kind)
    msgs = rng.integers(0, 256, (50, 64), dtype=np.uint8)
    msgs[0] = 0
    msgs[1] = 255
    got = O.hash64(kind, msgs)
    for m, d in zip(msgs, got):
        assert d.tobytes() == fn(m.tobytes()).digest()


def test_hash_golden():
    for case in _kernels()["hash"]:
        m = np.random.default_rng(case["seed"]).integers(0, 256, 64, dtype=np.uint8)
        assert O.hash64(0, m)[0].tobytes().hex() == case["sha3_256"]


def test_fft_golden():
    for case in _kernels()["fft"]:
        co = O.fe_random(case["seed"], case["coef_len"])
        lo = case["order"].bit_length() - 1
        assert _same(O.fft(co, case["order"], O.root_of_unity(lo)), case["output"]), case["order"]


def test_ifft_golden():
    for case in _kernels()["ifft"]:
        ev = O.fe_random(case["seed"], case["order"])
        lo = case["order"].bit_length() - 1
        assert _same(O.ifft(ev, case["coef_len"], O.root_of_unity(lo)), case["output"]), case["order"]


def test_merkle_golden():
    for case in _kernels()["tree"]:
        lv = np.random.default_rng(case["seed"]).integers(0, 256, (case["n"], 32), dtype=np.uint8)
        t = O.merkle_tree(0, lv)
        assert t[1].tobytes().hex() == case["root"]
        assert _same(t[1:], case["tree"])


def test_fft_roundtrip_and_edges():
    # interpolation followed by evaluation returns the input (RS_polynomial.cpp:53,226,234 asserts)
    for lo in [1, 3, 8, 10]:
        ev = O.fe_random(lo, 1 << lo)
        w = O.root_of_unity(lo)
        co = O.ifft(ev, 1 << lo, w)
        assert (O.fft(co, 1 << lo, w) == ev).all()
    zero = np.zeros((16, 2), np.uint64)
    assert (O.fft(zero, 64, O.root_of_unity(6)) == 0).all()


def test_root_of_unity_orders():
    one = np.array([0, 1], np.uint64)
    for k in [1, 5, 17, 24]:
        w = O.root_of_unity(k)
        x = np.ascontiguousarray(w.reshape(1, 2))
        for _ in range(k):
            y = np.zeros((1, 2), np.uint64)
            O.oracle().vo_fe_mul_arr(O.vp(x), O.vp(x), O.vp(y), O.L(1))
            x = y
        assert (x[0] == one).all()


REFKERN = os.path.join(O.REF_DIR, "libvirgo_refkern.so")


@pytest.mark.skipif(not os.path.exists(REFKERN), reason="reference routines not compiled here")
def test_oracle_matches_reference_routines():
    import ctypes
    R = ctypes.CDLL(REFKERN)
    R.ref_init()
    rng_seed = 77
    for lo in range(0, 13):
        for lc in range(0, lo + 1):
            if lo == 2 and lc == 2:
                continue   # reference defect: its size-4 FFT returns stale scratch (RS_polynomial.cpp:125-146)
            co = O.fe_random(rng_seed, 1 << lc)
            rng_seed += 1
            out = np.zeros((1 << lo, 2), np.uint64)
            R.ref_fft(O.vp(co), 1 << lc, 1 << lo, lo, O.vp(out))
            assert (O.fft(co, 1 << lo, O.root_of_unity(lo)) == out).all(), (lc, lo)
            if lc != 2:   # the inverse uses a size-coef_len forward transform
                ev = O.fe_random(rng_seed, 1 << lo)
                rng_seed += 1
                ri = np.zeros((1 << lc, 2), np.uint64)
                R.ref_ifft(O.vp(ev), 1 << lc, 1 << lo, lo, O.vp(ri))
                assert (O.ifft(ev, 1 << lc, O.root_of_unity(lo)) == ri).all(), ("ifft", lc, lo)
    for n in [1, 2, 7, 33, 256]:
        lv = np.random.default_rng(n).integers(0, 256, (n, 32), dtype=np.uint8)
        sz = 1
        while sz < n:
            sz *= 2
        t = np.zeros((2 * sz, 32), np.uint8)
        R.ref_create_tree(O.vp(lv), n, O.vp(t))
        assert (O.merkle_tree(0, lv)[1:] == t[1:]).all()


def test_commit_restatement_consistency():
    """Properties the reference asserts inside commit_public_array
    (poly_commit.h:156-193): RS codes agree with the data at every 32nd point,
    the mask codes with the masks at every gap-th point, and all_sum adds up to
    the inner product."""
    log_len = 11
    S = 1 << (log_len - 1)
    priv = O.fe_random(1, 1 << log_len)
    pub = O.fe_random(2, 1 << log_len)
    mask = O.fe_random(3, 40)
    l_eval, M = O.commit_private(priv, log_len, mask)
    assert M == 64
    R = S >> 5
    for s in range(64):
        assert (l_eval[s * S:(s + 1) * S:32] == priv[s * R:(s + 1) * R]).all()
    gap = S // M
    pm = np.zeros((M, 2), np.uint64)
    pm[:40] = mask
    assert (l_eval[64 * S::gap] == pm).all()
    pub_mask = O.fe_random(4, M)
    q, h, vo, sums = O.commit_public(l_eval, pub, log_len, pub_mask)
    # inner product over the committed points equals the sum of all_sum
    def mul(a, b):
        c = np.zeros_like(a)
        O.oracle().vo_fe_mul_arr(O.vp(a), O.vp(b), O.vp(c), O.L(len(a)))
        return c
    def total(a):
        acc = np.zeros((1, 2), np.uint64)
        for row in a:
            x = np.ascontiguousarray(row.reshape(1, 2))
            O.oracle().vo_fe_add_arr(O.vp(acc), O.vp(x), O.vp(acc), O.L(1))
        return acc[0]
    ip = total(np.concatenate([mul(np.ascontiguousarray(priv), np.ascontiguousarray(pub)), mul(pm, pub_mask)]))
    assert (total(sums) == ip).all()


def _pred_case(case):
    from virgo_b200 import circuits, sha256_circuit
    gen = sha256_circuit.sha256_blocks if case["generator"] == "sha256_blocks" else getattr(circuits, case["generator"])
    return gen(**case["params"])


def _pred_inputs(case_idx, layers, which):
    """the seeding of tests/golden/make_golden.py:pred_inputs"""
    lg = len(layers[which][0]).bit_length() - 1
    luv = len(layers[which - 1][0]).bit_length() - 1
    base = 6000 + 100 * case_idx + 10 * which
    return [O.fe_random(base + k, n) for k, n in enumerate([lg, lg, luv, luv, 1, 1])]


def test_predicates_golden():
    """The restatement of zk_verifier::predicates against the reference's own
    outputs (every layer of three circuits; every gate type the builders make,
    summation and exp-sum ranges, relays)."""
    cases = _kernels()["predicates"]
    nonzero = set()
    for ci, case in enumerate(cases):
        layers = _pred_case(case)
        assert len(case["layers"]) == len(layers) - 1
        for which in range(1, len(layers)):
            got = (np.zeros((14, 2), np.uint64) if which == 1
                   else O.predicates(layers, which, *_pred_inputs(ci, layers, which)))
            nonzero |= {t for t in range(14) if got[t].any()}
            assert _same(got, case["layers"][which - 1]) or \
                hashlib.sha256(got.tobytes()).hexdigest() == case["layers"][which - 1], (case["name"], which)
    assert {0, 1, 5, 6, 7, 8, 9, 10, 12, 13} <= nonzero


@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "libvirgo_refverifier.so")),
                    reason="reference verifier shim not built")
def test_predicates_match_reference_live():
    """Fresh random circuits straight through the reference function."""
    from virgo_b200 import circuits
    for seed, layers in enumerate([circuits.random_layered([7, 9, 8, 10, 6], seed=21),
                                   circuits.mixed_gates(8, log_width=5)]):
        for which in range(2, len(layers)):
            ins = _pred_inputs(50 + seed, layers, which)
            assert (O.predicates(layers, which, *ins) == O.ref_predicates(layers, which, *ins)).all(), (seed, which)


def test_fft_gkr_golden():
    """The fft_gkr restatement against the reference side prover's recorded
    sumcheck messages and phase values (lg 1..12, the reference's own
    unseeded rand() stream), and its proof-size count."""
    for case in _kernels()["fft_gkr"]:
        ok, msgs, vals, ps = O.fft_gkr(case["lg"], case["seed"])
        assert ok, case["lg"]
        assert len(msgs) == case["rounds"] and ps == case["proof_size"]
        assert _same(msgs, case["msgs"]), case["lg"]
        assert msgs[:4].tobytes().hex() == case["first"]
        assert vals.tobytes().hex() == case["vals"], case["lg"]


def test_fft_gkr_other_seed():
    """Another seed of the rand() stream gives another passing run with
    different messages."""
    ok1, m1, _, _ = O.fft_gkr(6, 1)
    ok2, m2, _, _ = O.fft_gkr(6, 12345)
    assert ok1 and ok2 and not (m1 == m2).all()


def _commit_cases():
    path = os.path.join(GOLD, "commit_ref.json")
    return {c["log_len"]: c for c in json.load(open(path))} if os.path.exists(path) else {}


@pytest.mark.parametrize("log_len", [11, 15])
def test_commit_path_restatement_matches_reference(log_len):
    """The restatement's commit path (RS encodings, virtual oracle, FRI folds
    with the reference's own randomness, leaf chains, trees, query answers)
    against the reference run through its poly_commit API
    (tests/golden/commit_ref.json, oracle/commit_ref.cpp): every root,
    all_sum, the final codeword and every query answer."""
    import sys
    sys.path.insert(0, GOLD)
    import make_commit_golden as G
    case = _commit_cases()[log_len]
    x = G.case_inputs(log_len)
    S = 1 << (log_len - 1)
    l_exp, M = O.commit_private(x["priv"], log_len, x["pri_mask"])
    assert M == case["n_pub_mask"]
    tree_l = O.merkle_tree(0, O.leaf_chain(0, l_exp, 65, S))
    assert tree_l[1].tobytes().hex() == case["roots"][0]
    _, h_exp, vo, sums = O.commit_public(l_exp, x["pub"], log_len, x["pub_mask"])
    assert sums.tobytes().hex() == case["all_sum"]
    tree_h = O.merkle_tree(0, O.leaf_chain(0, h_exp, 65, S))
    assert tree_h[1].tobytes().hex() == case["roots"][1]
    fri_r = np.frombuffer(bytes.fromhex(case["fri_r"]), np.uint64).reshape(-1, 2)
    sets = [(l_exp, S, tree_l), (h_exp, S, tree_h)]
    cw, n = vo, S
    for t in range(len(fri_r)):
        cw = O.fri_fold(cw, 65, n, O.root_of_unity(n.bit_length() - 1), fri_r[t])
        n //= 2
        tree = O.merkle_tree(0, O.leaf_chain(0, cw, 65, n))
        assert tree[1].tobytes().hex() == case["roots"][2 + t], ("level", t)
        sets.append((cw, n, tree))
    assert n == case["final_n"]
    assert hashlib.sha256(cw.tobytes()).hexdigest() == case["final_slice_major"]
    for q, (which, pos) in enumerate(zip(case["which"], case["pos"])):
        src, n, tree = sets[which]
        p = pos % (n // 2)
        vals = np.array([src[s * n + p + b * (n // 2)] for s in range(65) for b in (0, 1)], np.uint64)
        node, path = p + n // 2, []
        while node != 1:
            path.append(tree[node ^ 1].tobytes())
            node //= 2
        path.append(tree[p + n // 2].tobytes())
        assert len(path) == case["queries"][q]["path_len"]
        assert G.query_digest(vals, path) == case["queries"][q]["digest"], ("query", q, which)
