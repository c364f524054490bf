"""Kernel-level parity: every CUDA entry point against the C restatement on
the same seeded inputs, bit-exact (integer arithmetic)."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

import _oracle as O
import virgo_b200 as vb

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = vb.Context(0)
    yield c
    c.close()


def _ntt(ctx, inp, in_len, log_n, batch, root, scale=0):
    n = 1 << log_n
    src = ctx.buffer(np.ascontiguousarray(inp))
    dst = ctx.buffer(batch * n * 16)
    vb.check(vb.lib().vg_ntt(ctx.h, src.p, in_len, in_len, dst.p, log_n, n, batch, vb.to_fe(root), scale), "vg_ntt")
    out = dst.download(np.zeros((batch * n, 2), np.uint64))
    return out


@pytest.mark.parametrize("log_n,in_len,batch", [
    (0, 1, 1), (1, 2, 3), (2, 4, 2), (3, 8, 1), (4, 5, 2), (6, 64, 65), (8, 32, 4), (10, 1024, 2),
    (11, 64, 3), (12, 4096, 2), (13, 1000, 1), (16, 2048, 2), (17, 131072, 1), (20, 1 << 15, 1), (21, 1 << 21, 1),
])
def test_ntt_forward(ctx, log_n, in_len, batch):
    n = 1 << log_n
    co = O.fe_random(log_n * 100 + batch, batch * in_len)
    w = O.root_of_unity(log_n)
    got = _ntt(ctx, co, in_len, log_n, batch, w)
    for b in range(batch):
        exp = O.fft(co[b * in_len:(b + 1) * in_len], n, w)
        assert (got[b * n:(b + 1) * n] == exp).all(), (log_n, in_len, b)


@pytest.mark.parametrize("log_n,batch", [(1, 1), (5, 7), (9, 64), (14, 2), (18, 1)])
def test_ntt_inverse(ctx, log_n, batch):
    n = 1 << log_n
    ev = O.fe_random(log_n + 7, batch * n)
    w = O.root_of_unity(log_n)
    got = _ntt(ctx, ev, n, log_n, batch, O.inv(w), scale=1)
    for b in range(batch):
        assert (got[b * n:(b + 1) * n] == O.ifft(ev[b * n:(b + 1) * n], n, w)).all()


@pytest.mark.parametrize("kind", [0, 1])
def test_hash64(ctx, kind):
    vb.check(vb.lib().vg_ctx_set_hash(ctx.h, kind))
    rng = np.random.default_rng(kind)
    msgs = rng.integers(0, 256, (3000, 64), dtype=np.uint8)
    src, dst = ctx.buffer(msgs), ctx.buffer(3000 * 32)
    vb.check(vb.lib().vg_hash64(ctx.h, src.p, dst.p, 3000), "vg_hash64")
    got = dst.download(np.zeros((3000, 32), np.uint8))
    fn = hashlib.sha256 if kind else hashlib.sha3_256
    for m, d in zip(msgs[:200], got[:200]):
        assert d.tobytes() == fn(m.tobytes()).digest()
    assert (got == O.hash64(kind, msgs)).all()
    vb.check(vb.lib().vg_ctx_set_hash(ctx.h, 0))


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 1000, 4096, 70000])
def test_merkle_tree(ctx, kind, n):
    vb.check(vb.lib().vg_ctx_set_hash(ctx.h, kind))
    lv = np.random.default_rng(n).integers(0, 256, (n, 32), dtype=np.uint8)
    sz = 1
    while sz < n:
        sz *= 2
    src, dst = ctx.buffer(lv), ctx.buffer(2 * sz * 32)
    vb.check(vb.lib().vg_merkle_tree(ctx.h, src.p, n, dst.p), "vg_merkle_tree")
    got = dst.download(np.zeros((2 * sz, 32), np.uint8))
    assert (got[1:] == O.merkle_tree(kind, lv)[1:]).all()
    vb.check(vb.lib().vg_ctx_set_hash(ctx.h, 0))


@pytest.mark.parametrize("n_slices,n", [(1, 2), (65, 64), (65, 1 << 12), (3, 1 << 15)])
def test_leaf_chain(ctx, n_slices, n):
    cw = O.fe_random(n + n_slices, n_slices * n)
    src, dst = ctx.buffer(cw), ctx.buffer((n // 2) * 32)
    vb.check(vb.lib().vg_leaf_chain(ctx.h, src.p, n_slices, n, dst.p), "vg_leaf_chain")
    got = dst.download(np.zeros((n // 2, 32), np.uint8))
    assert (got == O.leaf_chain(0, cw, n_slices, n)).all()


def test_field_binop(ctx):
    edge = np.array([[0, 0], [O.P - 1, O.P - 1], [0, 1], [1, 0], [O.P - 1, 0], [0, O.P - 1], [5, O.P - 2]], np.uint64)
    a = np.concatenate([np.repeat(edge, len(edge), 0), O.fe_random(1, 5000)])
    b = np.concatenate([np.tile(edge, (len(edge), 1)), O.fe_random(2, 5000)])
    n = len(a)
    da, db, dc = ctx.buffer(a), ctx.buffer(b), ctx.buffer(n * 16)
    for op, name in [(0, "vo_fe_add_arr"), (1, "vo_fe_sub_arr"), (2, "vo_fe_mul_arr")]:
        vb.check(vb.lib().vg_fe_binop(ctx.h, op, da.p, db.p, dc.p, n))
        got = dc.download(np.zeros((n, 2), np.uint64))
        exp = np.zeros((n, 2), np.uint64)
        getattr(O.oracle(), name)(O.vp(a), O.vp(b), O.vp(exp), O.L(n))
        assert (got == exp).all(), name


def _pc(ctx):
    h = ctypes.c_void_p()
    vb.check(vb.lib().vg_pc_create(ctx.h, ctypes.byref(h)))
    return h


@pytest.mark.parametrize("log_len,n_mask", [(11, 40), (15, 300)])
def test_commitment_and_fri(ctx, log_len, n_mask):
    """commit_private / commit_public / FRI folding / query answers against the
    restatement: l_eval, h_eval, the virtual oracle (through the first fold),
    all_sum, every root and every query answer."""
    L = vb.lib()
    S = 1 << (log_len - 1)
    priv = O.fe_random(10 + log_len, 1 << log_len)
    pub = O.fe_random(20 + log_len, 1 << log_len)
    mask = O.fe_random(30 + log_len, n_mask)
    pc = _pc(ctx)
    try:
        M = ctypes.c_long()
        vb.check(L.vg_pc_encode_private(pc, vb.ptr(priv), log_len, vb.ptr(mask), n_mask, ctypes.byref(M)))
        l_exp, M_exp = O.commit_private(priv, log_len, mask)
        assert M.value == M_exp
        root_l = np.zeros(32, np.uint8)
        vb.check(L.vg_pc_init_commit(pc, 0, vb.ptr(root_l)))
        leaves = O.leaf_chain(0, l_exp, 65, S)
        assert (root_l == O.merkle_tree(0, leaves)[1]).all()

        pub_mask = O.fe_random(40 + log_len, M.value)
        sums = np.zeros((65, 2), np.uint64)
        inner = np.zeros(2, np.uint64)
        vb.check(L.vg_pc_encode_public(pc, vb.ptr(pub), vb.ptr(pub_mask), M.value, vb.ptr(sums), vb.ptr(inner)))
        q, h_exp, vo_exp, sums_exp = O.commit_public(l_exp, pub, log_len, pub_mask)
        assert (sums == sums_exp).all()
        root_h = np.zeros(32, np.uint8)
        vb.check(L.vg_pc_init_commit(pc, 1, vb.ptr(root_h)))
        assert (root_h == O.merkle_tree(0, O.leaf_chain(0, h_exp, 65, S))[1]).all()

        # FRI: fold the virtual oracle down to 32 entries per slice
        cw, n, t = vo_exp, S, 0
        rng = np.random.default_rng(log_len)
        while n > 32:
            r = np.array([rng.integers(0, O.P), rng.integers(0, O.P)], np.uint64)
            root = np.zeros(32, np.uint8)
            vb.check(L.vg_pc_fri_step(pc, vb.to_fe(r), vb.ptr(root)))
            w = O.root_of_unity((n).bit_length() - 1)
            cw = O.fri_fold(cw, 65, n, w, r)
            n //= 2
            assert (root == O.merkle_tree(0, O.leaf_chain(0, cw, 65, n))[1]).all(), ("level", t)
            t += 1
        data = np.zeros((n * 65, 2), np.uint64)
        msk = np.zeros((n, 2), np.uint64)
        nn = ctypes.c_long()
        vb.check(L.vg_pc_fri_final(pc, vb.ptr(data), vb.ptr(msk), ctypes.byref(nn)))
        assert nn.value == n
        for j in range(n // 2):
            for s in range(64):
                assert (data[(j << 7) | (s << 1)] == cw[s * n + j]).all()
                assert (data[(j << 7) | (s << 1) | 1] == cw[s * n + j + n // 2]).all()
            assert (msk[2 * j] == cw[64 * n + j]).all() and (msk[2 * j + 1] == cw[64 * n + j + n // 2]).all()

        # a query on the private oracle and on level 1
        vals = np.zeros((130, 2), np.uint64)
        path = np.zeros((log_len - 1, 32), np.uint8)
        p0 = S // 2 - 3
        vb.check(L.vg_pc_query_init(pc, p0, 0, vb.ptr(vals), vb.ptr(path)))
        for s in range(65):
            assert (vals[2 * s] == l_exp[s * S + p0]).all() and (vals[2 * s + 1] == l_exp[s * S + p0 + S // 2]).all()
        tree = O.merkle_tree(0, leaves)
        node = p0 + S // 2
        assert (path[log_len - 2] == tree[node]).all()
        for i in range(log_len - 2):
            assert (path[i] == tree[node ^ 1]).all()
            node //= 2
    finally:
        L.vg_pc_destroy(pc)


def _upload(ctx, layers):
    """raw prover-level circuit: layers[0] input values (u), others gates"""
    d = len(layers)
    bl = np.array([len(t).bit_length() - 1 for t, _, _ in layers], np.int32)
    keep = []
    tys, us, vs = (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)()
    for i, (t, u, v) in enumerate(layers):
        t, u, v = (np.ascontiguousarray(t, np.uint8), np.ascontiguousarray(u, np.int64), np.ascontiguousarray(v, np.int64))
        keep += [t, u, v]
        tys[i], us[i], vs[i] = t.ctypes.data, u.ctypes.data, v.ctypes.data
    h = ctypes.c_void_p()
    vb.check(vb.lib().vg_circuit_upload(ctx.h, d, vb.ptr(bl), tys, us, vs, ctypes.byref(h)), "vg_circuit_upload")
    return h


def _layers_values(layers):
    vals = [O.eval_input(layers[0][1])]
    for t, u, v in layers[1:]:
        vals.append(O.eval_layer(t, u, v, vals[-1]))
    return vals


def test_circuit_upload_rejects_bad_wires(ctx):
    layers = circuits_small()
    t, u, v = layers[1]
    u = u.copy()
    u[3] = 1 << 20   # out of range of the previous layer
    bad = [layers[0], (t, u, v)] + layers[2:]
    with pytest.raises(vb.VirgoError):
        _upload(ctx, bad)


def circuits_small():
    from virgo_b200 import circuits
    L = circuits.mixed_gates(11, log_width=6)
    return [L[0]] + L[1:]


@pytest.mark.parametrize("case", ["mixed", "random"])
def test_gkr_layer_pieces(ctx, case):
    """evaluate, V_res, phase-1/phase-2 scatter and every round's sums against
    the restatement, on all layers of a circuit with every gate type."""
    from virgo_b200 import circuits
    if case == "mixed":
        layers = circuits_small()
    else:
        layers = circuits.random_layered([9, 11, 10, 12, 8], seed=5)
    L = vb.lib()
    hc = _upload(ctx, layers)
    g = ctypes.c_void_p()
    vb.check(L.vg_gkr_create(ctx.h, hc, ctypes.byref(g)))
    try:
        vb.check(L.vg_gkr_evaluate(g))
        exp_vals = _layers_values(layers)
        for i, ev in enumerate(exp_vals):
            p = ctypes.c_void_p()
            vb.check(L.vg_gkr_layer_values(g, i, ctypes.byref(p)))
            got = np.zeros_like(ev)
            vb.check(L.vg_d2h(ctx.h, vb.ptr(got), p, got.nbytes))
            assert (got == ev).all(), ("layer", i)
        out_bl = len(exp_vals[-1]).bit_length() - 1
        r = O.fe_random(1, out_bl)
        vr = np.zeros(2, np.uint64)
        vb.check(L.vg_gkr_v_res(g, vb.ptr(r), out_bl, vb.ptr(vr)))
        assert (vr == O.v_res(exp_vals[-1], r)).all()

        rng = np.random.default_rng(7)
        rf = lambda k: O.fe_random(int(rng.integers(1 << 30)), k)  # noqa: E731
        for i in range(len(layers) - 1, 0, -1):
            t, u, v = layers[i]
            lg = len(t).bit_length() - 1
            lu = len(exp_vals[i - 1]).bit_length() - 1
            r0, r1, ab = rf(lg), rf(lg), rf(2)
            vb.check(L.vg_gkr_phase1_init(g, i, vb.ptr(r0), vb.ptr(r1), lg, vb.to_fe(ab[0]), vb.to_fe(ab[1])))
            bg = O.beta_g(lg, r0, r1, ab[0], ab[1])
            am, av = O.phase1_init(t, u, v, bg, exp_vals[i - 1])
            tabs = O.RoundTables(exp_vals[i - 1], av, am)
            ru = rf(lu)
            prev = np.zeros(2, np.uint64)
            last6 = np.zeros((6, 2), np.uint64)
            for j in range(lu):
                out3 = np.zeros((3, 2), np.uint64)
                vb.check(L.vg_gkr_round(g, vb.to_fe(prev), j, vb.ptr(out3), vb.ptr(last6)))
                assert (out3 == tabs.round(prev, j)).all(), ("phase1", i, j)
                prev = ru[j]
            # V_mult_add[0].eval(r) from the folded pair
            vu = rf(1)[0]
            vb.check(L.vg_gkr_phase2_init(g, vb.ptr(ru), lu, vb.to_fe(vu)))
            bu = O.beta_g(lu, ru, ru, np.array([0, 1], np.uint64), np.array([0, 0], np.uint64))
            am2, av2 = O.phase2_init(t, u, v, bg, bu, vu, len(exp_vals[i - 1]))
            tabs2 = O.RoundTables(exp_vals[i - 1], av2, am2)
            rv = rf(lu)
            prev = np.zeros(2, np.uint64)
            for j in range(lu):
                out3 = np.zeros((3, 2), np.uint64)
                vb.check(L.vg_gkr_round(g, vb.to_fe(prev), j, vb.ptr(out3), vb.ptr(last6)))
                assert (out3 == tabs2.round(prev, j)).all(), ("phase2", i, j)
                prev = rv[j]
    finally:
        L.vg_gkr_destroy(g)
        L.vg_circuit_destroy(hc)


def _mask_len(log_len, n_mask):
    S = 1 << (log_len - 1)
    gap = 1
    while gap * 2 <= S // n_mask:
        gap *= 2
    return S // gap


@pytest.mark.parametrize("log_len", [11, 20, 22, 24])
def test_commit_all_matches_step_api(ctx, log_len):
    """The kernel-level commit path at its full sizes (2^20, 2^22, 2^24): the
    one-call pipeline (fold-only FRI kernels, every leaf chain and tree in
    batched launches, one synchronisation) against the step API (the fused
    fold + leaf-chain kernel, per-set trees), which test_commitment_and_fri
    pins to the oracle: every root, all_sum, <l, q>, the final codeword and
    every query answer bit for bit."""
    L = vb.lib()
    n, S = 1 << log_len, 1 << (log_len - 1)
    nlevels = log_len - 6                      # fold until 32 entries per slice
    priv, pub = O.fe_random(50 + log_len, n), O.fe_random(60 + log_len, n)
    mask = O.fe_random(70 + log_len, 300)
    M = _mask_len(log_len, 300)
    pub_mask = O.fe_random(80 + log_len, M)
    fri_r = O.fe_random(90 + log_len, nlevels)
    rng = np.random.default_rng(log_len)
    which = np.array([0, 1] + [2 + t for t in range(nlevels)] * 2, np.int32)
    pos = np.array([rng.integers(0, S // 2) for _ in which], np.int64)
    nq = len(which)

    roots = np.zeros((2 + nlevels, 32), np.uint8)
    sums, inner = np.zeros((65, 2), np.uint64), np.zeros(2, np.uint64)
    fin = np.zeros((65 * 32, 2), np.uint64)
    qv, qp = np.zeros((nq * 130, 2), np.uint64), np.zeros((nq * 32, 32), np.uint8)
    pc = _pc(ctx)
    try:
        vb.check(L.vg_pc_commit_all(pc, vb.ptr(priv), log_len, vb.ptr(mask), 300, vb.ptr(pub), vb.ptr(pub_mask), M,
                                    vb.ptr(fri_r), nlevels, nq, vb.ptr(which), vb.ptr(pos), vb.ptr(roots), vb.ptr(sums),
                                    vb.ptr(inner), vb.ptr(fin), vb.ptr(qv), vb.ptr(qp)), "vg_pc_commit_all")
    finally:
        L.vg_pc_destroy(pc)

    pc = _pc(ctx)
    try:
        Mc = ctypes.c_long()
        vb.check(L.vg_pc_encode_private(pc, vb.ptr(priv), log_len, vb.ptr(mask), 300, ctypes.byref(Mc)))
        assert Mc.value == M
        r = np.zeros(32, np.uint8)
        vb.check(L.vg_pc_init_commit(pc, 0, vb.ptr(r)))
        assert (r == roots[0]).all()
        s2, i2 = np.zeros((65, 2), np.uint64), np.zeros(2, np.uint64)
        vb.check(L.vg_pc_encode_public(pc, vb.ptr(pub), vb.ptr(pub_mask), M, vb.ptr(s2), vb.ptr(i2)))
        assert (s2 == sums).all() and (i2 == inner).all()
        vb.check(L.vg_pc_init_commit(pc, 1, vb.ptr(r)))
        assert (r == roots[1]).all()
        for t in range(nlevels):
            vb.check(L.vg_pc_fri_step(pc, vb.to_fe(fri_r[t]), vb.ptr(r)))
            assert (r == roots[2 + t]).all(), ("level", t)
        data, msk, nn = np.zeros((32 * 65, 2), np.uint64), np.zeros((32, 2), np.uint64), ctypes.c_long()
        vb.check(L.vg_pc_fri_final(pc, vb.ptr(data), vb.ptr(msk), ctypes.byref(nn)))
        assert nn.value == 32
        for j in range(16):
            for s in range(64):
                assert (data[(j << 7) | (s << 1)] == fin[s * 32 + j]).all()
                assert (data[(j << 7) | (s << 1) | 1] == fin[s * 32 + j + 16]).all()
            assert (msk[2 * j] == fin[64 * 32 + j]).all() and (msk[2 * j + 1] == fin[64 * 32 + j + 16]).all()
        v2, p2 = np.zeros_like(qv), np.zeros_like(qp)
        plen = np.zeros(nq, np.int32)
        vb.check(L.vg_pc_query_batch(pc, nq, vb.ptr(which), vb.ptr(pos), vb.ptr(v2), vb.ptr(p2), vb.ptr(plen)))
        assert (v2 == qv).all()
        for q in range(nq):
            k = plen[q]
            assert (p2[q * 32:q * 32 + k] == qp[q * 32:q * 32 + k]).all(), ("query", q)
    finally:
        L.vg_pc_destroy(pc)


def _pred_inputs(seed, layers, which):
    lg = len(layers[which][0]).bit_length() - 1
    luv = len(layers[which - 1][0]).bit_length() - 1
    return [O.fe_random(seed + k, n) for k, n in enumerate([lg, lg, luv, luv, 1, 1])]


@pytest.mark.parametrize("case", ["mixed", "random", "sha4"])
def test_circuit_predicates(ctx, case):
    """vg_circuit_predicates (the verifier's wiring predicates as a reduction
    over the device circuit) on every layer against the restatement, and
    against the reference function itself where its shim was built; the
    4-block SHA-256 circuit has summation gates over wide ranges."""
    from virgo_b200 import circuits, sha256_circuit
    layers = {"mixed": circuits_small, "random": lambda: circuits.random_layered([9, 11, 10, 12, 8], seed=5),
              "sha4": lambda: sha256_circuit.sha256_blocks(4, seed=7)}[case]()
    hc = _upload(ctx, layers)
    try:
        for which in range(1, len(layers)):
            r0, r1, ru, rv, a, b = _pred_inputs(700 + 10 * which, layers, which)
            got = np.zeros((14, 2), np.uint64)
            vb.check(vb.lib().vg_circuit_predicates(ctx.h, hc, which, vb.ptr(r0), vb.ptr(r1), vb.ptr(ru), vb.ptr(rv),
                                                    vb.to_fe(a[0]), vb.to_fe(b[0]), vb.ptr(got)))
            if which == 1:
                assert not got.any()
                continue
            exp = O.predicates(layers, which, r0, r1, ru, rv, a, b)
            assert (got == exp).all(), (case, which)
            ref = O.ref_predicates(layers, which, r0, r1, ru, rv, a, b) if case != "sha4" else None
            assert ref is None or (got == ref).all(), (case, which)
    finally:
        vb.lib().vg_circuit_destroy(hc)


def _commit_ref_cases():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "commit_ref.json")
    with open(path) as f:
        return {c["log_len"]: c for c in json.load(f)}


@pytest.mark.parametrize("log_len", [11, 15, 20, 22])
def test_commit_all_matches_reference(ctx, log_len):
    """The kernel-level commit path (vg_pc_commit_all) against the reference
    itself run through its poly_commit API (commit_private_array,
    commit_public_array, commit_phase and the query answers of
    fri::request_init_value_with_merkle / request_step_commit), on the same
    seeded inputs and the reference's own FRI randomness, up to 2^22 inputs:
    every root, all_sum, the final codeword and every query answer with its
    authentication path, bit for bit (tests/golden/commit_ref.json)."""
    import hashlib
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_commit_golden as G
    case = _commit_ref_cases()[log_len]
    x = G.case_inputs(log_len)
    L = vb.lib()
    nlevels = x["nlevels"]
    fri_r = np.ascontiguousarray(np.frombuffer(bytes.fromhex(case["fri_r"]), np.uint64).reshape(-1, 2))
    which = np.array(case["which"], np.int32)
    pos = np.array(case["pos"], np.int64)
    nq = len(which)
    roots = np.zeros((2 + nlevels, 32), np.uint8)
    sums, inner = np.zeros((65, 2), np.uint64), np.zeros(2, np.uint64)
    fin = np.zeros((65 * case["final_n"], 2), np.uint64)
    qv, qp = np.zeros((nq * 130, 2), np.uint64), np.zeros((nq * 32, 32), np.uint8)
    pc = _pc(ctx)
    try:
        vb.check(L.vg_pc_commit_all(pc, vb.ptr(x["priv"]), log_len, vb.ptr(x["pri_mask"]), len(x["pri_mask"]),
                                    vb.ptr(x["pub"]), vb.ptr(x["pub_mask"]), x["n_pub_mask"], vb.ptr(fri_r), nlevels,
                                    nq, vb.ptr(which), vb.ptr(pos), vb.ptr(roots), vb.ptr(sums), vb.ptr(inner),
                                    vb.ptr(fin), vb.ptr(qv), vb.ptr(qp)), "vg_pc_commit_all")
    finally:
        L.vg_pc_destroy(pc)
    assert [r.tobytes().hex() for r in roots] == case["roots"]
    assert sums.tobytes().hex() == case["all_sum"]
    assert hashlib.sha256(fin.tobytes()).hexdigest() == case["final_slice_major"]
    for q in range(nq):
        k = case["queries"][q]["path_len"]
        path = [qp[q * 32 + i].tobytes() for i in range(k)]
        assert G.query_digest(qv[q * 130:(q + 1) * 130], path) == case["queries"][q]["digest"], ("query", q)
