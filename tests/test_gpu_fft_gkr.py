"""The fft_gkr side prover on the GPU against the reference's recorded
messages (tests/golden/kernels.json, lg 1..12), the restatement at larger
sizes and other seeds, and the reference binary itself where it was built;
every run must pass the reference's in-process checks."""
import json
import os
import subprocess

import numpy as np
import pytest

import _oracle as O
import virgo_b200 as vb

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kernels.json")


def _same(arr, stored):
    import hashlib
    if stored.startswith("sha256:"):
        return hashlib.sha256(arr.tobytes()).hexdigest() == stored[7:]
    return arr.tobytes().hex() == stored


@pytest.fixture(scope="module")
def prover():
    ctx = vb.Context(0)
    f = vb.FftGkr(ctx, 16)
    yield f
    f.close()
    ctx.close()


def test_fft_gkr_golden(prover):
    for case in json.load(open(GOLD))["fft_gkr"]:
        st, msgs, vals = prover.prove(case["lg"], case["seed"])
        assert st.pass_ == 1, case["lg"]
        assert st.rounds == case["rounds"] and st.proof_size == case["proof_size"]
        assert _same(msgs, case["msgs"]), case["lg"]
        assert vals.tobytes().hex() == case["vals"], case["lg"]
        assert st.launches > 0


@pytest.mark.parametrize("lg,seed", [(13, 1), (14, 1), (16, 1), (9, 12345), (11, 7)])
def test_fft_gkr_matches_restatement(prover, lg, seed):
    st, msgs, vals = prover.prove(lg, seed)
    ok, m, v, ps = O.fft_gkr(lg, seed)
    assert ok and st.pass_ == 1
    assert (msgs == m).all() and (vals == v).all()
    assert st.proof_size == ps


def test_fft_gkr_object_reuse_and_bounds(prover):
    """One object proves sizes in any order up to its maximum; the same size
    and seed give the same messages; sizes above the maximum are refused."""
    a = prover.prove(12)[1]
    prover.prove(3)
    b = prover.prove(12)[1]
    assert (a == b).all()
    with pytest.raises(vb.VirgoError):
        prover.prove(17)
    with pytest.raises(vb.VirgoError):
        prover.prove(0)


@pytest.mark.skipif(not os.path.exists(os.path.join(O.REF_DIR, "fft_gkr_rec")), reason="reference not built")
def test_fft_gkr_matches_reference_binary(prover, tmp_path):
    lg = 13
    rec, out = str(tmp_path / "r.rec"), str(tmp_path / "r.txt")
    subprocess.run([os.path.join(O.REF_DIR, "fft_gkr_rec"), str(lg), out, rec], check=True, cwd=str(tmp_path),
                   timeout=600)
    b = open(rec, "rb").read()
    q, i = [], 0
    while i < len(b):
        k = 4 if b[i:i + 1] == b"Q" else 3
        if k == 4:
            q.append(np.frombuffer(b[i + 1:i + 1 + 64], np.uint64).reshape(4, 2)[:3])
        i += 1 + 16 * k
    ref = np.array(q[0::3], np.uint64)
    st, msgs, _ = prover.prove(lg)
    assert (msgs == ref).all()
    assert st.proof_size == int(open(out).read().split()[1])


def test_fft_gkr_graph_replays_match_golden(prover):
    """A run repeating the previous one's size and seed is captured as a CUDA
    graph and later ones replay it: every run (plain, capture, replays, and
    after switching sizes and seeds in between) gives the recorded messages
    and passes the checks, with the same kernel count."""
    gold = {(c["lg"], c["seed"]): c for c in json.load(open(GOLD))["fft_gkr"]}
    a, b = gold[(8, next(s for l, s in gold if l == 8))], gold[(10, next(s for l, s in gold if l == 10))]
    launches = {}
    for case in (a, a, a, a, b, b, b, a, a, a, b):
        st, msgs, vals = prover.prove(case["lg"], case["seed"])
        assert st.pass_ == 1 and _same(msgs, case["msgs"]) and vals.tobytes().hex() == case["vals"], case["lg"]
        launches.setdefault(case["lg"], set()).add(st.launches)
        assert st.gpu_s > 0
    assert all(len(v) == 1 for v in launches.values()), launches
    # another seed at the same size: a new key, never the other key's graph
    for _ in range(3):
        st, msgs, vals = prover.prove(a["lg"], 777)
        ok, m, v, _ = O.fft_gkr(a["lg"], 777)
        assert ok and st.pass_ == 1 and (msgs == m).all() and (vals == v).all()
    st, msgs, _ = prover.prove(a["lg"], a["seed"])
    assert _same(msgs, a["msgs"])
