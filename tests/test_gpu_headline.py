"""The benchmarked path, pinned at the headline size.

bench.py times sessions in their deferred (launch pass + replay pass) mode: a
session on the 256x256 matmul circuit (2^24 product gates, 8 add layers,
32-bit entries) and fifteen forks of it, all proving at once, with paired
sumcheck rounds, the beta_g table, the launch shapes the autotuner picks, and
a new witness per proof through vg_session_set_inputs.  Here every prover
record of those proofs (sumcheck messages, commitment roots, all_sum, FRI
roots, final codeword, query answers) is compared with the reference
prover's own run on the same circuit, witness and seed: two witnesses (the
generator's entries and the bench's random 32-bit witness, which the
reference reads through its int truncation) times two seeds, under the
default shapes, the autotuner's choice and two hand-picked sets that move
every launch-shape parameter off its default."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import virgo_b200 as vb
from virgo_b200 import circuits, transcript

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

ALT_SHAPES = [
    dict(group_start=1 << 11, round_fuse=1, round_threads=128, ntt_max_log=8, ntt_tile_log=11, leaf_threads=128,
         leaf_warp_max=1 << 24, leaf_rot=1, beta_table=0, group_split=1),
    dict(group_start=1 << 22, round_fuse=2, round_threads=512, ntt_max_log=6, ntt_tile_log=13, leaf_threads=64,
         leaf_warp_max=0, leaf_rot=2, beta_table=1, group_split=0),
]


def _write_text(layers, cpath, mpath):
    L = vb.lib()
    d = len(layers)
    ns = np.array([len(t) for t, _, _ in layers], np.int64)
    tys, us, vs = (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)()
    keep = []
    for i, (t, u, v) in enumerate(layers):
        t, u, v = (np.ascontiguousarray(t, np.uint8), np.ascontiguousarray(u, np.int64),
                   np.ascontiguousarray(v, np.int64))
        keep.append((t, u, v))
        tys[i], us[i], vs[i] = t.ctypes.data, u.ctypes.data, v.ctypes.data
    vb.check(L.vg_circuit_write_text(d, ns.ctypes.data, tys, us, vs, cpath.encode(), mpath.encode()), "write text")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "zk_proof_ref")), reason="reference not compiled here")
def test_bench_session_path_matches_reference_matmul256(tmp_path):
    layers = circuits.matmul_addtree(256, 32, seed=1)
    u0 = np.ascontiguousarray(layers[0][1], np.int64)
    witnesses = {"gen": u0, "rand": np.random.default_rng(1234).integers(0, 1 << 32, len(u0), dtype=np.int64)}
    seeds = (11, 12)
    combos = [(w, s) for w in witnesses for s in seeds]

    # the reference prover on every (witness, seed), all at once on the host
    procs = {}
    for w, s in combos:
        d = tmp_path / ("%s_%d" % (w, s))
        d.mkdir()
        lay = [(layers[0][0], witnesses[w], layers[0][2])] + layers[1:]
        _write_text(lay, str(d / "c.txt"), str(d / "m.txt"))
        os.symlink(os.path.join(REF, "fft_gkr"), d / "fft_gkr")
        procs[(w, s)] = (subprocess.Popen([os.path.join(REF, "zk_proof_ref"), str(d / "c.txt"), str(d / "m.txt"),
                                           str(d / "res.txt"), str(s), str(d / "t.bin")], cwd=str(d),
                                          stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True), d)

    # the bench's session path while the reference runs
    base = vb.Session(layers)
    sessions = [base] + [base.fork() for _ in range(15)]
    got = {}
    try:
        vb.tune_reset(0)
        shapes = [("default", {})]
        chosen, _ = vb.autotune(sessions, seed=900, reps=1)
        shapes.append(("autotuned", chosen))
        shapes += [("alt%d" % k, a) for k, a in enumerate(ALT_SHAPES)]
        for name, shape in shapes:
            vb.tune_reset(0)
            if shape:
                vb.tune_set(0, **shape)
            for i, s in enumerate(sessions):
                s.set_inputs(witnesses[combos[i % 4][0]])
            res = vb.prove_batch(sessions, [combos[i % 4][1] for i in range(len(sessions))])
            for i, (st, blob) in enumerate(res):
                assert blob, (name, i)
                key = combos[i % 4]
                if key in got:
                    assert blob == got[key], ("proof differs between sessions or shapes", name, i, key)
                else:
                    got[key] = blob
    finally:
        vb.tune_reset(0)
        for s in sessions[1:]:
            s.close()
        base.close()

    for key, (p, d) in procs.items():
        out, err = p.communicate(timeout=900)
        assert p.returncode == 0 and "Pass" in out, (key, out[-1500:], err[-1500:])
        ref = transcript.prover_records(transcript.read(str(d / "t.bin")))
        mine = transcript.parse(got[key])
        assert len(mine) > 400
        assert transcript.first_difference(mine, ref) is None, key
