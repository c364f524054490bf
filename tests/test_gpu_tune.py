"""Launch-shape tuning: every value of every VG_TUNE_* parameter gives the
same results bit for bit (golden transcripts, oracle kernels), including the
one-warp-per-chain SHA3 leaf hashing and round groups that start on large
tables with CTAs looping over chunks; the autotuner keeps proofs unchanged."""
import ctypes
import json
import os

import numpy as np
import pytest

import _oracle as O
import virgo_b200 as vb
from virgo_b200 import circuits, transcript

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "transcripts.json")
# input padded to 2^17 (a 2^17-entry relay layer), a 2^15 input, 2^12 layers
CASES = ("matmul16_seed1", "random_3layer_pad15", "random_5layer")


@pytest.fixture(autouse=True)
def _defaults():
    vb.tune_reset(0)
    yield
    vb.tune_reset(0)


@pytest.fixture(scope="module")
def golden_sessions():
    gold = {c["name"]: c for c in json.load(open(GOLD))}
    out = []
    for name in CASES:
        c = gold[name]
        out.append((vb.Session(getattr(circuits, c["generator"])(**c["params"])), c))
    yield out
    for s, _ in out:
        s.close()


@pytest.mark.parametrize("knob,value", [
    ("group_start", 1 << 11), ("group_start", 1 << 13), ("group_start", 1 << 15), ("group_start", 1 << 19),
    ("group_start", 1 << 22), ("round_threads", 128), ("round_threads", 512), ("ntt_max_log", 6),
    ("ntt_max_log", 8), ("ntt_max_log", 9), ("ntt_tile_log", 10), ("ntt_tile_log", 11), ("ntt_tile_log", 13),
    ("leaf_threads", 64), ("leaf_threads", 128), ("leaf_warp_max", 1 << 24), ("leaf_rot", 0), ("leaf_rot", 1), ("leaf_rot", 2),
    ("beta_table", 0), ("group_split", 1), ("lazy_fold", 1), ("gather_fuse", 0),
])
def test_golden_transcripts_under_every_tuning(golden_sessions, knob, value):
    vb.tune_set(0, **{knob: value})
    assert vb.tune_get(0)[knob] == value
    for s, c in golden_sessions:
        _, blob = s.prove(c["seed"])
        assert transcript.digest(transcript.parse(blob)) == c["digest"], (c["name"], knob, value)


@pytest.mark.parametrize("fuse", [1, 2])
@pytest.mark.parametrize("group_start", [1 << 11, 1 << 13, 1 << 17])
def test_golden_transcripts_with_paired_rounds(golden_sessions, group_start, fuse):
    """Rounds above the group start one per launch or paired into two-round
    passes (the group start lowered so that the golden circuits have such
    rounds)."""
    vb.tune_set(0, group_start=group_start, round_fuse=fuse)
    for s, c in golden_sessions:
        _, blob = s.prove(c["seed"])
        assert transcript.digest(transcript.parse(blob)) == c["digest"], (c["name"], group_start)


def test_round_groups_loop_over_chunks_on_large_tables():
    """Tables of 2^20 entries with the group start at 2^20..2^22: groups of
    1024 chunks on at most 444 CTAs, each CTA folding several chunks."""
    layers = circuits.random_layered([20, 20, 19], seed=8)
    s = vb.Session(layers)
    try:
        base = s.prove(5)[1]
        for gs in (1 << 20, 1 << 21, 1 << 22):
            vb.tune_set(0, group_start=gs)
            assert s.prove(5)[1] == base, gs
        vb.tune_set(0, group_start=1 << 22, round_threads=512)
        assert s.prove(5)[1] == base
        vb.tune_set(0, group_start=1 << 11, round_threads=256)
        assert s.prove(5)[1] == base
        for gs, t, fuse in ((1 << 11, 128, 2), (1 << 13, 512, 2), (1 << 17, 256, 1), (1 << 11, 128, 1)):
            vb.tune_set(0, group_start=gs, round_threads=t, round_fuse=fuse)
            assert s.prove(5)[1] == base, (gs, t, fuse)
        vb.tune_set(0, beta_table=0)
        assert s.prove(5)[1] == base
        vb.tune_set(0, group_split=1, group_start=1 << 20)
        assert s.prove(5)[1] == base
    finally:
        s.close()


@pytest.fixture(scope="module")
def ctx():
    c = vb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("max_log,tile_log", [(6, 10), (8, 11), (9, 13), (10, 13), (7, 12)])
@pytest.mark.parametrize("log_n,batch", [(3, 2), (8, 3), (10, 1), (11, 2), (13, 1), (17, 1), (20, 1)])
def test_ntt_under_radix_and_tile(ctx, max_log, tile_log, log_n, batch):
    vb.tune_set(0, ntt_max_log=max_log, ntt_tile_log=tile_log)
    n = 1 << log_n
    co = O.fe_random(log_n * 31 + batch, batch * n)
    w = O.root_of_unity(log_n)
    src, dst = ctx.buffer(co), ctx.buffer(batch * n * 16)
    vb.check(vb.lib().vg_ntt(ctx.h, src.p, n, n, dst.p, log_n, n, batch, vb.to_fe(w), 0), "vg_ntt")
    got = dst.download(np.zeros((batch * n, 2), np.uint64))
    for b in range(batch):
        assert (got[b * n:(b + 1) * n] == O.fft(co[b * n:(b + 1) * n], n, w)).all(), (max_log, tile_log, log_n, b)


@pytest.mark.parametrize("mode", ["warp", "threads64", "threads128"])
@pytest.mark.parametrize("n_slices,n", [(1, 2), (65, 64), (65, 1 << 12), (3, 1 << 15)])
def test_leaf_chain_forms(ctx, mode, n_slices, n):
    if mode == "warp":
        vb.tune_set(0, leaf_warp_max=1 << 24)
    else:
        vb.tune_set(0, leaf_threads=int(mode[7:]))
    cw = O.fe_random(n + 3 * n_slices, n_slices * n)
    src, dst = ctx.buffer(cw), ctx.buffer((n // 2) * 32)
    vb.check(vb.lib().vg_leaf_chain(ctx.h, src.p, n_slices, n, dst.p), "vg_leaf_chain")
    got = dst.download(np.zeros((n // 2, 32), np.uint8))
    assert (got == O.leaf_chain(0, cw, n_slices, n)).all()


@pytest.mark.parametrize("rot,threads", [(1, 256), (2, 64), (2, 128)])
def test_multiply_pipe_rotations_in_batched_chains(rot, threads):
    """The SHA3 leaf chains with rho's rotations as multiplies: a proof's
    batched chains (every codeword set of the proof in one launch) give the
    golden transcript."""
    gold = {c["name"]: c for c in json.load(open(GOLD))}
    c = gold["random_5layer"]
    vb.tune_set(0, leaf_rot=rot, leaf_threads=threads)
    s = vb.Session(getattr(circuits, c["generator"])(**c["params"]))
    try:
        _, blob = s.prove(c["seed"])
    finally:
        s.close()
    assert transcript.digest(transcript.parse(blob)) == c["digest"]


def test_warp_leaf_chains_leave_sha256_per_thread(ctx):
    """The warp form is SHA3 only: with SHA-256 selected the same setting
    hashes per thread and still matches."""
    vb.tune_set(0, leaf_warp_max=1 << 24)
    vb.check(vb.lib().vg_ctx_set_hash(ctx.h, 1))
    try:
        n = 1 << 10
        cw = O.fe_random(77, 65 * n)
        src, dst = ctx.buffer(cw), ctx.buffer((n // 2) * 32)
        vb.check(vb.lib().vg_leaf_chain(ctx.h, src.p, 65, n, dst.p), "vg_leaf_chain")
        got = dst.download(np.zeros((n // 2, 32), np.uint8))
        assert (got == O.leaf_chain(1, cw, 65, n)).all()
    finally:
        vb.check(vb.lib().vg_ctx_set_hash(ctx.h, 0))


def test_autotune_keeps_proofs_and_picks_candidates(golden_sessions):
    s0, c = golden_sessions[2]
    forks = [s0.fork() for _ in range(2)]
    try:
        chosen, trials = vb.autotune([s0] + forks, seed=3, reps=1)
        assert len(trials) == 34   # every candidate of every key (autotune.cpp), the defaults included
        for name, v in chosen.items():
            assert any(t[0] == name and t[1] == v for t in trials) or v == vb.tune_get(0)[name]
            assert sum(1 for t in trials if t[0] == name and t[3]) == 1, name
        assert chosen == vb.tune_get(0)
        assert all(t[2] > 0 for t in trials)
        _, blob = s0.prove(c["seed"])
        assert transcript.digest(transcript.parse(blob)) == c["digest"]
        res = vb.prove_batch([s0] + forks, [c["seed"]] * 3)
        assert all(transcript.digest(transcript.parse(b)) == c["digest"] for _, b in res)
    finally:
        for f in forks:
            f.close()


def _family_launches(ctx, family):
    n, t, b = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
    vb.check(vb.lib().vg_ctx_profile_read(ctx, family, ctypes.byref(n), ctypes.byref(t), ctypes.byref(b)))
    return n.value


def test_table_builds_fused_into_first_paired_pass():
    """Tables above the group start (2^18, 2^19 entries): with the default
    shapes each phase's table build runs inside its first paired pass (the
    gather_round family of the per-launch profiler, 12 in common.cuh, counts
    those launches and the separate builds' families count none of them);
    with VG_TUNE_GATHER_FUSE = 0 the builds are launches of their own; the
    proofs are equal."""
    layers = circuits.random_layered([18, 19, 18, 17], seed=21)
    s = vb.Session(layers)
    try:
        base = s.prove(9)[1]
        cx = s.ctx()
        for fuse in (1, 0):
            vb.tune_set(0, gather_fuse=fuse)
            vb.check(vb.lib().vg_ctx_profile(cx, 1))
            blob = s.prove(9)[1]
            fused, builds = _family_launches(cx, 12), _family_launches(cx, 6) + _family_launches(cx, 7)
            vb.check(vb.lib().vg_ctx_profile(cx, 0))
            assert blob == base, fuse
            if fuse:
                assert fused >= 4, fused   # both phases of the layers over 2^18 and 2^19 entries
            else:
                assert fused == 0 and builds > 0
    finally:
        s.close()
