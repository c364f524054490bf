"""Proof server (continuous batching): every job's transcript is the same
alone and in the mix, bit for bit, whatever the admission order and the
memory budget."""
import pytest

import virgo_b200 as vb
from virgo_b200 import circuits

pytestmark = pytest.mark.gpu


def _mix():
    """circuits of different shapes and gate types, with their seeds"""
    return [
        (circuits.matmul_addtree(16, 16, seed=1), 1),
        (circuits.random_layered([10, 12, 11, 12, 9], seed=4), 5),
        (circuits.mixed_gates(seed=3), 7),
        (circuits.random_layered([14, 13, 15, 12, 14, 13], seed=9), 11),
        (circuits.matmul_addtree(8, 32, seed=2), 13),
        (circuits.random_layered([12, 16, 14], seed=21), 17),
    ]


def _alone(layers, seed):
    s = vb.Session(layers)
    try:
        return s.prove(seed)[1]
    finally:
        s.close()


def test_server_results_equal_alone():
    mix = _mix()
    want = [_alone(layers, seed) for layers, seed in mix]
    srv = vb.Server(slots=3)
    try:
        # twice over, so workers reload circuits of other shapes into used sessions
        jobs = [srv.submit(layers, seed) for layers, seed in mix + mix]
        got = [srv.wait(j) for j in jobs]
    finally:
        srv.close()
    for k, (info, data) in enumerate(got):
        assert info.status == 0
        assert info.latency_s >= info.run_s > 0
        assert data == want[k % len(mix)], ("job", k)


def test_server_small_budget_serialises_and_matches():
    """A budget that holds one job at a time: admission makes the workers
    take turns (idle workers give their memory back) and results still match."""
    mix = _mix()[:4]
    want = [_alone(layers, seed) for layers, seed in mix]
    budget = max(vb.job_footprint([len(t) for t, _, _ in layers]) for layers, _ in mix)
    srv = vb.Server(slots=4, hbm_budget=budget)
    try:
        jobs = [srv.submit(layers, seed, index_bytes=8) for layers, seed in mix]
        got = [srv.wait(j) for j in jobs]
    finally:
        srv.close()
    assert [d for _, d in got] == want


def test_server_reports_job_errors():
    bad = circuits.random_layered([10, 12, 11], seed=4)
    t, u, v = bad[2]
    u = u.copy()
    u[3] = 1 << 20   # wire beyond the previous layer
    bad[2] = (t, u, v)
    good = circuits.random_layered([10, 11], seed=5)
    srv = vb.Server(slots=2)
    try:
        jb = srv.submit(bad, 1)
        jg = srv.submit(good, 2)
        with pytest.raises(vb.VirgoError):
            srv.wait(jb)
        info, data = srv.wait(jg)
    finally:
        srv.close()
    assert info.status == 0 and data == _alone(good, 2)
