"""Captured sumcheck phases: a session queues each phase's round launches and
issues them together after one copy of their challenges into device memory;
the second time the same sequence comes (the same phase of the same circuit
in a later proof, whatever the seed) it is captured as a CUDA graph, and
replayed from then on.  The transcripts stay equal to the reference's
golden ones while proofs of two circuits and two seeds interleave: first
sight (plain launches), capture and replays."""
import json
import os

import pytest

import virgo_b200 as vb
from virgo_b200 import circuits, transcript

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "transcripts.json")


def test_phase_graph_replays_match_golden():
    """matmul16_seed1 and matmul16_seed7 share the wiring and differ in their
    input values (and proof seed): one session proves both, switching the
    witness with set_inputs, between proofs of another circuit."""
    gold = {c["name"]: c for c in json.load(open(GOLD))}
    a1, a7, b = gold["matmul16_seed1"], gold["matmul16_seed7"], gold["random_3layer_pad15"]
    la1 = getattr(circuits, a1["generator"])(**a1["params"])
    la7 = getattr(circuits, a7["generator"])(**a7["params"])
    inputs = {a1["name"]: la1[0][1], a7["name"]: la7[0][1]}
    sa = vb.Session(la1)
    sb = vb.Session(getattr(circuits, b["generator"])(**b["params"]))
    replays = captures = 0
    try:
        for it in range(4):
            for s, c in ((sa, a1), (sb, b), (sa, a7)):
                if s is sa:
                    s.set_inputs(inputs[c["name"]])
                st, blob = s.prove(c["seed"])
                assert transcript.digest(transcript.parse(blob)) == c["digest"], (it, c["name"])
                if it == 0 and c is not a7:
                    assert st.graph_replays == 0   # nothing replayed on first sight
                replays += st.graph_replays
                captures += st.graph_captures
    finally:
        sa.close()
        sb.close()
    assert captures > 0 and replays > captures


def test_phase_graphs_follow_launch_shapes():
    """A launch-shape change gives other launch sequences: new graphs, the
    same transcript."""
    gold = {c["name"]: c for c in json.load(open(GOLD))}
    c = gold["random_5layer"]
    s = vb.Session(getattr(circuits, c["generator"])(**c["params"]))
    try:
        for shape in ({}, {"group_start": 1 << 11, "round_fuse": 1}, {}, {"round_threads": 128}):
            vb.tune_reset(0)
            if shape:
                vb.tune_set(0, **shape)
            for _ in range(3):
                _, blob = s.prove(c["seed"])
                assert transcript.digest(transcript.parse(blob)) == c["digest"], shape
    finally:
        vb.tune_reset(0)
        s.close()
