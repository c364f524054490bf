#!/usr/bin/env python
"""Virgo prover benchmark: whole proofs of the 256 x 256 matrix-product circuit
(2^24 product gates, then 8 add-tree layers, seeded uniform 32-bit entries).

One step = one complete proof: layer evaluation, GKR sumcheck over every
layer, the polynomial commitment of the input (RS encoding, virtual oracle,
Merkle trees), the FRI commit phase, the answers to the verifier's 33 query
repetitions and the fft_gkr side proof (lg = 11) -- the prover side of the
reference's zk_proof run, all of what its Prove Time counts.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:       `value` = proofs/s with the circuit resident on the GPU (device
            time between CUDA events on the prover's stream, max over ranks);
            `e2e` = the same through the C ABI, wall clock: every proof takes
            a new witness from pinned host memory (vg_session_set_inputs) and
            downloads its transcript inside the step; `e2e_circuit` loads the
            whole circuit (vg_session_load, uint32 wires) for every proof.
reference:  the reference prover (compiled from its sources, oracle/_ref) on
            the host cores, one single-threaded proof per core, proofs/s from
            its own timers (Prove Time, which includes the fft_gkr side
            proof's prover time, plus evaluate).
Multi-GPU: replicas only (independent proofs per GPU, no collective on the
data path), launched by torchrun with one rank per GPU.
"""
from __future__ import annotations

import argparse
import ctypes
from concurrent.futures import ThreadPoolExecutor
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

# load every kernel when the CUDA context is created: with lazy loading (the
# CUDA 12 default) the first launch of a kernel in the timed region (e.g. a
# gate type or table shape seen for the first time by the server) loads its
# module mid-measurement
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")
# every session runs three streams (sumcheck, commitment, side proof): 32
# hardware work queues instead of CUDA's default 8, so that the streams of
# the proofs in flight do not share queues (the package sets the same default)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "matmul256_addtree_32bit"
METRIC = "proofs/s (256x256 matmul circuit, 2^24 product gates, full prover)"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "zk_proof_ref")
FFT_BIN = os.path.join(ROOT, "oracle", "_ref", "fft_gkr")
COMMIT_BIN = os.path.join(ROOT, "oracle", "_ref", "commit_ref")
FAMILIES = ["ntt_pass", "leaf_chain", "merkle_level", "fri_fold_leaf", "virtual_oracle", "eval_layer",
            "phase1_scatter", "phase2_scatter", "acc_finalize", "sumcheck_round", "reduce", "other", "gather_round"]
# DRAM bytes / algorithmic bytes measured by ncu on a full-size launch of
# the family's default kernel (profiles/k_round2_matmul256.txt: (403.0 +
# 173.3) MB read + written for 604 MB algorithmic on a 2^23-entry paired
# round)
TRAFFIC_RATIO = {"sumcheck_round": 0.954}
HBM_BOUND = {"ntt_pass", "virtual_oracle", "eval_layer", "phase1_scatter", "phase2_scatter", "acc_finalize",
             "sumcheck_round", "reduce", "gather_round"}


# Integer-ALU work of one proof of the matmul workload: warp instructions on
# the ALU pipe over every launch of a proof (ncu sm__inst_executed_pipe_alu
# per launch times launches per proof, profiles/alu_instructions_matmul256_proof.txt),
# a property of the code and the circuit, not of the run.  The pipe's peak is
# ncu's sm__inst_executed_pipe_alu.avg.peak_sustained, 2 warp instructions
# per SM cycle, on 148 SMs at the run's median SM clock.
ALU_WARP_INST_PER_PROOF = {"matmul256": 2.319e9}
# proofs the reference arm times per step (the step's sample)
REF_SAMPLE_PER_STEP = 8
ALU_PEAK_PER_SM_CYCLE = 2
NUM_SMS = 148


def alu_pipe(args, r):
    """The integer ALU pipe as the roofline of the whole step: the proofs'
    ALU instructions over the step's device time against the pipe's peak."""
    n = ALU_WARP_INST_PER_PROOF.get(args.workload)
    if not n:
        return None
    mhz = (r.get("clocks") or {}).get("sm_mhz") or 1965.0
    peak = ALU_PEAK_PER_SM_CYCLE * NUM_SMS * mhz * 1e6           # warp instructions / s
    floor_ms = 1e3 * n / peak                                      # one proof with the pipe always busy
    batch_ms = 1e3 * r["t_batch"] / (args.steps * args.batch)      # per proof, per GPU
    plain_ms = 1e3 * r["t_plain"] / args.steps
    return {"bound": "int_alu", "unit": "G warp instructions/s", "achieved": round(n / batch_ms / 1e6, 1),
            "peak": round(peak / 1e9, 1), "frac": round(floor_ms / batch_ms, 4),
            "plain_frac": round(floor_ms / plain_ms, 4), "alu_warp_inst_per_proof": n,
            "floor_ms_per_proof": round(floor_ms, 3), "max_batched_over_plain": round(plain_ms / floor_ms, 2),
            "source": "instructions per proof: a profile-derived constant (ncu counters, "
                      "profiles/alu_instructions_matmul256_proof.txt); times: this run's CUDA events; "
                      "peak: 2 warp instructions per SM cycle x 148 SMs x the run's median SM clock"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_workload(args):
    from virgo_b200 import circuits
    if args.workload == "matmul256":
        return circuits.matmul_addtree(256, 32, seed=1)
    if args.workload == "matmul16":
        return circuits.matmul_addtree(16, 16, seed=1)
    raise SystemExit("unknown workload " + args.workload)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Clocks and throttle reasons during a timed region: one background
    `nvidia-smi --query-gpu=... -lms 200` process for the whole region
    (started before it, stopped after it), parsed afterwards."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        self.out = tempfile.TemporaryFile(mode="w+")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)   # first sample before the region starts
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=10)
            except Exception:
                self.proc.kill()
                self.proc.wait()
        self.out.seek(0)
        for line in self.out.read().strip().splitlines():
            self.rows.append([x.strip() for x in line.split(",")])
        self.out.close()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------- reference arm
def ref_prover_seconds(workdir):
    err = open(os.path.join(workdir, "err.txt")).read()
    ev = float(re.search(r"total evaluation time: ([0-9.eE+-]+)", err).group(1))
    prove = float(re.search(r"^Prove Time ([0-9.eE+-]+)", err, re.M).group(1))
    gkr = float(re.search(r"GKR Prove Time ([0-9.eE+-]+)", err).group(1))
    fft = float(open(os.path.join(workdir, "log_fftgkr.txt")).read().split()[2])
    return ev + prove, {"evaluate_s": ev, "gkr_s": gkr, "prove_time_s": prove, "fft_gkr_s": fft}


def _ref_proof_dir():
    d = tempfile.mkdtemp(prefix="virgo_ref_")
    os.symlink(FFT_BIN, os.path.join(d, "fft_gkr"))   # the reference runs ./fft_gkr beside every proof
    return d


def _ref_launch(circuit, meta, seed):
    d = _ref_proof_dir()
    p = subprocess.Popen([REF_BIN, circuit, meta, os.path.join(d, "res.txt"), str(seed)], cwd=d,
                         stdout=open(os.path.join(d, "out.txt"), "w"), stderr=open(os.path.join(d, "err.txt"), "w"))
    return p, d


def run_reference_proofs(circuit, meta, count, seed0):
    """`count` concurrent single-threaded reference proofs; returns per-proof
    prover seconds and stage details."""
    procs = [_ref_launch(circuit, meta, seed0 + k) for k in range(count)]
    res = []
    for p, d in procs:
        p.wait()
        ok = "Pass" in open(os.path.join(d, "out.txt")).read()
        secs, detail = ref_prover_seconds(d)
        detail["verified"] = ok
        res.append((secs, detail))
        shutil.rmtree(d, ignore_errors=True)
    return res


def run_reference_pool(circuit, meta, n_warm, n_timed, width, seed0):
    """A pool of `width` concurrent single-threaded reference processes, one
    proof each: first n_warm warm-up proofs, then n_timed timed proofs; once
    every timed proof has started, filler proofs keep the pool full until the
    last timed proof ends (fillers are then stopped and not counted), so every
    timed proof runs beside width - 1 others.  Returns the timed proofs'
    (prover seconds, detail) and the wall-clock span from the first timed
    start to the last timed end."""
    pending = [("warm", seed0 + k) for k in range(n_warm)] + \
              [("timed", seed0 + n_warm + k) for k in range(n_timed)]
    running = []            # (kind, popen, dir, t_start)
    timed, t_first, t_last = [], None, None
    timed_left = n_timed
    filler_seed = seed0 + n_warm + n_timed
    fillers = 0
    while timed_left:
        while len(running) < width and (pending or timed_left):
            if pending:
                kind, seed = pending.pop(0)
            else:
                kind, seed = "filler", filler_seed
                filler_seed += 1
                fillers += 1
            p, d = _ref_launch(circuit, meta, seed)
            t0 = time.perf_counter()
            if kind == "timed" and t_first is None:
                t_first = t0
            running.append((kind, p, d, t0))
        time.sleep(0.02)
        still = []
        for kind, p, d, t0 in running:
            if p.poll() is None:
                still.append((kind, p, d, t0))
                continue
            if p.returncode != 0:
                raise RuntimeError("reference proof failed (rc %d) in %s" % (p.returncode, d))
            if kind == "timed":
                t_last = time.perf_counter()
                secs, detail = ref_prover_seconds(d)
                detail["verified"] = "Pass" in open(os.path.join(d, "out.txt")).read()
                timed.append((secs, detail))
                timed_left -= 1
            shutil.rmtree(d, ignore_errors=True)
        running = still
    for kind, p, d, t0 in running:   # warm-up stragglers and fillers: this process's own children
        p.kill()
        p.wait()
        shutil.rmtree(d, ignore_errors=True)
    return timed, t_last - t_first, fillers


def reference_sample(jobs):
    """Proves each (name, layers, seed) job with the reference prover, all
    jobs at once (one single-threaded process each); the circuit files are
    written by the library's text writer.  Returns (name, prover seconds,
    detail) per job, prover seconds from the reference's own timers (Prove
    Time, fft_gkr side proof included, plus evaluate)."""
    tmp = tempfile.mkdtemp(prefix="virgo_sample_")
    width = max(1, min(host_cores(), len(jobs)))
    try:
        files = []
        for k, (name, layers, seed) in enumerate(jobs):
            c, m = os.path.join(tmp, "c%d.txt" % k), os.path.join(tmp, "m%d.txt" % k)
            write_circuit_text(layers, c, m)
            files.append((name, c, m, seed))
        out, running = [], []
        while files or running:
            while files and len(running) < width:   # at most one process per core
                name, c, m, seed = files.pop(0)
                running.append((name, _ref_launch(c, m, seed)))
            time.sleep(0.02)
            still = []
            for name, (p, d) in running:
                if p.poll() is None:
                    still.append((name, (p, d)))
                    continue
                if p.returncode != 0:
                    raise RuntimeError("reference proof of %s failed (rc %d)" % (name, p.returncode))
                secs, detail = ref_prover_seconds(d)
                detail["verified"] = "Pass" in open(os.path.join(d, "out.txt")).read()
                out.append((name, secs, detail))
                shutil.rmtree(d, ignore_errors=True)
            running = still
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def cpu_baselines_batched_served(sample_random=8, seed_batch=4):
    """Bounded reference samples for the batched (64 random circuits) and
    served (job mix) workloads, all proved at once on the host cores:
    `sample_random` circuits drawn (seeded) from the 64 of the batch, and one
    job of each class of the served mix.  Throughput on all host cores is
    projected as cores / mean prover seconds (equal shares of the classes for
    the mix)."""
    from virgo_b200 import circuits, sha256_circuit
    cores = host_cores()
    batch = circuits.random_batch(64, seed_batch)
    pick = [int(i) for i in np.random.default_rng(17).choice(64, size=sample_random, replace=False)]
    jobs = [("random64[%d]" % i, batch[i], 100 + i) for i in pick]
    mix = [("random_2^14", circuits.random_by_gates(14, 16, seed=14000)),
           ("random_2^18", circuits.random_by_gates(18, 16, seed=18000)),
           ("random_2^22", circuits.random_by_gates(22, 16, seed=22000)),
           ("sha256_16_blocks", sha256_circuit.sha256_blocks(16, seed=41)),
           ("sha256_64_blocks", sha256_circuit.sha256_blocks(64, seed=61))]
    jobs += [(n, c, 500 + k) for k, (n, c) in enumerate(mix)]
    t0 = time.perf_counter()
    res = reference_sample(jobs)
    wall = time.perf_counter() - t0
    rnd = [(n, s) for n, s, _ in res if n.startswith("random64")]
    srv = [(n, s) for n, s, _ in res if not n.startswith("random64")]
    mean_r = statistics.mean(s for _, s in rnd)
    mean_s = statistics.mean(s for _, s in srv)
    common = {"unit": "proofs/s", "kind": "reference", "cores": cores,
              "note": "projected to all %d host cores as cores / mean prover seconds; the sample ran %d "
                      "single-threaded reference processes, at most one per core (%.1f s wall)"
                      % (cores, len(jobs), wall),
              "all_verified": all(d["verified"] for _, _, d in res)}
    return (dict(common, value=cores / mean_r, sample="%d of the 64 circuits (indices %s), prover seconds %s"
                 % (len(rnd), pick, [round(s, 3) for _, s in rnd])),
            dict(common, value=cores / mean_s, sample="one job of each class of the mix, prover seconds %s"
                 % {n: round(s, 3) for n, s in srv}))


def write_circuit_text(layers, circuit, meta):
    """The circuit in the reference text format through the library's writer
    (fast; used by this arm's cpu_baseline)."""
    import virgo_b200 as vb
    L = vb.lib()
    L.vg_circuit_write_text.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p]
    d = len(layers)
    ns = np.array([len(t) for t, _, _ in layers], np.int64)
    tys, us, vs = (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)()
    for i, (t, u, v) in enumerate(layers):
        tys[i], us[i], vs[i] = t.ctypes.data, u.ctypes.data, v.ctypes.data
    vb.check(L.vg_circuit_write_text(d, ns.ctypes.data, tys, us, vs, circuit.encode(), meta.encode()), "write text")


def bench_config(args, layers):
    """The workload description, identical on both arms."""
    return {"workload": WORKLOAD if args.workload == "matmul256" else args.workload,
            "circuit_gates": int(sum(len(t) for t, _, _ in layers)), "input_log2": 17 if args.workload == "matmul256" else None,
            "hash": "sha3-256", "proofs_per_step": args.batch,
            "l2": "inputs larger than L2 (circuit + tables > 1 GB per proof), no flush needed"}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def mem_available_gb():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 2 ** 20
    except Exception:
        pass
    return 64.0


def reference_arm(args, layers):
    """The reference prover (compiled from its own sources, unmodified apart
    from a main that seeds rand()) on the host cores: the same steps of
    `proofs_per_step` proofs as on the GPU arm, each timed on a bounded sample
    of at most REF_SAMPLE_PER_STEP of its proofs; W warm-up steps, then K
    timed steps, through a pool of single-threaded processes as wide as the
    cores (and memory) allow.  value = pool width x mean(1 / prover seconds) over
    the timed proofs, each timed by the reference's own timers (Prove Time,
    which includes the fft_gkr side proof, plus evaluate; zk_verifier.cpp
    :1244-1248); ms_per_step = wall-clock span of the timed proofs / K.  No
    library of this repository is loaded: the circuit file is written by the
    pure-numpy writer."""
    from virgo_b200 import circuits
    if not os.path.exists(REF_BIN):
        return {"impl": "reference", "unavailable": "reference prover not compiled (oracle/_ref missing)"}
    cores = host_cores()
    per_proof_gb = 4.5 if args.workload == "matmul256" else 1.0   # measured peak RSS 3.3 GB, plus margin
    width = max(1, min(cores, int(0.85 * mem_available_gb() // per_proof_gb)))
    tmp = tempfile.mkdtemp(prefix="virgo_circ_")
    circuit, meta = os.path.join(tmp, "c.txt"), os.path.join(tmp, "m.txt")
    circuits.write_text(layers, circuit, meta)
    # each step times a bounded sample of the step's proofs (at most
    # REF_SAMPLE_PER_STEP of them; a reference proof takes about 10 s of one
    # core), so that the K + W steps end within a few minutes
    per_step = min(args.batch, REF_SAMPLE_PER_STEP)
    try:
        timed, span, fillers = run_reference_pool(circuit, meta, args.warmup * per_step, args.steps * per_step,
                                                  width, seed0=1)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    secs = [x for x, _ in timed]
    value = width * statistics.mean(1.0 / x for x in secs)
    stage_means = {k: statistics.mean(d[k] for _, d in timed) for k in ("evaluate_s", "gkr_s", "prove_time_s", "fft_gkr_s")}
    return {
        "metric": METRIC, "value": value, "unit": "proofs/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * span / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64 (F_{p^2}, p = 2^61 - 1)", "data": "synthetic (seeded)",
        "config": bench_config(args, layers),
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": width, "kind": "reference",
                         "sample": "%d timed proofs of the workload (%d steps x %d of each step's %d proofs), %d "
                                   "single-threaded reference processes at a time on %d host cores, each proof "
                                   "timed by its own Prove Time (fft_gkr side proof included) plus evaluate"
                                   % (len(timed), args.steps, per_step, args.batch, width, cores)},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_pool": {"processes": width, "host_cores": cores, "proofs_timed": len(timed),
                           "proofs_warmup": args.warmup * per_step, "fillers_stopped": fillers,
                           "timed_span_s": round(span, 2),
                           "wall_proofs_s": round(len(timed) / span, 4),
                           "wall_note": "timed proofs / wall-clock span; each process also reads the circuit text "
                                        "and runs the verifier, which the prover timers exclude",
                           "all_verified": all(d["verified"] for _, d in timed),
                           "mean_stage_s": {k: round(v, 4) for k, v in stage_means.items()},
                           "build": "reference sources compiled unchanged with g++ -O3 -march=x86-64-v3 (its CMake "
                                    "uses -march=native; x86-64-v3 keeps AVX2/BMI2 and runs on any such host)"},
    }


# -------------------------------------------------------------------- ours
def session_arrays(layers, index_bytes=4):
    """pinned host copies of the layer arrays in the vg_session_load format:
    uint8 gate types, wires as uint32 (index_bytes=4) except the input
    layer's, whose u holds the int64 input values"""
    import torch
    pinned = []
    for i, (t, u, v) in enumerate(layers):
        dt = np.int64 if (i == 0 or index_bytes == 8) else np.uint32
        pt = torch.from_numpy(np.ascontiguousarray(t, np.uint8)).pin_memory()
        pu = torch.from_numpy(np.ascontiguousarray(u, dt).view(np.uint8)).pin_memory()
        pv = torch.from_numpy(np.ascontiguousarray(v, dt).view(np.uint8)).pin_memory()
        pinned.append((pt, pu, pv))
    return pinned


def load_from_pinned(session, pinned, index_bytes=4):
    """vg_session_load straight from pinned host buffers"""
    import virgo_b200 as vb
    d = len(pinned)
    ns = np.array([t.numel() for t, _, _ in pinned], np.int64)
    tys, us, vs = (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)()
    for i, (t, u, v) in enumerate(pinned):
        tys[i], us[i], vs[i] = t.data_ptr(), u.data_ptr(), v.data_ptr()
    vb.check(vb.lib().vg_session_load(session.h, d, ns.ctypes.data, tys, us, vs, index_bytes), "vg_session_load")


def local_device():
    return int(os.environ.get("VIRGO_DEVICE", "0"))


def ours(args, layers, rank, world):
    import virgo_b200 as vb
    L = vb.lib()
    base = vb.Session(layers)
    sessions = [base] + [base.fork() for _ in range(args.batch - 1)]
    from virgo_b200 import replicas
    seed0 = replicas.rank_seed_base(rank)

    def ctx_of(s):
        return s.ctx()

    # warm-up: every session proves once per warm-up step
    for w in range(args.warmup):
        vb.prove_batch(sessions, [seed0 + w * args.batch + i for i in range(args.batch)])

    # launch shapes: the autotuner times whole batches of the sessions under
    # each candidate (before any timed region; proofs are bit-identical under
    # every choice)
    tune = None
    if not args.no_autotune:
        defaults = vb.tune_get(local_device())
        chosen, trials = vb.autotune(sessions, seed=seed0 + 900, reps=3)
        tune = {"objective": "wall time of %d proofs in flight (best of 3 after 1 warm-up per candidate)"
                             % len(sessions),
                "defaults": defaults, "chosen": chosen,
                "trials": [[k, v, round(ms, 2), c] for k, v, ms, c in trials]}

    # ---- plain: one proof at a time on one stream (device time by CUDA events) ----
    barrier(world)
    timer = ctypes.c_void_p()
    ctx0 = ctx_of(base)
    stages = {"launch_s": 0.0, "wait_s": 0.0, "replay_s": 0.0, "fft_gkr_s": 0.0}
    vb.check(L.vg_timer_start(ctx0, ctypes.byref(timer)))
    for k in range(args.steps):
        st, _ = base.prove(seed0 + 100 + k, transcript=True)
        for key in stages:
            stages[key] += getattr(st, key)
    ms = ctypes.c_double()
    vb.check(L.vg_timer_stop(ctx0, timer, ctypes.byref(ms)))
    t_plain = max_over_ranks(ms.value / 1000.0, world)

    # ---- batched: each step proves `batch` proofs at once (one stream and one
    # host thread each; every thread takes its own transcript as soon as its
    # proof is done, so no host copy runs while the GPU waits) ----
    barrier(world)
    ctxs = (ctypes.c_void_p * len(sessions))(*[ctx_of(s).value for s in sessions])
    bpool = ThreadPoolExecutor(len(sessions))

    def prove_one(i, seed):
        return sessions[i].prove(seed, transcript=True)

    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        for s in sessions:
            vb.check(L.vg_ctx_sync(ctx_of(s)))
        timer = ctypes.c_void_p()
        vb.check(L.vg_timer_start(ctx0, ctypes.byref(timer)))
        n_launch = 0
        for k in range(args.steps):
            res = list(bpool.map(prove_one, range(len(sessions)),
                                 [seed0 + 300 + k * args.batch + i for i in range(args.batch)]))
            n_launch += sum(st.launches for st, _ in res)   # all three streams of every session
        ms = ctypes.c_double()
        vb.check(L.vg_timer_stop_multi(ctxs, len(sessions), timer, ctypes.byref(ms)))   # latest stream end
        t_batch = ms.value / 1000.0
    bpool.shutdown()
    t_batch = max_over_ranks(t_batch, world)

    # ---- per-kernel profile (separate pass, one stream, events around every launch) ----
    pctxs = (ctx0, base.commit_ctx())   # sumcheck stream and commitment stream
    for cx in pctxs:
        vb.check(L.vg_ctx_profile(cx, 1))
    for k in range(args.steps):
        base.prove(seed0 + 500 + k, transcript=False)
    fam = {}
    for i, name in enumerate(FAMILIES):
        tot_n, tot_t, tot_b = 0, 0.0, 0.0
        for cx in pctxs:
            n, t, b = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
            vb.check(L.vg_ctx_profile_read(cx, i, ctypes.byref(n), ctypes.byref(t), ctypes.byref(b)))
            tot_n, tot_t, tot_b = tot_n + n.value, tot_t + t.value, tot_b + b.value
        if tot_n:
            fam[name] = {"launches": tot_n / args.steps, "ms": tot_t / args.steps, "bytes": tot_b / args.steps}
    # the sumcheck stream's launches one by one: round launches that move at
    # least 100 MB (tables of 2^21 entries and up) against the rest
    cap = 20000
    tf, tm, tb = (ctypes.c_int * cap)(), (ctypes.c_double * cap)(), (ctypes.c_double * cap)()
    nt = ctypes.c_long()
    vb.check(L.vg_ctx_profile_trace(ctx0, tf, tm, tb, cap, ctypes.byref(nt)))
    rounds = [(tm[i], tb[i]) for i in range(min(nt.value, cap)) if tf[i] == FAMILIES.index("sumcheck_round")]
    big = [x for x in rounds if x[1] >= 100e6]
    large_rounds = {"launches_per_proof": len(big) / args.steps,
                    "ms": sum(t for t, _ in big) / args.steps, "bytes": sum(b for _, b in big) / args.steps} if big else None
    for cx in pctxs:
        vb.check(L.vg_ctx_profile(cx, 0))
    for s in sessions[1:]:
        s.close()

    # ---- e2e: every step, each of the `batch` sessions takes a new witness
    # (the input layer's values, int64, from pinned host memory; the wiring
    # stays on the device), proves and downloads its transcript: host ->
    # device -> host through the C ABI.  e2e_circuit: the same with the whole
    # circuit loaded from pinned host buffers (built and validated on the GPU)
    # for every proof ----
    import torch
    u0 = np.ascontiguousarray(layers[0][1], np.int64)
    rng = np.random.default_rng(1234)
    witnesses = [torch.from_numpy(u0.copy()).pin_memory(),
                 torch.from_numpy(rng.integers(0, 1 << 32, len(u0), dtype=np.int64)).pin_memory()]
    pinned = session_arrays(layers, 4)
    h2d_circuit = int(sum(t.numel() + u.numel() + v.numel() for t, u, v in pinned))
    sessions = [base] + [base.fork() for _ in range(args.batch - 1)]
    pool = ThreadPoolExecutor(len(sessions))

    def one(i, seed, full):
        if full:
            load_from_pinned(sessions[i], pinned, 4)
        else:
            sessions[i].set_inputs(witnesses[(seed + i) % 2])
        return len(sessions[i].prove(seed, transcript=True)[1])

    def e2e_run(full):
        def step(seed):
            return sum(pool.map(one, range(len(sessions)), [seed + i for i in range(len(sessions))],
                                [full] * len(sessions)))
        for w in range(args.warmup):
            step(seed0 + 700 + w * args.batch)
        barrier(world)
        d2h = 0
        t0 = time.perf_counter()
        for k in range(args.steps):
            d2h = step(seed0 + 200 + k * args.batch)
        return max_over_ranks(time.perf_counter() - t0, world), d2h

    # the clock sampler runs here too, so that both timed regions see the
    # same background NVML queries
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks_e2e:
        t_e2e, d2h = e2e_run(False)
    t_e2e_circuit, _ = e2e_run(True)
    pool.shutdown()
    for s in sessions[1:]:
        s.close()
    base.close()
    return {"t_plain": t_plain, "t_batch": t_batch, "t_e2e": t_e2e, "t_e2e_circuit": t_e2e_circuit,
            "clocks": clocks.summary(), "clocks_e2e": clocks_e2e.summary(), "families": fam, "launches": n_launch, "large_rounds": large_rounds,
            "stages": {k: v / args.steps for k, v in stages.items()}, "autotune": tune,
            "h2d": int(u0.nbytes) * args.batch, "h2d_circuit": h2d_circuit * args.batch, "d2h": d2h}


# ------------------------------------------------- batched and served forms
_PINNED = []


def _pinned_layers(layers):
    """numpy views of pinned copies in the vg_session_load layout (uint32
    wires above the input layer)"""
    import torch
    out = []
    for i, (t, u, v) in enumerate(layers):
        dt = np.int64 if i == 0 else np.uint32
        arrs = []
        for a, d in ((t, np.uint8), (u, dt), (v, dt)):
            pt = torch.from_numpy(np.ascontiguousarray(a, d)).pin_memory()
            _PINNED.append(pt)   # the numpy view below does not own the pinned storage
            arrs.append(pt.numpy())
        out.append(tuple(arrs))
    return out


def _pctl(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q * (len(xs) - 1)))))
    return xs[k]


def batched_random(count, seed, slots):
    """Random layered circuits (per circuit a depth in 8..32, per layer a width
    2^12..2^20, add/mult p = 0.5) proved through the server all at once, and
    the same circuits proved one after another on one session (the plain
    form).  Both are wall clock and include the circuit upload."""
    import virgo_b200 as vb
    from virgo_b200 import circuits
    batch = circuits.random_batch(count, seed)
    gates = int(sum(circuits.total_gates(c) for c in batch))
    # the client holds each circuit in pinned host memory, wires as uint32
    prepared = [_pinned_layers(c) for c in batch]
    # steady state: each form proves the whole batch once untimed (its buffers
    # reach their working size), then twice timed (the mean of the two passes)
    s = vb.Session(batch[0])
    t_plain = 0.0
    try:
        for rep in range(3):
            t0 = time.perf_counter()
            for k, c in enumerate(prepared):
                s.load(c, index_bytes=4)
                s.prove(100 + k, transcript=rep > 0)
            if rep:
                t_plain += (time.perf_counter() - t0) / 2
    finally:
        s.close()
    srv = vb.Server(slots=slots)
    t_batch = 0.0
    try:
        for rep in range(3):
            t0 = time.perf_counter()
            jobs = [srv.submit(c, 100 + k, transcript=rep > 0) for k, c in enumerate(prepared)]
            for j in jobs:
                srv.wait(j)
            if rep:
                t_batch += (time.perf_counter() - t0) / 2
    finally:
        srv.close()
    return {"value": count / t_batch, "unit": "proofs/s", "plain_value": count / t_plain,
            "speedup_vs_plain": round(t_plain / t_batch, 3), "circuits": count, "total_gates": gates,
            "slots": slots, "workload": "random layered circuits, depth U(8,32), widths 2^U(12,20), seed %d" % seed,
            "timing": "wall clock, circuit upload + proof + transcript download per job"}


def served(n_jobs, seed, slots, rate_factor=3.0, budget_ms=500.0, slo_factors=(0.5, 0.8, 1.0, 1.2, 1.5, 2.0, 3.0)):
    """Poisson arrivals of jobs mixing 2^14-, 2^18- and 2^22-gate random
    layered circuits (depth 16) and SHA-256 compression circuits.  The
    arrival rate is rate_factor x the plain form's throughput on the same
    mix; the server (continuous batching) and a one-slot server (the plain
    form with a queue) see the same arrival times.  Latency = submit to
    transcript on the host.  slo: both forms at arrival rates slo_factors x
    the plain form's saturated rate; each form's best throughput among the
    rates whose p99 stays within budget_ms."""
    import threading as th
    import virgo_b200 as vb
    from virgo_b200 import circuits
    from virgo_b200 import sha256_circuit
    rng = np.random.default_rng(seed)
    pool = {g: [circuits.random_by_gates(g, 16, seed=1000 * g + i) for i in range(3)] for g in (14, 18, 22)}
    # SHA-256 compression circuits over 2^4 and 2^6 blocks (2.1 M and 8.4 M gates)
    pool["sha4"] = [sha256_circuit.sha256_blocks(16, seed=41 + i) for i in range(2)]
    pool["sha6"] = [sha256_circuit.sha256_blocks(64, seed=61)]
    pool = {g: [_pinned_layers(c) for c in cs] for g, cs in pool.items()}
    classes = [14, 18, 22, "sha4", "sha6"]
    kinds = [classes[int(k)] for k in rng.integers(0, len(classes), size=n_jobs)]
    picks = [pool[g][int(rng.integers(len(pool[g])))] for g in kinds]

    def run(nslots, times):
        srv = vb.Server(slots=nslots)
        lat, done_at = [], []
        try:
            # warm every slot on the largest shapes (the largest input and the
            # widest layers), one wave per shape submitted at once, so each
            # idle worker takes one and grows its buffers before the timed
            # arrivals
            for big in (pool["sha6"][0], pool[22][0]):
                warm = [srv.submit(big, 1, transcript=False) for _ in range(nslots)]
                for j in warm:
                    srv.wait(j)
            ids = [None] * n_jobs
            t0 = time.perf_counter()

            def feeder():
                for k in range(n_jobs):
                    dt = t0 + times[k] - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                    ids[k] = srv.submit(picks[k], 500 + k)

            f = th.Thread(target=feeder)
            f.start()
            for k in range(n_jobs):
                while ids[k] is None:
                    time.sleep(0.0005)
                info, _ = srv.wait(ids[k])
                lat.append(info.latency_s)
                done_at.append(time.perf_counter() - t0)
            f.join()
        finally:
            srv.close()
        return lat, max(done_at)

    # the plain form's service rate on this mix (one job at a time)
    lat1, span1 = run(1, np.zeros(n_jobs))
    plain_rate = n_jobs / span1
    rate = rate_factor * plain_rate
    times = np.cumsum(rng.exponential(1.0 / rate, size=n_jobs))
    lat_s, span_s = run(slots, times)
    lat_p, span_p = run(1, times)
    sweep = []
    best = {"served": 0.0, "plain": 0.0}
    base = rng.exponential(1.0, size=n_jobs)   # one arrival pattern, scaled per rate
    for fct in slo_factors:
        ts = np.cumsum(base / (fct * plain_rate))
        row = {"arrival_factor": fct}
        for form, ns in (("served", slots), ("plain", 1)):
            lat, span = run(ns, ts)
            p99 = 1000 * _pctl(lat, 0.99)
            row[form] = {"proofs_s": round(n_jobs / span, 1), "p99_ms": round(p99, 1)}
            if p99 <= budget_ms:
                best[form] = max(best[form], n_jobs / span)
        sweep.append(row)
    return {"value": n_jobs / span_s, "unit": "proofs/s", "p50_ms": 1000 * _pctl(lat_s, 0.5),
            "p99_ms": 1000 * _pctl(lat_s, 0.99),
            "plain": {"value": n_jobs / span_p, "p50_ms": 1000 * _pctl(lat_p, 0.5), "p99_ms": 1000 * _pctl(lat_p, 0.99),
                      "saturated_value": plain_rate},
            "arrival_rate": rate, "jobs": n_jobs, "slots": slots,
            "slo": {"p99_budget_ms": budget_ms, "served_proofs_s": round(best["served"], 1),
                    "plain_proofs_s": round(best["plain"], 1),
                    "ratio": round(best["served"] / best["plain"], 3) if best["plain"] else None, "sweep": sweep},
            "workload": "Poisson arrivals at %.1fx the plain form's rate; equal shares of random layered circuits "
                        "of 2^14, 2^18, 2^22 gates (depth 16) and SHA-256 compression circuits over 2^4 and 2^6 "
                        "blocks" % rate_factor,
            "timing": "wall clock, submit to transcript on the host (circuit upload included)"}


def reference_commit_seconds(log_len, priv, pub, mask, pub_mask, which, pos):
    """The reference's commit path (oracle/_ref/commit_ref: commit_private_array,
    commit_public_array, commit_phase and the query answers through its
    poly_commit API) on the given inputs, one host core; returns its own
    stage timers in seconds."""
    import struct
    tmp = tempfile.mkdtemp(prefix="virgo_commit_")
    try:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<iiiIi", log_len, len(mask), len(pub_mask), 1, len(which)))
            for w, p in zip(which, pos):
                f.write(struct.pack("<iq", int(w), int(p)))
            for a in (priv, pub, mask, pub_mask):
                f.write(np.ascontiguousarray(a, np.uint64).tobytes())
        subprocess.run([COMMIT_BIN, fin, fout], check=True, capture_output=True)
        with open(fout, "rb") as f:
            f.seek(-24, 2)
            return struct.unpack("<ddd", f.read(24))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def commit_path(sizes=(20, 22, 24), reps=3, cpu_sizes=(20,)):
    """Config 2: the kernel-level commit path alone (vg_pc_commit_all: RS
    encodings of a private and a public vector of 2^L seeded F_p2 values,
    the virtual oracle, every FRI fold to 32 entries per slice, every leaf
    chain and Merkle tree, 2 + 2 (L - 6) query answers), host arrays in and
    out, wall clock per call after one warm-up call; Keccak-f count
    65 (2^(L-2) + 2^(L-2) + sum of the FRI levels' leaves)."""
    import virgo_b200 as vb
    L = vb.lib()
    P = (1 << 61) - 1
    ctx = vb.Context(0)
    out = []
    try:
        for log_len in sizes:
            n, S = 1 << log_len, 1 << (log_len - 1)
            rng = np.random.default_rng(log_len)
            fe = lambda k: rng.integers(0, P, (k, 2), dtype=np.uint64)  # noqa: E731
            nlevels = log_len - 6
            gap = 1
            while gap * 2 <= S // 300:
                gap *= 2
            M = S // gap
            priv, pub, mask, pub_mask, fri_r = fe(n), fe(n), fe(300), fe(M), fe(nlevels)
            which = np.array([0, 1] + [2 + t for t in range(nlevels)], np.int32)
            # positions below half the queried set's per-slice length (S for
            # the two committed oracles, S / 2^(t+1) for FRI level t)
            half = np.array([S // 2, S // 2] + [max(1, (S >> (t + 1)) // 2) for t in range(nlevels)], np.int64)
            pos = (rng.integers(0, 1 << 62, len(which)) % half).astype(np.int64)
            nq = len(which)
            roots = np.zeros((2 + nlevels, 32), np.uint8)
            sums, inner = np.zeros((65, 2), np.uint64), np.zeros(2, np.uint64)
            fin = np.zeros((65 * 32, 2), np.uint64)
            qv, qp = np.zeros((nq * 130, 2), np.uint64), np.zeros((nq * 32, 32), np.uint8)
            pc = ctypes.c_void_p()
            vb.check(L.vg_pc_create(ctx.h, ctypes.byref(pc)))
            try:
                ts = []
                for k in range(reps + 1):
                    t0 = time.perf_counter()
                    vb.check(L.vg_pc_commit_all(pc, vb.ptr(priv), log_len, vb.ptr(mask), 300, vb.ptr(pub),
                                                vb.ptr(pub_mask), M, vb.ptr(fri_r), nlevels, nq, vb.ptr(which),
                                                vb.ptr(pos), vb.ptr(roots), vb.ptr(sums), vb.ptr(inner), vb.ptr(fin),
                                                vb.ptr(qv), vb.ptr(qp)), "vg_pc_commit_all")
                    ts.append(time.perf_counter() - t0)
            finally:
                L.vg_pc_destroy(pc)
            t = min(ts[1:])
            leaves = 2 * (n >> 2) + sum(n >> (3 + i) for i in range(nlevels))
            row = {"log_len": log_len, "ms": round(1000 * t, 2), "keccak_f": 65 * leaves,
                   "keccak_f_per_s": round(65 * leaves / t / 1e9, 3), "unit": "G Keccak-f/s",
                   "h2d_bytes": int(priv.nbytes + pub.nbytes + mask.nbytes + pub_mask.nbytes)}
            if log_len in cpu_sizes and os.path.exists(COMMIT_BIN):
                secs = reference_commit_seconds(log_len, priv, pub, mask, pub_mask, which, pos)
                row["cpu_baseline"] = {"value": round(1.0 / sum(secs), 5), "unit": "commits/s", "cores": 1,
                                       "kind": "reference",
                                       "sample": "the same inputs through the reference's poly_commit API on one "
                                                 "host core (commit_private_array %.2f s, commit_public_array "
                                                 "%.2f s, commit_phase %.2f s, its own timers)" % secs}
            out.append(row)
    finally:
        ctx.close()
    return out


def barrier(world):
    from virgo_b200 import replicas
    replicas.barrier()


def max_over_ranks(x, world):
    from virgo_b200 import replicas
    return replicas.max_over_ranks(x)


def roofline(fam, hbm_peak, peak_kind, large=None):
    mem = {k: v for k, v in fam.items() if k in HBM_BOUND}
    if not mem:
        return None
    top = max(mem, key=lambda k: mem[k]["ms"])
    f = mem[top]
    gbs = f["bytes"] / (f["ms"] / 1000.0) / 1e9 if f["ms"] > 0 else 0.0
    per_launch = f["bytes"] / f["launches"]
    traffic = TRAFFIC_RATIO.get(top)
    g = fam.get("gather_round", {"bytes": 0.0, "ms": 0.0})
    both_b, both_ms = f["bytes"] + g["bytes"], f["ms"] + g["ms"]
    return {"bound": "hbm", "kernel": top, "achieved": round(gbs, 1), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(gbs / hbm_peak, 4),
            "traffic": round(per_launch * traffic) if traffic else None,
            "traffic_source": ("profile-derived constant, not measured in this run: the ratio of ncu "
                               "dram__bytes_read.sum + dram__bytes_write.sum to algorithmic bytes on a full-size "
                               "launch (profiles/k_round2_matmul256.txt, %.3f), times this run's average "
                               "algorithmic bytes per launch" % traffic) if traffic else None,
            "peak_source": peak_kind, "launches_per_proof": f["launches"],
            "avg_launch_us": round(1000.0 * f["ms"] / f["launches"], 2), "bytes_per_launch": per_launch,
            "large_launches": ({"achieved": round(large["bytes"] / (large["ms"] / 1000.0) / 1e9, 1),
                                "frac": round(large["bytes"] / (large["ms"] / 1000.0) / 1e9 / hbm_peak, 4),
                                "launches_per_proof": large["launches_per_proof"],
                                "share_of_family_ms": round(large["ms"] / f["ms"], 4),
                                "note": "the round launches that move at least 100 MB each (tables of 2^21 "
                                        "entries and up), same events"}
                               if (large and top == "sumcheck_round" and large["ms"] > 0) else None),
            "with_fused_builds": (
                {"achieved": round(both_b / (both_ms / 1000.0) / 1e9, 1),
                 "frac": round(both_b / (both_ms / 1000.0) / 1e9 / hbm_peak, 4),
                 "note": "the rounds together with the gather_round family: each phase's first two rounds above "
                         "the group start run inside its fused table build (k_gather_round2), so the family's "
                         "largest launches are there"}
                if top == "sumcheck_round" and g["ms"] > 0 else None),
            "alu_pipe_profile": {"frac_large_launches": 0.735, "frac_round_group": 0.33,
                                 "source": "profile-derived constants, not measured in this run: ncu "
                                           "sm__inst_executed_pipe_alu, pct of peak, of a paired round on a "
                                           "2^23-entry table (profiles/k_round2_matmul256.txt) and a 64-CTA "
                                           "round group (profiles/k_round_group_matmul256.txt)"},
            "note": "CUDA events on the launching stream; back-to-back launches share one event, so a "
                    "launch's time runs from the end of the one before it; the large launches are bound by "
                    "the integer ALU pipe (ALU 73.5%, math-pipe throttle the top stall), the round groups of "
                    "the last 17 rounds of each phase by latency"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["matmul256", "matmul16"], default="matmul256")
    ap.add_argument("--batch", type=int, default=16, help="proofs in flight at once (one session each)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-served", action="store_true", help="skip the batched-random and served measurements")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--tune", default="", help="launch shapes to set first, e.g. round_fuse=2,group_start=2048")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    layers = make_workload(args)

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args, layers)))
        return

    os.environ["VIRGO_DEVICE"] = str(local)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.tune:
        import virgo_b200 as vb
        vb.tune_set(local, **{k: int(v) for k, v in (kv.split("=") for kv in args.tune.split(","))})
    r = ours(args, layers, rank, world)
    if rank == 0:
        hbm, kind = peaks()
        total_ms = sum(f["ms"] for f in r["families"].values()) or 1.0
        fam = {k: dict(v, share=round(v["ms"] / total_ms, 4)) for k, v in r["families"].items()}
        line = {
            "metric": METRIC, "value": args.steps * args.batch * world / r["t_batch"], "unit": "proofs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * r["t_batch"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 (F_{p^2}, p = 2^61 - 1)", "data": "synthetic (seeded)",
            "config": bench_config(args, layers),
            "parallelism": ("replicas x%d, " % world if world > 1 else "") + "%d proofs in flight" % args.batch,
            "plain": {"value": args.steps * world / r["t_plain"], "unit": "proofs/s",
                      "ms_per_proof": 1000.0 * r["t_plain"] / args.steps,
                      "note": "one proof at a time on one stream, CUDA-event device time"},
            "e2e": {"value": args.steps * args.batch * world / r["t_e2e"], "unit": "proofs/s",
                    "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"], "clocks": r["clocks_e2e"],
                    "note": "%d proofs per step, wall clock: each session takes a new witness (the 2^17 input "
                            "values, int64) from pinned host memory with the wiring resident, proves, downloads "
                            "its transcript (the reference's timed Prove Time likewise excludes reading the "
                            "circuit)" % args.batch},
            "e2e_circuit": {"value": args.steps * args.batch * world / r["t_e2e_circuit"], "unit": "proofs/s",
                            "h2d_bytes_per_step": r["h2d_circuit"], "d2h_bytes_per_step": r["d2h"],
                            "note": "as e2e, but every proof loads its whole circuit from pinned host buffers "
                                    "(uint32 wires, built and validated on the GPU)"},
            "gpu_launches": r["launches"],
            "clocks": r["clocks"],
            "roofline": roofline(r["families"], hbm, kind, r["large_rounds"]),
            "roofline_alu": alu_pipe(args, r),
            "stages_s": r["stages"],
            "kernel_families": fam,
            "autotune": r["autotune"],
        }
        if not args.no_served and world == 1:
            line["commit_path"] = {"note": "config 2, best of 3 calls, wall clock incl. host<->device copies",
                                   "sizes": commit_path()}
            line["batched_random64"] = batched_random(64, seed=4, slots=args.batch)
            line["served"] = served(96, seed=5, slots=args.batch)
        if not args.no_cpu_baseline and world >= 1 and os.path.exists(REF_BIN):
            tmp = tempfile.mkdtemp(prefix="virgo_circ_")
            c, m = os.path.join(tmp, "c.txt"), os.path.join(tmp, "m.txt")
            write_circuit_text(layers, c, m)
            (secs, detail), = run_reference_proofs(c, m, 1, seed0=1)
            line["cpu_baseline"] = {"value": 1.0 / secs, "unit": "proofs/s", "cores": 1, "kind": "reference",
                                    "sample": "one reference proof of the workload on 1 core (Prove Time with "
                                              "the fft_gkr side proof, plus evaluate)", "detail": detail}
        else:
            line["cpu_baseline"] = None
        if (not args.no_cpu_baseline and not args.no_served and world == 1 and os.path.exists(REF_BIN)
                and args.workload == "matmul256"):
            cb_batch, cb_served = cpu_baselines_batched_served()
            line["batched_random64"]["cpu_baseline"] = cb_batch
            line["served"]["cpu_baseline"] = cb_served
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
