"""Host-side checks that need no GPU: the library builds and exports the C
ABI, fails loudly without a device, the circuit generators and transcript
format, and glibc's rand stream reproduction."""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

import virgo_b200 as vb
from virgo_b200 import circuits, transcript

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def built():
    if not os.path.exists(vb.LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(ROOT, "virgo_b200"), "-j8"], check=True, capture_output=True)
    return vb.lib()


def test_library_exports_every_declared_function(built):
    names = vb.header_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(built, n)]
    assert not missing, missing


def test_no_device_fails_loudly(built):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    h = ctypes.c_void_p()
    rc = built.vg_ctx_create(0, ctypes.byref(h))
    assert rc == 4   # VG_ERR_NO_DEVICE: no CPU fallback exists
    assert b"CUDA" in built.vg_last_error() or b"device" in built.vg_last_error()


def test_tuning_table_validates_and_resets(built):
    """Launch-shape parameters are host state: defaults, range checks,
    per-device values and reset need no GPU."""
    vb.tune_reset(0)
    vb.tune_reset(1)
    d = vb.tune_get(0)
    assert d == {"group_start": 1 << 17, "round_threads": 256, "ntt_max_log": 10, "ntt_tile_log": 12,
                 "leaf_threads": 256, "leaf_warp_max": 0, "round_fuse": 2, "leaf_rot": 3,
                 "beta_table": 1, "group_split": 0, "lazy_fold": 0, "gather_fuse": 1}
    vb.tune_set(0, group_start=1 << 13, ntt_max_log=8, leaf_warp_max=4096)
    assert vb.tune_get(0)["group_start"] == 1 << 13 and vb.tune_get(1) == d
    for bad in ({"group_start": 3000}, {"group_start": 1 << 10}, {"round_threads": 1024}, {"ntt_max_log": 11},
                {"ntt_tile_log": 14}, {"leaf_threads": 96}, {"leaf_warp_max": -1}, {"round_fuse": 3},
                {"round_fuse": 0}, {"leaf_rot": 4},
                {"beta_table": 2}, {"group_split": -1}, {"gather_fuse": 2}):
        with pytest.raises(vb.VirgoError):
            vb.tune_set(0, **bad)
    assert vb.tune_get(0)["ntt_max_log"] == 8   # a rejected value changes nothing
    lo, hi, df = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
    assert built.vg_tune_range(2, ctypes.byref(lo), ctypes.byref(hi), ctypes.byref(df)) == 0
    assert (lo.value, hi.value, df.value) == (6, 10, 10)
    assert built.vg_tune_range(12, None, None, None) == 2
    assert built.vg_tune_set(64, 0, 2048) == 2 and built.vg_tune_get(-1, 0, ctypes.byref(lo)) == 2
    vb.tune_reset(0)
    assert vb.tune_get(0) == d


def test_autotune_rejects_bad_arguments(built):
    n = ctypes.c_int()
    assert built.vg_autotune(None, 1, 1, 1, None, 0, ctypes.byref(n)) == 2
    hs = (ctypes.c_void_p * 1)(None)
    assert built.vg_autotune(hs, 1, 1, 1, None, 0, ctypes.byref(n)) == 2
    assert built.vg_autotune(hs, 1, 1, 0, None, 0, ctypes.byref(n)) == 2


def test_matmul_generator_shapes():
    L = circuits.matmul_addtree(4, 16, seed=0)
    assert [len(t) for t, _, _ in L] == [32, 64, 32, 16]
    ty, u, v = L[1]
    # gate (i, j, k) multiplies A[i][k] and B[k][j]
    g = (1 * 4 + 2) * 4 + 3
    assert ty[g] == 1 and u[g] == 1 * 4 + 3 and v[g] == 16 + 3 * 4 + 2
    ty, u, v = L[2]
    assert (u == 2 * np.arange(32)).all() and (v == u + 1).all() and (ty == 0).all()
    assert circuits.total_gates(circuits.matmul_addtree(256, 32, 1)) == 2 * 65536 + sum(1 << k for k in range(16, 25))


def test_random_layered_wires_in_range():
    L = circuits.random_layered([6, 8, 5, 7], seed=3)
    prev = 64
    for ty, u, v in L[1:]:
        assert set(np.unique(ty)) <= {0, 1}
        assert u.max() < prev and v.max() < prev and u.min() >= 0
        prev = len(ty)


def test_text_format_roundtrip(tmp_path):
    L = circuits.mixed_gates(9, log_width=4)
    c, m = str(tmp_path / "c.txt"), str(tmp_path / "m.txt")
    circuits.write_text(L, c, m)
    toks = open(c).read().split()
    d = int(toks[0])
    assert d == len(L)
    pos = 1
    for ty, u, v in L:
        n = int(toks[pos])
        rows = np.array(toks[pos + 1:pos + 1 + 4 * n], dtype=np.int64).reshape(n, 4)
        assert (rows[:, 0] == ty).all() and (rows[:, 1] == np.arange(n)).all()
        assert (rows[:, 2] == u).all() and (rows[:, 3] == v).all()
        pos += 1 + 4 * n
    assert open(m).read().count("0 0 1 0 0") == d


def test_transcript_parse_roundtrip():
    blob = b"R" + (1).to_bytes(4, "little") + bytes(range(16)) + b"C" + (2).to_bytes(4, "little") + bytes(32)
    recs = transcript.parse(blob)
    assert [t for t, _ in recs] == ["R", "C"] and len(recs[1][1]) == 32
    assert transcript.first_difference(recs, recs) is None


def test_golden_transcripts_are_consistent():
    with open(os.path.join(ROOT, "tests", "golden", "transcripts.json")) as f:
        cases = json.load(f)
    assert len(cases) >= 5
    for c in cases:
        tags = [t for t, _ in c["records"]]
        assert tags[0] == "R" and tags.count("C") == 2 and "X" in tags
        assert c["verdict"][0] == "V"
        # 33 query repetitions, each: two init answers (l, h) and L-6 step answers
        assert tags.count("I") == 66


def test_glibc_random_r_reproduces_rand():
    """Per-proof random streams (initstate_r + random_r with a 128-byte state)
    reproduce srand(seed)/rand(), the stream the reference draws from."""
    libc = ctypes.CDLL(None)
    for seed in [1, 7, 123456]:
        libc.srand(seed)
        a = [libc.rand() for _ in range(1000)]
        buf = ctypes.create_string_buffer(64)
        state = ctypes.create_string_buffer(128)
        assert libc.initstate_r(ctypes.c_uint(seed), state, ctypes.c_size_t(128), buf) == 0
        out = ctypes.c_int32()
        b = []
        for _ in range(1000):
            libc.random_r(buf, ctypes.byref(out))
            b.append(out.value)
        assert a == b


def test_job_footprint_is_monotone_and_covers_the_matmul(built):
    f = vb.job_footprint
    small, big = f([1 << 14] * 4), f([1 << 17, 1 << 24, 1 << 23])
    assert 0 < small < big
    assert f([1 << 17, 1 << 20]) < f([1 << 17, 1 << 21]) < f([1 << 18, 1 << 21])
    # tables + codewords of the 2^24-gate matmul (measured about 3.4 GB per session)
    assert 3.4e9 < big < 8e9


def test_random_batch_shapes():
    cs = circuits.random_batch(5, seed=3, log_width_range=(4, 6), depth_range=(2, 4))
    assert len(cs) == 5
    for c in cs:
        assert 2 <= len(c) <= 4
        prev = len(c[0][0])
        for t, u, v in c[1:]:
            assert 16 <= len(t) <= 64 and u.max() < prev and v.max() < prev
            prev = len(t)
    c = circuits.random_by_gates(14, 16, seed=1)
    assert len(c) == 16 and circuits.total_gates(c) == 1 << 14


def _read_binary_circuit(path):
    """independent numpy reader of the binary circuit layout"""
    raw = open(path, "rb").read()
    assert raw[:4] == b"VGC1"
    version, d, ib = np.frombuffer(raw, np.uint32, 3, 4)
    assert version == 1
    n = np.frombuffer(raw, np.int64, d, 16)
    pos = (16 + 8 * int(d) + 7) // 8 * 8
    out = []
    for i in range(d):
        wb = 8 if i == 0 else int(ib)
        dt = np.int64 if wb == 8 else np.uint32
        arrs = []
        for k, (cnt, width, t) in enumerate(((n[i], 1, np.uint8), (n[i], wb, dt), (n[i], wb, dt))):
            arrs.append(np.frombuffer(raw, t, int(cnt), pos))
            pos = (pos + int(cnt) * width + 7) // 8 * 8
        out.append(tuple(arrs))
    assert pos == len(raw)
    return out, int(ib)


@pytest.mark.parametrize("index_bytes", [4, 8])
def test_binary_circuit_file_roundtrip(built, tmp_path, index_bytes):
    layers = circuits.random_layered([9, 11, 10, 7], seed=3)
    path = str(tmp_path / "c.vgc")
    vb.write_circuit_binary(layers, path, index_bytes=index_bytes)
    assert vb.lib().vg_circuit_is_binary(path.encode()) == 1
    sizes, ib = vb.circuit_binary_info(path)
    assert sizes == [len(t) for t, _, _ in layers] and ib == index_bytes
    got, _ = _read_binary_circuit(path)
    for (t, u, v), (t2, u2, v2) in zip(layers, got):
        assert (t == t2).all() and (u == u2).all() and (v == v2).all()
    # a truncated file is rejected before any device work
    raw = open(path, "rb").read()
    open(path, "wb").write(raw[:-9])
    with pytest.raises(vb.VirgoError):
        vb.circuit_binary_info(path)
    txt = str(tmp_path / "c.txt")
    circuits.write_text(layers, txt, str(tmp_path / "m.txt"))
    assert vb.lib().vg_circuit_is_binary(txt.encode()) == 0


def test_sha256_compression_and_circuit():
    """The generator's compression equals hashlib's SHA-256 on padded single
    blocks, and its circuit, evaluated by the oracle, outputs only zeros
    (every addition and bit test holds for the witness)."""
    import hashlib
    import struct
    import sys
    from virgo_b200 import sha256_circuit as S
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import _oracle as O
    for m in (b"", b"abc", bytes(range(55))):
        blk = m + b"\x80" + b"\x00" * (55 - len(m)) + struct.pack(">Q", 8 * len(m))
        out = S.compress(S.H0, list(struct.unpack(">16I", blk)))["out"]
        assert b"".join(struct.pack(">I", x) for x in out) == hashlib.sha256(m).digest()
    L = S.sha256_blocks(1, seed=2)
    assert all(len(t) & (len(t) - 1) == 0 for t, _, _ in L)
    vals = O.eval_input(L[0][1])
    for t, u, v in L[1:]:
        vals = O.eval_layer(t, u, v, vals)
    assert not vals.any()


def _inc_table(name):
    """A brace-initialised table of numbers from csrc/hash_code.inc."""
    import re
    src = open(os.path.join(ROOT, "virgo_b200", "csrc", "hash_code.inc")).read()
    body = re.search(r"#define %s \{([^}]*)\}" % name, src).group(1)
    return [int(x.strip().rstrip("u"), 0) for x in body.replace("\\", "").split(",") if x.strip()]


def test_warp_keccak_lane_tables_give_sha3():
    """The one-warp-per-chain Keccak (lane x + 5y holds A[x, y]; theta from
    five column shuffles and two neighbour shuffles, rho on the own word, pi
    through the PI_SRC lane, chi from two neighbour shuffles) emulated lane
    by lane with the generated tables equals hashlib's SHA3-256; the
    multiply form of a rotation equals the shift form."""
    import hashlib
    M64 = (1 << 64) - 1
    rho, pi_src = _inc_table("VG_KECCAK_RHO"), _inc_table("VG_KECCAK_PI_SRC")
    rcl, rch = _inc_table("VG_KECCAK_RC_LO"), _inc_table("VG_KECCAK_RC_HI")
    assert len(rho) == len(pi_src) == 25 and sorted(pi_src) == list(range(25))

    def rotl(v, n):
        return ((v << n) | (v >> (64 - n))) & M64 if n else v

    def shfl(vals, src):
        return [vals[s] for s in src]

    def perm(A):
        A = A + [0] * 7
        x = [l % 5 for l in range(32)]
        y = [l // 5 for l in range(32)]
        own = lambda f: [f(l) if l < 25 else l for l in range(32)]  # noqa: E731
        for r in range(24):
            C = [0] * 32
            for yy in range(5):
                s = shfl(A, own(lambda l: x[l] + 5 * yy))
                C = [c ^ v for c, v in zip(C, s)]
            cm = shfl(C, own(lambda l: (x[l] + 4) % 5 + 5 * y[l]))
            cp = shfl(C, own(lambda l: (x[l] + 1) % 5 + 5 * y[l]))
            A = [a ^ m ^ rotl(p, 1) for a, m, p in zip(A, cm, cp)]
            R = [rotl(A[l], rho[l]) if l < 25 else 0 for l in range(32)]
            B = shfl(R, own(lambda l: pi_src[l]))
            b1 = shfl(B, own(lambda l: (x[l] + 1) % 5 + 5 * y[l]))
            b2 = shfl(B, own(lambda l: (x[l] + 2) % 5 + 5 * y[l]))
            A = [b ^ (~p & q & M64) for b, p, q in zip(B, b1, b2)]
            A[0] ^= rcl[r] | (rch[r] << 32)
        return A[:25]

    rng = np.random.default_rng(3)
    for _ in range(4):
        msg = rng.integers(0, 256, 64, dtype=np.uint8).tobytes()
        A = [int.from_bytes(msg[8 * i:8 * i + 8], "little") for i in range(8)] + [0] * 17
        A[8], A[16] = 0x06, 1 << 63
        out = perm(A)
        assert b"".join(out[i].to_bytes(8, "little") for i in range(4)) == hashlib.sha3_256(msg).digest()
    # VG_MROT_LO / VG_MROT_HI: lo * 2^n + umulhi(hi, 2^n) is the rotated low half
    for lo, hi in rng.integers(0, 1 << 32, (200, 2), dtype=np.uint64).tolist():
        for n in range(32):
            v = rotl((hi << 32) | lo, n)
            assert ((lo << n) & 0xFFFFFFFF) + ((hi << n) >> 32) == v & 0xFFFFFFFF
            assert ((hi << n) & 0xFFFFFFFF) + ((lo << n) >> 32) == v >> 32


def test_bench_roofline_fields():
    """bench.py's roofline object from per-family profiles: the dominant
    family, its fraction of the HBM peak, the large launches apart; JSON."""
    import sys
    sys.path.insert(0, ROOT)
    import bench
    fam = {"sumcheck_round": {"launches": 84.0, "ms": 5.3, "bytes": 7.5e9},
           "ntt_pass": {"launches": 22.0, "ms": 1.5, "bytes": 8.5e8}}
    large = {"launches_per_proof": 16.0, "ms": 2.3, "bytes": 6.0e9}
    r = bench.roofline(fam, 6650.0, "fallback", large)
    assert r["kernel"] == "sumcheck_round" and r["bound"] == "hbm"
    assert abs(r["achieved"] - 7.5e9 / 5.3e-3 / 1e9) < 0.1 and 0 < r["frac"] < 1
    assert r["large_launches"]["launches_per_proof"] == 16.0 and r["large_launches"]["frac"] > r["frac"]
    assert r["traffic"] is not None and r["alu_pipe_profile"]["frac_large_launches"] > 0
    json.dumps(r)
    assert bench.roofline(fam, 6650.0, "fallback", None)["large_launches"] is None
    assert r["with_fused_builds"] is None
    fam["gather_round"] = {"launches": 14.0, "ms": 3.0, "bytes": 3.2e9}
    w = bench.roofline(fam, 6650.0, "fallback", large)["with_fused_builds"]
    assert abs(w["achieved"] - (7.5e9 + 3.2e9) / 8.3e-3 / 1e9) < 0.1
    hbm, kind = bench.peaks()
    assert hbm > 0 and kind in ("measured", "fallback")


def test_bench_alu_roofline():
    """bench.py's integer-pipe roofline: the proofs' ALU instructions over the
    step's time against 2 warp instructions per SM cycle on 148 SMs; the
    floor per proof bounds the batched / plain ratio."""
    import argparse
    import sys
    sys.path.insert(0, ROOT)
    import bench
    args = argparse.Namespace(workload="matmul256", steps=10, batch=16)
    r = {"t_batch": 10 * 16 * 6.6e-3, "t_plain": 10 * 9.1e-3, "clocks": {"sm_mhz": 1965.0}}
    a = bench.alu_pipe(args, r)
    peak = 2 * 148 * 1965e6
    assert a["bound"] == "int_alu" and abs(a["peak"] - peak / 1e9) < 0.1
    floor = bench.ALU_WARP_INST_PER_PROOF["matmul256"] / peak
    assert abs(a["floor_ms_per_proof"] - 1e3 * floor) < 1e-3
    assert abs(a["frac"] - floor / 6.6e-3) < 1e-3 and abs(a["plain_frac"] - floor / 9.1e-3) < 1e-3
    assert abs(a["max_batched_over_plain"] - 9.1e-3 / floor) < 0.01
    json.dumps(a)
    assert bench.alu_pipe(argparse.Namespace(workload="matmul16", steps=1, batch=1), r) is None


def test_text_writer_matches_library_writer(built, tmp_path):
    """The pure-numpy text writer (used where no library of this repository
    may be loaded) writes the same bytes as vg_circuit_write_text, negative
    values and 32-bit inputs included."""
    for k, L in enumerate([circuits.mixed_gates(4, log_width=5), circuits.matmul_addtree(8, 32, seed=2),
                           circuits.random_layered([5, 6, 4], seed=3)]):
        L = [(t, u.copy(), v.copy()) for t, u, v in L]
        if k == 0:
            L[0][1][:4] = [-1, -(1 << 31), (1 << 32) - 1, -123456789012]
        a, am = str(tmp_path / "a.txt"), str(tmp_path / "am.txt")
        b, bm = str(tmp_path / "b.txt"), str(tmp_path / "bm.txt")
        circuits.write_text(L, a, am)
        d = len(L)
        ns = np.array([len(t) for t, _, _ in L], np.int64)
        arrs = [(np.ascontiguousarray(t, np.uint8), np.ascontiguousarray(u, np.int64),
                 np.ascontiguousarray(v, np.int64)) for t, u, v in L]
        tys, us, vs = (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)(), (ctypes.c_void_p * d)()
        for i, (t, u, v) in enumerate(arrs):
            tys[i], us[i], vs[i] = t.ctypes.data, u.ctypes.data, v.ctypes.data
        built.vg_circuit_write_text.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p]
        vb.check(built.vg_circuit_write_text(d, ns.ctypes.data, tys, us, vs, b.encode(), bm.encode()), "write")
        assert open(a, "rb").read().split() == open(b, "rb").read().split()
        assert open(am).read() == open(bm).read()
    x = np.array([0, -1, 9, 10, 9999, 10000, -10 ** 17 + 1, 10 ** 17 - 1, 1 << 33], np.int64)
    assert circuits._decimal_bytes(x, 32).decode().split() == [str(int(v)) for v in x]


def test_reference_pool_keeps_width_and_counts_timed(tmp_path, monkeypatch):
    """The reference arm's process pool: warm-up proofs first, then the timed
    ones; fillers keep it full until the last timed proof ends and are then
    stopped; only timed proofs are returned, each with its own timers.  A
    stand-in script plays the reference binary (same output lines)."""
    import sys
    import time
    sys.path.insert(0, ROOT)
    import bench
    fake = tmp_path / "fake_ref.sh"
    fake.write_text("#!/bin/sh\n"
                    "echo \"total evaluation time: 0.01 seconds.\" >&2\n"
                    "echo \"GKR Prove Time 0.05\" >&2\n"
                    "echo \"Prove Time 0.2\" >&2\n"
                    "echo \"x y 0.02\" > log_fftgkr.txt\n"
                    "sleep 0.3\n"
                    "echo Pass\n")
    fake.chmod(0o755)
    monkeypatch.setattr(bench, "REF_BIN", str(fake))
    monkeypatch.setattr(bench, "FFT_BIN", str(fake))
    t0 = time.perf_counter()
    timed, span, fillers = bench.run_reference_pool("c.txt", "m.txt", n_warm=3, n_timed=5, width=3, seed0=1)
    assert len(timed) == 5 and all(d["verified"] for _, d in timed)
    assert all(abs(s - 0.21) < 1e-9 for s, _ in timed)
    assert 0 < span < time.perf_counter() - t0
    assert fillers >= 1   # 8 proofs on 3 slots: the last wave is topped up


def test_replay_verifier_rejects_malformed_proof_files(tmp_path):
    """The verifier process for serialized proofs (oracle/_ref/zk_verify_file)
    refuses files that are not complete VGPF proofs before it verifies
    anything: wrong magic, a truncated body, trailing bytes."""
    binary = os.path.join(ROOT, "oracle", "_ref", "zk_verify_file")
    if not os.path.exists(binary):
        pytest.skip("replay verifier not built here")
    L = circuits.matmul_addtree(4, 8, seed=1)
    c, m = str(tmp_path / "c.txt"), str(tmp_path / "m.txt")
    circuits.write_text(L, c, m)
    header = b"VGPF" + (1).to_bytes(4, "little") + (5).to_bytes(4, "little") + (1).to_bytes(4, "little") + \
        (17).to_bytes(4, "little")
    cases = {"magic": b"XXXX" + header[4:] + bytes(64), "truncated": header + bytes(8),
             "trailing": header + (0).to_bytes(4, "little") * 3 + (1).to_bytes(8, "little") +
             (0).to_bytes(4, "little") + bytes(2 * 32 + 16 * (65 + 1 + 65)) + b"x"}
    for name, data in cases.items():
        p = str(tmp_path / (name + ".vgpf"))
        open(p, "wb").write(data)
        out = subprocess.run([binary, c, m, p, str(tmp_path / "r.txt")], capture_output=True, text=True, timeout=60)
        assert out.returncode == 2 and "VGPF" in out.stderr, (name, out.stderr)


def test_field_arithmetic_against_schoolbook(tmp_path):
    """The F_p2 product (two folds fewer than folding every partial product),
    x + a*b folded once (fe_fma), sums and differences of csrc/fp2.cuh, built
    for the host, against schoolbook 128-bit arithmetic reduced by % on
    every combination of edge values and on random inputs."""
    import shutil
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / "field_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "virgo_b200", "csrc"),
                    os.path.join(ROOT, "tests", "field_check.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe, "2000000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:]
    assert "cases agree" in out.stdout
