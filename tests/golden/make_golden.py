"""Generates the golden fixtures in this directory from the reference itself.

Run in a container where the reference sources are present:
    make -C oracle ref && python tests/golden/make_golden.py
It runs the reference prover + verifier (oracle/_ref/zk_proof_ref, compiled
from the reference's own sources with the transcript recorder wrapped around
every prover entry point) on seeded synthetic circuits, and single reference
routines (oracle/_ref/libvirgo_refkern.so) on seeded inputs, and writes:
  transcripts.json  per case: circuit generator and parameters, prover seed,
                    the number of records, a digest of all prover records,
                    the tag and a short SHA-256 of every record, and the raw
                    records of the first GKR layer (hex)
  kernels.json      FFT / inverse FFT outputs, Merkle roots and hashes
"""
import ctypes
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from virgo_b200 import circuits, transcript  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
P = (1 << 61) - 1

CASES = [
    # name, generator, params, prover seed
    ("matmul16_seed1", "matmul_addtree", {"n": 16, "bits": 16, "seed": 1}, 1),
    ("matmul16_seed7", "matmul_addtree", {"n": 16, "bits": 16, "seed": 2}, 7),
    ("mixed_gates", "mixed_gates", {"seed": 3}, 5),
    ("random_5layer", "random_layered", {"log_widths": [10, 12, 11, 12, 9], "seed": 4}, 11),
    ("random_3layer_pad15", "random_layered", {"log_widths": [8, 9, 8], "seed": 5}, 3),
    ("matmul8_32bit", "matmul_addtree", {"n": 8, "bits": 32, "seed": 6}, 2),
]


def make_circuit(gen, params):
    return getattr(circuits, gen)(**params)


def run_ref(layers, seed, workdir):
    c, m = os.path.join(workdir, "c.txt"), os.path.join(workdir, "m.txt")
    circuits.write_text(layers, c, m)
    fft = os.path.join(workdir, "fft_gkr")
    if not os.path.exists(fft):
        os.symlink(os.path.join(REF, "fft_gkr"), fft)
    tr = os.path.join(workdir, "tr.bin")
    out = subprocess.run([os.path.join(REF, "zk_proof_ref"), c, m, os.path.join(workdir, "r.txt"), str(seed), tr],
                         cwd=workdir, capture_output=True, text=True)
    assert out.returncode == 0 and "Pass" in out.stdout, out.stdout[-500:] + out.stderr[-500:]
    return transcript.read(tr)


def transcripts():
    res = []
    for name, gen, params, seed in CASES:
        with tempfile.TemporaryDirectory() as d:
            recs = run_ref(make_circuit(gen, params), seed, d)
        pr = transcript.prover_records(recs)
        first_layer = []
        for tag, data in pr[1:]:
            first_layer.append([tag, data.hex()])
            if tag == "h":
                break
        res.append({
            "name": name, "generator": gen, "params": params, "seed": seed,
            "n_records": len(pr), "digest": transcript.digest(pr),
            "records": [[t, h] for t, h in transcript.record_hashes(pr)],
            "v_res": pr[0][1].hex(), "first_layer": first_layer,
            "verdict": [recs[-1][0], recs[-1][1].hex()],
        })
        print(name, len(pr), res[-1]["digest"][:16])
    return res


def fe_random(seed, n):
    """Seeded canonical field elements, shape (n, 2) as (img, real)."""
    rng = np.random.default_rng(seed)
    a = np.empty((n, 2), dtype=np.uint64)
    a[:, 0] = rng.integers(0, P, n, dtype=np.uint64)
    a[:, 1] = rng.integers(0, P, n, dtype=np.uint64)
    return a


def kernels():
    """Inputs are regenerated from their seeds by the tests (fe_random, or
    numpy default_rng bytes); outputs are stored whole when small and as a
    SHA-256 otherwise."""
    import hashlib
    L = ctypes.CDLL(os.path.join(REF, "libvirgo_refkern.so"))
    L.ref_init()
    out = {"fft": [], "ifft": [], "tree": [], "hash": []}
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    keep = lambda a: a.tobytes().hex() if a.nbytes <= 4096 else "sha256:" + hashlib.sha256(a.tobytes()).hexdigest()  # noqa: E731
    for k, (lc, lo) in enumerate([(0, 3), (1, 1), (3, 3), (3, 6), (5, 9), (9, 9), (6, 12), (11, 11), (10, 15)]):
        co = fe_random(1000 + k, 1 << lc)
        r = np.zeros((1 << lo, 2), np.uint64)
        L.ref_fft(vp(co), 1 << lc, 1 << lo, lo, vp(r))
        out["fft"].append({"coef_len": 1 << lc, "order": 1 << lo, "seed": 1000 + k, "output": keep(r)})
        ev = fe_random(2000 + k, 1 << lo)
        ri = np.zeros((1 << lc, 2), np.uint64)
        L.ref_ifft(vp(ev), 1 << lc, 1 << lo, lo, vp(ri))
        out["ifft"].append({"coef_len": 1 << lc, "order": 1 << lo, "seed": 2000 + k, "output": keep(ri)})
    for k, n in enumerate([1, 2, 3, 5, 64, 100, 1000]):
        lv = np.random.default_rng(3000 + k).integers(0, 256, (n, 32), dtype=np.uint8)
        sz = 1
        while sz < n:
            sz *= 2
        t = np.zeros((2 * sz, 32), np.uint8)
        L.ref_create_tree(vp(lv), n, vp(t))
        out["tree"].append({"n": n, "seed": 3000 + k, "root": t[1].tobytes().hex(), "tree": keep(t[1:])})
    for k in range(8):
        m = np.random.default_rng(4000 + k).integers(0, 256, 64, dtype=np.uint8)
        d = np.zeros(32, np.uint8)
        L.ref_hash64(vp(m), vp(d))
        out["hash"].append({"seed": 4000 + k, "sha3_256": d.tobytes().hex()})
    out["predicates"] = predicates()
    out["fft_gkr"] = fft_gkr()
    return out


PRED_CASES = [
    # name, generator, params
    ("mixed_gates", "mixed_gates", {"seed": 3}),
    ("random_5layer", "random_layered", {"log_widths": [10, 12, 11, 12, 9], "seed": 4}),
    ("sha256_1block", "sha256_blocks", {"blocks": 1, "seed": 7}),
]


def pred_inputs(case_idx, layers, which):
    """r_0, r_1 (bit length of layer `which`), r_u, r_v (of the layer below),
    alpha, beta: seeded as fe_random(6000 + 100 * case + layer + k)."""
    lg = len(layers[which][0]).bit_length() - 1
    luv = len(layers[which - 1][0]).bit_length() - 1
    base = 6000 + 100 * case_idx + 10 * which
    return [fe_random(base + k, n) for k, n in enumerate([lg, lg, luv, luv, 1, 1])]


def predicates():
    """zk_verifier::predicates of every layer >= 1, through the shim
    oracle/_ref/libvirgo_refverifier.so over the reference's own objects."""
    import hashlib
    from virgo_b200 import sha256_circuit
    L = ctypes.CDLL(os.path.join(REF, "libvirgo_refverifier.so"))
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    out = []
    for ci, (name, gen, params) in enumerate(PRED_CASES):
        layers = (sha256_circuit.sha256_blocks(**params) if gen == "sha256_blocks"
                  else getattr(circuits, gen)(**params))
        d = len(layers)
        bl = np.array([len(t).bit_length() - 1 for t, _, _ in layers], np.int32)
        keep = [[np.ascontiguousarray(t, np.uint8), np.ascontiguousarray(u, np.int64),
                 np.ascontiguousarray(v, np.int64)] for t, u, v in layers]
        ptrs = [(ctypes.c_void_p * d)(*[k[j].ctypes.data for k in keep]) for j in range(3)]
        res = []
        for which in range(1, d):
            ins = pred_inputs(ci, layers, which)
            o = np.zeros((14, 2), np.uint64)
            L.ref_predicates(d, vp(bl), *ptrs, which, *[vp(x) for x in ins], vp(o))
            res.append(o.tobytes().hex())
        out.append({"name": name, "generator": gen, "params": params,
                    "layers": [hashlib.sha256(bytes.fromhex(h)).hexdigest() for h in res] if d > 12 else res})
    return out


def _fe_mul_add(a, x, b):
    """a * x + b in F_p[i]/(i^2 + 1), elements as (img, real)"""
    ai, ar = int(a[0]), int(a[1])
    xi, xr = int(x[0]), int(x[1])
    re = (ar * xr - ai * xi + int(b[1])) % P
    im = (ar * xi + ai * xr + int(b[0])) % P
    return np.array([im, re], np.uint64)


def fft_gkr_records(lg, workdir):
    """Runs oracle/_ref/fft_gkr_rec (the reference fft_gkr, its eval calls
    recorded); returns the sumcheck messages (rounds x 3 x (img, real)), the
    final value of every phase, and the reference's output line."""
    rec, out = os.path.join(workdir, "fg.rec"), os.path.join(workdir, "fg.txt")
    subprocess.run([os.path.join(REF, "fft_gkr_rec"), str(lg), out, rec], check=True, cwd=workdir)
    b = open(rec, "rb").read()
    q, lin, i = [], [], 0
    while i < len(b):
        k = 4 if b[i:i + 1] == b"Q" else 3
        a = np.frombuffer(b[i + 1:i + 1 + 16 * k], np.uint64).reshape(k, 2)
        (q if k == 4 else lin).append(a)
        i += 1 + 16 * k
    msgs = np.array([x[:3] for x in q[0::3]], np.uint64)   # eval(0), eval(1), eval(r) per message
    vals = np.array([_fe_mul_add(x[0], x[2], x[1]) for x in lin], np.uint64)
    return msgs, vals, open(out).read().split()


def fft_gkr():
    """The fft_gkr side prover's messages for lg 1..12 (the reference process
    never seeds rand(), so its stream is that of seed 1)."""
    import hashlib
    out = []
    with tempfile.TemporaryDirectory() as d:
        for lg in range(1, 13):
            msgs, vals, line = fft_gkr_records(lg, d)
            out.append({"lg": lg, "seed": 1, "rounds": len(msgs), "proof_size": int(line[1]),
                        "msgs": msgs.tobytes().hex() if msgs.nbytes <= 4096 else
                        "sha256:" + hashlib.sha256(msgs.tobytes()).hexdigest(),
                        "first": msgs[:4].tobytes().hex(), "vals": vals.tobytes().hex()})
    return out


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "kernels.json"), "w") as f:
        json.dump(kernels(), f, indent=0)
    with open(os.path.join(here, "transcripts.json"), "w") as f:
        json.dump(transcripts(), f, indent=0)
