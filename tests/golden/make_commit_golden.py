"""Generates tests/golden/commit_ref.json: the kernel-level commit path run by
the reference itself through its poly_commit API (oracle/_ref/commit_ref,
built from the reference's sources by `make -C oracle ref`).

Run where the reference has been compiled:
    python tests/golden/make_commit_golden.py

For each input length 2^log_len (11 and 15 for the restatement's CPU tests,
20 and 22 for the GPU test at the sizes the commit path is benchmarked on)
it draws seeded F_p2 vectors with numpy (tests/_oracle.fe_random: the
private and public arrays, 300 private mask values, the public mask at the
padded mask length), runs commit_private_array, commit_public_array and
commit_phase (srand(seed) first; one prime_field::random() per FRI level),
and answers one query on each of the two committed oracles and on every
FRI level.  It records the roots, all_sum, the FRI randomness, digests of
the final codeword and of every query answer, and the reference's own stage
times.  2^24 is not run: the reference's arrays at that size need about
60 GB of host memory.
"""
import hashlib
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import _oracle as O  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "commit_ref")
N_PRI_MASK = 300


def mask_len(log_len, n_mask):
    S = 1 << (log_len - 1)
    gap = 1
    while gap * 2 <= S // n_mask:
        gap *= 2
    return S // gap


def case_inputs(log_len):
    """The seeded inputs of one case (shared with the tests)."""
    n, S = 1 << log_len, 1 << (log_len - 1)
    nlevels = log_len - 6
    M = mask_len(log_len, N_PRI_MASK)
    rng = np.random.default_rng(5000 + log_len)
    which = [0, 1] + [2 + t for t in range(nlevels)]
    pos = [int(rng.integers(0, S // 2)) for _ in range(2)] + \
          [int(rng.integers(0, max(1, (S >> (t + 1)) // 2))) for t in range(nlevels)]
    return {"priv": O.fe_random(1000 + log_len, n), "pub": O.fe_random(2000 + log_len, n),
            "pri_mask": O.fe_random(3000 + log_len, N_PRI_MASK), "pub_mask": O.fe_random(4000 + log_len, M),
            "which": which, "pos": pos, "srand": 700 + log_len, "n_pub_mask": M, "nlevels": nlevels}


def sha(b):
    return hashlib.sha256(b).hexdigest()


def query_digest(values, path):
    """values: 130 field elements (16 bytes each), path: digests (32 bytes each)"""
    return sha(np.ascontiguousarray(values, np.uint64).tobytes() + b"".join(bytes(p) for p in path))


def run_reference(log_len):
    x = case_inputs(log_len)
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<iiiIi", log_len, N_PRI_MASK, x["n_pub_mask"], x["srand"], len(x["which"])))
            for w, p in zip(x["which"], x["pos"]):
                f.write(struct.pack("<iq", w, p))
            for k in ("priv", "pub", "pri_mask", "pub_mask"):
                f.write(np.ascontiguousarray(x[k], np.uint64).tobytes())
        out = subprocess.run([BIN, fin, fout], capture_output=True, text=True)
        if out.returncode:
            raise RuntimeError(out.stderr)
        b = open(fout, "rb").read()
    off = 0

    def take(nbytes):
        nonlocal off
        v = b[off:off + nbytes]
        off += nbytes
        return v

    nlevels = struct.unpack("<i", take(4))[0]
    assert nlevels == x["nlevels"]
    roots = [take(32).hex() for _ in range(2 + nlevels)]
    all_sum = take(65 * 16).hex()
    fri_r = take(nlevels * 16).hex()
    fin_n = struct.unpack("<i", take(4))[0]
    data = np.frombuffer(take(64 * fin_n * 16), np.uint64).reshape(-1, 2)
    msk = np.frombuffer(take(fin_n * 16), np.uint64).reshape(-1, 2)
    # the final level in slice-major order (slice s at s * n), the layout of
    # vg_pc_commit_all's final_cw: interleaved position (j << 7) | (s << 1) | b
    # holds entry j + b * n / 2 of slice s; the mask slice pairs (2j, 2j + 1)
    slice_major = np.zeros((65 * fin_n, 2), np.uint64)
    for s in range(64):
        for j in range(fin_n // 2):
            slice_major[s * fin_n + j] = data[(j << 7) | (s << 1)]
            slice_major[s * fin_n + j + fin_n // 2] = data[(j << 7) | (s << 1) | 1]
    for j in range(fin_n // 2):
        slice_major[64 * fin_n + j] = msk[2 * j]
        slice_major[64 * fin_n + j + fin_n // 2] = msk[2 * j + 1]
    queries = []
    for _ in x["which"]:
        vals = np.frombuffer(take(130 * 16), np.uint64).reshape(-1, 2)
        plen = struct.unpack("<i", take(4))[0]
        path = [take(32) for _ in range(plen)]
        queries.append({"values": sha(vals.tobytes()), "path_len": plen, "digest": query_digest(vals, path)})
    secs = struct.unpack("<ddd", take(24))
    assert off == len(b)
    return {"log_len": log_len, "n_pri_mask": N_PRI_MASK, "n_pub_mask": x["n_pub_mask"], "srand": x["srand"],
            "which": x["which"], "pos": x["pos"], "roots": roots, "all_sum": all_sum, "fri_r": fri_r,
            "final_n": fin_n, "final_slice_major": sha(slice_major.tobytes()), "queries": queries,
            "ref_seconds": {"commit_private_array": round(secs[0], 3), "commit_public_array": round(secs[1], 3),
                            "commit_phase": round(secs[2], 3)}}


def main():
    sizes = [int(a) for a in sys.argv[1:]] or [11, 15, 20, 22]
    path = os.path.join(HERE, "commit_ref.json")
    have = {c["log_len"]: c for c in json.load(open(path))} if os.path.exists(path) else {}
    for log_len in sizes:
        have[log_len] = run_reference(log_len)
        print(log_len, have[log_len]["ref_seconds"], flush=True)
    with open(path, "w") as f:
        json.dump([have[k] for k in sorted(have)], f, indent=1)


if __name__ == "__main__":
    main()
