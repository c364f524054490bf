"""Seeded synthetic layered circuits in the reference's text format.

A circuit is a list of file-level layers, input layer first; each layer is a
tuple (ty, u, v) of numpy arrays (uint8, int64, int64) with one entry per gate.
The input layer has type 3 gates whose u is the input value.  The text format
is the one of the reference's src/linear_gkr/README.md; the meta file holds
one "is_parallel block_size repeat_num log_block_size log_repeat_num" line per
layer, written as "0 0 1 0 0" (no data-parallel blocks), like the reference's
tests/matmul/gen.cpp.

Generators:
  matmul_addtree(n, bits, seed)  n x n matrix product: n^3 product gates, then
                                 log2(n) layers of pairwise add gates (the
                                 matmul circuits of the benchmark configs)
  random_layered(log_widths, seed, p_mult)  random add/mult layers with wires
                                 uniform over the previous layer
  mixed_gates(seed)              small circuit with every interior gate type
"""
from __future__ import annotations

import numpy as np

Layer = tuple  # (ty: uint8[n], u: int64[n], v: int64[n])


def matmul_addtree(n: int, bits: int, seed: int) -> list:
    assert n >= 2 and n & (n - 1) == 0
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 1 << bits, size=n * n, dtype=np.int64)
    b = rng.integers(0, 1 << bits, size=n * n, dtype=np.int64)
    vals = np.concatenate([a, b])
    layers = [(np.full(2 * n * n, 3, np.uint8), vals, np.zeros(2 * n * n, np.int64))]
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    # product gate (i, j, k) at g = (i n + j) n + k multiplies A[i][k] by B[k][j]
    u = (i * n + k).ravel().astype(np.int64)
    v = (n * n + k * n + j).ravel().astype(np.int64)
    layers.append((np.ones(n ** 3, np.uint8), u, v))
    width = n ** 3
    while width > n * n:
        width //= 2
        g = np.arange(width, dtype=np.int64)
        layers.append((np.zeros(width, np.uint8), 2 * g, 2 * g + 1))
    return layers


def random_layered(log_widths: list, seed: int, p_mult: float = 0.5, input_bits: int = 31) -> list:
    """log_widths[0] is the input layer; every other layer draws its gates
    add/mult with probability p_mult of mult and wires uniform over the
    previous layer."""
    rng = np.random.default_rng(seed)
    n0 = 1 << log_widths[0]
    vals = rng.integers(0, 1 << input_bits, size=n0, dtype=np.int64)
    layers = [(np.full(n0, 3, np.uint8), vals, np.zeros(n0, np.int64))]
    prev = n0
    for lw in log_widths[1:]:
        n = 1 << lw
        ty = (rng.random(n) < p_mult).astype(np.uint8)
        u = rng.integers(0, prev, size=n, dtype=np.int64)
        v = rng.integers(0, prev, size=n, dtype=np.int64)
        layers.append((ty, u, v))
        prev = n
    return layers


def random_batch(count: int, seed: int, log_width_range=(12, 20), depth_range=(8, 32), p_mult: float = 0.5) -> list:
    """Independent random layered circuits: per circuit a depth uniform in
    depth_range, per layer a width 2^k with k uniform in log_width_range,
    gates add/mult with probability p_mult, wires uniform over the previous
    layer, 31-bit inputs."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(count):
        depth = int(rng.integers(depth_range[0], depth_range[1] + 1))
        lw = [int(x) for x in rng.integers(log_width_range[0], log_width_range[1] + 1, size=depth)]
        out.append(random_layered(lw, seed=int(rng.integers(1 << 31)), p_mult=p_mult))
    return out


def random_by_gates(total_log: int, depth: int, seed: int, p_mult: float = 0.5) -> list:
    """A random layered circuit of 2^total_log gates spread evenly over
    `depth` layers (the input layer included)."""
    lw = max(1, total_log - int(np.log2(depth)))
    return random_layered([lw] * depth, seed=seed, p_mult=p_mult)


def mixed_gates(seed: int, log_width: int = 6) -> list:
    """Every gate type the reference proves in interior layers (0-2, 5-10,
    12, 13; type 3 constants are only evaluated, zk_prover.cpp:581-584 has no
    bookkeeping for them, and 4 is inserted by the reader) in each layer."""
    rng = np.random.default_rng(seed)
    n = 1 << log_width
    vals = rng.integers(0, 1 << 20, size=n, dtype=np.int64)
    vals[0] = -5  # negative input exercises the int truncation of evaluate()
    layers = [(np.full(n, 3, np.uint8), vals, np.zeros(n, np.int64))]
    types = [0, 1, 2, 5, 6, 7, 8, 9, 10, 12, 13]
    prev = n
    for _layer in range(3):
        ty = np.array([types[g % len(types)] for g in range(n)], np.uint8)
        u = rng.integers(0, prev, size=n, dtype=np.int64)
        v = rng.integers(0, prev, size=n, dtype=np.int64)
        for g in range(n):
            t = ty[g]
            if t == 2:
                u[g] = v[g] = 0
            elif t == 5:
                lo = int(rng.integers(0, prev - 4))
                u[g], v[g] = lo, lo + int(rng.integers(1, 4))
            elif t == 12:
                lo = int(rng.integers(0, prev - 8))
                u[g], v[g] = lo, lo + int(rng.integers(0, 7))
            elif t in (6, 10):
                v[g] = 0
            elif t == 13:
                v[g] = u[g]
        layers.append((ty, u, v))
        prev = n
    return layers


_DIGITS4 = np.array([list(b"%04d" % i) for i in range(10000)], np.uint8)
_POW10 = np.array([10 ** k for k in range(1, 19)], np.int64)


def _decimal_bytes(vals: np.ndarray, sep: int) -> bytes:
    """Integers (|x| < 10^18) as ASCII decimal, each followed by the byte
    `sep`, formatted with array operations: one fixed-width slot per number
    filled four digits at a time from a table, then the leading zeros masked
    out."""
    x = np.ascontiguousarray(vals, dtype=np.int64)
    if x.size == 0:
        return b""
    neg = x < 0
    a = np.abs(x)
    ndig = np.searchsorted(_POW10, a, side="right") + 1          # digits of |x|
    groups = (int(ndig.max()) + 3) // 4
    width = 4 * groups + 1                                        # sign + digits
    slots = np.empty((x.size, width + 1), np.uint8)
    slots[:, 0] = 45                                              # '-'
    slots[:, width] = sep
    q = a
    for g in range(groups - 1, -1, -1):
        q, r = np.divmod(q, 10000)
        slots[:, 1 + 4 * g:5 + 4 * g] = _DIGITS4[r]
    keep = np.empty((x.size, width + 1), bool)
    keep[:, 1:width] = np.arange(width - 1)[None, :] >= (width - 1 - ndig)[:, None]
    keep[:, 0] = neg
    keep[:, width] = True
    return slots[keep].tobytes()


def write_text(layers: list, circuit_path: str, meta_path: str) -> None:
    """Writes the reference text format (one line per layer: the gate count,
    then type, gate index, u, v of every gate), pure Python and numpy."""
    with open(circuit_path, "wb") as f:
        f.write(b"%d\n" % len(layers))
        for ty, u, v in layers:
            n = len(ty)
            f.write(b"%d " % n)
            chunk = 1 << 22
            for lo in range(0, n, chunk):
                hi = min(n, lo + chunk)
                rows = np.empty((hi - lo, 4), dtype=np.int64)
                rows[:, 0] = ty[lo:hi]
                rows[:, 1] = np.arange(lo, hi)
                rows[:, 2] = u[lo:hi]
                rows[:, 3] = v[lo:hi]
                b = _decimal_bytes(rows.ravel(), 32)
                f.write(b[:-1] if hi == n else b)
            f.write(b"\n")
    with open(meta_path, "w") as f:
        for _ in layers:
            f.write("0 0 1 0 0\n")


def total_gates(layers: list) -> int:
    return int(sum(len(t) for t, _, _ in layers))
