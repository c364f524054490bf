"""Proof transcripts: the ordered prover messages of one Virgo proof.

Both the oracle's recorder (around the reference prover under the reference
verifier) and vg_session_prove write the same records: a tag byte, a uint32
count of 16-byte units, then the units.  Tags:
  R V_res (1)           S mask sum after rho (1)   q/p phase-1 round (3/6)
  u v_u (1)             Q/P phase-2 round (3/6)     z final claims (2)
  f final round (3)     y/g/h mask queries (1 each) C commitment root (2)
  A all_sum (65)        B both roots (4)            T FRI level root (2)
  X/x final codeword, data / mask                   I/J query answers
  V verifier verdict and proof size (only from verifier-driven runs)
"""
from __future__ import annotations

import hashlib
import struct


def parse(blob: bytes) -> list:
    out, i = [], 0
    while i < len(blob):
        tag = chr(blob[i])
        (n,) = struct.unpack_from("<I", blob, i + 1)
        out.append((tag, blob[i + 5:i + 5 + 16 * n]))
        i += 5 + 16 * n
    return out


def read(path: str) -> list:
    with open(path, "rb") as f:
        return parse(f.read())


def prover_records(records: list) -> list:
    """Drops the verifier-only records (the verdict), keeping prover output."""
    return [r for r in records if r[0] != "V"]


def digest(records: list) -> str:
    h = hashlib.sha256()
    for tag, data in records:
        h.update(tag.encode())
        h.update(struct.pack("<I", len(data)))
        h.update(data)
    return h.hexdigest()


def record_hashes(records: list) -> list:
    return [(tag, hashlib.sha256(data).hexdigest()[:32]) for tag, data in records]


def first_difference(a: list, b: list):
    for k, (x, y) in enumerate(zip(a, b)):
        if x != y:
            return k, x[0], y[0]
    if len(a) != len(b):
        return min(len(a), len(b)), "len", "len"
    return None
