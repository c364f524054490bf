"""Builds layered circuits (every gate reads only the layer below) from a
gate graph of any depth: each value is relayed upward (type 10 gates) as far
as its last consumer needs it, packing gates (type 12, a weighted sum of a
contiguous range of wires) get their operands copied into a contiguous block
of relays in the layer below, and every layer is padded to a power of two
with dummy gates (type 2; input layer: zero inputs), as the reference's
reader expects full layers (src/linear_gkr/zk_verifier.cpp:15-217).

Gate types and their values (src/linear_gkr/zk_prover.cpp:60-157):
  0 a+b   1 a*b   6 1-a   7 a-b   8 a+b-2ab (xor)   9 b-ab (not-a-and-b)
  10 a (relay)   12 sum_j 2^j w_j over a contiguous range   13 a(1-a)
  5 sum of a contiguous range
"""
from __future__ import annotations

import numpy as np


class Builder:
    def __init__(self):
        self.inputs = []        # values of the input layer
        self.ty, self.a, self.b = [], [], []   # per node; a may be a tuple (range operand)
        self.depth = []
        self.outputs = []

    # ---- nodes ----
    def input(self, value: int) -> int:
        self.inputs.append(int(value))
        return self._node(3, None, None, 0)

    def _node(self, ty, a, b, depth):
        self.ty.append(ty)
        self.a.append(a)
        self.b.append(b)
        self.depth.append(depth)
        return len(self.ty) - 1

    def gate(self, ty: int, a: int, b: int | None = None) -> int:
        d = 1 + max(self.depth[a], self.depth[b] if b is not None else 0)
        return self._node(ty, a, b, d)

    def xor(self, a, b):
        return self.gate(8, a, b)

    def mul(self, a, b):
        return self.gate(1, a, b)

    def add(self, a, b):
        return self.gate(0, a, b)

    def sub(self, a, b):
        return self.gate(7, a, b)

    def naab(self, a, b):
        return self.gate(9, a, b)

    def bitcheck(self, a):
        return self.gate(13, a, a)

    def pack(self, bits: list) -> int:
        """sum_j 2^j bits[j] (at most 60 operands): one type-12 gate over a
        block of relays of the operands."""
        assert 1 <= len(bits) <= 60
        d = 2 + max(self.depth[x] for x in bits)
        return self._node(12, tuple(bits), None, d)

    def total(self, xs: list) -> int:
        """sum of xs: one type-5 gate over a block of relays of the operands."""
        d = 2 + max(self.depth[x] for x in xs)
        return self._node(5, tuple(xs), None, d)

    def add_tree(self, xs: list) -> int:
        xs = list(xs)
        while len(xs) > 1:
            nxt = [self.add(xs[i], xs[i + 1]) for i in range(0, len(xs) - 1, 2)]
            if len(xs) % 2:
                nxt.append(xs[-1])
            xs = nxt
        return xs[0]

    def output(self, x: int):
        self.outputs.append(x)

    # ---- layering ----
    def layers(self) -> list:
        n = len(self.ty)
        depth = self.depth
        D = max(depth[o] for o in self.outputs)
        need = [-1] * n   # last layer where the value must be present
        for x in range(n):
            t, a, b = self.ty[x], self.a[x], self.b[x]
            if isinstance(a, tuple):
                for y in a:
                    need[y] = max(need[y], depth[x] - 2)
            elif t != 3:
                need[a] = max(need[a], depth[x] - 1)
                if b is not None:
                    need[b] = max(need[b], depth[x] - 1)
        for o in self.outputs:
            need[o] = D
        outs = set(self.outputs)
        by_depth = [[] for _ in range(D + 1)]
        for x in range(n):
            if depth[x] <= D and self.ty[x] != 3 and (need[x] >= depth[x] or x in outs):
                by_depth[depth[x]].append(x)
        live_from = [[] for _ in range(D + 2)]   # values relayed from layer k on
        for x in range(n):
            for k in range(depth[x] + 1, need[x] + 1):
                live_from[k].append(x)
        ranged_at = [[] for _ in range(D + 2)]    # range gates whose block sits in layer k
        for x in range(n):
            if isinstance(self.a[x], tuple) and depth[x] <= D:
                ranged_at[depth[x] - 1].append(x)

        where = [dict() for _ in range(D + 1)]   # layer -> {value: index}
        block = {}                               # range gate -> (start, end) in its block layer
        out = []
        # input layer
        inputs = [x for x in range(n) if self.ty[x] == 3]
        vals = np.array([self.inputs[i] for i in range(len(inputs))], np.int64)
        for i, x in enumerate(inputs):
            where[0][x] = i
        w0 = 1 << max(1, (len(inputs) - 1).bit_length())
        ty0 = np.full(w0, 3, np.uint8)
        u0 = np.zeros(w0, np.int64)
        u0[:len(vals)] = vals
        out.append((ty0, u0, np.zeros(w0, np.int64)))
        for k in range(1, D + 1):
            T, U, V = [], [], []
            here = where[k]
            for r in ranged_at[k]:                # contiguous operand blocks first
                start = len(T)
                for y in self.a[r]:
                    T.append(10)
                    U.append(where[k - 1][y])
                    V.append(0)
                block[r] = (start, len(T))
            for x in by_depth[k]:
                t, a, b = self.ty[x], self.a[x], self.b[x]
                here[x] = len(T)
                if isinstance(a, tuple):
                    s, e = block[x]
                    T.append(t)
                    U.append(s)
                    V.append(e - 1 if t == 12 else e)   # 12: inclusive end, 5: exclusive
                else:
                    T.append(t)
                    U.append(where[k - 1][a])
                    V.append(where[k - 1][b] if b is not None else 0)
            for x in live_from[k]:
                here[x] = len(T)
                T.append(10)
                U.append(where[k - 1][x])
                V.append(0)
            w = 1 << max(1, (len(T) - 1).bit_length())
            ty = np.full(w, 2, np.uint8)
            u = np.zeros(w, np.int64)
            v = np.zeros(w, np.int64)
            ty[:len(T)] = T
            u[:len(U)] = U
            v[:len(V)] = V
            out.append((ty, u, v))
        return out
