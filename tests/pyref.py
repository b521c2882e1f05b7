"""Second, independent restatement of the reference hot path in pure Python
(small cases only). Used to cross-check the C oracle: two restatements
written separately from the reference source must agree bit for bit.

FP32 arithmetic is emulated with numpy float32 scalars, so every addition
rounds exactly as the reference's sequential float code does.

Reference files (SammithKanur/iitmGlobalRouter):
  bit_util.hpp:13-191  cost, Fenwick query/update, L-pattern
  gmst_util.hpp:164-341, mst_util.hpp:283-314  Boruvka rounds
  mst_bit_commit.hpp:17-235  GCELL walk of a committed edge
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32


def cost_of(c: int) -> np.float32:
    c = max(-256, min(1024, c))
    return F(math.exp(-0.5 * c))


class PyGrid:
    def __init__(self, X, Y, Z, cap):
        self.X, self.Y, self.Z = X, Y, Z
        self.cap0 = [int(v) for v in cap]
        self.capr = list(self.cap0)
        self.fen = [F(0)] * (X * Y * Z)
        # every cell adds its cost along its update path, cells in id order
        for e in range(X * Y * Z):
            self._add(e, cost_of(self.capr[e]))

    def enc(self, z, x, y):
        return z * self.X * self.Y + (x * self.Y + y if z & 1 else y * self.X + x)

    def dec(self, e):
        z, r = divmod(e, self.X * self.Y)
        if z & 1:
            x, y = divmod(r, self.Y)
        else:
            y, x = divmod(r, self.X)
        return z, x, y

    def _track(self, e):
        z, x, y = self.dec(e)
        p = y if z & 1 else x
        L = self.Y if z & 1 else self.X
        return e - p, p, L

    def _add(self, e, val):
        base, p, L = self._track(e)
        i = p + 1
        while i <= L:
            self.fen[base + i - 1] = F(self.fen[base + i - 1] + val)
            i += i & -i

    def query(self, z, x, y):
        res = F(0)
        if z & 1:
            i = y + 1
            while i > 0:
                res = F(res + self.fen[self.enc(z, x, i - 1)])
                i -= i & -i
        else:
            i = x + 1
            while i > 0:
                res = F(res + self.fen[self.enc(z, i - 1, y)])
                i -= i & -i
        return res

    def rq(self, z, x1, y1, x2, y2):
        return F(self.query(z, x2, y2) - self.query(z, x1, y1))

    # bit_util.hpp:91-117
    def _wire(self, c, z, x, y, x2, y2):
        if z & 1:
            if y < y2:
                c = F(c + self.rq(z, x, y - 1, x, y2))
            elif y > y2:
                c = F(c + self.rq(z, x, y2 - 1, x, y))
            return c, x, y2
        if x < x2:
            c = F(c + self.rq(z, x - 1, y, x2, y))
        elif x > x2:
            c = F(c + self.rq(z, x2 - 1, y, x, y))
        return c, x2, y

    def _via(self, c, za, zb, x, y):
        for i in range(min(za, zb), max(za, zb)):
            if i & 1:
                c = F(c + self.rq(i, x, y - 1, x, y))
            else:
                c = F(c + self.rq(i, x - 1, y, x, y))
        return c

    def pattern_cost(self, e1, e2, cpat):
        Z2 = (self.Z + 1) // 2
        z1, x1, y1 = self.dec(e1)
        z2, x2, y2 = self.dec(e2)
        via1, v = divmod(cpat, Z2)
        if via1 == 0:
            return None
        zs, xs, ys, c = z1, x1, y1, F(0)
        bth = xs != x2 and ys != y2
        if zs != via1:
            c = self._via(c, zs, via1, xs, ys)
            zs = via1
        c, xs, ys = self._wire(c, zs, xs, ys, x2, y2)
        via2 = 2 * v if zs & 1 else 2 * v + 1
        if bth and via2 != 0:
            if via2 >= self.Z:
                return None
            c = self._via(c, zs, via2, xs, ys)
            zs = via2
            c, xs, ys = self._wire(c, zs, xs, ys, x2, y2)
        if zs != z2:
            c = self._via(c, zs, z2, xs, ys)
            zs = z2
        if (xs, ys, zs) != (x2, y2, z2):
            return None
        return c

    def lpattern_pair(self, e1, e2):
        Z2 = (self.Z + 1) // 2
        best, bp, first = F(np.inf), -1, -1
        for cpat in range(self.Z * Z2):
            c = self.pattern_cost(e1, e2, cpat)
            if c is None:
                continue
            if first < 0:
                first = cpat
            if c < best:
                best, bp = c, cpat
        if bp < 0:
            return F(np.inf), first
        return best, bp

    # mst_bit_commit.hpp:36-67 and :209-231
    def edge_cells(self, e1, e2, cpat):
        Z2 = (self.Z + 1) // 2
        z1, x1, y1 = self.dec(e1)
        z2, x2, y2 = self.dec(e2)
        via1, v = divmod(cpat, Z2)
        cells = []

        def via(za, zb, x, y):
            for i in range(min(za, zb) + 1, max(za, zb)):
                cells.append(self.enc(i, x, y))

        def wire(z, x, y):
            if z & 1:
                for t in range(min(y, y2), max(y, y2) + 1):
                    cells.append(self.enc(z, x, t))
                return x, y2
            for t in range(min(x, x2), max(x, x2) + 1):
                cells.append(self.enc(z, t, y))
            return x2, y

        bth = x1 != x2 and y1 != y2
        d = 0
        if z1 != via1:
            via(z1, via1, x1, y1)
            d = abs(z1 - via1) - 1
            z1 = via1
        # mst_bit_commit.hpp:216 calls gpu_hash_gcell for the first wire even
        # for the threads of the first layer change's d interior cells, whose
        # local index is then -d..-1: they mark the d cells before the wire's
        # lower end (contiguous cell ids, into the previous track at 0)
        first = self.enc(z1, x1, min(y1, y2)) if z1 & 1 else self.enc(z1, min(x1, x2), y1)
        cells.extend(first - k for k in range(1, d + 1))
        x1, y1 = wire(z1, x1, y1)
        via2 = 2 * v if z1 & 1 else 2 * v + 1
        if bth and via2 != 0 and z1 != via2:
            via(z1, via2, x1, y1)
            z1 = via2
            x1, y1 = wire(z1, x1, y1)
        if z1 != z2:
            via(z1, z2, x1, y1)
        return cells

    def commit(self, marked):
        for e in sorted(set(marked)):
            inc = F(cost_of(self.capr[e] - 1) - cost_of(self.capr[e]))
            self.capr[e] -= 1
            self._add(e, inc)


def key(w, e):
    w = F(0) if w == 0 else F(w)
    u = int(np.array([w], dtype=np.float32).view(np.uint32)[0])
    u = (~u & 0xFFFFFFFF) if u & 0x80000000 else (u | 0x80000000)
    return (u << 32) | e


def decode(e):
    j = int((1 + math.isqrt(1 + 8 * e)) // 2)
    while j * (j - 1) // 2 > e:
        j -= 1
    while (j + 1) * j // 2 <= e:
        j += 1
    return j, e - j * (j - 1) // 2


def brvsk(n, w, local=0):
    """gmst_util.hpp:164-341 with ties to the lowest pair id and candidates
    processed in ascending root order; returns (slots, dist)."""
    dsu = list(range(n))

    def find(v):
        while dsu[v] != v:
            v = dsu[v]
        return v

    slots, d = [], F(0)
    while len(slots) < n - 1:
        root = [find(v) for v in range(n)]
        best = {}
        e = 0
        for j in range(1, n):
            for k in range(j):
                r1, r2 = root[j], root[k]
                if r1 != r2:
                    kk = key(w[e], e)
                    for r in (r1, r2):
                        if r not in best or kk < best[r]:
                            best[r] = kk
                e += 1
        sel = {}
        for r, kk in best.items():
            j, k = decode(kk & 0xFFFFFFFF)
            sel[r] = root[k] if root[j] == r else root[j]
        for r in sorted(sel):
            a, b = find(r), find(sel[r])
            if a == b:
                continue
            if a < b:
                dsu[a] = b
            else:
                dsu[b] = a
            j, k = decode(best[r] & 0xFFFFFFFF)
            d = F(d + F(w[j * (j - 1) // 2 + k]))
            slots.append((local << 30) | (r << 15) | sel[r])
    slots.append(-1)
    return slots[:n], d
