"""Writes the golden fixtures of tests/golden.

    python tests/golden/make_golden.py

The reference (SammithKanur/iitmGlobalRouter) ships no tests or golden data
for its -bit_pmodel path, so these fixtures are known answers derived by
hand from its source, each with the reasoning beside it, plus one small
routed design computed by tests/pyref.py (a pure-Python restatement written
independently of the C oracle).
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
import pyref  # noqa: E402


def cost_lut():
    # bit_util.hpp:13-15: cost(cap) = expf(-cap * 0.5); integer capacities
    vals = [[c, float(np.float32(math.exp(-0.5 * c)))] for c in (-20, -2, -1, 0, 1, 2, 3, 5, 8, 12, 16, 40)]
    return {"source": "bit_util.hpp:13-15", "values": vals}


def lpattern_kat():
    # Uniform-per-layer capacities; cells = GCELL terms of the cheapest
    # pattern, derived from bit_util.hpp:91-180: a via from za to zb adds the
    # point cost of layers [min, max) at its (x, y); a wire adds the inclusive
    # span along its layer's direction; pattern id = via1 * ceil(Z/2) + v.
    # Equal-cost patterns tie to the lowest id; where x-first and y-first
    # paths have equal cell counts their FP32 sums may round apart, so the
    # case lists every pattern id of minimal cell cost.
    c5 = float(np.float32(math.exp(-2.5)))
    cases = [
        # only x differs on layer 0: via1 = 2 (first even layer); v unused
        # cells: layers 0,1 at both ends (4) + x = 1..5 on layer 2 (5)
        dict(name="x_only", grid=[8, 8, 4], cap=5, src=[0, 1, 2], dst=[0, 5, 2], pattern=4, cells=9, cell_cost=c5),
        # only y differs: via1 = 1; layer 0 at both ends (2) + y = 1..6 (6)
        dict(name="y_only", grid=[8, 8, 4], cap=5, src=[0, 3, 1], dst=[0, 3, 6], pattern=2, cells=8, cell_cost=c5),
        # stacked pins (0,2,2)->(3,2,2): every valid pattern adds the points of
        # layers 0,1,2 in the same order, so costs tie exactly -> lowest id 2
        dict(name="stacked", grid=[8, 8, 4], cap=5, src=[0, 2, 2], dst=[3, 2, 2], pattern=2, cells=3, cell_cost=c5),
        # both pins on layer 1, y differs: no via, wire y = 1..4
        dict(name="layer1_wire", grid=[8, 8, 4], cap=5, src=[1, 1, 1], dst=[1, 1, 4], pattern=2, cells=4,
             cell_cost=c5),
    ]
    return {"source": "bit_util.hpp:91-191", "cases": cases}


def boruvka_kat():
    # gmst_util.hpp:164-341: per round each component root takes its cheapest
    # crossing pair; candidates are unioned in ascending root order
    # (smaller root -> larger root) and the RECORDED edge is
    # (root, other root) at the start of the round, packed
    # (net << 30) | (root << 15) | other. Pair id of (j, k), k < j: j(j-1)/2+k.
    cases = [
        dict(name="two_pins", w=[0.5], slots=[1, -1], dist=0.5, rounds=1),
        # triangle, w(1,0)=3 w(2,0)=1 w(2,1)=2: roots pick 0->2, 1->2, 2->0;
        # record (0,2) and (1,2); (2,0) closes a cycle
        dict(name="triangle", w=[3.0, 1.0, 2.0], slots=[(0 << 15) | 2, (1 << 15) | 2, -1], dist=3.0, rounds=1),
        # all ties: lowest pair id wins: 0->1, 1->0, 2->0 (pair (2,0) id 1);
        # record (0,1), then (2,0) -- 0 was a root when the round started
        dict(name="ties", w=[1.0, 1.0, 1.0], slots=[1, (2 << 15) | 0, -1], dist=2.0, rounds=1),
        # four pins, round 1 joins {0,1} and {2,3}; round 2 records the
        # roots (1,3) although the cheapest crossing pair is (2,1)
        dict(name="root_to_root", w=[1.0, 5.0, 2.0, 6.0, 7.0, 1.5],
             slots=[(0 << 15) | 1, (2 << 15) | 3, (1 << 15) | 3, -1], dist=4.5, rounds=2),
        dict(name="local_id", local=5, w=[0.5], slots=[(5 << 30) | 1, -1], dist=0.5, rounds=1),
    ]
    return {"source": "gmst_util.hpp:164-341, mst_util.hpp:289-314", "cases": cases}


def commit_kat():
    # mst_bit_commit.hpp:36-67,209-231: walk from the higher pin index (src)
    # to the lower; a via marks its interior layers only, a wire marks its
    # inclusive span. The first wire is walked (:216) also by the threads of
    # the first via's d interior cells, with local index -d..-1: they mark
    # the d cells below the wire's lower end. Cells as [z, x, y].
    cases = [
        # (0,5,2)->(0,1,2), pattern 4 = via1 2: via 0->2 marks layer 1 (d = 1),
        # wire x = 1..5 on layer 2 and the cell x = 0 below it, via 2->0 marks
        # layer 1
        dict(name="x_only", grid=[8, 8, 4], src=[0, 5, 2], dst=[0, 1, 2], pattern=4,
             cells=[[1, 5, 2], [2, 0, 2], [2, 1, 2], [2, 2, 2], [2, 3, 2], [2, 4, 2], [2, 5, 2], [1, 1, 2]]),
        # (3,2,2)->(0,2,2), pattern 2 = via1 1: via 3->1 marks layer 2 (d = 1),
        # the zero-length wire still marks its one cell on layer 1 and the
        # cell y = 1 below it (layer 1 runs along y)
        dict(name="stacked", grid=[8, 8, 4], src=[3, 2, 2], dst=[0, 2, 2], pattern=2,
             cells=[[2, 2, 2], [1, 2, 1], [1, 2, 2]]),
        # (0,4,5)->(0,1,1), pattern 3 = via1 1, v 1 -> via2 2: wire y = 1..5 on
        # layer 1 at x 4, wire x = 1..4 on layer 2 at y 1, via 2->0 marks 1
        dict(name="bend", grid=[8, 8, 4], src=[0, 4, 5], dst=[0, 1, 1], pattern=3,
             cells=[[1, 4, y] for y in range(1, 6)] + [[2, x, 1] for x in range(1, 5)] + [[1, 1, 1]]),
    ]
    return {"source": "mst_bit_commit.hpp:17-235", "cases": cases}


def route_small():
    """A 10x9x4 design of 18 nets in three batches, routed by pyref."""
    X, Y, Z = 10, 9, 4
    rng = np.random.default_rng(2024)
    cap = rng.integers(0, 5, size=X * Y * Z).astype(np.int32)
    p = pyref.PyGrid(X, Y, Z, cap)
    nets = []
    while len(nets) < 18:
        n = int(rng.integers(2, 7))
        x0, y0 = int(rng.integers(0, X - 4)), int(rng.integers(0, Y - 4))
        pins = sorted({p.enc(int(rng.integers(0, 2)), x0 + int(rng.integers(0, 5)), y0 + int(rng.integers(0, 5)))
                       for _ in range(n)})
        if len(pins) >= 2:
            nets.append(pins)
    pin_ofs = [0]
    for q in nets:
        pin_ofs.append(pin_ofs[-1] + len(q))
    net_ids = list(range(0, 18, 3)) + list(range(1, 18, 3)) + list(range(2, 18, 3))
    batch_ofs = [0, 6, 12, 18]
    mst, mst_pat = [], []
    for b in range(3):
        ids = net_ids[batch_ofs[b]:batch_ofs[b + 1]]
        res = []
        for nid in ids:
            q = nets[nid]
            res.append({(j, k): p.lpattern_pair(q[j], q[k]) for j in range(len(q)) for k in range(j)})
        marked = []
        for li, nid in enumerate(ids):
            q = nets[nid]
            n = len(q)
            w = [res[li][(j, k)][0] for j in range(n) for k in range(j)]
            slots, _ = pyref.brvsk(n, w, li)
            mst += slots
            for s in slots:
                if s == -1:
                    mst_pat.append(-1)
                    continue
                a, c = s & 0x7FFF, (s >> 15) & 0x7FFF
                hi, lo = max(a, c), min(a, c)
                pat = res[li][(hi, lo)][1]
                mst_pat.append(pat)
                marked += p.edge_cells(q[hi], q[lo], pat)
        p.commit(marked)
    demand = [int(a - b) for a, b in zip(p.cap0, p.capr)]
    fsum = int(np.array(p.fen, np.float32).view(np.uint32).astype(np.uint64).sum())
    return dict(grid=[X, Y, Z], cap=cap.tolist(), pin_ofs=pin_ofs, pins=[e for q in nets for e in q],
                batch_ofs=batch_ofs, net_ids=net_ids, mst=mst, mst_pat=mst_pat, demand=demand,
                fenwick_u32_sum=fsum)


def main():
    for name, fn in [("cost_lut", cost_lut), ("lpattern_kat", lpattern_kat), ("boruvka_kat", boruvka_kat),
                     ("commit_kat", commit_kat), ("route_small", route_small)]:
        (HERE / f"{name}.json").write_text(json.dumps(fn(), indent=None, separators=(",", ":")) + "\n")
        print("wrote", name)


if __name__ == "__main__":
    main()
