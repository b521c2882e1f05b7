"""CPU tests of the oracle: hand-derived known answers (tests/golden) and
agreement with the independent Python restatement (tests/pyref.py)."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
import pyref

GOLD = Path(__file__).resolve().parent / "golden"


def rand_grid(X, Y, Z, seed, lo=0, hi=9):
    rng = np.random.default_rng(seed)
    return rng.integers(lo, hi + 1, size=X * Y * Z).astype(np.int32)


def test_cost_lut_known_values():
    g = json.loads((GOLD / "cost_lut.json").read_text())
    for c, v in g["values"]:
        assert oracle.cost_of(c) == np.float32(v), c
        assert pyref.cost_of(c) == np.float32(v)
    # clamped ends: +inf below -177, 0 (or denormal) at large capacities
    assert math.isinf(oracle.cost_of(-300))
    assert oracle.cost_of(5000) == oracle.cost_of(1024)


@pytest.mark.parametrize("X,Y,Z", [(5, 4, 3), (9, 7, 4), (6, 11, 5)])
def test_fenwick_build_and_query(X, Y, Z):
    cap = rand_grid(X, Y, Z, 1)
    g = oracle.Grid(X, Y, Z, cap)
    p = pyref.PyGrid(X, Y, Z, cap)
    assert np.array_equal(g.fenwick().view(np.uint32), np.array(p.fen, dtype=np.float32).view(np.uint32))
    for z in range(Z):
        for x in range(X):
            for y in range(Y):
                assert g.query(z, x, y) == p.query(z, x, y)
                # the prefix query is a sum of costs along the track
                if z & 1:
                    s = sum(float(pyref.cost_of(int(cap[g.enc(z, x, t)]))) for t in range(y + 1))
                else:
                    s = sum(float(pyref.cost_of(int(cap[g.enc(z, t, y)]))) for t in range(x + 1))
                assert abs(g.query(z, x, y) - s) <= 1e-5 * max(1.0, s)


@pytest.mark.parametrize("Z", [3, 4, 5, 9, 10])
def test_lpattern_matches_python_restatement(Z):
    X, Y = 7, 6
    cap = rand_grid(X, Y, Z, Z, 0, 12)
    g = oracle.Grid(X, Y, Z, cap)
    p = pyref.PyGrid(X, Y, Z, cap)
    rng = np.random.default_rng(100 + Z)
    pairs = rng.integers(0, X * Y * Z, size=(120, 2)).astype(np.int32)
    # also stacked pins (same x, y) and pins sharing a row / column
    a = rng.integers(0, X * Y * Z, size=20)
    for e in a:
        z, x, y = p.dec(int(e))
        pairs = np.vstack([pairs, [[e, p.enc((z + 2) % Z, x, y)], [e, p.enc(z, (x + 3) % X, y)],
                                   [e, p.enc(z, x, (y + 2) % Y)]]]).astype(np.int32)
    cost, pat = g.lpattern(pairs.ravel())
    for i, (e1, e2) in enumerate(pairs):
        c, q = p.lpattern_pair(int(e1), int(e2))
        assert pat[i] == q, (i, e1, e2)
        assert np.float32(cost[i]).view(np.uint32) == np.float32(c).view(np.uint32)
        for cp in range(Z * ((Z + 1) // 2)):
            a1, a2 = g.pattern_cost(int(e1), int(e2), cp), p.pattern_cost(int(e1), int(e2), cp)
            assert (a1 is None) == (a2 is None)
            if a1 is not None:
                assert np.float32(a1) == a2


def test_odd_z_second_via_outside_grid_is_invalid():
    # Z=9: via1 even, v=4 gives layer 2*4+1 = 9 == Z (bit_util.hpp:157-164)
    X, Y, Z = 6, 6, 9
    g = oracle.Grid(X, Y, Z, np.full(X * Y * Z, 5, np.int32))
    e1, e2 = g.enc(0, 1, 1), g.enc(0, 4, 3)  # x and y differ
    Z2 = (Z + 1) // 2
    for via1 in range(2, Z, 2):
        assert g.pattern_cost(e1, e2, via1 * Z2 + 4) is None
    assert g.pattern_cost(e1, e2, 1 * Z2 + 4) is not None  # via1 odd: v2 = 8 < 9


def test_lpattern_known_answers():
    k = json.loads((GOLD / "lpattern_kat.json").read_text())
    for case in k["cases"]:
        X, Y, Z = case["grid"]
        g = oracle.Grid(X, Y, Z, np.full(X * Y * Z, case["cap"], np.int32))
        e1, e2 = g.enc(*case["src"]), g.enc(*case["dst"])
        cost, pat = g.lpattern(np.array([e1, e2], np.int32))
        assert int(pat[0]) == case["pattern"], case["name"]
        # cost = (number of GCELL terms) x per-cell cost, to FP32 rounding
        assert abs(float(cost[0]) - case["cells"] * case["cell_cost"]) <= 1e-5 * case["cells"] * case["cell_cost"]


def test_boruvka_known_answer_root_to_root_edges():
    k = json.loads((GOLD / "boruvka_kat.json").read_text())
    for case in k["cases"]:
        slots, d, rounds = oracle.brvsk_net(np.array(case["w"], np.float32), case.get("local", 0))
        assert slots.tolist() == case["slots"], case["name"]
        assert np.float32(d) == np.float32(case["dist"])
        assert rounds == case["rounds"]
        ps, pd = pyref.brvsk(len(case["slots"]), [np.float32(v) for v in case["w"]], case.get("local", 0))
        assert ps == case["slots"] and np.float32(pd) == np.float32(case["dist"])


@pytest.mark.parametrize("n,seed", [(2, 0), (3, 1), (5, 2), (8, 3), (13, 4), (31, 5), (64, 6)])
def test_boruvka_matches_python_restatement(n, seed):
    rng = np.random.default_rng(seed)
    P = n * (n - 1) // 2
    # few distinct values: many ties on cost
    w = rng.integers(0, 4, size=P).astype(np.float32) * np.float32(0.25)
    slots, d, rounds = oracle.brvsk_net(w, 7)
    ps, pd = pyref.brvsk(n, [np.float32(v) for v in w], 7)
    assert slots.tolist() == ps
    assert np.float32(d) == pd
    # spanning tree: n-1 edges connecting all pins, then the sentinel
    assert slots[n - 1] == -1
    par = list(range(n))

    def f(v):
        while par[v] != v:
            v = par[v]
        return v

    for s in slots[: n - 1]:
        assert s >> 30 == 7
        a, b = f(int(s) & 0x7FFF), f((int(s) >> 15) & 0x7FFF)
        assert a != b
        par[a] = b
    assert len({f(v) for v in range(n)}) == 1
    assert rounds <= max(1, math.ceil(math.log2(n)))


def test_commit_walk_known_answer():
    k = json.loads((GOLD / "commit_kat.json").read_text())
    for case in k["cases"]:
        X, Y, Z = case["grid"]
        p = pyref.PyGrid(X, Y, Z, [5] * (X * Y * Z))
        cells = p.edge_cells(p.enc(*case["src"]), p.enc(*case["dst"]), case["pattern"])
        assert sorted(set(cells)) == sorted(p.enc(*c) for c in case["cells"]), case["name"]
        # the oracle marks the same cells: one unit of demand each
        g = oracle.Grid(X, Y, Z, np.full(X * Y * Z, 5, np.int32))
        pins = np.array(sorted([g.enc(*case["src"]), g.enc(*case["dst"])]), np.int32)
        src_is_high = g.enc(*case["src"]) == pins[1]
        assert src_is_high, "the commit walks from the higher pin index"
        pp = np.zeros(1, np.int16) + case["pattern"]
        rc, mp = g.commit(np.array([0, 2]), pins, np.array([0]), np.array([(0 << 15) | 1, -1]), pp)
        assert rc == 0 and mp.tolist() == [case["pattern"], -1]
        dem = g.demand()
        assert sorted(np.nonzero(dem)[0].tolist()) == sorted(set(p.enc(*c) for c in case["cells"]))
        assert dem.max() == 1


def test_route_small_design_matches_python_restatement():
    """Multi-batch routing of a tiny design: oracle == pure-Python restatement
    (costs, patterns, trees, demand and every Fenwick node)."""
    X, Y, Z = 9, 8, 4
    rng = np.random.default_rng(11)
    cap = rng.integers(0, 4, size=X * Y * Z).astype(np.int32)
    g = oracle.Grid(X, Y, Z, cap)
    p = pyref.PyGrid(X, Y, Z, cap)
    nets = []
    for _ in range(14):
        n = int(rng.integers(2, 6))
        x0, y0 = int(rng.integers(0, X - 3)), int(rng.integers(0, Y - 3))
        pins = sorted({p.enc(int(rng.integers(0, 2)), x0 + int(rng.integers(0, 4)), y0 + int(rng.integers(0, 4)))
                       for _ in range(n)})
        if len(pins) >= 2:
            nets.append(pins)
    pin_ofs = np.cumsum([0] + [len(q) for q in nets]).astype(np.int64)
    pins = np.concatenate([np.array(q, np.int32) for q in nets])
    batches = [list(range(0, len(nets), 3)), list(range(1, len(nets), 3)), list(range(2, len(nets), 3))]
    for b in batches:
        r = g.route_batch(pin_ofs, pins, np.array(b, np.int32))
        assert r["rc"] == 0
        pairs = oracle.batch_pairs(pin_ofs, pins, b).reshape(-1, 2)
        exp = [p.lpattern_pair(int(a), int(c)) for a, c in pairs]
        assert [int(q) for q in r["pair_pat"]] == [q for _, q in exp]
        assert np.array_equal(r["pair_cost"].view(np.uint32), np.array([c for c, _ in exp], np.float32).view(np.uint32))
        marked, ofs, slot = [], 0, 0
        for li, nid in enumerate(b):
            q = nets[nid]
            n = len(q)
            w = [c for c, _ in exp[ofs: ofs + n * (n - 1) // 2]]
            slots, _ = pyref.brvsk(n, w, li)
            assert r["mst"][slot: slot + n].tolist() == slots
            for s in slots[: n - 1]:
                a, c = s & 0x7FFF, (s >> 15) & 0x7FFF
                hi, lo = max(a, c), min(a, c)
                pat = exp[ofs + hi * (hi - 1) // 2 + lo][1]
                marked += p.edge_cells(q[hi], q[lo], pat)
            ofs += n * (n - 1) // 2
            slot += n
        p.commit(marked)
        assert g.capr().tolist() == p.capr
        assert np.array_equal(g.fenwick().view(np.uint32), np.array(p.fen, np.float32).view(np.uint32))


def test_golden_design_fixture():
    """A committed fixture: routing the tiny design of golden/route_small.json
    reproduces its trees, patterns, demand and Fenwick checksum."""
    fx = json.loads((GOLD / "route_small.json").read_text())
    X, Y, Z = fx["grid"]
    g = oracle.Grid(X, Y, Z, np.array(fx["cap"], np.int32))
    rc, mst, mp = g.route_batches(fx["pin_ofs"], fx["pins"], fx["batch_ofs"], fx["net_ids"])
    assert rc == 0
    assert mst.tolist() == fx["mst"]
    assert mp.tolist() == fx["mst_pat"]
    assert g.demand().tolist() == fx["demand"]
    assert int(g.fenwick().view(np.uint32).astype(np.uint64).sum()) == fx["fenwick_u32_sum"]


def test_count_oob_pairs_matches_a_direct_count():
    """The odd-Z count (pairs whose pins differ in x and y, each with the
    patterns whose second via would be layer Z) against numpy on a small
    design; zero for even Z."""
    rng = np.random.default_rng(11)
    for Z, per in ((9, 4), (5, 2), (10, 0), (4, 0)):
        X, Y = 30, 20
        g = oracle.Grid(X, Y, Z, np.ones(X * Y * Z, np.int32))
        nets = [np.sort(rng.choice(X * Y * 2, size=int(n), replace=False)).astype(np.int32)
                for n in rng.integers(2, 15, size=40)]
        ofs = np.cumsum([0] + [len(q) for q in nets]).astype(np.int64)
        pins = np.concatenate(nets)
        ids = rng.permutation(len(nets)).astype(np.int32)
        want = 0
        for q in nets:
            dec = []
            for e in q:
                z, r = divmod(int(e), X * Y)
                dec.append((r // Y, r % Y) if z & 1 else (r % X, r // X))
            want += sum(1 for j in range(len(q)) for k in range(j) if dec[j][0] != dec[k][0] and dec[j][1] != dec[k][1])
        got = g.count_oob_pairs(ofs, pins, ids)
        assert got == ((want, per * want) if per else (0, 0)), (Z, got, want)
