"""CPU checks of the top-level scripts: every global name a function of
bench.py or __graft_entry__.py reads is defined (their GPU paths cannot run
here), and the benchmark's reference arm prints its JSON line."""
import builtins
import json
import subprocess
import sys
import symtable
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _undefined_globals(path: Path):
    top = symtable.symtable(path.read_text(), str(path), "exec")
    defined = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported()}
    defined |= set(dir(builtins)) | {"__file__", "__name__"}
    bad = []

    def walk(t):
        for s in t.get_symbols():
            if t.get_type() == "function" and s.is_global() and s.is_referenced() and s.get_name() not in defined:
                bad.append(f"{t.get_name()}: {s.get_name()}")
        for c in t.get_children():
            walk(c)

    walk(top)
    return bad


@pytest.mark.parametrize("name", ["bench.py", "__graft_entry__.py"])
def test_scripts_reference_only_defined_globals(name):
    assert _undefined_globals(ROOT / name) == []


def test_bench_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "1", "--steps", "1",
                        "--warmup", "0", "--cpu-pairs", "20000"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["unit"] == "nets/s" and out["value"] > 0
    assert out["cpu_baseline"]["kind"] == "port"  # the reference's kernels need Z = 9 or 10 (this design: 5)
    assert out["product_library_loaded"] is False
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["e2e"]["d2h_bytes_per_step"] == 0


def test_gather_bytes_matches_a_literal_walk():
    """The secondary measurement figure (bytes a direct Fenwick evaluation of
    every pattern would gather) equals a pair-by-pair count that follows the
    commit path's edge walk literally: a layer change costs one unit per
    interior cell, a wire two, stacked pins the union of their layers."""
    import numpy as np

    import iitmglobalrouter_b200 as gr

    d = gr.Design.generate(1, seed=3)
    dims = d.dims
    X, Y, Z = dims["X"], dims["Y"], dims["Z"]
    Z2 = (Z + 1) // 2
    ofs, pins = d.nets()

    def dec(e):
        z, r = divmod(int(e), X * Y)
        return (z, r // Y, r % Y) if z & 1 else (z, r % X, r // X)

    def walk(p, q, cp):
        (z1, x1, y1), (z2, x2, y2) = p, q
        via1, v = divmod(cp, Z2)
        bth = x1 != x2 and y1 != y2
        via2 = 2 * v if via1 & 1 else 2 * v + 1
        if via1 < 1 or via1 >= Z or (bth and via2 != 0 and via2 >= Z):
            return None
        if (x1, y1) == (x2, y2):
            cells = {via1} | set(range(min(z1, via1) + 1, max(z1, via1))) | set(range(min(via1, z2) + 1, max(via1, z2)))
            return len(cells)
        units = 0

        def via(a, b):
            return max(abs(a - b) - 1, 0)

        units += via(z1, via1)
        z = via1
        units += 2
        if z & 1:
            y1 = y2
        else:
            x1 = x2
        if bth and via2 != 0 and z != via2:
            units += via(z, via2) + 2
            z = via2
            if z & 1:
                y1 = y2
            else:
                x1 = x2
        units += via(z, z2)
        return units if (x1, y1) == (x2, y2) else None

    total = pats = 0
    for i in range(len(ofs) - 1):
        p = [dec(e) for e in pins[ofs[i]:ofs[i + 1]]]
        for a in range(len(p)):
            for b in range(a + 1, len(p)):
                for cp in range(Z * Z2):
                    u = walk(p[a], p[b], cp)
                    if u is not None:
                        total += u
                        pats += 1
    got = d.gather_bytes(threads=4)
    assert got["patterns"] == pats and got["bytes"] == 4 * total


def test_traffic_reduce_per_unit(tmp_path):
    """The profile helper's reduction: DRAM bytes of the captured launches of
    each kernel kind over that kind's units (L-pattern variants are one kind,
    the cluster Boruvka counts with k_mst_large)."""
    from iitmglobalrouter_b200 import traffic

    units = tmp_path / "u.json"
    units.write_text(json.dumps({"config": 3, "seed": 1, "batches": [5, 6],
                                 "units": {"k_lpat": 100, "k_mst_large": 50, "k_mst_warp": 0, "k_qtable": 10,
                                           "k_track_commit": 20}}))
    rows = ['"ID","Kernel Name","Metric Name","Metric Unit","Metric Value"']
    for i, (k, rd, wr) in enumerate([("void k_lpat_z<10>(GridC)", 700, 0), ("void k_lpat_zs<10, 4>(GridC)", 300, 0),
                                     ("k_mst_large(GridC)", 100, 0), ("void k_mst_cluster<4>(GridC)", 150, 50),
                                     ("k_track_commit(GridC)", 400, 40), ("k_fen_tracks(GridC)", 9, 9)]):
        rows.append(f'"{i}","{k}","dram__bytes_read.sum","byte","{rd}"')
        rows.append(f'"{i}","{k}","dram__bytes_write.sum","byte","{wr}"')
    csvf = tmp_path / "d.csv"
    csvf.write_text("==PROF== noise\n" + "\n".join(rows) + "\n")
    out = tmp_path / "o.json"
    traffic.reduce(type("A", (), {"units": str(units), "csv": str(csvf), "out": str(out)})())
    pu = json.loads(out.read_text())["per_unit"]
    assert pu["k_lpat"]["bytes"] == 10.0 and pu["k_lpat"]["launches"] == 2
    assert pu["k_mst_large"]["bytes"] == 6.0 and pu["k_mst_large"]["launches"] == 2
    assert pu["k_track_commit"]["bytes"] == 22.0
    assert "k_fen_tracks" not in pu and "k_mst_warp" not in pu
