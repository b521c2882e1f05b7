"""CPU tests of the native library: exported symbols, design I/O, batching,
route writing. Nothing here launches a kernel."""
import re
from pathlib import Path

import numpy as np
import pytest

import iitmglobalrouter_b200 as gr
from iitmglobalrouter_b200 import _capi

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "iitmgr_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gr_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = gr.lib()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
    # and the ctypes table covers every declaration
    assert set(names) <= set(_capi.SIGNATURES), set(names) - set(_capi.SIGNATURES)
    assert L.gr_version() >= 1


def test_context_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gr.GRError):
        gr.Router(4, 4, 3, np.ones(48, np.int32))


def test_generator_is_deterministic_and_follows_config():
    a = gr.Design.generate(1, seed=7)
    b = gr.Design.generate(1, seed=7)
    c = gr.Design.generate(1, seed=8)
    oa, pa = a.nets()
    ob, pb = b.nets()
    assert np.array_equal(oa, ob) and np.array_equal(pa, pb)
    assert np.array_equal(a.caps(), b.caps())
    assert not np.array_equal(a.caps(), c.caps())
    d = a.dims
    assert (d["X"], d["Y"], d["Z"]) == (64, 64, 5)
    assert d["n_nets"] + d["n_one_pin"] == 2000
    cap = a.caps()
    assert cap.min() >= 0 and cap.max() <= 8
    n = np.diff(oa)
    assert n.min() >= 2 and n.max() <= 60
    # pins ascending and distinct within every net, on layers 0..1
    for i in range(len(n)):
        q = pa[oa[i]:oa[i + 1]]
        assert np.all(np.diff(q) > 0)
    assert (pa // (64 * 64)).max() <= 1


def test_cap_net_text_round_trip(tmp_path):
    d = gr.Design.generate(1, seed=3, n_nets=300)
    d.write(tmp_path / "a.cap", tmp_path / "a.net")
    r = gr.Design.read(tmp_path / "a.cap", tmp_path / "a.net", new_fmt=True)
    assert r.dims == d.dims
    assert np.array_equal(r.caps(), d.caps())
    o1, p1 = d.nets()
    o2, p2 = r.nets()
    assert np.array_equal(o1, o2) and np.array_equal(p1, p2)
    assert r.net_name(0) == d.net_name(0)


def test_reader_grammar_and_pin_dedup(tmp_path):
    # 3 layers of 4x3 GCELLs; the .net holds a duplicated pin, a one-pin net
    # and a net whose pins come in descending cell order
    cap = "3 4 3\n0.5 4.0\n1.0 1.0 1.0\n0 0 0 0\n10 10 10\n10 10\n"
    for z in range(3):
        cap += f"metal{z + 1} {z & 1} 1\n" + "".join(" ".join(str(z + y) for _ in range(4)) + "\n" for y in range(3))
    (tmp_path / "t.cap").write_text(cap)
    net = ("netA\n(\n[p0, 0, (0, 3, 2)]\n[p1, 0, (1, 0, 0)]\n[p2, 0, (0, 3, 2)]\n)\n"
           "netB\n(\n[p0, 0, (1, 1, 1)]\n)\n"
           "netC\n(\n[p0, 0, (1, 2, 2)]\n[p1, 0, (0, 1, 0)]\n[p2, 0, (0, 0, 0)]\n)\n")
    (tmp_path / "t.net").write_text(net)
    d = gr.Design.read(tmp_path / "t.cap", tmp_path / "t.net")
    assert d.dims == dict(X=4, Y=3, Z=3, n_nets=2, n_pins=5, n_one_pin=1)
    cap_arr = d.caps()
    # cap[enc(z, x, y)] = z + y ; enc: even z -> z*12 + y*4 + x, odd z -> z*12 + x*3 + y
    assert cap_arr[0 * 12 + 2 * 4 + 1] == 2 and cap_arr[12 + 1 * 3 + 2] == 3
    ofs, pins = d.nets()
    assert ofs.tolist() == [0, 2, 5]
    assert pins[:2].tolist() == sorted([0 * 12 + 2 * 4 + 3, 12 + 0 * 3 + 0])
    assert pins[2:].tolist() == sorted([12 + 2 * 3 + 2, 1, 0])
    assert [d.net_name(0), d.net_name(1)] == ["netA", "netC"]


def test_reader_rejects_bad_input(tmp_path):
    (tmp_path / "t.cap").write_text("3 2 2\n")
    (tmp_path / "t.net").write_text("")
    with pytest.raises(gr.GRError):
        gr.Design.read(tmp_path / "t.cap", tmp_path / "t.net")
    with pytest.raises(gr.GRError):
        gr.Design.read(tmp_path / "missing.cap", tmp_path / "t.net")


def test_noninteger_capacity_is_rejected(tmp_path):
    cap = "3 2 2\n0.5 4.0\n1 1 1\n0 0 0 0\n10\n10\n"
    for z in range(3):
        cap += f"m{z} 0 1\n1.5 2\n3 4\n"
    (tmp_path / "t.cap").write_text(cap)
    (tmp_path / "t.net").write_text("n\n(\n[p, 0, (0, 0, 0)]\n[p, 0, (0, 1, 1)]\n)\n")
    d = gr.Design.read(tmp_path / "t.cap", tmp_path / "t.net")
    with pytest.raises(gr.GRError) as e:
        d.caps()
    assert e.value.code == -9


def boxes(d):
    ofs, pins = d.nets()
    X, Y = d.dims["X"], d.dims["Y"]
    XY = X * Y
    z = pins // XY
    r = pins % XY
    x = np.where(z & 1, r // Y, r % X)
    y = np.where(z & 1, r % Y, r // X)
    out = []
    for i in range(len(ofs) - 1):
        sl = slice(ofs[i], ofs[i + 1])
        out.append((x[sl].min(), x[sl].max(), y[sl].min(), y[sl].max()))
    return np.array(out)


@pytest.mark.parametrize("config,k", [(1, 4), (1, 1), (1, 7)])
def test_batcher_invariants(config, k):
    d = gr.Design.generate(config, seed=1)
    bofs, ids = d.batch(k)
    n = d.dims["n_nets"]
    assert bofs[0] == 0 and bofs[-1] == n
    assert sorted(ids.tolist()) == list(range(n))  # every net exactly once
    bx = boxes(d)
    ofs, _ = d.nets()
    npins = np.diff(ofs)
    for b in range(len(bofs) - 1):
        s = ids[bofs[b]:bofs[b + 1]]
        assert len(s) > 0
        assert np.all(np.diff(npins[s]) >= 0)  # sorted by pin count (net_part.hpp:347)
        B = bx[s]
        # closed boxes of a batch never intersect (NET_PART_CHECK, part_util.hpp:8-35)
        ox = (B[:, None, 0] <= B[None, :, 1]) & (B[None, :, 0] <= B[:, None, 1])
        oy = (B[:, None, 2] <= B[None, :, 3]) & (B[None, :, 2] <= B[:, None, 3])
        ov = ox & oy
        np.fill_diagonal(ov, False)
        assert not ov.any()


def test_batcher_deterministic():
    d = gr.Design.generate(1, seed=5)
    a = d.batch(4)
    b = d.batch(4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_route_writer_format(tmp_path):
    # one 2-pin net routed with pattern 4 (via1 = 2) on an 8x8x4 grid:
    # (0,5,2) -> (0,1,2): vias 0->1, 1->2 at x 5, wire x 1..5 on layer 2,
    # vias 2->1, 1->0 at x 1
    cap = "4 8 8\n0.5 4.0\n1 1 1 1\n0 0 0 0\n" + " ".join(["10"] * 7) + "\n" + " ".join(["10"] * 7) + "\n"
    for z in range(4):
        cap += f"metal{z + 1} {z & 1} 1\n" + ("5 " * 8 + "\n") * 8
    (tmp_path / "t.cap").write_text(cap)
    (tmp_path / "t.net").write_text("n0\n(\n[p, 0, (0, 5, 2)]\n[p, 0, (0, 1, 2)]\n)\n")
    d = gr.Design.read(tmp_path / "t.cap", tmp_path / "t.net")
    d.set_plan([0, 1], [0])
    wl, vias = d.write_routes(tmp_path / "r.txt", np.array([1, -1]), np.array([4, -1]), merge=True, rseg=False,
                              ppatch=True)
    lines = (tmp_path / "r.txt").read_text().splitlines()
    assert lines[0] == "n0" and lines[1] == "(" and lines[-1] == ")"
    segs = sorted(lines[2:-1])
    assert segs == sorted(["2 1 2 2 5 2", "0 1 2 0 1 2", "1 1 2 1 1 2", "0 5 2 0 5 2", "1 5 2 1 5 2"])
    assert (wl, vias) == (4, 4)
    d.write_routes(tmp_path / "g.txt", np.array([1, -1]), np.array([4, -1]), merge=True, rseg=True, ppatch=True)
    g = (tmp_path / "g.txt").read_text().splitlines()
    assert "6300 10500 metal3 23100 10500 metal3" in g  # 4200*x + 2100
    assert "23100 10500 metal1 23100 10500 metal2" in g
