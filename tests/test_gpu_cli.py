"""The `route` command line tool on a .cap/.net pair: its route file equals,
byte for byte, the route file written from the CPU oracle's trees and
patterns for the same design and plan."""
import json
import subprocess

import pytest

import iitmglobalrouter_b200 as gr
import oracle

@pytest.mark.gpu
@pytest.mark.parametrize("flags", [["-wrt_mrg", "-rseg_fmt", "-oprd_ppatch"], [], ["-wrt_mrg", "-graph"]])
def test_route_cli_matches_oracle(cuda, tmp_path, flags):
    d = gr.Design.generate(1, seed=4)
    cap, net, out = tmp_path / "d.cap", tmp_path / "d.net", tmp_path / "d.route"
    d.write(cap, net)
    cmd = [str(gr.LIB_PATH.parent / "route"), "-cap", str(cap), "-net", str(net), "-gr_out", str(out), "-new_fmt",
           "-bit_pmodel", "-batch_part", "-num_xdim_parts", "4", "-report", str(tmp_path / "r.json"), *flags]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    rep = json.loads((tmp_path / "r.json").read_text())
    # oracle route of the design as the reader leaves it
    rd = gr.Design.read(cap, net)
    dims = rd.dims
    ofs, pins = rd.nets()
    bofs, ids = rd.batch(4)
    g = oracle.Grid(dims["X"], dims["Y"], dims["Z"], rd.caps())
    rc, mst, mp = g.route_batches(ofs, pins, bofs, ids, nthreads=8)
    assert rc == 0
    ref = tmp_path / "oracle.route"
    wl, vias = rd.write_routes(ref, mst, mp, merge="-wrt_mrg" in flags, rseg="-rseg_fmt" in flags,
                               ppatch="-oprd_ppatch" in flags)
    assert out.read_bytes() == ref.read_bytes()
    assert rep["nets"] == dims["n_nets"] and rep["batches"] == len(bofs) - 1
    ev = rd.evaluate(g.demand())
    assert rep["overflow"] == ev["overflow"] and rep["demand"] == ev["demand"]
    if "-wrt_mrg" in flags:
        assert (rep["wirelength"], rep["vias"]) == (wl, vias)
    # every net, one-pin nets included, has a block in the file
    names = [ln for ln in out.read_text().splitlines() if ln and not ln[0].isdigit() and ln not in "()"]
    assert len(names) == dims["n_nets"] + dims["n_one_pin"]


def test_route_cli_rejects_other_modes(tmp_path):
    """Modes outside the Fenwick cost model stop before any device work (runs without a GPU)."""
    cmd = [str(gr.LIB_PATH.parent / "route"), "-cap", "x", "-net", "y", "-gr_out", "z", "-rbt_part"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=60)
    assert r.returncode == 2


def test_route_cli_rejects_bad_lookahead_files(tmp_path):
    """A network file that is not a one-dimensional float32 .npy, or settings
    out of range, stop the tool before any device work (runs without a GPU)."""
    import numpy as np

    route = str(gr.LIB_PATH.parent / "route")
    base = [route, "-cap", "x", "-net", "y", "-gr_out", "z", "-bit_pmodel", "-batch_part", "-lookahead"]
    np.save(tmp_path / "two_d.npy", np.zeros((3, 4), np.float32))
    np.save(tmp_path / "f64.npy", np.zeros(5, np.float64))
    (tmp_path / "junk.npy").write_bytes(b"not a numpy file")
    for name in ("two_d.npy", "f64.npy", "junk.npy", "missing.npy"):
        r = subprocess.run(base + [str(tmp_path / name)], capture_output=True, text=True, timeout=60)
        assert r.returncode == 2 and "float32 .npy" in r.stderr, (name, r.stderr)
    np.save(tmp_path / "ok.npy", np.zeros(5, np.float32))
    for extra in (["-la_mode", "sideways"], ["-la_every", "0"], ["-la_layers", "1"]):
        r = subprocess.run(base + [str(tmp_path / "ok.npy")] + extra, capture_output=True, text=True, timeout=60)
        assert r.returncode == 2 and "bad lookahead settings" in r.stderr, (extra, r.stderr)
