"""DRAM traffic per algorithmic unit of each route kernel, from a small ncu
capture (a measurement helper; nothing in the route uses it).

Two steps, the first on a GPU machine:

    # route the batches before b0, then batches [b0, b1) inside the NVTX
    # range "capture" (the only kernels ncu captures); their units go to UNITS.json
    python -m iitmglobalrouter_b200.traffic route --config 3 --batches 200:203 --units UNITS.json
    ncu --nvtx --nvtx-include "capture/" --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum \\
        --clock-control none --csv --log-file DRAM.csv  python -m iitmglobalrouter_b200.traffic route <same>

    # per kernel kind: DRAM bytes of its captured launches / their units
    python -m iitmglobalrouter_b200.traffic reduce --units UNITS.json --csv DRAM.csv --out dram_traffic.json

Units (the same as the benchmark's kernel_units): a pin pair for the
L-pattern kernels; a pin pair of a net above 32 pins for k_mst_large and the
cluster kernel (one kind in the router's own profile); a pin pair of a net
of 3..32 pins for k_mst_warp; a query-table entry (layer, distinct x,
distinct y of a net) for k_qtable; a committed GCELL for k_track_commit
(the demand the batch adds).
"""
from __future__ import annotations

import argparse
import csv
import json
from pathlib import Path

import numpy as np

KINDS = {
    "k_lpat": "pin pair",
    "k_mst_large": "pin pair of a net above 32 pins",
    "k_mst_warp": "pin pair of a net of 3..32 pins",
    "k_qtable": "query-table entry",
    "k_track_commit": "committed GCELL",
}


TABLE_MAX_CELLS = 1 << 20  # nx * ny of the largest per-net query table


def kind_of(kernel: str) -> str | None:
    """The profile kind of an ncu kernel name ('void k_lpat_z<10>(...)')."""
    name = kernel.replace("void ", "").split("(")[0].split("<")[0].strip()
    if name.startswith("k_lpat"):
        return "k_lpat"
    if name in ("k_mst_large", "k_mst_cluster"):
        return "k_mst_large"
    return name if name in KINDS else None


def batch_units(dims, ofs, pins, ids) -> dict:
    """Units of one batch per kernel kind, except the committed GCELLs."""
    n = np.diff(ofs)[ids].astype(np.int64)
    P = n * (n - 1) // 2
    X, Y = dims["X"], dims["Y"]
    XY = X * Y
    entries = 0
    for i in ids:
        p = pins[ofs[i]:ofs[i + 1]]
        z, r = p // XY, p % XY
        x = np.where(z & 1, r // Y, r % X)
        y = np.where(z & 1, r % Y, r // X)
        nx, ny = len(np.unique(x)), len(np.unique(y))
        if nx * ny <= TABLE_MAX_CELLS:  # larger nets' patterns gather from the Fenwick trees directly
            entries += dims["Z"] * nx * ny
    return {"k_lpat": int(P.sum()), "k_mst_large": int(P[n > 32].sum()),
            "k_mst_warp": int(P[(n > 2) & (n <= 32)].sum()), "k_qtable": int(entries)}


def route(args) -> None:
    import torch

    import iitmglobalrouter_b200 as gr

    b0, b1 = (int(v) for v in args.batches.split(":"))
    d = gr.Design.generate(args.config, seed=args.seed)
    dims = d.dims
    ofs, pins = d.nets()
    bofs, ids = d.batch(4)
    R = gr.Router(dims["X"], dims["Y"], dims["Z"], d.caps())
    R.set_nets(ofs, pins)
    R.plan_set(bofs, ids)
    from . import tune

    tune.apply(R, tune.load(tune.key(R)))  # the benchmark's launch shapes, when cached for this GPU and Z
    mst = torch.empty(R.plan_slots, dtype=torch.int64, device="cuda")
    pat = torch.empty(R.plan_slots, dtype=torch.int32, device="cuda")
    units = {k: 0 for k in KINDS}
    R.reset()
    R.route_plan(mst, pat, b0=0, b1=b0)
    R.sync()
    before = int(R.demand().sum())
    torch.cuda.nvtx.range_push("capture")
    R.route_plan(mst, pat, b0=b0, b1=b1)
    R.sync()
    torch.cuda.nvtx.range_pop()
    units["k_track_commit"] = int(R.demand().sum()) - before
    for b in range(b0, b1):
        for k, v in batch_units(dims, ofs, pins, ids[bofs[b]:bofs[b + 1]]).items():
            units[k] += v
    if R.status():
        raise SystemExit(f"device status {R.status():#x}")
    Path(args.units).write_text(json.dumps({"config": args.config, "seed": args.seed, "batches": [b0, b1],
                                            "units": units}, indent=1))
    R.close()


def reduce(args) -> None:
    meta = json.loads(Path(args.units).read_text())
    rows = list(csv.reader(open(args.csv)))
    hdr = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hdr]
    ki, mi, vi, ii = h.index("Kernel Name"), h.index("Metric Name"), h.index("Metric Value"), h.index("ID")
    per_launch = {}
    for r in rows[hdr + 1:]:
        if len(r) > vi:
            per_launch.setdefault((r[ii], r[ki]), {})[r[mi]] = float(r[vi].replace(",", ""))
    agg = {}
    for (_, name), m in per_launch.items():
        k = kind_of(name)
        if k is None:
            continue
        a = agg.setdefault(k, {"launches": 0, "bytes": 0.0})
        a["launches"] += 1
        a["bytes"] += m.get("dram__bytes_read.sum", 0.0) + m.get("dram__bytes_write.sum", 0.0)
    per_unit = {}
    for k, a in agg.items():
        u = meta["units"].get(k, 0)
        if u > 0:
            per_unit[k] = {"unit": KINDS[k], "bytes": round(a["bytes"] / u, 3), "launches": a["launches"],
                           "units": u, "dram_bytes": int(a["bytes"])}
    out = {"what": "DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic unit of each "
                   "route kernel kind over the captured batches",
           "workload": f"synthetic design config {meta['config']}, seed {meta['seed']}, batches "
                       f"{meta['batches'][0]}..{meta['batches'][1] - 1}",
           "per_unit": per_unit}
    Path(args.out).write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out, indent=1))


def main() -> None:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("route")
    r.add_argument("--config", type=int, default=3)
    r.add_argument("--seed", type=int, default=1)
    r.add_argument("--batches", default="200:203")
    r.add_argument("--units", required=True)
    d = sub.add_parser("reduce")
    d.add_argument("--units", required=True)
    d.add_argument("--csv", required=True)
    d.add_argument("--out", required=True)
    a = ap.parse_args()
    route(a) if a.cmd == "route" else reduce(a)


if __name__ == "__main__":
    main()
