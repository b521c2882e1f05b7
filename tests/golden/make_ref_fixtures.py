"""Fixtures from the reference router's own code (TEST INFRASTRUCTURE).

Two steps:

  python tests/golden/make_ref_fixtures.py run  --out DIR    (on a GPU machine)
  python tests/golden/make_ref_fixtures.py pack --src DIR    (anywhere)

`run` writes seeded synthetic designs as .cap/.net text (the package's
generator; the SHA-256 of every file is recorded) and runs
oracle/_ref/ref_harness -- the reference's reader, batcher, -bit_pmodel GPU
path and route writer, built from its sources by oracle/ref/build_ref.py --
on them, leaving the raw arrays in DIR/<design>/:
  small10   48x48x10, 800 nets: everything (every batch's pair costs and
            patterns, MST slots and slot patterns, the GCELLs each batch
            committed, the Fenwick and capacity state before three batches,
            the route file, the reference's cost function table)
  c1, c2    the 64x64x5 and 400x400x9 designs: reader and batcher only (the
            reference's L-pattern kernel needs Z = 9 or 10, and at Z = 9 it
            reads past the grid, so it is not run there)
  c3        the 1.2M-net 1000x1000x10 design: reader and batcher, then a
            second run that routes every batch with timing only
`pack` turns DIR into tests/golden/ref_<design>.npz (+ the small design's
text and the reference's route file, xz-compressed) and ref_timing.json.
tests/test_ref_fixtures.py compares the oracle and this library's host code
with them.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import lzma
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"
FLAGS = ["-new_fmt", "-num_xdim_parts", "4", "-wrt_mrg", "-rseg_fmt", "-oprd_ppatch"]

# name -> (how the design is made, harness mode)
DESIGNS = {
    "small10": ("custom", dict(X=48, Y=48, Z=10, cap_lo=4, cap_hi=8, n_nets=800, seed=3, hot_frac=0.1, hot_lo=0,
                               hot_hi=2, tail_frac=0.01, tail_hi=80, bbox_median=6.0, bbox_sigma=0.8), "full"),
    "c1": ("config", dict(config=1, seed=1), "no_route"),
    "c2": ("config", dict(config=2, seed=1), "no_route"),
    "c3": ("config", dict(config=3, seed=1), "no_route+time"),
}


def make_design(kind, kw):
    import iitmglobalrouter_b200 as gr

    if kind == "custom":
        return gr.Design.generate_custom(**kw)
    return gr.Design.generate(kw["config"], seed=kw["seed"])


def sha256(path: Path) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 22), b""):
            h.update(blk)
    return h.hexdigest()


def run(out: Path, only=None):
    out.mkdir(parents=True, exist_ok=True)
    if not HARNESS.exists():
        raise SystemExit(f"{HARNESS} is missing: build it with python -m oracle.ref.build_ref")
    for name, (kind, kw, mode) in DESIGNS.items():
        if only and name not in only:
            continue
        d = make_design(kind, kw)
        # the small design's raw results are kept; the large ones are packed
        # at once from a scratch directory (their text and arrays are large)
        dd = out / name if name == "small10" else Path(tempfile.mkdtemp(prefix=f"ref_{name}_"))
        dd.mkdir(parents=True, exist_ok=True)
        cap, net = dd / "design.cap", dd / "design.net"
        d.write(str(cap), str(net))
        meta = {"design": name, "kind": kind, "params": kw, "cap_sha256": sha256(cap), "net_sha256": sha256(net)}
        nb = None
        if mode == "full":
            cmd = [str(HARNESS), "-cap", str(cap), "-net", str(net), "-out", str(dd / "ref"), *FLAGS,
                   "-writer_threads", "4", "-mst_cpu_threads", "8"]
            # the Fenwick state before the first, a middle and the last batch
            pre = subprocess.run(cmd[:7] + FLAGS + ["-no_route"], capture_output=True, text=True, timeout=600)
            assert pre.returncode == 0, pre.stderr[-2000:]
            nb = json.loads((dd / "ref" / "summary.json").read_text())["batches"]
            cmd += ["-fen_at", f"0,{nb // 2},{nb - 1}"]
            runs = [cmd]
        else:
            runs = [[str(HARNESS), "-cap", str(cap), "-net", str(net), "-out", str(dd / "ref"), *FLAGS, "-no_route"]]
            if "time" in mode:
                runs.append([str(HARNESS), "-cap", str(cap), "-net", str(net), "-out", str(dd / "ref_time"), *FLAGS,
                             "-time_only", "-mst_cpu_threads", str(os.cpu_count() or 8)])
        for cmd in runs:
            print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=3000)
            (dd / ("log_" + Path(cmd[6]).name + ".txt")).write_text(r.stdout[-20000:] + "\n" + r.stderr[-20000:])
            if r.returncode != 0:
                raise SystemExit(f"{name}: ref_harness exited {r.returncode}: {r.stderr[-2000:]}")
        (dd / "meta.json").write_text(json.dumps(meta, indent=1))
        if name != "small10":
            pack(dd.parent, out / "packed", [name], dirname=dd.name)
            for log in dd.glob("log_*.txt"):
                (out / "packed" / f"{name}_{log.name}").write_text(log.read_text())
            shutil.rmtree(dd)


def _arr(d: Path, name, dtype):
    p = d / name
    return np.fromfile(p, dtype=dtype) if p.exists() else None


def pack(src: Path, dst: Path = HERE, only=None, dirname=None):
    dst.mkdir(parents=True, exist_ok=True)
    timing = {}
    for name in DESIGNS:
        dd = src / (dirname or name)
        if (only and name not in only) or not (dd / "meta.json").exists():
            continue
        meta = json.loads((dd / "meta.json").read_text())
        r = dd / "ref"
        summ = json.loads((r / "summary.json").read_text())
        ofs = _arr(r, "net_ofs.i64", np.int64)
        pins = _arr(r, "net_pins.i32", np.int32)
        names = (r / "net_names.txt").read_text().split("\n")[:-1]
        onames = (r / "odeg_names.txt").read_text().split("\n")[:-1]
        bofs = _arr(r, "npart_ofst.i32", np.int32).astype(np.int64)
        blen = _arr(r, "npart_len.i32", np.int32).astype(np.int64)
        ids = _arr(r, "npart_ids.i32", np.int32)
        caps = _arr(r, "caps.f32", np.float32)
        batch_of = np.full(len(ofs) - 1, -1, np.int32)
        for b in range(len(bofs)):
            batch_of[ids[bofs[b]:bofs[b] + blen[b]]] = b
        out = dict(meta=json.dumps(meta), summary=json.dumps(summ),
                   pins_sha256=hashlib.sha256(ofs.tobytes() + pins.tobytes()).hexdigest(),
                   names_sha256=hashlib.sha256("\n".join(names).encode()).hexdigest(),
                   odeg_names_sha256=hashlib.sha256("\n".join(onames).encode()).hexdigest(),
                   caps_sha256=hashlib.sha256(caps.astype(np.int32).tobytes()).hexdigest(),
                   caps_integral=bool(np.all(caps == np.round(caps))),
                   batch_of=batch_of, batch_len=blen.astype(np.int32))
        if name in ("small10", "c1"):
            out.update(net_ofs=ofs, net_pins=pins, batch_ids=ids, batch_ofs=bofs, net_names="\n".join(names),
                       odeg_names="\n".join(onames))
        if name == "small10":
            out.update(cost_table=_arr(r, "cost_table.f32", np.float32), caps=caps.astype(np.int16),
                       pairs=_arr(r, "pairs.i32", np.int32), pair_cost=_arr(r, "pair_cost.f32", np.float32),
                       pair_pat=_arr(r, "pair_pat.i16", np.int16), mst=_arr(r, "mst.i64", np.int64),
                       mst_pat=_arr(r, "mst_pat.i32", np.int32), marked=_arr(r, "marked.i32", np.int32),
                       marked_ofs=_arr(r, "marked_ofs.i64", np.int64),
                       final_capr=_arr(r, "final_capr.f32", np.float32).astype(np.int16),
                       final_fen=_arr(r, "final_fen.f32", np.float32))
            fen_at = sorted(int(p.stem.split("_b")[1]) for p in r.glob("fen_b*.f32"))
            out["fen_at"] = np.array(fen_at, np.int32)
            for b in fen_at:
                out[f"fen_b{b}"] = _arr(r, f"fen_b{b}.f32", np.float32)
                out[f"capr_b{b}"] = _arr(r, f"capr_b{b}.f32", np.float32).astype(np.int16)
            for fname, tgt in (("design.cap", "ref_small10.cap.xz"), ("design.net", "ref_small10.net.xz"),
                               ("ref/routes.txt", "ref_small10.routes.xz")):
                (dst / tgt).write_bytes(lzma.compress((dd / fname).read_bytes()))
        np.savez_compressed(dst / f"ref_{name}.npz", **out)
        if (dd / "ref_time" / "summary.json").exists():
            timing[name] = json.loads((dd / "ref_time" / "summary.json").read_text())
    if timing:
        tf = dst / "ref_timing.json"
        old = json.loads(tf.read_text()) if tf.exists() else {}
        old.update(timing)
        tf.write_text(json.dumps(old, indent=1) + "\n")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("step", choices=["run", "pack"])
    ap.add_argument("--out", default="ref_runs")
    ap.add_argument("--src", default="ref_runs")
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args()
    if a.step == "run":
        run(Path(a.out), a.only)
    else:
        pack(Path(a.src), HERE, a.only)
