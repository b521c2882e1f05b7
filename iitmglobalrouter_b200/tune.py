"""Autotuner for the launch shapes of the Borůvka size classes.

The routed result does not depend on these parameters (tests check that
every setting gives the same trees, patterns and demand); only the time per
batch does. Per parameter, in turn, every candidate value is timed as the
best of `reps` replays of a plan range (Fenwick reset + route, one CUDA
graph) on the router's own stream with CUDA events, and the fastest is kept
(coordinate descent, starting from the current values). Results are cached
as JSON keyed by GPU name and layer count Z.

    from iitmglobalrouter_b200 import tune
    best = tune.autotune(router, mst, pat, b0=0, b1=None)   # dict param -> value
    tune.save(best, tune.key(router), path)                  # path default: tuning.json beside this file
    tune.apply(router, tune.load(tune.key(router), path))
"""
from __future__ import annotations

import json
from pathlib import Path

from ._capi import (GR_TUNE_LPAT_SPLIT, GR_TUNE_MST_BIG_THREADS, GR_TUNE_MST_CLUSTER_MIN_PINS,
                    GR_TUNE_MST_CLUSTER_THREADS, GR_TUNE_MST_MID_THREADS, GR_TUNE_MST_QUEUE)

NAMES = {
    GR_TUNE_MST_MID_THREADS: "mst_mid_threads",
    GR_TUNE_MST_BIG_THREADS: "mst_big_threads",
    GR_TUNE_MST_CLUSTER_THREADS: "mst_cluster_threads",
    GR_TUNE_MST_CLUSTER_MIN_PINS: "mst_cluster_min_pins",
    GR_TUNE_LPAT_SPLIT: "lpat_split",
    GR_TUNE_MST_QUEUE: "mst_queue",
}
CANDIDATES = {
    GR_TUNE_MST_MID_THREADS: [128, 256, 384, 512, 768, 1024],
    GR_TUNE_MST_BIG_THREADS: [256, 512, 1024],
    GR_TUNE_MST_CLUSTER_THREADS: [256, 384, 512, 768, 1024],
    GR_TUNE_MST_CLUSTER_MIN_PINS: [0, 129, 160, 192],
    GR_TUNE_LPAT_SPLIT: [0, 1, 2, 4],
    GR_TUNE_MST_QUEUE: [0, 1],
}
DEFAULT_PATH = Path(__file__).resolve().parent / "tuning.json"


def key(router) -> str:
    import torch

    return f"{torch.cuda.get_device_name(router.device)}|Z={router.Z}"


def time_range(router, mst, pat, b0: int, b1: int | None, reps: int) -> float:
    """Best-of-reps milliseconds of reset + route of batches [b0, b1) replayed as one graph."""
    import torch

    s = torch.cuda.ExternalStream(router.stream, device=torch.device("cuda", router.device))
    best = float("inf")
    for i in range(reps + 1):  # the first replay captures the graph
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        router.reset()
        router.route_plan(mst, pat, b0=b0, b1=b1, graph=True)
        e1.record(s)
        e1.synchronize()
        if i:
            best = min(best, e0.elapsed_time(e1))
    router.sync()
    return best


def autotune(router, mst, pat, b0: int = 0, b1: int | None = None, reps: int = 3, log=None) -> dict:
    """Coordinate descent over CANDIDATES; leaves the router on the best values and returns them."""
    best_t = time_range(router, mst, pat, b0, b1, reps)
    for p, cands in CANDIDATES.items():
        cur = router.tune_get(p)
        choice = cur
        for v in cands:
            if v == cur:
                continue
            router.tune_set(p, v)
            t = time_range(router, mst, pat, b0, b1, reps)
            if log:
                log(f"{NAMES[p]}={v}: {t:.3f} ms (best {best_t:.3f} ms at {choice})")
            if t < best_t:
                best_t, choice = t, v
        router.tune_set(p, choice)
    return {NAMES[p]: router.tune_get(p) for p in CANDIDATES}


def apply(router, values: dict | None) -> None:
    if not values:
        return
    ids = {v: k for k, v in NAMES.items()}
    for name, v in values.items():
        if name in ids:
            router.tune_set(ids[name], int(v))


def load(k: str, path: Path | str = DEFAULT_PATH) -> dict | None:
    path = Path(path)
    if not path.exists():
        return None
    return json.loads(path.read_text()).get(k)


def save(values: dict, k: str, path: Path | str = DEFAULT_PATH) -> None:
    path = Path(path)
    data = json.loads(path.read_text()) if path.exists() else {}
    data[k] = values
    path.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")
