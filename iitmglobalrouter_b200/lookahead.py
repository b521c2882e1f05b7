"""Congestion lookahead: a small convolutional network over the routing grid.

The network (``gr_cnn_*`` in the C ABI) reads, per routing layer, the
current demand and capacity of every GCELL and predicts the demand the
remaining batches will still add. It is trained on snapshots of the router's
own runs (demand after 10/25/50/75 % of the batches against the final
demand) and its prediction becomes a lookahead term of the GCELL cost used
by the L-pattern stage.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from ._capi import check, lib, ptr


class LookaheadNet:
    """``n_layers`` 3x3 convolutions, ``hidden`` channels, ReLU between layers.

    Inputs and outputs are CUDA float32 tensors of shape (channels, H, W).
    Parameters per layer: weights (cout, cin, 3, 3) then biases (cout,).
    """

    def __init__(self, in_channels: int, out_channels: int, H: int, W: int, hidden: int = 32, n_layers: int = 4,
                 seed: int = 1, device: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        check(self._lib.gr_cnn_create(C.byref(h), device, in_channels, out_channels, hidden, n_layers, H, W, seed),
              "gr_cnn_create")
        self._h = h
        self.in_channels, self.out_channels, self.H, self.W = in_channels, out_channels, H, W
        self.hidden, self.n_layers, self.device = hidden, n_layers, device

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gr_cnn_destroy(self._h)
            self._h = None

    __del__ = close

    def check(self) -> None:
        """Waits for work enqueued by stream-ordered calls (a captured learned
        route) and raises if a convolution gave up waiting for its results."""
        check(self._lib.gr_cnn_check(self._h), "gr_cnn_check")

    @property
    def num_params(self) -> int:
        return int(self._lib.gr_cnn_num_params(self._h))

    def layer_shapes(self):
        """[(cin, cout)] per layer."""
        out = []
        for l in range(self.n_layers):
            cin = self.in_channels if l == 0 else self.hidden
            cout = self.out_channels if l + 1 == self.n_layers else self.hidden
            out.append((cin, cout))
        return out

    def get_params(self) -> np.ndarray:
        out = np.empty(self.num_params, dtype=np.float32)
        check(self._lib.gr_cnn_get_params(self._h, ptr(out)), "gr_cnn_get_params")
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params
        check(self._lib.gr_cnn_set_params(self._h, ptr(p)), "gr_cnn_set_params")

    def _check_in(self, x):
        import torch

        assert x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
        assert tuple(x.shape) == (self.in_channels, self.H, self.W), x.shape

    @staticmethod
    def _torch_done(x):
        """The network runs on its own stream: whatever torch's stream still
        has queued on x (or on memory it hands out next) finishes first."""
        import torch

        torch.cuda.current_stream(x.device).synchronize()

    def forward(self, x):
        import torch

        self._check_in(x)
        y = torch.empty((self.out_channels, self.H, self.W), dtype=torch.float32, device=x.device)
        self._torch_done(x)
        check(self._lib.gr_cnn_forward(self._h, x.data_ptr(), y.data_ptr()), "gr_cnn_forward")
        return y

    def grads(self, x, target):
        """(loss, gradients in parameter layout) of the mean squared error."""
        self._check_in(x)
        g = np.empty(self.num_params, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._torch_done(x)
        check(self._lib.gr_cnn_grads(self._h, x.data_ptr(), target.data_ptr(), ptr(g), ptr(loss)), "gr_cnn_grads")
        return float(loss[0]), g

    def train_step(self, x, target, lr: float = 1e-3) -> float:
        self._check_in(x)
        loss = np.zeros(1, dtype=np.float32)
        self._torch_done(x)
        check(self._lib.gr_cnn_train_step(self._h, x.data_ptr(), target.data_ptr(), C.c_float(lr), ptr(loss)),
              "gr_cnn_train_step")
        return float(loss[0])


# ---------------------------------------------------------------- data, training, routing

SCALE = 1.0 / 16  # demand and capacity units fed to the network


def _router_for(design, device=0):
    from .router import Router

    dims = design.dims
    R = Router(dims["X"], dims["Y"], dims["Z"], design.caps(), device=device)
    ofs, pins = design.nets()
    R.set_nets(ofs, pins)
    return R


def snapshot_samples(design, fracs=(0.10, 0.25, 0.50, 0.75), num_xdim_parts=4, device=0):
    """Training pairs from one plain route of the design: for each fraction f,
    the network input after round(f * batches) batches and the demand the
    remaining batches add (both scaled by SCALE). CUDA tensors."""
    import torch

    bofs, ids = design.batch(num_xdim_parts)
    R = _router_for(design, device)
    R.plan_set(bofs, ids)
    nb = len(bofs) - 1
    mst = torch.empty(R.plan_slots, dtype=torch.int64, device=f"cuda:{device}")
    pat = torch.empty(R.plan_slots, dtype=torch.int32, device=f"cuda:{device}")
    R.set_lookahead(None)
    R.reset()
    feats, prev = [], 0
    for f in fracs:
        b = min(nb, max(prev, int(round(f * nb))))
        R.route_plan(mst, pat, b0=prev, b1=b)
        feats.append(R.features(SCALE))
        prev = b
    R.route_plan(mst, pat, b0=prev, b1=nb)
    final = R.features(SCALE)
    R.sync()
    Z = R.Z
    out = [(x, (final[:Z] - x[:Z]).contiguous()) for x in feats]
    R.close()
    return out


def shard_seeds(n_designs: int, rank: int, world: int):
    """The design seeds 1..n_designs that rank `rank` of `world` generates:
    seed s goes to rank (s - 1) % world. The ranks share nothing, so the
    training data of many designs is made one design per GPU with no
    collective."""
    return [s for s in range(1, n_designs + 1) if (s - 1) % world == rank]


def write_shard(out_dir, n_designs: int, rank: int, world: int, make_samples) -> Path:
    """Generates this rank's designs' samples with make_samples(seed) -> list
    of (input, target) tensors and saves them, with their seeds, to
    out_dir/shard_<rank>.npz."""
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    xs, ts, seeds = [], [], []
    for s in shard_seeds(n_designs, rank, world):
        for x, t in make_samples(s):
            xs.append(x.detach().cpu().numpy())
            ts.append(t.detach().cpu().numpy())
            seeds.append(s)
    path = out / f"shard_{rank}.npz"
    if xs:
        np.savez(path, x=np.stack(xs), t=np.stack(ts), seed=np.array(seeds, np.int32))
    else:
        np.savez(path, x=np.zeros((0,), np.float32), t=np.zeros((0,), np.float32), seed=np.zeros((0,), np.int32))
    return path


def load_shards(in_dir, device="cpu"):
    """Every shard's samples, in design-seed order (within a design, in the
    order they were made): the same list one process generating every seed
    in turn would have made."""
    import torch

    parts = []
    for f in sorted(Path(in_dir).glob("shard_*.npz")):
        z = np.load(f)
        for i in range(len(z["seed"])):
            parts.append((int(z["seed"][i]), f.name, i, z["x"][i], z["t"][i]))
    parts.sort(key=lambda r: (r[0], r[2]))
    return [(torch.from_numpy(x).to(device), torch.from_numpy(t).to(device)) for _, _, _, x, t in parts]


def train(net, samples, epochs=20, lr=1e-3, seed=0, log=None):
    """Adam on the samples, one sample per step, shuffled every epoch; returns the mean loss per epoch."""
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        order = rng.permutation(len(samples))
        tot = 0.0
        for i in order:
            x, t = samples[i]
            tot += net.train_step(x, t, lr)
        hist.append(tot / len(samples))
        if log:
            log(f"epoch {ep}: loss {hist[-1]:.5f}")
    return hist


def route_lookahead(R, net, mst, pat, n_batches, every=64, beta=1.0, mode="demand"):
    """Route the plan from reset with the lookahead cost: before every block
    of `every` batches the network predicts, from the current demand and
    capacity, the demand still to come, and the cost becomes
    exp(-0.5 (cap_remaining - beta * p)) with p the prediction (mode
    "demand") or only its part beyond the capacity then remaining (mode
    "excess": cells expected to overflow). beta = 0 routes plainly."""
    import torch

    R.set_lookahead(None)
    R.reset()
    Z = R.Z
    for b0 in range(0, n_batches, every):
        b1 = min(n_batches, b0 + every)
        if beta > 0:
            f = R.features(SCALE)
            pred = net.forward(f) * (1.0 / SCALE)
            if mode == "excess":
                pred = torch.relu(pred - (f[Z:] - f[:Z]) * (1.0 / SCALE))
            R.set_lookahead(pred.contiguous(), beta)
        R.route_plan(mst, pat, b0=b0, b1=b1)
    R.sync()
    R.set_lookahead(None)


def quality(design, R, mst, pat):
    """Total overflow, overflowed GCELLs, demand, wirelength and vias of a routed plan."""
    q = design.evaluate(R.demand())
    import os

    wl, vias = design.write_routes(os.devnull, mst.cpu().numpy(), pat.cpu().numpy(), merge=True, rseg=True,
                                   ppatch=True, threads=8)
    return dict(q, wirelength=wl, vias=vias)


def evaluate(design, net, betas=(0.0, 0.5, 1.0, 2.0), every=64, num_xdim_parts=4, device=0, mode="demand"):
    """{beta: quality} of the design routed with each lookahead weight (0 = plain)."""
    import torch

    bofs, ids = design.batch(num_xdim_parts)
    R = _router_for(design, device)
    R.plan_set(bofs, ids)
    mst = torch.empty(R.plan_slots, dtype=torch.int64, device=f"cuda:{device}")
    pat = torch.empty(R.plan_slots, dtype=torch.int32, device=f"cuda:{device}")
    out = {}
    for beta in betas:
        route_lookahead(R, net, mst, pat, len(bofs) - 1, every=every, beta=beta, mode=mode)
        out[beta] = quality(design, R, mst, pat)
    R.close()
    return out


def main(argv=None):
    """Train the lookahead network on router snapshots of seeded 400x400x9
    designs and compare plain and lookahead routing on held-out seeds.

        python -m iitmglobalrouter_b200.lookahead --designs 50 --epochs 20 --out weights.npy --report report.json

    The samples can be made one design per GPU first (no collective; each
    process writes its own shard), then trained on in one process:

        torchrun --nproc-per-node 8 -m iitmglobalrouter_b200.lookahead --designs 50 --shard-dir shards
        python -m iitmglobalrouter_b200.lookahead --samples-dir shards --epochs 20 --out weights.npy
    """
    import argparse
    import json
    import time

    from .router import Design

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--designs", type=int, default=50)
    ap.add_argument("--nets", type=int, default=0, help="nets per design (0: the configuration's)")
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--hidden", type=int, default=32)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--every", type=int, default=64)
    ap.add_argument("--betas", default="0,0.25,0.5,1,2")
    ap.add_argument("--test-seeds", default="1001,1002,1003")
    ap.add_argument("--out", default="")
    ap.add_argument("--report", default="")
    ap.add_argument("--weights", default="", help="evaluate these parameters instead of training")
    ap.add_argument("--mode", default="demand", choices=["demand", "excess"])
    ap.add_argument("--shard-dir", default="",
                    help="only make this rank's share of the training samples (RANK / WORLD_SIZE / LOCAL_RANK "
                         "from the environment, one process per GPU) into this directory, then exit")
    ap.add_argument("--samples-dir", default="", help="train on the shards in this directory")
    a = ap.parse_args(argv)
    import os

    if a.shard_dir:
        import torch

        rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
        dev = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(dev)
        path = write_shard(a.shard_dir, a.designs, rank, world,
                           lambda s: snapshot_samples(Design.generate(a.config, seed=s, n_nets=a.nets), device=dev))
        print(f"rank {rank}/{world}: {path}")
        return {"shard": str(path)}
    t0 = time.time()
    d0 = Design.generate(a.config, seed=1, n_nets=a.nets).dims
    net = LookaheadNet(2 * d0["Z"], d0["Z"], d0["Y"], d0["X"], hidden=a.hidden, n_layers=a.layers, seed=7)
    samples, hist = [], []
    if a.weights:
        net.set_params(np.load(a.weights))
    elif a.samples_dir:
        samples = load_shards(a.samples_dir, device="cuda")
    else:
        for s in range(1, a.designs + 1):
            samples += snapshot_samples(Design.generate(a.config, seed=s, n_nets=a.nets))
    t1 = time.time()
    if not a.weights:
        hist = train(net, samples, epochs=a.epochs, lr=a.lr, log=print)
    t2 = time.time()
    if a.out:
        np.save(a.out, net.get_params())
    betas = [float(b) for b in a.betas.split(",")]
    results = {}
    for s in [int(x) for x in a.test_seeds.split(",")]:
        results[s] = evaluate(Design.generate(a.config, seed=s, n_nets=a.nets), net, betas=betas, every=a.every,
                              mode=a.mode)
        print(s, json.dumps(results[s]))
    rep = {"config": a.config, "mode": a.mode, "designs": a.designs, "samples": len(samples), "epochs": a.epochs, "lr": a.lr,
           "hidden": a.hidden, "layers": a.layers, "every": a.every, "loss": hist, "data_s": t1 - t0,
           "train_s": t2 - t1, "results": {str(k): {str(b): v for b, v in r.items()} for k, r in results.items()}}
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)
    return rep


if __name__ == "__main__":
    main()
