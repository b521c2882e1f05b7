"""Training samples made one design per GPU: each rank of a world-size-2 run
(spawned processes, a gloo process group for the launch only) writes the
samples of its own design seeds, and the shards load back as the same list,
in the same order, as one process making every seed in turn. The samples
here come from a CPU stand-in for the router's snapshots."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from iitmglobalrouter_b200 import lookahead


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def fake_samples(seed):
    g = torch.Generator().manual_seed(seed)
    n = 1 + seed % 3  # designs give different numbers of snapshots
    return [(torch.rand(4, 5, 6, generator=g), torch.rand(2, 5, 6, generator=g)) for _ in range(n)]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        lookahead.write_shard(out, 7, rank, world, fake_samples)
    finally:
        dist.destroy_process_group()


def test_shard_seeds_partition():
    for world in (1, 2, 3, 8):
        got = sorted(s for r in range(world) for s in lookahead.shard_seeds(50, r, world))
        assert got == list(range(1, 51))


def test_shards_of_two_ranks_equal_one_process(tmp_path):
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path / "two")), nprocs=2, join=True)
    lookahead.write_shard(tmp_path / "one", 7, 0, 1, fake_samples)
    two = lookahead.load_shards(tmp_path / "two")
    one = lookahead.load_shards(tmp_path / "one")
    ref = [p for s in range(1, 8) for p in fake_samples(s)]
    assert len(two) == len(one) == len(ref)
    for (x2, t2), (x1, t1), (xr, tr) in zip(two, one, ref):
        assert np.array_equal(x2.numpy(), xr.numpy()) and np.array_equal(t2.numpy(), tr.numpy())
        assert np.array_equal(x1.numpy(), xr.numpy()) and np.array_equal(t1.numpy(), tr.numpy())
