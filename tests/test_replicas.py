"""Replica bookkeeping for runs on N GPUs, checked with world-size-2 gloo
process groups on the CPU: each rank routes its own copy of a small design
(with the CPU oracle, as a stand-in for the device route), the replicas'
digests agree, the step time is the maximum over ranks and the whole-job
rate counts both ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out, corrupt_rank):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import iitmglobalrouter_b200 as gr
        import oracle
        from iitmglobalrouter_b200 import replicas

        d = gr.Design.generate(1, seed=2, n_nets=300)
        dims = d.dims
        ofs, pins = d.nets()
        bofs, ids = d.batch(4)
        g = oracle.Grid(dims["X"], dims["Y"], dims["Z"], d.caps())
        rc, mst, mp_ = g.route_batches(ofs, pins, bofs, ids, nthreads=1)
        assert rc == 0
        if rank == corrupt_rank:  # a replica whose result differs
            mst = mst.copy()
            mst[0] ^= 1
        ok = replicas.replicas_agree(replicas.digest(mst, mp_, g.demand()), dist)
        t = replicas.max_over_ranks(0.25 * (rank + 1), dist)
        rate = replicas.whole_job_rate(dims["n_nets"], t, dist.get_world_size())
        out.put((rank, ok, t, rate, dims["n_nets"]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _run(corrupt_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q, corrupt_rank)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(res)


def test_replicas_agree_and_timing_is_max_over_ranks():
    res = _run(corrupt_rank=-1)
    for rank, ok, t, rate, n in res:
        assert ok
        assert t == pytest.approx(0.5)
        assert rate == pytest.approx(2 * n / 0.5)


def test_replica_mismatch_is_detected_on_every_rank():
    res = _run(corrupt_rank=1)
    assert [ok for _, ok, *_ in res] == [False, False]


def test_single_process_helpers():
    from iitmglobalrouter_b200 import replicas

    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.replicas_agree(7)
    assert replicas.whole_job_rate(10, 2.0, 4) == 20.0
    assert replicas.digest(np.arange(3)) != replicas.digest(np.arange(4))
    with pytest.raises(ValueError):
        replicas.whole_job_rate(1, 0.0, 1)
