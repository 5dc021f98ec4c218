"""Multi-GPU timing of bench.py is replicas only: each rank runs its own grid and the job
reports the max device time over ranks.  Checked here with 2 gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    w, r, _ = bench.dist_setup(use_cuda=False)
    assert (w, r) == (world, rank)
    ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
    bench.dist_barrier(w)
    got = bench.dist_max(ms, w, use_cuda=False)
    out.put((rank, got))
    import torch.distributed as dist

    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 15.0, 1: 15.0}


def test_single_process_is_world_one(monkeypatch):
    import bench

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    assert bench.dist_setup(use_cuda=False)[0] == 1
    assert bench.dist_max(3.0, 1, False) == 3.0
