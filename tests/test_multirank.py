"""The multi-GPU path of bench.py (replicas, one process per GPU) on CPU:
two gloo ranks exchange their step times, each takes the maximum, and each
rank solves its own graph (seed = rank).  No GPU is used."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    dist = bench.dist_init(world, rank, backend="gloo")
    got = bench.ranks_max(10.0 * (rank + 1), dist, device="cpu")
    G = bench.graph_for(rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got, G.n, int(G.src[:50].sum())))


def test_two_gloo_ranks_max_and_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [20.0, 20.0]          # max over ranks, on every rank
    assert out[0][2] == out[1][2] == 50000             # same workload shape
    assert out[0][3] != out[1][3]                      # different graph per rank
    assert bench_single() == 7.5


def bench_single():
    import bench
    return bench.ranks_max(7.5, None)
