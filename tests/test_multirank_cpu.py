"""Multi-rank host logic on CPU (gloo, world size 2): the bench's max-over-ranks timing
reduction and the deterministic longest-first sharding of ensemble variants across ranks."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v = bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu")
        parts = bench.partition_by_cells([5, 9, 3, 7, 7, 1], world)
        out.put((rank, v, parts[rank]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_sharding_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    shards = [r[2] for r in res]
    assert sorted(i for s in shards for i in s) == list(range(6))
    loads = [sum([5, 9, 3, 7, 7, 1][i] for i in s) for s in shards]
    assert abs(loads[0] - loads[1]) <= 2


def test_partition_single_rank_and_identity_reduce():
    assert bench.partition_by_cells([3, 1, 2], 1) == [[0, 2, 1]]
    assert bench.partition_by_cells([4, 4], 3) == [[0], [1], []]
    assert bench.max_over_ranks(3.5) == 3.5
