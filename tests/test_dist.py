"""Multi-rank logic on CPU (gloo, world size 2): profile sharding covers
every profile exactly once and the max-over-ranks timing reduction."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from lblrtm_b200 import dist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _batch_worker(rank, world, port, costs, q):
    """The batched driver's sharding on CPU: each rank 'computes' its shard
    (a stub returning the shard's cost as its elapsed time and the profiles
    it did), times are reduced by max, summaries gathered."""
    import torch.distributed as td
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world)

    def work(idx):
        return float(sum(costs[i] for i in idx)), sorted(idx)

    mine, ms, got = dist.sharded_run(costs, work, rank, world, gather=True)
    q.put((rank, mine, ms, got))
    td.barrier()
    td.destroy_process_group()


def test_sharded_batch_driver_gloo():
    costs = [float(30 + (13 * i) % 61) * 1e5 for i in range(256)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    loads = [sum(costs[i] for i in r[1]) for r in res]
    for rank, mine, ms, got in res:
        assert ms == max(loads)                      # max over ranks
        assert [sorted(g) for g in got] == [sorted(r[1]) for r in res]
    assert sorted(i for r in res for i in r[1]) == list(range(256))


def test_sharded_run_single_process():
    mine, ms, got = dist.sharded_run([3.0, 1.0], lambda idx: (7.0, idx))
    assert mine == [0, 1] and ms == 7.0 and got == [[0, 1]]


def _worker(rank, world, port, costs, q):
    import torch
    import torch.distributed as td
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world)
    mine = dist.shard(costs, rank, world)
    got = [None] * world
    td.all_gather_object(got, mine)
    t = dist.max_over_ranks(1.5 + rank)
    q.put((rank, got, t))
    td.barrier()
    td.destroy_process_group()


def test_shard_and_max_over_ranks_gloo():
    costs = [float(30 + (7 * i) % 61) for i in range(256)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, t in res:
        assert t == pytest.approx(2.5)
        flat = sorted(i for s in got for i in s)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in s) for s in got]
        assert abs(loads[0] - loads[1]) <= max(costs)


def test_shard_single_rank():
    assert dist.shard([3.0, 1.0, 2.0], 0, 1) == [0, 1, 2]
