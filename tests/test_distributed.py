"""CPU: multi-process sharding and timing reductions over gloo with world size 2 (the same code
path the benchmark uses over NCCL, one process per GPU)."""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = torch.multiprocessing


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, queue):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from pycorrectedemissionct_b200 import distributed as d

    assert d.init("gloo", timeout_s=60)
    mine = d.shard(10, rank, world)
    elapsed = 1.0 + rank  # rank 1 is the slow one
    t_max = d.max_over_ranks(elapsed)
    n_total = d.sum_over_ranks(len(mine))
    d.barrier()
    queue.put((rank, list(mine), t_max, n_total))
    d.finalize()


def test_two_rank_sharding_and_max_timing():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == [0, 1, 2, 3, 4] and out[1][1] == [5, 6, 7, 8, 9]
    assert all(o[2] == 2.0 for o in out)  # max over ranks
    assert all(o[3] == 10 for o in out)   # every slice owned exactly once


def test_shard_partition_properties():
    from pycorrectedemissionct_b200.distributed import shard

    for total in (0, 1, 7, 64, 513):
        for world in (1, 2, 3, 8):
            parts = [shard(total, r, world) for r in range(world)]
            flat = [i for p in parts for i in p]
            assert flat == list(range(total))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(4, 2, 2)
