"""The N>1 path of bench.py on CPU: one process per rank over gloo (world
size 2).  The path shards as independent replicas (no data-path collective);
the only cross-rank steps are the barrier and the max over ranks of the
timings, which decide the whole-job throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    # rank 1 is the slow replica: its timings must win
    local = [1000.0 + 500.0 * rank, 2000.0 - 100.0 * rank, 0.05 * (rank + 1), 0.06]
    dist.barrier()
    m = bench.max_over_ranks(local, dist)
    v = bench.aggregate_throughput(3, world, m[0])
    q.put((rank, m, v))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, v in out:
        assert m == [1500.0, 2000.0, 0.1, 0.06]
        assert v == pytest.approx(3 * 2 / 1.5)


def test_single_process_is_identity():
    import bench
    assert bench.max_over_ranks([1.0, 2.0]) == [1.0, 2.0]
    assert bench.aggregate_throughput(5, 1, 1000.0) == pytest.approx(5.0)
