"""bench.py's multi-GPU form: one independent replica per rank (the north star fixes one GPU and
no sharding), whole-job throughput = every rank's queries over the slowest rank's time. The rank
aggregation runs here on two gloo ranks on the CPU."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch

    torch.distributed.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    slowest = bench.max_over_ranks(1.0 + rank, world, "cpu")       # rank r timed 1 + r seconds
    qps = bench.replica_qps(1000, 2.0 + 2.0 * rank, world, "cpu")  # 1000 queries per rank
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()
    out.put((rank, slowest, qps))


@pytest.mark.timeout(180)
def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.0, 2.0]
    assert [r[2] for r in res] == [2 * 1000 / 4.0] * 2


def test_one_rank_is_its_own_time():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.replica_qps(500, 2.0, 1, "cpu") == 250.0
