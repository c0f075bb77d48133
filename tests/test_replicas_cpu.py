"""The multi-GPU form of the bench is independent replicas: the collective carries only the
barrier and the max over ranks.  Two gloo ranks on the CPU check that path (no GPU)."""
import multiprocessing as mp
import os
import socket

import pytest


def _free_port():
    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def _rank(rank, world, port, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    ranks = bench.Ranks(collective=True, backend="gloo")
    ranks.barrier()
    slowest = ranks.max(100.0 + 50.0 * rank)       # per-rank device times of the timed region (ms)
    ranks.barrier()
    queue.put((rank, slowest, bench.replica_throughput(ranks.world, 10, slowest)))
    ranks.close()


def test_two_gloo_replicas_agree_on_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks see the slowest rank's time; throughput = all ranks' steps over that time
    assert [r[1] for r in results] == [150.0, 150.0]
    assert results[0][2] == pytest.approx(2 * 10 / 0.150)


def test_single_process_has_no_collective():
    import bench
    ranks = bench.Ranks(collective=True)
    assert ranks.dist is None and ranks.max(3.5) == 3.5
    assert bench.replica_throughput(1, 5, 500.0) == pytest.approx(10.0)
