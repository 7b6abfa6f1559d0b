"""The N > 1 host path of bench.py on CPU: two gloo ranks, one replica each (weak scaling, no
data-path collective). Every rank must agree on the slowest rank's time, and the whole-job rate is
world x steps / that time."""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    d = bench.Dist(world, backend="gloo")
    try:
        seconds = 1.0 + rank  # rank 1 is the slower one
        d.barrier()
        slowest = d.max(seconds)
        q.put((rank, slowest, bench.aggregate_rate(10, d.world, slowest)))
    finally:
        d.close()


def test_two_rank_replicas_time_by_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [2.0, 2.0]
    assert [g[2] for g in got] == [10.0, 10.0]  # 2 ranks x 10 steps / 2 s


def test_single_process_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    d = bench.Dist(1)
    assert d.pg is None and d.max(3.5) == 3.5
    assert bench.aggregate_rate(100, 1, 0.5) == 200.0
