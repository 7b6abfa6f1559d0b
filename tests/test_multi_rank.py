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


def _label_rank(rank: int, world: int, port: int, shard_dir: str, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import numpy as np
    import torch.distributed as dist

    from univeral_3d_reconstruction_system_b200.warmstart import generate_labels
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        done = []

        def label_fn(seed):
            done.append(seed)
            rows = 3 + seed % 4
            return np.full((rows, 134), seed, np.float32), np.full((rows, 11), -seed, np.float32)

        got = generate_labels(range(10, 17), label_fn, shard_dir, rank, world, dist.barrier, log=lambda *m: None)
        q.put((rank, done, None if got is None else (got[0][:, 0].tolist(), got[1][:, 0].tolist())))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_the_label_scenes(tmp_path):
    """Warm-start label generation with two ranks: each labels every other scene (no data-path
    collective); rank 0 then holds all rows in seed order."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_label_rank, args=(r, 2, port, str(tmp_path), q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict((r, (done, res)) for r, done, res in (q.get(timeout=5) for _ in range(2)))
    assert got[0][0] == [10, 12, 14, 16] and got[1][0] == [11, 13, 15]
    assert got[1][1] is None
    x0, t0 = got[0][1]
    expect = [float(s) for s in range(10, 17) for _ in range(3 + s % 4)]
    assert x0 == expect and t0 == [-v for v in expect]


def _batched_rank(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    from univeral_3d_reconstruction_system_b200.scenes import batched_specs
    d = bench.Dist(world, backend="gloo")
    try:
        specs = batched_specs(0, 16)
        mine = bench.batched_shard(len(specs), d.world, d.rank)
        iters = sum(specs[k].iterations for k in mine)
        # Per-rank device times and PSNR differences as a rank would measure them.
        got = bench.combine_batched(d, iters, 100.0 + 10 * rank, 300.0 - 50 * rank, 0.01 * rank)
        q.put((rank, mine, iters, got))
    finally:
        d.close()


def test_two_ranks_split_the_batched_scenes():
    """The batched leg with two gloo ranks: rank r trains scenes r, r + 2, ... (disjoint, covering all
    16), and every rank ends with the whole job's iteration count and the slowest rank's times."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batched_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict((r, rest) for r, *rest in (q.get(timeout=5) for _ in range(2)))
    assert got[0][0] == list(range(0, 16, 2)) and got[1][0] == list(range(1, 16, 2))
    total = got[0][1] + got[1][1]
    for r in (0, 1):
        assert got[r][2] == (total, 110.0, 300.0, 0.01)
