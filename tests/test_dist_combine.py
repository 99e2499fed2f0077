"""The cross-rank exchange step (twisty_b200.dist) on CPU with gloo, world size 2."""
import math
import os
import socket

import pytest
import torch.multiprocessing as mp

from twisty_b200 import dist as D


class R:
    def __init__(self, **kw):
        self.__dict__.update(kw)


PARTS = [
    dict(log10_weight=-290.25, rel_std_error=0.01, total_paths=1000, failed_paths=1, clamped_curvatures=3, num_chains=10),
    dict(log10_weight=-290.75, rel_std_error=0.02, total_paths=900, failed_paths=0, clamped_curvatures=1, num_chains=9),
]


def test_combine_math():
    c = D.combine([D.local_tuple(R(**p)) for p in PARTS])
    a, b = 10 ** 0.0, 10 ** -0.5   # relative to the larger
    assert c["log10_weight"] == pytest.approx(-290.25 + math.log10(a + b), abs=1e-12)
    assert c["rel_std_error"] == pytest.approx(math.hypot(0.01 * a, 0.02 * b) / (a + b), rel=1e-12)
    assert (c["total_paths"], c["failed_paths"], c["clamped_curvatures"], c["num_chains"]) == (1900, 1, 4, 19)
    # a rank with no valid path contributes nothing but its counts
    e = D.combine([D.local_tuple(R(**PARTS[0])),
                   [-math.inf, math.nan, 0, 5, 0, 4]])
    assert e["log10_weight"] == pytest.approx(-290.25) and e["failed_paths"] == 6


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, D.all_combine(R(**PARTS[rank]))))
    finally:
        dist.destroy_process_group()


def test_all_combine_gloo_two_ranks():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = D.combine([D.local_tuple(R(**p)) for p in PARTS])
    assert out[0] == out[1] == ref


BATCH = [[dict(PARTS[0]), dict(PARTS[1], log10_weight=-12.5)],
         [dict(PARTS[1]), dict(PARTS[0], log10_weight=-12.0, rel_std_error=0.03)]]   # [rank][experiment]


def _batch_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, D.all_combine_batch([R(**e) for e in BATCH[rank]])))
    finally:
        dist.destroy_process_group()


def test_all_combine_batch_gloo_two_ranks():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_batch_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for i in range(2):
        ref = D.combine([D.local_tuple(R(**BATCH[r][i])) for r in range(2)])
        assert out[0][i] == out[1][i] == ref


class X:
    def __init__(self, paths, num_segments):
        self.paths, self.num_segments = paths, num_segments


def test_partition_balances_work_and_covers_every_experiment():
    rng = __import__("numpy").random.default_rng(3)
    exps = [X(int(rng.integers(1000, 100000)), int(rng.integers(16, 1025))) for _ in range(257)]
    for world in (1, 2, 3, 8):
        parts = [D.partition_experiments(exps, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(exps)))
        for p in parts:
            assert p == list(range(p[0], p[0] + len(p))) if p else True   # contiguous
        loads = [sum(exps[i].paths * exps[i].num_segments for i in p) for p in parts]
        total = sum(loads)
        assert all(abs(ld - total / world) <= max(x.paths * x.num_segments for x in exps) for ld in loads)
        assert parts == [D.partition_experiments(exps, r, world) for r in range(world)]   # deterministic


# experiment i's result: fields derived from i so that every rank can check every row
def _result_of(i):
    return R(log10_weight=-10.0 - i, rel_std_error=0.01 * (i + 1), total_paths=1000 + i, failed_paths=i % 3,
             clamped_curvatures=i % 5, num_chains=8 + i)


def _partition_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        exps = [X(1000 * (1 + i % 7), 16 + 37 * i % 1000) for i in range(21)]
        mine = D.partition_experiments(exps, rank, world)
        q.put((rank, mine, D.gather_partitioned([_result_of(i) for i in mine], mine, len(exps))))
    finally:
        dist.destroy_process_group()


def test_partitioned_batch_gathers_on_every_rank_gloo_two_ranks():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_partition_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        rank, mine, out = q.get(timeout=120)
        got[rank] = (mine, out)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(got[0][0] + got[1][0]) == list(range(21)) and got[0][0] and got[1][0]
    assert got[0][1] == got[1][1]
    for i, row in enumerate(got[0][1]):
        assert row == D.combine([D.local_tuple(_result_of(i))])
