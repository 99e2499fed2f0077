"""Sharding over ranks (one process per GPU) and combining the results.

One experiment (the single-run forms): every rank runs the same experiment with a disjoint
range of chain ids (``chain_offset = rank * chains``), so the chains of all ranks are
independent draws of the same Markov process and the estimate is their sum. The one exchange
step combines the per-rank results: log10 sums by log-sum-exp, absolute standard errors in
quadrature (the ranks' chains are independent), counts by addition. It moves 6 doubles per
rank.

A batch (the receiver / pixel grids): experiments are independent, so the ranks split the
batch by experiment (``partition_experiments``: each rank takes a contiguous range holding its
share of the work, balanced by paths x segments) and run their own sub-batch with the
experiments' own Philox stream ids and bootstrap seeds (those of the full batch, so that the
result of an experiment does not depend on the number of ranks); ``gather_partitioned`` then
puts every experiment's result on every rank in one all-gather of n x 7 doubles.
"""
from __future__ import annotations

import math
from typing import Sequence

FIELDS = ("log10_weight", "rel_std_error", "total_paths", "failed_paths", "clamped_curvatures", "num_chains")


def combine(parts: Sequence[Sequence[float]]) -> dict:
    """Combine per-rank tuples ordered as FIELDS (the normaliser is a common factor)."""
    logs = [p[0] for p in parts if p[0] > -math.inf]
    if not logs:
        m = -math.inf
        total = 0.0
    else:
        m = max(logs)
        total = sum(10.0 ** (p[0] - m) for p in parts if p[0] > -math.inf)
    var = 0.0
    for p in parts:
        if p[0] > -math.inf and not math.isnan(p[1]):
            var += (p[1] * 10.0 ** (p[0] - m)) ** 2
    return {
        "log10_weight": m + math.log10(total) if total > 0 else -math.inf,
        "rel_std_error": math.sqrt(var) / total if total > 0 else math.nan,
        "total_paths": int(sum(p[2] for p in parts)),
        "failed_paths": int(sum(p[3] for p in parts)),
        "clamped_curvatures": int(sum(p[4] for p in parts)),
        "num_chains": int(sum(p[5] for p in parts)),
    }


def local_tuple(result) -> list:
    return [float(getattr(result, f)) for f in FIELDS]


def all_combine(result, group=None, device=None) -> dict:
    """All-gather the per-rank result tuples over torch.distributed and combine them."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(local_tuple(result), dtype=torch.float64, device=device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    return combine([p.tolist() for p in parts])


def all_combine_batch(results, group=None, device=None) -> list:
    """The batched form: every rank ran the same experiments (twisty_run_batch) on its own chain
    range; one all-gather of an n x 6 tensor, then experiment i combines the ranks' i-th tuples.
    Every rank must pass the same number of results."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([local_tuple(r) for r in results], dtype=torch.float64, device=device).reshape(-1, len(FIELDS))
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    rows = [p.tolist() for p in parts]
    return [combine([rows[r][i] for r in range(len(rows))]) for i in range(t.shape[0])]


def partition_experiments(experiments, rank: int, world: int) -> list:
    """Indices of the experiments rank `rank` of `world` runs: a contiguous range, cut where the
    running cost (paths x segments) crosses rank / world of the total, so every rank's share is
    within one experiment's cost of total / world. Contiguous, so that the sub-batch keeps the
    full batch's stream ids and bootstrap seeds: run it with experiment_id and bootstrap_seed
    raised by its first index (twisty_run_batch numbers experiments from those)."""
    cost = [float(x.paths) * float(x.num_segments) for x in experiments]
    total = sum(cost)

    def cut(r):
        if r <= 0:
            return 0
        if r >= world:
            return len(cost)
        target = total * r / world
        acc = 0.0
        for i, c in enumerate(cost):
            if acc + 0.5 * c > target:
                return i
            acc += c
        return len(cost)

    return list(range(cut(rank), cut(rank + 1)))


def gather_partitioned(results, indices, n: int, group=None, device=None) -> list:
    """Every experiment's result tuple (FIELDS) on every rank: each rank passes the results of
    the experiments it ran (`indices`, from partition_experiments) and receives a list of n
    dicts, experiment i's from the rank that ran it."""
    import torch
    import torch.distributed as dist
    t = torch.full((n, len(FIELDS) + 1), float("nan"), dtype=torch.float64, device=device)
    for i, r in zip(indices, results):
        t[i, :len(FIELDS)] = torch.tensor(local_tuple(r), dtype=torch.float64)
        t[i, len(FIELDS)] = 1.0   # row present
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    out = [None] * n
    for p in parts:
        rows = p.tolist()
        for i in range(n):
            if rows[i][len(FIELDS)] == 1.0:
                if out[i] is not None:
                    raise RuntimeError(f"experiment {i} ran on two ranks")
                out[i] = combine([rows[i][:len(FIELDS)]])
    missing = [i for i in range(n) if out[i] is None]
    if missing:
        raise RuntimeError(f"experiments {missing[:8]} ran on no rank")
    return out
