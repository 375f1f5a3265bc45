"""Host logic of running the pair sweep on several GPUs, one process per GPU.

Pairs are independent, so ranks never exchange data on the path: each rank either runs its own batch
(weak scaling, what bench.py measures) or takes a share of one cost-ordered batch, dealt so that every
rank holds the same mix of pair sizes (strong scaling).  The only collectives are host-side: the
slowest rank's time, and one gather of the per-rank results.
"""
from __future__ import annotations

import numpy as np


def pair_costs(tri_off, pair_mesh) -> np.ndarray:
    """nA * nB per pair: the triangle-pair count the reference's loop tests (src/main.cpp:2123-2145)."""
    n = np.diff(np.asarray(tri_off, np.int64))
    pm = np.asarray(pair_mesh).reshape(-1, 2)
    return n[pm[:, 0]] * n[pm[:, 1]]


def cost_balanced_ranges(costs, world: int) -> list[tuple[int, int]]:
    """Split pairs 0..n-1, in the order given, into `world` contiguous ranges of nearly equal total cost
    (each boundary at the first pair whose cumulative cost reaches r/world of the total)."""
    c = np.asarray(costs, np.float64)
    n = len(c)
    if world <= 1 or n == 0:
        return [(0, n)] + [(n, n)] * max(world - 1, 0)
    cum = np.cumsum(c)
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, total * r / world, side="left")) + 1 if total > 0 else n * r // world)
    cuts = [min(max(x, 0), n) for x in cuts] + [n]
    for i in range(1, len(cuts)):
        cuts[i] = max(cuts[i], cuts[i - 1])
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def rank_seed(base: int, rank: int) -> int:
    """Seed of a rank's own batch in the weak-scaling run (every rank a different batch)."""
    return int(base) + 1 + int(rank)


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over the ranks of the default process group (the time of the slowest rank);
    the value itself when no group is initialised."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_counts(count: int, device=None) -> list[int]:
    """Every rank's count (for example its contacts), on every rank."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [int(count)]
    t = torch.tensor([int(count)], dtype=torch.int64, device=device)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return [int(x.item()) for x in out]


def dealt(n: int, world: int) -> np.ndarray:
    """Rank of each position 0..n-1 of a descending cost order, dealt serpentine-wise: 0, 1, .., W-1,
    W-1, .., 0, 0, 1, ...  Every rank receives one pair of each run of W similar pairs, and the reversal
    of every other run cancels the first-dealt rank's edge within a run."""
    if world <= 1:
        return np.zeros(n, np.int64)
    i = np.arange(n, dtype=np.int64)
    run, pos = i // world, i % world
    return np.where(run % 2 == 0, pos, world - 1 - pos)


def strong_shards(tri_off, pair_mesh, world: int, mode: str = "dealt", costs=None) -> list[np.ndarray]:
    """Pair indices of each rank for one batch spread over `world` ranks, each rank's pairs in the work
    queue's cost order (descending, ties by index).

    mode "dealt": the cost-ordered pairs dealt to the ranks serpentine-wise, so that every rank holds the
    same mix of pair sizes.  Its balance does not depend on how real time grows with the cost: the certificate
    and culls leave about 1 % of nA * nB to test and the rebuild is linear in segments, so two ranges of
    equal nA * nB can differ severalfold in time, while two dealt shards of the same mix cannot.  It also
    keeps the largest pairs apart, one per rank, instead of leaving a few of them to one rank's SMs.
    mode "ranges": contiguous ranges of equal total cost (the cost-balanced cut).
    costs: per-pair costs to order by (for example a previous call's segment counts); nA * nB when None."""
    c = pair_costs(tri_off, pair_mesh) if costs is None else np.asarray(costs, np.float64)
    order = np.argsort(-c, kind="stable")
    if mode == "ranges":
        return [order[a:b] for a, b in cost_balanced_ranges(c[order], world)]
    if mode != "dealt":
        raise ValueError(f"unknown shard mode {mode!r}")
    r = dealt(len(order), world)
    return [order[r == k] for k in range(max(world, 1))]


def gather_rows(t, device=None) -> list:
    """Every rank's row block (a tensor of any length along dim 0, same trailing shape and dtype), on
    every rank: one gather of the lengths, then one of the blocks padded to the longest."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [t]
    n = gather_counts(int(t.shape[0]), device)
    m = max(max(n), 1)
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[: t.shape[0]] = t
    out = [torch.empty_like(pad) for _ in n]
    dist.all_gather(out, pad)
    return [o[:k] for o, k in zip(out, n)]
