"""Host logic of the multi-GPU sweep on two gloo ranks (CPU): the slowest rank's time and the counts
reach every rank, each rank draws a different batch, and the strong-scaling split covers every pair
once with balanced triangle-test work."""
import os

import numpy as np
import pytest


def _worker(rank, world, port, q):
    import torch.distributed as dist

    import torch

    from zdemx.replicas import gather_counts, gather_rows, max_over_ranks, rank_seed

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = max_over_ranks(1.5 + rank)
        counts = gather_counts(10 * (rank + 1))
        # row blocks of different lengths
        rows = torch.arange(3 * (2 - rank) * 4, dtype=torch.float64).reshape(-1, 4) + 100 * rank
        got = [g.tolist() for g in gather_rows(rows)]
        q.put((rank, t, counts, rank_seed(7, rank), got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [2.5, 2.5]
    assert all(r[2] == [10, 20] for r in res)
    assert res[0][3] != res[1][3]
    want = [np.arange(24.0).reshape(6, 4).tolist(), (np.arange(12.0).reshape(3, 4) + 100).tolist()]
    assert all(r[4] == want for r in res)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_cost_balanced_ranges(world):
    from zdemx.replicas import cost_balanced_ranges, pair_costs

    rng = np.random.default_rng(world)
    tri_off = np.r_[0, np.cumsum(20 * 4 ** rng.integers(1, 5, size=40))]
    pm = rng.integers(0, 40, size=(5000, 2))
    costs = pair_costs(tri_off, pm)
    order = np.argsort(-costs, kind="stable")          # the cost order of the work queue
    ranges = cost_balanced_ranges(costs[order], world)
    assert len(ranges) == world and ranges[0][0] == 0 and ranges[-1][1] == len(pm)
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    loads = [costs[order][a:b].sum() for a, b in ranges]
    assert max(loads) - min(loads) <= 2 * costs.max() + 1


@pytest.mark.parametrize("mode", ["dealt", "ranges"])
@pytest.mark.parametrize("world", [1, 2, 4, 7])
def test_strong_shards_cover_every_pair_once(world, mode):
    from zdemx.replicas import pair_costs, strong_shards

    rng = np.random.default_rng(10 + world)
    tri_off = np.r_[0, np.cumsum(20 * 4 ** rng.integers(1, 5, size=64))]
    pm = rng.integers(0, 64, size=(3000, 2))
    shards = strong_shards(tri_off, pm, world, mode=mode)
    assert len(shards) == world
    allp = np.sort(np.concatenate(shards))
    assert np.array_equal(allp, np.arange(len(pm)))
    costs = pair_costs(tri_off, pm)
    for s in shards:  # each shard in the work queue's cost order
        assert np.all(np.diff(costs[s]) <= 0)
    loads = [costs[s].sum() for s in shards]
    assert max(loads) - min(loads) <= 2 * costs.max() + 1
    if mode == "dealt":
        # the same mix of sizes on every rank: of each distinct cost, counts differ by at most 2
        for v in np.unique(costs):
            cnt = [int(np.sum(costs[s] == v)) for s in shards]
            assert max(cnt) - min(cnt) <= 2
        assert max(len(s) for s in shards) - min(len(s) for s in shards) <= 1


def test_dealt_order_is_serpentine():
    from zdemx.replicas import dealt

    assert dealt(10, 3).tolist() == [0, 1, 2, 2, 1, 0, 0, 1, 2, 2]
    assert dealt(4, 1).tolist() == [0, 0, 0, 0]


def test_strong_shards_take_given_costs():
    from zdemx.replicas import strong_shards

    tri_off = np.array([0, 10, 20, 30])
    pm = np.zeros((6, 2), np.int64)        # equal nA * nB everywhere
    seg = np.array([5, 60, 1, 40, 9, 7])   # measured per-pair costs of an earlier call
    shards = strong_shards(tri_off, pm, 2, costs=seg)
    assert [s.tolist() for s in shards] == [[1, 5, 0], [3, 4, 2]]
    with pytest.raises(ValueError):
        strong_shards(tri_off, pm, 2, mode="other")
