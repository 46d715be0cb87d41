"""The N > 1 host path on CPU: cost-balanced pair sharding, the max-over-ranks step time and the gathering
of per-pair scores, run as two gloo ranks (no GPU, no data-path collective)."""
import os
import socket

import numpy as np
import pytest

from semilocal_b200.shard import gather_scores, max_over_ranks, shard_pairs


def test_shard_pairs_covers_every_pair_once_and_balances():
    rng = np.random.default_rng(0)
    lens = np.exp(rng.uniform(np.log(256), np.log(65536), 4096)).astype(np.int64)
    costs = lens * lens
    for world in (1, 2, 3, 4, 8):
        shards = shard_pairs(costs, world)
        allidx = sorted(i for s in shards for i in s)
        assert allidx == list(range(len(costs)))
        loads = [int(costs[np.array(s, dtype=np.int64)].sum()) for s in shards]
        # LPT greedy: no rank exceeds the mean by more than the largest single pair
        assert max(loads) - sum(loads) / world <= costs.max()
    assert shard_pairs([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard_pairs([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard_pairs(costs, world)[rank]
        # a stand-in per-pair result: the pair's index and cost
        scores = [(i, int(costs[i])) for i in mine]
        step_ms = 10.0 + rank                           # rank 1 is the slow one
        t = max_over_ranks(step_ms, dist, "cpu")
        g = gather_scores(scores, dist, dst=0)
        q.put((rank, t, g, len(mine)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_time_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    costs = [int(x) for x in np.random.default_rng(1).integers(1, 10**6, 101)]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, t, g, n = q.get(timeout=120)
        out[rank] = (t, g, n)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 11.0                 # the job's step time is the slowest rank's
    assert out[1][1] is None
    gathered = out[0][1]
    idx = sorted(i for part in gathered for i, _ in part)
    assert idx == list(range(len(costs)))                 # every pair's result reached rank 0 exactly once
    assert out[0][2] + out[1][2] == len(costs)


def _fixed_shard_rank(rank, world, port, q):
    """One rank of bench.py --shard fixed on the host: the whole seed-5 batch, this rank's cost shard of it."""
    import datetime

    import torch.distributed as dist

    from semilocal_b200 import gen
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        costs = [len(a) * len(b) for a, b in gen.batch_pairs(4096, 256, 65536, seed=5)]   # as bench.py does
        mine = shard_pairs(costs, world)[rank]
        cells = sum(costs[i] for i in mine)
        g = gather_scores([(i, costs[i]) for i in mine], dist, dst=0)
        q.put((rank, cells, g))
    finally:
        dist.destroy_process_group()


def test_fixed_batch_shards_cover_the_batch_on_two_gloo_ranks():
    """Strong scaling of one 4096-pair batch over two ranks: the ranks' shards are disjoint, their union is the
    whole batch, and their cells differ by less than the largest pair."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fixed_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, cells, g = q.get(timeout=120)
        out[rank] = (cells, g)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    idx = [i for part in out[0][1] for i, _ in part]
    assert sorted(idx) == list(range(4096)) and len(set(idx)) == 4096
    costs = dict((i, c) for part in out[0][1] for i, c in part)
    assert abs(out[0][0] - out[1][0]) <= max(costs.values())
