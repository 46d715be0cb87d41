"""Serving loop (slcs_server_*): results against the oracle, identity of results alone and in a mix,
admission under a device-memory budget with eviction of resident braids, queries on resident braids."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pair(rng, m, n):
    a = rng.integers(0, 4, m).astype(np.uint8)
    b = rng.integers(0, 4, n).astype(np.uint8)
    return a, b


def _expected(a, b, q):
    kind, i, j = q
    if kind == 0:
        return O.lcs_dp(a, b)
    if kind == 1:
        return O.lcs_dp(a, b[i:j])
    if kind == 2:
        return O.lcs_dp(a[:i], b[j:])
    if kind == 3:
        return O.lcs_dp(a[i:], b[:j])
    if kind == 4:
        return O.lcs_dp(a[i:j], b)
    raise ValueError(kind)


def _random_query(rng, m, n):
    kind = int(rng.integers(0, 5))
    if kind == 0:
        return (0, 0, 0)
    if kind in (1,):
        i = int(rng.integers(0, n + 1)); j = int(rng.integers(i, n + 1))
        return (1, i, j)
    if kind in (2, 3):
        return (kind, int(rng.integers(0, m + 1)), int(rng.integers(0, n + 1)))
    i = int(rng.integers(0, m + 1)); j = int(rng.integers(i, m + 1))
    return (4, i, j)


def test_server_scores_and_braids_match_oracle(engine):
    import semilocal_b200 as S
    rng = np.random.default_rng(11)
    reqs = []
    for m, n in [(1, 1), (0, 5), (7, 0), (33, 700), (700, 33), (1000, 1000), (1500, 900), (64, 64), (2047, 2049)]:
        a, b = _pair(rng, m, n)
        reqs.append((a, b, _random_query(rng, m, n)))
    with S.Server(small_streams=2, big_cells=1_000_000) as srv:
        tickets = [srv.submit(a, b, q) for a, b, q in reqs]
        got = srv.wait_all(tickets)
        for t, (a, b, q) in zip(tickets, reqs):
            r = got[t]
            assert r["status"] == 0, r
            assert r["score"] == _expected(a, b, q), (len(a), len(b), q)
            assert r["t_submit"] <= r["t_admit"] <= r["t_done"]
            if len(a) and len(b):
                assert np.array_equal(srv.braid(t), O.comb_antidiag(a, b)), (len(a), len(b))
            else:
                assert np.array_equal(srv.braid(t), np.arange(len(a) + len(b)))


def test_server_results_same_alone_and_in_mix(engine):
    """Each request's answer and braid are bit-identical when it runs alone and inside a mixed load (small
    batches on several streams overlapping a big request on its own stream)."""
    import semilocal_b200 as S
    rng = np.random.default_rng(12)
    sizes = [(3000, 2800)] + [(int(x), int(x) + int(d)) for x, d in zip(rng.integers(50, 1500, 40), rng.integers(-20, 20, 40))]
    reqs = []
    for m, n in sizes:
        a, b = _pair(rng, m, max(n, 1))
        reqs.append((a, b, _random_query(rng, len(a), len(b))))
    alone = []
    with S.Server(small_streams=3, big_cells=4_000_000) as srv:
        for a, b, q in reqs:
            t = srv.submit(a, b, q)
            r = srv.wait_all([t])[t]
            alone.append((r["status"], r["score"], srv.braid(t)))
    with S.Server(small_streams=3, big_cells=4_000_000, max_batch=8) as srv:
        tickets = [srv.submit(a, b, q) for a, b, q in reqs]
        got = srv.wait_all(tickets)
        st = srv.stats()
        assert st["launches"] >= 3          # the mix really was split over several launches
        for t, (status, score, braid) in zip(tickets, alone):
            assert got[t]["status"] == status == 0
            assert got[t]["score"] == score
            assert np.array_equal(srv.braid(t), braid)


def test_server_admission_budget_and_eviction(engine):
    import semilocal_b200 as S
    rng = np.random.default_rng(13)
    reqs = [_pair(rng, 2000, 2000) for _ in range(12)]
    per_req = 2000 * 2 * (1 + 4 + 4) + 4096
    budget = 3 * per_req
    with S.Server(mem_budget=budget, small_streams=2, max_batch=2) as srv:
        tickets = [srv.submit(a, b) for a, b in reqs]
        got = srv.wait_all(tickets)
        for t, (a, b) in zip(tickets, reqs):
            assert got[t]["status"] == 0
            assert got[t]["score"] == O.lcs_dp(a, b)
        st = srv.stats()
        assert st["peak_bytes"] <= budget
        assert st["evicted"] > 0                       # resident braids made room for later requests
        assert st["resident_bytes"] <= budget
        # the oldest braids were evicted, the newest is still resident and answers queries
        with pytest.raises(S.SlcsError):
            srv.query(tickets[0], [(0, 0, 0)])
        a, b = reqs[-1]
        assert srv.query(tickets[-1], [(0, 0, 0)])[0] == O.lcs_dp(a, b)


def test_server_resident_queries_and_release(engine):
    import semilocal_b200 as S
    rng = np.random.default_rng(14)
    a, b = _pair(rng, 900, 1100)
    with S.Server() as srv:
        t = srv.submit(a, b, (2, 300, 400))
        r = srv.wait_all([t])[t]
        assert r["score"] == _expected(a, b, (2, 300, 400))
        qs = [_random_query(rng, len(a), len(b)) for _ in range(20)]
        out = srv.query(t, qs)
        assert [int(x) for x in out] == [_expected(a, b, q) for q in qs]
        win = srv.window_scores(t, 150)
        assert len(win) == len(b) - 150 + 1
        for s0 in (0, 1, 500, len(b) - 150):
            assert int(win[s0]) == O.lcs_dp(a, b[s0:s0 + 150])
        srv.release(t)
        with pytest.raises(S.SlcsError):
            srv.query(t, [(0, 0, 0)])
        assert srv.stats()["resident"] == 0


def test_server_rejects_bad_requests(engine):
    import semilocal_b200 as S
    a = np.zeros(100, np.uint8)
    with S.Server(mem_budget=1 << 20) as srv:
        with pytest.raises(S.SlcsError) as e:
            srv.submit(a, a, (1, 5, 200))            # substring end beyond n
        assert e.value.code == 1
        big = np.zeros(200_000, np.uint8)
        with pytest.raises(S.SlcsError) as e:
            srv.submit(big, big)                     # alone larger than the budget
        assert e.value.code == 3
    with S.Server(max_pending=1) as srv:
        codes = []
        for _ in range(64):
            try:
                srv.submit(np.zeros(4000, np.uint8), np.zeros(4000, np.uint8))
            except S.SlcsError as e:
                codes.append(e.code)
        assert not codes or set(codes) == {8}        # queue full -> SLCS_ERR_BUSY, never anything else
