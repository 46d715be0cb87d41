"""The ant passage's two forms, restated on the host and checked against the oracle's products.

The shared-memory steady-ant kernel combines two children either by walking c*(r) row by row (spans below 1024)
or by ranking the moving rows (spans from 1024 up): a row moves iff delta(r, x_r) puts its point on the wrong
side of c*(r), and the moving rows take their own columns in decreasing order.  Both forms are restated here on
the bottom-up tree of aligned power-of-two ranges the kernel uses (R:common/include/Permutations/
MongeMultuplicationStrategy.h:487-593 for the recursion, :244-323 for the ant passage it replaces) and must give
the reference's product exactly; the segment form of delta the kernel evaluates is checked against its
definition on the same nodes.
"""
import numpy as np
import pytest

from semilocal_b200 import gen


def delta(xs, hi, r, c):
    """delta(r, c) = #{hi points: row < r, col < c} - #{lo points: row >= r, col >= c}"""
    k = len(xs)
    return (sum(1 for q in range(r) if hi[q] and xs[q] < c)
            - sum(1 for q in range(r, k) if not hi[q] and xs[q] >= c))


def cstar(xs, hi, r):
    return next((c for c in range(len(xs) + 1) if delta(xs, hi, r, c) >= 0), len(xs) + 1)


def combine_walk(xs, hi):
    k = len(xs)
    res = xs.copy()
    for r in range(k):
        c = cstar(xs, hi, r)
        if 1 <= c <= k and ((xs[r] < c) if hi[r] else (xs[r] >= c)):
            res[r] = c - 1
    return res


def combine_rank(xs, hi):
    k = len(xs)
    moving = [r for r in range(k) if (delta(xs, hi, r, xs[r]) < 0) == bool(hi[r])]
    res = xs.copy()
    res[moving] = sorted(xs[moving], reverse=True)
    return res


def colind(ys, yhi, g, row):
    return (ys[g] < row) if yhi[g] else (ys[g] >= row)


def rowind(xs, hi, r, c):
    return (xs[r] < c) if hi[r] else (xs[r] >= c)


def segment_delta(xs, hi, ys, yhi, r, seg=32):
    """delta(r, x_r) from c* at the bottom of r's segment: #{g in [cb, x): colind(g, bot)} - #{r' in [r, bot):
    rowind(r', x)}"""
    k = len(xs)
    bot = min((r // seg + 1) * seg, k)
    cb = 0 if bot >= k else cstar(xs, hi, bot)
    x = xs[r]
    return (sum(1 for g in range(cb, x) if colind(ys, yhi, g, bot))
            - sum(1 for q in range(r, bot) if rowind(xs, hi, q, x)))


def multiply(pinv, q, combine, check_segments=False):
    n = len(pinv)
    nodes = [([int(pinv[j])], [int(q[j])], [0]) for j in range(n)]
    while len(nodes) > 1:
        nxt = []
        for i in range(0, len(nodes), 2):
            if i + 1 == len(nodes):
                nxt.append(nodes[i])
                continue
            (pl1, ql1, r1), (pl2, ql2, r2) = nodes[i], nodes[i + 1]
            pl, ql = sorted(pl1 + pl2), sorted(ql1 + ql2)
            k = len(pl)
            xs, hi = np.zeros(k, int), np.zeros(k, bool)
            for plc, qlc, rc, h in ((pl1, ql1, r1, False), (pl2, ql2, r2, True)):
                for r, c in enumerate(rc):
                    row, col = pl.index(plc[r]), ql.index(qlc[c])
                    xs[row], hi[row] = col, h
            if check_segments:
                ys, yhi = np.zeros(k, int), np.zeros(k, bool)
                ys[xs], yhi[xs] = np.arange(k), hi
                for r in range(k):
                    x = xs[r]
                    bot = min((r // 8 + 1) * 8, k)
                    cb = 0 if bot >= k else cstar(xs, hi, bot)
                    if x >= cb:
                        assert segment_delta(xs, hi, ys, yhi, r, seg=8) == delta(xs, hi, r, x)
                    else:
                        assert delta(xs, hi, r, x) < 0
            nxt.append((pl, ql, list(combine(xs, hi))))
        nodes = nxt
    pl, ql, res = nodes[0]
    out = np.zeros(n, dtype=np.int32)
    for r in range(n):
        out[pl[r]] = ql[res[r]]
    return out


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 13, 24, 31, 48, 64])
def test_walk_and_rank_match_the_oracle(oracle, n):
    for s in range(3):
        p, q = gen.permutation(n, 900 + s, 1), gen.permutation(n, 950 + s, 2)
        pinv = np.empty(n, dtype=np.int64)
        pinv[p] = np.arange(n)
        expect = oracle.steady_ant(p, q)
        assert np.array_equal(multiply(pinv, q, combine_walk), expect), (n, s)
        assert np.array_equal(multiply(pinv, q, combine_rank, check_segments=(n <= 31)), expect), (n, s)


def node_network(pl_leaves, ql_leaves, width=64):
    """The shared-memory kernel's lowest node, restated lane by lane: lane l holds positions 2l, 2l+1 of a node of
    `width` common indices (cnt <= width leaves, pads past cnt carry an infinite row).  The column ranks come from
    counting; an odd-even transposition sort of the rows (width rounds) swaps the carried ranks on each of its
    swaps where they are ascending (the 0-Hecke product).  Returns the sorted rows, the sorted columns and the
    node-local product (row rank -> column rank)."""
    inf = np.iinfo(np.int64).max
    cnt = len(pl_leaves)
    u = np.full(width, inf, dtype=np.int64)
    qv = np.full(width, inf, dtype=np.int64)
    u[:cnt], qv[:cnt] = pl_leaves, ql_leaves
    r = np.array([int(np.sum(qv < qv[j])) for j in range(width)])
    qs = np.full(width, inf, dtype=np.int64)
    qs[r[:cnt]] = qv[:cnt]
    for t in range(width):
        for i in range(t % 2, width - 1, 2):
            if u[i] > u[i + 1]:
                u[i], u[i + 1] = u[i + 1], u[i]
                if r[i] < r[i + 1]:
                    r[i], r[i + 1] = r[i + 1], r[i]
    return u[:cnt], qs[:cnt], r[:cnt]


@pytest.mark.parametrize("width,n", [(64, 1), (64, 7), (64, 100), (128, 2), (128, 33), (128, 128), (128, 300)])
def test_node_network_matches_the_oracle(oracle, width, n):
    """Each node of `width` leaves of the bottom-up tree (the trailing one partial) by the sorting network, then the tree's
    upper levels by the walk, gives the reference's product; and a node alone gives the product of its own
    sub-permutations."""
    for s in range(3):
        p, q = gen.permutation(n, 700 + s, 1), gen.permutation(n, 750 + s, 2)
        pinv = np.empty(n, dtype=np.int64)
        pinv[p] = np.arange(n)
        expect = oracle.steady_ant(p, q)
        nodes = []
        for o in range(0, n, width):
            pl, ql, res = node_network(pinv[o:o + width], q[o:o + width].astype(np.int64), width)
            nodes.append(([int(v) for v in pl], [int(v) for v in ql], [int(v) for v in res]))
            # the node alone: its rows and columns renumbered by rank, against the oracle's product of those
            k = len(pl)
            rank_r = {int(v): i for i, v in enumerate(pl)}
            rank_c = {int(v): i for i, v in enumerate(ql)}
            pn = np.array([rank_r[int(pinv[o + j])] for j in range(k)])
            pn_row_to_col = np.empty(k, dtype=np.int32)
            pn_row_to_col[pn] = np.arange(k)
            qn = np.array([rank_c[int(q[o + j])] for j in range(k)], dtype=np.int32)
            assert np.array_equal(np.asarray(res), oracle.steady_ant(pn_row_to_col, qn)), (n, s, o)
        while len(nodes) > 1:
            nxt = []
            for i in range(0, len(nodes), 2):
                if i + 1 == len(nodes):
                    nxt.append(nodes[i])
                    continue
                (pl1, ql1, r1), (pl2, ql2, r2) = nodes[i], nodes[i + 1]
                pl, ql = sorted(pl1 + pl2), sorted(ql1 + ql2)
                k = len(pl)
                xs, hi = np.zeros(k, int), np.zeros(k, bool)
                for plc, qlc, rc, h in ((pl1, ql1, r1, False), (pl2, ql2, r2, True)):
                    for rr, c in enumerate(rc):
                        xs[pl.index(plc[rr])], hi[pl.index(plc[rr])] = ql.index(qlc[c]), h
                nxt.append((pl, ql, list(combine_walk(xs, hi))))
            nodes = nxt
        pl, ql, res = nodes[0]
        out = np.zeros(n, dtype=np.int32)
        for rr in range(n):
            out[pl[rr]] = ql[res[rr]]
        assert np.array_equal(out, expect), (n, s)
