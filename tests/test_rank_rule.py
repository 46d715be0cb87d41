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
