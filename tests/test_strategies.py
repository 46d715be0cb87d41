"""The Python mirror of the reference's strategy classes (semilocal_b200/strategies.py) and its Permutation type, on
the CPU: the engine calls the classes make are answered by the oracle, so what is checked here is the classes' own
logic -- argument order, the (m, n) tags, the glue's result shape, the score read from a braid
(R:include/LCS/LCS.h:223-233), the result list of the duplicate searches.  The engine behind them is checked
against the oracle by the GPU tests."""
import numpy as np
import pytest

from semilocal_b200 import api
from semilocal_b200 import strategies as St
from semilocal_b200.api import Permutation


def _rand(rng, k, alpha):
    return rng.integers(0, alpha, k).astype(np.uint8)


@pytest.fixture
def on_oracle(monkeypatch, oracle):
    """The engine entry points the strategies call, answered by the oracle (and every call recorded)."""
    calls = []

    def comb(a, b, algo=0, tile=0, band_rows=0, want_col_to_row=False, sa_cutoff=0):
        calls.append(("comb", algo, tile, band_rows, sa_cutoff))
        braid = oracle.comb_antidiag(a, b)
        return braid, oracle.global_score(braid, len(a), len(b))

    def steady_ant(p, q, sa_cutoff=0):
        calls.append(("steady_ant", sa_cutoff))
        return oracle.steady_ant(p, q)

    def staggered_glue(p, pm, pn, q, qm, qn, row_glue):
        calls.append(("glue", pm, pn, qm, qn, row_glue))
        return oracle.staggered(p, pm, pn, q, qm, qn, row_glue)

    def duplicate_search(p, t, k, sparse=False):
        calls.append(("dup", sparse))
        return oracle.duplicate_search(p, t, k, sparse=sparse)

    monkeypatch.setattr(api, "comb", comb)
    monkeypatch.setattr(api, "steady_ant", steady_ant)
    monkeypatch.setattr(api, "staggered_glue", staggered_glue)
    monkeypatch.setattr(api, "lcs", lambda a, b: oracle.lcs_dp(a, b))
    monkeypatch.setattr(api, "bitcomb_llcs", lambda a, b: oracle.lcs_dp(a, b))
    monkeypatch.setattr(api, "duplicate_search", duplicate_search)
    return calls


def test_permutation_mirrors_the_reference_type():
    r2c = np.array([2, 0, 3, 1], np.int32)
    P = Permutation.from_row_to_col(r2c, 1, 3)
    assert (P.rows, P.cols, P.m, P.n) == (4, 4, 1, 3)
    assert [P.get_col_by_row(r) for r in range(4)] == [2, 0, 3, 1]
    assert all(P.get_row_by_col(P.get_col_by_row(r)) == r for r in range(4))
    assert P == Permutation.from_row_to_col(r2c.copy())
    assert P != Permutation.from_row_to_col(np.array([0, 1, 2, 3], np.int32))


def test_combing_strategies(on_oracle, oracle):
    rng = np.random.default_rng(80)
    a, b = _rand(rng, 70, 4), _rand(rng, 90, 4)
    exp = oracle.comb_antidiag(a, b)
    for solver in (St.GpuIterativeCombing(band_rows=64), St.GpuHybridCombing(tile=32, sa_cutoff=1024)):
        P = solver.compute(a, b)
        assert isinstance(P, Permutation) and (P.m, P.n) == (70, 90)
        assert np.array_equal(P.row_to_col, exp)
        assert np.array_equal(P.col_to_row[P.row_to_col], np.arange(160))
    assert on_oracle[0] == ("comb", 1, 0, 64, 0) and on_oracle[1] == ("comb", 2, 32, 0, 1024)


def test_lcs_strategies(on_oracle, oracle):
    rng = np.random.default_rng(81)
    for m, n in [(1, 1), (5, 40), (40, 5), (64, 64), (0, 7)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        s = oracle.lcs_dp(a, b)
        assert St.LCSBySemiLocal(St.GpuIterativeCombing()).compute(a, b) == s, (m, n)
        assert St.LCSBySemiLocal().compute(a, b) == s
        assert St.BitParallelLCS().compute(a, b) == s


def test_braid_multiplication_and_glue(on_oracle, oracle):
    from semilocal_b200 import gen
    p, q = gen.permutation(300, 82, 300), gen.permutation(300, 83, 300)
    R = St.GpuSteadyAntMultiplication(sa_cutoff=2048).multiply(Permutation.from_row_to_col(p), q)
    assert np.array_equal(R.row_to_col, oracle.steady_ant(p, q)) and on_oracle[-1] == ("steady_ant", 2048)
    # row glue: braids of (a_top, b) above (a_bottom, b) give the braid of (a_top a_bottom, b); column glue: braids
    # of (a, b_left) beside (a, b_right) give the braid of (a, b_left b_right)
    rng = np.random.default_rng(84)
    at, ab, b = _rand(rng, 30, 4), _rand(rng, 20, 4), _rand(rng, 25, 4)
    comb = St.GpuIterativeCombing()
    G = St.StaggeredStickyBraidMultiplication().staggered_sticky_multiplication(comb.compute(at, b), comb.compute(ab, b),
                                                                                True)
    assert (G.m, G.n) == (50, 25) and np.array_equal(G.row_to_col, oracle.comb_antidiag(np.concatenate([at, ab]), b))
    a, bl, br = _rand(rng, 30, 4), _rand(rng, 20, 4), _rand(rng, 25, 4)
    G = St.StaggeredStickyBraidMultiplication().staggered_sticky_multiplication(comb.compute(a, bl), comb.compute(a, br),
                                                                                False)
    assert (G.m, G.n) == (30, 45) and np.array_equal(G.row_to_col, oracle.comb_antidiag(a, np.concatenate([bl, br])))


def test_duplicate_search_classes_append(on_oracle, oracle):
    from semilocal_b200 import gen
    p, t = gen.planted_text(30, 2000, 5, 4, 85)
    for cls, sparse in ((St.InteractiveDuplicateSearchSemiDense, False), (St.InteractiveDuplicateSearchSemiSparse, True)):
        result = [("kept", 0, 0.0)]
        cls().find(p, t, 0.8, result)
        assert result[0] == ("kept", 0, 0.0)
        assert result[1:] == oracle.duplicate_search(p, t, 0.8, sparse=sparse) and len(result) > 1
        assert on_oracle[-1] == ("dup", sparse)
