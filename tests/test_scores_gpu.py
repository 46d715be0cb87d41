"""GPU score queries read from the braid, against the semi-local matrix computed by DP from its definition
and against LCS by DP on the corresponding substrings.  Bar: exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_every_matrix_entry(engine, oracle):
    rng = np.random.default_rng(40)
    for m, n in [(7, 9), (9, 7), (13, 13), (1, 12), (12, 1)]:
        a = rng.integers(0, 3, m).astype(np.uint8)
        b = rng.integers(0, 3, n).astype(np.uint8)
        H = oracle.semilocal_matrix(a, b)
        r2c, _ = engine.comb(a, b)
        qs = [(engine.Q_MATRIX, i, j) for i in range(m + n + 1) for j in range(m + n + 1)]
        got = engine.scores(r2c, m, n, qs)
        assert np.array_equal(got, H.ravel()), (m, n)


def test_named_queries_vs_dp(engine, oracle):
    rng = np.random.default_rng(41)
    m, n = 300, 400
    a = rng.integers(0, 4, m).astype(np.uint8)
    b = rng.integers(0, 4, n).astype(np.uint8)
    r2c, score = engine.comb(a, b)
    qs, exp = [(engine.Q_GLOBAL, 0, 0)], [oracle.lcs_dp(a, b)]
    for _ in range(40):
        i, j = sorted(int(x) for x in rng.integers(0, n + 1, 2))
        qs.append((engine.Q_STRING_SUBSTRING, i, j)); exp.append(oracle.lcs_dp(a, b[i:j]))
        i, j = int(rng.integers(0, m + 1)), int(rng.integers(0, n + 1))
        qs.append((engine.Q_PREFIX_SUFFIX, i, j)); exp.append(oracle.lcs_dp(a[:i], b[j:]))
        qs.append((engine.Q_SUFFIX_PREFIX, i, j)); exp.append(oracle.lcs_dp(a[i:], b[:j]))
        i, j = sorted(int(x) for x in rng.integers(0, m + 1, 2))
        qs.append((engine.Q_SUBSTRING_STRING, i, j)); exp.append(oracle.lcs_dp(a[i:j], b))
    assert list(engine.scores(r2c, m, n, qs)) == exp
    assert score == exp[0]


def test_out_of_range_query_is_an_error(engine):
    r2c, _ = engine.comb(np.array([1, 2], np.uint8), np.array([2, 1], np.uint8))
    with pytest.raises(engine.SlcsError):
        engine.scores(r2c, 2, 2, [(engine.Q_STRING_SUBSTRING, 2, 1)])


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,w", [(1, 1, 1), (5, 9, 3), (300, 200, 1), (300, 200, 200), (700, 1000, 64),
                                   (1200, 5000, 777), (50, 4200, 2049)])
def test_window_scores_match_dp(engine, oracle, m, n, w):
    import semilocal_b200 as S
    from semilocal_b200 import gen
    a = gen.uniform_string(m, 4, 70 + m, 1)
    b = gen.uniform_string(n, 4, 80 + n, 2)
    braid = oracle.comb_antidiag(a, b)
    got = S.window_scores(braid, m, n, w)
    assert len(got) == n - w + 1
    step = max(1, (n - w + 1) // 64)   # the DP per window is O(m w): check a spread of windows, and the last
    for s in list(range(0, n - w + 1, step)) + [n - w]:
        assert int(got[s]) == oracle.lcs_dp(a, b[s:s + w]), (s, w)
    # every window against the braid's own string-substring queries
    qs = [(S.Q_STRING_SUBSTRING, s, s + w) for s in range(n - w + 1)]
    assert np.array_equal(got, S.scores(braid, m, n, qs))
