"""GPU bit-parallel combing (LLCS) against the DP oracle, the reference's golden bit scores, and the integer
braid's score on the hybrid-config pair.  Bar: exact scores."""
import os

import numpy as np
import pytest

from semilocal_b200 import gen

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def test_small_all_shapes(engine, oracle):
    rng = np.random.default_rng(30)
    for m in list(range(0, 70, 3)) + [95, 96, 97]:
        for n in list(range(0, 70, 5)) + [127, 128, 129]:
            for alpha in (2, 4):
                a = rng.integers(0, alpha, m).astype(np.uint8)
                b = rng.integers(0, alpha, n).astype(np.uint8)
                assert engine.bitcomb_llcs(a, b) == oracle.lcs_dp(a, b), (m, n, alpha)


def test_golden_bit_scores(engine):
    g = np.load(GOLD)
    for k in range(int(g["bit_count"])):
        a, b = g[f"bit{k}_a"], g[f"bit{k}_b"]
        assert engine.bitcomb_llcs(a.astype(np.uint8), b.astype(np.uint8)) == int(g[f"bit{k}_score"]), k


@pytest.mark.parametrize("m,n", [(1000, 3000), (3000, 1000), (4097, 4095), (20000, 20001), (70000, 5000),
                                 (5000, 70000), (140000, 33)])
def test_mid_sizes(engine, oracle, m, n):
    rng = np.random.default_rng(m + n)
    a = rng.integers(0, 4, m).astype(np.uint8)
    b = rng.integers(0, 4, n).astype(np.uint8)
    assert engine.bitcomb_llcs(a, b) == oracle.lcs_dp(a, b)


def test_hybrid_pair_score_matches_braid(engine):
    """The hybrid-config pair at 2^18 (b mutated from a): the bit kernel's LLCS equals the integer braid's."""
    a, b = gen.hybrid_pair(1 << 18, seed=4)
    _, s_braid = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
    assert engine.bitcomb_llcs(a, b) == s_braid


def test_rejects_wide_symbols(engine):
    with pytest.raises(engine.SlcsError):
        engine.bitcomb_llcs(np.array([0, 4], np.uint8), np.array([1], np.uint8))
