"""GPU bit-parallel LLCS -- the braid-in-bits combing and the bit-vector (Hyyro) kernel -- against the DP oracle,
the reference's golden bit scores, and the integer braid's score on the hybrid-config pair.  Bar: exact scores."""
import os

import numpy as np
import pytest

from semilocal_b200 import gen

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")
KERNELS = ["bitcomb_llcs", "hyyro_llcs"]


@pytest.mark.parametrize("fn", KERNELS)
def test_small_all_shapes(engine, oracle, fn):
    llcs = getattr(engine, fn)
    rng = np.random.default_rng(30)
    for m in list(range(0, 70, 3)) + [95, 96, 97]:
        for n in list(range(0, 70, 5)) + [127, 128, 129]:
            for alpha in (2, 4):
                a = rng.integers(0, alpha, m).astype(np.uint8)
                b = rng.integers(0, alpha, n).astype(np.uint8)
                assert llcs(a, b) == oracle.lcs_dp(a, b), (m, n, alpha)


@pytest.mark.parametrize("fn", KERNELS)
def test_golden_bit_scores(engine, fn):
    llcs = getattr(engine, fn)
    g = np.load(GOLD)
    for k in range(int(g["bit_count"])):
        a, b = g[f"bit{k}_a"], g[f"bit{k}_b"]
        assert llcs(a.astype(np.uint8), b.astype(np.uint8)) == int(g[f"bit{k}_score"]), k


@pytest.mark.parametrize("m,n", [(1000, 3000), (3000, 1000), (4097, 4095), (20000, 20001), (70000, 5000),
                                 (5000, 70000), (140000, 33), (33, 140000), (1025, 1023), (2048, 31)])
@pytest.mark.parametrize("fn", KERNELS)
def test_mid_sizes(engine, oracle, m, n, fn):
    rng = np.random.default_rng(m + n)
    a = rng.integers(0, 4, m).astype(np.uint8)
    b = rng.integers(0, 4, n).astype(np.uint8)
    assert getattr(engine, fn)(a, b) == oracle.lcs_dp(a, b)


def test_hybrid_pair_score_matches_braid(engine):
    """The hybrid-config pair at 2^18 (b mutated from a): the bit kernel's LLCS equals the integer braid's."""
    a, b = gen.hybrid_pair(1 << 18, seed=4)
    _, s_braid = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
    assert engine.bitcomb_llcs(a, b) == s_braid
    assert engine.hyyro_llcs(a, b) == s_braid


@pytest.mark.parametrize("fn", KERNELS)
def test_rejects_wide_symbols(engine, fn):
    with pytest.raises(engine.SlcsError):
        getattr(engine, fn)(np.array([0, 4], np.uint8), np.array([1], np.uint8))


def test_hyyro_plan_graph_replays(engine, oracle):
    """A reusable bit-vector plan: eager run, then graph replays on the same buffers, scores exact each time."""
    import torch
    rng = np.random.default_rng(31)
    for m, n in [(5000, 7001), (7001, 5000), (40000, 40000)]:
        a = rng.integers(0, 4, m).astype(np.uint8)
        b = rng.integers(0, 4, n).astype(np.uint8)
        exp = oracle.hyyro_llcs(a, b)
        da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        sc = torch.zeros(1, dtype=torch.int32, device="cuda")
        pl = engine.PairPlan(m, n, engine.PLAN_HYYRO)
        for g in (False, True, True):
            pl.run(da.data_ptr(), db.data_ptr(), None, sc.data_ptr(), g)
            pl.check()
            assert int(sc.item()) == exp, (m, n, g)
        pl.close()
