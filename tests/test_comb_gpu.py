"""GPU parity of the integer combing kernels (wavefront and batched) against the CPU oracle and the
reference's golden braids.  Bar: bit-exact permutations and scores."""
import os

import numpy as np
import pytest

from semilocal_b200 import gen

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def _rand(rng, k, alpha):
    return rng.integers(0, alpha, k).astype(np.uint8)


def test_small_exhaustive(engine, oracle):
    """All m, n in 0..40 (m > n, m = 1, n = 1, empty) against the row-major definition."""
    rng = np.random.default_rng(10)
    for m in range(0, 41):
        for n in range(0, 41):
            a, b = _rand(rng, m, 4), _rand(rng, n, 4)
            r2c, score = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
            exp = oracle.comb_rowmajor(a, b)
            assert np.array_equal(r2c, exp), (m, n)
            assert score == oracle.global_score(exp, m, n), (m, n)


def test_golden_braids(engine):
    g = np.load(GOLD)
    for k in range(int(g["comb_count"])):
        a, b, perm = g[f"comb{k}_a"], g[f"comb{k}_b"], g[f"comb{k}_perm"]
        r2c, score = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
        assert np.array_equal(r2c, perm), k
        assert score == int(g[f"comb{k}_score"]), k


@pytest.mark.parametrize("band_rows", [32, 64, 128, 256, 512, 1024])
def test_band_heights(engine, oracle, band_rows):
    rng = np.random.default_rng(band_rows)
    for m, n in [(1000, 777), (777, 1000), (2049, 63), (63, 2049), (4096, 4096)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        r2c, _ = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT, band_rows=band_rows)
        assert np.array_equal(r2c, oracle.comb_antidiag(a, b, 4)), (m, n)


def test_wide_alphabet(engine, oracle):
    rng = np.random.default_rng(11)
    for m, n, alpha in [(300, 200, 150), (123, 456, 1000), (64, 64, 100000)]:
        a = rng.integers(-alpha, alpha, m).astype(np.int32)
        b = rng.integers(-alpha, alpha, n).astype(np.int32)
        r2c, _ = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
        assert np.array_equal(r2c, oracle.comb_rowmajor(a, b)), (m, n, alpha)


def test_plain_pair_8192(engine, oracle):
    """The reference's CPU-runnable case: a, b uniform over 4 letters, 8192 each."""
    a, b = gen.plain_pair(8192, seed=1)
    r2c, score, c2r = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT, want_col_to_row=True)
    exp = oracle.comb_antidiag(a, b, 8)
    assert np.array_equal(r2c, exp)
    assert np.array_equal(c2r[r2c], np.arange(16384))
    assert score == oracle.global_score(exp, 8192, 8192)


def test_batch_vs_single(engine, oracle):
    rng = np.random.default_rng(12)
    pairs = []
    for i in range(96):
        m = int(rng.integers(0, 3000)) if i % 7 else int(rng.integers(0, 3))
        n = int(rng.integers(0, 3000)) if i % 5 else int(rng.integers(0, 3))
        pairs.append((_rand(rng, m, 4), _rand(rng, n, 4)))
    res0, sc0 = engine.batch_comb(pairs, mode=0)
    res1, sc1 = engine.batch_comb(pairs, mode=1)
    for i, (a, b) in enumerate(pairs):
        exp = oracle.comb_antidiag(a, b, 4)
        assert np.array_equal(res0[i], exp), i
        assert np.array_equal(res1[i], exp), i
        assert sc0[i] == sc1[i] == oracle.global_score(exp, len(a), len(b)), i


@pytest.mark.parametrize("lane_cols", [4, 8])
@pytest.mark.parametrize("band_rows", [64, 128, 256, 512])
def test_tile_kernel_shapes(engine, oracle, band_rows, lane_cols):
    """The register-tile kernel of lone pairs: ragged widths (not multiples of 4 or 32), one band, a padded last
    band, fewer columns than lanes, and many bands; against the oracle, braids and scores."""
    rng = np.random.default_rng(band_rows + 7)
    shapes = [(1, 1), (1, 37), (37, 1), (5, 3), (31, 33), (band_rows, 4), (band_rows + 1, 129), (1000, 777),
              (777, 1000), (2049, 63), (63, 2049), (3 * band_rows - 5, 1023), (4096, 4099)]
    for m, n in shapes:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        r2c, score = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT, band_rows=band_rows, lane_cols=lane_cols)
        exp = oracle.comb_antidiag(a, b, 4)
        assert np.array_equal(r2c, exp), (m, n)
        assert score == oracle.global_score(exp, m, n), (m, n)


def test_tile_kernel_wide_alphabet_and_plan(engine, oracle):
    """int32 symbols through the tile kernel, and a reusable plan (graph replays) on the 8192 pair."""
    import torch
    rng = np.random.default_rng(12)
    for m, n, alpha in [(300, 201, 150), (123, 457, 1000), (640, 64, 100000)]:
        a = rng.integers(-alpha, alpha, m).astype(np.int32)
        b = rng.integers(-alpha, alpha, n).astype(np.int32)
        for lc in (4, 8):
            r2c, _ = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT, lane_cols=lc)
            assert np.array_equal(r2c, oracle.comb_rowmajor(a, b)), (m, n, alpha, lc)
    a, b = gen.plain_pair(8192, seed=1)
    exp = oracle.comb_antidiag(a, b, 8)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    r2c = torch.empty(16384, dtype=torch.int32, device="cuda")
    sc = torch.zeros(1, dtype=torch.int32, device="cuda")
    pl = engine.PairPlan(8192, 8192, engine.ALGO_WAVEFRONT, lane_cols=4)
    for g in (False, True, True, True):
        pl.run(da.data_ptr(), db.data_ptr(), r2c.data_ptr(), sc.data_ptr(), g)
        pl.check()
        assert np.array_equal(r2c.cpu().numpy(), exp), g
        assert int(sc.item()) == oracle.global_score(exp, 8192, 8192), g
    pl.close()
