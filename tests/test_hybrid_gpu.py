"""GPU hybrid (tiles combed independently, glued by the GPU steady ant) and the staggered glue, against the
CPU oracle, the reference's golden glue products and the GPU wavefront.  Bar: bit-exact braids."""
import os

import numpy as np
import pytest

from semilocal_b200 import gen

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def _rand(rng, k, alpha):
    return rng.integers(0, alpha, k).astype(np.uint8)


def test_golden_glues(engine):
    g = np.load(GOLD)
    for k in range(int(g["glue_count"])):
        p, q, out = g[f"glue{k}_p"], g[f"glue{k}_q"], g[f"glue{k}_out"]
        pm, pn, qm, qn, rg = (int(x) for x in g[f"glue{k}_dims"])
        assert np.array_equal(engine.staggered_glue(p, pm, pn, q, qm, qn, bool(rg)), out), k


def test_glue_vs_oracle(engine, oracle):
    rng = np.random.default_rng(20)
    for pm, pn, qm, qn, rg in [(700, 5000, 300, 5000, True), (5000, 700, 5000, 300, False),
                               (9000, 4500, 100, 4500, True), (33, 9000, 33, 17, False)]:
        if rg:
            b = _rand(rng, pn, 4)
            p = oracle.comb_antidiag(_rand(rng, pm, 4), b, 4)
            q = oracle.comb_antidiag(_rand(rng, qm, 4), b, 4)
        else:
            a = _rand(rng, pm, 4)
            p = oracle.comb_antidiag(a, _rand(rng, pn, 4), 4)
            q = oracle.comb_antidiag(a, _rand(rng, qn, 4), 4)
        assert np.array_equal(engine.staggered_glue(p, pm, pn, q, qm, qn, rg),
                              oracle.staggered(p, pm, pn, q, qm, qn, rg)), (pm, pn, qm, qn, rg)


@pytest.mark.parametrize("m,n,tile", [(1, 1, 1), (1, 50, 8), (50, 1, 8), (37, 41, 8), (300, 200, 64),
                                      (1000, 1300, 100), (1300, 1000, 96), (2000, 64, 128), (5000, 7000, 1024),
                                      (9000, 9000, 4096)])
def test_hybrid_vs_oracle(engine, oracle, m, n, tile):
    rng = np.random.default_rng(m * 7 + n)
    a, b = _rand(rng, m, 4), _rand(rng, n, 4)
    r2c, score = engine.comb(a, b, algo=engine.ALGO_HYBRID, tile=tile)
    exp = oracle.comb_antidiag(a, b, 8)
    assert np.array_equal(r2c, exp)
    assert score == oracle.global_score(exp, m, n)


def test_hybrid_equals_wavefront_mutated_pair(engine):
    """The hybrid-config shape (b mutated from a; 4096 tiles) at 2^16: both GPU paths give one braid."""
    a, b = gen.hybrid_pair(1 << 16, seed=4)
    h, sh = engine.comb(a, b, algo=engine.ALGO_HYBRID, tile=4096)
    w, sw = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
    assert np.array_equal(h, w) and sh == sw
    assert np.array_equal(np.sort(h), np.arange(len(a) + len(b)))


def test_cached_plan_outlives_the_callers_stream(engine, oracle):
    """The last hybrid plan of a device is kept for the next call of its shape.  It is made on the caller's
    stream, which the caller may destroy before the plan is replaced: replacing and freeing it afterwards must not
    touch that stream, and every result stays exact."""
    import ctypes

    import torch
    from cuda.bindings import runtime as rt

    S = engine
    rng = np.random.default_rng(33)
    first = (_rand(rng, 3000, 4), _rand(rng, 2500, 4))
    second = (_rand(rng, 1700, 4), _rand(rng, 3900, 4))

    def run(a, b, stream_handle):
        m, n = len(a), len(b)
        da = torch.from_numpy(a).cuda()
        db = torch.from_numpy(b).cuda()
        r2c = torch.full((m + n,), -1, dtype=torch.int32, device="cuda")
        o = S._lib.opts(S.ALGO_HYBRID, tile_rows=512, tile_cols=512)
        torch.cuda.synchronize()
        S._lib.check(S.lib().slcs_comb_u8_dev(da.data_ptr(), m, db.data_ptr(), n, r2c.data_ptr(), None, None,
                                              ctypes.byref(o), ctypes.c_void_p(stream_handle)))
        torch.cuda.synchronize()
        return r2c.cpu().numpy()

    err, st = rt.cudaStreamCreateWithFlags(rt.cudaStreamNonBlocking)
    assert err == rt.cudaError_t.cudaSuccess
    got = [run(*first, int(st))]                    # planned on the caller's stream and kept
    assert rt.cudaStreamDestroy(st)[0] == rt.cudaError_t.cudaSuccess
    got.append(run(*first, 0))                      # the kept plan, reused on another stream
    got.append(run(*second, 0))                     # another shape: the kept plan is replaced and freed
    got.append(run(*first, 0))                      # the first shape planned afresh
    exp = [oracle.comb_antidiag(*first, 4), oracle.comb_antidiag(*first, 4), oracle.comb_antidiag(*second, 4),
           oracle.comb_antidiag(*first, 4)]
    for k, (g, e) in enumerate(zip(got, exp)):
        assert np.array_equal(g, e), k


@pytest.mark.parametrize("m,n,similar", [(1 << 17, 1 << 17, False), (150001, 140003, True), (140003, 262147, False)])
def test_auto_takes_the_hybrid_and_matches_the_oracle(engine, oracle, m, n, similar):
    """AUTO takes the hybrid once both lengths reach 2^17 (tiles of about min(m, n) / 16, here 16384; ragged edges,
    both orientations): bit-exact against the oracle and against the wavefront forced by the caller."""
    if similar:
        a, b = gen.hybrid_pair(max(m, n), seed=9)
        a, b = a[:m], b[:n]
    else:
        rng = np.random.default_rng(m + 3 * n)
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
    r2c, score = engine.comb(a, b)
    exp = oracle.comb_antidiag(a, b, os.cpu_count() or 8)
    assert np.array_equal(r2c, exp)
    assert score == oracle.global_score(exp, m, n)
    w, sw = engine.comb(a, b, algo=engine.ALGO_WAVEFRONT)
    assert np.array_equal(w, exp) and sw == score
