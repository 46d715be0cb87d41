"""CPU tests of the oracle: the C restatement against the reference compiled in place (oracle/_ref) and
against the committed golden vectors (tests/golden/, produced by that reference library)."""
import os

import numpy as np
import pytest

from semilocal_b200 import gen

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _rand(rng, k, alpha):
    return rng.integers(0, alpha, k).astype(np.int32)


def test_comb_small_definitions_agree(oracle):
    """Row-major combing == anti-diagonal combing == DP-defined kernel, all m, n <= 10 (incl. m > n, 0)."""
    rng = np.random.default_rng(1)
    for m in range(0, 11):
        for n in range(0, 11):
            a, b = _rand(rng, m, 5), _rand(rng, n, 5)
            x = oracle.comb_rowmajor(a, b)
            assert np.array_equal(x, oracle.comb_antidiag(a, b, 2))
            if m and n:
                assert np.array_equal(x, oracle.comb_dp(a, b)), (m, n)


def test_rotate180_is_swap(oracle):
    rng = np.random.default_rng(2)
    for m, n in [(7, 13), (13, 7), (1, 30), (25, 25)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        assert np.array_equal(oracle.comb_rowmajor(a, b), oracle.rotate180(oracle.comb_rowmajor(b, a)))


def test_scores_against_dp(oracle):
    """Every semi-local matrix entry read from the braid equals the DP definition."""
    rng = np.random.default_rng(3)
    for m, n in [(5, 9), (9, 5), (12, 12), (1, 7)]:
        a, b = _rand(rng, m, 3), _rand(rng, n, 3)
        H = oracle.semilocal_matrix(a, b)
        perm = oracle.comb_rowmajor(a, b)
        for i in range(m + n + 1):
            for j in range(m + n + 1):
                assert oracle.semilocal_entry(perm, m, n, i, j) == H[i, j], (i, j)
        assert oracle.global_score(perm, m, n) == oracle.lcs_dp(a, b)


def test_steady_ant_vs_naive(oracle):
    for n in list(range(1, 24)) + [64, 100, 163]:
        p, q = gen.permutation(n, 31, n), gen.permutation(n, 32, n)
        assert np.array_equal(oracle.steady_ant(p, q), oracle.braid_naive(p, q)), n


def test_hybrid_equals_combing(oracle):
    rng = np.random.default_rng(4)
    for m, n, t in [(200, 300, 64), (301, 97, 50), (64, 1000, 128)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        assert np.array_equal(oracle.hybrid_iterative(a, b, 3, t, t), oracle.comb_rowmajor(a, b))


def test_bit_parallel_vs_dp(oracle):
    rng = np.random.default_rng(5)
    for m, n in [(32, 64), (64, 64), (96, 320), (512, 1024)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        assert oracle.bit_llcs_nary(a, b, 2) == oracle.lcs_dp(a, b)
    for m, n in [(64, 64), (128, 256)]:
        a, b = _rand(rng, m, 2), _rand(rng, n, 2)
        assert oracle.bit_llcs_binary(a, b) == oracle.lcs_dp(a, b)


ref_only = pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                               "libslcs_ref.so")),
                              reason="reference library oracle/_ref not built (needs the reference sources)")


def test_hyyro_vs_dp(oracle):
    """The bit-vector (Hyyro) restatement against the DP on ragged lengths (words of 64 rows, partial last words)."""
    rng = np.random.default_rng(9)
    for m, n in [(0, 5), (5, 0), (1, 1), (63, 64), (64, 65), (65, 63), (200, 333), (1000, 17)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        assert oracle.hyyro_llcs(a, b) == oracle.lcs_dp(a, b), (m, n)


@ref_only
def test_hyyro_matches_reference(oracle):
    """Pin: the restatement equals the reference's own lllcs_hyyro (its sequential and anti-diagonal forms)."""
    rng = np.random.default_rng(10)
    for m, n in [(1, 1), (63, 200), (64, 64), (130, 500), (700, 900), (2000, 300)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        exp = oracle.hyyro_llcs(a, b)
        assert oracle.ref_hyyro(a, b) == exp, (m, n)
        if n > (m + 63) // 64:
            assert oracle.ref_hyyro(a, b, 4) == exp, (m, n)


@ref_only
def test_restatement_matches_reference(oracle):
    rng = np.random.default_rng(6)
    for m, n in [(1, 1), (1, 9), (9, 1), (17, 33), (300, 200), (1000, 999)]:
        a, b = _rand(rng, m, 11), _rand(rng, n, 11)
        x = oracle.comb_rowmajor(a, b)
        assert np.array_equal(x, oracle.ref_comb(a, b, "simple"))
        assert np.array_equal(x, oracle.ref_comb(a, b, "openmp", 3))
        assert oracle.lcs_dp(a, b) == oracle.ref_lcs(a, b)
    for n in [2, 7, 100, 1000, 4097]:
        p, q = gen.permutation(n, 41, n), gen.permutation(n, 42, n)
        assert np.array_equal(oracle.steady_ant(p, q), oracle.ref_braid(p, q, "seq"))
    for m, n in [(320, 640), (1024, 1024)]:
        a, b = _rand(rng, m, 4), _rand(rng, n, 4)
        assert oracle.bit_llcs_nary(a, b, 2) == oracle.ref_bit_nary(a, b, 4)


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "golden.npz")), reason="golden vectors not generated")
def test_oracle_against_golden(oracle):
    """The C restatement reproduces every vector the reference produced (tests/golden/make_golden.py)."""
    g = np.load(os.path.join(GOLD, "golden.npz"))
    ncomb = int(g["comb_count"])
    for k in range(ncomb):
        a, b, perm = g[f"comb{k}_a"], g[f"comb{k}_b"], g[f"comb{k}_perm"]
        assert np.array_equal(oracle.comb_rowmajor(a, b), perm), k
        assert oracle.global_score(perm, len(a), len(b)) == int(g[f"comb{k}_score"])
    for k in range(int(g["sa_count"])):
        p, q, r = g[f"sa{k}_p"], g[f"sa{k}_q"], g[f"sa{k}_r"]
        assert np.array_equal(oracle.steady_ant(p, q), r), k
    for k in range(int(g["glue_count"])):
        p, q, out = g[f"glue{k}_p"], g[f"glue{k}_q"], g[f"glue{k}_out"]
        pm, pn, qm, qn, rg = (int(x) for x in g[f"glue{k}_dims"])
        assert np.array_equal(oracle.staggered(p, pm, pn, q, qm, qn, bool(rg)), out), k
    for k in range(int(g["bit_count"])):
        a, b = g[f"bit{k}_a"], g[f"bit{k}_b"]
        assert oracle.bit_llcs_nary(a, b, 2) == int(g[f"bit{k}_score"]), k


@ref_only
def test_reference_test_grids(oracle):
    """The oracle against the reference on the grids of the reference's own GoogleTest comparators (sizes, steps
    and alphabets as there; strings and permutations seeded here): SemiLocalLCSTest.cpp:47-55 (Dummy vs Simple,
    5..49 squared, 5 letters) and :57-68 (Simple vs OpenMP, 4900..4999 step 11, 11 letters), SteadyAntTest.cpp:
    43-56 (Naive vs SimpleSticky, 100..299, every 3rd size here) and :59-67 (SimpleSticky vs MemoryOptimized, 1000..29999 step 111),
    LCSTest.cpp:65-86 (Dummy vs SemiLocal vs SequentialMem, 5..499 with 15 letters; every 7th size pair here), and the
    combined and hybrid strategies of SemiLocalLCSTest.cpp:88-130 on parts of their grids."""
    rng = np.random.default_rng(50)
    for m in range(5, 50):
        for n in range(5, 50):
            a, b = _rand(rng, m, 5), _rand(rng, n, 5)
            x = oracle.comb_rowmajor(a, b)
            assert np.array_equal(x, oracle.ref_comb(a, b, "dummy")), (m, n)
            assert np.array_equal(x, oracle.ref_comb(a, b, "simple")), (m, n)
    for m in range(4900, 5000, 11):
        for n in range(4900, 5000, 33):
            a, b = _rand(rng, m, 11), _rand(rng, n, 11)
            assert np.array_equal(oracle.comb_antidiag(a, b, 4), oracle.ref_comb(a, b, "openmp", 4)), (m, n)
    for n in range(100, 300, 3):
        p, q = gen.permutation(n, 60 + n, n), gen.permutation(n, 61 + n, n)
        assert np.array_equal(oracle.steady_ant(p, q), oracle.ref_braid(p, q, "naive")), n
    for n in range(1000, 30000, 111):
        p, q = gen.permutation(n, 62 + n, n), gen.permutation(n, 63 + n, n)
        assert np.array_equal(oracle.steady_ant(p, q), oracle.ref_braid(p, q, "seq")), n
    for m in range(5, 500, 7):
        for n in range(5, 500, 49):
            a, b = _rand(rng, m, 15), _rand(rng, n, 15)
            s = oracle.lcs_dp(a, b)
            assert s == oracle.ref_lcs(a, b, "dummy") == oracle.ref_lcs(a, b, "semilocal") == oracle.ref_lcs(a, b), (m, n)
    # SemiLocalLCSTest.cpp:88-130: OpenMP vs Combined (3000..3339, 150 letters), vs HybridRecursive (3900..3999) and
    # vs HybridIterative (one 10^5 pair there; 20000 here, tiles 4096), every few sizes of each grid
    for m in range(3000, 3340, 110):
        for n in range(3000, 3340, 110):
            a, b = _rand(rng, m, 150), _rand(rng, n, 150)
            assert np.array_equal(oracle.comb_antidiag(a, b, 4), oracle.ref_comb(a, b, "combined", 2)), (m, n)
    for m, n in [(3900, 3955), (3977, 3911)]:
        a, b = _rand(rng, m, 150), _rand(rng, n, 150)
        assert np.array_equal(oracle.comb_antidiag(a, b, 4), oracle.ref_hybrid_recursive(a, b, 2, 6, 400)), (m, n)
    a, b = _rand(rng, 20000, 150), _rand(rng, 20037, 150)
    assert np.array_equal(oracle.comb_antidiag(a, b, 8), oracle.ref_hybrid_iterative(a, b, 4, 4096, 4096))


legacy_only = pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                                  "libslcs_ref_legacy.so")),
                                 reason="legacy reference library oracle/_ref not built (needs the reference sources)")


@legacy_only
def test_legacy_second_oracle(oracle):
    """The reference's legacy implementations (R:semi_local.h, R:unit_monge_mult/steady_ant.h) as a second oracle,
    on the same grids as test_reference_test_grids: sticky_braid_mpi (:212-276) against the restatement on the
    5..49 squared grid (1 and 3 threads) and the 4900..4999 grid; steady_ant_parallel_wrapper (:811-844), nested
    and sequential, against the restatement on 100..299 and 1000..29999; hybrid_iterative_wrapper (:740-790) on a
    pair above its 32000-row tile bound."""
    rng = np.random.default_rng(51)
    for m in range(5, 50, 2):
        for n in range(5, 50, 3):
            a, b = _rand(rng, m, 5), _rand(rng, n, 5)
            x = oracle.comb_rowmajor(a, b)
            assert np.array_equal(x, oracle.legacy_comb(a, b, 1)), (m, n)
            assert np.array_equal(x, oracle.legacy_comb(a, b, 3)), (m, n)
    for m in range(4900, 5000, 33):
        for n in range(4900, 5000, 33):
            a, b = _rand(rng, m, 11), _rand(rng, n, 11)
            assert np.array_equal(oracle.comb_antidiag(a, b, 4), oracle.legacy_comb(a, b, 4)), (m, n)
    for n in range(100, 300, 7):
        p, q = gen.permutation(n, 70 + n, n), gen.permutation(n, 71 + n, n)
        assert np.array_equal(oracle.steady_ant(p, q), oracle.legacy_steady_ant(p, q, 3, 5)), n
    for n in range(1000, 30000, 1111):
        p, q = gen.permutation(n, 72 + n, n), gen.permutation(n, 73 + n, n)
        exp = oracle.steady_ant(p, q)
        assert np.array_equal(exp, oracle.legacy_steady_ant(p, q, 3, 5)), n
        assert np.array_equal(exp, oracle.legacy_steady_ant(p, q, 0, 5)), n
    a, b = _rand(rng, 40000, 4), _rand(rng, 33001, 4)
    assert np.array_equal(oracle.comb_antidiag(a, b, 8), oracle.legacy_hybrid_iterative(a, b, 4))
