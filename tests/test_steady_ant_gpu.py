"""GPU steady ant (unit-Monge braid multiplication) against the CPU oracle, the O(n^3) definition and the
reference's golden products.  Bar: bit-exact permutations."""
import os

import numpy as np
import pytest

from semilocal_b200 import gen

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def test_small_vs_naive(engine, oracle):
    for n in list(range(1, 40)) + [63, 64, 65, 100, 127, 128, 129, 255, 300]:
        for s in range(2):
            p, q = gen.permutation(n, 500 + s, n), gen.permutation(n, 600 + s, n)
            assert np.array_equal(engine.steady_ant(p, q), oracle.braid_naive(p, q)), (n, s)


def test_extremes(engine, oracle):
    for n in [5, 32, 33, 1000, 4096, 5000, 9000]:
        I = np.arange(n, dtype=np.int32)
        Rv = I[::-1].copy()
        for p, q in [(I, I), (Rv, I), (I, Rv), (Rv, Rv)]:
            assert np.array_equal(engine.steady_ant(p, q), oracle.steady_ant(p, q)), n


def test_golden_products(engine):
    g = np.load(GOLD)
    for k in range(int(g["sa_count"])):
        p, q, r = g[f"sa{k}_p"], g[f"sa{k}_q"], g[f"sa{k}_r"]
        assert np.array_equal(engine.steady_ant(p, q), r), k


@pytest.mark.parametrize("n", [511, 4095, 4096, 4097, 8192, 10007, 33333, 65536, 100000, 262144])
def test_mid_sizes(engine, oracle, n):
    p, q = gen.permutation(n, 700, n), gen.permutation(n, 701, n)
    assert np.array_equal(engine.steady_ant(p, q), oracle.steady_ant(p, q))


@pytest.mark.parametrize("cutoff", [1024, 2048, 4096])
def test_cutoffs_and_partial_nodes(engine, oracle, cutoff):
    """Every shared-memory subtree size the tuner may pick; sizes whose last node at each span has one child, two
    unequal children, or exactly fills it (the walked spans below 1024 and the ranked spans from 1024 up)."""
    for n in [1536, 1537, 2047, 2049, 3000, 3071, 6143, 12289, 20000]:
        p, q = gen.permutation(n, 710 + n % 7, n), gen.permutation(n, 711 + n % 5, n)
        assert np.array_equal(engine.steady_ant(p, q, sa_cutoff=cutoff), oracle.steady_ant(p, q)), (n, cutoff)


def test_large_properties(engine, oracle):
    """2^22 (the headline size): exact against the sequential oracle (a few seconds on the host)."""
    n = 1 << 22
    p, q = gen.steady_ant_pair(n)
    r = engine.steady_ant(p, q)
    assert np.array_equal(np.sort(r), np.arange(n))
    assert np.array_equal(r, oracle.steady_ant(p, q))
