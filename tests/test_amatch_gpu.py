"""Approximate pattern search on the GPU (slcs_duplicate_search_*): the result vectors of the reference's
InteractiveDuplicateSearchSemiDense::find and ...SemiSparse::find, bit for bit, against the reference's own golden results and the
oracle's restatement, through the C ABI."""
import json
import os

import numpy as np
import pytest

import semilocal_b200 as S
from semilocal_b200 import gen

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "amatch_golden.json")


@pytest.mark.parametrize("sparse", [False, True])
def test_golden(engine, sparse):
    for c in json.load(open(GOLDEN))["cases"]:
        p, t = gen.planted_text(c["m"], c["n"], c["copies"], c["alphabet"], c["seed"])
        got = engine.duplicate_search(p, t, c["k"], sparse=sparse)
        assert [list(x) for x in got] == c["intervals_sparse" if sparse else "intervals"], (c["m"], c["n"], c["k"])


def test_sparse_random_vs_oracle(engine, oracle):
    rng = np.random.default_rng(9)
    for trial in range(25):
        m = int(rng.integers(1, 120))
        k = float(rng.choice([0.5, 0.75, 0.9, 1.0, rng.uniform(0.3, 1.0)]))
        n = int(rng.integers(int(m / k), int(m / k) + 6000))
        p, t = gen.planted_text(m, n, int(rng.integers(0, 30)), int(rng.choice([2, 4])), 1900 + trial)
        assert engine.duplicate_search(p, t, k, sparse=True) == oracle.duplicate_search(p, t, k, sparse=True), (m, n, k)


@pytest.mark.parametrize("symbols", ["u8", "i32"])
def test_random_vs_oracle(engine, oracle, symbols):
    rng = np.random.default_rng(7 if symbols == "u8" else 8)
    for trial in range(40):
        m = int(rng.integers(1, 300))
        k = float(rng.choice([0.5, 0.6, 0.75, 0.8, 0.9, 0.95, 1.0, rng.uniform(0.25, 1.0)]))
        n = int(rng.integers(int(m / k), int(m / k) + 20000))
        p, t = gen.planted_text(m, n, int(rng.integers(0, 30)), int(rng.choice([2, 4, 20])), 900 + trial)
        if symbols == "i32":
            p, t = p.astype(np.int32) * 1000 - 7, t.astype(np.int32) * 1000 - 7
        assert engine.duplicate_search(p, t, k) == oracle.duplicate_search(p, t, k), (m, n, k)


@pytest.mark.parametrize("sparse", [False, True])
def test_i32_symbols_equal_to_padding_codes(engine, oracle, sparse):
    """int32 symbols are arbitrary values compared for equality, including the two codes the combing kernel keeps
    for its padding rows and columns (-2^30 and -2^30 - 1): the results stay the reference's."""
    table = np.array([-(1 << 30), -(1 << 30) - 1, 5, (1 << 31) - 1], dtype=np.int64)
    for m, n, k, seed in [(37, 3000, 0.8, 61), (200, 9000, 0.9, 62), (1, 40, 1.0, 63)]:
        p, t = gen.planted_text(m, n, 6, 4, seed)
        p, t = table[p].astype(np.int32), table[t].astype(np.int32)
        assert engine.duplicate_search(p, t, k, sparse=sparse) == oracle.duplicate_search(p, t, k, sparse=sparse), \
            (m, n, k)


def test_edges(engine, oracle):
    # window of one end (k = 1), the text exactly one window long, a one-symbol pattern, intervals down to length 0
    for m, n, k in [(1, 50, 1.0), (40, 40, 1.0), (40, 41, 1.0), (8, 17, 0.5), (1, 9, 0.2), (3, 3000, 0.34)]:
        p, t = gen.planted_text(m, n, 3, 4, 70 + m + n)
        assert engine.duplicate_search(p, t, k) == oracle.duplicate_search(p, t, k), (m, n, k)


def test_large(engine, oracle):
    p, t = gen.planted_text(1000, 1 << 18, 60, 4, 77)
    got = engine.duplicate_search(p, t, 0.9)
    assert len(got) > 0
    assert got == oracle.duplicate_search(p, t, 0.9)


def test_bad_arguments(engine):
    p, t = gen.planted_text(10, 100, 2, 4, 1)
    for k in (0.0, -1.0, 1.5):
        with pytest.raises(S.SlcsError):
            engine.duplicate_search(p, t, k)
    with pytest.raises(S.SlcsError):
        engine.duplicate_search(p, t[:15], 0.5)
