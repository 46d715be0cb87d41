"""Autotuner: the measured table is well formed, results stay bit-exact under tuned parameters, and
get / set / reset round-trip."""
import numpy as np
import pytest

from oracle import oracle as O
from semilocal_b200 import gen

pytestmark = pytest.mark.gpu


def test_autotune_table_and_results_bit_exact(engine, tmp_path):
    import semilocal_b200 as S
    S.set_tuning(None)
    cache = str(tmp_path / "tuning.json")
    table = S.autotune(cache=cache)
    for k in range(32):
        assert table["band_rows_batch"][k] in (32, 64, 128, 256, 512, 1024)
        assert table["band_rows_single"][k] in (32, 64, 128, 256, 512, 1024)
    assert table["tile"] in (2048, 4096, 8192)
    assert table["sa_cutoff"] in (1024, 2048, 4096)
    assert S.tuning() == table
    # a second call with the cache loads the same table without measuring
    S.set_tuning(None)
    assert S.autotune(cache=cache) == table and S.tuning() == table
    # every path that reads the table still matches the oracle
    rng = np.random.default_rng(3)
    pairs = []
    for i, L in enumerate(rng.integers(100, 5000, 12)):
        a = gen.uniform_string(int(L), 4, 40 + i, 1)
        pairs.append((a, gen.mutate(a, 0.1, 0.005, 0.005, 4, 50 + i)))
    braids, scores = S.batch_comb(pairs)
    for (a, b), r2c in zip(pairs, braids):
        assert np.array_equal(r2c, O.comb_antidiag(a, b))
    a, b = gen.hybrid_pair(1 << 14, seed=4)
    exp = O.comb_antidiag(a, b)
    assert np.array_equal(S.comb(a, b, algo=S.ALGO_WAVEFRONT)[0], exp)
    assert np.array_equal(S.comb(a, b, algo=S.ALGO_HYBRID, tile=1024)[0], exp)
    p, q = gen.steady_ant_pair(1 << 14)
    assert np.array_equal(S.steady_ant(p, q), O.steady_ant(p, q))
    S.set_tuning(None)
    assert S.tuning()["tile"] == 0
