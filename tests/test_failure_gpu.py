"""Failure detection on the GPU without a fault: a combing band waits on a progress counter that nothing sets;
its bounded wait must give up (about 2 s of the GPU timer), the engine must report SLCS_ERR_TIMEOUT, and the
next calls must work and stay exact."""
import ctypes
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_engine_stays_usable(engine, oracle):
    import semilocal_b200 as S
    st = ctypes.c_int32(-1)
    t0 = time.monotonic()
    S._lib.check(S.lib().slcs_selftest_wait_timeout(ctypes.byref(st)))
    dt = time.monotonic() - t0
    assert st.value == 4, st.value            # SLCS_ERR_TIMEOUT
    assert 1.0 < dt < 30.0, dt                # the limit is about 2 s of GPU time
    a = np.random.default_rng(7).integers(0, 4, 3000).astype(np.uint8)
    b = np.random.default_rng(8).integers(0, 4, 2500).astype(np.uint8)
    r2c, score = S.comb(a, b, algo=S.ALGO_WAVEFRONT)
    assert np.array_equal(r2c, oracle.comb_antidiag(a, b))
    from semilocal_b200 import gen
    p, q = gen.steady_ant_pair(5000)
    assert np.array_equal(S.steady_ant(p, q), oracle.steady_ant(p, q))


def test_permutation_check(engine):
    import semilocal_b200 as S
    from semilocal_b200 import gen
    a, b = gen.hybrid_pair(1 << 14, seed=4)
    r2c, _ = S.comb(a, b, algo=S.ALGO_HYBRID, tile=1024)
    assert S.check_permutation(r2c) == 0
    bad = r2c.copy()
    bad[5] = bad[6]                   # one repeat
    bad[7] = len(bad) + 3             # one out of range
    assert S.check_permutation(bad) == 2
    p, q = gen.steady_ant_pair(1 << 16)
    assert S.check_permutation(S.steady_ant(p, q)) == 0
