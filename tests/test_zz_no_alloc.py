"""The allocation-free combing entry point (slcs_comb_u8_dev_noalloc) against the regular device entry
point (slcs_comb_u8_dev), called through the C ABI on torch-owned device buffers.

It exists for callers that cannot let the engine allocate device memory (a fixed device-memory budget
owned by the host, a plugin in an application whose allocator reserved the device memory up front, a
serving loop that must not touch the allocator); its scratch is a static device array shared by all calls.  Braids are integers,
so the tolerance is exact equality.  Two calls in a row check that the shared scratch is cleared between
calls.  This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

from semilocal_b200 import gen

pytestmark = pytest.mark.gpu


def _run(S, torch, fn_name, a, b, noalloc):
    m, n = len(a), len(b)
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    r2c = torch.full((m + n,), -7, dtype=torch.int32, device="cuda")
    c2r = torch.full((m + n,), -7, dtype=torch.int32, device="cuda")
    sc = torch.full((1,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    L = S.lib()
    if noalloc:
        rc = L.slcs_comb_u8_dev_noalloc(da.data_ptr(), m, db.data_ptr(), n, r2c.data_ptr(), c2r.data_ptr(),
                                        sc.data_ptr(), sh)
    else:
        o = S._lib.opts(S.ALGO_WAVEFRONT)
        rc = L.slcs_comb_u8_dev(da.data_ptr(), m, db.data_ptr(), n, r2c.data_ptr(), c2r.data_ptr(), sc.data_ptr(),
                                ctypes.byref(o), sh)
    S._lib.check(rc)
    torch.cuda.synchronize()
    return r2c.cpu().numpy(), c2r.cpu().numpy(), int(sc.item())


def test_noalloc_matches_regular_entry_point_twice(engine):
    import torch
    S = engine
    cases = [gen.plain_pair(3000, seed=21), (gen.uniform_string(5000, 4, 22, 1), gen.uniform_string(777, 4, 22, 2))]
    for a, b in cases:   # two calls in a row, different sizes: the shared scratch must not leak between them
        got = _run(S, torch, "noalloc", a, b, True)
        exp = _run(S, torch, "regular", a, b, False)
        assert np.array_equal(got[0], exp[0])
        assert np.array_equal(got[1], exp[1])
        assert got[2] == exp[2]


def test_noalloc_against_the_oracle_and_edges(engine, oracle):
    """The allocation-free call against the CPU oracle: the identity braid of an empty string on either side, and
    a pair long enough for 32-row lanes (1024-row bands) whose last band is padded."""
    import torch
    S = engine
    for m, n in [(0, 0), (0, 17), (23, 0), (1, 1), (131072 + 500, 3001)]:
        a, b = gen.uniform_string(m, 4, 23, 1), gen.uniform_string(n, 4, 23, 2)
        r2c, c2r, score = _run(S, torch, "noalloc", a, b, True)
        exp = oracle.comb_antidiag(a, b, 8)
        assert np.array_equal(r2c, exp), (m, n)
        assert np.array_equal(c2r[exp], np.arange(m + n)), (m, n)
        assert score == oracle.global_score(exp, m, n), (m, n)


def test_noalloc_call_allocates_no_device_memory(engine):
    """After its first call on the device (which resolves the scratch array's address), a call leaves the free
    device memory unchanged: nothing is allocated, not even from a pool."""
    import torch
    S = engine
    a, b = gen.uniform_string(70000, 4, 24, 1), gen.uniform_string(5000, 4, 24, 2)
    m, n = len(a), len(b)
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    r2c = torch.empty(m + n, dtype=torch.int32, device="cuda")
    c2r = torch.empty(m + n, dtype=torch.int32, device="cuda")
    sc = torch.empty(1, dtype=torch.int32, device="cuda")
    sh = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = S.lib()
    call = lambda: S._lib.check(L.slcs_comb_u8_dev_noalloc(da.data_ptr(), m, db.data_ptr(), n, r2c.data_ptr(),
                                                           c2r.data_ptr(), sc.data_ptr(), sh))
    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_its_scratch(engine):
    S = engine
    rc = S.lib().slcs_comb_u8_dev_noalloc(ctypes.c_void_p(1), 9_000_000, ctypes.c_void_p(1), 10, ctypes.c_void_p(1),
                                          ctypes.c_void_p(1), None, None)
    assert rc == 5   # SLCS_ERR_TOO_LARGE, rejected before any device work
    assert b"8388608" in S.lib().slcs_last_error()
