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


def test_noalloc_rejects_sizes_beyond_its_scratch(engine):
    S = engine
    rc = S.lib().slcs_comb_u8_dev_noalloc(ctypes.c_void_p(1), 9_000_000, ctypes.c_void_p(1), 10, ctypes.c_void_p(1),
                                          ctypes.c_void_p(1), None, None)
    assert rc == 5   # SLCS_ERR_TOO_LARGE, rejected before any device work
    assert b"8388608" in S.lib().slcs_last_error()
