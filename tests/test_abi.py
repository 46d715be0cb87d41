"""CPU checks of the C ABI: the library loads without a GPU and exports every function include/slcs.h
declares; calls without a device fail loudly (SLCS_ERR_NO_DEVICE), never silently on the CPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "slcs.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(slcs_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["slcs_comb_u8", "slcs_steady_ant", "slcs_bitcomb_llcs_u8", "slcs_scores", "slcs_batch_comb_u8",
                 "slcs_staggered_glue", "slcs_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from semilocal_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    from semilocal_b200 import _lib
    names = set(declared_functions()) - {"slcs_last_error"}
    covered = set(_lib.SIGNATURES) | set(_lib.OTHER_SIGNATURES)
    assert names <= covered, sorted(names - covered)


def test_no_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    import semilocal_b200 as S
    with pytest.raises(S.SlcsError) as e:
        S.comb(np.array([1, 2, 3], np.uint8), np.array([1, 2], np.uint8))
    assert e.value.code == 6
    with pytest.raises(S.SlcsError):
        S.steady_ant(np.array([1, 0], np.int32), np.array([0, 1], np.int32))
    with pytest.raises(S.SlcsError) as e:
        S.Server()
    assert e.value.code == 6


def test_struct_layouts_match_header():
    """The ctypes mirrors have the sizes the C structs have (x86-64 ABI)."""
    from semilocal_b200 import _lib
    assert ctypes.sizeof(_lib.Query) == 12
    assert ctypes.sizeof(_lib.Opts) == 32
    assert ctypes.sizeof(_lib.ServerOpts) == 72
    assert ctypes.sizeof(_lib.Result) == 64
    assert ctypes.sizeof(_lib.ServerStats) == 96
    assert ctypes.sizeof(_lib.Tuning) == 288
