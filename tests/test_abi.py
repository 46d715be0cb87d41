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


def test_sizes_beyond_the_limit_are_rejected_before_device_work():
    """Every entry point taking a pair, a braid or a permutation refuses m + n (or n) >= 2^30 with
    SLCS_ERR_TOO_LARGE before it touches a device, so this holds on a host without a GPU too."""
    from semilocal_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    L.slcs_last_error.restype = ctypes.c_char_p
    big, p = 1 << 29, ctypes.c_void_p(16)   # m = n = 2^29: m + n = 2^30; p is never dereferenced
    q = _lib.Query()
    calls = {
        "slcs_comb_u8": lambda: L.slcs_comb_u8(p, big, p, big, p, None, None, None),
        "slcs_scores": lambda: L.slcs_scores(p, big, big, ctypes.byref(q), 1, p),
        "slcs_scores_dev": lambda: L.slcs_scores_dev(p, big, big, ctypes.byref(q), 1, p, None),
        "slcs_window_scores": lambda: L.slcs_window_scores(p, big, big, 5, p),
        "slcs_window_scores_dev": lambda: L.slcs_window_scores_dev(p, p, big, big, 5, p, None),
        "slcs_bitcomb_llcs_u8_dev": lambda: L.slcs_bitcomb_llcs_u8_dev(p, big, p, big, p, None),
        "slcs_hyyro_llcs_u8_dev": lambda: L.slcs_hyyro_llcs_u8_dev(p, big, p, big, p, None),
        "slcs_staggered_glue": lambda: L.slcs_staggered_glue(p, big, big, p, big, big, 1, p),
        "slcs_steady_ant": lambda: L.slcs_steady_ant(p, p, 1 << 30, p, None),
        "slcs_comb_i32": lambda: L.slcs_comb_i32(p, big, p, big, p, None, None, None),
        "slcs_lcs_u8": lambda: L.slcs_lcs_u8(p, big, p, big, p),
    }
    for name, call in calls.items():
        assert call() == 5, (name, L.slcs_last_error())


def test_bad_arguments_are_status_codes_not_crashes():
    """Negative lengths and NULL buffers come back as SLCS_ERR_ARG from the host entry points, before anything is
    read, allocated or sent to a device."""
    from semilocal_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    L.slcs_last_error.restype = ctypes.c_char_p
    p = ctypes.c_void_p(16)   # never dereferenced
    score = ctypes.c_int32()
    assert L.slcs_lcs_u8(p, -5, p, 3, ctypes.byref(score)) == 1
    assert L.slcs_lcs_u8(None, 4, p, 3, ctypes.byref(score)) == 1
    assert L.slcs_comb_i32(None, 4, p, 3, p, None, None, None) == 1
    assert L.slcs_comb_i32(p, 4, None, 3, p, None, None, None) == 1
    assert L.slcs_comb_u8(p, -1, p, 3, p, None, None, None) == 1
    assert L.slcs_comb_u8_dev(p, 4, p, 3, None, None, None, None, None) == 1   # the device output is required
    assert L.slcs_comb_u8_dev(None, 4, p, 3, p, None, None, None, None) == 1


def test_int32_symbol_map(tmp_path):
    """The int32 combing entry point's symbol map (semilocal_b200/csrc/symbol_codes.h) applies exactly when the
    symbols span at most 256 values and keeps every (in)equality between them (tests/cpp/symbol_codes_check.cpp)."""
    import subprocess
    exe = str(tmp_path / "symbol_codes_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(ROOT, "semilocal_b200", "csrc"), os.path.join(ROOT, "tests", "cpp", "symbol_codes_check.cpp"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
