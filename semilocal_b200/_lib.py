"""Loader of libslcs.so (the CUDA engine) and ctypes signatures of its C ABI (include/slcs.h).

The library is built in-tree for sm_100a by semilocal_b200/build.py.  There is no CPU fallback: if the
library cannot be loaded, or the device is not usable, every call raises SlcsError.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libslcs.so")

SLCS_OK = 0
ERRORS = {
    1: "SLCS_ERR_ARG", 2: "SLCS_ERR_CUDA", 3: "SLCS_ERR_OOM", 4: "SLCS_ERR_TIMEOUT", 5: "SLCS_ERR_TOO_LARGE",
    6: "SLCS_ERR_NO_DEVICE", 7: "SLCS_ERR_INTERNAL", 8: "SLCS_ERR_BUSY",
}

ALGO_AUTO, ALGO_WAVEFRONT, ALGO_HYBRID = 0, 1, 2
PLAN_BITPARALLEL = 3
PLAN_HYYRO = 4
Q_GLOBAL, Q_STRING_SUBSTRING, Q_PREFIX_SUFFIX, Q_SUFFIX_PREFIX, Q_SUBSTRING_STRING, Q_MATRIX = range(6)


class SlcsError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_int), ("tile_rows", ctypes.c_int), ("tile_cols", ctypes.c_int),
                ("band_rows", ctypes.c_int), ("sa_cutoff", ctypes.c_int), ("lane_cols", ctypes.c_int),
                ("reserved", ctypes.c_int * 2)]


class Query(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("i", ctypes.c_int32), ("j", ctypes.c_int32)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("mem_budget", ctypes.c_int64), ("max_pending", ctypes.c_int32), ("small_streams", ctypes.c_int32),
                ("big_cells", ctypes.c_int64), ("big_warps", ctypes.c_int32), ("small_warps", ctypes.c_int32),
                ("max_batch", ctypes.c_int32), ("band_rows", ctypes.c_int32), ("big_streams", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 7)]


class Result(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("status", ctypes.c_int32), ("score", ctypes.c_int32),
                ("m", ctypes.c_int32), ("n", ctypes.c_int32), ("query", Query), ("pad", ctypes.c_int32),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double)]


class Interval(ctypes.Structure):
    """slcs_interval: [start, end) of the text and its score."""
    _fields_ = [("start", ctypes.c_int32), ("end", ctypes.c_int32), ("score", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("submitted", "completed", "rejected", "evicted", "resident",
                                             "resident_bytes", "used_bytes", "peak_bytes", "budget", "launches",
                                             "cells")] + [("pending", ctypes.c_int32), ("inflight", ctypes.c_int32)]


class Tuning(ctypes.Structure):
    _fields_ = [("band_rows_batch", ctypes.c_int32 * 32), ("band_rows_single", ctypes.c_int32 * 32),
                ("tile", ctypes.c_int32), ("sa_cutoff", ctypes.c_int32), ("reserved", ctypes.c_int32 * 6)]


TUNE_BANDS_BATCH, TUNE_BANDS_SINGLE, TUNE_TILE, TUNE_SA_CUTOFF, TUNE_ALL = 1, 2, 4, 8, 15

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p
_int = ctypes.c_int
_optp = ctypes.POINTER(Opts)
_qp = ctypes.POINTER(Query)

# name -> argtypes (all return int status except where noted)
SIGNATURES = {
    "slcs_version": [],
    "slcs_set_device": [_int],
    "slcs_release": [],
    "slcs_comb_u8": [_u8p, _int, _u8p, _int, _i32p, _i32p, _i32p, _optp],
    "slcs_comb_i32": [_i32p, _int, _i32p, _int, _i32p, _i32p, _i32p, _optp],
    "slcs_comb_u8_dev": [_vp, _int, _vp, _int, _vp, _vp, _vp, _optp, _vp],
    "slcs_comb_u8_dev_noalloc": [_vp, _int, _vp, _int, _vp, _vp, _vp, _vp],
    "slcs_lcs_u8": [_u8p, _int, _u8p, _int, _i32p],
    "slcs_bitcomb_llcs_u8": [_u8p, _int, _u8p, _int, _i32p],
    "slcs_bitcomb_llcs_u8_dev": [_vp, _int, _vp, _int, _vp, _vp],
    "slcs_hyyro_llcs_u8": [_u8p, _int, _u8p, _int, _i32p],
    "slcs_hyyro_llcs_u8_dev": [_vp, _int, _vp, _int, _vp, _vp],
    "slcs_steady_ant": [_i32p, _i32p, _int, _i32p, _optp],
    "slcs_steady_ant_dev": [_vp, _vp, _int, _vp, _optp, _vp],
    "slcs_sa_plan_create": [_int, ctypes.POINTER(_vp)],
    "slcs_sa_plan_run": [_vp, _vp, _vp, _vp, _int, _vp],
    "slcs_sa_plan_check": [_vp, _vp],
    "slcs_sa_plan_launches": [_vp, _i32p],
    "slcs_sa_plan_destroy": [_vp],
    "slcs_staggered_glue": [_i32p, _int, _int, _i32p, _int, _int, _int, _i32p],
    "slcs_scores": [_i32p, _int, _int, _qp, _int, _i32p],
    "slcs_scores_dev": [_vp, _int, _int, _vp, _int, _vp, _vp],
    "slcs_batch_comb_u8": [_u8p, _i64p, _i32p, _u8p, _i64p, _i32p, _int, _i32p, _i32p, _int, _optp],
    "slcs_batch_create": [_i32p, _i32p, _int, _int, _optp, ctypes.POINTER(_vp)],
    "slcs_batch_upload": [_vp, _vp, _i64p, _vp, _i64p, _vp],
    "slcs_batch_run": [_vp, _int, _vp],
    "slcs_batch_download": [_vp, _vp, _vp, _vp],
    "slcs_batch_kernel_ms": [_vp, ctypes.POINTER(ctypes.c_float)],
    "slcs_batch_info": [_vp, _i64p, _i32p, _i64p, _i64p],
    "slcs_batch_destroy": [_vp],
    "slcs_probe_cell_peak": [ctypes.POINTER(ctypes.c_double)],
    "slcs_pair_plan_create": [_int, _int, _int, _optp, ctypes.POINTER(_vp)],
    "slcs_pair_plan_run": [_vp, _vp, _vp, _vp, _vp, _int, _vp],
    "slcs_pair_plan_check": [_vp, _vp],
    "slcs_pair_plan_kernel_ms": [_vp, ctypes.POINTER(ctypes.c_float)],
    "slcs_pair_plan_launches": [_vp, _i32p],
    "slcs_pair_plan_destroy": [_vp],
    "slcs_server_create": [ctypes.POINTER(ServerOpts), ctypes.POINTER(_vp)],
    "slcs_server_submit": [_vp, _u8p, _int, _u8p, _int, _qp, ctypes.POINTER(ctypes.c_uint64)],
    "slcs_server_poll": [_vp, ctypes.POINTER(Result), _int, _i32p, _int],
    "slcs_server_query": [_vp, ctypes.c_uint64, _qp, _int, _i32p],
    "slcs_server_braid": [_vp, ctypes.c_uint64, _i32p],
    "slcs_server_release": [_vp, ctypes.c_uint64],
    "slcs_server_stats_get": [_vp, ctypes.POINTER(ServerStats)],
    "slcs_server_destroy": [_vp],
    "slcs_window_scores": [_i32p, _int, _int, _int, _i32p],
    "slcs_window_scores_dev": [_vp, _vp, _int, _int, _int, _vp, _vp],
    "slcs_duplicate_search_u8": [_u8p, _int, _u8p, _int, ctypes.c_double, ctypes.POINTER(Interval), _int, _i32p],
    "slcs_duplicate_search_i32": [_i32p, _int, _i32p, _int, ctypes.c_double, ctypes.POINTER(Interval), _int, _i32p],
    "slcs_duplicate_search_sparse_u8": [_u8p, _int, _u8p, _int, ctypes.c_double, ctypes.POINTER(Interval), _int,
                                        _i32p],
    "slcs_duplicate_search_sparse_i32": [_i32p, _int, _i32p, _int, ctypes.c_double, ctypes.POINTER(Interval), _int,
                                         _i32p],
    "slcs_server_window": [_vp, ctypes.c_uint64, _int, _i32p],
    "slcs_selftest_wait_timeout": [_i32p],
    "slcs_check_permutation": [_i32p, _int, _i32p],
    "slcs_check_permutation_dev": [_vp, _int, _i32p, _vp],
    "slcs_autotune": [_int, ctypes.POINTER(Tuning)],
    "slcs_tuning_get": [ctypes.POINTER(Tuning)],
    "slcs_tuning_set": [ctypes.POINTER(Tuning)],
}
# name -> (argtypes, restype) for entry points that do not return a status
OTHER_SIGNATURES = {
    "slcs_server_now": ([_vp], ctypes.c_double),
}

_lock = threading.Lock()
_lib = None


def _ensure_built() -> None:
    if os.path.exists(LIB_PATH):
        from . import build as _b
        if not _b.stale():
            return
        try:
            _b.build()
        except Exception:
            # a stale but present library still works; a rebuild failure is reported on the next build()
            return
        return
    from . import build as _b
    _b.build()


def lib() -> ctypes.CDLL:
    """The loaded engine library (built on first use when nvcc is available)."""
    global _lib
    with _lock:
        if _lib is None:
            _ensure_built()
            if not os.path.exists(LIB_PATH):
                raise SlcsError(6, f"libslcs.so not found at {LIB_PATH}; run semilocal_b200/build.py")
            L = ctypes.CDLL(LIB_PATH)
            for name, args in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = ctypes.c_int
            for name, (args, res) in OTHER_SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
            L.slcs_last_error.argtypes = []
            L.slcs_last_error.restype = ctypes.c_char_p
            _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != SLCS_OK:
        msg = lib().slcs_last_error()
        raise SlcsError(rc, msg.decode(errors="replace") if msg else "")


def opts(algo: int = ALGO_AUTO, tile_rows: int = 0, tile_cols: int = 0, band_rows: int = 0, sa_cutoff: int = 0,
         lane_cols: int = 0):
    o = Opts()
    o.algo, o.tile_rows, o.tile_cols, o.band_rows, o.sa_cutoff = algo, tile_rows, tile_cols, band_rows, sa_cutoff
    o.lane_cols = lane_cols
    return o
