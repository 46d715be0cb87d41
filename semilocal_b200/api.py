"""Function-level API over the C ABI (host numpy arrays in, host numpy arrays out)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def _u8(x) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x))
    if a.dtype != np.uint8:
        if a.size and (a.min() < 0 or a.max() > 255):
            raise ValueError("uint8 symbols expected; use comb(..., ) with int32 input for wider alphabets")
        a = a.astype(np.uint8)
    return a


def _p(x: np.ndarray, t):
    return x.ctypes.data_as(t)


@dataclass
class Permutation:
    """Mirror of common::Permutation (R:common/include/Permutations/Matrices.h:16-96): both maps plus the
    (m, n) tags the hybrid attaches (:698-699)."""
    row_to_col: np.ndarray
    col_to_row: np.ndarray
    m: int = 0
    n: int = 0

    @property
    def rows(self) -> int:
        return len(self.row_to_col)

    @property
    def cols(self) -> int:
        return len(self.col_to_row)

    def get_col_by_row(self, r: int) -> int:
        return int(self.row_to_col[r])

    def get_row_by_col(self, c: int) -> int:
        return int(self.col_to_row[c])

    @staticmethod
    def from_row_to_col(r2c: np.ndarray, m: int = 0, n: int = 0) -> "Permutation":
        r2c = np.ascontiguousarray(r2c, dtype=np.int32)
        c2r = np.full(len(r2c), -1, dtype=np.int32)
        ok = r2c >= 0
        c2r[r2c[ok]] = np.nonzero(ok)[0].astype(np.int32)
        return Permutation(r2c, c2r, m, n)

    def __eq__(self, other) -> bool:
        return (isinstance(other, Permutation) and np.array_equal(self.row_to_col, other.row_to_col)
                and np.array_equal(self.col_to_row, other.col_to_row))


def comb(a, b, algo: int = _lib.ALGO_AUTO, tile: int = 0, band_rows: int = 0, want_col_to_row: bool = False,
         sa_cutoff: int = 0, lane_cols: int = 0) -> Tuple[np.ndarray, int]:
    """Braid (row->col, m+n int32) and global LLCS of the pair (a, b).  lane_cols picks the wavefront kernel of a
    lone pair (4: register tiles, 1: one column per lane step, 0: automatic)."""
    a_arr = np.ascontiguousarray(np.asarray(a))
    b_arr = np.ascontiguousarray(np.asarray(b))
    m, n = len(a_arr), len(b_arr)
    r2c = np.empty(m + n, dtype=np.int32)
    c2r = np.empty(m + n, dtype=np.int32) if want_col_to_row else None
    score = ctypes.c_int32(0)
    o = _lib.opts(algo, tile, tile, band_rows, sa_cutoff, lane_cols)
    wide = a_arr.dtype != np.uint8 or b_arr.dtype != np.uint8
    if wide and ((a_arr.size and (a_arr.min() < 0 or a_arr.max() > 255)) or
                 (b_arr.size and (b_arr.min() < 0 or b_arr.max() > 255))):
        a32 = np.ascontiguousarray(a_arr, dtype=np.int32)
        b32 = np.ascontiguousarray(b_arr, dtype=np.int32)
        check(lib().slcs_comb_i32(_p(a32, _i32p), m, _p(b32, _i32p), n, _p(r2c, _i32p),
                                  _p(c2r, _i32p) if c2r is not None else None, ctypes.byref(score), ctypes.byref(o)))
    else:
        au, bu = _u8(a_arr), _u8(b_arr)
        check(lib().slcs_comb_u8(_p(au, _u8p), m, _p(bu, _u8p), n, _p(r2c, _i32p),
                                 _p(c2r, _i32p) if c2r is not None else None, ctypes.byref(score), ctypes.byref(o)))
    if want_col_to_row:
        return r2c, int(score.value), c2r
    return r2c, int(score.value)


def lcs(a, b) -> int:
    au, bu = _u8(a), _u8(b)
    s = ctypes.c_int32(0)
    check(lib().slcs_lcs_u8(_p(au, _u8p), len(au), _p(bu, _u8p), len(bu), ctypes.byref(s)))
    return int(s.value)


def bitcomb_llcs(a, b) -> int:
    """LLCS by the bit-parallel kernel (symbols < 4)."""
    au, bu = _u8(a), _u8(b)
    s = ctypes.c_int32(0)
    check(lib().slcs_bitcomb_llcs_u8(_p(au, _u8p), len(au), _p(bu, _u8p), len(bu), ctypes.byref(s)))
    return int(s.value)


def hyyro_llcs(a, b) -> int:
    """LLCS by the bit-vector (Hyyro) kernel (symbols < 4)."""
    au, bu = _u8(a), _u8(b)
    s = ctypes.c_int32(0)
    check(lib().slcs_hyyro_llcs_u8(_p(au, _u8p), len(au), _p(bu, _u8p), len(bu), ctypes.byref(s)))
    return int(s.value)


def steady_ant(p, q, sa_cutoff: int = 0) -> np.ndarray:
    """Unit-Monge product r = p (.) q of two permutations (row->col int32)."""
    p = np.ascontiguousarray(p, dtype=np.int32)
    q = np.ascontiguousarray(q, dtype=np.int32)
    if len(p) != len(q):
        raise ValueError("p and q must have the same size")
    r = np.empty(len(p), dtype=np.int32)
    o = _lib.opts(sa_cutoff=sa_cutoff)
    check(lib().slcs_steady_ant(_p(p, _i32p), _p(q, _i32p), len(p), _p(r, _i32p), ctypes.byref(o)))
    return r


def staggered_glue(p, pm: int, pn: int, q, qm: int, qn: int, row_glue: bool) -> np.ndarray:
    p = np.ascontiguousarray(p, dtype=np.int32)
    q = np.ascontiguousarray(q, dtype=np.int32)
    k = pn if row_glue else pm
    out = np.empty(pm + pn + qm + qn - k, dtype=np.int32)
    check(lib().slcs_staggered_glue(_p(p, _i32p), pm, pn, _p(q, _i32p), qm, qn, int(bool(row_glue)),
                                    _p(out, _i32p)))
    return out


def check_permutation(perm) -> int:
    """Number of entries of `perm` that are out of range or repeat a value (0 for a permutation), on the GPU."""
    p = np.ascontiguousarray(perm, dtype=np.int32)
    bad = ctypes.c_int32(0)
    rc = lib().slcs_check_permutation(_p(p, _i32p), len(p), ctypes.byref(bad))
    if rc not in (0, 7):
        check(rc)
    return int(bad.value)


def window_scores(row_to_col, m: int, n: int, w: int) -> np.ndarray:
    """LCS(a, b[s..s+w)) for every window s = 0..n-w, read from the braid in one pass on the device."""
    r2c = np.ascontiguousarray(row_to_col, dtype=np.int32)
    out = np.empty(max(n - w + 1, 1), dtype=np.int32)
    check(lib().slcs_window_scores(_p(r2c, _i32p), m, n, w, _p(out, _i32p)))
    return out[:max(n - w + 1, 0)]


def duplicate_search(pattern, text, k: float, sparse: bool = False) -> List[Tuple[int, int, float]]:
    """Approximate copies of `pattern` in `text` as (start, end, score) intervals: the result vector of the
    reference's InteractiveDuplicateSearchSemiDense::find (sparse=False) or ...SemiSparse::find (sparse=True)
    (R:approximate_matching/ApproximateMatching.h:252-420) for the same symbols and k (0 < k <= 1), computed from
    one braid on the device."""
    p = np.asarray(pattern)
    t = np.asarray(text)
    suffix = "sparse_" if sparse else ""
    if p.dtype == np.uint8 and t.dtype == np.uint8:
        fn, ptr = getattr(lib(), f"slcs_duplicate_search_{suffix}u8"), _u8p
    else:
        p, t = p.astype(np.int32), t.astype(np.int32)
        fn, ptr = getattr(lib(), f"slcs_duplicate_search_{suffix}i32"), _i32p
    p, t = np.ascontiguousarray(p), np.ascontiguousarray(t)
    # the picked intervals do not overlap and are at least int(m k) long
    cap = len(t) // max(int(len(p) * k), 1) + 2 if k > 0 else 1
    while True:
        out = (_lib.Interval * cap)()
        cnt = ctypes.c_int32(0)
        check(fn(_p(p, ptr), len(p), _p(t, ptr), len(t), ctypes.c_double(k), out, cap, ctypes.byref(cnt)))
        if cnt.value <= cap:
            return [(out[i].start, out[i].end, out[i].score) for i in range(cnt.value)]
        cap = cnt.value


def scores(row_to_col, m: int, n: int, queries: Sequence[Tuple[int, int, int]]) -> np.ndarray:
    """Answer (kind, i, j) queries against a braid; see SLCS_Q_* in include/slcs.h."""
    r2c = np.ascontiguousarray(row_to_col, dtype=np.int32)
    nq = len(queries)
    qarr = (_lib.Query * max(nq, 1))()
    for k, (kind, i, j) in enumerate(queries):
        qarr[k].kind, qarr[k].i, qarr[k].j = int(kind), int(i), int(j)
    out = np.empty(max(nq, 1), dtype=np.int32)
    check(lib().slcs_scores(_p(r2c, _i32p), m, n, qarr, nq, _p(out, _i32p)))
    return out[:nq]


def batch_comb(pairs: Sequence[Tuple[np.ndarray, np.ndarray]], mode: int = 0, band_rows: int = 0
               ) -> Tuple[List[np.ndarray], np.ndarray]:
    """Braids and global scores of many independent pairs: mode 0 = one persistent batched launch,
    mode 1 = one launch per pair."""
    npairs = len(pairs)
    ms = np.array([len(a) for a, _ in pairs], dtype=np.int32)
    ns = np.array([len(b) for _, b in pairs], dtype=np.int32)
    a_off = np.zeros(npairs, dtype=np.int64)
    b_off = np.zeros(npairs, dtype=np.int64)
    if npairs:
        a_off[1:] = np.cumsum(ms[:-1], dtype=np.int64)
        b_off[1:] = np.cumsum(ns[:-1], dtype=np.int64)
    a_cat = np.ascontiguousarray(np.concatenate([_u8(a) for a, _ in pairs]) if npairs else np.zeros(1, np.uint8))
    b_cat = np.ascontiguousarray(np.concatenate([_u8(b) for _, b in pairs]) if npairs else np.zeros(1, np.uint8))
    total = int((ms.astype(np.int64) + ns).sum())
    out = np.empty(max(total, 1), dtype=np.int32)
    sc = np.zeros(max(npairs, 1), dtype=np.int32)
    o = _lib.opts(band_rows=band_rows)
    check(lib().slcs_batch_comb_u8(_p(a_cat, _u8p), _p(a_off, _i64p), _p(ms, _i32p), _p(b_cat, _u8p),
                                   _p(b_off, _i64p), _p(ns, _i32p), npairs, _p(out, _i32p), _p(sc, _i32p), mode,
                                   ctypes.byref(o)))
    res = []
    off = 0
    for i in range(npairs):
        sz = int(ms[i]) + int(ns[i])
        res.append(out[off:off + sz])
        off += sz
    return res, sc[:npairs]


class BatchPlan:
    """A reusable device-resident batch (include/slcs.h: slcs_batch_*).  upload() copies the concatenated
    strings (host numpy arrays, pinned or not), run() is the device-only step (optionally replayed from a
    CUDA graph), download() copies braids and scores back."""

    def __init__(self, ms, ns, mode: int = 0, band_rows: int = 0):
        self.ms = np.ascontiguousarray(ms, dtype=np.int32)
        self.ns = np.ascontiguousarray(ns, dtype=np.int32)
        self.npairs = len(self.ms)
        self.total = int((self.ms.astype(np.int64) + self.ns).sum())
        o = _lib.opts(band_rows=band_rows)
        h = ctypes.c_void_p()
        check(lib().slcs_batch_create(_p(self.ms, _i32p), _p(self.ns, _i32p), self.npairs, mode, ctypes.byref(o),
                                      ctypes.byref(h)))
        self.h = h

    def upload(self, a_cat: np.ndarray, a_off: np.ndarray, b_cat: np.ndarray, b_off: np.ndarray, stream=None):
        self._keep = (a_cat, b_cat)
        self.a_off = np.ascontiguousarray(a_off, dtype=np.int64)
        self.b_off = np.ascontiguousarray(b_off, dtype=np.int64)
        check(lib().slcs_batch_upload(self.h, a_cat.ctypes.data, _p(self.a_off, _i64p), b_cat.ctypes.data,
                                      _p(self.b_off, _i64p), stream))

    def run(self, use_graph: bool = False, stream=None):
        check(lib().slcs_batch_run(self.h, int(bool(use_graph)), stream))

    def download(self, out: np.ndarray, scores: np.ndarray, stream=None):
        check(lib().slcs_batch_download(self.h, out.ctypes.data, scores.ctypes.data, stream))

    def kernel_ms(self) -> float:
        v = ctypes.c_float(0)
        check(lib().slcs_batch_kernel_ms(self.h, ctypes.byref(v)))
        return float(v.value)

    def info(self):
        cells, h2d, d2h = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        launches = ctypes.c_int32(0)
        check(lib().slcs_batch_info(self.h, ctypes.byref(cells), ctypes.byref(launches), ctypes.byref(h2d),
                                    ctypes.byref(d2h)))
        return {"cells": cells.value, "launches": launches.value, "h2d_bytes": h2d.value, "d2h_bytes": d2h.value}

    def close(self):
        if getattr(self, "h", None):
            lib().slcs_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def concat_pairs(pairs):
    """Concatenate (a, b) pairs into the batch layout: a_cat, a_off, ms, b_cat, b_off, ns."""
    ms = np.array([len(a) for a, _ in pairs], dtype=np.int32)
    ns = np.array([len(b) for _, b in pairs], dtype=np.int32)
    a_off = np.zeros(len(pairs), dtype=np.int64)
    b_off = np.zeros(len(pairs), dtype=np.int64)
    if len(pairs):
        a_off[1:] = np.cumsum(ms[:-1], dtype=np.int64)
        b_off[1:] = np.cumsum(ns[:-1], dtype=np.int64)
    a_cat = np.ascontiguousarray(np.concatenate([_u8(a) for a, _ in pairs])) if len(pairs) else np.zeros(1, np.uint8)
    b_cat = np.ascontiguousarray(np.concatenate([_u8(b) for _, b in pairs])) if len(pairs) else np.zeros(1, np.uint8)
    return a_cat, a_off, ms, b_cat, b_off, ns


class PairPlan:
    """A reusable single-pair plan on device buffers (include/slcs.h: slcs_pair_plan_*): kind is ALGO_WAVEFRONT,
    ALGO_HYBRID, PLAN_BITPARALLEL or PLAN_HYYRO.  run() takes device pointers (ints) and a stream handle."""

    def __init__(self, m: int, n: int, kind: int, tile: int = 0, band_rows: int = 0, lane_cols: int = 0):
        o = _lib.opts(kind if kind not in (_lib.PLAN_BITPARALLEL, _lib.PLAN_HYYRO) else 0, tile, tile, band_rows, 0,
                      lane_cols)
        h = ctypes.c_void_p()
        check(lib().slcs_pair_plan_create(m, n, kind, ctypes.byref(o), ctypes.byref(h)))
        self.h, self.m, self.n, self.kind = h, m, n, kind

    def run(self, d_a: int, d_b: int, d_r2c, d_score, use_graph: bool = False, stream=None):
        check(lib().slcs_pair_plan_run(self.h, d_a, d_b, d_r2c, d_score, int(bool(use_graph)), stream))

    def check(self, stream=None):
        check(lib().slcs_pair_plan_check(self.h, stream))

    def kernel_ms(self) -> float:
        v = ctypes.c_float(0)
        check(lib().slcs_pair_plan_kernel_ms(self.h, ctypes.byref(v)))
        return float(v.value)

    def launches(self) -> int:
        v = ctypes.c_int32(0)
        check(lib().slcs_pair_plan_launches(self.h, ctypes.byref(v)))
        return int(v.value)

    def close(self):
        if getattr(self, "h", None):
            lib().slcs_pair_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SteadyAntPlan:
    """A reusable steady-ant plan of size n (include/slcs.h: slcs_sa_plan_*)."""

    def __init__(self, n: int):
        h = ctypes.c_void_p()
        check(lib().slcs_sa_plan_create(n, ctypes.byref(h)))
        self.h, self.n = h, n

    def run(self, d_p: int, d_q: int, d_r: int, use_graph: bool = False, stream=None):
        check(lib().slcs_sa_plan_run(self.h, d_p, d_q, d_r, int(bool(use_graph)), stream))

    def check(self, stream=None):
        check(lib().slcs_sa_plan_check(self.h, stream))

    def launches(self) -> int:
        v = ctypes.c_int32(0)
        check(lib().slcs_sa_plan_launches(self.h, ctypes.byref(v)))
        return int(v.value)

    def close(self):
        if getattr(self, "h", None):
            lib().slcs_sa_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop over the C ABI (slcs_server_*): continuous batching of comparison requests on one GPU.

    submit() copies the pair and returns a ticket at once; a worker thread inside the library admits requests
    by a device-memory budget, overlaps their launches on the device and keeps finished braids resident;
    poll() returns finished results.  Results are identical alone and in any mix.
    """

    def __init__(self, mem_budget: int = 0, small_streams: int = 0, big_cells: int = 0, max_batch: int = 0,
                 big_warps: int = 0, small_warps: int = 0, band_rows: int = 0, max_pending: int = 0,
                 big_streams: int = 0):
        self._h = ctypes.c_void_p()
        o = _lib.ServerOpts(mem_budget=mem_budget, max_pending=max_pending, small_streams=small_streams,
                            big_cells=big_cells, big_warps=big_warps, small_warps=small_warps, max_batch=max_batch,
                            band_rows=band_rows, big_streams=big_streams)
        _lib.check(_lib.lib().slcs_server_create(ctypes.byref(o), ctypes.byref(self._h)))
        self._sizes = {}

    def submit(self, a, b, query: Tuple[int, int, int] = (0, 0, 0)) -> int:
        a, b = _u8(a), _u8(b)
        t = ctypes.c_uint64()
        q = _lib.Query(*query)
        _lib.check(_lib.lib().slcs_server_submit(self._h, _p(a, _u8p), len(a), _p(b, _u8p),
                                                 len(b), ctypes.byref(q), ctypes.byref(t)))
        self._sizes[t.value] = (len(a), len(b))
        return t.value

    def poll(self, cap: int = 1024, timeout_ms: int = 0):
        buf = (_lib.Result * max(cap, 1))()
        cnt = ctypes.c_int32()
        _lib.check(_lib.lib().slcs_server_poll(self._h, buf, cap, ctypes.byref(cnt), timeout_ms))
        out = []
        for r in buf[:cnt.value]:
            out.append({"ticket": r.ticket, "status": r.status, "score": r.score, "m": r.m, "n": r.n,
                        "query": (r.query.kind, r.query.i, r.query.j), "t_submit": r.t_submit,
                        "t_admit": r.t_admit, "t_done": r.t_done})
        return out

    def wait_all(self, tickets, timeout_s: float = 600.0):
        """Polls until every ticket has a result; returns {ticket: result}."""
        import time
        want, got = set(tickets), {}
        t_end = time.monotonic() + timeout_s
        while want - set(got):
            if time.monotonic() > t_end:
                raise TimeoutError(f"{len(want - set(got))} requests unfinished")
            for r in self.poll(timeout_ms=50):
                got[r["ticket"]] = r
        return got

    def query(self, ticket: int, queries: Sequence[Tuple[int, int, int]]) -> np.ndarray:
        qs = (_lib.Query * max(len(queries), 1))(*[_lib.Query(*q) for q in queries])
        out = np.zeros(len(queries), np.int32)
        _lib.check(_lib.lib().slcs_server_query(self._h, ticket, qs, len(queries), _p(out, _i32p)))
        return out

    def window_scores(self, ticket: int, w: int) -> np.ndarray:
        """LCS(a, b[s..s+w)) for every window of the resident braid of `ticket`."""
        m, n = self._sizes[ticket]
        out = np.zeros(max(n - w + 1, 1), np.int32)
        _lib.check(_lib.lib().slcs_server_window(self._h, ticket, w, _p(out, _i32p)))
        return out[:max(n - w + 1, 0)]

    def braid(self, ticket: int) -> np.ndarray:
        m, n = self._sizes[ticket]
        out = np.zeros(max(m + n, 1), np.int32)
        _lib.check(_lib.lib().slcs_server_braid(self._h, ticket, _p(out, _i32p)))
        return out[:m + n]

    def release(self, ticket: int) -> None:
        _lib.check(_lib.lib().slcs_server_release(self._h, ticket))

    def stats(self) -> dict:
        st = _lib.ServerStats()
        _lib.check(_lib.lib().slcs_server_stats_get(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _lib.ServerStats._fields_}

    def now(self) -> float:
        return _lib.lib().slcs_server_now(self._h)

    def close(self) -> None:
        if self._h:
            _lib.lib().slcs_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tuning() -> dict:
    """The current device's tuning table (zeros = built-in defaults)."""
    t = _lib.Tuning()
    check(lib().slcs_tuning_get(ctypes.byref(t)))
    return {"band_rows_batch": list(t.band_rows_batch), "band_rows_single": list(t.band_rows_single),
            "tile": t.tile, "sa_cutoff": t.sa_cutoff}


def set_tuning(table: Optional[dict]) -> None:
    """Installs a tuning table (None restores the built-in defaults)."""
    if table is None:
        check(lib().slcs_tuning_set(None))
        return
    t = _lib.Tuning()
    for i, v in enumerate(table.get("band_rows_batch", [])[:32]):
        t.band_rows_batch[i] = int(v)
    for i, v in enumerate(table.get("band_rows_single", [])[:32]):
        t.band_rows_single[i] = int(v)
    t.tile = int(table.get("tile", 0))
    t.sa_cutoff = int(table.get("sa_cutoff", 0))
    check(lib().slcs_tuning_set(ctypes.byref(t)))


def autotune(flags: int = _lib.TUNE_ALL, cache: Optional[str] = None) -> dict:
    """Measures and installs the tuning table of the current device.  With `cache` (a JSON file path) a table
    saved for the same device name and library version is loaded instead of measuring, and a measured table
    is saved there."""
    import json
    import os
    key = None
    if cache:
        try:
            import torch
            key = f"{torch.cuda.get_device_name()}|v{lib().slcs_version()}"
        except Exception:
            key = f"device|v{lib().slcs_version()}"
        if os.path.exists(cache):
            try:
                with open(cache) as f:
                    saved = json.load(f)
                if key in saved:
                    set_tuning(saved[key])
                    return saved[key]
            except (OSError, ValueError):
                pass
    t = _lib.Tuning()
    check(lib().slcs_autotune(flags, ctypes.byref(t)))
    table = tuning()
    if cache:
        saved = {}
        if os.path.exists(cache):
            try:
                with open(cache) as f:
                    saved = json.load(f)
            except (OSError, ValueError):
                saved = {}
        saved[key] = table
        with open(cache, "w") as f:
            json.dump(saved, f)
    return table
