"""ctypes face of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The libraries wrapped:
  * liboracle.so   -- the C restatement in oracle/slcs_oracle.c (always built; `make -C oracle`);
  * _ref/libslcs_ref.so -- the reference's own headers compiled by oracle/build_ref.sh (present when the
    reference sources were available at build time; the file travels with the repository snapshot);
  * _ref/libslcs_ref_am.so -- the reference's approximate pattern search, compiled the same way;
  * _ref/libslcs_ref_legacy.so -- the reference's legacy combing, steady ant and hybrid (second oracle).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libslcs_ref.so")
REF_AM_PATH = os.path.join(HERE, "_ref", "libslcs_ref_am.so")
REF_LEGACY_PATH = os.path.join(HERE, "_ref", "libslcs_ref_legacy.so")

_lock = threading.Lock()
_lib = None
_ref = None
_ref_tried = False

_i32p = ctypes.POINTER(ctypes.c_int32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)
_ref_am = None
_ref_legacy = None


def build() -> str:
    """(Re)build liboracle.so if it is missing or older than its sources."""
    srcs = [os.path.join(HERE, f) for f in ("slcs_oracle.c", "amatch_oracle.cpp")]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(LIB_PATH) < os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(LIB_PATH)
            L.slo_comb_rowmajor.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, _i32p]
            L.slo_comb_antidiag.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, _i32p]
            L.slo_rotate180.argtypes = [_i32p, ctypes.c_int, _i32p]
            L.slo_semilocal_matrix.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, _i32p]
            L.slo_kernel_from_matrix.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, _i32p]
            L.slo_global_score.argtypes = [_i32p, ctypes.c_int, ctypes.c_int]
            L.slo_semilocal_entry.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            L.slo_lcs_dp.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int]
            L.slo_braid_mult_naive.argtypes = [_i32p, _i32p, ctypes.c_int, _i32p]
            L.slo_steady_ant.argtypes = [_i32p, _i32p, ctypes.c_int, _i32p]
            L.slo_staggered.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p]
            L.slo_hybrid_iterative.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, _i32p]
            L.slo_encode_u64.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, _u64p]
            L.slo_encode_reverse_u64.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, _u64p]
            L.slo_bit_llcs_nary_u64.argtypes = [_u64p, ctypes.c_int, _u64p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            L.slo_bit_llcs_binary_u64.argtypes = [_u64p, ctypes.c_int, _u64p, ctypes.c_int, ctypes.c_int]
            L.slo_comb_score.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int]
            L.slo_hyyro_llcs.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int]
            L.slo_duplicate_search.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_double, _i32p, _i32p,
                                               _f64p, ctypes.c_int]
            L.slo_duplicate_search_sparse.argtypes = L.slo_duplicate_search.argtypes
            _lib = L
    return _lib


def ref():
    """The reference-compiled library, or None when it was not built."""
    global _ref, _ref_tried
    with _lock:
        if not _ref_tried:
            _ref_tried = True
            if os.path.exists(REF_PATH):
                R = ctypes.CDLL(REF_PATH)
                R.ref_comb_simple.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, _i32p]
                R.ref_comb_openmp.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, _i32p]
                R.ref_comb_dummy.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, _i32p]
                R.ref_comb_combined.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, _i32p]
                R.ref_hybrid_iterative.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p]
                R.ref_hybrid_recursive.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_int, _i32p]
                R.ref_braid_naive.argtypes = [_i32p, _i32p, ctypes.c_int, _i32p]
                R.ref_braid_simple.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, _i32p]
                R.ref_braid_seq.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, _i32p]
                R.ref_braid_omp.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p]
                R.ref_precalc_warm.argtypes = [ctypes.c_int]
                R.ref_staggered.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, _i32p]
                R.ref_lcs_seqmem.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int]
                R.ref_lcs_dummy.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int]
                R.ref_lcs_by_semilocal.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int]
                R.ref_bit_nary_u64.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
                R.ref_bit_binary_u64.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int]
                R.ref_hyyro_u64.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int]
                _ref = R
    return _ref


def _i32(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


def _p(x: np.ndarray):
    return x.ctypes.data_as(_i32p)


def _pu(x: np.ndarray):
    return x.ctypes.data_as(_u64p)


# --------------------------------------------------------------------------------------------------
# C restatement
# --------------------------------------------------------------------------------------------------

def comb_rowmajor(a, b) -> np.ndarray:
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    lib().slo_comb_rowmajor(_p(a), len(a), _p(b), len(b), _p(out))
    return out


def comb_antidiag(a, b, threads: int = 1) -> np.ndarray:
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    lib().slo_comb_antidiag(_p(a), len(a), _p(b), len(b), threads, _p(out))
    return out


def rotate180(perm) -> np.ndarray:
    perm = _i32(perm)
    out = np.full(len(perm), -1, dtype=np.int32)
    lib().slo_rotate180(_p(perm), len(perm), _p(out))
    return out


def semilocal_matrix(a, b) -> np.ndarray:
    a, b = _i32(a), _i32(b)
    s = len(a) + len(b) + 1
    H = np.empty(s * s, dtype=np.int32)
    lib().slo_semilocal_matrix(_p(a), len(a), _p(b), len(b), _p(H))
    return H.reshape(s, s)


def kernel_from_matrix(H, m: int, n: int) -> np.ndarray:
    H = _i32(H).ravel()
    out = np.empty(m + n, dtype=np.int32)
    lib().slo_kernel_from_matrix(_p(H), m, n, _p(out))
    return out


def comb_dp(a, b) -> np.ndarray:
    """Braid from the DP definition of the semi-local matrix (small sizes only)."""
    return kernel_from_matrix(semilocal_matrix(a, b), len(a), len(b))


def global_score(perm, m: int, n: int) -> int:
    perm = _i32(perm)
    return int(lib().slo_global_score(_p(perm), m, n))


def semilocal_entry(perm, m: int, n: int, i: int, j: int) -> int:
    perm = _i32(perm)
    return int(lib().slo_semilocal_entry(_p(perm), m, n, i, j))


def lcs_dp(a, b) -> int:
    a, b = _i32(a), _i32(b)
    return int(lib().slo_lcs_dp(_p(a), len(a), _p(b), len(b)))


def braid_naive(p, q) -> np.ndarray:
    p, q = _i32(p), _i32(q)
    out = np.empty(len(p), dtype=np.int32)
    lib().slo_braid_mult_naive(_p(p), _p(q), len(p), _p(out))
    return out


def steady_ant(p, q) -> np.ndarray:
    p, q = _i32(p), _i32(q)
    out = np.empty(len(p), dtype=np.int32)
    rc = lib().slo_steady_ant(_p(p), _p(q), len(p), _p(out))
    if rc != 0:
        raise RuntimeError("oracle steady ant failed")
    return out


def staggered(p, pm: int, pn: int, q, qm: int, qn: int, row_glue: bool) -> np.ndarray:
    p, q = _i32(p), _i32(q)
    k = pn if row_glue else pm
    out = np.empty(pm + pn + qm + qn - k, dtype=np.int32)
    rc = lib().slo_staggered(_p(p), pm + pn, _p(q), qm + qn, k, int(bool(row_glue)), _p(out))
    if rc != 0:
        raise RuntimeError("oracle staggered glue failed")
    return out


def hybrid_iterative(a, b, threads: int = 1, cols: int = 4096, rows: int = 4096) -> np.ndarray:
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    rc = lib().slo_hybrid_iterative(_p(a), len(a), _p(b), len(b), threads, cols, rows, _p(out))
    if rc != 0:
        raise RuntimeError("oracle hybrid failed")
    return out


def encode_u64(s, bps: int) -> np.ndarray:
    s = _i32(s)
    S = 64 // bps
    out = np.zeros(max(1, (len(s) + S - 1) // S), dtype=np.uint64)
    w = lib().slo_encode_u64(_p(s), len(s), bps, _pu(out))
    return out[:w]


def encode_reverse_u64(s, bps: int) -> np.ndarray:
    s = _i32(s)
    S = 64 // bps
    out = np.zeros(max(1, (len(s) + S - 1) // S), dtype=np.uint64)
    w = lib().slo_encode_reverse_u64(_p(s), len(s), bps, _pu(out))
    return out[:w]


def bit_llcs_nary(a, b, bps: int = 2) -> int:
    """Reference-domain n-ary bit combing (lengths multiples of 64/bps, |a| <= |b|)."""
    ar = encode_reverse_u64(a, bps)
    be = encode_u64(b, bps)
    return int(lib().slo_bit_llcs_nary_u64(_pu(ar), len(ar), _pu(be), len(be), len(a), bps))


def bit_llcs_binary(a, b) -> int:
    ar = encode_reverse_u64(a, 1)
    be = encode_u64(b, 1)
    return int(lib().slo_bit_llcs_binary_u64(_pu(ar), len(ar), _pu(be), len(be), len(a)))


def hyyro_llcs(a, b) -> int:
    """Bit-vector LLCS (Allison-Dix / Hyyro recurrence) over 64-bit words of `a`, looping over `b`."""
    a, b = _i32(a), _i32(b)
    return int(lib().slo_hyyro_llcs(_p(a), len(a), _p(b), len(b)))


def comb_score(a, b, threads: int = 1) -> int:
    a, b = _i32(a), _i32(b)
    return int(lib().slo_comb_score(_p(a), len(a), _p(b), len(b), threads))


# --------------------------------------------------------------------------------------------------
# Reference-compiled checker (None-returning when absent)
# --------------------------------------------------------------------------------------------------

def ref_available() -> bool:
    return ref() is not None


def ref_comb(a, b, kind: str = "simple", threads: int = 1) -> np.ndarray:
    R = ref()
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    if kind == "simple":
        R.ref_comb_simple(_p(a), len(a), _p(b), len(b), _p(out))
    elif kind == "openmp":
        R.ref_comb_openmp(_p(a), len(a), _p(b), len(b), threads, _p(out))
    elif kind == "dummy":
        R.ref_comb_dummy(_p(a), len(a), _p(b), len(b), _p(out))
    elif kind == "combined":
        R.ref_comb_combined(_p(a), len(a), _p(b), len(b), threads, _p(out))
    else:
        raise ValueError(kind)
    return out


def ref_hybrid_iterative(a, b, threads=1, cols=4096, rows=4096, precalc=0) -> np.ndarray:
    R = ref()
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    R.ref_hybrid_iterative(_p(a), len(a), _p(b), len(b), threads, cols, rows, precalc, _p(out))
    return out


def ref_hybrid_recursive(a, b, parallel_depth=1, depth=6, sum_bound=400) -> np.ndarray:
    R = ref()
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    R.ref_hybrid_recursive(_p(a), len(a), _p(b), len(b), parallel_depth, depth, sum_bound, _p(out))
    return out


def ref_braid(p, q, kind: str = "seq", precalc: int = 0, depth: int = 3) -> np.ndarray:
    R = ref()
    p, q = _i32(p), _i32(q)
    out = np.empty(len(p), dtype=np.int32)
    if kind == "naive":
        R.ref_braid_naive(_p(p), _p(q), len(p), _p(out))
    elif kind == "simple":
        R.ref_braid_simple(_p(p), _p(q), len(p), precalc, _p(out))
    elif kind == "seq":
        R.ref_braid_seq(_p(p), _p(q), len(p), precalc, _p(out))
    elif kind == "omp":
        R.ref_braid_omp(_p(p), _p(q), len(p), depth, precalc, _p(out))
    else:
        raise ValueError(kind)
    return out


def ref_staggered(p, pm, pn, q, qm, qn, row_glue: bool) -> np.ndarray:
    R = ref()
    p, q = _i32(p), _i32(q)
    k = pn if row_glue else pm
    out = np.empty(pm + pn + qm + qn - k, dtype=np.int32)
    R.ref_staggered(_p(p), pm, pn, _p(q), qm, qn, int(bool(row_glue)), _p(out))
    return out


def ref_lcs(a, b, kind: str = "seqmem") -> int:
    R = ref()
    a, b = _i32(a), _i32(b)
    f = {"seqmem": R.ref_lcs_seqmem, "dummy": R.ref_lcs_dummy, "semilocal": R.ref_lcs_by_semilocal}[kind]
    return int(f(_p(a), len(a), _p(b), len(b)))


def ref_bit_nary(a, b, alphabet: int = 4, threads: int = 1) -> int:
    R = ref()
    a, b = _i32(a), _i32(b)
    return int(R.ref_bit_nary_u64(_p(a), len(a), _p(b), len(b), alphabet, threads))


def ref_hyyro(vec, seq, threads: int = 1) -> int:
    """The reference's lllcs_hyyro (bit vector over `vec`, loop over `seq`; threads > 1: its anti-diagonal form,
    which wants len(seq) > words of vec)."""
    R = ref()
    vec, seq = _i32(vec), _i32(seq)
    return int(R.ref_hyyro_u64(_p(vec), len(vec), _p(seq), len(seq), threads))


def ref_bit_binary(a, b, threads: int = 1) -> int:
    R = ref()
    a, b = _i32(a), _i32(b)
    return int(R.ref_bit_binary_u64(_p(a), len(a), _p(b), len(b), threads))


# --------------------------------------------------------------------------------------------------
# Approximate pattern search: the restatement and the reference's own code
# --------------------------------------------------------------------------------------------------

def _intervals(fn, pattern, text, k):
    p, t = _i32(pattern), _i32(text)
    cap = max(len(t), 1)
    st, en = np.empty(cap, np.int32), np.empty(cap, np.int32)
    sc = np.empty(cap, np.float64)
    cnt = fn(_p(p), len(p), _p(t), len(t), ctypes.c_double(k), _p(st), _p(en), sc.ctypes.data_as(_f64p), cap)
    if cnt < 0:
        raise ValueError("bad arguments")
    return [(int(st[i]), int(en[i]), float(sc[i])) for i in range(cnt)]


def duplicate_search(pattern, text, k: float, sparse: bool = False):
    """The restatement of InteractiveDuplicateSearchSemiDense::find, or ...SemiSparse::find with sparse=True
    (oracle/amatch_oracle.cpp)."""
    return _intervals(lib().slo_duplicate_search_sparse if sparse else lib().slo_duplicate_search, pattern, text, k)


def ref_am():
    """The reference-compiled approximate pattern search, or None when it was not built."""
    global _ref_am
    with _lock:
        if _ref_am is None and os.path.exists(REF_AM_PATH):
            R = ctypes.CDLL(REF_AM_PATH)
            for f in (R.ref_dup_search_dense, R.ref_dup_search_sparse):
                f.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_double, _i32p, _i32p, _f64p, ctypes.c_int]
            _ref_am = R
    return _ref_am


def ref_duplicate_search(pattern, text, k: float, kind: str = "dense"):
    """The reference's own InteractiveDuplicateSearchSemiDense (kind "dense") or ...SemiSparse ("sparse")."""
    R = ref_am()
    return _intervals(R.ref_dup_search_dense if kind == "dense" else R.ref_dup_search_sparse, pattern, text, k)


# --------------------------------------------------------------------------------------------------
# The reference's legacy implementations (second oracle; oracle/ref_legacy_shim.cpp)
# --------------------------------------------------------------------------------------------------

def ref_legacy():
    """The reference's legacy combing / steady ant / hybrid (R:semi_local.h, R:unit_monge_mult/steady_ant.h)
    compiled from its sources, or None when it was not built."""
    global _ref_legacy
    with _lock:
        if _ref_legacy is None and os.path.exists(REF_LEGACY_PATH):
            R = ctypes.CDLL(REF_LEGACY_PATH)
            R.ref_legacy_sticky_braid_mpi.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int, _i32p]
            R.ref_legacy_steady_ant.argtypes = [_i32p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i32p]
            R.ref_legacy_hybrid_iterative.argtypes = [_i32p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_int, _i32p]
            _ref_legacy = R
    return _ref_legacy


def legacy_comb(a, b, threads: int = 1) -> np.ndarray:
    """semi_local::sticky_braid_mpi<int, false, false> (R:semi_local.h:212-276)."""
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    ref_legacy().ref_legacy_sticky_braid_mpi(_p(a), len(a), _p(b), len(b), threads, _p(out))
    return out


def legacy_steady_ant(p, q, nested_lvls: int = 3, precalc: int = 5) -> np.ndarray:
    """steady_ant_parallel_wrapper (R:unit_monge_mult/steady_ant.h:811-844)."""
    p, q = _i32(p), _i32(q)
    out = np.empty(len(p), dtype=np.int32)
    ref_legacy().ref_legacy_steady_ant(_p(p), _p(q), len(p), nested_lvls, precalc, _p(out))
    return out


def legacy_hybrid_iterative(a, b, threads: int = 4, precalc: int = 5) -> np.ndarray:
    """semi_local::hybrid_iterative_wrapper<false> (R:semi_local.h:740-790): symbols as unsigned short."""
    a, b = _i32(a), _i32(b)
    out = np.empty(len(a) + len(b), dtype=np.int32)
    ref_legacy().ref_legacy_hybrid_iterative(_p(a), len(a), _p(b), len(b), threads, precalc, _p(out))
    return out
