"""Strategy classes with the reference's interface shapes, backed by the CUDA engine.

Reference interfaces (R: = source/cpu/ of NikitaMishin/semilocal):
  semi_local::SemiLocalStrategy<Input>::compute(a, aSize, b, bSize, Permutation&)   R:include/SemiLocal/SemiLocalLCS.h:7-11
  common::BraidMultiplicationStrategy::multiply(P, Q, Permutation&)                 R:common/include/Permutations/MongeMultuplicationStrategy.h:18-21
  common::StaggeredStickyBraidMultiplication::staggeredStickyMultiplication<RowGlue> R:common/include/Permutations/MongeMultuplicationStrategy.h:679-758
  lcs::LCSStrategy<Input>::compute(a, sizeA, b, sizeB) -> int                        R:include/LCS/LCS.h:9-13
  lcs::LCSBySemiLocal                                                               R:include/LCS/LCS.h:216-238
Python returns the output instead of filling an out-parameter; errors raise SlcsError.
"""
from __future__ import annotations

import numpy as np

from . import _lib, api
from .api import Permutation


class SemiLocalStrategy:
    def compute(self, a, b) -> Permutation:  # pragma: no cover - interface
        raise NotImplementedError


class GpuIterativeCombing(SemiLocalStrategy):
    """Tiled wavefront combing over the whole grid (the GPU counterpart of OpenMPIterativeCombing,
    R:include/SemiLocal/SemiLocalLCS.h:231-306)."""

    def __init__(self, band_rows: int = 0):
        self.band_rows = band_rows

    def compute(self, a, b) -> Permutation:
        r2c, _ = api.comb(a, b, algo=_lib.ALGO_WAVEFRONT, band_rows=self.band_rows)
        return Permutation.from_row_to_col(r2c, len(a), len(b))


class GpuHybridCombing(SemiLocalStrategy):
    """Tiles combed independently and glued by the GPU steady ant (the GPU counterpart of
    OpenMPHybridIterative, R:include/SemiLocal/SemiLocalLCS.h:594-794)."""

    def __init__(self, tile: int = 4096, sa_cutoff: int = 0):
        self.tile = tile
        self.sa_cutoff = sa_cutoff

    def compute(self, a, b) -> Permutation:
        r2c, _ = api.comb(a, b, algo=_lib.ALGO_HYBRID, tile=self.tile, sa_cutoff=self.sa_cutoff)
        return Permutation.from_row_to_col(r2c, len(a), len(b))


class BraidMultiplicationStrategy:
    def multiply(self, p: Permutation, q: Permutation) -> Permutation:  # pragma: no cover - interface
        raise NotImplementedError


class GpuSteadyAntMultiplication(BraidMultiplicationStrategy):
    """Steady-ant unit-Monge product on the GPU (counterpart of
    SequentialMemoryOptimizedStickBraidMultiplication / OpenMPStickyBraid,
    R:common/include/Permutations/MongeMultuplicationStrategy.h:548-673)."""

    def __init__(self, sa_cutoff: int = 0):
        self.sa_cutoff = sa_cutoff

    def multiply(self, p, q) -> Permutation:
        pr = p.row_to_col if isinstance(p, Permutation) else np.asarray(p)
        qr = q.row_to_col if isinstance(q, Permutation) else np.asarray(q)
        return Permutation.from_row_to_col(api.steady_ant(pr, qr, self.sa_cutoff))


class StaggeredStickyBraidMultiplication:
    """Glue of two braids sharing k strands (R:common/include/Permutations/MongeMultuplicationStrategy.h:675-802)."""

    def staggered_sticky_multiplication(self, p: Permutation, q: Permutation, row_glue: bool) -> Permutation:
        out = api.staggered_glue(p.row_to_col, p.m, p.n, q.row_to_col, q.m, q.n, row_glue)
        m = p.m + q.m if row_glue else p.m
        n = p.n if row_glue else p.n + q.n
        return Permutation.from_row_to_col(out, m, n)


class LCSStrategy:
    def compute(self, a, b) -> int:  # pragma: no cover - interface
        raise NotImplementedError


class LCSBySemiLocal(LCSStrategy):
    """Global LCS read from the braid: m - #{left strands ending on the right} (R:include/LCS/LCS.h:223-233)."""

    def __init__(self, solver: SemiLocalStrategy | None = None):
        self.solver = solver

    def compute(self, a, b) -> int:
        if self.solver is None:
            return api.lcs(a, b)
        perm = self.solver.compute(a, b)
        m, n = len(a), len(b)
        return m - int(np.count_nonzero(perm.row_to_col[:m] >= n))


class BitParallelLCS(LCSStrategy):
    """LLCS by bit-parallel combing (counterpart of llcs_nary_symbol_smart_combing with 2 bits per symbol,
    R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:668-736)."""

    def compute(self, a, b) -> int:
        return api.bitcomb_llcs(a, b)


class InteractiveDuplicateSearchSemiDense:
    """InteractiveDuplicateSearchSemiDense::find (R:approximate_matching/ApproximateMatching.h:320-420): appends the
    (start, end, score) intervals the reference finds to `result`."""

    sparse = False

    def find(self, p, text, k: float, result: list) -> None:
        result.extend(api.duplicate_search(p, text, k, sparse=self.sparse))


class InteractiveDuplicateSearchSemiSparse(InteractiveDuplicateSearchSemiDense):
    """InteractiveDuplicateSearchSemiSparse::find (R:approximate_matching/ApproximateMatching.h:252-318)."""

    sparse = True
