"""semilocal_b200 -- a B200-native (sm_100a) semi-local LCS engine.

Host-side mirror (Python) of the reference's strategy interfaces (NikitaMishin/semilocal, source/cpu/):
  * SemiLocalStrategy.compute(a, b) -> Permutation      (R:include/SemiLocal/SemiLocalLCS.h:7-11)
  * BraidMultiplicationStrategy.multiply(p, q) -> Permutation
                                                         (R:common/include/Permutations/MongeMultuplicationStrategy.h:18-21)
  * LCSStrategy.compute(a, b) -> int                      (R:include/LCS/LCS.h:9-13)
over the C ABI of libslcs.so (include/slcs.h).  All compute runs in CUDA kernels; there is no CPU path.
"""
from ._lib import (ALGO_AUTO, ALGO_HYBRID, ALGO_WAVEFRONT, PLAN_BITPARALLEL, PLAN_HYYRO, Q_GLOBAL, Q_MATRIX, Q_PREFIX_SUFFIX,
                   Q_STRING_SUBSTRING, Q_SUBSTRING_STRING, Q_SUFFIX_PREFIX, SlcsError, lib)
from .api import (BatchPlan, PairPlan, Server, SteadyAntPlan, Permutation, autotune, set_tuning, tuning, batch_comb, concat_pairs, bitcomb_llcs, hyyro_llcs, comb, lcs, scores, staggered_glue, steady_ant, window_scores, check_permutation, duplicate_search)
from .strategies import (BitParallelLCS, BraidMultiplicationStrategy, GpuHybridCombing, GpuIterativeCombing,
                         GpuSteadyAntMultiplication, InteractiveDuplicateSearchSemiDense,
                         InteractiveDuplicateSearchSemiSparse, LCSBySemiLocal, LCSStrategy, SemiLocalStrategy,
                         StaggeredStickyBraidMultiplication)

__all__ = [
    "ALGO_AUTO", "ALGO_HYBRID", "ALGO_WAVEFRONT", "PLAN_BITPARALLEL", "PLAN_HYYRO", "Q_GLOBAL", "Q_MATRIX", "Q_PREFIX_SUFFIX", "Q_STRING_SUBSTRING",
    "Q_SUBSTRING_STRING", "Q_SUFFIX_PREFIX", "SlcsError", "lib", "BatchPlan", "PairPlan", "Server", "autotune", "set_tuning", "tuning", "SteadyAntPlan", "concat_pairs", "Permutation", "batch_comb", "bitcomb_llcs", "hyyro_llcs",
    "comb", "lcs", "scores", "staggered_glue", "steady_ant", "window_scores", "check_permutation", "duplicate_search", "BitParallelLCS", "BraidMultiplicationStrategy",
    "GpuHybridCombing", "GpuIterativeCombing", "GpuSteadyAntMultiplication", "LCSBySemiLocal", "LCSStrategy",
    "SemiLocalStrategy", "StaggeredStickyBraidMultiplication", "InteractiveDuplicateSearchSemiDense",
    "InteractiveDuplicateSearchSemiSparse",
]
