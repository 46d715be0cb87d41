"""Generate tests/golden/golden.npz from the reference's own code (oracle/_ref/libslcs_ref.so, built from the
reference sources by oracle/build_ref.sh).  Run in a container where the reference is present:

    oracle/build_ref.sh && python tests/golden/make_golden.py

Cases (all inputs seeded, see semilocal_b200/gen.py):
  comb*  : braids from SimpleIterativeCombing (checked against OpenMPIterativeCombing and, for small sizes,
           DummyPrefixLCSStrategy) + global scores from SequentialMemLCS;
  sa*    : steady-ant products from SequentialMemoryOptimizedStickBraidMultiplication (checked against
           NaiveBraidMultiplication for n <= 64 and OpenMPStickyBraid);
  glue*  : staggeredStickyMultiplication<RowGlue> for both glue directions;
  bit*   : llcs_nary_symbol_smart_combing<uint64_t> (2 bits per symbol) on aligned lengths.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from semilocal_b200 import gen  # noqa: E402


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libslcs_ref.so missing: run oracle/build_ref.sh first")
    out = {}
    k = 0
    sizes = [(m, n) for m in range(1, 9) for n in range(1, 9)]
    sizes += [(1, 64), (64, 1), (31, 33), (33, 31), (100, 37), (37, 100), (257, 255), (500, 500), (1000, 1500),
              (2047, 513), (4096, 4096)]
    for idx, (m, n) in enumerate(sizes):
        alpha = [2, 4, 5, 11, 150][idx % 5]
        a = (gen.uniform_string(m, 256, 9000 + idx, 1).astype(np.int32) % alpha)
        b = (gen.uniform_string(n, 256, 9000 + idx, 2).astype(np.int32) % alpha)
        perm = O.ref_comb(a, b, "simple")
        assert np.array_equal(perm, O.ref_comb(a, b, "openmp", 4))
        if m + n <= 16:
            assert np.array_equal(perm, O.ref_comb(a, b, "dummy"))
        out[f"comb{k}_a"], out[f"comb{k}_b"], out[f"comb{k}_perm"] = a, b, perm
        out[f"comb{k}_score"] = np.int32(O.ref_lcs(a, b, "seqmem"))
        k += 1
    out["comb_count"] = np.int32(k)

    k = 0
    for n in list(range(1, 17)) + [31, 32, 33, 64, 100, 255, 256, 1000, 4096, 10007]:
        p, q = gen.permutation(n, 7000 + n, 1), gen.permutation(n, 7000 + n, 2)
        r = O.ref_braid(p, q, "seq")
        if n <= 64:
            assert np.array_equal(r, O.ref_braid(p, q, "naive"))
        assert np.array_equal(r, O.ref_braid(p, q, "omp", depth=2))
        out[f"sa{k}_p"], out[f"sa{k}_q"], out[f"sa{k}_r"] = p, q, r
        k += 1
    out["sa_count"] = np.int32(k)

    k = 0
    for (pm, pn, qm, qn, rg) in [(5, 7, 3, 7, 1), (40, 13, 21, 13, 1), (7, 5, 7, 3, 0), (13, 40, 13, 21, 0),
                                 (300, 256, 200, 256, 1), (256, 300, 256, 200, 0), (1, 1, 1, 1, 1), (1, 1, 1, 1, 0)]:
        a1 = gen.uniform_string(pm if rg else pm, 4, 5100 + k, 1)
        # braids of real sub-grids so that the glue is the hybrid's glue
        if rg:   # p above q: same columns b, a split in two
            b = gen.uniform_string(pn, 4, 5100 + k, 2)
            a2 = gen.uniform_string(qm, 4, 5100 + k, 3)
            p = O.ref_comb(a1.astype(np.int32), b.astype(np.int32), "simple")
            q = O.ref_comb(a2.astype(np.int32), b.astype(np.int32), "simple")
        else:    # p left of q: same rows a, b split in two
            b1 = gen.uniform_string(pn, 4, 5100 + k, 2)
            b2 = gen.uniform_string(qn, 4, 5100 + k, 3)
            p = O.ref_comb(a1.astype(np.int32), b1.astype(np.int32), "simple")
            q = O.ref_comb(a1.astype(np.int32), b2.astype(np.int32), "simple")
        o = O.ref_staggered(p, pm, pn, q, qm, qn, bool(rg))
        out[f"glue{k}_p"], out[f"glue{k}_q"], out[f"glue{k}_out"] = p, q, o
        out[f"glue{k}_dims"] = np.array([pm, pn, qm, qn, rg], dtype=np.int32)
        k += 1
    out["glue_count"] = np.int32(k)

    k = 0
    for (m, n) in [(32, 32), (32, 96), (64, 320), (320, 640), (1024, 2048), (2048, 2048)]:
        a = gen.uniform_string(m, 4, 6100 + k, 1).astype(np.int32)
        b = gen.uniform_string(n, 4, 6100 + k, 2).astype(np.int32)
        out[f"bit{k}_a"], out[f"bit{k}_b"] = a, b
        out[f"bit{k}_score"] = np.int32(O.ref_bit_nary(a, b, 4, 2))
        assert int(out[f"bit{k}_score"]) == O.ref_lcs(a, b)
        k += 1
    out["bit_count"] = np.int32(k)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
