"""Generate tests/golden/amatch_golden.json: the results of the reference's own approximate pattern search,
InteractiveDuplicateSearchSemiDense::find and ...SemiSparse::find (R:approximate_matching/ApproximateMatching.h:
252-420, compiled from the
reference sources into oracle/_ref/libslcs_ref_am.so by oracle/build_ref.sh), on seeded inputs with planted
copies (semilocal_b200.gen.planted_text).  Run where the reference is present:

    oracle/build_ref.sh && python tests/golden/make_amatch_golden.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from semilocal_b200 import gen  # noqa: E402

# (m, n, copies, alphabet, seed, k)
CASES = [(1, 40, 3, 4, 21, 1.0), (5, 90, 4, 2, 22, 0.5), (12, 300, 6, 4, 23, 0.8), (20, 600, 8, 4, 24, 0.9),
         (33, 1200, 10, 4, 25, 0.75), (50, 3000, 20, 4, 26, 0.9), (64, 2500, 15, 2, 27, 0.6),
         (100, 8000, 25, 4, 28, 0.85), (200, 12000, 20, 4, 29, 0.95), (17, 17, 1, 4, 30, 1.0)]


def main():
    if O.ref_am() is None:
        raise SystemExit("reference library missing: run oracle/build_ref.sh first")
    out = []
    for m, n, copies, alpha, seed, k in CASES:
        p, t = gen.planted_text(m, n, copies, alpha, seed)
        res = O.ref_duplicate_search(p, t, k)
        sp = O.ref_duplicate_search(p, t, k, kind="sparse")
        out.append({"m": m, "n": n, "copies": copies, "alphabet": alpha, "seed": seed, "k": k,
                    "intervals": [[s, e, sc] for s, e, sc in res],
                    "intervals_sparse": [[s, e, sc] for s, e, sc in sp]})
    path = os.path.join(ROOT, "tests", "golden", "amatch_golden.json")
    with open(path, "w") as f:
        json.dump({"source": "InteractiveDuplicateSearchSemiDense / SemiSparse::find of the reference, int symbols", "cases": out}, f)
    print(path, sum(len(c["intervals"]) for c in out), "intervals")


if __name__ == "__main__":
    main()
