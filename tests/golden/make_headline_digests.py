#!/usr/bin/env python
"""Digests of the reference's own results on the headline workloads (TEST FIXTURE GENERATOR).

Runs the reference's CPU code compiled from its sources (oracle/_ref/libslcs_ref.so, built by
oracle/build_ref.sh) on the seeded synthetic workloads the GPU is timed on, and writes
tests/golden/headline_digests.json:

* batch_4096: the batched comparison -- gen.batch_pairs(4096, 256, 65536, seed=5), each pair combed by
  OpenMPIterativeCombing<int,false>(1) (R:include/SemiLocal/SemiLocalLCS.h:231-306) on a pool of host
  threads (the reference has no batch API; this is the harness-level loop over pairs).  Per pair the first
  16 hex digits of sha256(row_to_col as little-endian int32) and the global score; over the batch the sha256
  of the concatenated per-pair full digests.
* hybrid_2p20: the single-pair hybrid workload -- gen.hybrid_pair(2^20, seed=4) -- combed by
  OpenMPHybridIterative<int,false>(threads, 4096, 4096) (R:include/SemiLocal/SemiLocalLCS.h:594-794):
  sha256 of the braid, its global score and a few semi-local scores read from it.
* bit_2p20: nary::llcs_nary_symbol_smart_combing<uint64_t> with 2 bits per symbol
  (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:668-736) on the same pair trimmed to the
  reference routine's domain: both lengths multiples of 32, |a| <= |b|.

Usage: python tests/golden/make_headline_digests.py [--threads T]   (about 3 minutes on 8 cores)
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from semilocal_b200 import gen  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "headline_digests.json")


def braid_digest(r2c: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(r2c, dtype="<i4").tobytes()).hexdigest()


def batch_digest(full_digests) -> str:
    h = hashlib.sha256()
    for d in full_digests:
        h.update(bytes.fromhex(d))
    return h.hexdigest()


def semilocal_queries(m: int, n: int):
    """Query positions recorded beside the hybrid braid: (kind, i, j) with kind 1 = string-substring
    LCS(a, b[i:j]) and 2 = prefix-suffix LCS(a[:i], b[j:])."""
    return [(1, 0, n), (1, n // 3, 2 * n // 3), (1, 12345, 12345 + 4096), (2, m // 2, n // 2), (2, m, 0),
            (2, 1000, n - 1000)]


def semilocal_value(r2c: np.ndarray, m: int, n: int, kind: int, i: int, j: int) -> int:
    """A score read from the braid through the semi-local matrix H (R:include/SemiLocal/SemiLocalLCS.h:13-63):
    string-substring LCS(a, b[i:j]) = H(m + i, j); prefix-suffix LCS(a[:i], b[j:]) = H(m + j, m + n - i) - (m - i).
    H comes from the oracle's dominance count over the reference's braid."""
    if kind == 1:
        return O.semilocal_entry(r2c, m, n, m + i, j)
    return O.semilocal_entry(r2c, m, n, m + j, m + n - i) - (m - i)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default="", help="comma list of batch,hybrid,bit")
    args = ap.parse_args()
    if not O.ref_available():
        sys.exit("the reference library oracle/_ref/libslcs_ref.so is not built (oracle/build_ref.sh)")
    only = set(args.only.split(",")) if args.only else {"batch", "hybrid", "bit"}
    out = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            out = json.load(f)
    out["generator"] = "tests/golden/make_headline_digests.py"

    if "batch" in only:
        pairs = gen.batch_pairs(4096, 256, 65536, seed=5)
        digests = [None] * len(pairs)
        scores = [0] * len(pairs)
        order = sorted(range(len(pairs)), key=lambda i: -len(pairs[i][0]) * len(pairs[i][1]))
        lock = threading.Lock()
        nxt = [0]

        def worker():
            while True:
                with lock:
                    if nxt[0] >= len(order):
                        return
                    k = order[nxt[0]]
                    nxt[0] += 1
                a, b = pairs[k]
                r2c = O.ref_comb(a.astype(np.int32), b.astype(np.int32), "openmp", 1)
                digests[k] = braid_digest(r2c)
                scores[k] = O.global_score(r2c, len(a), len(b))

        t0 = time.time()
        ths = [threading.Thread(target=worker) for _ in range(args.threads)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        out["batch_4096"] = {
            "workload": "gen.batch_pairs(4096, 256, 65536, seed=5)",
            "reference": "OpenMPIterativeCombing<int,false>(1) per pair (SemiLocalLCS.h:231-306)",
            "cells": int(sum(len(a) * len(b) for a, b in pairs)),
            "batch_sha256": batch_digest(digests),
            "pair_sha256_16": [d[:16] for d in digests],
            "global_scores": scores,
        }
        print(f"batch: {time.time() - t0:.1f} s", file=sys.stderr)

    if "hybrid" in only or "bit" in only:
        a, b = gen.hybrid_pair(1 << 20, seed=4)
        m, n = len(a), len(b)
    if "hybrid" in only:
        t0 = time.time()
        r2c = O.ref_hybrid_iterative(a.astype(np.int32), b.astype(np.int32), args.threads, 4096, 4096)
        qs = semilocal_queries(m, n)
        out["hybrid_2p20"] = {
            "workload": "gen.hybrid_pair(2^20, seed=4)", "m": m, "n": n,
            "reference": "OpenMPHybridIterative<int,false>(threads, 4096, 4096) (SemiLocalLCS.h:594-794)",
            "sha256": braid_digest(r2c),
            "global_score": O.global_score(r2c, m, n),
            "queries": [[k, i, j, semilocal_value(r2c, m, n, k, i, j)] for k, i, j in qs],
        }
        print(f"hybrid: {time.time() - t0:.1f} s", file=sys.stderr)
    if "bit" in only:
        t0 = time.time()
        la, lb = (m // 32) * 32, (n // 32) * 32
        ta, tb = a[:la], b[:lb]
        if la > lb:
            ta, tb = tb, ta
        score = O.ref_bit_nary(ta.astype(np.int32), tb.astype(np.int32), 4, args.threads)
        out["bit_2p20"] = {
            "workload": "gen.hybrid_pair(2^20, seed=4), a[:32*(m//32)] and b[:32*(n//32)], shorter first",
            "reference": "nary::llcs_nary_symbol_smart_combing<uint64_t>, 2 bits per symbol "
                         "(transposition_network_binary_alphabet.h:668-736)",
            "len_a": int(len(ta)), "len_b": int(len(tb)), "a_is_first": bool(la <= lb), "llcs": score,
        }
        print(f"bit: {time.time() - t0:.1f} s", file=sys.stderr)

    with open(OUT, "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print(OUT)


if __name__ == "__main__":
    main()
