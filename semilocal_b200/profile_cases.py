"""Small, self-contained runs of each hot kernel for profiling (ncu) and quick timing.

    python -m semilocal_b200.profile_cases batch  [pairs]     # persistent batched combing (comb_kernel)
    python -m semilocal_b200.profile_cases bit    [log2 n]    # bit-parallel combing (bit_kernel)
    python -m semilocal_b200.profile_cases wave   [log2 n]    # wavefront combing of one pair (comb_kernel)
    python -m semilocal_b200.profile_cases hybrid [log2 n] [tile]  # hybrid: tile combing + glue tree (tile 4096)
    python -m semilocal_b200.profile_cases hyyro  [log2 n]    # bit-vector LLCS (hyyro_kernel)
    python -m semilocal_b200.profile_cases plain  [n]         # one n x n pair, register-tile kernel (comb_tile_kernel)
    python -m semilocal_b200.profile_cases amatch [log2 n]    # approximate search: pattern 1000, planted text
    python -m semilocal_b200.profile_cases sa     [log2 n]    # steady ant (sa_* kernels)
    python -m semilocal_b200.profile_cases probe              # the combing roofline probe (probe_cells_kernel)

Each case runs its plan three times (the first run binds and captures nothing; the runs are plain launches)
and prints one timing line.  Inputs are the seeded synthetic workloads of semilocal_b200.gen.
"""
from __future__ import annotations

import ctypes
import sys
import time

import numpy as np


def main(argv):
    import torch

    import semilocal_b200 as S
    from semilocal_b200 import gen
    case = argv[1] if len(argv) > 1 else "bit"
    arg = int(argv[2]) if len(argv) > 2 else None
    st = torch.cuda.Stream()
    sh = ctypes.c_void_p(st.cuda_stream)
    if case == "batch":
        npairs = arg or 256
        pairs = gen.batch_pairs(npairs, 256, 16384, seed=5)
        a_cat, a_off, ms, b_cat, b_off, ns = S.concat_pairs(pairs)
        plan = S.BatchPlan(ms, ns, mode=0)
        plan.upload(a_cat, a_off, b_cat, b_off, sh)
        cells = plan.info()["cells"]
        for _ in range(3):
            plan.run(False, sh)
        torch.cuda.synchronize()
        k = plan.kernel_ms()
        print(f"batch pairs={npairs} cells={cells} kernel_ms={k:.3f} gcups={cells / k / 1e6:.1f}")
        return
    if case in ("bit", "wave", "hybrid", "hyyro", "plain"):
        lg = arg or 18
        if case == "plain":
            a, b = gen.plain_pair(arg or 8192, seed=1)
            lg = int(np.log2(len(a)))
        else:
            a, b = gen.hybrid_pair(1 << lg, seed=4)
        m, n = len(a), len(b)
        da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        kind = {"bit": S.PLAN_BITPARALLEL, "wave": S.ALGO_WAVEFRONT, "hybrid": S.ALGO_HYBRID, "hyyro": S.PLAN_HYYRO,
                "plain": S.ALGO_WAVEFRONT}[case]
        tile = (int(argv[3]) if len(argv) > 3 else 4096) if case == "hybrid" else 0
        pl = S.PairPlan(m, n, kind, tile=tile)
        r2 = torch.empty(m + n, dtype=torch.int32, device="cuda") if case not in ("bit", "hyyro") else None
        sc = torch.zeros(1, dtype=torch.int32, device="cuda")
        t0 = time.perf_counter()
        for _ in range(3):
            pl.run(da.data_ptr(), db.data_ptr(), r2.data_ptr() if r2 is not None else None, sc.data_ptr(), False, sh)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / 3
        pl.check(sh)
        print(f"{case} n=2^{lg} score={int(sc.item())} kernel_ms={pl.kernel_ms():.3f} wall_ms={dt * 1e3:.2f}")
        return
    if case == "probe":
        peak = ctypes.c_double(0)
        S._lib.check(S.lib().slcs_probe_cell_peak(ctypes.byref(peak)))
        print(f"probe cells/s={peak.value:.4g}")
        return
    if case == "sa":
        lg = arg or 20
        p, q = gen.steady_ant_pair(1 << lg)
        dp, dq = torch.from_numpy(p).cuda(), torch.from_numpy(q).cuda()
        dr = torch.empty(1 << lg, dtype=torch.int32, device="cuda")
        sp = S.SteadyAntPlan(1 << lg)
        t0 = time.perf_counter()
        for _ in range(3):
            sp.run(dp.data_ptr(), dq.data_ptr(), dr.data_ptr(), False, sh)
        torch.cuda.synchronize()
        sp.check(sh)
        print(f"sa n=2^{lg} wall_ms={(time.perf_counter() - t0) / 3 * 1e3:.2f} ok={bool(np.array_equal(np.sort(dr.cpu().numpy()), np.arange(1 << lg)))}")
        return
    if case == "amatch":
        lg = arg or 22
        p, t = gen.planted_text(1000, 1 << lg, 200, 4, 31)
        t0 = time.perf_counter()
        for _ in range(3):
            found = S.duplicate_search(p, t, 0.9)
        print(f"amatch pattern=1000 text=2^{lg} k=0.9 intervals={len(found)} "
              f"wall_ms={(time.perf_counter() - t0) / 3 * 1e3:.2f}")
        return
    raise SystemExit(f"unknown case {case}")


if __name__ == "__main__":
    main(sys.argv)
