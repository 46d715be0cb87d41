#!/usr/bin/env python
"""Benchmark of the B200 semi-local LCS engine: one JSON line on rank 0.

Default workload (N GPUs, weak scaling): the batched comparison -- 4096 pairs per GPU, |a| log-uniform in
[256, 65536] over 4 letters, b = a with 10 % substitutions and 1 % indels -- combed into int32 braids by
one persistent, length-bucketed launch replayed from a CUDA graph.  metric = GCUPS (sum m*n per second,
whole job).  Beside it: the same plan launched once per pair (the plain per-pair baseline), the
reference's CPU path on a bounded sample (cpu_baseline), the roofline of the combing kernel, clocks.

--impl reference times the reference's own CPU code (oracle/_ref, compiled from the reference sources;
the C restatement in oracle/ when absent) on the same workload, all host threads, bounded samples.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from semilocal_b200 import gen  # noqa: E402
from semilocal_b200.shard import max_over_ranks, shard_pairs  # noqa: E402

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
OPS_PER_CELL = 5     # compare, compare, or, two selects (R:include/SemiLocal/SemiLocalLCS.h:158-172)
# DRAM bytes (read + write) per cell of comb_kernel, from one ncu capture of the 2048-pair batch case
# (`python -m semilocal_b200.profile_cases batch 2048`: 16.68 + 10.24 MB for 6.5112e10 cells); a launch's traffic grows
# with its bands x columns, i.e. with its cells at a fixed band height, so the bench scales it by cells.
COMB_DRAM_BYTES_PER_CELL = 26.925e6 / 6.5112e10
# Pipe split of comb_kernel from ncu (profiles/comb_kernel_batch_2048_pairs.md): the ALU pipe carries the cell's
# compares and select, the FMA pipe its two IMADs; the issue slots are two-thirds used.
COMB_PIPE_SPLIT = {"alu_pct_of_peak": 60.6, "fma_pct_of_peak": 31.6, "issue_pct": 69.3,
                   "source": "ncu --set full, comb_kernel, 2048-pair batch (profiles/comb_kernel_batch_2048_pairs.md)"}
SM_COUNT = 148
# bit-parallel ops per cell: 17 ops per step, 2S - 1 steps per S x S word cell, S = 32 symbols per 64-bit word
BIT_OPS_PER_CELL = 17 * (2 * 32 - 1) / (32 * 32)
# the bit-vector (Hyyro) kernel: 55.25 warp instructions per step of a lane's 32 rows x 4 columns (ncu instruction
# count of one band, 1024 x 262144: 3.62e6 instructions over 65567 steps), i.e. lane-ops per cell
HY_OPS_PER_CELL = 55.25 / 128
DIGESTS_PATH = os.path.join(ROOT, "tests", "golden", "headline_digests.json")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def issue_ceiling_gops(clocks) -> float:
    """Integer-op ceiling of the SM issue slots: every SMSP issues one warp instruction (32 lane-ops) per clock,
    at the median SM clock sampled under load (the maximum clock when no sample was taken)."""
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    return SM_COUNT * 4 * 32 * mhz * 1e6 / 1e9


def check_against_reference(braids, scores, ms, ns, shard):
    """Every braid of a timed batch against the digests of the reference's results on the seed-5 batch
    (OpenMPIterativeCombing<int,false>(1) per pair, tests/golden/headline_digests.json).  `shard` maps the
    plan's pairs to indices of that batch (None: not that batch)."""
    import hashlib
    if shard is None:
        return {"bit_exact_vs_reference": None, "checked_pairs": 0,
                "note": "this rank's batch has another seed; checked against the per-pair launches only"}
    try:
        with open(DIGESTS_PATH) as f:
            ref = json.load(f)["batch_4096"]
    except (OSError, KeyError, ValueError) as e:
        return {"bit_exact_vs_reference": None, "checked_pairs": 0, "note": f"no reference digests: {e}"}
    off = 0
    bad = []
    for k, i in enumerate(shard):
        sz = int(ms[k]) + int(ns[k])
        d = hashlib.sha256(np.ascontiguousarray(braids[off:off + sz], dtype="<i4").tobytes()).hexdigest()
        if d[:16] != ref["pair_sha256_16"][i] or int(scores[k]) != ref["global_scores"][i]:
            bad.append(i)
        off += sz
    return {"bit_exact_vs_reference": not bad, "checked_pairs": len(shard), "mismatched_pairs": bad[:16],
            "reference": "sha256 of each pair's int32 braid from OpenMPIterativeCombing<int,false>(1), "
                         "the reference compiled from its sources (tests/golden/headline_digests.json)"}


def check_pair_2p20(braids, bit_scores, m, n):
    """The 2^20 pair's braids against the digest of the reference's OpenMPHybridIterative braid and its bit
    scores against the reference braid's global score (tests/golden/headline_digests.json)."""
    import hashlib
    try:
        with open(DIGESTS_PATH) as f:
            ref = json.load(f)["hybrid_2p20"]
    except (OSError, KeyError, ValueError) as e:
        return {"note": f"no reference digests: {e}"}
    out = {name + "_bit_exact_vs_reference":
           hashlib.sha256(np.ascontiguousarray(r, dtype="<i4").tobytes()).hexdigest() == ref["sha256"]
           for name, r in braids.items()}
    for name, sc in bit_scores.items():
        out[name + "_score_equals_reference"] = int(sc) == ref["global_score"] and (m, n) == (ref["m"], ref["n"])
    out["reference"] = "OpenMPHybridIterative<int,false>(threads, 4096, 4096), the reference compiled from its sources"
    return out


def load_peaks():
    try:
        with open(PEAKS_PATH) as f:
            return json.load(f)
    except Exception:
        return {}


# ------------------------------------------------------------------------------------------------------
# workloads
# ------------------------------------------------------------------------------------------------------

def batch_workload(seed: int):
    pairs = gen.batch_pairs(4096, 256, 65536, seed=seed)
    return pairs


def cpu_reference_batch_sample(pairs, budget_s: float, threads: int):
    """Reference CPU path over a bounded sample of the batch: a pool of host threads, each combing whole
    pairs with OpenMPIterativeCombing<int,false>(1) (the reference has no batch API; this is the
    harness-level loop over pairs).  Returns (cells, seconds, kind, sample description)."""
    from oracle import oracle as O
    use_ref = O.ref_available()
    kind = "reference" if use_ref else "port"
    # sample: pairs in a fixed shuffled order until the estimated CPU work fills the budget
    order = np.random.default_rng(0).permutation(len(pairs))
    est_rate = 3.0e9 * threads          # cells/s, conservative estimate to size the sample
    target = est_rate * budget_s
    chosen, cells = [], 0
    for i in order:
        a, b = pairs[i]
        c = len(a) * len(b)
        if cells + c > target and chosen:
            continue
        chosen.append(i)
        cells += c
        if cells >= target:
            break
    work = [(np.ascontiguousarray(pairs[i][0], dtype=np.int32), np.ascontiguousarray(pairs[i][1], dtype=np.int32))
            for i in chosen]
    lock = threading.Lock()
    nxt = [0]

    def worker():
        while True:
            with lock:
                k = nxt[0]
                nxt[0] += 1
            if k >= len(work):
                return
            a, b = work[k]
            if use_ref:
                O.ref_comb(a, b, "openmp", 1)
            else:
                O.comb_antidiag(a, b, 1)

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    dt = time.perf_counter() - t0
    desc = (f"{len(work)} of the batch's pairs ({cells / 1e9:.2f} Gcells), each combed by "
            f"{'OpenMPIterativeCombing<int,false>(1) from the reference sources' if use_ref else 'the C restatement'}"
            f" on a pool of {threads} host threads")
    return cells, dt, kind, desc


# ------------------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------------------

def run_ours(args, rank, world, local):
    import torch

    import semilocal_b200 as S
    torch.cuda.set_device(local)
    S._lib.check(S.lib().slcs_set_device(local))
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    # band heights by length class, hybrid tile and steady-ant cutoff for this device (outside timing)
    t_tune = time.perf_counter()
    table = S.autotune(cache=args.tuning_cache or None)
    t_tune = time.perf_counter() - t_tune
    if args.shard == "fixed":
        # one batch for the whole job, split over the ranks by cost; no data-path collective
        full = batch_workload(5)
        shard = shard_pairs([len(a) * len(b) for a, b in full], world)[rank]
        pairs = [full[i] for i in shard]
        job_cells = sum(len(a) * len(b) for a, b in full)
        del full
    else:
        # weak scaling: every rank its own batch (rank 0 the seed the reference digests are taken on)
        pairs = batch_workload(5 + 1000 * rank)
        shard = list(range(len(pairs))) if rank == 0 else None
        job_cells = None
    a_cat, a_off, ms, b_cat, b_off, ns = S.concat_pairs(pairs)
    # pinned host copies for the end-to-end leg
    a_pin = torch.from_numpy(a_cat).pin_memory()
    b_pin = torch.from_numpy(b_cat).pin_memory()
    plan = S.BatchPlan(ms, ns, mode=0)
    info = plan.info()
    cells = info["cells"]
    out_pin = torch.empty(plan.total, dtype=torch.int32).pin_memory()
    sc_pin = torch.empty(len(pairs), dtype=torch.int32).pin_memory()
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    plan.upload(a_pin.numpy(), a_off, b_pin.numpy(), b_off, sh)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident step (value) ----
    for _ in range(args.warmup):
        plan.run(use_graph=True, stream=sh)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kern_ms = []
    with Clocks(local) as clk:
        barrier()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                plan.run(use_graph=True, stream=sh)
            ev1.record(stream)
        ev1.synchronize()
        barrier()
    total_ms = ev0.elapsed_time(ev1)
    t_max = max_over_ranks(total_ms, dist, "cuda")
    ms_per_step = t_max / args.steps
    value = (job_cells if job_cells is not None else cells * world) / (ms_per_step * 1e-3) / 1e9
    # the braids of the timed plan: every one against the reference's digests (pairs of the seed-5 batch)
    plan.download(out_pin.numpy(), sc_pin.numpy(), sh)
    torch.cuda.synchronize()
    braids = out_pin.numpy().copy()
    scores = sc_pin.numpy().copy()
    parity = check_against_reference(braids, scores, ms, ns, shard)
    # per-launch time of the combing kernel: the mean over replays, each read from the events recorded
    # around the kernel on the launching stream inside the graph
    for _ in range(args.steps):
        plan.run(use_graph=True, stream=sh)
        stream.synchronize()
        kern_ms.append(plan.kernel_ms())

    # ---- end to end through the public API: pinned H2D, run, D2H of braids + scores, every step ----
    # Two plans alternate (double buffering) on three streams: step i's strings go up on the upload stream, its
    # run waits for them on the compute stream, its braids and scores come down on the download stream; so step
    # i+1's upload and step i's download overlap the runs.  A plan's next upload waits for its previous run (the
    # strings are read while combing) and its next run for its previous download (the braids are overwritten).
    # Every step's copies lie inside the timed region; the host consumes each step's braids (download returns
    # after its copy and the device error check).
    plan2 = S.BatchPlan(ms, ns, mode=0)
    plans = (plan, plan2)
    s_up, s_dn = torch.cuda.Stream(), torch.cuda.Stream()
    h_up, h_dn = ctypes.c_void_p(s_up.cuda_stream), ctypes.c_void_p(s_dn.cuda_stream)
    e2e_steps = max(2, args.steps)

    def e2e_pipeline(nsteps, e_start=None, e_end=None):
        ran = [None, None]      # event after each plan's last run
        fetched = [None, None]  # event after each plan's last download
        pending = None          # (plan index, run event) whose download is not issued yet
        if e_start is not None:
            e_start.record(s_up)
        for i in range(nsteps + 1):
            if i < nsteps:
                k = i % 2
                if ran[k] is not None:
                    s_up.wait_event(ran[k])
                plans[k].upload(a_pin.numpy(), a_off, b_pin.numpy(), b_off, h_up)
                up = torch.cuda.Event()
                up.record(s_up)
                stream.wait_event(up)
                if fetched[k] is not None:
                    stream.wait_event(fetched[k])
                plans[k].run(use_graph=True, stream=sh)
                ev = torch.cuda.Event()
                ev.record(stream)
                ran[k] = ev
            if pending is not None:   # the previous step's braids come down while this step combs
                kp, evp = pending
                s_dn.wait_event(evp)
                plans[kp].download(out_pin.numpy(), sc_pin.numpy(), h_dn)
                fe = torch.cuda.Event()
                fe.record(s_dn)
                fetched[kp] = fe
            pending = (i % 2, ran[i % 2]) if i < nsteps else None
        if e_end is not None:
            e_end.record(s_dn)

    e2e_pipeline(2)                  # capture both plans' graphs, warm the copy paths
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_pipeline(e2e_steps, e0, e1)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, dist, "cuda")
    e2e_value = (job_cells if job_cells is not None else cells * world) / (e2e_ms * 1e-3) / 1e9
    e2e_check = bool(np.array_equal(out_pin.numpy(), braids) and np.array_equal(sc_pin.numpy(), scores))
    plan2.close()

    # ---- plain per-pair launches on the same plan (baseline for the batched launch) ----
    plain = S.BatchPlan(ms, ns, mode=1)
    plain.upload(a_pin.numpy(), a_off, b_pin.numpy(), b_off, sh)
    plain.run(use_graph=False, stream=sh)
    plain.run(use_graph=True, stream=sh)     # capture + instantiate outside the timed region
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        p0.record(stream)
        plain.run(use_graph=True, stream=sh)
        p1.record(stream)
    p1.synchronize()
    plain_ms = p0.elapsed_time(p1)
    plain_gcups = cells / (plain_ms * 1e-3) / 1e9
    plain_info = plain.info()
    plain.download(out_pin.numpy(), sc_pin.numpy(), sh)
    torch.cuda.synchronize()
    parity["per_pair_launches_equal_batched"] = bool(np.array_equal(out_pin.numpy(), braids) and
                                                     np.array_equal(sc_pin.numpy(), scores))
    plain.close()

    # ---- roofline of the combing kernel ----
    peak_cells = ctypes.c_double(0)
    S._lib.check(S.lib().slcs_probe_cell_peak(ctypes.byref(peak_cells)))
    k_ms = float(np.mean(kern_ms))
    achieved_gops = OPS_PER_CELL * cells / (k_ms * 1e-3) / 1e9
    peak_gops = OPS_PER_CELL * peak_cells.value / 1e9
    clk_summary = clk.summary()
    issue_peak_gops = issue_ceiling_gops(clk_summary)

    result = {
        "metric": "GCUPS", "value": round(value, 2), "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
        "scaling": "strong" if args.shard == "fixed" else "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded splitmix64)",
        "config": {"workload": "batched combing: 4096 pairs per GPU, |a| log-uniform [256, 65536], 4 letters, "
                               "b = a with 10% subst + 1% indels; int32 braids; persistent length-bucketed "
                               "launch replayed from a CUDA graph",
                   "pairs_per_gpu": len(pairs), "cells_per_gpu": cells,
                   "parallelism": (f"one 4096-pair batch split by cost over {world} GPU" if args.shard == "fixed"
                                   else f"a 4096-pair batch per GPU, {world} GPU"),
                   "l2": "inputs + braids (~%d MB) exceed the 126 MB L2" % ((a_cat.nbytes + b_cat.nbytes + 8 * plan.total) >> 20),
                   "tuning": {"band_rows_by_log2_len": {str(k): table["band_rows_batch"][k] for k in range(8, 17)},
                              "hybrid_tile": table["tile"], "steady_ant_cutoff": table["sa_cutoff"],
                              "autotune_s": round(t_tune, 2)}},
        "e2e": {"value": round(e2e_value, 2), "unit": "GCUPS", "h2d_bytes_per_step": info["h2d_bytes"],
                "d2h_bytes_per_step": info["d2h_bytes"], "steps": e2e_steps,
                "pipeline": "public batch API on two plans: step i+1's H2D and step i's D2H on copy streams overlap "
                            "the runs; every step's copies inside the timed region",
                "last_step_braids_equal_timed_braids": e2e_check},
        "gpu_launches": info["launches"] * args.steps,
        "parity": parity,
        "plain_per_pair": {"value": round(plain_gcups, 2), "unit": "GCUPS", "launches": plain_info["launches"],
                           "batched_over_plain": round(value / world / plain_gcups, 2)},
        "roofline": {"bound": "int32-issue", "achieved": round(achieved_gops, 1), "peak": round(peak_gops, 1),
                     "unit": "Gop/s", "frac": round(achieved_gops / peak_gops, 4),
                     "traffic": int(COMB_DRAM_BYTES_PER_CELL * cells),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of comb_kernel on the "
                                       "2048-pair batch case, scaled to this launch by cells",
                     "kernel": "comb_kernel", "kernel_ms": round(k_ms, 3),
                     "kernel_ms_source": f"mean of {len(kern_ms)} graph replays' kernel events",
                     "peak_source": "slcs_probe_cell_peak (cell instruction mix, full occupancy), x5 ops/cell",
                     "issue_ceiling": {"peak": round(issue_peak_gops, 1), "unit": "Gop/s",
                                       "frac": round(achieved_gops / issue_peak_gops, 4),
                                       "source": "148 SM x 4 SMSP x 32 lanes x median SM clock, one lane-op "
                                                 "per issue slot, x5 ops/cell"},
                     "pipes": COMB_PIPE_SPLIT},
        "clocks": clk_summary,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        c_cells, c_s, kind, desc = cpu_reference_batch_sample(pairs, args.cpu_budget, os.cpu_count() or 1)
        result["cpu_baseline"] = {"value": round(c_cells / c_s / 1e9, 3), "unit": "GCUPS",
                                  "cores": os.cpu_count() or 1, "kind": kind, "sample": desc}
    if rank == 0 and world == 1 and not args.no_suite:
        result["workloads"] = run_suite(torch, S, peak_cells.value, load_peaks())
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    plan.close()
    if rank == 0:
        print(json.dumps(result), flush=True)


# ------------------------------------------------------------------------------------------------------
# the other workloads (rank 0, N = 1): plain pair, steady ant, hybrid pair -- GPU device-resident timings,
# parity spot checks, and the reference's CPU path beside each (bounded samples)
# ------------------------------------------------------------------------------------------------------

def _time_stream(torch, stream, fn, K, W):
    for _ in range(W):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(K):
            fn()
        e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / K


def _cpu_time(fn, reps=1):
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best


def run_suite(torch, S, peak_cells, peaks):
    from oracle import oracle as O
    ncpu = os.cpu_count() or 1
    use_ref = O.ref_available()
    st = torch.cuda.Stream()
    sh = ctypes.c_void_p(st.cuda_stream)
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    out = {}

    # ---- plain pair: a, b uniform over 4 letters, 8192 each; the wavefront on one pair ----
    a, b = gen.plain_pair(8192, seed=1)
    m, n = len(a), len(b)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    r2c = torch.empty(m + n, dtype=torch.int32, device="cuda")
    sc = torch.zeros(1, dtype=torch.int32, device="cuda")
    pl = S.PairPlan(m, n, S.ALGO_WAVEFRONT)
    ms = _time_stream(torch, st, lambda: pl.run(da.data_ptr(), db.data_ptr(), r2c.data_ptr(), sc.data_ptr(), True, sh),
                      10, 3)
    pl.check(sh)
    exp = O.ref_comb(a.astype(np.int32), b.astype(np.int32), "openmp", ncpu) if use_ref else O.comb_antidiag(a, b, ncpu)
    ok = bool(np.array_equal(r2c.cpu().numpy(), exp))
    t1 = _cpu_time(lambda: (O.ref_comb(a, b, "openmp", 1) if use_ref else O.comb_antidiag(a, b, 1)), 3)
    tn = _cpu_time(lambda: (O.ref_comb(a, b, "openmp", ncpu) if use_ref else O.comb_antidiag(a, b, ncpu)), 3)
    out["plain_pair_8192"] = {
        "gpu_ms": round(ms, 3), "gcups": round(m * n / ms / 1e6, 1), "bit_exact_vs_cpu": ok,
        "cpu_ref": {"kind": "reference" if use_ref else "port", "gcups_1t": round(m * n / t1 / 1e9, 2),
                    "gcups_nt": round(m * n / tn / 1e9, 2), "threads": ncpu,
                    "impl": "OpenMPIterativeCombing<int,false>"}}
    pl.close()

    # ---- steady ant: two uniform permutations, n = 2^16 .. 2^24 (headline 2^22) ----
    sweep = {}
    for lg in (16, 18, 20, 22, 24):
        nn = 1 << lg
        p, q = gen.steady_ant_pair(nn)
        dp, dq = torch.from_numpy(p).cuda(), torch.from_numpy(q).cuda()
        dr = torch.empty(nn, dtype=torch.int32, device="cuda")
        sp = S.SteadyAntPlan(nn)
        ms = _time_stream(torch, st, lambda: sp.run(dp.data_ptr(), dq.data_ptr(), dr.data_ptr(), True, sh), 5, 3)
        sp.check(sh)
        balg = 16 * nn * (max(0, int(np.ceil(np.log2(nn / 4096)))) + 1)
        ent = {"gpu_ms": round(ms, 3), "gbs_alg": round(balg / ms / 1e6, 1),
               "hbm_frac": round(balg / ms / 1e6 / hbm_peak, 4), "launches": sp.launches()}
        if lg == 22:
            rr = dr.cpu().numpy()
            if use_ref:
                O.ref().ref_precalc_warm(5)
                t0 = time.perf_counter()
                ref_r = O.ref_braid(p, q, "seq", precalc=5)
                t_seq = time.perf_counter() - t0
                t0 = time.perf_counter()
                O.ref_braid(p, q, "omp", precalc=5, depth=3)
                t_omp = time.perf_counter() - t0
            else:
                t0 = time.perf_counter()
                ref_r = O.steady_ant(p, q)
                t_seq = t_omp = time.perf_counter() - t0
            ent["bit_exact_vs_cpu"] = bool(np.array_equal(rr, ref_r))
            ent["cpu_ref"] = {"kind": "reference" if use_ref else "port", "seq_s": round(t_seq, 3),
                              "openmp_depth3_s": round(t_omp, 3), "threads": ncpu,
                              "impl": "SequentialMemoryOptimizedStickBraidMultiplication / OpenMPStickyBraid(3), "
                                      "precalc 5"}
        sweep[str(nn)] = ent
        sp.close()
        del dp, dq, dr
    out["steady_ant"] = sweep

    # ---- hybrid pair: a uniform 2^20, b = a with 5 % subst, 0.5 % ins, 0.5 % del; tiles 4096 ----
    a, b = gen.hybrid_pair(1 << 20, seed=4)
    m, n = len(a), len(b)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    res = {}
    braids = {}
    # the hybrid with the configuration's 4096 x 4096 tiles, and with 65536 x 65536 tiles (the reference's own
    # OpenMPHybridIterative(threads, 65536, 65536): 256 tiles, 8 glue levels instead of 16)
    for name, kind, tile in (("hybrid_tiles_4096", S.ALGO_HYBRID, 4096), ("hybrid_tiles_65536", S.ALGO_HYBRID, 65536),
                             ("wavefront", S.ALGO_WAVEFRONT, 0), ("bit_parallel", S.PLAN_BITPARALLEL, 0),
                             ("bit_vector_hyyro", S.PLAN_HYYRO, 0)):
        score_only = kind in (S.PLAN_BITPARALLEL, S.PLAN_HYYRO)
        pl = S.PairPlan(m, n, kind, tile=tile)
        r2 = torch.empty(m + n, dtype=torch.int32, device="cuda") if not score_only else None
        sc2 = torch.zeros(1, dtype=torch.int32, device="cuda")
        fn = lambda: pl.run(da.data_ptr(), db.data_ptr(), r2.data_ptr() if r2 is not None else None,
                            sc2.data_ptr(), True, sh)
        ms = _time_stream(torch, st, fn, 3, 3)
        pl.check(sh)
        kms = pl.kernel_ms()
        ent = {"gpu_ms": round(ms, 2), "gcups": round(m * n / ms / 1e6, 1), "score": int(sc2.item()),
               "comb_kernel_ms": round(kms, 2), "launches": pl.launches()}
        if not score_only:
            # whole run (tiles + glue for the hybrid) and combing kernel alone, against the cell-mix probe
            ent["roofline_frac_whole_run"] = round(m * n / (ms * 1e-3) / peak_cells, 4)
            ent["roofline_frac_comb_kernel"] = round(m * n / (kms * 1e-3) / peak_cells, 4)
            braids[name] = r2.cpu().numpy()
        else:
            # ops per cell: the braid-in-bits convention, 17 ops per step of a 32-symbol word cell, 2S - 1 = 63
            # steps per S^2 = 1024 cells (R:prefix_lcs/bitwise/transposition_network_binary_alphabet.h:351-370);
            # the bit-vector kernel's own measured instruction count; against the SM issue ceiling (one lane-op per
            # issue slot) at the sampled clock
            opc = BIT_OPS_PER_CELL if kind == S.PLAN_BITPARALLEL else HY_OPS_PER_CELL
            ops = opc * m * n
            ceiling = issue_ceiling_gops({}) * 1e9
            ent["int_ops_per_cell"] = round(opc, 4)
            ent["roofline_frac_whole_run"] = round(ops / (ms * 1e-3) / ceiling, 4)
            ent["roofline_frac_kernel"] = round(ops / (kms * 1e-3) / ceiling, 4)
            ent["roofline_peak"] = "SM issue ceiling, 148 SM x 4 SMSP x 32 lanes x 1965 MHz"
            # the same ops against the integer-pipe peak the combing is measured on (probe cells/s x 5 ops)
            ent["roofline_frac_kernel_vs_probe"] = round(ops / (kms * 1e-3) / (OPS_PER_CELL * peak_cells), 4)
        res[name] = ent
        pl.close()
    res["hybrid_equals_wavefront"] = bool(np.array_equal(braids["hybrid_tiles_4096"], braids["wavefront"]) and
                                          np.array_equal(braids["hybrid_tiles_65536"], braids["wavefront"]))
    res["scores_agree"] = len({res[k]["score"] for k in ("hybrid_tiles_4096", "hybrid_tiles_65536", "wavefront",
                                                           "bit_parallel", "bit_vector_hyyro")}) == 1
    res["parity"] = check_pair_2p20(braids, {k: res[k]["score"] for k in ("bit_parallel", "bit_vector_hyyro")}, m, n)
    # the reference's hybrid on a bounded sample: the leading 2^16 x 2^16 corner of the same pair
    sa, sb = a[:1 << 16].astype(np.int32), b[:1 << 16].astype(np.int32)
    if use_ref:
        t = _cpu_time(lambda: O.ref_hybrid_iterative(sa, sb, ncpu, 4096, 4096), 1)
        tbit_a = a[:1 << 17].astype(np.int32)
        tbit_b = b[:1 << 17].astype(np.int32)
        tb = _cpu_time(lambda: O.ref_bit_nary(tbit_a, tbit_b, 4, ncpu), 1)
        res["cpu_ref"] = {"kind": "reference", "threads": ncpu,
                          "hybrid_gcups": round(len(sa) * len(sb) / t / 1e9, 2),
                          "hybrid_sample": "OpenMPHybridIterative<int,false>(threads, 4096, 4096) on the leading "
                                           "2^16 x 2^16 corner",
                          "bit_gcups": round(len(tbit_a) * len(tbit_b) / tb / 1e9, 2),
                          "bit_sample": "llcs_nary_symbol_smart_combing<uint64_t>, 2 bits/symbol, leading 2^17 x 2^17"}
    out["hybrid_pair_2p20"] = res
    out["approximate_search"] = run_approximate_search(S, O, use_ref)
    out["serving"] = run_serving(S, O, use_ref, ncpu)
    return out


def run_approximate_search(S, O, use_ref):
    """Approximate copies of a 1000-symbol pattern in a 2^22-symbol text (4 letters, 200 planted copies with 10 %
    substitutions and 2 % indels), k = 0.9, through the public call (host buffers in, intervals out): the dense and
    the sparse search.  The reference's own searches run on a bounded sample, the leading 2^18 (dense) or 2^16
    (sparse) symbols of the text, and the GPU result on that sample is compared with theirs."""
    p, t = gen.planted_text(1000, 1 << 22, 200, 4, 31)
    k = 0.9
    res = {"pattern": len(p), "text": len(t), "k": k, "cells": len(p) * len(t)}
    for name, sparse in (("dense", False), ("sparse", True)):
        S.duplicate_search(p, t, k, sparse=sparse)   # warm-up
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            found = S.duplicate_search(p, t, k, sparse=sparse)
            times.append(time.perf_counter() - t0)
        best = min(times)
        ent = {"e2e_ms": round(best * 1e3, 2), "intervals": len(found),
               "gcups_e2e": round(len(p) * len(t) / best / 1e9, 1)}
        ts = t[:1 << (16 if sparse else 18)]   # the reference's sparse search spends ~90 us per symbol
        if use_ref and O.ref_am() is not None:
            t0 = time.perf_counter()
            ref = O.ref_duplicate_search(p, ts, k, "sparse" if sparse else "dense")
            rt = time.perf_counter() - t0
            ent["equal_to_reference_on_sample"] = S.duplicate_search(p, ts, k, sparse=sparse) == ref
            ent["cpu_ref"] = {"kind": "reference", "threads": 1,
                              "sample": f"leading {len(ts)} symbols of the text",
                              "seconds": round(rt, 3), "gcups": round(len(p) * len(ts) / rt / 1e9, 3),
                              "impl": "InteractiveDuplicateSearchSemi" + ("Sparse" if sparse else "Dense") + "::find"}
        res[name] = ent
    return res


def _serving_query(r):
    """Query of one generated request: kind uniform over global / string-substring / prefix-suffix, its
    positions from the request's two uniform draws."""
    m, n = len(r["a"]), len(r["b"])
    if r["kind"] == "global":
        return (0, 0, 0)
    if r["kind"] == "string_substring":
        i = int(r["u"] * n)
        return (1, i, i + int(r["v"] * (n - i)))
    return (2, int(r["u"] * m), int(r["v"] * n))


def run_serving(S, O, use_ref, ncpu, count=160, rates=(20.0, None), server_opts=None):
    """Poisson arrivals of comparison requests (|a| log-uniform [1k, 1M], 4 letters, b = a with 5 % subst +
    1 % indels, query uniform over global / string-substring / prefix-suffix) through the serving loop.
    Latency = result on the host minus the scheduled arrival.  rate None = every request at t = 0
    (saturation throughput)."""
    reqs = gen.serving_requests(count, 20.0, seed=6)
    cells_all = sum(len(r["a"]) * len(r["b"]) for r in reqs)
    base = np.array([r["t"] for r in reqs]) * 20.0   # unit-rate arrival times, rescaled per run
    out = {"requests": count, "cells": cells_all, "lengths": "log-uniform [1e3, 1e6]"}
    for rate in rates:
        arrivals = base / rate if rate else np.zeros(count)
        with S.Server(**(server_opts or {})) as srv:
            t0 = srv.now()
            tick_arrival, results, nxt = {}, {}, 0
            while len(results) < count:
                now = srv.now() - t0
                while nxt < count and arrivals[nxt] <= now:
                    r = reqs[nxt]
                    t = srv.submit(r["a"], r["b"], _serving_query(r))
                    tick_arrival[t] = (t0 + arrivals[nxt], nxt)
                    nxt += 1
                wait = 1 if nxt < count else 50
                for res in srv.poll(timeout_ms=wait):
                    results[res["ticket"]] = res
            st = srv.stats()
        lat = np.array([res["t_done"] - tick_arrival[t][0] for t, res in results.items()])
        t_end = max(res["t_done"] for res in results.values())
        bad = [res for res in results.values() if res["status"] != 0]
        # answers of the smallest requests against the oracle's DP
        small = sorted(results.items(), key=lambda kv: kv[1]["m"] * kv[1]["n"])[:6]
        ok = all(res["score"] == _serving_dp(O, reqs[tick_arrival[t][1]]) for t, res in small)
        p99 = float(np.percentile(lat, 99))
        # the request at the 99th percentile (the smallest latency at or above it), run again alone on an idle
        # server: how much of its latency in the mix was queueing and sharing
        tickets = list(results.keys())
        at_p99 = min((t for t in tickets if results[t]["t_done"] - tick_arrival[t][0] >= p99 - 1e-9),
                     key=lambda t: results[t]["t_done"] - tick_arrival[t][0])
        r99 = reqs[tick_arrival[at_p99][1]]
        with S.Server(**(server_opts or {})) as srv:
            alone = []
            for _ in range(2):
                t0a = srv.now()
                tk = srv.submit(r99["a"], r99["b"], _serving_query(r99))
                got = []
                while not got:
                    got = srv.poll(timeout_ms=50)
                alone.append(got[0]["t_done"] - t0a)
                srv.release(tk)
        alone_s = min(alone)
        out["poisson_%g_hz" % rate if rate else "saturation"] = {
            "p50_ms": round(1e3 * float(np.percentile(lat, 50)), 2),
            "p99_ms": round(1e3 * p99, 2),
            "p99_request": {"m": len(r99["a"]), "n": len(r99["b"]), "alone_ms": round(1e3 * alone_s, 2),
                            "p99_over_alone": round(p99 / alone_s, 3)},
            "mean_ms": round(1e3 * float(lat.mean()), 2),
            "gcups": round(cells_all / (t_end - t0) / 1e9, 1),
            "wall_s": round(t_end - t0, 3), "failed": len(bad), "smallest_6_match_oracle": ok,
            "launches": st["launches"], "peak_device_bytes": st["peak_bytes"], "budget_bytes": st["budget"]}
    # the reference's own CPU combing on a bounded sample: the smallest requests, one after another, each with
    # OpenMPIterativeCombing<int,false>(all host threads)
    order = sorted(range(count), key=lambda i: len(reqs[i]["a"])) if ncpu > 0 else []
    chosen, c = [], 0
    for i in order:
        cc = len(reqs[i]["a"]) * len(reqs[i]["b"])
        if c + cc > 1.5e10:
            break
        chosen.append(i)
        c += cc
    t0 = time.perf_counter()
    for i in chosen:
        a, b = reqs[i]["a"].astype(np.int32), reqs[i]["b"].astype(np.int32)
        if use_ref:
            O.ref_comb(a, b, "openmp", ncpu)
        else:
            O.comb_antidiag(a, b, ncpu)
    dt = time.perf_counter() - t0
    if ncpu <= 0:
        return out
    out["cpu_ref"] = {"kind": "reference" if use_ref else "port", "threads": ncpu, "gcups": round(c / dt / 1e9, 2),
                      "sample": f"the {len(chosen)} smallest requests ({c / 1e9:.1f} Gcells) in sequence, "
                                f"OpenMPIterativeCombing<int,false>({ncpu})"}
    return out


def _serving_dp(O, r):
    kind, i, j = _serving_query(r)
    a, b = r["a"], r["b"]
    if kind == 0:
        return O.lcs_dp(a, b)
    if kind == 1:
        return O.lcs_dp(a, b[i:j])
    return O.lcs_dp(a[:i], b[j:])


# ------------------------------------------------------------------------------------------------------
# reference arm
# ------------------------------------------------------------------------------------------------------

def run_reference(args, rank, world, local):
    if rank != 0:
        return
    pairs = batch_workload(5)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference_batch_sample(pairs, args.ref_step_s, threads)
    cells_tot, sec_tot, kind, desc = 0, 0.0, None, None
    for _ in range(args.steps):
        c, s, kind, desc = cpu_reference_batch_sample(pairs, args.ref_step_s, threads)
        cells_tot += c
        sec_tot += s
    value = cells_tot / sec_tot / 1e9
    result = {
        "impl": "reference", "metric": "GCUPS", "value": round(value, 3), "unit": "GCUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * sec_tot / args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded splitmix64)",
        "config": {"workload": "batched combing: 4096 pairs, |a| log-uniform [256, 65536], 4 letters, "
                               "b = a with 10% subst + 1% indels; int32 braids",
                   "sample_per_step": desc},
        "cpu_baseline": {"value": round(value, 3), "unit": "GCUPS", "cores": threads, "kind": kind, "sample": desc},
        "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(result), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU work for cpu_baseline")
    ap.add_argument("--ref-step-s", type=float, default=6.0, help="seconds of CPU work per reference step")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-suite", action="store_true", help="skip the plain / steady-ant / hybrid workloads")
    ap.add_argument("--tuning-cache", default="", help="JSON file: load the autotuned table if saved there for "
                                                        "this device, else measure and save it")
    ap.add_argument("--shard", default="weak", choices=["weak", "fixed"],
                    help="weak: every rank combs its own 4096-pair batch; fixed: one 4096-pair batch split over "
                         "the ranks by cost (strong scaling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world, local)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
