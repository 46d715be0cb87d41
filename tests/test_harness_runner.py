"""The harness executables (semilocal_b200/harness/): the reference's benchmark protocol (R:utils/runners.py) --
seven stdout lines, the braid hash of R:test_utils.h -- pinned against the reference's own executable's output
(tests/golden/runner_golden.json), the hash restated here against the oracle's braid, and the GPU runners."""
import importlib.util
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "runner_golden.json")
HARNESS = os.path.join(ROOT, "semilocal_b200", "harness")
_spec = importlib.util.spec_from_file_location("mkrg", os.path.join(ROOT, "tests", "golden", "make_runner_golden.py"))
MK = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(MK)


def braid_hash(col_to_row):
    """R:test_utils.h:8-18 (h = (R h + x) mod M on 64-bit signed integers, wrapping like the reference build)."""
    R, M = 4294967279, 4294967291
    h = 0
    for x in col_to_row:
        t = (R * h + int(x)) & ((1 << 64) - 1)
        if t >= 1 << 63:
            t -= 1 << 64
        q = abs(t) % M
        h = q if t >= 0 else -q
    return h


def _write(tmp_path, case):
    a, b = MK.inputs(case["m"], case["n"], case["seed"])
    pa, pb = tmp_path / "a.fna", tmp_path / "b.fna"
    pa.write_text(MK.fna_text(f"a{case['seed']}", a))
    pb.write_text(MK.fna_text(f"b{case['seed']}", b))
    return a, b, str(pa), str(pb)


def test_hash_restatement_matches_reference_runner_golden(tmp_path):
    for case in json.load(open(GOLDEN)):
        a, b, _, _ = _write(tmp_path, case)
        r2c = O.comb_antidiag(a, b)
        c2r = np.empty_like(r2c)
        c2r[r2c] = np.arange(len(r2c))
        assert braid_hash(c2r) == case["hash"], case


def test_runner_fails_loudly_without_device(tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    exe = os.path.join(HARNESS, "slcs_comb_runner")
    if not os.path.exists(exe):
        pytest.skip("harness runners not built")
    _, _, pa, pb = _write(tmp_path, json.load(open(GOLDEN))[1])
    r = subprocess.run([exe, "1", pa, pb], capture_output=True, text=True)
    assert r.returncode == 1 and "status 6" in r.stderr


@pytest.mark.gpu
def test_runners_speak_the_reference_protocol(engine, tmp_path):
    for case in json.load(open(GOLDEN)):
        a, b, pa, pb = _write(tmp_path, case)
        out = subprocess.run([os.path.join(HARNESS, "slcs_comb_runner"), "16", pa, pb], capture_output=True,
                             text=True, timeout=120)
        assert out.returncode == 0 and out.stderr == "", out.stderr
        lines = out.stdout.split("\n")
        assert len(lines) == case["lines"] == 7
        int(lines[0]), int(lines[1])
        assert int(lines[2]) == case["hash"]
        assert [int(lines[3]), int(lines[4])] == [len(a), len(b)]
        assert lines[5:7] == case["names"]
        out = subprocess.run([os.path.join(HARNESS, "slcs_lcs_runner"), "16", pa, pb], capture_output=True,
                             text=True, timeout=120)
        assert out.returncode == 0
        assert int(out.stdout.split("\n")[2]) == O.lcs_dp(a, b)
