"""The C++ adapter (include/slcs.hpp): a driver in the reference's test style compiled with g++ against the
library, and -- where oracle/build_ref.sh built it -- the reference's own strategies with the GPU engine
plugged in (tests/cpp/reference_plugin.cpp)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from semilocal_b200 import gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "semilocal_b200")
PLUGIN = os.path.join(ROOT, "oracle", "_ref", "reference_plugin")


def _build_demo(tmp_path):
    exe = str(tmp_path / "adapter_demo")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "adapter_demo.cpp"), "-L", LIBDIR, "-lslcs",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_adapter_builds_and_fails_loudly_without_device(tmp_path):
    if _gpu_present():
        pytest.skip("a GPU is present")
    exe = _build_demo(tmp_path)
    r = subprocess.run([exe], input="2 2 0 1 1 0 0", capture_output=True, text=True)
    assert r.returncode == 3 and r.stdout.startswith("error 6"), r.stdout


@pytest.mark.gpu
def test_adapter_matches_oracle(engine, tmp_path):
    exe = _build_demo(tmp_path)
    a = gen.uniform_string(1500, 4, 91, 1)
    b = gen.mutate(a, 0.1, 0.005, 0.005, 4, 92)
    m, n = len(a), len(b)
    k = 777
    p, q = gen.steady_ant_pair(k)
    stdin = " ".join(map(str, [m, n, *a, *b, k, *p, *q]))
    r = subprocess.run([exe], input=stdin, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = {ln.split()[0]: [int(x) for x in ln.split()[1:]] for ln in r.stdout.strip().splitlines()}
    braid = O.comb_antidiag(a, b)
    assert np.array_equal(out["comb"], braid)
    assert np.array_equal(out["hybrid"], braid) and out["same"] == [1]
    score = O.lcs_dp(a, b)
    assert out["lcs"] == [score] and out["bit"] == [score]
    assert out["queries"] == [score, O.lcs_dp(a, b[n // 4:n // 2]), O.lcs_dp(a[:m // 3], b[n // 5:])]
    assert np.array_equal(out["sa"], O.steady_ant(p, q))
    assert np.array_equal(out["glue"], braid)
    dup = O.duplicate_search(a[:40], b, 0.8)
    assert len(dup) > 0 and out["dup"] == [int(v) for iv in dup for v in iv]


@pytest.mark.gpu
def test_reference_strategies_with_gpu_engine_plugged_in(engine):
    if not os.path.exists(PLUGIN):
        pytest.skip("reference plugin not built (oracle/build_ref.sh needs the reference sources)")
    r = subprocess.run([PLUGIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
