"""Approximate pattern search on the host: the oracle's restatements of InteractiveDuplicateSearchSemiDense and
...SemiSparse (oracle/amatch_oracle.cpp) against the reference's own result vectors (tests/golden/amatch_golden.json, made by the
reference compiled from its sources) and, where that library is present, against the reference on seeded inputs."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from semilocal_b200 import gen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "amatch_golden.json")


def golden_cases():
    return json.load(open(GOLDEN))["cases"]


@pytest.mark.parametrize("sparse", [False, True])
def test_oracle_matches_golden(sparse):
    for c in golden_cases():
        p, t = gen.planted_text(c["m"], c["n"], c["copies"], c["alphabet"], c["seed"])
        got = O.duplicate_search(p, t, c["k"], sparse=sparse)
        assert [list(x) for x in got] == c["intervals_sparse" if sparse else "intervals"], (c["m"], c["n"], c["k"])


@pytest.mark.parametrize("sparse", [False, True])
def test_oracle_matches_reference(sparse):
    if O.ref_am() is None:
        pytest.skip("reference library not built here")
    rng = np.random.default_rng(11 + sparse)
    for trial in range(80):
        m = int(rng.integers(1, 60))
        k = float(rng.choice([0.5, 0.7, 0.8, 0.9, 1.0, rng.uniform(0.3, 1.0)]))
        n = int(rng.integers(int(m / k), int(m / k) + 800))
        p, t = gen.planted_text(m, n, int(rng.integers(0, 8)), int(rng.choice([2, 4])), 500 + trial)
        assert O.duplicate_search(p, t, k, sparse) == O.ref_duplicate_search(p, t, k, "sparse" if sparse else "dense")


def test_oracle_rejects_bad_arguments():
    p, t = gen.planted_text(10, 100, 2, 4, 1)
    for k in (0.0, -0.5, 1.5):
        with pytest.raises(ValueError):
            O.duplicate_search(p, t, k)
    with pytest.raises(ValueError):
        O.duplicate_search(p, t[:11], 0.5)   # text shorter than the window int(m / k) = 20


def test_host_pick_steps_match_plain_restatement(tmp_path):
    """The search's host steps after the device (order by window start, distinct intervals, sort, greedy pick:
    semilocal_b200/csrc/amatch_pick.h) against a plain restatement of the reference's steps on random candidate
    sets (tests/cpp/amatch_pick_check.cpp)."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "amatch_pick_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I",
                    os.path.join(root, "semilocal_b200", "csrc"), os.path.join(root, "tests", "cpp", "amatch_pick_check.cpp"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
