"""Generate tests/golden/runner_golden.json: the stdout of the reference's own benchmark executables
(R:cpu_impl/semi_local_naive_iterative.cpp, built from the reference sources into oracle/_ref by
oracle/build_ref.sh) on seeded .fna inputs.  Run where the reference is present:

    oracle/build_ref.sh && python tests/golden/make_runner_golden.py
"""
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from semilocal_b200 import gen  # noqa: E402

CASES = [(1, 1, 11), (37, 64, 12), (700, 500, 13), (1500, 1499, 14), (4000, 2500, 15)]


def fna_text(name, s):
    return name + "\n" + str(len(s)) + "\n" + ",".join(map(str, s)) + ","


def inputs(m, n, seed):
    a = gen.uniform_string(m, 4, seed, 1)
    b = gen.mutate(a, 0.1, 0.005, 0.005, 4, seed + 100)[:n] if n <= m else gen.uniform_string(n, 4, seed, 2)
    return a, b


def main():
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_semi_local_naive_iterative")
    if not os.path.exists(exe):
        raise SystemExit("reference runner missing: run oracle/build_ref.sh first")
    out = []
    with tempfile.TemporaryDirectory() as d:
        for m, n, seed in CASES:
            a, b = inputs(m, n, seed)
            pa, pb = os.path.join(d, "a.fna"), os.path.join(d, "b.fna")
            open(pa, "w").write(fna_text(f"a{seed}", a))
            open(pb, "w").write(fna_text(f"b{seed}", b))
            lines = subprocess.run([exe, "1", pa, pb], capture_output=True, text=True, check=True).stdout.split("\n")
            out.append({"m": m, "n": len(b), "seed": seed, "hash": int(lines[2]), "lines": len(lines),
                        "names": lines[5:7]})
    json.dump(out, open(os.path.join(os.path.dirname(__file__), "runner_golden.json"), "w"), indent=1)


if __name__ == "__main__":
    main()
