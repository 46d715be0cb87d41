"""Build recipe of the engine: compiles semilocal_b200/csrc/*.cu for sm_100a into semilocal_b200/libslcs.so.

Invoked by __graft_entry__.build() and by the package loader when the library is missing or stale.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libslcs.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
         "-cudart", "static", "-Xptxas", "-warn-spills"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in sources() + headers())


def build(verbose: bool = False, force: bool = False, extra=None) -> str:
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, *(extra or []), "-I", os.path.join(HERE, "..", "include"), "-dc"
               if False else "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode):
            sys.stderr.write(out.decode())
        if p.returncode:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_runners()
    return LIB


def build_runners() -> None:
    """The harness executables (semilocal_b200/harness/): combing (braid hash) and LCS (score)."""
    src = os.path.join(HERE, "harness", "slcs_runner.cpp")
    inc = os.path.join(HERE, "..", "include")
    for name, defs in (("slcs_comb_runner", []), ("slcs_lcs_runner", ["-DSLCS_RUNNER_LCS"])):
        out = os.path.join(HERE, "harness", name)
        subprocess.run(["g++", "-std=c++17", "-O2", *defs, "-I", inc, src, "-L", HERE, "-lslcs",
                        "-Wl,-rpath,$ORIGIN/..", "-o", out], check=True)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
