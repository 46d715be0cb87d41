#!/usr/bin/env bash
# Compile the reference's own CPU headers (NikitaMishin/semilocal, source/cpu/) in place into
# oracle/_ref/libslcs_ref.so through oracle/ref_shim.cpp.  TEST INFRASTRUCTURE ONLY: the library is the
# parity pin for the C oracle, the generator of tests/golden/, and the "reference" CPU baseline of bench.py.
#
# The reference's CMake build is not used (its configure step needs GTest and a missing test file).
# Only the header-only library code is compiled; nothing is copied out of the reference tree.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
ref="${1:-/root/reference}"
src="$ref/source/cpu"
if [ ! -d "$src" ]; then
  echo "build_ref: reference sources not found at $src; skipping" >&2
  exit 0
fi
mkdir -p "$here/_ref"
# -march=x86-64-v3: portable across the build container and the GPU hosts (the reference's own CMake uses
# -march=native, which would tie the binary to this CPU).
/usr/bin/g++ -std=c++17 -O3 -march=x86-64-v3 -fopenmp -fPIC -shared -w \
  -I"$src" "$here/ref_shim.cpp" -o "$here/_ref/libslcs_ref.so.tmp" -Wl,--no-undefined
mv "$here/_ref/libslcs_ref.so.tmp" "$here/_ref/libslcs_ref.so"
echo "build_ref: wrote $here/_ref/libslcs_ref.so"
# The approximate pattern search (legacy permutation types: its own library)
/usr/bin/g++ -std=c++17 -O3 -march=x86-64-v3 -fPIC -shared -w \
  -I"$src" "$here/ref_am_shim.cpp" -o "$here/_ref/libslcs_ref_am.so.tmp" -Wl,--no-undefined
mv "$here/_ref/libslcs_ref_am.so.tmp" "$here/_ref/libslcs_ref_am.so"
echo "build_ref: wrote $here/_ref/libslcs_ref_am.so"
# The legacy combing, steady ant and hybrid (source/cpu/semi_local.h, unit_monge_mult/steady_ant.h): second oracle
/usr/bin/g++ -std=c++17 -O3 -march=x86-64-v3 -fopenmp -fPIC -shared -w \
  -I"$src" "$here/ref_legacy_shim.cpp" -o "$here/_ref/libslcs_ref_legacy.so.tmp" -Wl,--no-undefined
mv "$here/_ref/libslcs_ref_legacy.so.tmp" "$here/_ref/libslcs_ref_legacy.so"
echo "build_ref: wrote $here/_ref/libslcs_ref_legacy.so"
# Two of the reference's own benchmark executables (its harness protocol: R:utils/runners.py), as the pin of the
# harness runners in semilocal_b200/harness/.
for f in semi_local_naive_iterative semi_local_hybrid_iterative; do
  /usr/bin/g++ -std=c++17 -O2 -march=x86-64-v3 -fopenmp -w -I"$src" "$src/cpu_impl/$f.cpp" -o "$here/_ref/ref_$f"
done
echo "build_ref: wrote the reference runners"
# The reference's own strategies with the GPU engine plugged in through include/slcs.hpp (needs the engine).
repo="$(cd "$here/.." && pwd)"
if [ -f "$repo/semilocal_b200/libslcs.so" ]; then
  /usr/bin/g++ -std=c++17 -O2 -march=x86-64-v3 -fopenmp -w -I"$src" -I"$repo/include" \
    "$repo/tests/cpp/reference_plugin.cpp" -L"$repo/semilocal_b200" -lslcs \
    -Wl,-rpath,'$ORIGIN/../../semilocal_b200' -o "$here/_ref/reference_plugin"
  echo "build_ref: wrote $here/_ref/reference_plugin"
fi
