#!/usr/bin/env bash
# Attempt to compile the reference's own GPU path (the "reference-GPU oracle") from its sources
# where they lie, with nvcc and the CUDA toolkit only: no CMake, no fetched dependencies.
# Test infrastructure: nothing in the library uses it.  Objects and the log go to oracle/_ref/.
#
#   bash oracle/ref_build_attempt.sh path/to/reference
#
# The files are the ones the per-window path runs on the reference's GPU: Fresnel, angular
# spectrum, PCA (cuBLAS Gram + cuSOLVER eigensolver), and holonp FFT / RFFT / Mean.  Each is
# compiled on its own; the first error of each is printed.
set -u
if [ $# -ne 1 ]; then echo "usage: bash oracle/ref_build_attempt.sh path/to/reference" >&2; exit 2; fi
REF="$1"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
mkdir -p "$OUT"
LOG="$OUT/build_attempt.log"
: > "$LOG"
INC=(-I "$REF/src/curaii/include" -I "$REF/src/holoflow/include" -I "$REF/src/holoflow/src"
     -I "$REF/src/holoflow_event/include" -I "$REF/src/holonp/include" -I "$REF/src/holonp/src"
     -I "$REF/src/holotask/include" -I "$REF/src/holotask/src")
# Header-only copies of two of the fetched dependencies ship inside installed Python packages
# (nlohmann/json with cudnn_frontend, spdlog with flashinfer); use them when present, so that the
# attempt gets past the first missing header.
SITE="$(python3 -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])' 2>/dev/null)"
for d in "$SITE/include/cudnn_frontend/thirdparty" "$SITE/flashinfer/data/spdlog/include"; do
  if [ -d "$d" ]; then INC+=(-I "$d"); echo "include $d" >> "$LOG"; fi
done
FILES=(src/holotask/src/syncs/fresnel_diffraction.cu src/holotask/src/syncs/angular_spectrum.cu
       src/holotask/src/syncs/pca.cc src/holotask/src/syncs/pca_heev.cc
       src/holonp/src/fft.cu src/holonp/src/rfft.cu src/holonp/src/mean.cu
       src/holoflow/src/core/tasks.cc src/holoflow/src/core/tensor.cc)
# The syncs use logger() and HOLOVIBES_CHECK without including their headers (the reference's
# CMake build supplies them); force-include both so the attempt reaches the next error.
PRE=()
for h in "$REF/src/holotask/src/logger.hh" "$REF/src/holotask/src/bug.hh"; do
  if [ -f "$h" ]; then PRE+=(-include "$h"); fi
done
fail=0
for f in "${FILES[@]}"; do
  obj="$OUT/$(basename "$f").o"
  one="$OUT/$(basename "$f").log"
  if nvcc -std=c++20 -x cu -gencode arch=compute_100a,code=sm_100a "${INC[@]}" "${PRE[@]}" -c "$REF/$f" -o "$obj" > "$one" 2>&1; then
    echo "ok      $f"
  else
    fail=1
    echo "FAILED  $f: $(grep -m1 -E 'error' "$one")"
  fi
  { echo "== $f"; cat "$one"; } >> "$LOG"
done
exit $fail
