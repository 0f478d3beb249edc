#!/usr/bin/env bash
# Builds oracle/_ref/libcuvslam_ref.so: the reference's own hot-path CUDA kernels, compiled
# unchanged from the read-only reference checkout, plus oracle/ref_harness.cu (our host-side
# restatement of the reference wrappers' launch sequences).  Test infrastructure only.
#
# The reference's C++ (Eigen-based) CPU tracker is not built: Eigen, gflags and googletest are
# fetched over the network by the reference's CMake and are absent here.
#
# Usage: oracle/build_ref.sh <cuVSLAM checkout>   (or with CUVSLAM_REFERENCE set).  Without either,
# or when the checkout has no kernels, nothing is built and the script exits 0.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CUVSLAM_REFERENCE:-}}"
if [ -z "$REF" ]; then
  echo "no cuVSLAM checkout given (argument or CUVSLAM_REFERENCE); oracle/_ref not built" >&2
  exit 0
fi
K="$REF/libs/cuda_modules/cuda_kernels"
if [ ! -d "$K" ]; then
  echo "reference kernels not found under $REF; oracle/_ref not built" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
OUT="$HERE/_ref/libcuvslam_ref.so"
if [ -f "$OUT" ] && [ "$OUT" -nt "$HERE/ref_harness.cu" ] && [ "$OUT" -nt "$K/lk_tracker.cu" ] && [ "$OUT" -nt "$HERE/build_ref.sh" ]; then
  exit 0
fi
nvcc -gencode arch=compute_100a,code=sm_100a -O3 -DNDEBUG -std=c++17 -lineinfo \
  -Xcompiler -fPIC -shared -I "$REF/libs" \
  "$K/image_cast.cu" "$K/image_pyramid.cu" "$K/convolutions.cu" "$K/gftt.cu" \
  "$K/selection_v2.cu" "$K/sort.cu" "$K/lk_tracker.cu" "$K/st_tracker.cu" \
  "$HERE/ref_harness.cu" -o "$HERE/_ref/libcuvslam_ref.so"
echo "built $HERE/_ref/libcuvslam_ref.so"
