#!/usr/bin/env bash
# TEST INFRASTRUCTURE ONLY. Compiles the reference's own CUDA interaction
# kernels (included in place from the Octo-Tiger source tree, never copied)
# around oracle/ref_gpu_driver.cu for sm_100a, with --fmad=false so that their
# arithmetic is the reference CPU kernels' (IEEE operations in the templates'
# order), into oracle/_ref/libotfmm_ref_gpu.so. Needs the reference tree:
# $OCTOTIGER_REFERENCE, else the recipe's default location below; exits with
# status 3 when neither holds it.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${OCTOTIGER_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/src/multipole_interactions/legacy/multipole_cuda_kernel.cpp" ]; then
    echo "build_ref_gpu: reference tree not found at $REF" >&2
    exit 3
fi
mkdir -p "$OUT"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
DEFS="-DOCTOTIGER_HAVE_CUDA -DOCTOTIGER_GRIDDIM=8 -DOCTOTIGER_THETA_MINIMUM=0.34 -DOCTOTIGER_KOKKOS_MULTIPOLE_TASKS=1 -DOCTOTIGER_KOKKOS_MONOPOLE_TASKS=1"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 --fmad=false -std=c++17 --expt-relaxed-constexpr \
    --extended-lambda -Xcompiler -fPIC -shared $DEFS -diag-suppress 177 \
    -I "$HERE/ref_gpu_shim" -I "$HERE/ref_shim" -I "$REF" \
    "$HERE/ref_gpu_driver.cu" -o "$OUT/libotfmm_ref_gpu.so.tmp"
mv "$OUT/libotfmm_ref_gpu.so.tmp" "$OUT/libotfmm_ref_gpu.so"
echo "build_ref_gpu: built $OUT/libotfmm_ref_gpu.so"
