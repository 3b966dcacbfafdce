#!/usr/bin/env bash
# TEST INFRASTRUCTURE ONLY. Compiles the reference's own kernel arithmetic
# (header templates + stencil generators, included in place from the
# Octo-Tiger source tree) around oracle/ref_driver.cpp into oracle/_ref/.
# Needs the reference tree: $OCTOTIGER_REFERENCE, else the recipe's default
# location below; exits with status 3 when neither holds it. Outputs go only
# to oracle/_ref/. Two builds: AVX-512 (8 SIMD lanes, the reference's host
# AVX-512 configuration) and AVX2 (4 lanes) for hosts without AVX-512.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${OCTOTIGER_REFERENCE:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/octotiger/multipole_interactions/kernel/compute_kernel_templates.hpp" ]; then
    echo "build_ref: reference tree not found at $REF" >&2
    exit 3
fi
mkdir -p "$OUT"
DEFS="-DOCTOTIGER_GRIDDIM=8 -DOCTOTIGER_THETA_MINIMUM=0.34 -DOCTOTIGER_KOKKOS_MULTIPOLE_TASKS=1 -DOCTOTIGER_KOKKOS_MONOPOLE_TASKS=1"
FLAGS="-std=c++17 -O3 -ffp-contract=off -fPIC -shared -pthread"
for variant in "avx512:x86-64-v4" "avx2:x86-64-v3"; do
    name="${variant%%:*}"; march="${variant##*:}"
    g++ $FLAGS -march=$march $DEFS -I "$HERE/ref_shim" -I "$REF" -I "$HERE" \
        "$HERE/ref_driver.cpp" -o "$OUT/libotfmm_ref_$name.so.tmp"
    mv "$OUT/libotfmm_ref_$name.so.tmp" "$OUT/libotfmm_ref_$name.so"
done
git -C "$REF" rev-parse HEAD > "$OUT/REFERENCE_COMMIT" 2>/dev/null || echo unknown > "$OUT/REFERENCE_COMMIT"
echo "build_ref: built $(ls "$OUT"/*.so | tr '\n' ' ')"
