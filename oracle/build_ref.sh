#!/usr/bin/env bash
# Builds the reference's own executor (and its bytecode passes) from the
# sources where they lie in the reference tree, together with the harness in
# oracle/ref_harness/, into oracle/_ref/libclifft_ref.so.
#
# Test infrastructure only: the library pins the oracle restatement and times
# the reference's CPU executor. Two builds of the same sources:
#   libclifft_ref.so         generic x86-64 baseline plus the reference's
#                            per-ISA kernel translation units
#                            (src/clifft/CMakeLists.txt:33-43); the CPUID
#                            dispatcher picks avx512 / avx2 / scalar at run
#                            time, so it loads on any x86-64 host. Parity
#                            tests use this one.
#   libclifft_ref_native.so  -march=native -mtune=native on every unit, the
#                            reference's default CLIFFT_CPU_BASELINE=native
#                            (CMakeLists.txt:52,116), for timing. It only runs
#                            on hosts with this build host's instruction set;
#                            oracle/pyoracle.py probes it in a child process
#                            before using it.
# Both use the Release flags -O3 -ffast-math (CMakeLists.txt:93-131).
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT   (or CLIFFT_REFERENCE_ROOT set)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CLIFFT_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
    echo "usage: $0 REFERENCE_ROOT (or set CLIFFT_REFERENCE_ROOT): the reference checkout to build from" >&2
    exit 2
fi
SRC="$REF/src"
OUT="$HERE/_ref"
OBJ="$OUT/obj"
if [ ! -f "$SRC/clifft/svm/svm.cc" ]; then
    echo "reference sources not found under $SRC" >&2
    exit 2
fi
mkdir -p "$OBJ"
CXX="${CXX:-g++}"
COMMON=(-std=c++20 -O3 -ffast-math -fopenmp -fPIC -DNDEBUG -DCLIFFT_ENABLE_RUNTIME_DISPATCH
        -I"$SRC" -I"$HERE/ref_harness" -I"$HERE/../include")
compile() {  # src obj extra-flags...
    local src="$1" obj="$2"; shift 2
    "$CXX" "${COMMON[@]}" "$@" -c "$src" -o "$obj"
}
# Link libgomp by path: this image's g++ driver has no libgomp.spec, so
# -fopenmp works when compiling but not when linking.
GOMP="$(ls /usr/lib/x86_64-linux-gnu/libgomp.so.1 2>/dev/null || echo -lgomp)"
build_variant() {  # object-dir library extra-flags...
    local od="$1" lib="$2"; shift 2
    mkdir -p "$od"
    local pids=()
    for f in svm/svm.cc svm/svm_state.cc svm/svm_scalar.cc svm/svm_forced_kernels.cc \
             api/record_probabilities.cc optimizer/bytecode_pass.cc optimizer/noise_block_pass.cc \
             optimizer/multi_gate_pass.cc optimizer/expand_t_pass.cc optimizer/swap_meas_pass.cc \
             optimizer/tile_axis_fusion_pass.cc optimizer/single_axis_fusion_pass.cc; do
        compile "$SRC/clifft/$f" "$od/$(echo "$f" | tr / _).o" "$@" & pids+=($!)
    done
    compile "$SRC/clifft/svm/svm_avx2.cc" "$od/svm_avx2.o" "$@" -mavx2 -mbmi2 -mfma & pids+=($!)
    compile "$SRC/clifft/svm/svm_avx512.cc" "$od/svm_avx512.o" "$@" -mavx2 -mbmi2 -mfma -mavx512f -mavx512dq \
        & pids+=($!)
    compile "$HERE/ref_harness/ref_driver.cc" "$od/ref_driver.o" "$@" & pids+=($!)
    for p in "${pids[@]}"; do wait "$p"; done
    "$CXX" -shared -o "$OUT/$lib" "$od"/*.o "$GOMP" -lpthread
    echo "built $OUT/$lib"
}
build_variant "$OBJ" libclifft_ref.so
build_variant "$OUT/obj_native" libclifft_ref_native.so -march=native -mtune=native
