#!/usr/bin/env bash
# Test infrastructure: builds the reference's own GPU program (mriSolver) from
# the reference sources (default /root/reference, override with REF_ROOT) for
# sm_100a into oracle/_ref/mriSolver_ref.  It is used only to generate golden
# outputs of the Toeplitz path, which has no CPU code in the reference
# (tests/golden/gen_toeplitz_golden.py).  Nothing is copied into the repository.
#
# Two build fixes relative to the reference's own Makefiles, which are not run:
#   * toeplitz/GPU_kernels.cu is #included by toeplitz/CUDA_interface.cu and is
#     not compiled on its own;
#   * deviceQuery's main() is left out (it would clash with mriSolver's).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
R="${REF_ROOT:-/root/reference}"
OUT="$HERE/_ref"
CUDA="${CUDA_HOME:-/usr/local/cuda}"
if [ ! -d "$R/toeplitz" ]; then
    echo "build_ref_gpu: reference sources not found at $R; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
INC=(-I"$R" -I"$R/cuda_sdk/inc" -I"$R/bruteForce" -I"$R/toeplitz" -I"$R/kernels"
     -I"$R/deviceQuery" -I"$R/xcpplib")
CU=("$R/main_mri.cu" "$R/deviceQuery/deviceQuery.cu")
for f in "$R"/kernels/*.cu "$R"/bruteForce/*.cu "$R"/toeplitz/*.cu "$R"/xcpplib/*.cu; do
    [ -e "$f" ] || continue
    [ "$(basename "$f")" = "GPU_kernels.cu" ] && continue
    CU+=("$f")
done
CPP=("$R/main.cpp")
for f in "$R"/kernels/*.cpp "$R"/bruteForce/*.cpp "$R"/toeplitz/*.cpp "$R"/xcpplib/*.cpp; do
    CPP+=("$f")
done
for k in cutil stopwatch stopwatch_linux multithreading cmd_arg_reader bank_checker; do
    CPP+=("$R/cuda_sdk/src/$k.cpp")
done
pids=()
for f in "${CU[@]}"; do
    "$CUDA/bin/nvcc" -gencode arch=compute_100a,code=sm_100a -O2 -w -DUNIX "${INC[@]}" \
        -Xcompiler -fpermissive -c "$f" -o "$TMP/$(basename "$f").o" &
    pids+=($!)
done
for f in "${CPP[@]}"; do
    g++ -O2 -w -fpermissive -DUNIX "${INC[@]}" -I"$CUDA/include" -c "$f" \
        -o "$TMP/$(basename "$f").o" &
    pids+=($!)
done
for p in "${pids[@]}"; do wait "$p"; done
"$CUDA/bin/nvcc" -gencode arch=compute_100a,code=sm_100a -o "$OUT/mriSolver_ref" "$TMP"/*.o \
    -lcufft -lpthread
echo "build_ref_gpu: $OUT/mriSolver_ref"
