#!/usr/bin/env bash
# Test infrastructure: builds the reference's own CPU brute-force path from the
# reference sources where they lie (default /root/reference, override with
# REF_ROOT) into oracle/_ref/ (git-ignored, travels with the repo snapshot).
# Nothing is copied into the repository.
#
#   oracle/_ref/libref_bf64.so      FP64 build (-DENABLE_DOUBLE_PRECISION): the pinning oracle
#   oracle/_ref/libref_bf32.so      FP32 build: "reference FP32" comparisons
#   oracle/_ref/libref_bf32_omp.so  FP32 + OpenMP: the timed CPU reference leg of bench.py
#
# The OpenMP variant needs one token added to two `default(none)` clauses of
# kernels/ftCpu.cpp (:163-166, :249-252) that GCC >= 9 rejects because the
# loop bound is not listed as shared; the patched copy lives only in a temp dir.
# Only g++ is used; the reference's own Makefiles are not run.  The reference
# headers include cuda_runtime.h, so the CUDA include dir is needed, and
# cutil.cpp references libcudart symbols, which are linked but never called
# by the CPU path.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
R="${REF_ROOT:-/root/reference}"
OUT="$HERE/_ref"
CUDA="${CUDA_HOME:-/usr/local/cuda}"
if [ ! -d "$R/kernels" ]; then
    echo "build_ref: reference sources not found at $R; skipping" >&2
    exit 0
fi
mkdir -p "$OUT"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT

SRCS=("$R/bruteForce/bruteForceCpu.cpp")
for k in ft add dotProduct multiply pointMult Dhori2d Dverti2d DHWD2d smvm parImaging; do
    SRCS+=("$R/kernels/${k}Cpu.cpp")
done
SRCS+=("$R/kernels/structures.cpp" "$R/kernels/tools.cpp" "$R/kernels/mmio.cpp")
for f in "$R"/xcpplib/*.cpp; do SRCS+=("$f"); done
for k in cutil stopwatch stopwatch_linux multithreading cmd_arg_reader bank_checker; do
    SRCS+=("$R/cuda_sdk/src/$k.cpp")
done
INC=(-I"$R" -I"$R/kernels" -I"$R/xcpplib" -I"$R/cuda_sdk/inc" -I"$R/bruteForce" -I"$CUDA/include")

# patched copy of ftCpu.cpp for the OpenMP build
sed -e 's/shared(i, kx_N, ky_N/shared(i, num_i, kx_N, ky_N/' \
    -e 's/shared(j, ktraj, t,/shared(j, num_k, ktraj, t,/' \
    "$R/kernels/ftCpu.cpp" > "$TMP/ftCpu_omp.cpp"

build() {  # name, extra flags...
    local name="$1"; shift
    local obj="$TMP/$name"; mkdir -p "$obj"
    local objs=()
    local omp=0
    for fl in "$@"; do [ "$fl" = "-DENABLE_OPENMP" ] && omp=1; done
    local pids=()
    for src in "${SRCS[@]}" "$HERE/ref_driver.cpp"; do
        local s="$src"
        if [ $omp = 1 ] && [ "$(basename "$src")" = "ftCpu.cpp" ]; then s="$TMP/ftCpu_omp.cpp"; fi
        local o="$obj/$(basename "$src").o"
        g++ -O2 -fPIC -fpermissive -w -DUNIX "$@" "${INC[@]}" -c "$s" -o "$o" &
        pids+=($!)
        objs+=("$o")
    done
    for p in "${pids[@]}"; do wait "$p"; done
    local omplink=""
    [ $omp = 1 ] && omplink="-fopenmp"
    g++ -shared -o "$OUT/lib$name.so" "${objs[@]}" $omplink -L"$CUDA/lib64" -lcudart \
        -Wl,-rpath,"$CUDA/lib64"
    echo "build_ref: $OUT/lib$name.so"
}

build ref_bf64 -DENABLE_DOUBLE_PRECISION
build ref_bf32
build ref_bf32_omp -DENABLE_OPENMP -fopenmp
