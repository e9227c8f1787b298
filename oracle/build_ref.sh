#!/bin/sh
# Builds the reference's own code, from its sources where they lie, into
# oracle/_ref/ (TEST INFRASTRUCTURE ONLY: parity checks and the measured
# reference baselines, nothing else).
#
#   sh oracle/build_ref.sh REFERENCE_ROOT      (or CTC_REFERENCE_ROOT=...)
#
#   libref_host.so          sgpu/{ciss,io,sptensor,util,base,matrixprocess}.c
#                           -- tt_read, tt_write_binary and ciss_alloc
#   libref_ga_host.so       the GA-tunable CISS builder (ga/ciss.c)
#   libref_{als,ccd,sgd}.so ref_kernels_harness.cu compiled around
#                           sgpu/{als,ccd,sgd}.cu (+ the host .c files they
#                           link against), sm_100a, rank 16 (the reference's
#                           DEFAULT_NFACTORS)
#   libref_{als,ccd,sgd}_r32.so  the same at rank 32 (the 100M workload's rank)
#
# sgpu/base.h:13-14 includes CUDA 10.2 headers by absolute path; the build
# predefines its include guard and force-includes ref_base_shim.h instead.
# Nothing is written outside oracle/_ref/.  Exits 0 without building when no
# reference tree is given or found there (the GPU box uses the prebuilt
# files).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=${1:-$CTC_REFERENCE_ROOT}
if [ -z "$ROOT" ]; then
    echo "build_ref: no reference root given (argument or CTC_REFERENCE_ROOT); skipping"
    exit 0
fi
SRC="$ROOT/software/single GPU/sgpu"
OUT="$HERE/_ref"
if [ ! -f "$SRC/ciss.c" ]; then
    echo "build_ref: reference sources not found under $ROOT; skipping"
    exit 0
fi
mkdir -p "$OUT"
CUDA=${CUDA_HOME:-/usr/local/cuda}
HOST_SRCS="ciss.c io.c sptensor.c util.c base.c matrixprocess.c"

# host objects of the reference at rank $1 into $OUT/r$1_*.o
host_objs() {
    SHIM="-DBASE_H -include $HERE/ref_base_shim.h -DREF_RANK=$1"
    for f in $HOST_SRCS completion.c; do
        /usr/bin/gcc -O2 -fPIC -std=gnu99 -D_GNU_SOURCE -w -I$CUDA/include $SHIM -c "$SRC/$f" \
            -o "$OUT/r$1_${f%.c}.o"
    done
}

host_objs 16
HOST_OBJS=""
for f in $HOST_SRCS; do HOST_OBJS="$HOST_OBJS $OUT/r16_${f%.c}.o"; done
/usr/bin/gcc -shared -o "$OUT/libref_host.so" $HOST_OBJS -lm

# the GA-tunable CISS builder (runtime tile length, ga/ciss.c:69-212); its
# base.h includes <cuda.h> normally, so no shim is needed
GA="$ROOT/software/autotuning/performance_GA"
if [ -f "$GA/ciss.c" ]; then
    GAOBJS=""
    for f in ciss.c sptensor.c io.c util.c base.c matrixprocess.c; do
        o="$OUT/ga_${f%.c}.o"
        /usr/bin/gcc -O2 -fPIC -std=gnu99 -D_GNU_SOURCE -fopenmp -w -I"$CUDA/include" -c "$GA/$f" -o "$o"
        GAOBJS="$GAOBJS $o"
    done
    /usr/bin/gcc -shared -fopenmp -o "$OUT/libref_ga_host.so" $GAOBJS -lm
fi

# kernel libraries at rank $1, file suffix $2
kernel_libs() {
    RANK=$1
    SUF=$2
    SHIM="-DBASE_H -include $HERE/ref_base_shim.h -DREF_RANK=$RANK"
    NVFLAGS="-O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -w $SHIM"
    OBJS=""
    for f in $HOST_SRCS completion.c; do OBJS="$OBJS $OUT/r${RANK}_${f%.c}.o"; done
    # every harness links all three drivers through completion.c, so each
    # library compiles all three reference .cu files; the harness TU
    # replaces one of them.
    for alg in als ccd sgd; do
        UP=$(echo $alg | tr a-z A-Z)
        OTHERS=""
        for o in als ccd sgd; do
            if [ "$o" != "$alg" ]; then
                "$CUDA/bin/nvcc" $NVFLAGS -c "$SRC/$o.cu" -o "$OUT/k${RANK}_${alg}_$o.o"
                OTHERS="$OTHERS $OUT/k${RANK}_${alg}_$o.o"
            fi
        done
        "$CUDA/bin/nvcc" $NVFLAGS -DREF_HARNESS_$UP "-DREF_SOURCE=\"$SRC/$alg.cu\"" \
            -c "$HERE/ref_kernels_harness.cu" -o "$OUT/k${RANK}_${alg}_harness.o"
        "$CUDA/bin/nvcc" -shared -gencode arch=compute_100a,code=sm_100a \
            -o "$OUT/libref_$alg$SUF.so" "$OUT/k${RANK}_${alg}_harness.o" $OTHERS $OBJS \
            -lcusolver -lcudart -lm
    done
}

if command -v "$CUDA/bin/nvcc" >/dev/null 2>&1; then
    kernel_libs 16 ""
    host_objs 32
    kernel_libs 32 "_r32"
fi
rm -f "$OUT"/*.o
echo "build_ref: built $(ls "$OUT" | tr '\n' ' ')"
