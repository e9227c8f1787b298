#!/bin/sh
# Builds the reference's own code, from its sources where they lie, into
# oracle/_ref/ (TEST INFRASTRUCTURE ONLY: parity checks and nothing else).
#
#   libref_host.so          sgpu/{ciss,io,sptensor,util,base,matrixprocess}.c
#                           -- tt_read and ciss_alloc for the bit-exact tests
#   libref_{als,ccd,sgd}.so ref_kernels_harness.cu compiled around
#                           sgpu/{als,ccd,sgd}.cu (+ the host .c files they
#                           link against), sm_100a, rank REF_RANK (16)
#
# sgpu/base.h:13-14 includes CUDA 10.2 headers by absolute path; the build
# predefines its include guard and force-includes ref_base_shim.h instead.
# Nothing is written outside oracle/_ref/.  Exits 0 without building when
# the reference tree is absent (the GPU box uses the prebuilt files).
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=${CTC_REFERENCE_ROOT:-/root/reference}
SRC="$ROOT/software/single GPU/sgpu"
OUT="$HERE/_ref"
RANK=${REF_RANK:-16}
if [ ! -f "$SRC/ciss.c" ]; then
    echo "build_ref: reference sources not found under $ROOT; skipping"
    exit 0
fi
mkdir -p "$OUT"
CUDA=${CUDA_HOME:-/usr/local/cuda}
SHIM="-DBASE_H -include $HERE/ref_base_shim.h -DREF_RANK=$RANK"
CFLAGS="-O2 -fPIC -std=gnu99 -D_GNU_SOURCE -w -I$CUDA/include $SHIM"

HOST_SRCS="ciss.c io.c sptensor.c util.c base.c matrixprocess.c"
OBJS=""
for f in $HOST_SRCS completion.c; do
    o="$OUT/host_${f%.c}.o"
    /usr/bin/gcc $CFLAGS -c "$SRC/$f" -o "$o"
    OBJS="$OBJS $o"
done
HOST_OBJS=""
for f in $HOST_SRCS; do HOST_OBJS="$HOST_OBJS $OUT/host_${f%.c}.o"; done
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

if command -v "$CUDA/bin/nvcc" >/dev/null 2>&1; then
    NVFLAGS="-O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -w $SHIM"
    # every harness links all three drivers through completion.c, so each
    # library compiles all three reference .cu files; the harness TU
    # replaces one of them.
    for alg in als ccd sgd; do
        UP=$(echo $alg | tr a-z A-Z)
        OTHERS=""
        for o in als ccd sgd; do
            if [ "$o" != "$alg" ]; then
                "$CUDA/bin/nvcc" $NVFLAGS -c "$SRC/$o.cu" -o "$OUT/k_${alg}_$o.o"
                OTHERS="$OTHERS $OUT/k_${alg}_$o.o"
            fi
        done
        "$CUDA/bin/nvcc" $NVFLAGS -DREF_HARNESS_$UP "-DREF_SOURCE=\"$SRC/$alg.cu\"" \
            -c "$HERE/ref_kernels_harness.cu" -o "$OUT/k_${alg}_harness.o"
        "$CUDA/bin/nvcc" -shared -gencode arch=compute_100a,code=sm_100a \
            -o "$OUT/libref_$alg.so" "$OUT/k_${alg}_harness.o" $OTHERS $OBJS \
            -lcusolver -lcudart -lm
    done
fi
rm -f "$OUT"/*.o
echo "build_ref: built $(ls "$OUT" | tr '\n' ' ')"
