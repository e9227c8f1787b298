/*
 * ref_base_shim.h -- stands in for the reference's sgpu/base.h when the
 * reference sources are compiled for the parity checks (TEST INFRASTRUCTURE
 * ONLY).
 *
 * sgpu/base.h:13-14 includes CUDA 10.2 headers by absolute path, which do
 * not exist here.  The build passes -DBASE_H (so the reference header's
 * include guard skips its body) and force-includes this file, which provides
 * the same declarations (sgpu/base.h:18-90) against the installed CUDA.  The
 * constant values are the reference's; REF_RANK overrides the compile-time
 * rank DEFAULT_NFACTORS (sgpu/base.h:21) so the kernels can be built at
 * another rank.
 */
#ifndef CTC_REF_BASE_SHIM_H
#define CTC_REF_BASE_SHIM_H

#include <time.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <limits.h>
#include <assert.h>
#include <cuda.h>
#include <cuda_runtime.h>

typedef uint64_t idx_t;

#ifndef REF_RANK
#define REF_RANK 16
#endif

#define DEFAULT_ITERATE 50
#define DEFAULT_NFACTORS REF_RANK
#define DEFAULT_MAX_ITERATE 1000
#define DEFAULT_ERROR_ALS 1e-8
#define DEFAULT_ERROR_SGD 1e-8
#define DEFAULT_ERROR_CCD 1e-8
#define DEFAULT_RANK REF_RANK
#define MAX_NMODES 4
#define NUM_INNER 1
#define MAX_SECONDS -1
#define MAX_BADEPOCHS 3
#define NBADEPOCHS 0
#define BEST_EPOCH 0
#define BEST_RMSE 10000000
#define TOLERANCE 1e-4
#define SGD_REGULARIZATION 1e-3
#define CCD_REGULARIZATION 100
#define ALS_REGULARIZATION 10
#define SGD_MODIFICATIONA 1e-5
#define SGD_MODIFICATIONB 1e-5
#define SGD_MODIFICATIONC 1e-5
#define ALS_WARPSIZE 32
#define CCD_WARPSIZE 32
#define SGD_WARPSIZE 16
#define ALS_BLOCKSIZE 256
#define ALS_BUFSIZE 2048
#define LEARN_RATE 1e-3
#define DEFAULT_BLOCKSIZE 256
#define DEFAULT_T_TILE_LENGTH 32
#define UNIT_LENGTH 134217728
#define DEFAULT_T_TILE_WIDTH 3
#define SS_MIN(x, y) ((x) < (y) ? (x) : (y))
#define SS_MAX(x, y) ((x) > (y) ? (x) : (y))

#ifdef __cplusplus
extern "C" {
#endif
idx_t argmax_elem(idx_t const *const arr, idx_t const N);
#ifdef __cplusplus
}
#endif

#define HANDLE_ERROR(err) (ctc_ref_handle_error((err), __FILE__, __LINE__))
static inline void ctc_ref_handle_error(cudaError_t err, const char *file, int line)
{
    if (err != cudaSuccess) {
        fprintf(stderr, "ERROR: %s in %s at line %d (error-code %d)\n",
                cudaGetErrorString(err), file, line, (int)err);
        fflush(stdout);
        exit(-1);
    }
}

#endif
