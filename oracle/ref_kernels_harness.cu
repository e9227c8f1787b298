/*
 * ref_kernels_harness.cu -- runs the reference's own CUDA kernels, compiled
 * from the reference sources for sm_100a, one mode update at a time
 * (TEST INFRASTRUCTURE ONLY; the parity tests use it to pin the oracle's
 * compat restatement on a B200).
 *
 * Built three times by oracle/build_ref.sh with REF_SOURCE set to the
 * reference's sgpu/als.cu, sgpu/ccd.cu or sgpu/sgd.cu and one of
 * REF_HARNESS_ALS / _CCD / _SGD defined.  The reference file is compiled as
 * part of this translation unit so its __global__ kernels can be launched
 * directly; its host drivers (tc_als, ...) are compiled but never called.
 *
 * Each entry point repeats the per-mode launch sequence of the reference
 * driver with the reference's grid shapes, on caller-supplied CISS arrays
 * and factors (row-major, R = DEFAULT_NFACTORS):
 *   ALS: sgpu/als.cu:691-716   (memset, p_mttkrp_gpu_as, p_update_matrice,
 *                               cusolverDnDpotrf/potrsBatched)
 *   CCD: sgpu/ccd.cu:561-569   (memset, update_frac_gpu_as with the
 *                               reference grid tilenum/256+1, update_ccd_gpu)
 *   SGD: sgpu/sgd.cu:270-287   (p_update_sgd_gpu, one epoch)
 * Directory and dcounter get one padding slot so that the reference's reads
 * one past the last directory position stay inside the allocation.  SGD is
 * refused when nnz % 32 == 0 (its terminator-only tile has bitmap 0 and
 * sgpu/sgd.cu:50 would loop forever).
 */
#include REF_SOURCE

#include <stdint.h>

namespace {

struct DevCiss {
    ciss_t host;          /* host copy holding device pointers */
    ciss_t *dev = nullptr;
    idx_t *d_dir = nullptr, *d_dc = nullptr, *d_dims = nullptr;
    double *d_ent = nullptr;
};

static int put_ciss(DevCiss &c, const double *entries, uint64_t size_rows,
                    const uint64_t *directory, const uint64_t *dcounter, uint64_t dlength,
                    uint64_t nnz, const uint64_t *dims)
{
    if (cudaMalloc(&c.d_dir, (dlength + 1) * sizeof(idx_t))) return -1;
    if (cudaMalloc(&c.d_dc, (dlength + 2) * sizeof(idx_t))) return -1;
    if (cudaMalloc(&c.d_ent, size_rows * 3 * sizeof(double))) return -1;
    if (cudaMalloc(&c.d_dims, 3 * sizeof(idx_t))) return -1;
    if (cudaMalloc(&c.dev, sizeof(ciss_t))) return -1;
    cudaMemset(c.d_dir, 0, (dlength + 1) * sizeof(idx_t));
    cudaMemset(c.d_dc, 0, (dlength + 2) * sizeof(idx_t));
    cudaMemcpy(c.d_dir, directory, dlength * sizeof(idx_t), cudaMemcpyHostToDevice);
    if (dcounter)
        cudaMemcpy(c.d_dc, dcounter, (dlength + 1) * sizeof(idx_t), cudaMemcpyHostToDevice);
    cudaMemcpy(c.d_ent, entries, size_rows * 3 * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(c.d_dims, dims, 3 * sizeof(idx_t), cudaMemcpyHostToDevice);
    c.host.nmodes = 3;
    c.host.nnz = nnz;
    c.host.size = size_rows;
    c.host.dlength = dlength;
    c.host.dims = c.d_dims;
    c.host.directory = c.d_dir;
    c.host.dcounter = c.d_dc;
    c.host.entries = c.d_ent;
    cudaMemcpy(c.dev, &c.host, sizeof(ciss_t), cudaMemcpyHostToDevice);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

static void free_ciss(DevCiss &c)
{
    cudaFree(c.d_dir);
    cudaFree(c.d_dc);
    cudaFree(c.d_ent);
    cudaFree(c.d_dims);
    cudaFree(c.dev);
}

struct DevMat {
    ordi_matrix *dev = nullptr;
    double *vals = nullptr;
    uint64_t rows = 0;
};

static int put_mat(DevMat &m, const double *vals, uint64_t rows)
{
    m.rows = rows;
    if (cudaMalloc(&m.vals, rows * DEFAULT_NFACTORS * sizeof(double))) return -1;
    if (cudaMalloc(&m.dev, sizeof(ordi_matrix))) return -1;
    cudaMemcpy(m.vals, vals, rows * DEFAULT_NFACTORS * sizeof(double), cudaMemcpyHostToDevice);
    ordi_matrix h;
    h.I = rows;
    h.J = DEFAULT_NFACTORS;
    h.values = m.vals;
    h.row_col_flag = 1;
    cudaMemcpy(m.dev, &h, sizeof(ordi_matrix), cudaMemcpyHostToDevice);
    return 0;
}

static void get_mat(const DevMat &m, double *vals)
{
    cudaMemcpy(vals, m.vals, m.rows * DEFAULT_NFACTORS * sizeof(double), cudaMemcpyDeviceToHost);
}

static void free_mat(DevMat &m)
{
    cudaFree(m.vals);
    cudaFree(m.dev);
}

}  // namespace

extern "C" int refh_rank(void) { return DEFAULT_NFACTORS; }

namespace {
// Three mode CISS copies and the three factors resident on the device, for
// timing the reference's per-epoch kernel sequences (refh_*_bench).
struct Resident {
    DevCiss c[3];
    DevMat U[3];
    bool ok = true;
    Resident(const double *const *entries, const uint64_t *size_rows, const uint64_t *const *directory,
             const uint64_t *const *dcounter, const uint64_t *dlength, uint64_t nnz, const uint64_t *dims3,
             const double *const *U0, int ncopies)
    {
        for (int m = 0; m < ncopies && ok; ++m)
            ok = put_ciss(c[m], entries[m], size_rows[m], directory[m], dcounter ? dcounter[m] : nullptr, dlength[m],
                          nnz, dims3) == 0;
        for (int m = 0; m < 3 && ok; ++m) ok = put_mat(U[m], U0[m], dims3[m]) == 0;
        used = ncopies;
    }
    ~Resident()
    {
        for (int m = 0; m < used; ++m) free_ciss(c[m]);
        for (int m = 0; m < 3; ++m) free_mat(U[m]);
    }
    void get(double *const *U1)
    {
        for (int m = 0; m < 3; ++m) get_mat(U[m], U1[m]);
    }
    int used = 0;
};

static float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}
}  // namespace

#ifdef REF_HARNESS_ALS
/* Update factor `t` (target) from CISS of its mode; b and c are the factors
 * of the CISS's first and second stored index (sgpu/als.cu:701, 726, 753). */
extern "C" int refh_als_mode(const double *entries, uint64_t size_rows,
                             const uint64_t *directory, uint64_t dlength, uint64_t nnz,
                             const uint64_t *dims3, double *ft, uint64_t It,
                             const double *fb, uint64_t Ib, const double *fc, uint64_t Ic,
                             double lambda)
{
    DevCiss c;
    DevMat A, B, C;
    int rc = put_ciss(c, entries, size_rows, directory, nullptr, dlength, nnz, dims3);
    rc |= put_mat(A, ft, It) | put_mat(B, fb, Ib) | put_mat(C, fc, Ic);
    double *hbuf = nullptr, **hptr = nullptr, **fptr = nullptr;
    int *info = nullptr;
    cusolverDnHandle_t handle = nullptr;
    if (!rc) {
        rc |= cudaMalloc(&hbuf, (size_t)DEFAULT_NFACTORS * DEFAULT_NFACTORS * dlength * sizeof(double));
        rc |= cudaMalloc(&hptr, dlength * sizeof(double *));
        rc |= cudaMalloc(&fptr, dlength * sizeof(double *));
        rc |= cudaMalloc(&info, dlength * sizeof(int));
    }
    if (!rc && cusolverDnCreate(&handle) != CUSOLVER_STATUS_SUCCESS) rc = -2;
    if (!rc) {
        idx_t tilenum = nnz / DEFAULT_T_TILE_LENGTH + 1;
        idx_t blocknum_m = tilenum / (((idx_t)DEFAULT_BLOCKSIZE) / ((idx_t)ALS_WARPSIZE)) + 1;
        idx_t blocknum_u = dlength / DEFAULT_BLOCKSIZE + 1;
        cudaMemset(hbuf, 0, (size_t)DEFAULT_NFACTORS * DEFAULT_NFACTORS * dlength * sizeof(double));
        cudaMemset(A.vals, 0, It * DEFAULT_NFACTORS * sizeof(double));
        p_mttkrp_gpu_as<<<blocknum_m, DEFAULT_BLOCKSIZE, 0>>>(c.dev, A.dev, B.dev, C.dev, hbuf, tilenum);
        p_update_matrice<<<blocknum_u, DEFAULT_BLOCKSIZE, 0>>>(c.dev, A.vals, hbuf, hptr, fptr, dlength, lambda);
        cublasFillMode_t uplo = CUBLAS_FILL_MODE_UPPER;
        if (cusolverDnDpotrfBatched(handle, uplo, DEFAULT_NFACTORS, hptr, DEFAULT_NFACTORS, info, (int)dlength) != CUSOLVER_STATUS_SUCCESS) rc = -3;
        if (!rc && cusolverDnDpotrsBatched(handle, uplo, DEFAULT_NFACTORS, 1, hptr, DEFAULT_NFACTORS, fptr, DEFAULT_NFACTORS, info, (int)dlength) != CUSOLVER_STATUS_SUCCESS) rc = -4;
        if (cudaDeviceSynchronize() != cudaSuccess) rc = -5;
        if (!rc) get_mat(A, ft);
    }
    if (handle) cusolverDnDestroy(handle);
    cudaFree(hbuf);
    cudaFree(hptr);
    cudaFree(fptr);
    cudaFree(info);
    free_ciss(c);
    free_mat(A);
    free_mat(B);
    free_mat(C);
    return rc;
}

/* `iters` ALS iterations (modes 0, 1, 2, each with the reference driver's
 * kernel sequence, sgpu/als.cu:691-716 and its case 1 / case 2) on
 * resident copies; *ms = device time per iteration (CUDA events, after one
 * untimed warm-up iteration); U (host, row-major) in and out. */
extern "C" int refh_als_bench(const double *const *entries, const uint64_t *size_rows,
                              const uint64_t *const *directory, const uint64_t *dlength, uint64_t nnz,
                              const uint64_t *dims3, double *const *U, double lambda, int iters, double *ms)
{
    Resident S(entries, size_rows, directory, nullptr, dlength, nnz, dims3, U, 3);
    if (!S.ok) return -1;
    uint64_t maxd = 0;
    for (int m = 0; m < 3; ++m) maxd = dlength[m] > maxd ? dlength[m] : maxd;
    double *hbuf = nullptr, **hptr = nullptr, **fptr = nullptr;
    int *info = nullptr;
    int rc = 0;
    rc |= cudaMalloc(&hbuf, (size_t)DEFAULT_NFACTORS * DEFAULT_NFACTORS * maxd * sizeof(double));
    rc |= cudaMalloc(&hptr, maxd * sizeof(double *));
    rc |= cudaMalloc(&fptr, maxd * sizeof(double *));
    rc |= cudaMalloc(&info, maxd * sizeof(int));
    cusolverDnHandle_t handle = nullptr;
    if (!rc && cusolverDnCreate(&handle) != CUSOLVER_STATUS_SUCCESS) rc = -2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    idx_t tilenum = nnz / DEFAULT_T_TILE_LENGTH + 1;
    idx_t blocknum_m = tilenum / (((idx_t)DEFAULT_BLOCKSIZE) / ((idx_t)ALS_WARPSIZE)) + 1;
    cublasFillMode_t uplo = CUBLAS_FILL_MODE_UPPER;
    for (int it = 0; it <= iters && !rc; ++it) {
        if (it == 1) cudaEventRecord(e0);
        for (int m = 0; m < 3 && !rc; ++m) {
            const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
            idx_t blocknum_u = dlength[m] / DEFAULT_BLOCKSIZE + 1;
            cudaMemset(hbuf, 0, (size_t)DEFAULT_NFACTORS * DEFAULT_NFACTORS * dlength[m] * sizeof(double));
            cudaMemset(S.U[m].vals, 0, dims3[m] * DEFAULT_NFACTORS * sizeof(double));
            p_mttkrp_gpu_as<<<blocknum_m, DEFAULT_BLOCKSIZE, 0>>>(S.c[m].dev, S.U[m].dev, S.U[m1].dev, S.U[m2].dev,
                                                                  hbuf, tilenum);
            p_update_matrice<<<blocknum_u, DEFAULT_BLOCKSIZE, 0>>>(S.c[m].dev, S.U[m].vals, hbuf, hptr, fptr,
                                                                   dlength[m], lambda);
            if (cusolverDnDpotrfBatched(handle, uplo, DEFAULT_NFACTORS, hptr, DEFAULT_NFACTORS, info,
                                        (int)dlength[m]) != CUSOLVER_STATUS_SUCCESS)
                rc = -3;
            if (!rc && cusolverDnDpotrsBatched(handle, uplo, DEFAULT_NFACTORS, 1, hptr, DEFAULT_NFACTORS, fptr,
                                               DEFAULT_NFACTORS, info, (int)dlength[m]) != CUSOLVER_STATUS_SUCCESS)
                rc = -4;
        }
    }
    cudaEventRecord(e1);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = -5;
    if (!rc) {
        *ms = iters > 0 ? elapsed(e0, e1) / iters : 0.0;
        S.get(U);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (handle) cusolverDnDestroy(handle);
    cudaFree(hbuf);
    cudaFree(hptr);
    cudaFree(fptr);
    cudaFree(info);
    return rc;
}
#endif

#ifdef REF_HARNESS_CCD
extern "C" int refh_ccd_mode(const double *entries, uint64_t size_rows,
                             const uint64_t *directory, uint64_t dlength, uint64_t nnz,
                             const uint64_t *dims3, double *ft, uint64_t It,
                             const double *fb, uint64_t Ib, const double *fc, uint64_t Ic,
                             double lambda)
{
    DevCiss c;
    DevMat A, B, C;
    int rc = put_ciss(c, entries, size_rows, directory, nullptr, dlength, nnz, dims3);
    rc |= put_mat(A, ft, It) | put_mat(B, fb, Ib) | put_mat(C, fc, Ic);
    double *num = nullptr, *den = nullptr;
    if (!rc) {
        rc |= cudaMalloc(&num, (size_t)DEFAULT_NFACTORS * dlength * sizeof(double));
        rc |= cudaMalloc(&den, (size_t)DEFAULT_NFACTORS * dlength * sizeof(double));
    }
    if (!rc) {
        idx_t tilenum = nnz / DEFAULT_T_TILE_LENGTH + 1;
        idx_t blocknum_m = tilenum / ((idx_t)DEFAULT_BLOCKSIZE) + 1;
        idx_t blocknum_u = dlength / DEFAULT_BLOCKSIZE + 1;
        cudaMemset(num, 0, (size_t)DEFAULT_NFACTORS * dlength * sizeof(double));
        cudaMemset(den, 0, (size_t)DEFAULT_NFACTORS * dlength * sizeof(double));
        update_frac_gpu_as<<<blocknum_m, DEFAULT_BLOCKSIZE, 0>>>(c.dev, A.dev, B.dev, C.dev, num, den, tilenum);
        update_ccd_gpu<<<blocknum_u, DEFAULT_BLOCKSIZE, 0>>>(c.dev, A.dev, num, den, dlength, lambda);
        if (cudaDeviceSynchronize() != cudaSuccess) rc = -5;
        if (!rc) get_mat(A, ft);
    }
    cudaFree(num);
    cudaFree(den);
    free_ciss(c);
    free_mat(A);
    free_mat(B);
    free_mat(C);
    return rc;
}

/* `iters` reference CCD+ iterations (modes 0, 1, 2 with the driver's
 * sequence and grid, sgpu/ccd.cu:561-586) on resident copies; *ms per
 * iteration after one untimed warm-up iteration. */
extern "C" int refh_ccd_bench(const double *const *entries, const uint64_t *size_rows,
                              const uint64_t *const *directory, const uint64_t *dlength, uint64_t nnz,
                              const uint64_t *dims3, double *const *U, double lambda, int iters, double *ms)
{
    Resident S(entries, size_rows, directory, nullptr, dlength, nnz, dims3, U, 3);
    if (!S.ok) return -1;
    uint64_t maxd = 0;
    for (int m = 0; m < 3; ++m) maxd = dlength[m] > maxd ? dlength[m] : maxd;
    double *num = nullptr, *den = nullptr;
    int rc = 0;
    rc |= cudaMalloc(&num, (size_t)DEFAULT_NFACTORS * maxd * sizeof(double));
    rc |= cudaMalloc(&den, (size_t)DEFAULT_NFACTORS * maxd * sizeof(double));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    idx_t tilenum = nnz / DEFAULT_T_TILE_LENGTH + 1;
    idx_t blocknum_m = tilenum / ((idx_t)DEFAULT_BLOCKSIZE) + 1;
    for (int it = 0; it <= iters && !rc; ++it) {
        if (it == 1) cudaEventRecord(e0);
        for (int m = 0; m < 3; ++m) {
            const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
            idx_t blocknum_u = dlength[m] / DEFAULT_BLOCKSIZE + 1;
            cudaMemset(num, 0, (size_t)DEFAULT_NFACTORS * dlength[m] * sizeof(double));
            cudaMemset(den, 0, (size_t)DEFAULT_NFACTORS * dlength[m] * sizeof(double));
            update_frac_gpu_as<<<blocknum_m, DEFAULT_BLOCKSIZE, 0>>>(S.c[m].dev, S.U[m].dev, S.U[m1].dev,
                                                                     S.U[m2].dev, num, den, tilenum);
            update_ccd_gpu<<<blocknum_u, DEFAULT_BLOCKSIZE, 0>>>(S.c[m].dev, S.U[m].dev, num, den, dlength[m],
                                                                 lambda);
        }
    }
    cudaEventRecord(e1);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = -5;
    if (!rc) {
        *ms = iters > 0 ? elapsed(e0, e1) / iters : 0.0;
        S.get(U);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(num);
    cudaFree(den);
    return rc;
}
#endif

#ifdef REF_HARNESS_SGD
/* One Hogwild epoch of the reference kernel on the mode-1 CISS; factors
 * a, b, c are updated in place. */
extern "C" int refh_sgd_epoch(const double *entries, uint64_t size_rows,
                              const uint64_t *directory, const uint64_t *dcounter,
                              uint64_t dlength, uint64_t nnz, const uint64_t *dims3,
                              double *fa, uint64_t Ia, double *fb, uint64_t Ib,
                              double *fc, uint64_t Ic, double lr, double lambda)
{
    if (nnz % DEFAULT_T_TILE_LENGTH == 0) return -10;
    DevCiss c;
    DevMat A, B, C;
    int rc = put_ciss(c, entries, size_rows, directory, dcounter, dlength, nnz, dims3);
    rc |= put_mat(A, fa, Ia) | put_mat(B, fb, Ib) | put_mat(C, fc, Ic);
    if (!rc) {
        idx_t tilenum = nnz / DEFAULT_T_TILE_LENGTH + 1;
        idx_t blocknum_m = tilenum / DEFAULT_BLOCKSIZE + 1;
        p_update_sgd_gpu<<<blocknum_m, DEFAULT_BLOCKSIZE, 0>>>(c.dev, A.dev, B.dev, C.dev, lr, lambda, tilenum);
        if (cudaDeviceSynchronize() != cudaSuccess) rc = -5;
        if (!rc) {
            get_mat(A, fa);
            get_mat(B, fb);
            get_mat(C, fc);
        }
    }
    free_ciss(c);
    free_mat(A);
    free_mat(B);
    free_mat(C);
    return rc;
}

/* `epochs` reference SGD epochs (sgpu/sgd.cu:270-287) on the resident
 * mode-1 copy; *ms per epoch after one untimed warm-up epoch.  Refused
 * when nnz % 32 == 0, as refh_sgd_epoch. */
extern "C" int refh_sgd_bench(const double *entries, uint64_t size_rows, const uint64_t *directory,
                              const uint64_t *dcounter, uint64_t dlength, uint64_t nnz, const uint64_t *dims3,
                              double *const *U, double lr, double lambda, int epochs, double *ms)
{
    if (nnz % DEFAULT_T_TILE_LENGTH == 0) return -10;
    const double *e[1] = {entries};
    const uint64_t *d[1] = {directory}, *dc[1] = {dcounter};
    Resident S(e, &size_rows, d, dc, &dlength, nnz, dims3, U, 1);
    if (!S.ok) return -1;
    int rc = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    idx_t tilenum = nnz / DEFAULT_T_TILE_LENGTH + 1;
    idx_t blocknum_m = tilenum / DEFAULT_BLOCKSIZE + 1;
    for (int ep = 0; ep <= epochs; ++ep) {
        if (ep == 1) cudaEventRecord(e0);
        p_update_sgd_gpu<<<blocknum_m, DEFAULT_BLOCKSIZE, 0>>>(S.c[0].dev, S.U[0].dev, S.U[1].dev, S.U[2].dev, lr,
                                                                lambda, tilenum);
    }
    cudaEventRecord(e1);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = -5;
    if (!rc) {
        *ms = epochs > 0 ? elapsed(e0, e1) / epochs : 0.0;
        S.get(U);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}
#endif
