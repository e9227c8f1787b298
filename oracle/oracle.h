/*
 * oracle.h -- FP64 CPU restatement of the cuTC single-GPU completion path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine
 * in cutc_b200/: the parity tests, the smoke check and the CPU-baseline leg of
 * bench.py call it.  The engine never links, loads or calls it.
 *
 * Every function states the reference file:line it restates.  Paths are
 * relative to the reference project root, with "sgpu/" meaning
 * "software/single GPU/sgpu/" and "ga/" meaning
 * "software/autotuning/performance_GA/".
 *
 * Conventions
 *   - tensors are COO with the indices exactly as read from a .tns file
 *     (1-based, as the reference kernels require: sgpu/als.cu:256-258);
 *   - factor matrices are row-major double, dims[m] x R, row r = index-1;
 *   - "sorted for mode m" means sorted by (ind[m], ind[(m+1)%3]) with ties
 *     kept in file order (software/scripts/stensor.py:36-43).
 */
#ifndef CTC_ORACLE_H
#define CTC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nmodes;
    uint64_t nnz;
    uint64_t dims[4];
    uint64_t *ind[4];
    double *vals;
} orc_tensor;

typedef struct {
    uint64_t nnz, dlength, size_rows, tile_len;
    uint64_t *directory;   /* dlength           */
    uint64_t *dcounter;    /* dlength + 1       */
    double *entries;       /* size_rows * 3     */
    uint8_t *written;      /* size_rows * 3: 1 where the reference writes */
} orc_ciss;

/* .tns reader: sgpu/io.c:58-106 (p_tt_read_file), io.c:234-308 (tt_get_dims) */
int orc_tns_read(const char *path, orc_tensor *out);
void orc_tensor_free(orc_tensor *t);

/* CISS builder: sgpu/ciss.c:68-195 (tile length 32), ga/ciss.c:69-212 (any). */
int orc_ciss_build(const orc_tensor *t, int mode0, int tile_len, orc_ciss *out);
/* The same with the GA builder's directory counters (ga/ciss.c:101-120
 * counts the first nonzero too: dcounter[k] = start of slice k). */
int orc_ciss_build_ga(const orc_tensor *t, int mode0, int tile_len, orc_ciss *out);
void orc_ciss_free(orc_ciss *c);

/* Reference double->idx_t store of a value into a CISS entry
 * (sgpu/ciss.c:163 "tmpv = newtensor->vals[m]" with tmpv an idx_t), as the
 * x86-64 gcc conversion sequence produces it. */
double orc_ref_value_trunc(double v);

/* Per-nonzero multiplicity that the reference warp kernels give each
 * nonzero of a 32-long CISS tile (sgpu/als.cu:243-312, sgpu/ccd.cu:120-200):
 * 0 for the tile's first row segment (lane 0 never writes), 1 + extra for
 * lane 31 when it continues a segment (shfl_down at lane 31 returns its own
 * value), and for CCD (kernel=1) 0 for every tile at or past
 * 8 * (tilenum/256 + 1) (sgpu/ccd.cu:520).  nnz % 32 must be 0 so that no
 * lane reads an inactive neighbour (undefined in the reference).  w has nnz
 * entries in CISS (= sorted) order. */
int orc_compat_weights(const orc_ciss *c, int kernel, double *w);

/* sum of squared errors, sgpu/completion.c:166-189, rows indexed 0-based */
double orc_sq_loss(const orc_tensor *t, double *const *U, int R);
/* lambda * sum ||U_m||^2, sgpu/completion.c:193-214 */
double orc_frob(int nmodes, const uint64_t *dims, double *const *U, int R, double lambda);

/* One ALS mode update (sgpu/als.cu:689-781 for one mode_n):
 * U[m] := 0, then for each row i present in t (sorted for mode m)
 *   (sum_n w_n h_n h_n^T + lambda I) u_i = sum_n w_n x_n h_n,
 * h_n = U[m+1](j) o U[m+2](k).  w may be NULL (all ones).  If trunc, x_n is
 * orc_ref_value_trunc(x_n).  Returns the number of non-SPD rows. */
int orc_als_mode(const orc_tensor *t, int m, double **U, int R, double lambda,
                 const double *w, int trunc);

/* One reference "CCD+" mode update (sgpu/ccd.cu:82-206 + 318-348):
 * for each row i present in t (sorted for mode m), all columns at once,
 *   e_n = x_n - U[m](i).h_n (old U[m]),  num_f = sum w e h_f,  den_f = sum w h_f^2,
 *   U[m](i,f) = num_f / (lambda + den_f).  Rows absent keep their values. */
void orc_ccd_compat_mode(const orc_tensor *t, int m, double **U, int R, double lambda,
                         const double *w, int trunc);

/* One CCD++ outer iteration (rank-one residual form; the column loop that
 * sgpu/ccd.cu:531-556 leaves commented out): for f in 0..R-1: add back the
 * f-th rank-one term, `inner` sweeps of the three column updates
 * U[m](i,f) = sum r h / (lambda + sum h^2) (rows absent -> 0), subtract the
 * new term.  resid (nnz, in t's order) holds x - model on entry and exit. */
void orc_ccdpp_outer(const orc_tensor *t, double **U, int R, double lambda,
                     int inner, double *resid);
/* resid = x - model */
void orc_residual(const orc_tensor *t, double *const *U, int R, double *resid);

/* One SGD epoch in the deterministic order (tile-major, entry-minor = the
 * mode-1 sorted order) with the reference's per-nonzero rule
 * (sgpu/sgd.cu:86-99):  e = x - sum a.b.c ;
 *   a_f += lr*scale*(e b_f c_f - lambda a_f)  (same for b, c from the
 *   pre-update rows). */
void orc_sgd_epoch(const orc_tensor *t, double **U, int R, double lr,
                   double lambda, double scale, int trunc);
/* The same rule, OpenMP Hogwild over `nthreads` contiguous slices. */
void orc_sgd_epoch_hogwild(const orc_tensor *t, double **U, int R, double lr,
                           double lambda, double scale, int nthreads);

/* Gradient of 1/2 sum_Omega (x - xhat)^2 + lambda sum_m ||U_m||^2
 * (the masked CP loss) for every factor; G has the layout of U. */
void orc_grad(const orc_tensor *t, double *const *U, int R, double lambda, double **G);
double orc_objective(const orc_tensor *t, double *const *U, int R, double lambda);

/* OpenMP variants used as the timed CPU baseline (same results up to
 * summation order). */
int orc_als_mode_omp(const orc_tensor *t, int m, double **U, int R, double lambda,
                     int nthreads);
void orc_ccdpp_outer_omp(const orc_tensor *t, double **U, int R, double lambda,
                         int inner, double *resid, int nthreads);
double orc_sq_loss_omp(const orc_tensor *t, double *const *U, int R, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
