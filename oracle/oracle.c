/*
 * oracle.c -- FP64 CPU restatement of the cuTC single-GPU completion path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine (parity tests,
 * smoke check, CPU-baseline leg of bench.py).  The engine never uses it.
 * Reference citations are file:line relative to the reference project root
 * ("sgpu/" = "software/single GPU/sgpu/", "ga/" = the GA-tunable copy).
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* .tns reader                                                          */
/* ------------------------------------------------------------------ */

/* sgpu/io.c:234-308 (tt_get_dims) and sgpu/io.c:58-106 (p_tt_read_file):
 * three passes -- mode count from the first data line (strtok on " \t",
 * minus the value token), max/min index per mode, then the fill with
 * strtoul/strtod.  Lines of length <= 1 and lines starting with '#' are
 * skipped.  dims[m] = max index, +1 when the smallest index is 0.  Indices
 * are kept as read. */
int orc_tns_read(const char *path, orc_tensor *out)
{
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char *line = NULL;
    size_t cap = 0;
    ssize_t rd;
    int ntok = 0;
    while ((rd = getline(&line, &cap, f)) != -1) {
        if (rd > 1 && line[0] != '#') {
            char *p = strtok(line, " \t");
            while (p) { ++ntok; p = strtok(NULL, " \t"); }
            break;
        }
    }
    int nmodes = ntok - 1;
    if (nmodes < 1 || nmodes > 4) { free(line); fclose(f); return -2; }
    uint64_t dims[4] = {0, 0, 0, 0}, offs[4] = {1, 1, 1, 1};
    uint64_t nnz = 0;
    rewind(f);
    while ((rd = getline(&line, &cap, f)) != -1) {
        if (rd > 1 && line[0] != '#') {
            char *p = line;
            for (int m = 0; m < nmodes; ++m) {
                uint64_t v = strtoull(p, &p, 10);
                if (v > dims[m]) dims[m] = v;
                if (v < offs[m]) offs[m] = v;
            }
            strtod(p, &p);
            ++nnz;
        }
    }
    for (int m = 0; m < nmodes; ++m)
        if (offs[m] == 0) ++dims[m];
    out->nmodes = nmodes;
    out->nnz = nnz;
    for (int m = 0; m < nmodes; ++m) {
        out->dims[m] = dims[m];
        out->ind[m] = (uint64_t *)malloc((nnz ? nnz : 1) * sizeof(uint64_t));
    }
    out->vals = (double *)malloc((nnz ? nnz : 1) * sizeof(double));
    rewind(f);
    uint64_t n = 0;
    while ((rd = getline(&line, &cap, f)) != -1 && n < nnz) {
        if (rd > 1 && line[0] != '#') {
            char *p = line;
            for (int m = 0; m < nmodes; ++m) out->ind[m][n] = strtoul(p, &p, 10);
            out->vals[n++] = strtod(p, &p);
        }
    }
    free(line);
    fclose(f);
    return 0;
}

void orc_tensor_free(orc_tensor *t)
{
    for (int m = 0; m < 4; ++m) free(t->ind[m]);
    free(t->vals);
    memset(t, 0, sizeof(*t));
}

/* ------------------------------------------------------------------ */
/* CISS builder                                                         */
/* ------------------------------------------------------------------ */

/* The value store "tmpv = vals[m]" into an idx_t (sgpu/ciss.c:163,
 * ga/ciss.c:173), as the x86-64 gcc sequence does it: values below 2^63 go
 * through a signed truncation (out of range -> 0x8000000000000000), larger
 * ones are offset by 2^63 first and get bit 63 flipped. */
static uint64_t ref_d2u(double v)
{
    const double two63 = 9223372036854775808.0;
    if (isnan(v)) return 0x8000000000000000ULL;
    if (v < two63) {
        if (v < -two63) return 0x8000000000000000ULL;
        return (uint64_t)(int64_t)v;
    }
    double w = v - two63;
    uint64_t r = (w < two63) ? (uint64_t)(int64_t)w : 0x8000000000000000ULL;
    return r ^ 0x8000000000000000ULL;
}

double orc_ref_value_trunc(double v) { return (double)ref_d2u(v); }

/* sgpu/ciss.c:68-195 and ga/ciss.c:69-212 (one partition covering all rows).
 * Directory: distinct mode indices in order of appearance; dcounter[k] =
 * inclusive end of slice k-1 (dcounter[0]=0, dcounter[dlength]=nnz-1).
 * Entries: tiles of (T+1) rows x 3 doubles.  Header row
 * [-dir_pos_at_tile_start, -last_dir_pos_changed_to, bitmap]; body rows
 * (ind[mode+1], ind[mode+2], value-as-idx_t); terminator (-1,-1,-1) after
 * the last nonzero.  `written` marks the slots the reference writes; the
 * rest stay 0 here (uninitialised heap in the reference). */
static int ciss_build_impl(const orc_tensor *t, int mode, int T, int ga, orc_ciss *c)
{
    memset(c, 0, sizeof(*c));
    if (t->nmodes != 3 || t->nnz == 0 || T < 1 || mode < 0 || mode > 2) return -1;
    const uint64_t nnz = t->nnz;
    const uint64_t *im = t->ind[mode];
    const uint64_t *ij = t->ind[(mode + 1) % 3];
    const uint64_t *ik = t->ind[(mode + 2) % 3];
    uint64_t *tdir = (uint64_t *)malloc(nnz * sizeof(uint64_t));
    uint64_t *tdc = (uint64_t *)calloc(nnz + 1, sizeof(uint64_t));
    uint64_t counter = 1, last = im[0];
    tdir[0] = last;
    tdc[0] = 0;
    for (uint64_t m = 1; m < nnz; ++m) {
        if (last != im[m]) {
            tdir[counter] = im[m];
            counter++;
            tdc[counter] += tdc[counter - 1];
            last = im[m];
        }
        tdc[counter]++;
    }
    c->nnz = nnz;
    c->dlength = counter;
    c->tile_len = (uint64_t)T;
    c->directory = (uint64_t *)malloc(counter * sizeof(uint64_t));
    c->dcounter = (uint64_t *)malloc((counter + 1) * sizeof(uint64_t));
    memcpy(c->directory, tdir, counter * sizeof(uint64_t));
    memcpy(c->dcounter, tdc, counter * sizeof(uint64_t));
    c->dcounter[counter] = nnz - 1;
    if (ga) {
        /* ga/ciss.c:101-120 starts its count at the first nonzero itself, so
         * every running count is one larger: dcounter[k] = start(slice k). */
        for (uint64_t k = 1; k < counter; ++k) c->dcounter[k] += 1;
    }

    const uint64_t tilesize = nnz / (uint64_t)T + 1;
    c->size_rows = tilesize + nnz + 1;
    const uint64_t cap = c->size_rows * 3;
    c->entries = (double *)calloc(cap, sizeof(double));
    c->written = (uint8_t *)calloc(cap, 1);
    uint64_t npos = 0, nl = 0, m = 0;
#define W(off, val)                                          \
    do {                                                     \
        uint64_t o_ = npos + (off);                          \
        if (o_ >= cap) { rc = -3; goto done; }               \
        c->entries[o_] = (val);                              \
        c->written[o_] = 1;                                  \
    } while (0)
    int rc = 0;
    while (m < nnz + 1) {
        uint64_t bitmap = 1;
        uint64_t ns = nl;
        uint64_t niv = tdir[ns];
        uint64_t lc = 1;
        W(0, -1.0 * (double)ns);
        while (lc <= (uint64_t)T) {
            if (m == nnz) {
                W(lc * 3, -1.0);
                W(lc * 3 + 1, -1.0);
                W(lc * 3 + 2, -1.0);
                m++;
                break;
            }
            uint64_t ti = im[m];
            if (ti == niv) {
                bitmap = (bitmap << 1) + 1;
            } else {
                bitmap = bitmap << 1;
                niv = ti;
                nl++;
                W(1, -1.0 * (double)nl);
            }
            W(lc * 3, (double)ij[m]);
            W(lc * 3 + 1, (double)ik[m]);
            W(lc * 3 + 2, (double)ref_d2u(t->vals[m]));
            W(2, (double)bitmap);
            m++;
            lc++;
        }
        npos += ((uint64_t)T + 1) * 3;
    }
#undef W
done:
    free(tdir);
    free(tdc);
    if (rc) orc_ciss_free(c);
    return rc;
}

int orc_ciss_build(const orc_tensor *t, int mode, int T, orc_ciss *c)
{
    return ciss_build_impl(t, mode, T, 0, c);
}

int orc_ciss_build_ga(const orc_tensor *t, int mode, int T, orc_ciss *c)
{
    return ciss_build_impl(t, mode, T, 1, c);
}

void orc_ciss_free(orc_ciss *c)
{
    free(c->directory);
    free(c->dcounter);
    free(c->entries);
    free(c->written);
    memset(c, 0, sizeof(*c));
}

/* ------------------------------------------------------------------ */
/* Reference warp-kernel multiplicities                                 */
/* ------------------------------------------------------------------ */

static uint64_t brev64(uint64_t x)
{
    uint64_t r = 0;
    for (int i = 0; i < 64; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* Lane-exact restatement of the segmented shuffle reduction in
 * sgpu/als.cu:227-312 (and the same loop in sgpu/ccd.cu:126-200):
 *   bitmap' = brev(bitmap) with the leading sentinel removed, so bit l is 1
 *   when nonzero l continues the previous row (l=0 compares with the row
 *   at the tile start); lane 0 is forced to mybit=1 and never writes;
 *   itercounter K = popc(bitmap') - bit0; the head h of a segment ending at
 *   lane e accumulates v_h..v_e, plus (K - (31-h)) extra copies of v_31 when
 *   e = 31 > h (shfl_down at lane 31 returns lane 31's own value). */
int orc_compat_weights(const orc_ciss *c, int kernel, double *w)
{
    if (c->tile_len != 32 || c->nnz % 32 != 0) return -1;
    const uint64_t nnz = c->nnz;
    const uint64_t tilenum = nnz / 32 + 1;
    uint64_t covered = tilenum;
    if (kernel == 1) {
        uint64_t cov = 8 * (tilenum / 256 + 1);   /* sgpu/ccd.cu:520 */
        if (cov < covered) covered = cov;
    }
    for (uint64_t n = 0; n < nnz; ++n) w[n] = 0.0;
    for (uint64_t tile = 0; tile < tilenum && tile < covered; ++tile) {
        uint64_t base = tile * 33 * 3;
        uint64_t first = tile * 32;
        if (first >= nnz) break;
        uint64_t B = (uint64_t)c->entries[base + 2];
        if (B == 0) continue;
        uint64_t b = brev64(B);
        while ((b & 1) == 0) b >>= 1;
        b >>= 1;
        int K = __builtin_popcountll(b) - (int)(b & 1);
        int flag[32];
        for (int l = 0; l < 32; ++l) flag[l] = (int)((b >> l) & 1);
        flag[0] = 1; /* lane 0: mybit forced to 1 */
        int h = -1;
        for (int l = 0; l <= 32; ++l) {
            int is_head = (l < 32) && (l > 0) && (flag[l] == 0);
            if (l == 32 || is_head) {
                if (h >= 1) {
                    int e = l - 1;
                    for (int q = h; q <= e; ++q) w[first + q] = 1.0;
                    if (e == 31 && h < 31) w[first + 31] += (double)(K - (31 - h));
                }
                h = l;
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Evaluation                                                           */
/* ------------------------------------------------------------------ */

static inline double predict3(const orc_tensor *t, double *const *U, int R, uint64_t n)
{
    const double *a = U[0] + (t->ind[0][n] - 1) * (uint64_t)R;
    const double *b = U[1] + (t->ind[1][n] - 1) * (uint64_t)R;
    const double *c = U[2] + (t->ind[2][n] - 1) * (uint64_t)R;
    double est = 0;
    for (int f = 0; f < R; ++f) est += a[f] * b[f] * c[f];
    return est;
}

/* sgpu/completion.c:166-189 with p_predict_val3 (completion.c:29-51) read
 * at row index-1 (the reference reads row index, one past the row). */
double orc_sq_loss(const orc_tensor *t, double *const *U, int R)
{
    double s = 0;
    for (uint64_t n = 0; n < t->nnz; ++n) {
        double e = t->vals[n] - predict3(t, U, R, n);
        s += e * e;
    }
    return s;
}

double orc_sq_loss_omp(const orc_tensor *t, double *const *U, int R, int nthreads)
{
    double s = 0;
    const int64_t nnz = (int64_t)t->nnz;
#pragma omp parallel for reduction(+ : s) num_threads(nthreads) schedule(static)
    for (int64_t n = 0; n < nnz; ++n) {
        double e = t->vals[n] - predict3(t, U, R, (uint64_t)n);
        s += e * e;
    }
    return s;
}

/* sgpu/completion.c:193-214 */
double orc_frob(int nmodes, const uint64_t *dims, double *const *U, int R, double lambda)
{
    double reg = 0;
    for (int m = 0; m < nmodes; ++m) {
        double acc = 0;
        for (uint64_t x = 0; x < dims[m] * (uint64_t)R; ++x) acc += U[m][x] * U[m][x];
        reg += lambda * acc;
    }
    return reg;
}

/* ------------------------------------------------------------------ */
/* ALS                                                                  */
/* ------------------------------------------------------------------ */

/* Cholesky solve of the SPD system A u = b (A is R x R row-major, lower
 * triangle used, overwritten).  Returns 0, or 1 when a pivot is not
 * positive (u is then set to 0). */
static int chol_solve(double *A, double *b, double *u, int R)
{
    for (int j = 0; j < R; ++j) {
        double d = A[j * R + j];
        for (int k = 0; k < j; ++k) d -= A[j * R + k] * A[j * R + k];
        if (!(d > 0)) {
            for (int q = 0; q < R; ++q) u[q] = 0;
            return 1;
        }
        d = sqrt(d);
        A[j * R + j] = d;
        for (int i = j + 1; i < R; ++i) {
            double s = A[i * R + j];
            for (int k = 0; k < j; ++k) s -= A[i * R + k] * A[j * R + k];
            A[i * R + j] = s / d;
        }
    }
    for (int i = 0; i < R; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= A[i * R + k] * u[k];
        u[i] = s / A[i * R + i];
    }
    for (int i = R - 1; i >= 0; --i) {
        double s = u[i];
        for (int k = i + 1; k < R; ++k) s -= A[k * R + i] * u[k];
        u[i] = s / A[i * R + i];
    }
    return 0;
}

static void als_row(const orc_tensor *t, int m, double **U, int R, double lambda,
                    const double *w, int trunc, uint64_t s, uint64_t e,
                    double *G, double *rhs, double *h, int *bad)
{
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
    memset(G, 0, sizeof(double) * R * R);
    memset(rhs, 0, sizeof(double) * R);
    for (uint64_t n = s; n < e; ++n) {
        double wn = w ? w[n] : 1.0;
        if (wn == 0.0) continue;
        const double *b = U[m1] + (t->ind[m1][n] - 1) * (uint64_t)R;
        const double *c = U[m2] + (t->ind[m2][n] - 1) * (uint64_t)R;
        double x = trunc ? orc_ref_value_trunc(t->vals[n]) : t->vals[n];
        for (int f = 0; f < R; ++f) h[f] = b[f] * c[f];
        for (int p = 0; p < R; ++p) {
            for (int q = 0; q <= p; ++q) G[p * R + q] += wn * h[p] * h[q];
            rhs[p] += wn * x * h[p];
        }
    }
    for (int p = 0; p < R; ++p) G[p * R + p] += lambda;
    double *u = U[m] + (t->ind[m][s] - 1) * (uint64_t)R;
    *bad += chol_solve(G, rhs, u, R);
}

/* sgpu/als.cu:689-781 for one mode: memset the target factor (als.cu:699),
 * accumulate Gram + MTTKRP per directory row (als.cu:186-317), add lambda to
 * the diagonal (als.cu:467-491), Cholesky solve in place (als.cu:715-716). */
int orc_als_mode(const orc_tensor *t, int m, double **U, int R, double lambda,
                 const double *w, int trunc)
{
    const uint64_t nnz = t->nnz;
    memset(U[m], 0, sizeof(double) * t->dims[m] * (uint64_t)R);
    double *G = (double *)malloc(sizeof(double) * R * R);
    double *rhs = (double *)malloc(sizeof(double) * R);
    double *h = (double *)malloc(sizeof(double) * R);
    int bad = 0;
    uint64_t s = 0;
    while (s < nnz) {
        uint64_t e = s + 1;
        while (e < nnz && t->ind[m][e] == t->ind[m][s]) ++e;
        als_row(t, m, U, R, lambda, w, trunc, s, e, G, rhs, h, &bad);
        s = e;
    }
    free(G);
    free(rhs);
    free(h);
    return bad;
}

static uint64_t *row_starts(const orc_tensor *t, int m, uint64_t *nrows)
{
    uint64_t cnt = 0;
    for (uint64_t n = 0; n < t->nnz; ++n)
        if (n == 0 || t->ind[m][n] != t->ind[m][n - 1]) ++cnt;
    uint64_t *st = (uint64_t *)malloc((cnt + 1) * sizeof(uint64_t));
    cnt = 0;
    for (uint64_t n = 0; n < t->nnz; ++n)
        if (n == 0 || t->ind[m][n] != t->ind[m][n - 1]) st[cnt++] = n;
    st[cnt] = t->nnz;
    *nrows = cnt;
    return st;
}

int orc_als_mode_omp(const orc_tensor *t, int m, double **U, int R, double lambda,
                     int nthreads)
{
    memset(U[m], 0, sizeof(double) * t->dims[m] * (uint64_t)R);
    uint64_t nrows;
    uint64_t *st = row_starts(t, m, &nrows);
    int bad = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : bad)
    {
        double *G = (double *)malloc(sizeof(double) * R * R);
        double *rhs = (double *)malloc(sizeof(double) * R);
        double *h = (double *)malloc(sizeof(double) * R);
        int lbad = 0;
#pragma omp for schedule(dynamic, 16)
        for (int64_t r = 0; r < (int64_t)nrows; ++r)
            als_row(t, m, U, R, lambda, NULL, 0, st[r], st[r + 1], G, rhs, h, &lbad);
        bad += lbad;
        free(G);
        free(rhs);
        free(h);
    }
    free(st);
    return bad;
}

/* ------------------------------------------------------------------ */
/* CCD                                                                  */
/* ------------------------------------------------------------------ */

/* sgpu/ccd.cu:82-206 (update_frac_gpu_as) and ccd.cu:318-348
 * (update_ccd_gpu): per directory row, all columns at once, residual taken
 * with the old row of the target factor. */
void orc_ccd_compat_mode(const orc_tensor *t, int m, double **U, int R, double lambda,
                         const double *w, int trunc)
{
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
    const uint64_t nnz = t->nnz;
    double *num = (double *)malloc(sizeof(double) * R);
    double *den = (double *)malloc(sizeof(double) * R);
    double *h = (double *)malloc(sizeof(double) * R);
    uint64_t s = 0;
    while (s < nnz) {
        uint64_t e = s + 1;
        while (e < nnz && t->ind[m][e] == t->ind[m][s]) ++e;
        double *a = U[m] + (t->ind[m][s] - 1) * (uint64_t)R;
        for (int f = 0; f < R; ++f) num[f] = den[f] = 0;
        for (uint64_t n = s; n < e; ++n) {
            double wn = w ? w[n] : 1.0;
            if (wn == 0.0) continue;
            const double *b = U[m1] + (t->ind[m1][n] - 1) * (uint64_t)R;
            const double *c = U[m2] + (t->ind[m2][n] - 1) * (uint64_t)R;
            double x = trunc ? orc_ref_value_trunc(t->vals[n]) : t->vals[n];
            for (int f = 0; f < R; ++f) {
                h[f] = b[f] * c[f];
                x -= a[f] * h[f];
            }
            for (int f = 0; f < R; ++f) {
                den[f] += wn * h[f] * h[f];
                num[f] += wn * h[f] * x;
            }
        }
        for (int f = 0; f < R; ++f) a[f] = num[f] / (lambda + den[f]);
        s = e;
    }
    free(num);
    free(den);
    free(h);
}

void orc_residual(const orc_tensor *t, double *const *U, int R, double *resid)
{
    for (uint64_t n = 0; n < t->nnz; ++n) resid[n] = t->vals[n] - predict3(t, U, R, n);
}

static inline double rank1(const orc_tensor *t, double *const *U, int R, int f, uint64_t n)
{
    return U[0][(t->ind[0][n] - 1) * (uint64_t)R + f] *
           U[1][(t->ind[1][n] - 1) * (uint64_t)R + f] *
           U[2][(t->ind[2][n] - 1) * (uint64_t)R + f];
}

/* CCD++ (the rank-one residual loop sketched, commented out, at
 * sgpu/ccd.cu:531-556): per column f, r += a_f o b_f o c_f; `inner` sweeps
 * over the modes of u_i = sum(r h) / (lambda + sum h^2); r -= new term. */
static void ccdpp_impl(const orc_tensor *t, double **U, int R, double lambda, int inner,
                       double *resid, int nthreads)
{
    const uint64_t nnz = t->nnz;
    uint64_t maxd = 0;
    for (int m = 0; m < 3; ++m) if (t->dims[m] > maxd) maxd = t->dims[m];
    int nt = nthreads > 0 ? nthreads : 1;
    double *num = (double *)calloc(maxd * (uint64_t)nt, sizeof(double));
    double *den = (double *)calloc(maxd * (uint64_t)nt, sizeof(double));
    for (int f = 0; f < R; ++f) {
#pragma omp parallel for num_threads(nt) schedule(static) if (nt > 1)
        for (int64_t n = 0; n < (int64_t)nnz; ++n) resid[n] += rank1(t, U, R, f, (uint64_t)n);
        for (int it = 0; it < inner; ++it) {
            for (int m = 0; m < 3; ++m) {
                const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
                const uint64_t D = t->dims[m];
                memset(num, 0, sizeof(double) * D * nt);
                memset(den, 0, sizeof(double) * D * nt);
#pragma omp parallel num_threads(nt) if (nt > 1)
                {
                    int tid = 0;
#ifdef _OPENMP
                    tid = omp_get_thread_num();
#endif
                    double *nu = num + (uint64_t)tid * D, *de = den + (uint64_t)tid * D;
#pragma omp for schedule(static)
                    for (int64_t n = 0; n < (int64_t)nnz; ++n) {
                        double h = U[m1][(t->ind[m1][n] - 1) * (uint64_t)R + f] *
                                   U[m2][(t->ind[m2][n] - 1) * (uint64_t)R + f];
                        uint64_t row = t->ind[m][n] - 1;
                        nu[row] += resid[n] * h;
                        de[row] += h * h;
                    }
                }
                for (uint64_t r = 0; r < D; ++r) {
                    double a = 0, b = 0;
                    for (int q = 0; q < nt; ++q) { a += num[(uint64_t)q * D + r]; b += den[(uint64_t)q * D + r]; }
                    U[m][r * (uint64_t)R + f] = a / (lambda + b);
                }
            }
        }
#pragma omp parallel for num_threads(nt) schedule(static) if (nt > 1)
        for (int64_t n = 0; n < (int64_t)nnz; ++n) resid[n] -= rank1(t, U, R, f, (uint64_t)n);
    }
    free(num);
    free(den);
}

void orc_ccdpp_outer(const orc_tensor *t, double **U, int R, double lambda, int inner,
                     double *resid)
{
    ccdpp_impl(t, U, R, lambda, inner, resid, 1);
}

void orc_ccdpp_outer_omp(const orc_tensor *t, double **U, int R, double lambda, int inner,
                         double *resid, int nthreads)
{
    ccdpp_impl(t, U, R, lambda, inner, resid, nthreads);
}

/* ------------------------------------------------------------------ */
/* SGD                                                                  */
/* ------------------------------------------------------------------ */

/* sgpu/sgd.cu:75-99: rows gathered, e = x - sum (a*b)*c, then
 * a_f += (lr*moda)*scale with moda = (e*b_f)*c_f - lambda*a_f,
 * modb = (e*a_f)*c_f - lambda*b_f, modc = (e*b_f)*a_f - lambda*c_f. */
static inline void sgd_one(const orc_tensor *t, double **U, int R, double lr, double lambda,
                           double scale, int trunc, uint64_t n, double *ta, double *tb,
                           double *tc)
{
    double *a = U[0] + (t->ind[0][n] - 1) * (uint64_t)R;
    double *b = U[1] + (t->ind[1][n] - 1) * (uint64_t)R;
    double *c = U[2] + (t->ind[2][n] - 1) * (uint64_t)R;
    double x = trunc ? orc_ref_value_trunc(t->vals[n]) : t->vals[n];
    for (int f = 0; f < R; ++f) { ta[f] = a[f]; tb[f] = b[f]; tc[f] = c[f]; }
    double p = 0;
    for (int f = 0; f < R; ++f) p += ta[f] * tb[f] * tc[f];
    double e = x - p;
    for (int f = 0; f < R; ++f) {
        double moda = (e * tb[f] * tc[f]) - (lambda * ta[f]);
        double modb = (e * ta[f] * tc[f]) - (lambda * tb[f]);
        double modc = (e * tb[f] * ta[f]) - (lambda * tc[f]);
        a[f] += lr * moda * scale;
        b[f] += lr * modb * scale;
        c[f] += lr * modc * scale;
    }
}

void orc_sgd_epoch(const orc_tensor *t, double **U, int R, double lr, double lambda,
                   double scale, int trunc)
{
    double *tmp = (double *)malloc(sizeof(double) * 3 * R);
    for (uint64_t n = 0; n < t->nnz; ++n)
        sgd_one(t, U, R, lr, lambda, scale, trunc, n, tmp, tmp + R, tmp + 2 * R);
    free(tmp);
}

void orc_sgd_epoch_hogwild(const orc_tensor *t, double **U, int R, double lr, double lambda,
                           double scale, int nthreads)
{
#pragma omp parallel num_threads(nthreads)
    {
        double *tmp = (double *)malloc(sizeof(double) * 3 * R);
#pragma omp for schedule(static)
        for (int64_t n = 0; n < (int64_t)t->nnz; ++n)
            sgd_one(t, U, R, lr, lambda, scale, 0, (uint64_t)n, tmp, tmp + R, tmp + 2 * R);
        free(tmp);
    }
}

/* ------------------------------------------------------------------ */
/* Adjoint of the masked CP loss                                        */
/* ------------------------------------------------------------------ */

double orc_objective(const orc_tensor *t, double *const *U, int R, double lambda)
{
    return 0.5 * orc_sq_loss(t, U, R) + orc_frob(t->nmodes, t->dims, U, R, lambda);
}

void orc_grad(const orc_tensor *t, double *const *U, int R, double lambda, double **G)
{
    for (int m = 0; m < 3; ++m)
        for (uint64_t x = 0; x < t->dims[m] * (uint64_t)R; ++x) G[m][x] = 2.0 * lambda * U[m][x];
    for (uint64_t n = 0; n < t->nnz; ++n) {
        uint64_t i = t->ind[0][n] - 1, j = t->ind[1][n] - 1, k = t->ind[2][n] - 1;
        const double *a = U[0] + i * R, *b = U[1] + j * R, *c = U[2] + k * R;
        double e = t->vals[n] - predict3(t, U, R, n);
        for (int f = 0; f < R; ++f) {
            G[0][i * R + f] -= e * b[f] * c[f];
            G[1][j * R + f] -= e * a[f] * c[f];
            G[2][k * R + f] -= e * a[f] * b[f];
        }
    }
}
