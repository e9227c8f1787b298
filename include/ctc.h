/*
 * ctc.h -- C ABI of the B200-native sparse tensor-completion engine
 * (libctc.so, built from cutc_b200/csrc/).
 *
 * Drop-in for the single-GPU driver of cuTC (abovekumo/cuTC).  Each entry
 * point names the reference interface it replaces, as file:line relative to
 * the reference project ("sgpu/" = "software/single GPU/sgpu/", "ga/" =
 * "software/autotuning/performance_GA/").
 *
 * Conventions
 *   - every function returns CTC_OK (0) or a negative CTC_E_* code and
 *     leaves a message for ctc_last_error() (thread-local); nothing exits
 *     the process (the reference calls exit(-1), sgpu/base.h:79-90);
 *   - handles are caller-owned and freed with the matching *_free/destroy;
 *   - a ctc_ctx owns one CUDA device and one stream; calls on one context
 *     are serialised by the caller, different contexts are independent;
 *   - tensors keep their indices exactly as read (1-based .tns files, as the
 *     reference kernels require: sgpu/als.cu:256-258) and their values in
 *     double; factors cross the ABI as row-major double, dims[m] x rank.
 */
#ifndef CTC_H
#define CTC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CTC_OK 0
#define CTC_E_ARG (-1)      /* invalid argument                        */
#define CTC_E_IO (-2)       /* file could not be opened / parsed        */
#define CTC_E_CUDA (-3)     /* CUDA runtime error                        */
#define CTC_E_NOMEM (-4)    /* host or device allocation failed          */
#define CTC_E_UNSUP (-5)    /* unsupported rank / order / combination    */
#define CTC_E_NUMERIC (-6)  /* non-finite result                          */
#define CTC_E_TIMEOUT (-7)  /* bounded device wait expired                */
#define CTC_E_NOGPU (-8)    /* no CUDA device                             */
#define CTC_E_NOTFOUND (-9) /* no entry (tuning cache lookup)             */

typedef struct ctc_ctx ctc_ctx;
typedef struct ctc_tensor ctc_tensor;
typedef struct ctc_ciss ctc_ciss;
typedef struct ctc_model ctc_model;
typedef struct ctc_dataset ctc_dataset;

/* ---------------------------------------------------------------- */
/* errors, version                                                   */
/* ---------------------------------------------------------------- */
const char *ctc_last_error(void);
const char *ctc_version(void);

/* ---------------------------------------------------------------- */
/* context                                                           */
/* ---------------------------------------------------------------- */
/* Select `device` and create the context's stream.  The reference picks
 * device 0 inside every driver (sgpu/als.cu:535, sgpu/sgd.cu:178). */
int ctc_ctx_create(int device, ctc_ctx **out);
int ctc_ctx_destroy(ctc_ctx *ctx);
/* Number of kernels this library launched on the context so far. */
int ctc_ctx_kernel_launches(const ctc_ctx *ctx, uint64_t *out);
/* The context's cudaStream_t, for callers timing with CUDA events. */
void *ctc_ctx_stream(ctc_ctx *ctx);

/* ---------------------------------------------------------------- */
/* tensors (host)                                                    */
/* ---------------------------------------------------------------- */
/* Replaces tt_read (sgpu/sptensor.c:64 -> sgpu/io.c:195-217, text form
 * io.c:58-106 + tt_get_dims io.c:234-308): whitespace "i j k v" lines,
 * '#' and empty lines skipped, mode count from the first data line,
 * dims[m] = max index (+1 when an index 0 occurs).  Parsed in parallel.
 * Files ending in ".ctcb" use the binary form of ctc_tensor_save_bin;
 * files ending in ".bin" are SPLATT binary coordinate tensors (see
 * ctc_tensor_save_splatt).  A binary file too short for its header's
 * nonzero count is rejected (CTC_E_IO) before anything is allocated. */
int ctc_tensor_load_tns(const char *path, ctc_tensor **out);
/* SPLATT binary coordinate form, the reference's .bin path
 * (sgpu/io.c:116-150 p_write_tt_binary_header, io.c:347-431
 * tt_write_binary_file; header sgpu/io.h:67-84): int32 magic 0, u64
 * idx_width, u64 val_width, then idx_width-byte nmodes, dims[nmodes], nnz,
 * the index arrays (as stored: 1-based from .tns files) and nnz values of
 * val_width bytes.  The reference writes idx_width 8 and, through a
 * comparison of a double with itself (io.c:137-143), always val_width 4,
 * and its reader exits on idx_width 8 (io.c:444-449): its own files are
 * unreadable.  Here the loader reads idx_width 4 or 8 and val_width 4 or 8
 * (so the reference's files too), and the writer uses 4-byte words when
 * every count and index fits, 4-byte values only when every value is
 * exactly a float. */
int ctc_tensor_save_splatt(const ctc_tensor *t, const char *path);
/* Text output, one line per nonzero: the indices as stored ("%llu "), then
 * the value with "%.<digits>f" (digits 0..40), or "%.17g" (round trip of
 * the double) when digits < 0.  The reference's data-prep scripts write
 * "%d %d %d %.1f" (software/scripts/tvtensor.py:122-129, stensor.py:39-43):
 * digits = 1 gives their bytes. */
int ctc_tensor_write_tns(const ctc_tensor *t, const char *path, int digits);
/* Seeded train / test / validation split of software/scripts/tvtensor.py
 * (:64-120): the nonzeros are sorted stably by (ind[0], ind[1]) (:103),
 * then each in that order draws flag = random.randint(0, 9) from Python's
 * Mersenne Twister seeded by random.seed(seed) (the script leaves it
 * unseeded) and goes to train (flag < 8), test (flag == 8) or validation
 * (flag == 9).  Outputs keep that order; dims are each output's maximum
 * index.  Any output pointer may be NULL.  The script's mode-2 and mode-3
 * copies (stensor.py:36-43) are ctc_tensor_sort(t, 1) and (t, 2) of the
 * training output. */
int ctc_tensor_split(const ctc_tensor *t, uint64_t seed, ctc_tensor **train, ctc_tensor **test,
                     ctc_tensor **val);
/* Binary form (replaces the broken .bin path, sgpu/io.c:125, 444-476):
 * header "CTCB", u32 version, u32 nmodes, u64 nnz, u64 dims[nmodes], then
 * nmodes arrays of u64 indices and one array of f64 values. */
int ctc_tensor_save_bin(const ctc_tensor *t, const char *path);
/* Build from caller arrays (copied).  dims may be NULL (max index). */
int ctc_tensor_from_coo(int nmodes, uint64_t nnz, const uint64_t *dims,
                        const uint64_t *const *ind, const double *vals,
                        ctc_tensor **out);
int ctc_tensor_info(const ctc_tensor *t, int *nmodes, uint64_t *nnz, uint64_t *dims);
/* Copy out: ind[m] must hold nnz u64, vals nnz doubles (either may be NULL). */
int ctc_tensor_export(const ctc_tensor *t, uint64_t *const *ind, double *vals);
/* Stable sort by (ind[mode], ind[(mode+1)%n]) in place (mode 0-based), the
 * ordering the reference's input files carry
 * (software/scripts/stensor.py:36-43, tvtensor.py:103). */
int ctc_tensor_sort(ctc_tensor *t, int mode);
int ctc_tensor_free(ctc_tensor *t);

/* ---------------------------------------------------------------- */
/* CISS (TB-COO) tiling                                              */
/* ---------------------------------------------------------------- */
/* Replaces ciss_alloc (sgpu/ciss.c:68-195, mode 1-based, tile length 32)
 * and cissbasic_alloc (ga/ciss.c:69-212, runtime tile length).  The
 * tensor must already be sorted for `mode` (the reference's contract).
 * Bit-exact with the reference on every slot it writes; slots it leaves
 * uninitialised (header[1] of a tile without a row change, the bitmap of a
 * terminator-only tile, the unused tail) are 0.0 here.  tile_len in
 * [1, 64]; bitmaps above 53 bits round as the reference's do. */
int ctc_ciss_build(const ctc_tensor *t, int mode, int tile_len, ctc_ciss **out);
/* The GA builder's form (ga/ciss.c:69-212 with one partition covering all
 * rows): identical tiles; its directory counters count the first nonzero
 * too (ga/ciss.c:101-120), so dcounter[k] = start of slice k. */
int ctc_ciss_build_ga(const ctc_tensor *t, int mode, int tile_len, ctc_ciss **out);
/* The same CISS built on the GPU of `ctx`, bit-exact with ctc_ciss_build
 * (CTC_CISS_GA: with ctc_ciss_build_ga's counters).  With CTC_CISS_SORT
 * the nonzeros are first sorted for `mode` on the device (stable by the
 * mode index, then the next mode's index: the order of the reference's
 * traina/b/c files); without it `t` must already be in that order, as for
 * ciss_alloc.  Same ownership and export as ctc_ciss_build. */
#define CTC_CISS_GA 1
#define CTC_CISS_SORT 2
int ctc_ciss_build_gpu(ctc_ctx *ctx, const ctc_tensor *t, int mode, int tile_len, int flags,
                       ctc_ciss **out);
int ctc_ciss_sizes(const ctc_ciss *c, uint64_t *nnz, uint64_t *dlength,
                   uint64_t *size_rows, int *tile_len);
/* directory: dlength u64; dcounter: dlength+1 u64; entries: size_rows*3 f64;
 * written (may be NULL): size_rows*3 bytes, 1 where the reference writes. */
int ctc_ciss_export(const ctc_ciss *c, uint64_t *directory, uint64_t *dcounter,
                    double *entries, uint8_t *written);
int ctc_ciss_free(ctc_ciss *c);

/* Work-tile plan of a copy sorted for one mode (ind: that mode's 1-based
 * indices, n of them): at most tile_len nonzeros per tile, whole rows
 * packed, longer rows split into pieces.  tiles: 4 int32 per tile {first
 * nonzero, length, heavy-row index or -1, piece}; heavy: 4 uint32 per long
 * row {row (0-based), first tile, tiles, 0}.  from_runs = 1 builds it from
 * the rows' run lengths (the planner of the device staging), 0 from the
 * index array (the host staging's planner); the two give the same plan.
 * The counts are always written, each array only when its capacity holds
 * it.  CTC_E_ARG when ind is not sorted. */
int ctc_plan_tiles(const uint64_t *ind, uint64_t n, uint32_t tile_len, int from_runs, int32_t *tiles,
                   uint64_t tiles_cap, uint64_t *ntiles, uint32_t *heavy, uint64_t heavy_cap,
                   uint64_t *nheavy);

/* ---------------------------------------------------------------- */
/* factor model                                                      */
/* ---------------------------------------------------------------- */
/* Replaces the factor arrays of tc_main_ciss (sgpu/completion.c:422-450,
 * matrix_randomize / fill_rand sgpu/matrixprocess.c:156-165, 568-577). */
int ctc_model_create(int nmodes, const uint64_t *dims, int rank, ctc_model **out);
/* Seeded U(0,1)*scale init (scale 1/sqrt(rank) in the workloads); a
 * counter-based generator, so the result depends only on (seed, mode,
 * row, column). */
int ctc_model_init_uniform(ctc_model *m, uint64_t seed, double scale);
int ctc_model_set(ctc_model *m, int mode, const double *rowmajor);
int ctc_model_get(const ctc_model *m, int mode, double *rowmajor);
/* Factor output and checkpoints.  write_text: factor `mode` (0-based) as the
 * reference's mat_write (sgpu/io.c:554-591, unused by its drivers): one row
 * per line, each value "%+0.8le ".  save / load: an exact binary checkpoint
 * of all factors (FP64 bits), to resume a run with ctc_run or a dataset;
 * load allocates the model (free with ctc_model_free). */
int ctc_model_write_text(const ctc_model *m, int mode, const char *path);
int ctc_model_save(const ctc_model *m, const char *path);
int ctc_model_load(const char *path, ctc_model **out);
int ctc_model_copy(const ctc_model *src, ctc_model *dst);
int ctc_model_info(const ctc_model *m, int *nmodes, uint64_t *dims, int *rank);
int ctc_model_free(ctc_model *m);

/* ---------------------------------------------------------------- */
/* algorithms                                                        */
/* ---------------------------------------------------------------- */
enum ctc_alg {
    CTC_ALG_ALS = 0,        /* tc_als, sgpu/als.cu:512-843                   */
    CTC_ALG_SGD = 1,        /* tc_sgd, sgpu/sgd.cu:155-342                   */
    CTC_ALG_CCD = 2,        /* tc_ccd ("CCD+"), sgpu/ccd.cu:359-661           */
    CTC_ALG_CCDPP = 3       /* rank-one CCD++ (the loop sgpu/ccd.cu:531-556
                               leaves commented out)                          */
};
enum ctc_precision {
    CTC_PREC_F32 = 0,       /* FP32 factors and accumulation (plain form)     */
    CTC_PREC_F64 = 1,       /* FP64 throughout (the reference's arithmetic)   */
    CTC_PREC_MIXED = 2      /* BF16 factor reads, FP32 masters/accumulation   */
};
enum ctc_lr_schedule {
    CTC_LR_BOLD_DRIVER = 0, /* x1.05 / x0.5 from epoch 2 (sgpu/sgd.cu:315-321) */
    CTC_LR_EXP_DECAY = 1,   /* lr *= lr_decay after every epoch                */
    CTC_LR_CONSTANT = 2
};
enum ctc_sgd_order {
    CTC_SGD_HOGWILD = 0,    /* tiles in parallel, lock-free updates           */
    CTC_SGD_SEQUENTIAL = 1  /* one warp, tile-major entry-minor: deterministic */
};

typedef struct {
    int alg;               /* enum ctc_alg                                          */
    int rank;              /* 8, 16, 32 or 64 (reference: DEFAULT_NFACTORS 16)      */
    double lambda;         /* regularisation (reference: ALS 10, SGD 1e-3, CCD 100) */
    double lr;             /* SGD learning rate (reference LEARN_RATE 1e-3)         */
    double lr_scale;       /* SGD step multiplier (reference SGD_MODIFICATION 1e-5) */
    int lr_schedule;       /* enum ctc_lr_schedule                                  */
    double lr_decay;       /* factor for CTC_LR_EXP_DECAY                           */
    int iters;             /* epochs (reference DEFAULT_MAX_ITERATE 1000)           */
    int inner;             /* CCD++ inner sweeps per column                         */
    int tile_len;          /* nonzeros per warp work unit (0 = tuned)               */
    int threads_per_block; /* Hogwild SGD threads per block, the reference GA's
                              block-size gene (ga/sgd.cu:66-78, fitness.c:67-75:
                              2^(2..9)): 32, 64, 128, 256 or 512; 0 = 256 (an
                              autotuner axis).  4-16 are rejected (CTC_E_UNSUP:
                              a block is whole warps here).  1024 is accepted
                              for sgd_atomic 3 when a lane holds at most two
                              16-byte slices of a row (threads_per_row >=
                              rank / 8), else CTC_E_UNSUP.  The other
                              algorithms' kernels have fixed block shapes and do
                              not read it                                        */
    int precision;         /* enum ctc_precision                                    */
    int compat;            /* 1: reference kernel semantics (values stored through
                              an integer, sgpu/ciss.c:163; ALS/CCD per-tile lane
                              multiplicities; CCD grid coverage, sgpu/ccd.cu:520)   */
    int early_stop;        /* 1: tc_converge rule (sgpu/completion.c:296-362)       */
    double tolerance;      /* early-stop tolerance (reference TOLERANCE 1e-4)       */
    int max_bad_epochs;    /* reference MAX_BADEPOCHS 3                             */
    int mode_start;        /* first mode of the rotation (reference: rand()%3,
                              sgpu/als.cu:684-685; fixed here)                      */
    int sgd_order;         /* enum ctc_sgd_order                                    */
    int sgd_atomic;        /* Hogwild: 2 = each nonzero's three row deltas added by
                              three bulk row reductions from shared memory (FP32;
                              the default), 1 = vector atomic adds, 0 = plain
                              stores, 3 = block-merged hot rows (FP32): the
                              block's groups step together, one nonzero each, and
                              the deltas of each mode's 32 most frequent rows are
                              summed in shared memory and added once per step
                              (the step's nonzeros act as simultaneous Hogwild
                              updates); the other rows as in 1                     */
    int eval_every;        /* evaluate RMSE every n epochs (0 = only at the end)    */
    int use_graph;         /* capture the epoch in a CUDA graph when possible       */
    uint64_t seed;         /* reserved for stochastic modes                          */
    int sgd_groups;        /* Hogwild: nonzero groups in flight (0 = default)       */
    int sgd_conflicts;     /* Hogwild: bound K on the expected number of in-flight
                              updates of one row, G * nnz(row) / nnz; rows above it
                              take steps scaled by K / that number, so a hot row
                              moves by at most ~K single steps per wave of stale
                              updates (0 = 128, < 0 = no scaling).  With one group
                              in flight (sequential order) no row is scaled.       */
    int threads_per_row;   /* SGD: lanes per nonzero (each holds rank/lanes values of
                              the three rows); 0 = rank/4 (FP32) or rank/2 (FP64).
                              The reference uses one thread per nonzero
                              (sgpu/sgd.cu:32)                                      */
    int smem_budget;       /* CCD++: shared memory per block (bytes) for the factor
                              columns a pass gathers; columns that fit are staged
                              there once per block.  0 = 110 KiB, < 0 = none.  A
                              column's first pass stages both gathered modes'
                              half packs in one 1024-thread block per SM when
                              they fit twice the budget (0: the block's whole
                              shared memory)                                        */
} ctc_params;

/* Reference-default parameters for an algorithm (sgpu/base.h:19-64). */
int ctc_params_default(int alg, ctc_params *p);
/* The checks ctc_run / ctc_dataset_create / ctc_autotune make on `p`
 * (algorithm, precision, rank, tile length, block size ...), on the host:
 * CTC_OK, or the code and message those calls would fail with.  Lets a
 * parameter search (the reference's GA, ga/fitness.c:67-79) drop invalid
 * candidates without a device. */
int ctc_params_check(const ctc_params *p);

typedef struct {
    int epoch;
    double loss;       /* training sum of squared errors (sgpu/completion.c:166) */
    double frob;       /* lambda * sum ||U||^2                                    */
    double rmse_tr, rmse_vl, rmse_te;   /* -1 when the tensor was not given     */
    double ms_epoch;   /* device time of the epoch's update kernels              */
    double lr;
} ctc_epoch_stats;

/* Called after every evaluated epoch; a non-zero return stops the run. */
typedef int (*ctc_epoch_cb)(void *user, const ctc_epoch_stats *s);

typedef struct {
    int epochs_run;
    int best_epoch;
    double best_rmse;       /* best validation RMSE (train RMSE without one)   */
    double final_rmse_tr, final_rmse_vl, final_rmse_te;
    double total_ms;        /* device time of all update kernels                */
    uint64_t nonspd_rows;   /* ALS rows whose system needed a diagonal shift    */
} ctc_result;

/* Replaces tc_als / tc_sgd / tc_ccd (sgpu/als.cuh:20-33, sgd.cuh:18-32,
 * ccd.cuh:20-33) and tc_main_ciss (sgpu/completion.c:422-497):
 * train[m] is the training tensor sorted for mode m (the reference's
 * traina/b/c); train[1], train[2] may be NULL: those copies are then sorted
 * on the device from train[0] in ctc_tensor_sort's order (stable by the
 * mode index, then the next mode's), so a run with only train[0] equals
 * one with the three host-sorted copies.  CCD++ orders the nonzeros of
 * each row further by the other two indices (the larger mode first),
 * whichever copies are given.  Only train[0] crosses PCIe when the others
 * are NULL.  val/test may be NULL.  `model` holds the initial factors
 * and receives the final ones; `best` (may be NULL) receives the factors of
 * the best validation epoch (tc_converge's best_mats).  Everything is
 * staged to the device inside the call and released before it returns. */
int ctc_run(ctc_ctx *ctx, const ctc_tensor *const train[3], const ctc_tensor *val,
            const ctc_tensor *test, ctc_model *model, ctc_model *best,
            const ctc_params *p, ctc_epoch_cb cb, void *user, ctc_result *res);

/* Device-resident form of the same run: the tensors are staged once
 * (records, tiles, sorted copies) and epochs run on HBM-resident data.
 * The factor rows are the maximum index over train/val/test per mode
 * (ctc_dataset_dims); models given to the dataset must have those rows. */
int ctc_dataset_create(ctc_ctx *ctx, const ctc_tensor *const train[3],
                       const ctc_tensor *val, const ctc_tensor *test,
                       const ctc_params *p, ctc_dataset **out);
int ctc_dataset_dims(const ctc_dataset *d, uint64_t *dims);
int ctc_dataset_free(ctc_dataset *d);
/* The whole epoch loop of ctc_run on the staged tensors; `p` may change
 * the run-time parameters but not alg/precision/compat/tile_len. */
int ctc_dataset_run(ctc_dataset *d, ctc_model *model, ctc_model *best,
                    const ctc_params *p, ctc_epoch_cb cb, void *user, ctc_result *res);
/* Step-wise control of the same device session (one iteration of the loop
 * in sgpu/als.cu:678-810, sgd.cu:277-324, ccd.cu:521-620 without the host
 * round trip of the factors):
 *   set_model  stages factors (and, for CCD++, the residuals x - model);
 *   epochs     enqueues n update epochs on the context stream and returns
 *              without waiting (no evaluation in between);
 *   set_lr     the SGD step (lr * step scale) of later epochs;
 *   evaluate   waits, then fills loss, frob and the three RMSEs;
 *   get_model  copies the factors out. */
int ctc_dataset_set_model(ctc_dataset *d, const ctc_model *model);
int ctc_dataset_epochs(ctc_dataset *d, int n);
int ctc_dataset_set_lr(ctc_dataset *d, double lr);
int ctc_dataset_evaluate(ctc_dataset *d, ctc_epoch_stats *st);
int ctc_dataset_get_model(ctc_dataset *d, ctc_model *model);
/* Bounded device waits (the tensor-core Gram's wait for its MMAs, the
 * CCD++ pass's wait for its staged columns) give up after about 2 s and
 * set the session's error flag; the next ctc_dataset_evaluate (or the
 * evaluation inside ctc_dataset_run) returns CTC_E_TIMEOUT once and clears
 * the flag, as does ctc_dataset_set_model.  probe_wait is a self-test of
 * that path with no reference counterpart: it enqueues one kernel whose
 * bounded wait, on a barrier nothing arrives at, expires after limit_ns
 * (at most 2e9) and sets the flag. */
int ctc_dataset_probe_wait(ctc_dataset *d, uint64_t limit_ns);

/* Batches of independent completion problems (no reference counterpart;
 * the reference runs one problem per process).  Instance b's training and
 * test tensors (1-based indices, any order) are stacked into one
 * block-diagonal tensor whose mode-m rows of instance b start after the
 * rows of instances 0..b-1, so each epoch is one launch per kernel over all
 * instances, load-balanced by one tile plan.  ALS, CCD and SGD (not CCD++,
 * not compat).  Instance dims are the maximum index over its train/test
 * tensors.  test may be NULL. */
typedef struct ctc_batch ctc_batch;
int ctc_batch_create(ctc_ctx *ctx, int ninst, const ctc_tensor *const *train,
                     const ctc_tensor *const *test, const ctc_params *p, ctc_batch **out);
int ctc_batch_free(ctc_batch *b);
int ctc_batch_info(const ctc_batch *b, int *ninst, uint64_t *nnz_train, uint64_t *nnz_test);
/* Called after every evaluated epoch with each instance's train and test
 * RMSE (test: -1 without test tensors); non-zero stops the run. */
typedef int (*ctc_batch_cb)(void *user, int epoch, int ninst, const double *rmse_tr,
                            const double *rmse_te, double ms_epoch);
/* Runs p->iters epochs of all instances.  models[b]: instance b's initial
 * factors (rank p->rank, at least its dims), replaced by the final ones.
 * The SGD schedule is shared; the bold driver follows the summed training
 * error.  res (may be NULL): totals over all instances. */
int ctc_batch_run(ctc_batch *b, ctc_model *const *models, const ctc_params *p, ctc_batch_cb cb,
                  void *user, ctc_result *res);

/* Autotuner (replaces the reference's offline genetic search over tile
 * length and threads per block, ga/ciss.c:69-75, ga/sgd.cu:66-78,
 * fitness.c:67-79).  For the shape of train[0] (dims, nonzeros, rounded to
 * half powers of two), the algorithm, precision and rank of `p` and this
 * device's SM count, it times update epochs over a candidate set: tile
 * length (ALS, CCD, CCD++, SGD), lanes per nonzero (SGD threads_per_row),
 * the FP32 Hogwild reduction mode (SGD sgd_atomic 1, 2 or 3), the SGD
 * block size (threads_per_block, around each tile length's best), CCD++ column
 * staging on/off (smem_budget), and writes the fastest into
 * `out` (a copy of `p` with those fields replaced).  With cache_path, a
 * cached entry for the shape is returned without a search (unless
 * CTC_TUNE_FORCE), and a search stores its winner there (unless
 * CTC_TUNE_NO_WRITE).  trials (may be NULL) receives up to max_trials
 * timings; ntrials the number run (1 with cached = 1 on a cache hit). */
#define CTC_TUNE_FORCE 1
#define CTC_TUNE_NO_WRITE 2
typedef struct {
    int tile_len, threads_per_row, smem_budget;
    double ms_epoch;   /* device time of one update epoch */
    int cached;
    int sgd_atomic;    /* SGD: the Hogwild reduction mode tried */
    int threads_per_block; /* SGD: the block size tried (0 = 256) */
} ctc_tune_trial;
int ctc_autotune(ctc_ctx *ctx, const ctc_tensor *const train[3], const ctc_params *p,
                 const char *cache_path, int flags, ctc_params *out, ctc_tune_trial *trials,
                 int max_trials, int *ntrials);
/* The cached entry for the shape of `train` on a device with sm_count SMs,
 * without a device: CTC_E_NOTFOUND when there is none. */
int ctc_tune_lookup(const char *cache_path, const ctc_tensor *train, const ctc_params *p, int sm_count,
                    ctc_params *out);
/* The cache key of that shape (NUL-terminated, at most len bytes). */
int ctc_tune_key(const ctc_tensor *train, const ctc_params *p, int sm_count, char *buf, int len);

/* First-order training driven by the adjoint (no reference counterpart;
 * the reference's first-order method is per-nonzero SGD, sgpu/sgd.cu:21-143,
 * whose step is the negative gradient of 1/2 e^2 + 1/2 lambda ||a||^2, i.e.
 * lambda twice the lambda below).  Loss of an order-3 or order-4 tensor:
 *     f = 1/2 sum_Omega (x - [[U_1, ..., U_d]])^2 + lambda sum_m ||U_m||^2.
 * Each step takes the gradient of a minibatch of `batch` nonzeros (scaled by
 * nonzeros / batch; batch 0 = full gradient) in one pass, residuals
 * recomputed, and applies Adam to FP32 master factors; with precision
 * CTC_PREC_MIXED the pass gathers BF16 copies of the factors (refreshed by
 * the Adam step) and accumulates in FP32.  The training nonzeros are
 * shuffled once on the device (seeded); each epoch visits the minibatches
 * in a seeded random order. */
typedef struct {
    int rank;           /* 8, 16, 32 or 64 */
    int precision;      /* CTC_PREC_F32 or CTC_PREC_MIXED (BF16 gathers)      */
    double lambda;
    double lr, beta1, beta2, eps;   /* Adam */
    uint64_t batch;     /* nonzeros per step; 0 = the whole tensor            */
    int epochs;
    uint64_t seed;      /* shuffle and minibatch order                         */
    int eval_every;     /* epochs between evaluations; 0 = only the last       */
} ctc_fo_params;
typedef struct ctc_fo ctc_fo;
int ctc_fo_params_default(ctc_fo_params *p);
int ctc_fo_create(ctc_ctx *ctx, const ctc_tensor *train, const ctc_tensor *test,
                  const ctc_fo_params *p, ctc_fo **out);
int ctc_fo_free(ctc_fo *f);
int ctc_fo_dims(const ctc_fo *f, int *order, uint64_t *dims);
/* model: order and rows of the tensors (ctc_fo_dims), rank p->rank; initial
 * factors in, final factors out.  cb gets loss (training SSE), frob
 * (lambda sum ||U||^2) and the train/test RMSE after evaluated epochs. */
int ctc_fo_run(ctc_fo *f, ctc_model *model, const ctc_fo_params *p, ctc_epoch_cb cb, void *user,
               ctc_result *res);
/* The gradient the training step uses, for checking it: at `model`, over
 * every training nonzero of f in one pass of the minibatch adjoint kernel
 * (scale 1), with the precision and lambda f was created with (FP32 or
 * BF16 gathers, FP32 accumulation), plus 2 lambda U added in FP64.
 * grads[m]: dims[m] x rank row-major doubles; obj (may be NULL): the
 * pass's FP64 loss sum + lambda sum ||U||^2.  ctc_grad gives the same
 * quantities in FP64. */
int ctc_fo_grad(ctc_fo *f, const ctc_model *model, double *const *grads, double *obj);

/* Per-kernel device time: with profiling on, every launch of this library
 * on the context is bracketed by a CUDA event pair; kernel_time sums the
 * launches whose kernel name contains `name` (count, milliseconds).  No
 * reference counterpart (the reference times with gettimeofday around
 * kernels and copies, sgpu/als.cu:682-799). */
int ctc_ctx_set_profiling(ctc_ctx *ctx, int on);
int ctc_ctx_kernel_time(ctc_ctx *ctx, const char *name, uint64_t *count, double *total_ms);
int ctc_ctx_reset_kernel_times(ctc_ctx *ctx);

/* RMSE of `model` on tensor `t` on the GPU (sgpu/completion.c:123-130 with
 * rows read at index-1).  The reduction is deterministic (fixed order). */
int ctc_rmse(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double *rmse);

/* Squared-error sum over nonzeros already on the device, allocating no
 * device memory.  No counterpart in the reference.  For callers that cannot
 * call cudaMalloc (a process whose GPU memory another allocator has fully
 * reserved, or a loop that cannot take an allocation's device-wide
 * synchronisation).  rec: n device records {i0, i1, i2, value bits} (uint4,
 * 0-based indices, FP32 value); U0..U2: device row-major FP32 factors
 * (dims x rank); out_sse: one device double receiving sum (x - xhat)^2;
 * stream: a cudaStream_t (NULL = legacy default stream).  Asynchronous.
 * rec, U0, U1, U2 must be 16-byte aligned and out_sse 8-byte aligned
 * (CTC_E_ARG otherwise, before any launch); every record's i0, i1, i2 must
 * be below the row count of U0, U1, U2 (not checked: there is no dims
 * argument, and an index past the rows reads out of bounds).
 * Scratch is a fixed 512 KiB file-scope device array (65536 partial sums
 * of 16384 nonzeros), held until exit by every GPU that loads the library:
 * n above 2^30 is rejected (CTC_E_ARG).  All calls share that array, so
 * calls that overlap on the GPU race.  The first call on a device looks up
 * the array's address (make it before any stream capture there); under
 * CUDA's lazy module loading that first call, or the library's first kernel
 * launch on the device, also loads the array, which takes device memory:
 * make it before another allocator reserves the device. */
int ctc_sse_noalloc(const void *rec, uint64_t n, const float *U0, const float *U1,
                    const float *U2, int rank, double *out_sse, void *stream);

/* Adjoint of the masked CP loss 1/2 ||P_Omega(X - [[U_1,...,U_d]])||^2 +
 * lambda sum ||U_m||^2 (order d = 3 or 4, FP64): every factor gradient from
 * one pass over the tensor, residuals recomputed, not stored.  grads[m]:
 * dims[m] x rank row-major doubles.  obj (may be NULL) receives the loss
 * value.  No reference counterpart (the reference has no gradient path). */
int ctc_grad(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double lambda,
             double *const *grads, double *obj);

#ifdef __cplusplus
}
#endif
#endif
