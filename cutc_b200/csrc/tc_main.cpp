// tc_main.cpp -- the `tc` command line, with the reference driver's surface
// (sgpu/tc.c:17-60, run as `tc traina trainb trainc validation test`,
// sgpu/run.sh:16) plus run-time options in place of the reference's
// compile-time constants (sgpu/base.h:19-64, tc.c:22).
//
// Output per evaluated epoch, as sgpu/completion.c:111-113, with the test
// RMSE and the epoch's device time added:
//   epoch:%d   loss: %0.5e   RMSE-tr: %0.5e   RMSE-vl: %0.5e   RMSE-te: %0.5e   ms: %.3f
#include "ctc.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

static void usage()
{
    fprintf(stderr,
            "usage: tc traina.tns trainb.tns trainc.tns validation.tns test.tns [options]\n"
            "  --alg als|sgd|ccd|ccdpp   algorithm (default sgd, the reference's algorithm_index 1)\n"
            "  --rank R                  8, 16, 32 or 64 (default 16)\n"
            "  --lambda L                regularisation (default: the reference's per algorithm)\n"
            "  --lr LR                   SGD learning rate (default 1e-3)\n"
            "  --lr-scale S              SGD step multiplier (default 1e-5)\n"
            "  --decay D                 SGD: lr *= D per epoch instead of the bold driver\n"
            "  --iters N                 epochs (default 1000)\n"
            "  --inner K                 CCD++ inner sweeps (default 1)\n"
            "  --tile-len T              nonzeros per warp work unit (default tuned)\n"
            "  --precision f32|f64|mixed (default f32; mixed: ALS tensor-core Gram at rank 32/64,\n"
            "                            CCD++ packed residual slots)\n"
            "  --threads-per-block B     SGD block size, 32..512 (default 256)\n"
            "  --compat                  reference kernel semantics\n"
            "  --no-early-stop           run all epochs\n"
            "  --seed S                  factor initialisation seed (default 0)\n"
            "  --device D                CUDA device (default 0)\n"
            "  --load-model F            start from the checkpoint F (ctc_model_save) instead of a seeded init\n"
            "  --save-model F            write the final factors to checkpoint F\n"
            "  --write-factors PREFIX    write the best-epoch factors as PREFIX1.txt .. PREFIX3.txt\n"
            "                            (one row per line, the reference's mat_write format)\n");
}

static int check(int rc, const char *what)
{
    if (rc != CTC_OK) {
        fprintf(stderr, "tc: %s failed (%d): %s\n", what, rc, ctc_last_error());
        exit(1);
    }
    return rc;
}

static int print_epoch(void *, const ctc_epoch_stats *s)
{
    printf("epoch:%d   loss: %0.5e   RMSE-tr: %0.5e   RMSE-vl: %0.5e   RMSE-te: %0.5e   ms: %.3f\n", s->epoch,
           s->loss, s->rmse_tr, s->rmse_vl, s->rmse_te, s->ms_epoch);
    fflush(stdout);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 6) {
        usage();
        return 2;
    }
    int alg = CTC_ALG_SGD, rank = 16, iters = -1, inner = -1, tile = 0, prec = CTC_PREC_F32, compat = 0;
    int early = 1, device = 0, tpb = 0;
    double lambda = NAN, lr = NAN, lr_scale = NAN, decay = NAN;
    unsigned long long seed = 0;
    const char *load_path = nullptr, *save_path = nullptr, *factors_prefix = nullptr;
    for (int i = 6; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&]() -> const char * {
            if (i + 1 >= argc) {
                usage();
                exit(2);
            }
            return argv[++i];
        };
        if (a == "--alg") {
            std::string v = next();
            alg = v == "als" ? CTC_ALG_ALS : v == "sgd" ? CTC_ALG_SGD : v == "ccd" ? CTC_ALG_CCD
                : v == "ccdpp" ? CTC_ALG_CCDPP : -1;
            if (alg < 0) {
                usage();
                return 2;
            }
        } else if (a == "--rank") rank = atoi(next());
        else if (a == "--lambda") lambda = atof(next());
        else if (a == "--lr") lr = atof(next());
        else if (a == "--lr-scale") lr_scale = atof(next());
        else if (a == "--decay") decay = atof(next());
        else if (a == "--iters") iters = atoi(next());
        else if (a == "--inner") inner = atoi(next());
        else if (a == "--tile-len") tile = atoi(next());
        else if (a == "--precision") {
            const std::string v = next();
            prec = v == "f64" ? CTC_PREC_F64 : v == "mixed" ? CTC_PREC_MIXED : v == "f32" ? CTC_PREC_F32 : -1;
            if (prec < 0) {
                usage();
                return 2;
            }
        } else if (a == "--threads-per-block") tpb = atoi(next());
        else if (a == "--compat") compat = 1;
        else if (a == "--no-early-stop") early = 0;
        else if (a == "--seed") seed = strtoull(next(), nullptr, 10);
        else if (a == "--device") device = atoi(next());
        else if (a == "--load-model") load_path = next();
        else if (a == "--save-model") save_path = next();
        else if (a == "--write-factors") factors_prefix = next();
        else {
            usage();
            return 2;
        }
    }
    ctc_tensor *t[5] = {};
    for (int k = 0; k < 5; ++k) check(ctc_tensor_load_tns(argv[1 + k], &t[k]), argv[1 + k]);
    uint64_t dims[3] = {0, 0, 0};
    for (int k = 0; k < 5; ++k) {
        uint64_t d[4];
        int nm = 0;
        check(ctc_tensor_info(t[k], &nm, nullptr, d), "tensor info");
        if (nm != 3) {
            fprintf(stderr, "tc: %s is not an order-3 tensor\n", argv[1 + k]);
            return 1;
        }
        for (int m = 0; m < 3; ++m) dims[m] = d[m] > dims[m] ? d[m] : dims[m];
    }
    ctc_params p;
    check(ctc_params_default(alg, &p), "params");
    p.rank = rank;
    if (!std::isnan(lambda)) p.lambda = lambda;
    if (!std::isnan(lr)) p.lr = lr;
    if (!std::isnan(lr_scale)) p.lr_scale = lr_scale;
    if (!std::isnan(decay)) {
        p.lr_schedule = CTC_LR_EXP_DECAY;
        p.lr_decay = decay;
    }
    if (iters >= 0) p.iters = iters;
    if (inner > 0) p.inner = inner;
    p.tile_len = tile;
    p.precision = prec;
    p.compat = compat;
    p.early_stop = early;
    p.threads_per_block = tpb;
    check(ctc_params_check(&p), "parameters");
    ctc_ctx *ctx = nullptr;
    check(ctc_ctx_create(device, &ctx), "context");
    ctc_model *model = nullptr, *best = nullptr;
    if (load_path) {
        check(ctc_model_load(load_path, &model), load_path);
    } else {
        check(ctc_model_create(3, dims, rank, &model), "model");
        check(ctc_model_init_uniform(model, seed, 1.0 / std::sqrt((double)rank)), "init");
    }
    check(ctc_model_create(3, dims, rank, &best), "model");
    const ctc_tensor *train[3] = {t[0], t[1], t[2]};
    ctc_result res;
    check(ctc_run(ctx, train, t[3], t[4], model, best, &p, print_epoch, nullptr, &res), "run");
    printf("best epoch %d  best RMSE-vl %0.5e  final RMSE-te %0.5e  update time %.3f ms\n", res.best_epoch,
           res.best_rmse, res.final_rmse_te, res.total_ms);
    if (save_path) check(ctc_model_save(model, save_path), save_path);
    if (factors_prefix)
        for (int m = 0; m < 3; ++m) {
            const std::string f = std::string(factors_prefix) + std::to_string(m + 1) + ".txt";
            check(ctc_model_write_text(best, m, f.c_str()), f.c_str());
        }
    ctc_model_free(model);
    ctc_model_free(best);
    for (int k = 0; k < 5; ++k) ctc_tensor_free(t[k]);
    ctc_ctx_destroy(ctx);
    return 0;
}
