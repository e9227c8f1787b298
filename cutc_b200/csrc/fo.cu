// fo.cu -- first-order (adjoint-driven) training: full-gradient or
// minibatch Adam on the masked CP loss of order-3 and order-4 tensors, with
// FP32 master factors, optional BF16 copies for the gathers, FP32 gradient
// accumulation and FP64 loss sums; and the FP64 order-4 gradient behind
// ctc_grad.  No reference counterpart: the reference's only first-order
// method is per-nonzero SGD (sgpu/sgd.cu:21-143), whose per-nonzero step is
// the negative gradient of 1/2 e^2 + 1/2 lambda ||a||^2 (so its lambda is
// twice the lambda of the loss above).
#include "ctc_internal.h"
#include "runtime.cuh"
#include "fo.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <random>

namespace ctc {

static void fo_validate(const ctc_tensor *t, const uint64_t *dims, int D, const char *what)
{
    if (!t) fail(CTC_E_ARG, "%s: null tensor", what);
    if (t->nmodes != D) fail(CTC_E_ARG, "%s: order %d, expected %d", what, t->nmodes, D);
    if (t->nnz == 0) fail(CTC_E_ARG, "%s: empty tensor", what);
    if (t->nnz >= 0xfffffff0ull) fail(CTC_E_UNSUP, "%s: more than 2^32 nonzeros", what);
    std::atomic<int> bad{0};
    for (int m = 0; m < D; ++m) {
        const uint64_t *ind = t->ind[m].data();
        par_for(t->nnz, [&](uint64_t b, uint64_t e) {
            for (uint64_t i = b; i < e; ++i)
                if (ind[i] == 0 || ind[i] > dims[m]) {
                    bad = 1;
                    return;
                }
        });
    }
    if (bad) fail(CTC_E_ARG, "%s: index 0 or beyond the dimension (indices are 1-based)", what);
}

// records {i0, i1, i2, i3} (0-based; i3 = 0 at order 3) and values (T)
template <typename T>
static void fo_stage(ctc_ctx *ctx, const ctc_tensor *t, int D, DevBuf<uint4> &idx, DevBuf<T> &val)
{
    const uint64_t n = t->nnz;
    idx.alloc(n);
    val.alloc(n);
    const uint64_t *in[4] = {t->ind[0].data(), t->ind[1].data(), t->ind[2].data(), D > 3 ? t->ind[3].data() : nullptr};
    upload_filled(ctx, idx.p, n, [&](uint64_t b, uint64_t e, uint4 *h) {
        for (uint64_t i = b; i < e; ++i)
            h[i - b] = make_uint4((uint32_t)(in[0][i] - 1), (uint32_t)(in[1][i] - 1), (uint32_t)(in[2][i] - 1),
                                  in[3] ? (uint32_t)(in[3][i] - 1) : 0u);
    });
    const double *v = t->vals.data();
    upload_filled(ctx, val.p, n, [&](uint64_t b, uint64_t e, T *h) {
        for (uint64_t i = b; i < e; ++i) h[i - b] = (T)v[i];
    });
    CK(cudaStreamSynchronize(ctx->stream));
}

// a seeded permutation of the records, on the device (radix sort of
// counter-based random keys)
template <typename T>
static void fo_shuffle(ctc_ctx *ctx, DevBuf<uint4> &idx, DevBuf<T> &val, uint64_t seed)
{
    const uint64_t n = idx.n;
    DevBuf<uint64_t> k_in, k_out;
    DevBuf<uint32_t> p_in, p_out;
    k_in.alloc(n);
    k_out.alloc(n);
    p_in.alloc(n);
    p_out.alloc(n);
    LAUNCH(ctx, fo::k_fo_keys, grid_for(n, 256, kSMs * 16), 256, 0, k_in.p, p_in.p, n, seed);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k_in.p, k_out.p, p_in.p, p_out.p, (int)n, 0, 64, ctx->stream));
    DevBuf<unsigned char> scratch;
    scratch.alloc(tmp);
    CK(cub::DeviceRadixSort::SortPairs(scratch.p, tmp, k_in.p, k_out.p, p_in.p, p_out.p, (int)n, 0, 64,
                                       ctx->stream));
    k_in.release();
    k_out.release();
    scratch.release();
    DevBuf<uint4> idx2;
    DevBuf<T> val2;
    idx2.alloc(n);
    val2.alloc(n);
    LAUNCH(ctx, fo::k_fo_gather<T>, grid_for(n, 256, kSMs * 16), 256, 0, (const uint32_t *)p_out.p,
           (const uint4 *)idx.p, (const T *)val.p, idx2.p, val2.p, n);
    CK(cudaStreamSynchronize(ctx->stream));
    std::swap(idx.p, idx2.p);
    std::swap(val.p, val2.p);
}

// shared memory per block for privatised gradient rows
constexpr uint32_t kFoPrivBytes = 48 * 1024;

}  // namespace ctc

struct ctc_fo {
    ctc_ctx *ctx = nullptr;
    int D = 3;
    uint64_t dims[4] = {0, 0, 0, 0};
    uint64_t ntrain = 0, ntest = 0;
    ctc_fo_params p{};
    ctc::DevBuf<uint4> idx, tidx;
    ctc::DevBuf<float> val, tval;
    // parameters of the current run (all modes concatenated, row-major)
    int R = 0;
    uint64_t off[5] = {0, 0, 0, 0, 0};
    ctc::DevBuf<float> U, M, V, G;
    ctc::DevBuf<__nv_bfloat16> Ub;
};

namespace ctc {

static void fo_alloc(ctc_fo *f, int R)
{
    if (f->R == R) return;
    f->R = R;
    f->off[0] = 0;
    for (int m = 0; m < f->D; ++m) f->off[m + 1] = f->off[m] + f->dims[m] * (uint64_t)R;
    const uint64_t n = f->off[f->D];
    f->U.alloc(n);
    f->M.alloc(n);
    f->V.alloc(n);
    f->G.alloc(n);
    f->Ub.alloc(n);
}

template <typename GT, int R, int D, bool GRAD>
static void fo_pass(ctc_fo *f, const uint4 *idx, const float *val, uint64_t b, uint64_t e, double scale,
                    const void *const U[4])
{
    ctc_ctx *ctx = f->ctx;
    fo::FoArgs a{};
    a.idx = idx;
    a.val = val;
    a.begin = b;
    a.end = e;
    uint32_t priv = 0;
    for (int m = 0; m < D; ++m) {
        a.U[m] = U[m];
        a.G[m] = f->G.p + f->off[m];
        a.dims[m] = (uint32_t)f->dims[m];
        const uint32_t need = (uint32_t)(f->dims[m] * R);
        if (GRAD && (priv + need) * sizeof(float) <= kFoPrivBytes) {
            a.priv[m] = 1;
            a.priv_off[m] = priv;
            priv += need;
        }
    }
    a.priv_elems = priv;
    a.scale = scale;
    // bulk row reductions: two staged slots of D rows per nonzero group
    a.bulk = GRAD ? 1 : 0;
    constexpr int kGroups = 8 * (32 / (R / fo::Gather<float, GT>::VE));
    const size_t smem = (priv + (GRAD ? (size_t)kGroups * 2 * D * R : 0)) * sizeof(float);
    if (smem > 48 * 1024)
        CK(cudaFuncSetAttribute(fo::k_fo<float, GT, R, D, GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
    const unsigned g = grid_for(e - b, 256, kMaxPartials);
    // named apart so that per-kernel times separate the adjoint from evaluation
    launch_named(ctx, GRAD ? "fo::k_fo_grad" : "fo::k_fo_eval", fo::k_fo<float, GT, R, D, GRAD>, g, 256, smem, a,
                 ctx->partial.p);
}

template <int R, int D>
static double fo_sse(ctc_fo *f, const uint4 *idx, const float *val, uint64_t n)
{
    ctc_ctx *ctx = f->ctx;
    const void *U[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int m = 0; m < D; ++m) U[m] = f->U.p + f->off[m];
    fo_pass<float, R, D, false>(f, idx, val, 0, n, 1.0, U);
    const unsigned g = grid_for(n, 256, kMaxPartials);
    LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p + 8);
    double half = 0;
    CK(cudaMemcpyAsync(&half, ctx->scalars.p + 8, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 2.0 * half;
}

static double fo_sumsq(ctc_fo *f)
{
    std::vector<float> h(f->U.n);
    CK(cudaMemcpyAsync(h.data(), f->U.p, h.size() * sizeof(float), cudaMemcpyDeviceToHost, f->ctx->stream));
    CK(cudaStreamSynchronize(f->ctx->stream));
    double s = 0;
    for (float v : h) s += (double)v * (double)v;
    return s;
}

template <int R, int D>
static void fo_run(ctc_fo *f, ctc_model *model, const ctc_fo_params &p, ctc_epoch_cb cb, void *user,
                   ctc_result *res)
{
    ctc_ctx *ctx = f->ctx;
    fo_alloc(f, R);
    {
        std::vector<float> h(f->U.n);
        for (int m = 0; m < D; ++m)
            for (uint64_t i = 0; i < f->dims[m] * (uint64_t)R; ++i) h[f->off[m] + i] = (float)model->U[m][i];
        f->U.upload(h.data(), h.size(), ctx->stream);
    }
    const uint64_t n = f->U.n;
    CK(cudaMemsetAsync(f->M.p, 0, n * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(f->V.p, 0, n * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(f->G.p, 0, n * sizeof(float), ctx->stream));
    const bool bf = p.precision == CTC_PREC_MIXED;
    const unsigned ga = grid_for(n, 256, kSMs * 16);
    // BF16 copies of the starting factors (an Adam step with lr 0 is a copy)
    if (bf)
        LAUNCH(ctx, fo::k_fo_adam, ga, 256, 0, f->U.p, f->M.p, f->V.p, f->G.p, f->Ub.p, n, 0.f, 0.f, 0.f, 1.f,
               1.f, 1.f, 0.f);
    const uint64_t batch = (p.batch == 0 || p.batch >= f->ntrain) ? f->ntrain : p.batch;
    const uint64_t nb = (f->ntrain + batch - 1) / batch;
    std::mt19937_64 rng(p.seed ^ 0x5DEECE66DULL);
    std::vector<uint64_t> order(nb);
    uint64_t step = 0;
    double total_ms = 0;
    ctc_epoch_stats st{};
    auto report = [&](int epoch, double ms) -> bool {
        const double sse_tr = fo_sse<R, D>(f, f->idx.p, f->val.p, f->ntrain);
        const double sse_te = f->ntest ? fo_sse<R, D>(f, f->tidx.p, f->tval.p, f->ntest) : 0.0;
        st.epoch = epoch;
        st.loss = sse_tr;
        st.frob = p.lambda * fo_sumsq(f);
        st.rmse_tr = std::sqrt(sse_tr / (double)f->ntrain);
        st.rmse_vl = -1.0;
        st.rmse_te = f->ntest ? std::sqrt(sse_te / (double)f->ntest) : -1.0;
        st.ms_epoch = ms;
        st.lr = p.lr;
        if (!std::isfinite(st.loss)) fail(CTC_E_NUMERIC, "training loss is not finite at epoch %d", epoch);
        return cb ? cb(user, &st) != 0 : false;
    };
    bool stop = report(0, 0.0);
    int e = 1;
    const void *Ug[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int m = 0; m < D; ++m) Ug[m] = bf ? (const void *)(f->Ub.p + f->off[m]) : (const void *)(f->U.p + f->off[m]);
    for (; !stop && e <= p.epochs; ++e) {
        for (uint64_t j = 0; j < nb; ++j) order[j] = j;
        std::shuffle(order.begin(), order.end(), rng);
        CK(cudaEventRecord(ctx->ev0, ctx->stream));
        for (uint64_t j : order) {
            const uint64_t b = j * batch, en = std::min(f->ntrain, b + batch);
            const double scale = (double)f->ntrain / (double)(en - b);
            if (bf) fo_pass<__nv_bfloat16, R, D, true>(f, f->idx.p, f->val.p, b, en, scale, Ug);
            else fo_pass<float, R, D, true>(f, f->idx.p, f->val.p, b, en, scale, Ug);
            ++step;
            const double c1 = 1.0 / (1.0 - std::pow(p.beta1, (double)step));
            const double c2 = 1.0 / (1.0 - std::pow(p.beta2, (double)step));
            LAUNCH(ctx, fo::k_fo_adam, ga, 256, 0, f->U.p, f->M.p, f->V.p, f->G.p,
                   bf ? f->Ub.p : (__nv_bfloat16 *)nullptr, n, (float)p.lr, (float)p.beta1, (float)p.beta2,
                   (float)p.eps, (float)c1, (float)c2, (float)(2.0 * p.lambda));
        }
        CK(cudaEventRecord(ctx->ev1, ctx->stream));
        CK(cudaEventSynchronize(ctx->ev1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        total_ms += ms;
        if (e == p.epochs || (p.eval_every > 0 && e % p.eval_every == 0)) stop = report(e, ms);
    }
    {
        std::vector<float> h(f->U.n);
        CK(cudaMemcpyAsync(h.data(), f->U.p, h.size() * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int m = 0; m < D; ++m)
            for (uint64_t i = 0; i < f->dims[m] * (uint64_t)R; ++i) model->U[m][i] = (double)h[f->off[m] + i];
    }
    if (res) {
        *res = ctc_result{};
        res->epochs_run = e - 1;
        res->best_epoch = e - 1;
        res->best_rmse = st.rmse_tr;
        res->final_rmse_tr = st.rmse_tr;
        res->final_rmse_vl = -1.0;
        res->final_rmse_te = st.rmse_te;
        res->total_ms = total_ms;
    }
}

// Gradient of the whole training loss at `model` through the minibatch
// kernel: one pass over every staged training nonzero (scale 1), with the
// precision the first-order training was created with (FP32 or BF16
// gathers, FP32 accumulation); the lambda term is added in FP64.
template <int R, int D>
static void fo_grad_pass(ctc_fo *f, const ctc_model *model, double *const *grads, double *obj)
{
    ctc_ctx *ctx = f->ctx;
    fo_alloc(f, R);
    {
        std::vector<float> h(f->U.n);
        for (int m = 0; m < D; ++m)
            for (uint64_t i = 0; i < f->dims[m] * (uint64_t)R; ++i) h[f->off[m] + i] = (float)model->U[m][i];
        f->U.upload(h.data(), h.size(), ctx->stream);
    }
    const uint64_t n = f->U.n;
    CK(cudaMemsetAsync(f->G.p, 0, n * sizeof(float), ctx->stream));
    const bool bf = f->p.precision == CTC_PREC_MIXED;
    if (bf) {
        // BF16 copies (an Adam step with lr 0 is a copy)
        CK(cudaMemsetAsync(f->M.p, 0, n * sizeof(float), ctx->stream));
        CK(cudaMemsetAsync(f->V.p, 0, n * sizeof(float), ctx->stream));
        LAUNCH(ctx, fo::k_fo_adam, grid_for(n, 256, kSMs * 16), 256, 0, f->U.p, f->M.p, f->V.p, f->G.p, f->Ub.p, n,
               0.f, 0.f, 0.f, 1.f, 1.f, 1.f, 0.f);
    }
    const void *Ug[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int m = 0; m < D; ++m) Ug[m] = bf ? (const void *)(f->Ub.p + f->off[m]) : (const void *)(f->U.p + f->off[m]);
    if (bf) fo_pass<__nv_bfloat16, R, D, true>(f, f->idx.p, f->val.p, 0, f->ntrain, 1.0, Ug);
    else fo_pass<float, R, D, true>(f, f->idx.p, f->val.p, 0, f->ntrain, 1.0, Ug);
    const unsigned g = grid_for(f->ntrain, 256, kMaxPartials);
    LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p + 8);
    double half = 0;
    CK(cudaMemcpyAsync(&half, ctx->scalars.p + 8, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<float> h(n);
    CK(cudaMemcpyAsync(h.data(), f->G.p, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double lam = f->p.lambda;
    double reg = 0;
    for (int m = 0; m < D; ++m) {
        const std::vector<double> &u = model->U[m];
        for (uint64_t i = 0; i < u.size(); ++i) {
            grads[m][i] = (double)h[f->off[m] + i] + 2.0 * lam * u[i];
            reg += u[i] * u[i];
        }
    }
    if (obj) *obj = half + lam * reg;
}

template <typename F>
static void with_rank_order(int R, int D, F &&f)
{
    with_rank(R, [&](auto RC) {
        if (D == 4) f(RC, std::integral_constant<int, 4>{});
        else f(RC, std::integral_constant<int, 3>{});
    });
}

// FP64 gradient of the whole objective at `model` (order 3 or 4): the
// adjoint kernel in FP64, no privatisation, no BF16
template <int R, int D>
static void fo_grad_f64(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double lambda,
                        double *const *grads, double *obj)
{
    DevBuf<uint4> idx;
    DevBuf<double> val;
    fo_stage<double>(ctx, t, D, idx, val);
    DevBuf<double> U[4], G[4];
    fo::FoArgs a{};
    a.idx = idx.p;
    a.val = val.p;
    a.begin = 0;
    a.end = t->nnz;
    a.scale = 1.0;
    for (int m = 0; m < D; ++m) {
        U[m].upload(model->U[m].data(), model->U[m].size(), ctx->stream);
        G[m].alloc(model->U[m].size());
        CK(cudaMemsetAsync(G[m].p, 0, G[m].n * sizeof(double), ctx->stream));
        a.U[m] = U[m].p;
        a.G[m] = G[m].p;
        a.dims[m] = (uint32_t)model->dims[m];
    }
    const unsigned g = grid_for(t->nnz, 256, kMaxPartials);
    LAUNCH(ctx, (fo::k_fo<double, double, R, D, true>), g, 256, 0, a, ctx->partial.p);
    LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p + 8);
    double half = 0;
    CK(cudaMemcpyAsync(&half, ctx->scalars.p + 8, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    double reg = 0;
    for (int m = 0; m < D; ++m) {
        CK(cudaMemcpyAsync(grads[m], G[m].p, G[m].n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const std::vector<double> &u = model->U[m];
        for (size_t i = 0; i < u.size(); ++i) {
            grads[m][i] += 2.0 * lambda * u[i];
            reg += u[i] * u[i];
        }
    }
    if (obj) *obj = half + lambda * reg;
}

}  // namespace ctc

// order-4 (and order-3) FP64 gradient, used by ctc_grad for order 4
void ctc::ctc_grad_fo(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double lambda,
                      double *const *grads, double *obj)
{
    if (model->nmodes != t->nmodes) fail(CTC_E_ARG, "model order %d, tensor order %d", model->nmodes, t->nmodes);
    fo_validate(t, model->dims, t->nmodes, "tensor");
    with_rank_order(model->rank, t->nmodes, [&](auto RC, auto DC) {
        fo_grad_f64<decltype(RC)::value, decltype(DC)::value>(ctx, t, model, lambda, grads, obj);
    });
}

extern "C" int ctc_fo_params_default(ctc_fo_params *p)
{
    return guarded([&] {
        if (!p) fail(CTC_E_ARG, "null params");
        *p = ctc_fo_params{};
        p->rank = 16;
        p->precision = CTC_PREC_F32;
        p->lambda = 0.0;
        p->lr = 1e-3;
        p->beta1 = 0.9;
        p->beta2 = 0.999;
        p->eps = 1e-8;
        p->batch = (uint64_t)1 << 20;
        p->epochs = 10;
        p->seed = 1;
        p->eval_every = 1;
    });
}

static void fo_check(const ctc_fo_params *p)
{
    if (!p) fail(CTC_E_ARG, "null params");
    if (p->rank != 8 && p->rank != 16 && p->rank != 32 && p->rank != 64) fail(CTC_E_UNSUP, "rank %d", p->rank);
    if (p->precision != CTC_PREC_F32 && p->precision != CTC_PREC_MIXED)
        fail(CTC_E_UNSUP, "first-order training runs in FP32 or mixed (BF16 gathers) precision");
    if (!(p->lr > 0) || !(p->beta1 >= 0 && p->beta1 < 1) || !(p->beta2 >= 0 && p->beta2 < 1) || !(p->eps > 0))
        fail(CTC_E_ARG, "Adam parameters out of range");
    if (p->lambda < 0) fail(CTC_E_ARG, "lambda < 0");
    if (p->epochs < 0) fail(CTC_E_ARG, "epochs < 0");
}

extern "C" int ctc_fo_create(ctc_ctx *ctx, const ctc_tensor *train, const ctc_tensor *test, const ctc_fo_params *p,
                             ctc_fo **out)
{
    using namespace ctc;
    return guarded([&] {
        if (!ctx || !train || !out) fail(CTC_E_ARG, "null argument");
        fo_check(p);
        if (train->nmodes != 3 && train->nmodes != 4) fail(CTC_E_UNSUP, "order %d (3 or 4)", train->nmodes);
        CK(cudaSetDevice(ctx->device));
        auto f = std::make_unique<ctc_fo>();
        f->ctx = ctx;
        f->D = train->nmodes;
        f->p = *p;
        for (int m = 0; m < f->D; ++m) {
            f->dims[m] = std::max(train->dims[m], test ? test->dims[m] : 0);
            if (f->dims[m] >= 0xfffffff0ull) fail(CTC_E_UNSUP, "dimension %d too large", m + 1);
        }
        fo_validate(train, f->dims, f->D, "training tensor");
        fo_stage<float>(ctx, train, f->D, f->idx, f->val);
        fo_shuffle<float>(ctx, f->idx, f->val, p->seed);
        f->ntrain = train->nnz;
        if (test) {
            fo_validate(test, f->dims, f->D, "test tensor");
            fo_stage<float>(ctx, test, f->D, f->tidx, f->tval);
            f->ntest = test->nnz;
        }
        *out = f.release();
    });
}

extern "C" int ctc_fo_free(ctc_fo *f)
{
    if (f) {
        cudaSetDevice(f->ctx->device);
        cudaStreamSynchronize(f->ctx->stream);
        delete f;
    }
    return CTC_OK;
}

extern "C" int ctc_fo_dims(const ctc_fo *f, int *order, uint64_t *dims)
{
    return guarded([&] {
        if (!f) fail(CTC_E_ARG, "null argument");
        if (order) *order = f->D;
        if (dims)
            for (int m = 0; m < f->D; ++m) dims[m] = f->dims[m];
    });
}

extern "C" int ctc_fo_run(ctc_fo *f, ctc_model *model, const ctc_fo_params *p, ctc_epoch_cb cb, void *user,
                          ctc_result *res)
{
    using namespace ctc;
    return guarded([&] {
        if (!f || !model) fail(CTC_E_ARG, "null argument");
        fo_check(p);
        if (model->nmodes != f->D || model->rank != p->rank) fail(CTC_E_ARG, "model order/rank mismatch");
        for (int m = 0; m < f->D; ++m)
            if (model->dims[m] != f->dims[m]) fail(CTC_E_ARG, "model mode %d has %llu rows, the tensors need %llu",
                                                   m, (unsigned long long)model->dims[m],
                                                   (unsigned long long)f->dims[m]);
        CK(cudaSetDevice(f->ctx->device));
        with_rank_order(p->rank, f->D, [&](auto RC, auto DC) {
            fo_run<decltype(RC)::value, decltype(DC)::value>(f, model, *p, cb, user, res);
        });
    });
}

extern "C" int ctc_fo_grad(ctc_fo *f, const ctc_model *model, double *const *grads, double *obj)
{
    using namespace ctc;
    return guarded([&] {
        if (!f || !model || !grads) fail(CTC_E_ARG, "null argument");
        if (model->nmodes != f->D || model->rank != f->p.rank) fail(CTC_E_ARG, "model order/rank mismatch");
        for (int m = 0; m < f->D; ++m)
            if (model->dims[m] != f->dims[m]) fail(CTC_E_ARG, "model mode %d has %llu rows, the tensors need %llu",
                                                   m, (unsigned long long)model->dims[m],
                                                   (unsigned long long)f->dims[m]);
        CK(cudaSetDevice(f->ctx->device));
        with_rank_order(f->p.rank, f->D, [&](auto RC, auto DC) {
            fo_grad_pass<decltype(RC)::value, decltype(DC)::value>(f, model, grads, obj);
        });
    });
}
