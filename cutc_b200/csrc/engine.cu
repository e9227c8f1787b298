// engine.cu -- device-side orchestration of libctc: staging of the mode
// copies, the device-resident session (factors, residuals, scratch), the
// ALS / CCD / CCD++ / SGD epochs (optionally replayed as a CUDA graph),
// evaluation, early stop, and the C ABI entry points that need the GPU.
#include "ctc_internal.h"
#include "runtime.cuh"
#include "kernels.cuh"
#include "als_tc.cuh"
#include "stage_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <type_traits>

double ctc_value_through_idx(double v);

namespace ctc {

namespace {
struct PoolSlot {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
};
std::mutex g_pool_mu;
PoolSlot g_pools[64];

PoolSlot &pool_slot()
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail(CTC_E_UNSUP, "device %d: at most 64 devices", dev);
    std::lock_guard<std::mutex> g(g_pool_mu);
    PoolSlot &s = g_pools[dev];
    if (!s.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        CK(cudaMemPoolCreate(&s.pool, &props));
        uint64_t keep = ~0ull;
        CK(cudaMemPoolSetAttribute(s.pool, cudaMemPoolAttrReleaseThreshold, &keep));
        CK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    }
    return s;
}
}  // namespace

void *dev_alloc(size_t bytes)
{
    PoolSlot &s = pool_slot();
    void *p = nullptr;
    CK(cudaMallocFromPoolAsync(&p, bytes, s.pool, s.stream));
    CK(cudaStreamSynchronize(s.stream));
    return p;
}

void dev_free(void *p) noexcept
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || !g_pools[dev].stream) {
        cudaFree(p);
        return;
    }
    cudaDeviceSynchronize();
    cudaFreeAsync(p, g_pools[dev].stream);
    cudaStreamSynchronize(g_pools[dev].stream);
}

void dev_pool_trim() noexcept
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (g_pools[dev].pool) cudaMemPoolTrimTo(g_pools[dev].pool, 0);
}

// One tensor staged on the device as 16-byte records (+ FP64 values in
// FP64 runs), optionally with its row-aligned work tiles for one mode and
// the reference lane multiplicities.
template <typename T>
struct DevTensor {
    DevBuf<uint4> rec;
    DevBuf<double> v64;
    uint32_t n = 0;
    int mode = -1;
    DevBuf<int4> tiles;
    uint32_t ntiles = 0;
    DevBuf<uint4> heavy;
    DevBuf<uint32_t> pieces;  // tile indices of the heavy pieces
    uint32_t npieces = 0;
    uint32_t nheavy = 0;
    DevBuf<T> w;
    bool has_w = false;
    // CCD++ copies: packed keys, residual, values (no rec)
    DevBuf<uint64_t> keys;
    DevBuf<T> res, x;
    k::KeyShape ks{};
    uint32_t nslots = 0;  // CCD++: ntiles * slot length (lane-interleaved tiles)
    DevBuf<int4> tasks;   // CCD++ warp tasks (light tiles, groups of pieces)
    uint32_t ntasks = 0;
    uint64_t nrows = 0;   // rows of the copy's mode that hold nonzeros (0: not counted)
};

static int bits_for(uint64_t d)
{
    int b = 1;
    while (b < 64 && (1ull << b) < d) ++b;
    return b;
}

// CCD++ copy of mode m: packed 64-bit keys row | q1 | q2 (row = index in
// mode m, q1/q2 = indices in modes m+1, m+2, each in just enough bits) and
// values in the tile slots of `plan` (slot length S = 32 * E): entry p of
// tile t sits at t*S + (p % E)*32 + p / E, so that lane p / E of the warp
// owning the tile holds its E consecutive entries and every warp load is
// coalesced.  Unused slot entries hold kPadKey, value 0 and residual 0.
// The slots are gathered on the device from records in mode-m order
// (rec, or rec through perm); the residual is formed on the device.
// packed (mixed precision, FP32 only): the residual lives in the key word's
// low rbits = min(32, 64 - key bits) bits (at least 16), so a slot entry is
// 8 bytes instead of 12 and there is no residual array.
static int ccdpp_packed_rbits(const uint64_t *dims)
{
    const int kb = bits_for(dims[0]) + bits_for(dims[1]) + bits_for(dims[2]);
    return std::min(32, 64 - kb);
}

template <typename T>
static void stage_keys(ctc_ctx *ctx, const DevTensor<T> &src, const uint32_t *perm, int m, const uint64_t *dims,
                       const TilePlan &plan, int E, bool packed, DevTensor<T> &d)
{
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
    const int b0 = bits_for(dims[m]), b1 = bits_for(dims[m1]), b2 = bits_for(dims[m2]);
    if (b0 + b1 + b2 > 64) fail(CTC_E_UNSUP, "CCD++ keys need %d bits (> 64) for these dimensions", b0 + b1 + b2);
    const int rb = packed ? ccdpp_packed_rbits(dims) : 0;
    if (packed && (rb < 16 || sizeof(T) != 4))
        fail(CTC_E_UNSUP, "mixed-precision CCD++ packs an FP32 residual of at least 16 bits beside the %d key bits",
             b0 + b1 + b2);
    d.ks.s_row = (uint32_t)(b1 + b2 + rb);
    d.ks.s_q1 = (uint32_t)(b2 + rb);
    d.ks.s_q2 = (uint32_t)rb;
    d.ks.rbits = (uint32_t)rb;
    d.ks.m_q1 = (b1 == 64) ? ~0ull : ((1ull << b1) - 1);
    d.ks.m_q2 = (b2 == 64) ? ~0ull : ((1ull << b2) - 1);
    int eshift = 0;
    while ((1 << eshift) < E) ++eshift;
    if ((1 << eshift) != E) fail(CTC_E_ARG, "CCD++ lanes per tile must be a power of two");
    const uint64_t S = 32ull * (uint64_t)E;
    const uint64_t ntiles = plan.ntiles();
    const uint64_t nslots = ntiles * S;
    if (nslots >= 0xfffffff0ull) fail(CTC_E_UNSUP, "CCD++: more than 2^32 slot entries");
    d.keys.alloc(nslots);
    d.x.alloc(nslots);
    dev_fill_slots<T>(ctx, src.rec.p, sizeof(T) == 8 ? src.v64.p : nullptr, perm, m, d.tiles.p, nslots, eshift,
                      d.ks.s_row, d.ks.s_q1, d.ks.s_q2, d.keys.p, d.x.p);
    // warp tasks: a light tile, or up to kCcdppGroup consecutive pieces of a
    // long row; the long-row table becomes {row, first group, groups, 0}
    std::vector<int32_t> tasks;
    std::vector<uint32_t> hv;
    tasks.reserve((size_t)ntiles * 4);
    uint32_t gslot = 0;
    for (uint32_t tt = 0; tt < (uint32_t)ntiles;) {
        const int32_t h = plan.tiles[4 * tt + 2];
        if (h < 0) {
            tasks.insert(tasks.end(), {(int32_t)tt, plan.tiles[4 * tt + 1], -1, 0});
            ++tt;
            continue;
        }
        const uint32_t np = plan.heavy_rows[4 * h + 2];
        const uint32_t ng = (np + k::kCcdppGroup - 1) / k::kCcdppGroup;
        hv.insert(hv.end(), {plan.heavy_rows[4 * h], gslot, ng, 0u});
        for (uint32_t g = 0; g < ng; ++g)
            tasks.insert(tasks.end(), {(int32_t)(tt + g * k::kCcdppGroup),
                                       (int32_t)std::min<uint32_t>(k::kCcdppGroup, np - g * k::kCcdppGroup), h,
                                       (int32_t)gslot++});
        tt += np;
    }
    d.ntasks = (uint32_t)(tasks.size() / 4);
    d.tasks.upload(reinterpret_cast<const int4 *>(tasks.data()), d.ntasks, ctx->stream);
    d.heavy.upload(reinterpret_cast<const uint4 *>(hv.data()), hv.size() / 4, ctx->stream);
    d.n = src.n;
    d.nslots = (uint32_t)nslots;
    if (!packed) {
        d.res.alloc(nslots);
        CK(cudaMemsetAsync(d.res.p, 0, nslots * sizeof(T), ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
}

// nonzeros per lane of the CCD++ pass for a tile length
static int ccdpp_lanes(int tile_len)
{
    return tile_len <= 128 ? 4 : (tile_len <= 256 ? 8 : 16);
}

// Order, size and dimension checks; the staging pass that reads the
// indices (stage_tensor with check dims) checks their range.
static void check_shape(const ctc_tensor *t, const uint64_t *dims, const char *what)
{
    if (!t) fail(CTC_E_ARG, "%s: null tensor", what);
    if (t->nmodes != 3) fail(CTC_E_UNSUP, "%s: only order-3 tensors are supported (got %d)", what, t->nmodes);
    if (t->nnz == 0) fail(CTC_E_ARG, "%s: empty tensor", what);
    if (t->nnz >= 0xfffffff0ull) fail(CTC_E_UNSUP, "%s: more than 2^32 nonzeros", what);
    for (int m = 0; m < 3; ++m)
        if (dims[m] == 0 || dims[m] >= 0xfffffff0ull)
            fail(CTC_E_UNSUP, "%s: bad dimension %llu", what, (unsigned long long)dims[m]);
}

static void validate_tensor(const ctc_tensor *t, const uint64_t *dims, const char *what)
{
    check_shape(t, dims, what);
    std::atomic<int> bad{0};
    par_for(t->nnz, [&](uint64_t b, uint64_t e) {
        for (int m = 0; m < 3; ++m) {
            const uint64_t *ind = t->ind[m].data();
            for (uint64_t i = b; i < e; ++i)
                if (ind[i] == 0 || ind[i] > dims[m]) {
                    bad = 1;
                    return;
                }
        }
    });
    if (bad) fail(CTC_E_ARG, "%s: indices must be 1-based and within the model dimensions", what);
}

// check: when given, every index is checked against these dimensions in
// the same pass (failing with `what` in the message before any kernel
// reads the records).
template <typename T>
static void stage_tensor(ctc_ctx *ctx, const ctc_tensor *t, bool trunc, DevTensor<T> &d,
                         const uint64_t *check = nullptr, const char *what = "tensor")
{
    const uint64_t n = t->nnz;
    d.n = (uint32_t)n;
    d.rec.alloc(n);
    const uint64_t *i0 = t->ind[0].data(), *i1 = t->ind[1].data(), *i2 = t->ind[2].data();
    const double *vals = t->vals.data();
    const uint64_t c0 = check ? check[0] : ~0ull, c1 = check ? check[1] : ~0ull, c2 = check ? check[2] : ~0ull;
    std::atomic<int> bad{0};
    upload_filled(ctx, d.rec.p, n, [&](uint64_t b, uint64_t e, uint4 *h) {
        bool oob = false;
        for (uint64_t i = b; i < e; ++i) {
            double v = vals[i];
            if (trunc) v = ctc_value_through_idx(v);
            const float vf = (float)v;
            uint32_t bits;
            memcpy(&bits, &vf, 4);
            const uint64_t a0 = i0[i] - 1, a1 = i1[i] - 1, a2 = i2[i] - 1;
            oob |= (a0 >= c0) | (a1 >= c1) | (a2 >= c2);
            stream_store16(h + (i - b), (uint32_t)a0, (uint32_t)a1, (uint32_t)a2, bits);
        }
        stream_fence();
        if (oob) bad = 1;
    });
    if (check) {
        CK(cudaStreamSynchronize(ctx->stream));
        if (bad) fail(CTC_E_ARG, "%s: indices must be 1-based and within the model dimensions", what);
    }
    if (std::is_same<T, double>::value) {
        d.v64.alloc(n);
        upload_filled(ctx, d.v64.p, n, [&](uint64_t b, uint64_t e, double *h) {
            for (uint64_t i = b; i < e; ++i) h[i - b] = trunc ? ctc_value_through_idx(vals[i]) : vals[i];
        });
    }
    CK(cudaStreamSynchronize(ctx->stream));
}

template <typename T>
static void upload_plan(ctc_ctx *ctx, const TilePlan &p, int mode, DevTensor<T> &d);

// host planner over the copy's index array (the compat ALS / CCD path)
template <typename T>
static TilePlan stage_plan(ctc_ctx *ctx, const ctc_tensor *t, int mode, uint32_t tile_len, DevTensor<T> &d)
{
    const uint64_t n = t->nnz;
    if (n >= 0x7fffffffull) fail(CTC_E_UNSUP, "tile plans index at most 2^31 - 1 nonzeros");
    bool unsorted = false;
    TilePlan p = plan_tiles_chunked(t->ind[mode].data(), n, tile_len, &unsorted);
    if (unsorted) fail(CTC_E_ARG, "training tensor %d is not sorted for mode %d", mode + 1, mode + 1);
    upload_plan(ctx, p, mode, d);
    return p;
}

// the plan's tiles, long rows and piece list on the device
template <typename T>
static void upload_plan(ctc_ctx *ctx, const TilePlan &p, int mode, DevTensor<T> &d)
{
    d.mode = mode;
    d.ntiles = p.ntiles();
    d.nheavy = p.nheavy();
    d.tiles.upload(reinterpret_cast<const int4 *>(p.tiles.data()), p.ntiles(), ctx->stream);
    d.heavy.upload(reinterpret_cast<const uint4 *>(p.heavy_rows.data()), p.nheavy(), ctx->stream);
    // the tiles that are pieces of long rows, in order: each long row's
    // pieces are the consecutive tiles first .. first + count - 1, and the
    // long rows are numbered in tile order
    std::vector<uint32_t> pieces;
    size_t np = 0;
    for (uint32_t h = 0; h < p.nheavy(); ++h) np += p.heavy_rows[4 * h + 2];
    pieces.resize(np);
    np = 0;
    for (uint32_t h = 0; h < p.nheavy(); ++h)
        for (uint32_t q = 0; q < p.heavy_rows[4 * h + 2]; ++q) pieces[np++] = p.heavy_rows[4 * h + 1] + q;
    d.npieces = (uint32_t)pieces.size();
    d.pieces.upload(pieces.data(), pieces.size(), ctx->stream);
    CK(cudaStreamSynchronize(ctx->stream));
}

template <typename T>
static void stage_weights(ctc_ctx *ctx, const ctc_tensor *t, int mode, int kernel, DevTensor<T> &d)
{
    ctc_ciss *cp = nullptr;
    if (ctc_ciss_build(t, mode + 1, 32, &cp) != CTC_OK) fail(CTC_E_ARG, "%s", ctc_last_error());
    std::unique_ptr<ctc_ciss, int (*)(ctc_ciss *)> guard(cp, ctc_ciss_free);
    std::vector<double> w;
    compat_weights(*cp, kernel, w);
    std::vector<T> wt(w.begin(), w.end());
    d.w.upload(wt.data(), wt.size(), ctx->stream);
    d.has_w = true;
    CK(cudaStreamSynchronize(ctx->stream));
}

// Device-resident state of one run: factors (row-major, or column-major
// for CCD++), best-epoch copy, CCD++ residuals in the staged records,
// scratch, the SGD step on the device, and the captured epoch graph.
struct SessionBase {
    virtual ~SessionBase() = default;
    virtual void set_model(const ctc_model *m) = 0;
    virtual void get_model(ctc_model *m, bool best) = 0;
    virtual void epochs(int n) = 0;
    virtual void evaluate(ctc_epoch_stats *st) = 0;
    virtual void set_lr(double lr) = 0;
    virtual void save_best() = 0;
    virtual uint64_t nonspd() = 0;
    virtual void set_params(const ctc_params &p) = 0;
    virtual void probe_wait(uint64_t limit_ns) = 0;
    // squared error per batch instance over instance-aligned chunks of the
    // mode-1 training copy (which = 0) or the test tensor (which = 1)
    virtual void seg_sse(int which, const uint4 *chunks, uint32_t nchunks, const uint32_t *first, int ninst,
                         double *partial, double *out) = 0;
};

}  // namespace ctc

// ---------------------------------------------------------------------
// dataset: staged tensors for one algorithm / precision + its session
// ---------------------------------------------------------------------
struct ctc_dataset {
    ctc_ctx *ctx = nullptr;
    ctc_params p{};
    uint64_t dims[3] = {0, 0, 0};
    uint64_t nnz_train = 0;
    bool has_val = false, has_test = false;
    struct Base {
        virtual ~Base() = default;
    };
    std::unique_ptr<Base> impl;
    std::unique_ptr<ctc::SessionBase> session;
    int session_rank = 0;
};

namespace ctc {

template <typename T>
struct DatasetImpl : ctc_dataset::Base {
    DevTensor<T> copy[3];
    DevTensor<T> val, test;
    std::vector<uint32_t> rowcnt[3];  // SGD: nonzeros per row of each mode
};

static int default_tile(int alg)
{
    switch (alg) {
    case CTC_ALG_ALS: return 512;
    case CTC_ALG_SGD: return 256;
    default: return 256;
    }
}

// The three mode copies of ALS / CCD / CCD++ staged through the device:
// the records of train[0] (mode-1 order) are uploaded once; copy m is the
// caller's train[m] uploaded as records when given, else the stable
// (mode m, mode m+1) order of train[0] sorted on the device (the order
// ctc_tensor_sort gives).  CCD++ copies are further sorted by the full key
// (row, larger other mode, smaller other mode).  The rows' run lengths
// come back to the host for the tile plan (plan_tiles_runs: the plan of the
// host planner), and the CCD++ slots or the record copy are gathered on
// the device.
// CCD++ pass: quarters of its tasks taken on a fixed stride before the rest
// are claimed (its grid is exactly the resident blocks).  On the 100M
// tensor, tile 256, CCD++ outer iteration: 93.1 ms with every task claimed,
// 91.0 ms with half on the stride, 93.1 ms with three quarters, 100.6 ms
// with all but the remainder.
constexpr uint32_t kCcdppStrideQuarters = 2;
// CCD++ later sweeps staging one column of at least this many bytes while
// gathering the other through L1 run as one 1024-thread block per SM
constexpr size_t kCcdppBigStaged = 32 * 1024;
// Mixed ALS: the row length above which a row takes tiles of its own and a
// tensor-core Gram, below the tile length that packs the light rows (on the
// 100M rank-32 tensor, tile 1024: 21.1 ms per iteration with the tile
// length as the threshold, 20.2 / 19.7 / 19.7 ms with 512 / 256 / 128, test
// RMSE after 10 iterations 0.2934-0.2939 against 0.2940 in FP32; every row
// above R/2 nonzeros moved the factors 0.25 from the oracle on a 2M sample)
constexpr uint32_t kMixedHeavyMin = 256;
template <typename T>
static void stage_copies_dev(ctc_ctx *ctx, const ctc_params &p, uint32_t tl, const ctc_tensor *const train[3],
                             const uint64_t *dims, bool trunc, DatasetImpl<T> &impl)
{
    const uint64_t n = train[0]->nnz;
    if (n >= 0x7fffffffull) fail(CTC_E_UNSUP, "tile plans index at most 2^31 - 1 nonzeros");
    const bool ccdpp = p.alg == CTC_ALG_CCDPP;
    DevTensor<T> base;
    {
        TracePhase tp("records + upload");
        stage_tensor<T>(ctx, train[0], trunc, base, dims, "training tensor");
    }
    // copy 1 last: it can take over the base records (ALS / CCD)
    for (int m : {1, 2, 0}) {
        const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
        DevTensor<T> given;
        const DevTensor<T> *src = &base;
        DevBuf<uint32_t> perm;
        bool in_order = m == 0;  // src already sorted for mode m (copy 1, or the caller's copy)
        if (m > 0 && train[m]) {
            TracePhase tp("records + upload");
            stage_tensor<T>(ctx, train[m], trunc, given, dims, "training tensor");
            src = &given;
            in_order = true;
        }
        if (in_order && dev_unsorted(ctx, src->rec.p, (uint32_t)n, m))
            fail(CTC_E_ARG, "training tensor %d is not sorted for mode %d", m + 1, m + 1);
        if (ccdpp) {
            // CCD++ slots: within each row, the larger of the other two modes
            // in increasing order (then the smaller), so that the gathers from
            // the column that cannot be staged in shared memory sweep it
            // instead of jumping; the full key makes the order unique for
            // distinct coordinates, whichever copy it starts from
            TracePhase tp("device sort");
            const int kb = bits_for(dims[0]) + bits_for(dims[1]) + bits_for(dims[2]);
            if (kb > 64) fail(CTC_E_UNSUP, "CCD++ keys need %d bits (> 64) for these dimensions", kb);
            const int big = dims[m2] > dims[m1] ? m2 : m1, small = big == m1 ? m2 : m1;
            const int k[3] = {m, big, small};
            const int b[3] = {bits_for(dims[m]), bits_for(dims[big]), bits_for(dims[small])};
            perm.alloc(n);
            dev_sort_order(ctx, src->rec.p, (uint32_t)n, k, b, perm.p);
        } else if (!in_order) {
            TracePhase tp("device sort");
            const int k[3] = {m, m1, m1};
            const int b[3] = {bits_for(dims[m]), bits_for(dims[m1]), 0};
            perm.alloc(n);
            dev_sort_order(ctx, base.rec.p, (uint32_t)n, k, b, perm.p);
        }
        const uint32_t *pp = perm.p;
        DevTensor<T> &d = impl.copy[m];
        TilePlan plan;
        {
            TracePhase tp("row runs + tile plan");
            std::vector<uint32_t> rows, counts;
            if (dev_row_runs(ctx, src->rec.p, pp, (uint32_t)n, m, rows, counts))
                fail(CTC_E_ARG, "training tensor %d is not sorted for mode %d", m + 1, m + 1);
            // mixed ALS: rows longer than kMixedHeavyMin get tiles of their
            // own, whose Grams the tensor cores form
            const bool tc_rows = p.alg == CTC_ALG_ALS && p.precision == CTC_PREC_MIXED &&
                                 (p.rank == 32 || p.rank == 64) && p.compat == 0;
            plan = plan_tiles_runs(rows.data(), counts.data(), rows.size(), tl, tc_rows ? kMixedHeavyMin : 0u);
            upload_plan(ctx, plan, m, d);
            d.nrows = rows.size();  // one run per row: the copy is sorted by its mode
        }
        if (ccdpp) {
            TracePhase tp("CCD++ slots");
            stage_keys<T>(ctx, *src, pp, m, dims, plan, (int)(tl / 32), p.precision == CTC_PREC_MIXED, d);
            continue;
        }
        TracePhase tp("record copy");
        d.n = (uint32_t)n;
        if (pp) {
            d.rec.alloc(n);
            if (sizeof(T) == 8) d.v64.alloc(n);
            dev_gather_records(ctx, base.rec.p, sizeof(T) == 8 ? base.v64.p : nullptr, pp, (uint32_t)n, d.rec.p,
                               d.v64.p);
            CK(cudaStreamSynchronize(ctx->stream));
        } else {
            DevTensor<T> &from = (m == 0) ? base : given;
            d.rec.swap(from.rec);
            d.v64.swap(from.v64);
        }
    }
}

template <typename T>
static void build_dataset(ctc_dataset *ds, const ctc_tensor *const train[3], const ctc_tensor *val,
                          const ctc_tensor *test)
{
    auto impl = std::make_unique<DatasetImpl<T>>();
    ctc_ctx *ctx = ds->ctx;
    const ctc_params &p = ds->p;
    const bool trunc = p.compat != 0;
    uint32_t tl = (uint32_t)(p.tile_len > 0 ? p.tile_len : default_tile(p.alg));
    // CCD++: tiles fill slots of 32*E entries
    if (p.alg == CTC_ALG_CCDPP) tl = 32u * (uint32_t)ccdpp_lanes((int)tl);
    for (int m = 0; m < 3; ++m)
        if (train[m]) {
            check_shape(train[m], ds->dims, "training tensor");
            if (train[m]->nnz != train[0]->nnz) fail(CTC_E_ARG, "training copies differ in size");
        }
    if (p.alg == CTC_ALG_SGD) {
        {
            TracePhase tp("records + upload");
            stage_tensor<T>(ctx, train[0], trunc, impl->copy[0], ds->dims, "training tensor");
        }
        // SGD tiles are plain chunks of the mode-1 order (sgpu/sgd.cu:32-34)
        impl->copy[0].mode = 0;
        impl->copy[0].ntiles = (uint32_t)((impl->copy[0].n + tl - 1) / tl);
        TracePhase tp("SGD row counts");
        for (int m = 0; m < 3; ++m)
            dev_row_counts(ctx, impl->copy[0].rec.p, impl->copy[0].n, m, (uint32_t)ds->dims[m], impl->rowcnt[m]);
    } else if (trunc && (p.alg == CTC_ALG_ALS || p.alg == CTC_ALG_CCD)) {
        // the reference's lane multiplicities come from the host CISS of
        // every sorted copy, so these copies are sorted and planned on the host
        std::unique_ptr<ctc_tensor> own[3];
        for (int m = 0; m < 3; ++m) {
            const ctc_tensor *t = train[m];
            if (!t) {
                own[m].reset(new ctc_tensor(*train[0]));
                if (ctc_tensor_sort(own[m].get(), m) != CTC_OK) fail(CTC_E_ARG, "%s", ctc_last_error());
                t = own[m].get();
            }
            stage_tensor<T>(ctx, t, trunc, impl->copy[m], ds->dims, "training tensor");
            stage_plan<T>(ctx, t, m, tl, impl->copy[m]);
            stage_weights<T>(ctx, t, m, p.alg == CTC_ALG_CCD ? 1 : 0, impl->copy[m]);
        }
    } else {
        stage_copies_dev<T>(ctx, p, tl, train, ds->dims, trunc, *impl);
    }
    if (val) {
        TracePhase tp("validation tensor");
        check_shape(val, ds->dims, "validation tensor");
        stage_tensor<T>(ctx, val, false, impl->val, ds->dims, "validation tensor");
    }
    if (test) {
        TracePhase tp("test tensor");
        check_shape(test, ds->dims, "test tensor");
        stage_tensor<T>(ctx, test, false, impl->test, ds->dims, "test tensor");
    }
    ds->impl = std::move(impl);
}

template <typename T, int R>
struct Session : SessionBase {
    ctc_ctx *ctx;
    ctc_dataset *ds;
    DatasetImpl<T> *D;
    ctc_params p;
    uint32_t dims[3];
    bool colmajor;
    uint32_t tile_len;
    DevBuf<T> U[3], Ubest[3], Urow[3], slot, slot2, lr_dev;
    DevBuf<k::Pack3<T>> pk[3];  // CCD++ per-column {cur, prev, old}
    DevBuf<k::Pack2<T>> pk2[3];  // ... and {old, prev} (+2: staged copies read whole 16-byte words)
    DevBuf<unsigned int> hcnt[3];  // CCD++ pieces arrived per heavy row (reset by the finaliser)
    // {next, done} task claim counters of the kernels that claim their warp
    // tasks (k::TaskClaim); every launch leaves them at zero
    DevBuf<unsigned int> claim;
    // mixed-precision ALS at rank 64: BF16 copies of the factors feed the
    // tensor-core Gram of long-row pieces; err flags an expired bounded wait
    bool tc = false;
    DevBuf<__nv_bfloat16> Ubf[3];
    DevBuf<int> dev_err;
    DevBuf<unsigned long long> nonspd_dev;
    cudaGraphExec_t graph = nullptr;
    bool model_set = false;

    Session(ctc_dataset *d) : ctx(d->ctx), ds(d), p(d->p)
    {
        D = static_cast<DatasetImpl<T> *>(d->impl.get());
        for (int m = 0; m < 3; ++m) dims[m] = (uint32_t)d->dims[m];
        colmajor = p.alg == CTC_ALG_CCDPP;
        tile_len = (uint32_t)(p.tile_len > 0 ? p.tile_len : default_tile(p.alg));
        nonspd_dev.alloc(1);
        lr_dev.alloc(1);
        dev_err.alloc(1);
        CK(cudaMemsetAsync(dev_err.p, 0, sizeof(int), ctx->stream));
        for (int m = 0; m < 3; ++m) {
            const size_t sz = (size_t)dims[m] * R;
            // (+4: the CCD++ column staging copies whole 16-byte words and
            // may read up to 15 bytes past the last column)
            U[m].alloc(sz + 4);
            CK(cudaMemsetAsync(U[m].p, 0, (sz + 4) * sizeof(T), ctx->stream));
            Ubest[m].alloc(sz);
            if (colmajor) {
                Urow[m].alloc(sz);
                pk[m].alloc(dims[m]);
                pk2[m].alloc(dims[m] + 2);
                CK(cudaMemsetAsync(pk2[m].p, 0, pk2[m].n * sizeof(k::Pack2<T>), ctx->stream));
                hcnt[m].alloc(D->copy[m].nheavy);
                CK(cudaMemsetAsync(hcnt[m].p, 0, hcnt[m].n * sizeof(unsigned int), ctx->stream));
            }
        }
        claim.alloc(2);
        CK(cudaMemsetAsync(claim.p, 0, 2 * sizeof(unsigned int), ctx->stream));
        // scratch sized once so an epoch can be captured as a graph
        size_t need = 1;
        for (int m = 0; m < 3; ++m) {
            const DevTensor<T> &c = D->copy[m];
            if (!c.nheavy && p.alg != CTC_ALG_CCDPP) continue;
            if (p.alg == CTC_ALG_ALS) need = std::max<size_t>(need, (size_t)c.ntiles * (R * R + R));
            else if (p.alg == CTC_ALG_CCD) need = std::max<size_t>(need, (size_t)c.ntiles * 2 * R);
            else if (p.alg == CTC_ALG_CCDPP) need = std::max<size_t>(need, (size_t)c.ntiles);
        }
        slot.alloc(need);
        if (p.alg == CTC_ALG_CCDPP) slot2.alloc(need);
        if (p.alg == CTC_ALG_CCDPP) {
            set_ccdpp_smem<4>();
            set_ccdpp_smem<8>();
            set_ccdpp_smem<16>();
        }
        tc = p.alg == CTC_ALG_ALS && p.precision == CTC_PREC_MIXED && (R == 64 || R == 32) &&
             std::is_same<T, float>::value;
        if constexpr (R == 64 || R == 32) {
            if (tc) {
                for (int m = 0; m < 3; ++m) Ubf[m].alloc((size_t)dims[m] * R);
                CK(cudaFuncSetAttribute(tc::k_als_gram_tc<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tc::gram_smem_bytes<R>()));
            }
        }
        if (p.alg == CTC_ALG_SGD && std::is_same<T, float>::value) {
            // bulk row reductions stage 2 x 3 rows per group in shared memory
            set_sgd_smem<1>();
            set_sgd_smem<2>();
            set_sgd_smem<4>();
        }
        if (p.alg == CTC_ALG_ALS) {
            // both kernels park one warp's systems per warp of a 4-warp block
            const int smem_tile = (int)(4 * k::AlsBatch<T, R>::warp_doubles * sizeof(double));
            CK(cudaFuncSetAttribute(k::k_als_tile<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_tile));
            CK(cudaFuncSetAttribute(k::k_als_fix<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_tile));
        }
        CK(cudaStreamSynchronize(ctx->stream));
    }

    ~Session() override
    {
        if (graph) cudaGraphExecDestroy(graph);
    }

    // run-time parameters (lambda, inner, lr, schedule, order ...); the
    // staged layout (alg, precision, compat, tile length) stays
    template <int E>
    void set_ccdpp_smem()
    {
        // the largest budget ctc_params.smem_budget may ask for
        const int smem = ccdpp_smem_max();
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, true, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, false, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, true, E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem));
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, false, E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem));
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, true, E, false, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, true, E, true, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, false, E, false, false, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        CK(cudaFuncSetAttribute(k::k_ccdpp_pass<T, false, E, true, false, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    }

    // shared memory per block of a CCD++ pass for staged factor columns: two
    // 512-thread blocks per SM share the 228 KiB
    size_t ccdpp_budget() const
    {
        if (p.smem_budget < 0) return 0;
        const size_t b = p.smem_budget > 0 ? (size_t)p.smem_budget : (size_t)110 * 1024;
        return std::min<size_t>(b, (size_t)ccdpp_smem_max());
    }

    // opt-in dynamic shared memory of a block, less room for the pass's
    // static mbarrier (and a margin)
    static int ccdpp_smem_max()
    {
        int dev = 0, optin = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        return optin - 1024;
    }

    void set_params(const ctc_params &np) override
    {
        p = np;
        if (graph) {
            cudaGraphExecDestroy(graph);
            graph = nullptr;
        }
        damp_ready = false;
    }

    // Hogwild step scale per row: min(1, K / (G * nnz(row) / nnz)), G the
    // groups in flight (see ctc_params.sgd_conflicts)
    DevBuf<float> damp[3];
    bool damp_ready = false, damp_on = false;
    // block-merged hot rows (sgd_atomic 3): slot codes per nonzero of copy 0
    // and the rows of the slots, mode-major
    DevBuf<uint32_t> hot_codes, hot_rows;
    bool hot_ready = false;
    bool eager_done = false;  // the session's first epoch ran without a graph
    void prepare_hot()
    {
        hot_ready = true;
        const DevTensor<T> &c = D->copy[0];
        std::vector<uint32_t> rows(3 * k::kSgdHot, 0u);
        DevBuf<uint16_t> map[3];
        for (int m = 0; m < 3; ++m) {
            // the kSgdHot most frequent rows (ties: lower row first)
            const auto &cnt = D->rowcnt[m];
            std::vector<uint32_t> order(dims[m]);
            std::iota(order.begin(), order.end(), 0u);
            const size_t h = std::min<size_t>(k::kSgdHot, order.size());
            auto count = [&](uint32_t r) -> uint32_t { return r < cnt.size() ? cnt[r] : 0u; };
            std::partial_sort(order.begin(), order.begin() + h, order.end(), [&](uint32_t a, uint32_t b) {
                return count(a) != count(b) ? count(a) > count(b) : a < b;
            });
            std::vector<uint16_t> mp(dims[m], (uint16_t)k::kSgdCold);
            for (size_t s = 0; s < h; ++s) {
                mp[order[s]] = (uint16_t)s;
                rows[m * k::kSgdHot + s] = order[s];
            }
            map[m].upload(mp.data(), mp.size(), ctx->stream);
        }
        hot_rows.upload(rows.data(), rows.size(), ctx->stream);
        hot_codes.alloc(c.n);
        LAUNCH(ctx, k::k_sgd_hot_codes, grid_for(c.n, 256, kSMs * 16), 256, 0, (const uint4 *)c.rec.p, c.n,
               (const uint16_t *)map[0].p, (const uint16_t *)map[1].p, (const uint16_t *)map[2].p, hot_codes.p);
        CK(cudaStreamSynchronize(ctx->stream));
    }
    unsigned sgd_grid(int gpb) const
    {
        const unsigned cap = p.sgd_groups > 0 ? (unsigned)std::max(1, p.sgd_groups / gpb) : kSMs * 8;
        return grid_for(D->copy[0].ntiles, gpb, cap);
    }
    void prepare_damping(int gpb)
    {
        damp_ready = true;
        damp_on = false;
        if (p.sgd_order == CTC_SGD_SEQUENTIAL || p.sgd_conflicts < 0) return;
        const double K = p.sgd_conflicts > 0 ? (double)p.sgd_conflicts : 128.0;
        const double G = std::min<double>((double)sgd_grid(gpb) * gpb, (double)D->copy[0].ntiles);
        const double n = (double)D->copy[0].n;
        for (int m = 0; m < 3; ++m) {
            std::vector<float> h(dims[m], 1.0f);
            const auto &cnt = D->rowcnt[m];
            for (size_t r = 0; r < cnt.size() && r < h.size(); ++r) {
                const double conc = G * (double)cnt[r] / n;
                if (conc > K) {
                    h[r] = (float)(K / conc);
                    damp_on = true;
                }
            }
            damp[m].upload(h.data(), h.size(), ctx->stream);
        }
        CK(cudaStreamSynchronize(ctx->stream));
    }

    // rows x cols row-major -> cols x rows row-major on the device
    void transpose(const T *in, uint64_t rows, uint64_t cols, T *out)
    {
        const dim3 grid((unsigned)((rows + 31) / 32), (unsigned)std::min<uint64_t>((cols + 31) / 32, 65535));
        LAUNCH(ctx, k::k_transpose<T>, grid, dim3(32, 8), 0, in, rows, cols, out);
    }

    // The factors stream through the pinned buffer as rows of T (converted
    // on the host threads); CCD++'s column-major factors are transposed on
    // the device.
    void set_model(const ctc_model *mdl) override
    {
        DevBuf<T> rowmajor;
        for (int m = 0; m < 3; ++m) {
            const uint64_t d = dims[m], n = d * R;
            const double *src = mdl->U[m].data();
            T *dst = U[m].p;
            if (colmajor) {
                rowmajor.ensure(n);
                dst = rowmajor.p;
            }
            upload_filled(ctx, dst, n, [&](uint64_t b, uint64_t e, T *h) {
                for (uint64_t i = b; i < e; ++i) h[i - b] = (T)src[i];
            });
            if (colmajor) transpose(rowmajor.p, d, R, U[m].p);
            CK(cudaMemcpyAsync(Ubest[m].p, U[m].p, n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
        CK(cudaMemsetAsync(nonspd_dev.p, 0, sizeof(unsigned long long), ctx->stream));
        CK(cudaMemsetAsync(dev_err.p, 0, sizeof(int), ctx->stream));
        set_lr(p.lr * (p.lr_scale > 0 ? p.lr_scale : 1.0));
        if (colmajor) ccdpp_init();
        if (tc)
            for (int m = 0; m < 3; ++m) refresh_bf16(m);
        CK(cudaStreamSynchronize(ctx->stream));
        model_set = true;
    }

    void get_model(ctc_model *mdl, bool best) override
    {
        DevBuf<T> *src = best ? Ubest : U;
        DevBuf<T> rowmajor;
        for (int m = 0; m < 3; ++m) {
            const uint64_t d = dims[m], n = d * R;
            const T *from = src[m].p;
            if (colmajor) {
                rowmajor.ensure(n);
                transpose(src[m].p, R, d, rowmajor.p);
                from = rowmajor.p;
            }
            double *dst = mdl->U[m].data();
            download_drained(ctx, from, n, [&](uint64_t b, uint64_t e, const T *h) {
                for (uint64_t i = b; i < e; ++i) dst[i] = (double)h[i - b];
            });
        }
    }

    void set_lr(double lr) override
    {
        T v = (T)lr;
        CK(cudaMemcpyAsync(lr_dev.p, &v, sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }

    void save_best() override
    {
        for (int m = 0; m < 3; ++m)
            CK(cudaMemcpyAsync(Ubest[m].p, U[m].p, (size_t)dims[m] * R * sizeof(T), cudaMemcpyDeviceToDevice,
                               ctx->stream));
    }

    uint64_t nonspd() override
    {
        unsigned long long v = 0;
        CK(cudaMemcpyAsync(&v, nonspd_dev.p, sizeof(v), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        return v;
    }

    // ---- reductions into ctx->scalars[s]
    void sse_into(const DevTensor<T> &t, const T *const Urm[3], int s)
    {
        const unsigned g = grid_for(t.n, 256, kMaxPartials);
        LAUNCH(ctx, k::k_sse<T, R>, g, 256, 0, (const uint4 *)t.rec.p, (const double *)t.v64.p, t.n,
               Urm[0], Urm[1], Urm[2], ctx->partial.p);
        LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p + s);
    }
    void sumsq_into(const T *x, uint64_t n, int s)
    {
        const unsigned g = grid_for(n, 256, kMaxPartials);
        LAUNCH(ctx, k::k_sumsq<T>, g, 256, 0, x, n, ctx->partial.p);
        LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p + s);
    }

    // ---- epochs
    void als_epoch()
    {
        const size_t smem = 4 * k::AlsBatch<T, R>::warp_doubles * sizeof(double);
        for (int q = 0; q < 3; ++q) {
            const int m = (p.mode_start + q) % 3;
            const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
            DevTensor<T> &c = D->copy[m];
            CK(cudaMemsetAsync(U[m].p, 0, (size_t)dims[m] * R * sizeof(T), ctx->stream));
            LAUNCH(ctx, k::k_als_tile<T, R>, grid_for(c.ntiles, 4, kSMs * 16), 128,
                   4 * k::AlsBatch<T, R>::warp_doubles * sizeof(double), (const int4 *)c.tiles.p,
                   c.ntiles, (const uint4 *)c.rec.p, (const double *)c.v64.p,
                   (const T *)(c.has_w ? c.w.p : nullptr), m, U[m].p, (const T *)U[m1].p, (const T *)U[m2].p,
                   (T)p.lambda, slot.p, nonspd_dev.p, tc ? 1 : 0, k::TaskClaim{claim.p, 0u});
            if (tc && c.npieces) als_gram_tc(c, m);
            if (c.nheavy) {
                // pieces summed element-parallel first; the solve reads one slot per row
                LAUNCH(ctx, k::k_als_sum_pieces<T, R>,
                       grid_for((uint64_t)c.nheavy * (R * R + R), 256, kSMs * 16), 256, 0,
                       (const uint4 *)c.heavy.p, c.nheavy, slot.p);
                LAUNCH(ctx, k::k_als_fix<T, R>, grid_for(c.nheavy, 4, kSMs * 16), 128, smem,
                       (const uint4 *)c.heavy.p, c.nheavy, (const T *)slot.p, U[m].p, (T)p.lambda, nonspd_dev.p, 1);
            }
            if (tc) refresh_bf16(m);
        }
    }

    void refresh_bf16(int m)
    {
        if constexpr (std::is_same<T, float>::value)
            LAUNCH(ctx, tc::k_to_bf16, grid_for((uint64_t)dims[m] * R, 256, kSMs * 8), 256, 0, (const float *)U[m].p,
                   Ubf[m].p, (uint64_t)dims[m] * R);
    }

    void als_gram_tc(DevTensor<T> &c, int m)
    {
        if constexpr (std::is_same<T, float>::value && (R == 64 || R == 32)) {
            const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
            const unsigned g = std::min<unsigned>(c.npieces, (R == 64 ? 2 : 4) * kSMs);
            LAUNCH(ctx, tc::k_als_gram_tc<R>, g, tc::kThreads, tc::gram_smem_bytes<R>(), (const int4 *)c.tiles.p,
                   (const uint32_t *)c.pieces.p, c.npieces, (const uint4 *)c.rec.p, m,
                   (const __nv_bfloat16 *)Ubf[m1].p, (const __nv_bfloat16 *)Ubf[m2].p, (float *)slot.p, dev_err.p);
        }
    }

    // device-side error flag: 1 = the tensor-core Gram's bounded wait for
    // its MMAs expired, 2 = a CCD++ pass's bounded wait for its staged
    // columns expired (the pass left the column unfinished), 3 = the
    // bounded-wait self-test expired (ctc_dataset_probe_wait).  An error is
    // reported once: the flag is cleared when it is read here, and when a
    // model is staged.
    void check_errors()
    {
        int e = 0;
        CK(cudaMemcpyAsync(&e, dev_err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (!e) return;
        CK(cudaMemsetAsync(dev_err.p, 0, sizeof(int), ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (e == 1) fail(CTC_E_TIMEOUT, "tensor-core Gram: a bounded wait for the MMAs expired");
        if (e == 3) fail(CTC_E_TIMEOUT, "bounded-wait self-test: the wait expired");
        fail(CTC_E_TIMEOUT, "CCD++ pass: a bounded wait for the staged factor columns expired");
    }

    void probe_wait(uint64_t limit_ns) override
    {
        LAUNCH(ctx, k::k_wait_probe, 1, 32, 0, dev_err.p, 3, limit_ns);
    }

    void ccd_epoch()
    {
        for (int q = 0; q < 3; ++q) {
            const int m = (p.mode_start + q) % 3;
            const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
            DevTensor<T> &c = D->copy[m];
            LAUNCH(ctx, k::k_ccdc_tile<T, R>, grid_for(c.ntiles, 4, kSMs * 16), 128, 0, (const int4 *)c.tiles.p,
                   c.ntiles, (const uint4 *)c.rec.p, (const double *)c.v64.p,
                   (const T *)(c.has_w ? c.w.p : nullptr), m, U[m].p, (const T *)U[m1].p, (const T *)U[m2].p,
                   (T)p.lambda, slot.p);
            if (c.nheavy)
                LAUNCH(ctx, k::k_ccdc_fix<T, R>, grid_for(c.nheavy, 4, kSMs * 16), 128, 0,
                       (const uint4 *)c.heavy.p, c.nheavy, (const T *)slot.p, U[m].p, (T)p.lambda);
        }
    }

    // 16-byte vectors per lane of the SGD kernel (1, 2 or 4): the lanes per
    // nonzero are R / (vector width * C), ctc_params.threads_per_row.  The
    // default is one vector per lane (R/4 lanes per FP32 nonzero), the
    // fastest setting measured at R = 32 on the 100M-nonzero Zipf tensor
    // (35 ms per epoch against 63 ms with two vectors and 79 ms with four).
    int sgd_vectors() const
    {
        constexpr int base = R / k::Vec<T>::n;
        if (p.sgd_order == CTC_SGD_SEQUENTIAL) return 1;
        int c = p.threads_per_row > 0 ? base / p.threads_per_row : 1;
        if (c >= 4 && base % 4 == 0) return 4;
        if (c >= 2 && base % 2 == 0) return 2;
        return 1;
    }
    // Hogwild threads per block: ctc_params.threads_per_block (the
    // reference GA's block-size gene, ga/sgd.cu:66-78), 256 when 0
    int sgd_block() const { return p.threads_per_block > 0 ? p.threads_per_block : 256; }
    int sgd_groups_per_block() const
    {
        return (sgd_block() / 32) * (32 / (R / k::Vec<T>::n / sgd_vectors()));
    }
    template <int C>
    void set_sgd_smem()
    {
        if constexpr ((R / k::Vec<T>::n) % C == 0 && R / k::Vec<T>::n / C <= 32) {
            // the largest block (512 threads) sets the opt-in
            const int gpb = 16 * (32 / (R / k::Vec<T>::n / C));
            const int smem = gpb * 2 * 3 * R * (int)sizeof(T);
            if (smem > 48 * 1024)
                CK(cudaFuncSetAttribute(k::k_sgd<T, R, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        }
    }

    void sgd_epoch()
    {
        switch (sgd_vectors()) {
        case 4: sgd_launch<4>(); break;
        case 2: sgd_launch<2>(); break;
        default: sgd_launch<1>(); break;
        }
    }

    template <int C>
    void sgd_launch()
    {
        DevTensor<T> &c = D->copy[0];
        const int gpb = sgd_groups_per_block();
        const bool seq = p.sgd_order == CTC_SGD_SEQUENTIAL;
        const unsigned g = seq ? 1 : sgd_grid(gpb);
        const float *d0 = damp_on ? damp[0].p : nullptr;
        const float *d1 = damp_on ? damp[1].p : nullptr;
        const float *d2 = damp_on ? damp[2].p : nullptr;
        // a prime stride that does not divide the tile count
        uint64_t stride = 1;
        if (!seq) {
            for (uint64_t pr : {1000003ull, 999983ull, 999979ull, 104729ull})
                if (c.ntiles % pr != 0) {
                    stride = pr % c.ntiles ? pr : 1;
                    break;
                }
        }
        if constexpr (std::is_same<T, float>::value && (R / 4) % C == 0 && R / 4 / C <= 32) {
            if (!seq && p.sgd_atomic == 3) {
                // block-merged hot rows: a block's groups step together
                const int blk = sgd_block();
                const int gpb_h = (blk / 32) * (32 / (R / 4 / C));
                LAUNCH(ctx, (k::k_sgd_hot<R, C>), sgd_grid(gpb_h), blk, 0, (const uint4 *)c.rec.p,
                       (const uint32_t *)hot_codes.p, c.n, tile_len, c.ntiles, U[0].p, U[1].p, U[2].p,
                       (const float *)lr_dev.p, (float)p.lambda, stride, d0, d1, d2, (const uint32_t *)hot_rows.p);
                return;
            }
        }
        // bulk row reductions: two staged deltas of three rows per group
        const bool bulk = !seq && p.sgd_atomic == 2 && std::is_same<T, float>::value;
        const size_t smem = bulk ? (size_t)gpb * 2 * 3 * R * sizeof(T) : 0;
        if constexpr ((R / k::Vec<T>::n) % C == 0)
            LAUNCH(ctx, k::k_sgd<T, R, C>, g, seq ? 32 : sgd_block(), smem, (const uint4 *)c.rec.p,
                   (const double *)c.v64.p,
                   c.n, tile_len, c.ntiles, U[0].p, U[1].p, U[2].p, (const T *)lr_dev.p, (T)p.lambda, p.sgd_atomic,
                   seq ? 1 : 0, stride, d0, d1, d2);
    }

    void ccdpp_init()
    {
        for (int m = 0; m < 3; ++m)
            LAUNCH(ctx, k::k_col_to_row<T>, grid_for((uint64_t)dims[m] * R, 256, kSMs * 8), 256, 0,
                   (const T *)U[m].p, Urow[m].p, dims[m], R);
        for (int m = 0; m < 3; ++m) {
            DevTensor<T> &c = D->copy[m];
            if (c.ks.rbits)
                LAUNCH(ctx, (k::k_ccdpp_init<T, R, true>), grid_for(c.nslots, 256, kSMs * 16), 256, 0, c.keys.p,
                       (const T *)c.x.p, c.res.p, c.nslots, c.ks, m, (const T *)Urow[0].p, (const T *)Urow[1].p,
                       (const T *)Urow[2].p);
            else
                LAUNCH(ctx, (k::k_ccdpp_init<T, R, false>), grid_for(c.nslots, 256, kSMs * 16), 256, 0, c.keys.p,
                       (const T *)c.x.p, c.res.p, c.nslots, c.ks, m, (const T *)Urow[0].p, (const T *)Urow[1].p,
                       (const T *)Urow[2].p);
        }
    }

    // fresh: the column's first pass (no mode swept yet in this column)
    template <int E>
    void ccdpp_pass(int m, int f, bool first, bool fresh)
    {
        DevTensor<T> &c = D->copy[m];
        T *out = U[m].p + (size_t)f * dims[m];
        k::CcdppCols<T> cols{};
        size_t need[2], need2[2];
        for (int q = 0; q < 2; ++q) {
            const int n = (m + 1 + q) % 3;
            cols.col[q] = U[n].p + (size_t)f * dims[n];
            cols.pk[q] = pk[n].p;
            cols.pk2[q] = pk2[n].p;
            cols.dim[q] = dims[n];
            // bytes one copy takes (the column copy may start up to 15
            // bytes early to reach a 16-byte boundary)
            need[q] = first ? (size_t)dims[n] * sizeof(k::Pack3<T>) : (((size_t)dims[n] * sizeof(T) + 15 + 15) & ~15ull);
            need2[q] = ((size_t)dims[n] * sizeof(k::Pack2<T>) + 15) & ~15ull;
        }
        // the column's first pass: both gathered modes' half packs staged in
        // a 1024-thread block per SM, when they fit its shared memory
        if (fresh && p.smem_budget >= 0 &&
            need2[0] + need2[1] <= std::min<size_t>((size_t)ccdpp_smem_max(),
                                                    p.smem_budget > 0 ? 2 * (size_t)p.smem_budget : SIZE_MAX)) {
            cols.stage[0] = cols.stage[1] = 1;
            const unsigned g = grid_for((uint64_t)c.ntasks, 32, kSMs);
            if (c.ks.rbits)
                ccdpp_launch_fresh<E, true>(c, g, need2[0] + need2[1], cols, out, m);
            else
                ccdpp_launch_fresh<E, false>(c, g, need2[0] + need2[1], cols, out, m);
            return;
        }
        // stage both when they fit, else the one that fits
        const size_t budget = ccdpp_budget();
        if (need[0] + need[1] <= budget) {
            cols.stage[0] = cols.stage[1] = 1;
        } else if (need[0] <= budget || need[1] <= budget) {
            const int q = (need[0] <= budget && (need[1] > budget || need[0] >= need[1])) ? 0 : 1;
            cols.stage[q] = 1;
        }
        const size_t smem = (cols.stage[0] ? need[0] : 0) + (cols.stage[1] ? need[1] : 0);
        // a later sweep that stages one sizeable column and gathers the other
        // through L1: one 1024-thread block per SM holds the staged column
        // once, which leaves L1 more room for the other
        if (!first && (cols.stage[0] ^ cols.stage[1]) && smem >= kCcdppBigStaged) {
            const unsigned g = grid_for((uint64_t)c.ntasks, 32, kSMs);
            if (c.ks.rbits)
                ccdpp_launch_big<E, true>(c, g, smem, cols, out, m);
            else
                ccdpp_launch_big<E, false>(c, g, smem, cols, out, m);
            return;
        }
        const unsigned g = grid_for((uint64_t)c.ntasks, 16, kSMs * 2);
        if (c.ks.rbits)
            ccdpp_launch<E, true>(c, first, g, smem, cols, out, m);
        else
            ccdpp_launch<E, false>(c, first, g, smem, cols, out, m);
    }

    template <int E, bool PK>
    void ccdpp_launch_big(DevTensor<T> &c, unsigned g, size_t smem, const k::CcdppCols<T> &cols, T *out, int m)
    {
        LAUNCH(ctx, (k::k_ccdpp_pass<T, false, E, PK, false, true>), g, 1024, smem, (const int4 *)c.tasks.p,
               c.ntasks, c.keys.p, c.res.p, c.ks, pk[m].p, cols, out, (T)p.lambda, slot.p, slot2.p,
               (const uint4 *)c.heavy.p, hcnt[m].p, dev_err.p, k::TaskClaim{claim.p, kCcdppStrideQuarters});
    }

    template <int E, bool PK>
    void ccdpp_launch(DevTensor<T> &c, bool first, unsigned g, size_t smem, const k::CcdppCols<T> &cols, T *out,
                      int m)
    {
        if (first)
            LAUNCH(ctx, (k::k_ccdpp_pass<T, true, E, PK>), g, 512, smem, (const int4 *)c.tasks.p, c.ntasks, c.keys.p,
                   c.res.p, c.ks, pk[m].p, cols, out, (T)p.lambda, slot.p, slot2.p, (const uint4 *)c.heavy.p,
                   hcnt[m].p, dev_err.p, k::TaskClaim{claim.p, kCcdppStrideQuarters});
        else
            LAUNCH(ctx, (k::k_ccdpp_pass<T, false, E, PK>), g, 512, smem, (const int4 *)c.tasks.p, c.ntasks,
                   c.keys.p, c.res.p, c.ks, pk[m].p, cols, out, (T)p.lambda, slot.p, slot2.p,
                   (const uint4 *)c.heavy.p, hcnt[m].p, dev_err.p, k::TaskClaim{claim.p, kCcdppStrideQuarters});
    }

    template <int E, bool PK>
    void ccdpp_launch_fresh(DevTensor<T> &c, unsigned g, size_t smem, const k::CcdppCols<T> &cols, T *out, int m)
    {
        LAUNCH(ctx, (k::k_ccdpp_pass<T, true, E, PK, true>), g, 1024, smem, (const int4 *)c.tasks.p, c.ntasks,
               c.keys.p, c.res.p, c.ks, pk[m].p, cols, out, (T)p.lambda, slot.p, slot2.p, (const uint4 *)c.heavy.p,
               hcnt[m].p, dev_err.p, k::TaskClaim{claim.p, kCcdppStrideQuarters});
    }

    // One CCD++ outer iteration: per column f, the {cur, prev, old} packs,
    // then `inner` sweeps over the modes of the column update (the first
    // sweep of each copy also refreshes its residual); finally one pass per
    // copy removes the last column's term, leaving r = x - model in every
    // copy and the training SSE in scalars[0].
    void ccdpp_outer()
    {
        const int inner = p.inner > 0 ? p.inner : 1;
        const int lanes = ccdpp_lanes((int)tile_len);
        for (int f = 0; f < R; ++f) {
            k::PackArgs pa{};
            for (int n = 0; n < 3; ++n) {
                pa.pk[n] = pk[n].p;
                pa.pk2[n] = pk2[n].p;
                pa.col[n] = U[n].p + (size_t)f * dims[n];
                pa.pcol[n] = f > 0 ? (const void *)(U[n].p + (size_t)(f - 1) * dims[n]) : nullptr;
                pa.dims[n] = dims[n];
            }
            LAUNCH(ctx, k::k_ccdpp_pack<T>, grid_for((uint64_t)dims[0] + dims[1] + dims[2], 256, kSMs * 8), 256, 0,
                   pa);
            for (int it = 0; it < inner; ++it) {
                for (int q = 0; q < 3; ++q) {
                    const int m = (p.mode_start + q) % 3;
                    // a row without nonzeros gets u = 0 / (lambda + 0): the
                    // pass writes only the rows it sees
                    if (D->copy[m].nrows != dims[m])
                        CK(cudaMemsetAsync(U[m].p + (size_t)f * dims[m], 0, dims[m] * sizeof(T), ctx->stream));
                    const bool fresh = it == 0 && q == 0;
                    if (lanes == 4) ccdpp_pass<4>(m, f, it == 0, fresh);
                    else if (lanes == 8) ccdpp_pass<8>(m, f, it == 0, fresh);
                    else ccdpp_pass<16>(m, f, it == 0, fresh);
                }
            }
        }
        for (int m = 0; m < 3; ++m) {
            DevTensor<T> &c = D->copy[m];
            const unsigned g = grid_for(c.nslots, 256, kMaxPartials);
            const T *c0 = U[0].p + (size_t)(R - 1) * dims[0], *c1 = U[1].p + (size_t)(R - 1) * dims[1],
                    *c2 = U[2].p + (size_t)(R - 1) * dims[2];
            double *part = m == 0 ? ctx->partial.p : (double *)nullptr;
            if (c.ks.rbits)
                LAUNCH(ctx, (k::k_ccdpp_finish<T, true>), g, 256, 0, c.keys.p, c.res.p, c.nslots, c.ks, m, c0, c1, c2,
                       part);
            else
                LAUNCH(ctx, (k::k_ccdpp_finish<T, false>), g, 256, 0, c.keys.p, c.res.p, c.nslots, c.ks, m, c0, c1,
                       c2, part);
            if (m == 0)
                LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p + 0);
        }
    }

    void one_epoch()
    {
        switch (p.alg) {
        case CTC_ALG_ALS: als_epoch(); break;
        case CTC_ALG_CCD: ccd_epoch(); break;
        case CTC_ALG_CCDPP: ccdpp_outer(); break;
        case CTC_ALG_SGD: sgd_epoch(); break;
        }
    }

    void epochs(int n) override
    {
        if (!model_set) fail(CTC_E_ARG, "no model staged on the dataset");
        if (p.alg == CTC_ALG_SGD && !damp_ready) {
            TracePhase tp("SGD damping");
            prepare_damping(sgd_groups_per_block());
        }
        if constexpr (std::is_same<T, float>::value)
            if (p.alg == CTC_ALG_SGD && p.sgd_atomic == 3 && p.sgd_order != CTC_SGD_SEQUENTIAL && !hot_ready) {
                TracePhase tp("SGD hot rows");
                prepare_hot();
            }
        const bool use_graph = p.use_graph && !ctx->kt.on && p.sgd_order != CTC_SGD_SEQUENTIAL;
        for (int i = 0; i < n; ++i) {
            if (!use_graph) {
                one_epoch();
                continue;
            }
            // the first epoch of a session runs its launches directly: a
            // single-epoch run (the reference-shaped ctc_run) does not pay
            // for capturing and instantiating a graph it would launch once
            if (!graph && !eager_done) {
                eager_done = true;
                one_epoch();
                continue;
            }
            if (!graph) {
                TracePhase tp("epoch graph capture");
                cudaGraph_t g = nullptr;
                ctx->capturing = true;
                CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
                try {
                    one_epoch();
                } catch (...) {
                    cudaStreamEndCapture(ctx->stream, &g);
                    if (g) cudaGraphDestroy(g);
                    ctx->capturing = false;
                    throw;
                }
                CK(cudaStreamEndCapture(ctx->stream, &g));
                ctx->capturing = false;
                CK(cudaGraphInstantiate(&graph, g, 0));
                CK(cudaGraphDestroy(g));
            }
            CK(cudaGraphLaunch(graph, ctx->stream));
            ctx->launches += 1;
        }
    }

    // scalars: 0 train SSE, 2 val SSE, 3 test SSE, 4..6 sum of squares of U
    // row-major device factors (CCD++ keeps them column-major: converted)
    void row_factors(const T *Urm[3])
    {
        for (int m = 0; m < 3; ++m) {
            if (colmajor) {
                LAUNCH(ctx, k::k_col_to_row<T>, grid_for((uint64_t)dims[m] * R, 256, kSMs * 8), 256, 0,
                       (const T *)U[m].p, Urow[m].p, dims[m], R);
                Urm[m] = Urow[m].p;
            } else {
                Urm[m] = U[m].p;
            }
        }
    }

    void seg_sse(int which, const uint4 *chunks, uint32_t nchunks, const uint32_t *first, int ninst, double *partial,
                 double *out) override
    {
        if (colmajor) fail(CTC_E_UNSUP, "per-instance errors need the record layout (not CCD++)");
        const DevTensor<T> &t = which == 0 ? D->copy[0] : D->test;
        const T *Urm[3];
        row_factors(Urm);
        if (nchunks)
            LAUNCH(ctx, k::k_sse_chunks<T, R>, std::min<uint32_t>(nchunks, kSMs * 8), 256, 0, (const uint4 *)t.rec.p,
                   (const double *)t.v64.p, chunks, nchunks, Urm[0], Urm[1], Urm[2], partial);
        LAUNCH(ctx, k::k_fold_segments, grid_for((uint64_t)ninst, 128, 64), 128, 0, (const double *)partial, first,
               ninst, out);
    }

    void evaluate(ctc_epoch_stats *st) override
    {
        check_errors();
        const T *Urm[3];
        row_factors(Urm);
        if (colmajor && D->copy[0].ks.rbits) {
            // packed slots of copy 0 hold r = x - model in the key words
            const DevTensor<T> &c = D->copy[0];
            const unsigned g = grid_for(c.nslots, 256, kMaxPartials);
            LAUNCH(ctx, k::k_ccdpp_res_sumsq, g, 256, 0, (const uint64_t *)c.keys.p, c.nslots, c.ks.rbits,
                   ctx->partial.p);
            LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p + 0);
        } else if (colmajor) {
            // copy 0 holds r = x - model: its SSE is the sum of squares
            sumsq_into(D->copy[0].res.p, D->copy[0].nslots, 0);
        } else {
            sse_into(D->copy[0], Urm, 0);
        }
        for (int m = 0; m < 3; ++m) sumsq_into(U[m].p, (uint64_t)dims[m] * R, 4 + m);
        if (ds->has_val) sse_into(D->val, Urm, 2);
        if (ds->has_test) sse_into(D->test, Urm, 3);
        CK(cudaMemcpyAsync(ctx->h_scalars, ctx->scalars.p, kScalars * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        const double *s = ctx->h_scalars;
        st->loss = s[0];
        st->frob = p.lambda * (s[4] + s[5] + s[6]);
        st->rmse_tr = std::sqrt(s[0] / (double)ds->nnz_train);
        st->rmse_vl = ds->has_val ? std::sqrt(s[2] / (double)D->val.n) : -1.0;
        st->rmse_te = ds->has_test ? std::sqrt(s[3] / (double)D->test.n) : -1.0;
    }
};

static SessionBase *session_for(ctc_dataset *d, int rank)
{
    if (d->session && d->session_rank == rank) return d->session.get();
    d->session.reset();
    with_rank(rank, [&](auto RC) {
        constexpr int R = decltype(RC)::value;
        if (d->p.precision == CTC_PREC_F64) d->session.reset(new Session<double, R>(d));
        else d->session.reset(new Session<float, R>(d));
    });
    d->session_rank = rank;
    return d->session.get();
}

// The epoch loop of tc_als / tc_sgd / tc_ccd with tc_converge's bookkeeping
// (sgpu/completion.c:296-362) and the SGD learning-rate schedule
// (sgpu/sgd.cu:315-323).
static void run_loop(ctc_dataset *ds, SessionBase *S, ctc_model *model, ctc_model *best, const ctc_params &p,
                     ctc_epoch_cb cb, void *user, ctc_result *res)
{
    ctc_ctx *ctx = ds->ctx;
    {
        TracePhase tp("set model");
        S->set_model(model);
    }
    TracePhase tp_loop("epochs + evaluation");
    double lr_base = p.lr;
    const double scale = p.lr_scale > 0 ? p.lr_scale : 1.0;
    double best_rmse = 10000000.0;  // BEST_RMSE, sgpu/base.h:35
    int nbad = 0, best_epoch = 0;
    double prev_obj = 0, total_ms = 0;
    ctc_epoch_stats st{};
    // tc_converge runs after every epoch from the first (sgpu/als.cu:803-806):
    // the starting point (epoch 0) is reported but not tracked, so the first
    // epoch always becomes the best one, as in the reference
    auto report = [&](int epoch, double ms) -> bool {
        S->evaluate(&st);
        st.epoch = epoch;
        st.ms_epoch = ms;
        st.lr = lr_base * scale;
        if (!std::isfinite(st.loss)) fail(CTC_E_NUMERIC, "training loss is not finite at epoch %d", epoch);
        if (epoch == 0) return cb ? cb(user, &st) != 0 : false;
        const double conv = ds->has_val ? st.rmse_vl : st.rmse_tr;
        bool converged = false;
        if (conv - best_rmse < -p.tolerance) {
            nbad = 0;
            best_rmse = conv;
            best_epoch = epoch;
            S->save_best();
        } else if (++nbad == p.max_bad_epochs) {
            converged = true;
        }
        int stop = cb ? cb(user, &st) : 0;
        return stop != 0 || (p.early_stop && converged);
    };
    bool stop = report(0, 0.0);
    prev_obj = st.loss + st.frob;
    int e = 1;
    for (; !stop && e <= p.iters; ++e) {
        CK(cudaEventRecord(ctx->ev0, ctx->stream));
        S->epochs(1);
        CK(cudaEventRecord(ctx->ev1, ctx->stream));
        CK(cudaEventSynchronize(ctx->ev1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        total_ms += ms;
        const bool bold = p.alg == CTC_ALG_SGD && p.lr_schedule == CTC_LR_BOLD_DRIVER;
        const bool need = p.early_stop || bold || e == p.iters || (p.eval_every > 0 && e % p.eval_every == 0);
        if (need) stop = report(e, ms);
        if (p.alg == CTC_ALG_SGD) {
            if (bold) {
                const double obj = st.loss + st.frob;
                if (e > 1) lr_base *= (obj < prev_obj) ? 1.05 : 0.50;
                prev_obj = obj;
            } else if (p.lr_schedule == CTC_LR_EXP_DECAY) {
                lr_base *= p.lr_decay;
            }
            S->set_lr(lr_base * scale);
        }
    }
    if (res) {
        res->epochs_run = e - 1;
        res->best_epoch = best_epoch;
        res->best_rmse = best_rmse;
        res->final_rmse_tr = st.rmse_tr;
        res->final_rmse_vl = st.rmse_vl;
        res->final_rmse_te = st.rmse_te;
        res->total_ms = total_ms;
        res->nonspd_rows = S->nonspd();
    }
    TracePhase tp("get model");
    S->get_model(model, false);
    if (best) {
        if (best->nmodes != 3 || best->rank != model->rank) *best = *model;
        S->get_model(best, true);
    }
}

// 16-byte slices of an FP32 row per lane (1, 2 or 4) of a Hogwild launch for
// this rank and ctc_params.threads_per_row, as the SGD launch picks them
static int sgd_vectors_for(int rank, int threads_per_row)
{
    const int base = rank / 4;
    const int c = threads_per_row > 0 ? base / threads_per_row : 1;
    if (c >= 4 && base % 4 == 0) return 4;
    if (c >= 2 && base % 2 == 0) return 2;
    return 1;
}

static void check_params(const ctc_params *p)
{
    if (!p) fail(CTC_E_ARG, "null params");
    if (p->alg < CTC_ALG_ALS || p->alg > CTC_ALG_CCDPP) fail(CTC_E_ARG, "unknown algorithm %d", p->alg);
    if (p->precision != CTC_PREC_F32 && p->precision != CTC_PREC_F64 && p->precision != CTC_PREC_MIXED)
        fail(CTC_E_ARG, "unknown precision %d", p->precision);
    if (p->precision == CTC_PREC_MIXED && !(p->alg == CTC_ALG_ALS && (p->rank == 64 || p->rank == 32)) &&
        p->alg != CTC_ALG_CCDPP)
        fail(CTC_E_UNSUP, "mixed precision is available for ALS at ranks 32 and 64 (BF16 tensor-core Gram) and for "
                          "CCD++ (packed residual slots)");
    if (p->rank != 8 && p->rank != 16 && p->rank != 32 && p->rank != 64)
        fail(CTC_E_UNSUP, "rank %d not supported (8, 16, 32, 64)", p->rank);
    if (p->tile_len < 0 || p->tile_len > (1 << 20)) fail(CTC_E_ARG, "tile_len %d", p->tile_len);
    if (p->iters < 0) fail(CTC_E_ARG, "iters %d", p->iters);
    if (p->mode_start < 0 || p->mode_start > 2) fail(CTC_E_ARG, "mode_start %d", p->mode_start);
    if (p->sgd_atomic < 0 || p->sgd_atomic > 3) fail(CTC_E_ARG, "sgd_atomic %d (0 to 3)", p->sgd_atomic);
    if (p->alg == CTC_ALG_SGD && p->sgd_atomic == 3 && p->precision == CTC_PREC_F64)
        fail(CTC_E_UNSUP, "sgd_atomic 3 (block-merged hot rows) is FP32 only");
    const int tpb = p->threads_per_block;
    if (tpb < 0 || (tpb & (tpb - 1)) != 0 || tpb > 1024)
        fail(CTC_E_ARG, "threads_per_block %d: 0 or a power of two up to 1024", tpb);
    if (tpb > 0 && tpb < 32)
        fail(CTC_E_UNSUP, "threads_per_block %d: SGD blocks are whole warps here (32 to 512 threads)", tpb);
    if (tpb == 1024 && (p->sgd_atomic != 3 || p->sgd_order == CTC_SGD_SEQUENTIAL ||
                        sgd_vectors_for(p->rank, p->threads_per_row) > 2))
        fail(CTC_E_UNSUP, "threads_per_block 1024: block-merged hot-row SGD (sgd_atomic 3) with "
                          "threads_per_row >= rank / 8 only");
}

static void check_model(const ctc_dataset *d, const ctc_model *model, int rank)
{
    if (!model) fail(CTC_E_ARG, "null model");
    if (model->nmodes != 3 || model->rank != rank) fail(CTC_E_ARG, "model shape does not match the rank");
    for (int m = 0; m < 3; ++m)
        if (model->dims[m] != d->dims[m])
            fail(CTC_E_ARG, "model mode %d has %llu rows, the dataset %llu", m, (unsigned long long)model->dims[m],
                 (unsigned long long)d->dims[m]);
}

}  // namespace ctc

// ---------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------
extern "C" int ctc_ctx_create(int device, ctc_ctx **out)
{
    return guarded([&] {
        if (!out) fail(CTC_E_ARG, "null out");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            fail(CTC_E_NOGPU, "no CUDA device available");
        }
        if (device < 0 || device >= n) fail(CTC_E_ARG, "device %d out of range (%d devices)", device, n);
        CK(cudaSetDevice(device));
        auto c = std::make_unique<ctc_ctx>();
        c->device = device;
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        CK(cudaEventCreate(&c->ev0));
        CK(cudaEventCreate(&c->ev1));
        c->partial.alloc(kMaxPartials);
        c->scalars.alloc(kScalars);
        CK(cudaMemset(c->scalars.p, 0, kScalars * sizeof(double)));
        CK(cudaMallocHost(&c->h_scalars, kScalars * sizeof(double)));
        *out = c.release();
    });
}

extern "C" int ctc_ctx_destroy(ctc_ctx *ctx)
{
    if (!ctx) return CTC_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &e : ctx->kt.pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    ctx->partial.release();
    ctx->scalars.release();
    if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
    for (int q = 0; q < 2; ++q) {
        if (ctx->pin[q]) cudaFreeHost(ctx->pin[q]);
        if (ctx->pin_ev[q]) cudaEventDestroy(ctx->pin_ev[q]);
    }
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    dev_pool_trim();
    return CTC_OK;
}

extern "C" int ctc_ctx_kernel_launches(const ctc_ctx *ctx, uint64_t *out)
{
    return guarded([&] {
        if (!ctx || !out) fail(CTC_E_ARG, "null argument");
        *out = ctx->launches;
    });
}

extern "C" void *ctc_ctx_stream(ctc_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" int ctc_ctx_set_profiling(ctc_ctx *ctx, int on)
{
    return guarded([&] {
        if (!ctx) fail(CTC_E_ARG, "null context");
        kt_flush(ctx);
        ctx->kt.on = on != 0;
    });
}

extern "C" int ctc_ctx_kernel_time(ctc_ctx *ctx, const char *name, uint64_t *count, double *total_ms)
{
    return guarded([&] {
        if (!ctx || !name) fail(CTC_E_ARG, "null argument");
        kt_flush(ctx);
        uint64_t c = 0;
        double ms = 0;
        for (auto &kv : ctx->kt.acc)
            if (kv.first.find(name) != std::string::npos) {
                c += kv.second.first;
                ms += kv.second.second;
            }
        if (count) *count = c;
        if (total_ms) *total_ms = ms;
    });
}

extern "C" int ctc_ctx_reset_kernel_times(ctc_ctx *ctx)
{
    return guarded([&] {
        if (!ctx) fail(CTC_E_ARG, "null context");
        kt_flush(ctx);
        ctx->kt.acc.clear();
    });
}

extern "C" int ctc_params_check(const ctc_params *p)
{
    return guarded([&] { check_params(p); });
}

extern "C" int ctc_params_default(int alg, ctc_params *p)
{
    return guarded([&] {
        if (!p) fail(CTC_E_ARG, "null params");
        memset(p, 0, sizeof(*p));
        p->alg = alg;
        p->rank = 16;                 // DEFAULT_NFACTORS, sgpu/base.h:21
        p->lambda = alg == CTC_ALG_ALS ? 10.0 : (alg == CTC_ALG_SGD ? 1e-3 : 100.0);  // base.h:39-41
        p->lr = 1e-3;                 // LEARN_RATE, base.h:58
        p->lr_scale = 1e-5;           // SGD_MODIFICATION*, base.h:42-44
        p->lr_schedule = CTC_LR_BOLD_DRIVER;
        p->lr_decay = 0.95;
        p->iters = 1000;              // DEFAULT_MAX_ITERATE, base.h:22
        p->inner = 1;                 // NUM_INNER, base.h:30
        p->precision = CTC_PREC_F32;
        p->early_stop = 1;
        p->tolerance = 1e-4;          // TOLERANCE, base.h:36
        p->max_bad_epochs = 3;        // MAX_BADEPOCHS, base.h:32
        p->sgd_order = CTC_SGD_HOGWILD;
        p->sgd_atomic = 2;
        p->eval_every = 1;
    });
}

extern "C" int ctc_dataset_create(ctc_ctx *ctx, const ctc_tensor *const train[3], const ctc_tensor *val,
                                  const ctc_tensor *test, const ctc_params *p, ctc_dataset **out)
{
    return guarded([&] {
        if (!ctx || !train || !train[0] || !out) fail(CTC_E_ARG, "null argument");
        check_params(p);
        CK(cudaSetDevice(ctx->device));
        auto ds = std::make_unique<ctc_dataset>();
        ds->ctx = ctx;
        ds->p = *p;
        for (int m = 0; m < 3; ++m) {
            uint64_t d = 0;
            for (const ctc_tensor *t : {train[0], val, test})
                if (t && t->nmodes == 3) d = std::max(d, t->dims[m]);
            ds->dims[m] = d;
        }
        ds->nnz_train = train[0]->nnz;
        ds->has_val = val != nullptr;
        ds->has_test = test != nullptr;
        if (p->precision == CTC_PREC_F64) build_dataset<double>(ds.get(), train, val, test);
        else build_dataset<float>(ds.get(), train, val, test);
        *out = ds.release();
    });
}

extern "C" int ctc_dataset_dims(const ctc_dataset *d, uint64_t *dims)
{
    return guarded([&] {
        if (!d || !dims) fail(CTC_E_ARG, "null argument");
        for (int m = 0; m < 3; ++m) dims[m] = d->dims[m];
    });
}

extern "C" int ctc_dataset_free(ctc_dataset *d)
{
    if (d) {
        cudaSetDevice(d->ctx->device);
        cudaStreamSynchronize(d->ctx->stream);
        delete d;
    }
    return CTC_OK;
}

static void check_run_params(const ctc_dataset *d, const ctc_params *p)
{
    check_params(p);
    if (p->alg != d->p.alg || p->precision != d->p.precision || p->compat != d->p.compat ||
        p->tile_len != d->p.tile_len)
        fail(CTC_E_ARG, "parameters differ from the dataset's (alg/precision/compat/tile_len)");
}

extern "C" int ctc_dataset_run(ctc_dataset *d, ctc_model *model, ctc_model *best, const ctc_params *p,
                               ctc_epoch_cb cb, void *user, ctc_result *res)
{
    return guarded([&] {
        if (!d) fail(CTC_E_ARG, "null dataset");
        check_run_params(d, p);
        check_model(d, model, p->rank);
        CK(cudaSetDevice(d->ctx->device));
        d->p = *p;
        SessionBase *S;
        {
            TracePhase tp("session");
            S = session_for(d, p->rank);
            S->set_params(*p);
        }
        run_loop(d, S, model, best, *p, cb, user, res);
    });
}

extern "C" int ctc_dataset_set_model(ctc_dataset *d, const ctc_model *model)
{
    return guarded([&] {
        if (!d) fail(CTC_E_ARG, "null dataset");
        check_model(d, model, model ? model->rank : 0);
        CK(cudaSetDevice(d->ctx->device));
        d->p.rank = model->rank;
        session_for(d, model->rank)->set_model(model);
    });
}

extern "C" int ctc_dataset_epochs(ctc_dataset *d, int n)
{
    return guarded([&] {
        if (!d || n < 0) fail(CTC_E_ARG, "bad argument");
        if (!d->session) fail(CTC_E_ARG, "no model staged on the dataset");
        CK(cudaSetDevice(d->ctx->device));
        d->session->epochs(n);
    });
}

extern "C" int ctc_dataset_set_lr(ctc_dataset *d, double lr)
{
    return guarded([&] {
        if (!d || !d->session) fail(CTC_E_ARG, "no model staged on the dataset");
        d->session->set_lr(lr);
    });
}

extern "C" int ctc_dataset_evaluate(ctc_dataset *d, ctc_epoch_stats *st)
{
    return guarded([&] {
        if (!d || !st) fail(CTC_E_ARG, "null argument");
        if (!d->session) fail(CTC_E_ARG, "no model staged on the dataset");
        CK(cudaSetDevice(d->ctx->device));
        memset(st, 0, sizeof(*st));
        d->session->evaluate(st);
    });
}

extern "C" int ctc_dataset_probe_wait(ctc_dataset *d, uint64_t limit_ns)
{
    return guarded([&] {
        if (!d || !d->session) fail(CTC_E_ARG, "no model staged on the dataset");
        if (limit_ns == 0 || limit_ns > 2000000000ull) fail(CTC_E_ARG, "limit_ns must be in (0, 2e9]");
        CK(cudaSetDevice(d->ctx->device));
        d->session->probe_wait(limit_ns);
    });
}

extern "C" int ctc_dataset_get_model(ctc_dataset *d, ctc_model *model)
{
    return guarded([&] {
        if (!d || !d->session) fail(CTC_E_ARG, "no model staged on the dataset");
        check_model(d, model, d->session_rank);
        d->session->get_model(model, false);
    });
}

extern "C" int ctc_run(ctc_ctx *ctx, const ctc_tensor *const train[3], const ctc_tensor *val,
                       const ctc_tensor *test, ctc_model *model, ctc_model *best, const ctc_params *p,
                       ctc_epoch_cb cb, void *user, ctc_result *res)
{
    ctc_dataset *ds = nullptr;
    int rc = ctc_dataset_create(ctx, train, val, test, p, &ds);
    if (rc != CTC_OK) return rc;
    // the factor rows cover the tensors' index range (reference: traina
    // dims, sgpu/completion.c:439-446); a model with more rows is fine
    rc = guarded([&] {
        if (!model) fail(CTC_E_ARG, "null model");
        for (int m = 0; m < 3; ++m) {
            if (model->dims[m] < ds->dims[m])
                fail(CTC_E_ARG, "model mode %d has %llu rows, the tensors need %llu", m,
                     (unsigned long long)model->dims[m], (unsigned long long)ds->dims[m]);
            ds->dims[m] = model->dims[m];
        }
    });
    if (rc == CTC_OK) rc = ctc_dataset_run(ds, model, best, p, cb, user, res);
    TracePhase tp("free dataset");
    ctc_dataset_free(ds);
    return rc;
}

namespace ctc {
template <typename T, int R>
static double rmse_impl(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model)
{
    DevTensor<T> d;
    stage_tensor<T>(ctx, t, false, d);
    DevBuf<T> U[3];
    for (int m = 0; m < 3; ++m) {
        std::vector<T> h(model->U[m].begin(), model->U[m].end());
        U[m].upload(h.data(), h.size(), ctx->stream);
    }
    const unsigned g = grid_for(d.n, 256, kMaxPartials);
    LAUNCH(ctx, k::k_sse<T, R>, g, 256, 0, (const uint4 *)d.rec.p, (const double *)d.v64.p, d.n, (const T *)U[0].p,
           (const T *)U[1].p, (const T *)U[2].p, ctx->partial.p);
    LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p);
    double s = 0;
    CK(cudaMemcpyAsync(&s, ctx->scalars.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return std::sqrt(s / (double)d.n);
}

template <typename T, int R>
static void grad_impl(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double lambda,
                      double *const *grads, double *obj)
{
    // mode-0-sorted copy so the mode-0 gradient rows stay in registers
    ctc_tensor s(*t);
    if (ctc_tensor_sort(&s, 0) != CTC_OK) fail(CTC_E_ARG, "%s", ctc_last_error());
    DevTensor<T> d;
    stage_tensor<T>(ctx, &s, false, d);
    DevBuf<T> U[3], G[3];
    for (int m = 0; m < 3; ++m) {
        std::vector<T> h(model->U[m].begin(), model->U[m].end());
        U[m].upload(h.data(), h.size(), ctx->stream);
        G[m].alloc(h.size());
        LAUNCH(ctx, k::k_scale<T>, grid_for(h.size(), 256, kSMs * 8), 256, 0, (const T *)U[m].p, G[m].p,
               (uint64_t)h.size(), (T)(2.0 * lambda));
    }
    const uint32_t tl = 256;
    const uint32_t ntiles = (d.n + tl - 1) / tl;
    constexpr int GR = R / k::Vec<T>::n;
    const unsigned g = grid_for(ntiles, 8 * (32 / GR), kMaxPartials);
    LAUNCH(ctx, k::k_grad<T, R>, g, 256, 0, (const uint4 *)d.rec.p, (const double *)d.v64.p, d.n, tl, ntiles,
           (const T *)U[0].p, (const T *)U[1].p, (const T *)U[2].p, G[0].p, G[1].p, G[2].p, ctx->partial.p);
    LAUNCH(ctx, k::k_sum_partials, 1, 256, 0, (const double *)ctx->partial.p, (int)g, ctx->scalars.p);
    double half_sse = 0;
    CK(cudaMemcpyAsync(&half_sse, ctx->scalars.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    for (int m = 0; m < 3; ++m) {
        std::vector<T> h(G[m].n);
        CK(cudaMemcpyAsync(h.data(), G[m].p, h.size() * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (size_t i = 0; i < h.size(); ++i) grads[m][i] = (double)h[i];
    }
    if (obj) {
        double reg = 0;
        for (int m = 0; m < 3; ++m)
            for (double v : model->U[m]) reg += v * v;
        *obj = half_sse + lambda * reg;
    }
}
}  // namespace ctc

extern "C" int ctc_rmse(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double *rmse)
{
    return guarded([&] {
        if (!ctx || !t || !model || !rmse) fail(CTC_E_ARG, "null argument");
        CK(cudaSetDevice(ctx->device));
        validate_tensor(t, model->dims, "tensor");
        with_rank(model->rank, [&](auto RC) {
            constexpr int R = decltype(RC)::value;
            *rmse = rmse_impl<float, R>(ctx, t, model);
        });
    });
}

extern "C" int ctc_grad(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double lambda,
                        double *const *grads, double *obj)
{
    return guarded([&] {
        if (!ctx || !t || !model || !grads) fail(CTC_E_ARG, "null argument");
        CK(cudaSetDevice(ctx->device));
        if (t->nmodes == 4) {
            ctc_grad_fo(ctx, t, model, lambda, grads, obj);
            return;
        }
        validate_tensor(t, model->dims, "tensor");
        with_rank(model->rank, [&](auto RC) {
            constexpr int R = decltype(RC)::value;
            grad_impl<double, R>(ctx, t, model, lambda, grads, obj);
        });
    });
}

// ---------------------------------------------------------------------
// Batches of independent completion problems.  Instance b's tensors are
// stacked into one block-diagonal tensor: its mode-m indices are shifted by
// off[m][b] = sum of the earlier instances' dimensions, so rows of different
// instances never meet.  One dataset over the stacked tensor then trains
// every instance with one launch per kernel and epoch, the tile plan
// balancing the work across instance boundaries; the ALS row solves, the
// SGD updates and the reference CCD+ updates of an instance see only its
// own nonzeros.  Errors are kept per instance: the mode-1 training copy and
// the test tensor are instance-contiguous, cut into chunks that never
// straddle two instances, and summed per instance in chunk order.
// ---------------------------------------------------------------------
struct ctc_batch {
    ctc_ctx *ctx = nullptr;
    int ninst = 0;
    ctc_params p{};
    std::unique_ptr<ctc_dataset> ds;
    std::vector<uint64_t> off[3], idims[3];
    std::vector<uint64_t> ntr, nte;
    bool has_test = false;
    ctc::DevBuf<uint4> ch_tr, ch_te;
    ctc::DevBuf<uint32_t> first_tr, first_te;
    uint32_t nch_tr = 0, nch_te = 0;
    ctc::DevBuf<double> partial, sse;  // sse: [0, ninst) train, [ninst, 2 ninst) test
};

namespace ctc {

static constexpr uint32_t kBatchChunk = 16384;

// chunks of [start_b, start_b + n_b) per instance, and each instance's first
// chunk (ninst + 1 entries)
static void batch_chunks(const std::vector<uint64_t> &n, std::vector<uint4> &ch, std::vector<uint32_t> &first)
{
    ch.clear();
    first.assign(n.size() + 1, 0);
    uint64_t start = 0;
    for (size_t b = 0; b < n.size(); ++b) {
        first[b] = (uint32_t)ch.size();
        for (uint64_t s = 0; s < n[b]; s += kBatchChunk)
            ch.push_back(make_uint4((uint32_t)(start + s), (uint32_t)(start + std::min<uint64_t>(n[b], s + kBatchChunk)),
                                    (uint32_t)b, 0u));
        start += n[b];
    }
    first[n.size()] = (uint32_t)ch.size();
}

static void batch_eval(ctc_batch *B, SessionBase *S, std::vector<double> &rtr, std::vector<double> &rte)
{
    const int n = B->ninst;
    S->seg_sse(0, B->ch_tr.p, B->nch_tr, B->first_tr.p, n, B->partial.p, B->sse.p);
    if (B->has_test) S->seg_sse(1, B->ch_te.p, B->nch_te, B->first_te.p, n, B->partial.p, B->sse.p + n);
    std::vector<double> h(2 * (size_t)n, 0.0);
    CK(cudaMemcpyAsync(h.data(), B->sse.p, (B->has_test ? 2 : 1) * (size_t)n * sizeof(double),
                       cudaMemcpyDeviceToHost, B->ctx->stream));
    CK(cudaStreamSynchronize(B->ctx->stream));
    rtr.resize(n);
    rte.resize(n);
    for (int b = 0; b < n; ++b) {
        rtr[b] = B->ntr[b] ? std::sqrt(h[b] / (double)B->ntr[b]) : 0.0;
        rte[b] = (B->has_test && B->nte[b]) ? std::sqrt(h[n + b] / (double)B->nte[b]) : -1.0;
        if (!std::isfinite(rtr[b])) fail(CTC_E_NUMERIC, "instance %d: training error is not finite", b);
    }
}

}  // namespace ctc

extern "C" int ctc_batch_create(ctc_ctx *ctx, int ninst, const ctc_tensor *const *train,
                                const ctc_tensor *const *test, const ctc_params *p, ctc_batch **out)
{
    return guarded([&] {
        if (!ctx || !train || !out || ninst <= 0) fail(CTC_E_ARG, "null argument or no instances");
        check_params(p);
        if (p->alg == CTC_ALG_CCDPP) fail(CTC_E_UNSUP, "batches run ALS, CCD and SGD");
        if (p->compat) fail(CTC_E_UNSUP, "batches run the plain update rules (compat = 0)");
        CK(cudaSetDevice(ctx->device));
        auto B = std::make_unique<ctc_batch>();
        B->ctx = ctx;
        B->ninst = ninst;
        B->p = *p;
        B->has_test = test != nullptr;
        uint64_t ntot = 0, ttot = 0;
        for (int m = 0; m < 3; ++m) {
            B->off[m].assign(ninst + 1, 0);
            B->idims[m].assign(ninst, 0);
        }
        B->ntr.assign(ninst, 0);
        B->nte.assign(ninst, 0);
        for (int b = 0; b < ninst; ++b) {
            const ctc_tensor *tr = train[b], *te = test ? test[b] : nullptr;
            if (!tr || tr->nmodes != 3 || tr->nnz == 0) fail(CTC_E_ARG, "instance %d: empty or not order-3 training tensor", b);
            if (test && (!te || te->nmodes != 3)) fail(CTC_E_ARG, "instance %d: missing or not order-3 test tensor", b);
            for (int m = 0; m < 3; ++m) {
                B->idims[m][b] = std::max(tr->dims[m], te ? te->dims[m] : 0);
                B->off[m][b + 1] = B->off[m][b] + B->idims[m][b];
            }
            B->ntr[b] = tr->nnz;
            B->nte[b] = te ? te->nnz : 0;
            ntot += tr->nnz;
            ttot += B->nte[b];
        }
        for (int m = 0; m < 3; ++m)
            if (B->off[m][ninst] >= 0xfffffff0ull) fail(CTC_E_UNSUP, "stacked dimension %d exceeds 2^32", m + 1);
        if (ntot >= 0x7fffffffull || ttot >= 0x7fffffffull) fail(CTC_E_UNSUP, "more than 2^31 stacked nonzeros");
        // stacked tensors (1-based indices shifted by the instance offsets)
        auto stack = [&](const ctc_tensor *const *src, uint64_t total, const std::vector<uint64_t> &cnt) {
            auto t = std::make_unique<ctc_tensor>();
            t->nmodes = 3;
            t->nnz = total;
            for (int m = 0; m < 3; ++m) {
                t->dims[m] = B->off[m][ninst];
                t->ind[m].resize(total);
            }
            t->vals.resize(total);
            std::vector<uint64_t> start(ninst + 1, 0);
            for (int b = 0; b < ninst; ++b) start[b + 1] = start[b] + cnt[b];
            // (indices were checked against the instance dims, which are
            // their maxima; 0 is the one bad value left)
            std::atomic<int> bad{-1};
            for (int b = 0; b < ninst; ++b) {
                const ctc_tensor *s = src[b];
                for (int m = 0; m < 3; ++m) {
                    const uint64_t o = B->off[m][b];
                    const uint64_t *in = s->ind[m].data();
                    uint64_t *dst = t->ind[m].data() + start[b];
                    par_for(cnt[b], [&](uint64_t i0, uint64_t i1) {
                        for (uint64_t i = i0; i < i1; ++i) {
                            if (in[i] == 0) bad = b;
                            dst[i] = in[i] + o;
                        }
                    });
                }
                std::copy(s->vals.begin(), s->vals.end(), t->vals.begin() + start[b]);
            }
            if (bad >= 0) fail(CTC_E_ARG, "instance %d: 0 index in a 1-based tensor", bad.load());
            return t;
        };
        std::unique_ptr<ctc_tensor> st = stack(train, ntot, B->ntr);
        // mode-1 order of the stacked tensor is instance-major: instance b's
        // training nonzeros are [sum of earlier counts, + ntr[b]) in copy 0
        if (ctc_tensor_sort(st.get(), 0) != CTC_OK) fail(CTC_E_ARG, "%s", ctc_last_error());
        std::unique_ptr<ctc_tensor> tt;
        if (test) tt = stack(test, ttot, B->nte);
        auto ds = std::make_unique<ctc_dataset>();
        ds->ctx = ctx;
        ds->p = *p;
        for (int m = 0; m < 3; ++m) ds->dims[m] = B->off[m][ninst];
        ds->nnz_train = ntot;
        ds->has_val = false;
        ds->has_test = test != nullptr;
        const ctc_tensor *tr3[3] = {st.get(), nullptr, nullptr};
        if (p->precision == CTC_PREC_F64) build_dataset<double>(ds.get(), tr3, nullptr, tt.get());
        else build_dataset<float>(ds.get(), tr3, nullptr, tt.get());
        B->ds = std::move(ds);
        std::vector<uint4> ch;
        std::vector<uint32_t> first;
        batch_chunks(B->ntr, ch, first);
        B->nch_tr = (uint32_t)ch.size();
        B->ch_tr.upload(ch.data(), ch.size(), ctx->stream);
        B->first_tr.upload(first.data(), first.size(), ctx->stream);
        size_t nparts = ch.size();
        if (test) {
            batch_chunks(B->nte, ch, first);
            B->nch_te = (uint32_t)ch.size();
            B->ch_te.upload(ch.data(), ch.size(), ctx->stream);
            B->first_te.upload(first.data(), first.size(), ctx->stream);
            nparts = std::max(nparts, ch.size());
        }
        B->partial.alloc(std::max<size_t>(nparts, 1));
        B->sse.alloc(2 * (size_t)ninst);
        CK(cudaStreamSynchronize(ctx->stream));
        *out = B.release();
    });
}

extern "C" int ctc_batch_free(ctc_batch *b)
{
    if (b) {
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
        delete b;
    }
    return CTC_OK;
}

extern "C" int ctc_batch_info(const ctc_batch *b, int *ninst, uint64_t *nnz_train, uint64_t *nnz_test)
{
    return guarded([&] {
        if (!b) fail(CTC_E_ARG, "null batch");
        if (ninst) *ninst = b->ninst;
        uint64_t a = 0, c = 0;
        for (int i = 0; i < b->ninst; ++i) {
            a += b->ntr[i];
            c += b->nte[i];
        }
        if (nnz_train) *nnz_train = a;
        if (nnz_test) *nnz_test = c;
    });
}

extern "C" int ctc_batch_run(ctc_batch *B, ctc_model *const *models, const ctc_params *p, ctc_batch_cb cb,
                             void *user, ctc_result *res)
{
    return guarded([&] {
        if (!B || !models) fail(CTC_E_ARG, "null argument");
        check_params(p);
        if (p->alg != B->p.alg || p->precision != B->p.precision || p->compat != B->p.compat ||
            p->tile_len != B->p.tile_len)
            fail(CTC_E_ARG, "parameters differ from the batch's (alg/precision/compat/tile_len)");
        const int n = B->ninst, R = p->rank;
        // the stacked model: instance b's rows at off[m][b]
        ctc_model sm;
        sm.nmodes = 3;
        sm.rank = R;
        for (int m = 0; m < 3; ++m) {
            sm.dims[m] = B->off[m][n];
            sm.U[m].assign(sm.dims[m] * (uint64_t)R, 0.0);
        }
        for (int b = 0; b < n; ++b) {
            const ctc_model *mb = models[b];
            if (!mb || mb->nmodes != 3 || mb->rank != R) fail(CTC_E_ARG, "instance %d: model missing or of another rank", b);
            for (int m = 0; m < 3; ++m) {
                if (mb->dims[m] < B->idims[m][b]) fail(CTC_E_ARG, "instance %d: model smaller than its tensors", b);
                std::copy(mb->U[m].begin(), mb->U[m].begin() + B->idims[m][b] * R,
                          sm.U[m].begin() + B->off[m][b] * R);
            }
        }
        ctc_ctx *ctx = B->ctx;
        CK(cudaSetDevice(ctx->device));
        B->ds->p = *p;
        SessionBase *S = session_for(B->ds.get(), R);
        S->set_params(*p);
        S->set_model(&sm);
        double lr_base = p->lr, total_ms = 0, prev_obj = 0;
        const double scale = p->lr_scale > 0 ? p->lr_scale : 1.0;
        std::vector<double> rtr, rte;
        auto report = [&](int epoch, double ms) -> bool {
            batch_eval(B, S, rtr, rte);
            return cb ? cb(user, epoch, n, rtr.data(), rte.data(), ms) != 0 : false;
        };
        bool stop = report(0, 0.0);
        int e = 1;
        for (; !stop && e <= p->iters; ++e) {
            CK(cudaEventRecord(ctx->ev0, ctx->stream));
            S->epochs(1);
            CK(cudaEventRecord(ctx->ev1, ctx->stream));
            CK(cudaEventSynchronize(ctx->ev1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            total_ms += ms;
            const bool bold = p->alg == CTC_ALG_SGD && p->lr_schedule == CTC_LR_BOLD_DRIVER;
            if (bold || e == p->iters || (p->eval_every > 0 && e % p->eval_every == 0)) stop = report(e, ms);
            if (p->alg == CTC_ALG_SGD) {
                if (bold) {
                    // the schedule follows the summed training error of all instances
                    double obj = 0;
                    for (int b = 0; b < n; ++b) obj += rtr[b] * rtr[b] * (double)B->ntr[b];
                    if (e > 1) lr_base *= (obj < prev_obj) ? 1.05 : 0.50;
                    prev_obj = obj;
                } else if (p->lr_schedule == CTC_LR_EXP_DECAY) {
                    lr_base *= p->lr_decay;
                }
                S->set_lr(lr_base * scale);
            }
        }
        S->get_model(&sm, false);
        for (int b = 0; b < n; ++b)
            for (int m = 0; m < 3; ++m)
                std::copy(sm.U[m].begin() + B->off[m][b] * R, sm.U[m].begin() + (B->off[m][b] + B->idims[m][b]) * R,
                          models[b]->U[m].begin());
        if (res) {
            *res = ctc_result{};
            res->epochs_run = e - 1;
            res->total_ms = total_ms;
            res->best_epoch = e - 1;
            double se_tr = 0, se_te = 0, ntr = 0, nte = 0;
            for (int b = 0; b < n; ++b) {
                se_tr += rtr[b] * rtr[b] * (double)B->ntr[b];
                ntr += (double)B->ntr[b];
                if (B->has_test) {
                    se_te += rte[b] * rte[b] * (double)B->nte[b];
                    nte += (double)B->nte[b];
                }
            }
            res->final_rmse_tr = ntr > 0 ? std::sqrt(se_tr / ntr) : 0.0;
            res->final_rmse_te = nte > 0 ? std::sqrt(se_te / nte) : -1.0;
            res->final_rmse_vl = -1.0;
            res->best_rmse = res->final_rmse_tr;
            res->nonspd_rows = S->nonspd();
        }
    });
}

// ---------------------------------------------------------------------
// Autotuner: per tensor shape, the tile length (all algorithms), the lanes
// per nonzero (SGD) and the shared-memory staging budget (CCD++) are
// searched by timing update epochs on the device, and the winner is cached
// in a text file -- this project's replacement for the reference's offline
// genetic search over tile length and block size (ga/, fitness.c:67-79).
// ---------------------------------------------------------------------
namespace ctc {

struct TuneCand {
    int tile_len = 0, threads_per_row = 0, smem_budget = 0, sgd_atomic = 0, threads_per_block = 0;
};

// shape key: algorithm, precision, rank, compat, SGD order, dimensions and
// nonzeros rounded to half powers of two, and the device's SM count
static std::string tune_key(const ctc_params &p, const uint64_t dims[3], uint64_t nnz, int sms)
{
    auto b = [](uint64_t x) { return (long)std::lround(2.0 * std::log2((double)std::max<uint64_t>(x, 1))); };
    char buf[256];
    snprintf(buf, sizeof buf, "alg=%d,prec=%d,rank=%d,compat=%d,order=%d,I=%ld,J=%ld,K=%ld,nnz=%ld,sms=%d", p.alg,
             p.precision, p.rank, p.compat, p.alg == CTC_ALG_SGD ? p.sgd_order : 0, b(dims[0]), b(dims[1]),
             b(dims[2]), b(nnz), sms);
    return buf;
}

// cache lines: "<key> tile_len=<t> threads_per_row=<c> smem_budget=<s> ms=<x>"
static bool tune_read(const char *path, const std::string &key, TuneCand &c, double &ms)
{
    if (!path) return false;
    FILE *f = fopen(path, "r");
    if (!f) return false;
    char line[512];
    bool found = false;
    while (fgets(line, sizeof line, f)) {
        char k[300];
        TuneCand t;
        double x = 0;
        if (sscanf(line, "%299s tile_len=%d threads_per_row=%d smem_budget=%d sgd_atomic=%d threads_per_block=%d ms=%lf",
                   k, &t.tile_len, &t.threads_per_row, &t.smem_budget, &t.sgd_atomic, &t.threads_per_block,
                   &x) == 7 &&
            key == k) {
            c = t;  // the last entry for a key wins
            ms = x;
            found = true;
        }
    }
    fclose(f);
    return found;
}

static void tune_write(const char *path, const std::string &key, const TuneCand &c, double ms)
{
    if (!path) return;
    std::vector<std::string> keep;
    if (FILE *f = fopen(path, "r")) {
        char line[512];
        while (fgets(line, sizeof line, f)) {
            char k[300];
            if (sscanf(line, "%299s", k) == 1 && key == k) continue;
            keep.emplace_back(line);
        }
        fclose(f);
    }
    FILE *f = fopen(path, "w");
    if (!f) fail(CTC_E_IO, "cannot write the tuning cache %s", path);
    for (const std::string &l : keep) fputs(l.c_str(), f);
    fprintf(f, "%s tile_len=%d threads_per_row=%d smem_budget=%d sgd_atomic=%d threads_per_block=%d ms=%.6f\n",
            key.c_str(), c.tile_len, c.threads_per_row, c.smem_budget, c.sgd_atomic, c.threads_per_block, ms);
    fclose(f);
}

static std::vector<TuneCand> tune_space(const ctc_params &p)
{
    std::vector<TuneCand> v;
    auto add = [&](int t, int c, int s, int a = -1) {
        TuneCand x;
        x.tile_len = t;
        x.threads_per_row = c;
        x.smem_budget = s;
        x.sgd_atomic = a < 0 ? p.sgd_atomic : a;
        x.threads_per_block = p.threads_per_block;
        v.push_back(x);
    };
    switch (p.alg) {
    case CTC_ALG_ALS:
        // mixed precision: shorter tiles send more rows to the tensor-core Gram
        if (p.precision == CTC_PREC_MIXED) add(128, 0, 0);
        for (int t : {256, 512, 1024, 2048}) add(t, 0, 0);
        break;
    case CTC_ALG_CCD:
        if (p.compat) add(32, 0, 0);  // the reference multiplicities need 32-long tiles
        else
            for (int t : {256, 512, 1024}) add(t, 0, 0);
        break;
    case CTC_ALG_CCDPP:
        for (int t : {128, 256, 512})
            for (int s : {0, -1}) add(t, 0, s);
        break;
    case CTC_ALG_SGD: {
        const int base = p.rank / (p.precision == CTC_PREC_F64 ? 2 : 4);  // lanes at one vector each
        if (p.sgd_order == CTC_SGD_SEQUENTIAL) {
            add(p.tile_len, 0, 0);
            break;
        }
        // FP32: vector atomic adds, bulk row reductions or block-merged hot
        // rows (which one is faster depends on how hot the hottest rows are)
        const bool f32 = p.precision != CTC_PREC_F64;
        for (int t : {128, 256, 512, 1024})
            for (int c : {base, base / 2, base / 4})
                if (c >= 1) {
                    if (f32 && p.sgd_atomic != 0) {
                        add(t, c, 0, 1);
                        add(t, c, 0, 2);
                        add(t, c, 0, 3);
                    } else {
                        add(t, c, 0);
                    }
                }
        break;
    }
    }
    return v;
}

static int device_sms(int dev)
{
    int n = 0;
    CK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

}  // namespace ctc

extern "C" int ctc_tune_key(const ctc_tensor *train, const ctc_params *p, int sm_count, char *buf, int len)
{
    return guarded([&] {
        if (!train || !p || !buf || len <= 0) fail(CTC_E_ARG, "null argument");
        const std::string key = tune_key(*p, train->dims, train->nnz, sm_count);
        if ((int)key.size() >= len) fail(CTC_E_ARG, "buffer of %d bytes is too small", len);
        memcpy(buf, key.c_str(), key.size() + 1);
    });
}

extern "C" int ctc_tune_lookup(const char *cache_path, const ctc_tensor *train, const ctc_params *p, int sm_count,
                               ctc_params *out)
{
    return guarded([&] {
        if (!cache_path || !train || !p || !out) fail(CTC_E_ARG, "null argument");
        const std::string key = tune_key(*p, train->dims, train->nnz, sm_count);
        TuneCand c;
        double ms = 0;
        if (!tune_read(cache_path, key, c, ms)) fail(CTC_E_NOTFOUND, "no tuned entry for %s", key.c_str());
        *out = *p;
        out->tile_len = c.tile_len;
        out->threads_per_row = c.threads_per_row;
        out->smem_budget = c.smem_budget;
        out->sgd_atomic = c.sgd_atomic;
        out->threads_per_block = c.threads_per_block;
    });
}

extern "C" int ctc_autotune(ctc_ctx *ctx, const ctc_tensor *const train[3], const ctc_params *p,
                            const char *cache_path, int flags, ctc_params *out, ctc_tune_trial *trials,
                            int max_trials, int *ntrials)
{
    return guarded([&] {
        if (!ctx || !train || !train[0] || !p || !out) fail(CTC_E_ARG, "null argument");
        check_params(p);
        CK(cudaSetDevice(ctx->device));
        const int sms = device_sms(ctx->device);
        const std::string key = tune_key(*p, train[0]->dims, train[0]->nnz, sms);
        *out = *p;
        int nt = 0;
        TuneCand best;
        double best_ms = 0;
        if (!(flags & CTC_TUNE_FORCE) && tune_read(cache_path, key, best, best_ms)) {
            if (trials && max_trials > 0) {
                trials[0] = ctc_tune_trial{best.tile_len, best.threads_per_row, best.smem_budget, best_ms, 1,
                                           best.sgd_atomic, best.threads_per_block};
                nt = 1;
            }
        } else {
            const std::vector<TuneCand> space = tune_space(*p);
            best_ms = 1e300;
            std::vector<int> tiles;
            for (const TuneCand &c : space)
                if (std::find(tiles.begin(), tiles.end(), c.tile_len) == tiles.end()) tiles.push_back(c.tile_len);
            for (int tl : tiles) {
                // one staging per tile length; the other knobs are run-time
                ctc_params q = *p;
                q.tile_len = tl;
                q.early_stop = 0;
                q.use_graph = 0;
                auto ds = std::make_unique<ctc_dataset>();
                ds->ctx = ctx;
                ds->p = q;
                for (int m = 0; m < 3; ++m) ds->dims[m] = train[0]->dims[m];
                ds->nnz_train = train[0]->nnz;
                if (q.precision == CTC_PREC_F64) build_dataset<double>(ds.get(), train, nullptr, nullptr);
                else build_dataset<float>(ds.get(), train, nullptr, nullptr);
                ctc_model mdl;
                mdl.nmodes = 3;
                mdl.rank = q.rank;
                for (int m = 0; m < 3; ++m) {
                    mdl.dims[m] = ds->dims[m];
                    mdl.U[m].resize(mdl.dims[m] * (uint64_t)q.rank);
                }
                if (ctc_model_init_uniform(&mdl, 12345, 1.0 / std::sqrt((double)q.rank)) != CTC_OK)
                    fail(CTC_E_ARG, "%s", ctc_last_error());
                SessionBase *S = session_for(ds.get(), q.rank);
                auto trial = [&](const TuneCand &c) {
                    q.threads_per_row = c.threads_per_row;
                    q.smem_budget = c.smem_budget;
                    q.sgd_atomic = c.sgd_atomic;
                    q.threads_per_block = c.threads_per_block;
                    ds->p = q;
                    S->set_params(q);
                    S->set_model(&mdl);
                    S->epochs(1);  // warm-up
                    CK(cudaEventRecord(ctx->ev0, ctx->stream));
                    S->epochs(2);
                    CK(cudaEventRecord(ctx->ev1, ctx->stream));
                    CK(cudaEventSynchronize(ctx->ev1));
                    float ms = 0;
                    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
                    const double per = ms / 2.0;
                    if (trials && nt < max_trials)
                        trials[nt] = ctc_tune_trial{c.tile_len, c.threads_per_row, c.smem_budget, per, 0,
                                                    c.sgd_atomic, c.threads_per_block};
                    ++nt;
                    return per;
                };
                TuneCand tile_best;
                double tile_ms = 1e300;
                for (const TuneCand &c : space) {
                    if (c.tile_len != tl) continue;
                    const double per = trial(c);
                    if (per < tile_ms) {
                        tile_ms = per;
                        tile_best = c;
                    }
                }
                // Hogwild SGD: the block size (the reference GA's other gene)
                // around this tile length's fastest candidate
                if (q.alg == CTC_ALG_SGD && q.sgd_order == CTC_SGD_HOGWILD)
                    for (int b : {128, 512, 1024}) {
                        TuneCand c = tile_best;
                        if (b == 1024 && (c.sgd_atomic != 3 || sgd_vectors_for(q.rank, c.threads_per_row) > 2))
                            continue;
                        c.threads_per_block = b;
                        const double per = trial(c);
                        if (per < tile_ms) {
                            tile_ms = per;
                            tile_best = c;
                        }
                    }
                if (tile_ms < best_ms) {
                    best_ms = tile_ms;
                    best = tile_best;
                }
                ds.reset();
            }
            if (!(flags & CTC_TUNE_NO_WRITE)) tune_write(cache_path, key, best, best_ms);
        }
        out->tile_len = best.tile_len;
        out->threads_per_row = best.threads_per_row;
        out->smem_budget = best.smem_budget;
        out->sgd_atomic = best.sgd_atomic;
        out->threads_per_block = best.threads_per_block;
        if (ntrials) *ntrials = nt;
    });
}
