// runtime.cuh -- host-side runtime shared by the library's CUDA sources:
// CUDA error checks, device buffers, host parallel loops, the context
// (stream, events, reduction scratch, pinned staging buffers), timed kernel
// launches (LAUNCH), and host-to-device staging through pinned memory.
#pragma once

#include "ctc_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#if defined(__SSE2__)
#include <emmintrin.h>
#endif

namespace ctc {

static void check_cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        // clear a non-sticky error so that it is not reported again by the
        // next launch check of an unrelated call
        (void)cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? CTC_E_NOMEM : CTC_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
}
#define CK(x) check_cuda((x), #x)

// Device memory of the library comes from one stream-ordered pool per
// device that keeps freed blocks (release threshold: unlimited), so that
// datasets, sessions and staging scratch that come and go reuse mapped
// memory instead of mapping and unmapping gigabytes on every call.
// dev_alloc returns a block ready for use on any stream; dev_free first
// waits for the device, as cudaFree does, so that a block is idle before
// the pool hands it out again.  (Defined once, in engine.cu.)
void *dev_alloc(size_t bytes);
void dev_free(void *p) noexcept;
// unused pool memory back to the driver
void dev_pool_trim() noexcept;

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) dev_free(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count)
    {
        release();
        if (count == 0) count = 1;
        p = static_cast<T *>(dev_alloc(count * sizeof(T)));
        n = count;
    }
    void ensure(size_t count)
    {
        if (n < count) alloc(count);
    }
    void swap(DevBuf &o)
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
    void upload(const T *h, size_t count, cudaStream_t s)
    {
        ensure(count);
        if (count) CK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

template <typename F>
static void par_for(uint64_t n, F &&fn)
{
    int P = host_threads();
    if (n < 65536 || P == 1) {
        fn((uint64_t)0, n);
        return;
    }
    const std::function<void(int)> task = [&](int p) { fn(n * p / P, n * (p + 1) / P); };
    host_run(P, task);
}

template <typename F>
static void with_rank(int R, F &&f)
{
    switch (R) {
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    case 32: f(std::integral_constant<int, 32>{}); break;
    case 64: f(std::integral_constant<int, 64>{}); break;
    default: fail(CTC_E_UNSUP, "rank %d not supported (8, 16, 32, 64)", R);
    }
}

constexpr int kSMs = 148;
constexpr int kMaxPartials = kSMs * 8;
constexpr int kScalars = 16;

// CTC_TRACE=1 in the environment prints the host staging phases' wall
// times to stderr
static bool trace_on()
{
    static const bool on = [] {
        const char *e = getenv("CTC_TRACE");
        return e && *e && *e != '0';
    }();
    return on;
}

struct TracePhase {
    const char *what;
    std::chrono::steady_clock::time_point t0;
    explicit TracePhase(const char *w) : what(w), t0(std::chrono::steady_clock::now()) {}
    ~TracePhase()
    {
        if (trace_on())
            fprintf(stderr, "[ctc] %-28s %8.3f s\n", what,
                    std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
};

static unsigned grid_for(uint64_t work, unsigned per_block, unsigned cap)
{
    uint64_t g = (work + per_block - 1) / per_block;
    if (g < 1) g = 1;
    return (unsigned)std::min<uint64_t>(g, cap);
}

// per-kernel device time, from an event pair around every launch
struct KernelTimes {
    bool on = false;
    std::vector<std::pair<const char *, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
    std::map<std::string, std::pair<uint64_t, double>> acc;  // name -> (count, ms)
    size_t used = 0;
};

}  // namespace ctc

using namespace ctc;

struct ctc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DevBuf<double> partial;   // per-block reduction partials
    DevBuf<double> scalars;   // reduction results
    double *h_scalars = nullptr;  // pinned mirror
    bool capturing = false;
    KernelTimes kt;
    // pinned double buffer for host-to-device staging (first use allocates)
    unsigned char *pin[2] = {nullptr, nullptr};
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};
};

namespace ctc {

// Host-to-device staging through the context's pinned double buffer:
// fill(b, e, h) writes elements [b, e) of the device array to h (pinned
// host memory, element b at h[0]); the copy of one chunk runs while the
// next one is filled on the host threads.
constexpr size_t kPinBytes = (size_t)32 << 20;

// 16 bytes into pinned staging memory (16-byte aligned) with a streaming
// store where the host has one: the staging buffers are written once and
// then read by the copy engine, so a normal store's fetch of the line it
// is about to overwrite is wasted host memory traffic.  A thread that
// streamed calls stream_fence() before its data may be copied.
static inline void stream_store16(void *dst, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
#if defined(__SSE2__)
    _mm_stream_si128(reinterpret_cast<__m128i *>(dst), _mm_set_epi32((int)d, (int)c, (int)b, (int)a));
#else
    const uint32_t v[4] = {a, b, c, d};
    memcpy(dst, v, sizeof(v));
#endif
}

static inline void stream_fence()
{
#if defined(__SSE2__)
    _mm_sfence();
#endif
}

static void ensure_pinned(ctc_ctx *ctx)
{
    if (!ctx->pin[0])
        for (int q = 0; q < 2; ++q) {
            CK(cudaMallocHost(&ctx->pin[q], kPinBytes));
            CK(cudaEventCreateWithFlags(&ctx->pin_ev[q], cudaEventDisableTiming));
        }
}

template <typename E, typename F>
static void upload_filled(ctc_ctx *ctx, E *dev, uint64_t n, F &&fill)
{
    ensure_pinned(ctx);
    const uint64_t per = kPinBytes / sizeof(E);
    int q = 0;
    for (uint64_t b = 0; b < n; b += per, q ^= 1) {
        const uint64_t e = std::min(n, b + per);
        CK(cudaEventSynchronize(ctx->pin_ev[q]));  // this buffer's previous copy is done
        E *h = reinterpret_cast<E *>(ctx->pin[q]);
        par_for(e - b, [&](uint64_t i0, uint64_t i1) { fill(b + i0, b + i1, h + i0); });
        CK(cudaMemcpyAsync(dev + b, h, (e - b) * sizeof(E), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaEventRecord(ctx->pin_ev[q], ctx->stream));
    }
}

// Device-to-host through the same pinned double buffer: consume(b, e, h)
// reads elements [b, e) of the device array from h (element b at h[0]) on
// the host threads while the copy of the next chunk runs.
template <typename E, typename F>
static void download_drained(ctc_ctx *ctx, const E *dev, uint64_t n, F &&consume)
{
    ensure_pinned(ctx);
    const uint64_t per = kPinBytes / sizeof(E);
    const uint64_t nch = (n + per - 1) / per;
    auto issue = [&](uint64_t c) {
        const int q = (int)(c & 1);
        const uint64_t b = c * per, e = std::min(n, b + per);
        CK(cudaEventSynchronize(ctx->pin_ev[q]));  // an earlier copy through this buffer is done
        CK(cudaMemcpyAsync(ctx->pin[q], dev + b, (e - b) * sizeof(E), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaEventRecord(ctx->pin_ev[q], ctx->stream));
    };
    if (nch) issue(0);
    for (uint64_t c = 0; c < nch; ++c) {
        if (c + 1 < nch) issue(c + 1);
        const int q = (int)(c & 1);
        const uint64_t b = c * per, e = std::min(n, b + per);
        CK(cudaEventSynchronize(ctx->pin_ev[q]));
        const E *h = reinterpret_cast<const E *>(ctx->pin[q]);
        par_for(e - b, [&](uint64_t i0, uint64_t i1) { consume(b + i0, b + i1, h + i0); });
    }
}

static void kt_flush(ctc_ctx *ctx)
{
    KernelTimes &k = ctx->kt;
    if (k.pending.empty()) return;
    CK(cudaStreamSynchronize(ctx->stream));
    for (auto &pe : k.pending) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, pe.second.first, pe.second.second));
        auto &a = k.acc[pe.first];
        a.first += 1;
        a.second += ms;
    }
    k.pending.clear();
    k.used = 0;
}

template <typename Kern, typename... Args>
static void launch_named(ctc_ctx *ctx, const char *name, Kern kern, dim3 grid, dim3 block, size_t smem,
                         Args... args)
{
    KernelTimes &k = ctx->kt;
    const bool timed = k.on && !ctx->capturing;
    std::pair<cudaEvent_t, cudaEvent_t> ev{};
    if (timed) {
        if (k.used >= 4096) kt_flush(ctx);
        if (k.used == k.pool.size()) {
            cudaEvent_t a, b;
            CK(cudaEventCreate(&a));
            CK(cudaEventCreate(&b));
            k.pool.push_back({a, b});
        }
        ev = k.pool[k.used++];
        CK(cudaEventRecord(ev.first, ctx->stream));
    }
    kern<<<grid, block, smem, ctx->stream>>>(args...);
    ctx->launches++;
    CK(cudaGetLastError());
    if (timed) {
        CK(cudaEventRecord(ev.second, ctx->stream));
        k.pending.push_back({name, ev});
    }
}
#define LAUNCH(ctx, kern, ...) launch_named(ctx, #kern, kern, __VA_ARGS__)

}  // namespace ctc
