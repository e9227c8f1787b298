// ctc_internal.h -- internal types of libctc (host side).
#pragma once

#include "ctc.h"

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <functional>
#include <memory>
#include <utility>
#include <vector>

namespace ctc {

// An error carried to the C ABI boundary as (code, message).
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const char *fmt, ...);
void set_last_error(const char *msg);

// Runs fn, converting exceptions into a status code + ctc_last_error().
template <typename F>
int guarded(F &&fn)
{
    try {
        fn();
        return CTC_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return CTC_E_NOMEM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return CTC_E_ARG;
    }
}

// Number of host threads used by the parallel host passes.
int host_threads();
// task(0 .. ntasks-1) on the persistent host workers and the calling thread
void host_run(int ntasks, const std::function<void(int)> &task);

// Row-aligned work tiles over one mode-sorted copy of the nonzeros.
//   light tile: whole rows packed up to `tile_len` nonzeros (heavy == -1)
//   heavy piece: `tile_len` nonzeros of a row longer than tile_len
//                (heavy = index of that row in `heavy_rows`)
struct TilePlan {
    std::vector<int32_t> tiles;       // 4 ints per tile: start, len, heavy, piece
    std::vector<uint32_t> heavy_rows; // 4 uints per heavy row: row, first_tile, ntiles, 0
    uint32_t ntiles() const { return (uint32_t)(tiles.size() / 4); }
    uint32_t nheavy() const { return (uint32_t)(heavy_rows.size() / 4); }
};
TilePlan plan_tiles_chunked(const uint64_t *ind, uint64_t n, uint32_t tile_len, bool *unsorted);
// heavy_min: rows longer than this get tiles of their own (pieces of at
// most tile_len); 0 means tile_len, the planners' common rule
TilePlan plan_tiles_runs(const uint32_t *rows, const uint32_t *counts, uint64_t nruns, uint32_t tile_len,
                         uint32_t heavy_min = 0);

// FP64 gradient of the masked CP loss for order-3/4 tensors (fo.cu)
void ctc_grad_fo(ctc_ctx *ctx, const ctc_tensor *t, const ctc_model *model, double lambda, double *const *grads,
                 double *obj);

// Reference warp-kernel multiplicity of each nonzero (see ciss.cpp).
void compat_weights(const ctc_ciss &c, int kernel, std::vector<double> &w);

}  // namespace ctc

struct ctc_tensor {
    int nmodes = 0;
    uint64_t nnz = 0;
    uint64_t dims[4] = {0, 0, 0, 0};
    std::vector<uint64_t> ind[4];
    std::vector<double> vals;
};

namespace ctc {
// An allocator whose value-less construct leaves the element uninitialised:
// vectors that are filled right after resize (in parallel, or by a
// device-to-host copy) skip a serial zero fill.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept
    {
    }
    template <typename U>
    void construct(U *p) noexcept
    {
        ::new ((void *)p) U;
    }
    template <typename U, typename... A>
    void construct(U *p, A &&...a)
    {
        ::new ((void *)p) U(std::forward<A>(a)...);
    }
};
}  // namespace ctc

struct ctc_ciss {
    uint64_t nnz = 0, dlength = 0, size_rows = 0;
    int tile_len = 32;
    std::vector<uint64_t> directory, dcounter;
    std::vector<double, ctc::NoInitAlloc<double>> entries;  // every slot is written by the builders
    std::vector<uint8_t, ctc::NoInitAlloc<uint8_t>> written;
};

struct ctc_model {
    int nmodes = 0;
    int rank = 0;
    uint64_t dims[4] = {0, 0, 0, 0};
    std::vector<double> U[4];  // row-major dims[m] x rank
};
