// ciss_gpu.cu -- the reference's CISS layout (sgpu/ciss.c:68-195, the
// runtime-tile-length form of ga/ciss.c:69-212) built on the device,
// bit-exact with the host builder:
//   1. optional stable sort by (mode index, next mode index): two stable
//      radix-sort passes, the minor key first;
//   2. row starts f[m] = (im[m] != im[m-1]) and their inclusive prefix sum:
//      every nonzero's directory index;
//   3. directory / dcounter from the row starts;
//   4. the entries, one thread per layout row: a body row is the nonzero's
//      (j, k, value stored through an integer), a header row
//      [-dir index at the tile start, -last dir index changed to, bitmap] is
//      rebuilt from the same-row bits of the tile's nonzeros, the
//      terminator (-1, -1, -1) follows the last nonzero.
// Slots the host builder leaves unwritten are 0 here too, and the written
// mask is produced alongside (for ctc_ciss_export).
#include "ctc_internal.h"
#include "runtime.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace ctc {
namespace cg {

// sgpu/ciss.c:163 stores the value through an idx_t; the x86-64 conversion
// sequence: signed truncation below 2^63, offset and top-bit flip above,
// 0x8000000000000000 for NaN and out-of-range values
__device__ __forceinline__ double through_idx(double v)
{
    const double two63 = 9223372036854775808.0;
    uint64_t r;
    if (isnan(v) || v < -two63) {
        r = 0x8000000000000000ull;
    } else if (v < two63) {
        r = (uint64_t)(long long)v;
    } else {
        const double w = v - two63;
        r = ((w < two63) ? (uint64_t)(long long)w : 0x8000000000000000ull) ^ 0x8000000000000000ull;
    }
    return (double)r;
}

static __global__ void k_row_starts(const uint64_t *__restrict__ im, uint64_t n, uint32_t *__restrict__ f)
{
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < n; m += (uint64_t)gridDim.x * blockDim.x)
        f[m] = (m > 0 && im[m] != im[m - 1]) ? 1u : 0u;
}

static __global__ void k_directory(const uint64_t *__restrict__ im, const uint32_t *__restrict__ f,
                                   const uint32_t *__restrict__ rowid, uint64_t n, int ga,
                                   uint64_t *__restrict__ dir, uint64_t *__restrict__ dcounter)
{
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < n; m += (uint64_t)gridDim.x * blockDim.x) {
        if (m == 0) {
            dir[0] = im[0];
            dcounter[0] = 0;
        } else if (f[m]) {
            const uint32_t k = rowid[m];
            dir[k] = im[m];
            dcounter[k] = ga ? m : m - 1;
        }
    }
}

// one thread per layout row r = tile * (T + 1) + lc
static __global__ void k_entries(const uint64_t *__restrict__ im, const uint64_t *__restrict__ ij,
                                 const uint64_t *__restrict__ ik, const double *__restrict__ vals,
                                 const uint32_t *__restrict__ rowid, uint64_t n, int T, uint64_t rows,
                                 double *__restrict__ E, uint8_t *__restrict__ W)
{
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t tile = r / (uint64_t)(T + 1), lc = r % (uint64_t)(T + 1);
        const uint64_t first = tile * (uint64_t)T;
        double *e = E + 3 * r;
        uint8_t *w = W + 3 * r;
        if (first > n) continue;  // past the terminator's tile: unwritten
        if (lc > 0) {
            const uint64_t m = first + lc - 1;
            if (m < n) {
                e[0] = (double)ij[m];
                e[1] = (double)ik[m];
                e[2] = through_idx(vals[m]);
                w[0] = w[1] = w[2] = 1;
            } else if (m == n) {
                e[0] = e[1] = e[2] = -1.0;
                w[0] = w[1] = w[2] = 1;
            }
            continue;
        }
        // header: the directory index current at the tile start
        const uint64_t ns = tile == 0 ? 0 : rowid[first - 1];
        e[0] = -1.0 * (double)ns;
        w[0] = 1;
        const uint64_t last = min(first + (uint64_t)T, n);
        if (last > first) {
            uint64_t bitmap = 1;
            int64_t changed = -1;
            for (uint64_t m = first; m < last; ++m) {
                const bool same = (m == 0) || im[m] == im[m - 1];
                bitmap = (bitmap << 1) + (same ? 1u : 0u);
                if (!same) changed = (int64_t)m;
            }
            e[2] = (double)bitmap;
            w[2] = 1;
            if (changed >= 0) {
                e[1] = -1.0 * (double)rowid[changed];
                w[1] = 1;
            }
        }
    }
}

static __global__ void k_gather_u64(const uint32_t *__restrict__ perm, const uint64_t *__restrict__ in,
                                    uint64_t *__restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[perm[i]];
}

static __global__ void k_gather_f64(const uint32_t *__restrict__ perm, const double *__restrict__ in,
                                    double *__restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[perm[i]];
}

static __global__ void k_iota(uint32_t *__restrict__ p, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (uint32_t)i;
}

static __global__ void k_gather_key(const uint32_t *__restrict__ perm, const uint64_t *__restrict__ key,
                                    uint64_t *__restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = key[perm[i]];
}

}  // namespace cg

static void ciss_build_gpu(ctc_ctx *ctx, const ctc_tensor &t, int mode, int T, bool ga, bool sort, ctc_ciss &c)
{
    if (t.nmodes != 3) fail(CTC_E_UNSUP, "CISS needs an order-3 tensor (got %d)", t.nmodes);
    if (t.nnz == 0) fail(CTC_E_ARG, "CISS of an empty tensor");
    if (T < 1 || T > 64) fail(CTC_E_ARG, "tile length %d outside [1, 64]", T);
    if (mode < 0 || mode > 2) fail(CTC_E_ARG, "mode %d outside [0, 2]", mode);
    const uint64_t n = t.nnz;
    if (n >= 0x7fffffffull) fail(CTC_E_UNSUP, "more than 2^31 nonzeros");
    const int m1 = (mode + 1) % 3, m2 = (mode + 2) % 3;
    DevBuf<uint64_t> im, ij, ik;
    DevBuf<double> v;
    auto up = [&](DevBuf<uint64_t> &d, const uint64_t *src) {
        d.alloc(n);
        upload_filled(ctx, d.p, n, [&](uint64_t b, uint64_t e, uint64_t *h) { memcpy(h, src + b, (e - b) * 8); });
    };
    up(im, t.ind[mode].data());
    up(ij, t.ind[m1].data());
    up(ik, t.ind[m2].data());
    v.alloc(n);
    upload_filled(ctx, v.p, n, [&](uint64_t b, uint64_t e, double *h) { memcpy(h, t.vals.data() + b, (e - b) * 8); });
    const unsigned g = grid_for(n, 256, kSMs * 16);
    if (sort) {
        // stable by (im, ij), ties in input order: LSD radix passes, minor key first
        DevBuf<uint32_t> pa, pb;
        DevBuf<uint64_t> ka, kb;
        pa.alloc(n);
        pb.alloc(n);
        ka.alloc(n);
        kb.alloc(n);
        LAUNCH(ctx, cg::k_iota, g, 256, 0, pa.p, n);
        size_t tmp = 0, tmp2 = 0;
        CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ij.p, ka.p, pa.p, pb.p, (int)n, 0, 64, ctx->stream));
        DevBuf<unsigned char> scratch;
        scratch.alloc(tmp);
        CK(cub::DeviceRadixSort::SortPairs(scratch.p, tmp, ij.p, ka.p, pa.p, pb.p, (int)n, 0, 64, ctx->stream));
        // major key in the order of the first pass
        LAUNCH(ctx, cg::k_gather_key, g, 256, 0, (const uint32_t *)pb.p, (const uint64_t *)im.p, ka.p, n);
        CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp2, ka.p, kb.p, pb.p, pa.p, (int)n, 0, 64, ctx->stream));
        if (tmp2 > tmp) scratch.alloc(tmp2);
        size_t avail = std::max(tmp, tmp2);
        CK(cub::DeviceRadixSort::SortPairs(scratch.p, avail, ka.p, kb.p, pb.p, pa.p, (int)n, 0, 64, ctx->stream));
        scratch.release();
        // pa: the sorted order; gather all four arrays
        DevBuf<uint64_t> tmpu;
        tmpu.alloc(n);
        for (DevBuf<uint64_t> *d : {&im, &ij, &ik}) {
            LAUNCH(ctx, cg::k_gather_u64, g, 256, 0, (const uint32_t *)pa.p, (const uint64_t *)d->p, tmpu.p, n);
            std::swap(d->p, tmpu.p);
        }
        DevBuf<double> tmpv;
        tmpv.alloc(n);
        LAUNCH(ctx, cg::k_gather_f64, g, 256, 0, (const uint32_t *)pa.p, (const double *)v.p, tmpv.p, n);
        std::swap(v.p, tmpv.p);
    }
    DevBuf<uint32_t> f, rowid;
    f.alloc(n);
    rowid.alloc(n);
    LAUNCH(ctx, cg::k_row_starts, g, 256, 0, (const uint64_t *)im.p, n, f.p);
    {
        size_t tmp = 0;
        CK(cub::DeviceScan::InclusiveSum(nullptr, tmp, f.p, rowid.p, (int)n, ctx->stream));
        DevBuf<unsigned char> scratch;
        scratch.alloc(tmp);
        CK(cub::DeviceScan::InclusiveSum(scratch.p, tmp, f.p, rowid.p, (int)n, ctx->stream));
    }
    uint32_t lastid = 0;
    CK(cudaMemcpyAsync(&lastid, rowid.p + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const uint64_t dlength = (uint64_t)lastid + 1;
    DevBuf<uint64_t> dir, dcnt;
    dir.alloc(dlength);
    dcnt.alloc(dlength + 1);
    LAUNCH(ctx, cg::k_directory, g, 256, 0, (const uint64_t *)im.p, (const uint32_t *)f.p,
           (const uint32_t *)rowid.p, n, ga ? 1 : 0, dir.p, dcnt.p);
    const uint64_t last = n - 1;
    CK(cudaMemcpyAsync(dcnt.p + dlength, &last, sizeof(uint64_t), cudaMemcpyHostToDevice, ctx->stream));
    const uint64_t tilesize = n / (uint64_t)T + 1;
    const uint64_t size_rows = tilesize + n + 1;
    DevBuf<double> E;
    DevBuf<uint8_t> W;
    E.alloc(size_rows * 3);
    W.alloc(size_rows * 3);
    CK(cudaMemsetAsync(E.p, 0, size_rows * 3 * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(W.p, 0, size_rows * 3, ctx->stream));
    LAUNCH(ctx, cg::k_entries, grid_for(size_rows, 256, kSMs * 16), 256, 0, (const uint64_t *)im.p,
           (const uint64_t *)ij.p, (const uint64_t *)ik.p, (const double *)v.p, (const uint32_t *)rowid.p, n, T,
           size_rows, E.p, W.p);
    c.nnz = n;
    c.tile_len = T;
    c.dlength = dlength;
    c.size_rows = size_rows;
    c.directory.resize(dlength);
    c.dcounter.resize(dlength + 1);
    c.entries.resize(size_rows * 3);
    c.written.resize(size_rows * 3);
    CK(cudaMemcpyAsync(c.directory.data(), dir.p, dlength * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(c.dcounter.data(), dcnt.p, (dlength + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    // the layout and the written mask come back through the pinned double
    // buffer, drained into the (not yet touched) host arrays on the host
    // threads while the next chunk copies
    double *ent = c.entries.data();
    uint8_t *wr = c.written.data();
    download_drained(ctx, (const double *)E.p, size_rows * 3,
                     [&](uint64_t b, uint64_t e, const double *h) { memcpy(ent + b, h, (e - b) * sizeof(double)); });
    download_drained(ctx, (const uint8_t *)W.p, size_rows * 3,
                     [&](uint64_t b, uint64_t e, const uint8_t *h) { memcpy(wr + b, h, e - b); });
    CK(cudaStreamSynchronize(ctx->stream));
}

}  // namespace ctc

extern "C" int ctc_ciss_build_gpu(ctc_ctx *ctx, const ctc_tensor *t, int mode, int tile_len, int flags,
                                  ctc_ciss **out)
{
    using namespace ctc;
    return guarded([&] {
        if (!ctx || !t || !out) fail(CTC_E_ARG, "null argument");
        CK(cudaSetDevice(ctx->device));
        auto c = std::make_unique<ctc_ciss>();
        ciss_build_gpu(ctx, *t, mode - 1, tile_len, (flags & CTC_CISS_GA) != 0, (flags & CTC_CISS_SORT) != 0, *c);
        *out = c.release();
    });
}
