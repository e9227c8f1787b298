// stage_gpu.cu -- the mode copies made on the device from one upload of
// the training records (16 bytes per nonzero): a stable radix sort gives
// the (mode m, mode m+1) order of ctc_tensor_sort, a run-length encoding
// of the rows feeds the host's tile planner (plan_tiles_runs, which makes
// the plan plan_tiles_chunked makes from the index array), and one gather
// lays out the CCD++ slots or the record copy.  The host reads each
// training tensor once instead of once per copy and phase.
#include "stage_gpu.h"

#include "ctc_internal.h"
#include "runtime.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>

namespace ctc {
namespace sg {

constexpr uint64_t kPadKey = ~0ull;

__device__ __forceinline__ uint32_t field(const uint4 &r, int m) { return m == 0 ? r.x : (m == 1 ? r.y : r.z); }

static __global__ void k_order_keys(const uint4 *__restrict__ rec, uint32_t n, int k0, int k1, int k2, int b1,
                                    int b2, uint64_t *__restrict__ keys, uint32_t *__restrict__ ids)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 r = rec[i];
        uint64_t key = ((uint64_t)field(r, k0) << (b1 + b2)) | ((uint64_t)field(r, k1) << b2);
        if (b2) key |= field(r, k2);
        keys[i] = key;
        ids[i] = i;
    }
}

static __global__ void k_check_sorted(const uint4 *__restrict__ rec, uint32_t n, int m, int *__restrict__ unsorted)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x + 1; i < n; i += gridDim.x * blockDim.x)
        if (field(rec[i], m) < field(rec[i - 1], m)) *unsorted = 1;
}

static __global__ void k_rows_in_order(const uint4 *__restrict__ rec, const uint32_t *__restrict__ perm, uint32_t n,
                                       int m, uint32_t *__restrict__ rows, int *__restrict__ unsorted)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t row = field(rec[perm ? perm[i] : i], m);
        rows[i] = row;
        if (!perm && i > 0 && row < field(rec[i - 1], m)) *unsorted = 1;
    }
}

template <typename T>
__global__ void k_fill_slots(const uint4 *__restrict__ rec, const double *__restrict__ v64,
                             const uint32_t *__restrict__ perm, int m, const int4 *__restrict__ tiles,
                             uint64_t nslots, int eshift, uint32_t s_row, uint32_t s_q1, uint32_t s_q2,
                             uint64_t *__restrict__ keys, T *__restrict__ x)
{
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
    const int sshift = 5 + eshift;
    const uint64_t smask = (1ull << sshift) - 1;
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslots;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t o = s & smask;
        const uint32_t q = (uint32_t)(((o & 31) << eshift) | (o >> 5));
        const int4 t = tiles[s >> sshift];
        uint64_t key = kPadKey;
        T v = T(0);
        if (q < (uint32_t)t.y) {
            const uint32_t p = (uint32_t)t.x + q;
            const uint32_t j = perm ? perm[p] : p;
            const uint4 r = rec[j];
            key = ((uint64_t)field(r, m) << s_row) | ((uint64_t)field(r, m1) << s_q1) |
                  ((uint64_t)field(r, m2) << s_q2);
            if constexpr (sizeof(T) == 8) v = v64[j];
            else v = __uint_as_float(r.w);
        }
        keys[s] = key;
        x[s] = v;
    }
}

static __global__ void k_gather_records(const uint4 *__restrict__ rec, const double *__restrict__ v64,
                                        const uint32_t *__restrict__ perm, uint32_t n, uint4 *__restrict__ out,
                                        double *__restrict__ v64_out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t j = perm[i];
        out[i] = rec[j];
        if (v64) v64_out[i] = v64[j];
    }
}

// per-block histogram in shared memory, added to the global counts
static __global__ void k_row_hist_smem(const uint4 *__restrict__ rec, uint32_t n, int m, uint32_t dim,
                                       uint32_t *__restrict__ counts)
{
    extern __shared__ uint32_t hist[];
    for (uint32_t r = threadIdx.x; r < dim; r += blockDim.x) hist[r] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&hist[field(rec[i], m)], 1u);
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < dim; r += blockDim.x)
        if (hist[r]) atomicAdd(&counts[r], hist[r]);
}

// global counts; lanes of a warp with the same row add once
static __global__ void k_row_hist_global(const uint4 *__restrict__ rec, uint32_t n, int m,
                                         uint32_t *__restrict__ counts)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) - lane; base < n; base += stride) {
        const uint64_t i = base + lane;
        const bool valid = i < n;
        const unsigned active = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const uint32_t row = field(rec[i], m);
            const unsigned peers = __match_any_sync(active, row);
            if ((int)lane == __ffs(peers) - 1) atomicAdd(&counts[row], (uint32_t)__popc(peers));
        }
    }
}

}  // namespace sg

void dev_sort_order(ctc_ctx *ctx, const uint4 *rec, uint32_t n, const int k[3], const int b[3], uint32_t *perm)
{
    const int end_bit = b[0] + b[1] + b[2];
    if (end_bit > 64) fail(CTC_E_UNSUP, "sort keys need %d bits (> 64) for these dimensions", end_bit);
    DevBuf<uint64_t> k_in, k_out;
    DevBuf<uint32_t> ids;
    k_in.alloc(n);
    k_out.alloc(n);
    ids.alloc(n);
    LAUNCH(ctx, sg::k_order_keys, grid_for(n, 256, kSMs * 16), 256, 0, rec, n, k[0], k[1], k[2], b[1], b[2], k_in.p,
           ids.p);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, k_in.p, k_out.p, ids.p, perm, (int)n, 0, end_bit,
                                       ctx->stream));
    DevBuf<unsigned char> scratch;
    scratch.alloc(tmp);
    CK(cub::DeviceRadixSort::SortPairs(scratch.p, tmp, k_in.p, k_out.p, ids.p, perm, (int)n, 0, end_bit,
                                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
}

bool dev_unsorted(ctc_ctx *ctx, const uint4 *rec, uint32_t n, int m)
{
    DevBuf<int> flag;
    flag.alloc(1);
    CK(cudaMemsetAsync(flag.p, 0, sizeof(int), ctx->stream));
    LAUNCH(ctx, sg::k_check_sorted, grid_for(n, 256, kSMs * 16), 256, 0, rec, n, m, flag.p);
    int h = 0;
    CK(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return h != 0;
}

bool dev_row_runs(ctc_ctx *ctx, const uint4 *rec, const uint32_t *perm, uint32_t n, int m,
                  std::vector<uint32_t> &rows, std::vector<uint32_t> &counts)
{
    DevBuf<uint32_t> in, uniq, cnt;
    DevBuf<int> flags;  // [0] unsorted, [1] number of runs
    in.alloc(n);
    uniq.alloc(n);
    cnt.alloc(n);
    flags.alloc(2);
    CK(cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), ctx->stream));
    LAUNCH(ctx, sg::k_rows_in_order, grid_for(n, 256, kSMs * 16), 256, 0, rec, perm, n, m, in.p, flags.p);
    size_t tmp = 0;
    CK(cub::DeviceRunLengthEncode::Encode(nullptr, tmp, in.p, uniq.p, cnt.p, flags.p + 1, (int)n, ctx->stream));
    DevBuf<unsigned char> scratch;
    scratch.alloc(tmp);
    CK(cub::DeviceRunLengthEncode::Encode(scratch.p, tmp, in.p, uniq.p, cnt.p, flags.p + 1, (int)n, ctx->stream));
    int h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, flags.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const size_t nr = (size_t)std::max(h[1], 0);
    rows.resize(nr);
    counts.resize(nr);
    if (nr) {
        CK(cudaMemcpyAsync(rows.data(), uniq.p, nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(counts.data(), cnt.p, nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return h[0] != 0;
}

template <typename T>
void dev_fill_slots(ctc_ctx *ctx, const uint4 *rec, const double *v64, const uint32_t *perm, int m,
                    const int4 *tiles, uint64_t nslots, int eshift, uint32_t s_row, uint32_t s_q1, uint32_t s_q2,
                    uint64_t *keys, T *x)
{
    LAUNCH(ctx, sg::k_fill_slots<T>, grid_for(nslots, 256, kSMs * 16), 256, 0, rec, v64, perm, m, tiles, nslots,
           eshift, s_row, s_q1, s_q2, keys, x);
}
template void dev_fill_slots<float>(ctc_ctx *, const uint4 *, const double *, const uint32_t *, int, const int4 *,
                                    uint64_t, int, uint32_t, uint32_t, uint32_t, uint64_t *, float *);
template void dev_fill_slots<double>(ctc_ctx *, const uint4 *, const double *, const uint32_t *, int, const int4 *,
                                     uint64_t, int, uint32_t, uint32_t, uint32_t, uint64_t *, double *);

void dev_gather_records(ctc_ctx *ctx, const uint4 *rec, const double *v64, const uint32_t *perm, uint32_t n,
                        uint4 *out, double *v64_out)
{
    LAUNCH(ctx, sg::k_gather_records, grid_for(n, 256, kSMs * 16), 256, 0, rec, v64, perm, n, out, v64_out);
}

void dev_row_counts(ctc_ctx *ctx, const uint4 *rec, uint32_t n, int m, uint32_t dim, std::vector<uint32_t> &counts)
{
    DevBuf<uint32_t> c;
    c.alloc(dim);
    CK(cudaMemsetAsync(c.p, 0, (size_t)dim * sizeof(uint32_t), ctx->stream));
    constexpr uint32_t kSmemRows = 40960;  // 160 KiB of shared counters
    if (dim <= kSmemRows) {
        const size_t smem = (size_t)dim * sizeof(uint32_t);
        if (smem > 48 * 1024)
            CK(cudaFuncSetAttribute(sg::k_row_hist_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        LAUNCH(ctx, sg::k_row_hist_smem, grid_for(n, 1024, kSMs), 1024, smem, rec, n, m, dim, c.p);
    } else {
        LAUNCH(ctx, sg::k_row_hist_global, grid_for(n, 256, kSMs * 8), 256, 0, rec, n, m, c.p);
    }
    counts.resize(dim);
    CK(cudaMemcpyAsync(counts.data(), c.p, (size_t)dim * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
}

}  // namespace ctc
