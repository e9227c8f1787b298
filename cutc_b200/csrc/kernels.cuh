// kernels.cuh -- sm_100a kernels of the completion engine.
//
// Data layout in HBM (one copy of the training nonzeros per mode, sorted
// for that mode, the order of the reference's traina/b/c files):
//   rec[n]  : uint4 {i0, i1, i2, value bits}  -- 16 B, one 128-bit load per
//             nonzero; indices 0-based; the value is FP32 (in FP64 runs it
//             lives in v64[n] instead, and CCD++ keeps its residual there)
//   tiles[t]: int4 {start, len, heavy, piece}  -- row-aligned work tiles:
//             whole rows packed to <= tile_len nonzeros (heavy = -1), or one
//             tile_len piece of a longer row (heavy = its heavy-row id)
//   heavy[h]: uint4 {row, first_tile, ntiles, 0}
// A warp owns a tile: rows inside a light tile are reduced and finalised by
// that warp alone (no atomics); pieces of heavy rows write per-tile partials
// that a fixup kernel sums in piece order (deterministic).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "ptx.cuh"

namespace ctc {
namespace k {

constexpr uint32_t kNoKey = 0xffffffffu;

template <typename T>
struct Vec;
template <>
struct Vec<float> {
    using type = float4;
    static constexpr int n = 4;
};
template <>
struct Vec<double> {
    using type = double2;
    static constexpr int n = 2;
};

__device__ __forceinline__ float vget(const float4 &v, int i)
{
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}
__device__ __forceinline__ double vget(const double2 &v, int i) { return i == 0 ? v.x : v.y; }
__device__ __forceinline__ void vset(float4 &v, int i, float x)
{
    if (i == 0) v.x = x;
    else if (i == 1) v.y = x;
    else if (i == 2) v.z = x;
    else v.w = x;
}
__device__ __forceinline__ void vset(double2 &v, int i, double x)
{
    if (i == 0) v.x = x;
    else v.y = x;
}

__device__ __forceinline__ uint32_t key_of(const uint4 &r, int m)
{
    return m == 0 ? r.x : (m == 1 ? r.y : r.z);
}

template <typename T>
__device__ __forceinline__ T value_of(const uint4 &r, const double *v64, uint64_t n)
{
    if constexpr (sizeof(T) == 8) return v64[n];
    else return __uint_as_float(r.w);
}

template <typename T>
__device__ __forceinline__ void store_value(uint4 *rec, double *v64, uint64_t n, T v)
{
    if constexpr (sizeof(T) == 8) v64[n] = v;
    else rec[n].w = __float_as_uint(v);
}

__device__ __forceinline__ void vatomic_add(float4 *p, const float4 &d) { atomicAdd(p, d); }
__device__ __forceinline__ void vatomic_add(double2 *p, const double2 &d)
{
    atomicAdd(&p->x, d.x);
    atomicAdd(&p->y, d.y);
}

// Warp tasks claimed one at a time from a counter pair {next, done} that
// every launch leaves at zero: a warp claims indices until it draws one past
// the end, then counts itself done, and the last warp of the grid to finish
// zeroes both for the next launch on the stream.  Every warp of the grid
// calls finish() exactly once.  Warps that drew short tasks thus take more,
// where a fixed stride would leave the grid waiting on the unluckiest warp.
struct TaskClaim {
    unsigned int *ctr;
    // quarters of the tasks handed out on a fixed stride before any is
    // claimed (0: all claimed), for grids whose warps are all resident: the
    // stride takes part of them without an atomic, and the claimed rest
    // evens out the finish
    uint32_t stride_quarters;
    __device__ __forceinline__ uint32_t next(int lane) const
    {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(ctr, 1u);
        return __shfl_sync(0xffffffffu, t, 0);
    }
    __device__ __forceinline__ void finish(int lane) const
    {
        if (lane == 0) {
            const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
            __threadfence();  // this warp's claims come before its count
            if (atomicAdd(ctr + 1, 1u) == nwarps - 1u) {
                __threadfence();
                ctr[0] = 0u;
                ctr[1] = 0u;
            }
        }
    }
};

// A warp's task indices under a TaskClaim: its fixed-stride share first
// (warp, warp + nwarps, ... for stride_quarters / 4 of the tasks), then
// indices claimed after that share.  Warp-uniform.
struct WarpTaskSeq {
    TaskClaim c;
    uint32_t warp, nwarps, per, k, base;
    __device__ __forceinline__ WarpTaskSeq(const TaskClaim &tc, uint32_t ntasks) : c(tc), k(0)
    {
        warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        nwarps = (gridDim.x * blockDim.x) >> 5;
        per = (uint32_t)(((uint64_t)ntasks * tc.stride_quarters / 4u) / nwarps);
        base = per * nwarps;
    }
    __device__ __forceinline__ uint32_t next(int lane)
    {
        if (k < per) return warp + (k++) * nwarps;
        return base + c.next(lane);
    }
};

// Block-wide double sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = (l < nw) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

// ---------------------------------------------------------------------
// Squared error (the residual/RMSE kernel).  A warp takes 32 consecutive
// nonzeros with one coalesced 512-byte load of their records, then walks
// them GPW at a time: a group of GL = R / VN lanes per nonzero, lane gl
// reading the 16-byte slice gl of each of the three factor rows, so one
// warp load covers whole 64/128-byte rows instead of 32 scattered slices.
// The group's partial products meet in a butterfly; lane 0 of the group
// adds e^2 to its double accumulator.  Per-block double partials, folded
// in a fixed order afterwards, keep the result deterministic.
// ---------------------------------------------------------------------
template <typename T, int R>
__device__ __forceinline__ double sse_span(const uint4 *__restrict__ rec, const double *__restrict__ v64,
                                           uint64_t first, uint64_t end, uint64_t stride,
                                           const T *__restrict__ U0, const T *__restrict__ U1,
                                           const T *__restrict__ U2)
{
    using V = typename Vec<T>::type;
    constexpr int VN = Vec<T>::n;
    constexpr int GL = R / VN;
    static_assert(GL >= 1 && 32 % GL == 0, "lanes per nonzero");
    const int lane = threadIdx.x & 31;
    const int gl = lane % GL, gw = lane / GL;
    double acc = 0;
    // group gw takes the GL consecutive records gw*GL .. gw*GL+GL-1 of the
    // 32, so in a copy sorted by (mode 0, mode 1) it mostly sees one mode-0
    // row, and runs of one mode-1 row inside it: each row's slice stays in
    // registers until its index changes.  One record ahead took an
    // evaluation of the 100M workload from 2.11 to 2.02 ms; gathering for
    // four records before using any (80 registers) was slower, 2.61 ms.
    uint32_t cur0 = 0xffffffffu, cur1 = 0xffffffffu;
    V va{}, vb{};
    for (uint64_t base = first; base < end; base += stride) {
        const uint64_t mine = base + lane;
        uint4 r = make_uint4(0u, 0u, 0u, 0u);  // row 0 for the tail: in bounds, result unused
        T x = 0;
        if (mine < end) {
            r = rec[mine];
            x = value_of<T>(r, v64, mine);
        }
        const uint64_t cnt = end - base;
        // one record ahead: the slices of record j + 1 are loaded while
        // record j is multiplied
        auto fetch = [&](int src, V &a, V &b, V &c) {
            const uint32_t i0 = __shfl_sync(0xffffffffu, r.x, src);
            const uint32_t i1 = __shfl_sync(0xffffffffu, r.y, src);
            const uint32_t i2 = __shfl_sync(0xffffffffu, r.z, src);
            if (i0 != cur0) a = reinterpret_cast<const V *>(U0 + (size_t)i0 * R)[gl];
            if (i1 != cur1) b = reinterpret_cast<const V *>(U1 + (size_t)i1 * R)[gl];
            c = reinterpret_cast<const V *>(U2 + (size_t)i2 * R)[gl];
            cur0 = i0;
            cur1 = i1;
        };
        V na = va, nb = vb, nc;
        fetch(gw * GL, na, nb, nc);
#pragma unroll
        for (int j = 0; j < GL; ++j) {
            const int src = gw * GL + j;
            const T xv = __shfl_sync(0xffffffffu, x, src);
            const V a = na, b = nb, c = nc;
            if (j + 1 < GL) fetch(src + 1, na, nb, nc);
            T p = 0;
#pragma unroll
            for (int v = 0; v < VN; ++v) p += vget(a, v) * vget(b, v) * vget(c, v);
#pragma unroll
            for (int o = GL / 2; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
            if (gl == 0 && (uint64_t)src < cnt) {
                const T e = xv - p;
                acc += (double)e * (double)e;
            }
        }
        va = na;  // the slices of the rows cur0 / cur1 name
        vb = nb;
    }
    return acc;
}

template <typename T, int R>
__global__ void __launch_bounds__(256) k_sse(const uint4 *__restrict__ rec,
                                             const double *__restrict__ v64, uint32_t n,
                                             const T *__restrict__ U0, const T *__restrict__ U1,
                                             const T *__restrict__ U2, double *__restrict__ partial)
{
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    double acc = sse_span<T, R>(rec, v64, warp * 32, n, nwarps * 32, U0, U1, U2);
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Squared error over chunks that each lie inside one instance of a batch
// (chunk = {begin, end, instance, 0}): block per chunk, one double partial
// per chunk; k_fold_segments sums each instance's chunks in order.
template <typename T, int R>
__global__ void __launch_bounds__(256) k_sse_chunks(const uint4 *__restrict__ rec, const double *__restrict__ v64,
                                                    const uint4 *__restrict__ chunks, uint32_t nchunks,
                                                    const T *__restrict__ U0, const T *__restrict__ U1,
                                                    const T *__restrict__ U2, double *__restrict__ partial)
{
    const uint64_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const uint4 ch = chunks[c];
        double acc = sse_span<T, R>(rec, v64, ch.x + w * 32, ch.y, nw * 32, U0, U1, U2);
        acc = block_sum(acc);
        if (threadIdx.x == 0) partial[c] = acc;
        __syncthreads();  // block_sum's shared slots are reused by the next chunk
    }
}

// out = transpose of in: in is rows x cols row-major, out[c * rows + r] =
// in[r * cols + c].  32 x 32 tiles through shared memory (padded rows), so
// both the reads and the writes are coalesced; 32 x 8 threads per block,
// blocks over row tiles in x and (looping) column tiles in y.
template <typename T>
__global__ void __launch_bounds__(256) k_transpose(const T *__restrict__ in, uint64_t rows, uint64_t cols,
                                                   T *__restrict__ out)
{
    __shared__ T tile[32][33];
    const uint64_t r0 = (uint64_t)blockIdx.x * 32;
    for (uint64_t c0 = (uint64_t)blockIdx.y * 32; c0 < cols; c0 += (uint64_t)gridDim.y * 32) {
        for (int i = threadIdx.y; i < 32; i += 8) {
            const uint64_t r = r0 + i, c = c0 + threadIdx.x;
            if (r < rows && c < cols) tile[i][threadIdx.x] = in[r * cols + c];
        }
        __syncthreads();
        for (int i = threadIdx.y; i < 32; i += 8) {
            const uint64_t c = c0 + i, r = r0 + threadIdx.x;
            if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][i];
        }
        __syncthreads();
    }
}

// out[i] = sum of partial[first[i] .. first[i+1]) in order (thread per
// instance)
static __global__ void k_fold_segments(const double *__restrict__ partial, const uint32_t *__restrict__ first, int ninst,
                                double *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ninst; i += gridDim.x * blockDim.x) {
        double acc = 0;
        for (uint32_t c = first[i]; c < first[i + 1]; ++c) acc += partial[c];
        out[i] = acc;
    }
}

// Sum of squares of a dense array (for lambda * ||U||^2).
template <typename T>
__global__ void __launch_bounds__(256) k_sumsq(const T *__restrict__ x, uint64_t n,
                                               double *__restrict__ partial)
{
    double acc = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        acc += (double)x[i] * (double)x[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// out[slot] = sum of partial[0..n) in a fixed order (one block).
static __global__ void __launch_bounds__(256) k_sum_partials(const double *__restrict__ partial, int n,
                                                      double *__restrict__ out)
{
    double acc = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

// ---------------------------------------------------------------------
// SGD (sgpu/sgd.cu:21-143 rule).  A group of G = R/(VN*C) lanes handles one
// tile of consecutive mode-0-sorted nonzeros; each lane holds C 16-byte
// slices of the three rows (C is the "threads per row" knob: fewer lanes
// per nonzero put more nonzeros in flight per warp).
//   e = x - sum a.b.c ;  a += s*((e*b*c) - lambda*a) ; b, c likewise from
//   the pre-update rows, s = lr * step scale (times a per-row factor when
//   damping is on, see ctc_params.sgd_conflicts).
// sequential != 0: one group walks all tiles in order (deterministic); the
//   mode-0 row stays in registers while it does not change (exact there).
// Hogwild: groups run tiles concurrently, in a scattered tile order; each
//   nonzero reads its three rows fresh and adds its deltas atomically
//   (vector red.add), or stores the new rows (atomic == 0, lossy under
//   contention).  The next nonzero's record is fetched while the current
//   one is processed.
// ---------------------------------------------------------------------
template <typename T, int R, int C>
__global__ void __launch_bounds__(512) k_sgd(const uint4 *__restrict__ rec,
                                             const double *__restrict__ v64, uint32_t n,
                                             uint32_t tile_len, uint32_t ntiles, T *U0, T *U1,
                                             T *U2, const T *__restrict__ lr_dev, T lambda,
                                             int atomic, int sequential, uint64_t tile_stride,
                                             const float *__restrict__ damp0,
                                             const float *__restrict__ damp1,
                                             const float *__restrict__ damp2)
{
    using V = typename Vec<T>::type;
    constexpr int VN = Vec<T>::n;
    constexpr int G = R / (VN * C);
    static_assert(G >= 1 && G <= 32 && (32 % G) == 0 && G * VN * C == R, "unsupported rank / lanes");
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int gl = lane % G;
    const int gw = lane / G;
    const uint32_t gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (gw * G));
    uint64_t group = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * GPW + gw;
    uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x >> 5) * GPW;
    if (sequential) {
        if (group != 0) return;
        ngroups = 1;
    }
    const T s = *lr_dev;
    // atomic == 2 (FP32 Hogwild): a nonzero's three row deltas are staged in
    // the group's shared buffer (two of them, alternating) and added by
    // three bulk reductions of whole rows, issued by the group's lane 0
    extern __shared__ __align__(16) unsigned char sgd_smem[];
    const bool bulk = std::is_same<T, float>::value && atomic == 2 && !sequential;
    T *gbuf = reinterpret_cast<T *>(sgd_smem) + (size_t)((threadIdx.x >> 5) * GPW + gw) * (2 * 3 * R);
    uint32_t nstaged = 0;
    for (uint64_t t = group; t < ntiles; t += ngroups) {
        // Hogwild: tiles in flight together are spread over the tensor
        // (tile_stride is coprime to ntiles), so a long row of the sorted
        // mode is not updated by every group at once; sequential: stride 1
        const uint64_t tile = (t * tile_stride) % ntiles;
        const uint64_t start = tile * tile_len;
        const uint64_t end = min(start + tile_len, (uint64_t)n);
        uint32_t cur = kNoKey;
        V a[C], a0[C];
        V *arow = nullptr;
        uint4 rn = start < end ? rec[start] : make_uint4(0, 0, 0, 0);
        for (uint64_t p = start; p < end; ++p) {
            const uint4 r = rn;
            if (p + 1 < end) rn = rec[p + 1];
            const T x = value_of<T>(r, v64, p);
            if (!sequential) {
                // every row read fresh: the staleness of a hot row is bounded
                // by the updates in flight
                arow = reinterpret_cast<V *>(U0 + (size_t)r.x * R) + gl * C;
#pragma unroll
                for (int q = 0; q < C; ++q) a0[q] = a[q] = bulk ? __ldcg(arow + q) : arow[q];
            } else if (r.x != cur) {
                if (arow)
#pragma unroll
                    for (int q = 0; q < C; ++q) arow[q] = a[q];
                cur = r.x;
                arow = reinterpret_cast<V *>(U0 + (size_t)r.x * R) + gl * C;
#pragma unroll
                for (int q = 0; q < C; ++q) a[q] = arow[q];
            }
            V *brow = reinterpret_cast<V *>(U1 + (size_t)r.y * R) + gl * C;
            V *crow = reinterpret_cast<V *>(U2 + (size_t)r.z * R) + gl * C;
            V b[C], c[C];
            // bulk reductions are applied at L2 and leave stale lines in L1,
            // so that mode reads the rows from L2
#pragma unroll
            for (int q = 0; q < C; ++q) {
                b[q] = bulk ? __ldcg(brow + q) : brow[q];
                c[q] = bulk ? __ldcg(crow + q) : crow[q];
            }
            T part = 0;
#pragma unroll
            for (int q = 0; q < C; ++q)
#pragma unroll
                for (int v = 0; v < VN; ++v) part += vget(a[q], v) * vget(b[q], v) * vget(c[q], v);
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) part += __shfl_xor_sync(gmask, part, o);
            const T e = x - part;
            T sa = s, sb = s, sc = s;
            if (damp0) {
                sa *= (T)damp0[r.x];
                sb *= (T)damp1[r.y];
                sc *= (T)damp2[r.z];
            }
            T *buf = gbuf + (nstaged & 1) * (3 * R);
            if (bulk) {
                // the buffer staged two nonzeros ago has been read by its reductions
                if (gl == 0) px::bulk_wait_read<1>();
                __syncwarp(gmask);
            }
#pragma unroll
            for (int q = 0; q < C; ++q) {
                V an, db, dc;
#pragma unroll
                for (int v = 0; v < VN; ++v) {
                    const T av = vget(a[q], v), bv = vget(b[q], v), cv = vget(c[q], v);
                    vset(an, v, av + sa * ((e * bv * cv) - lambda * av));
                    vset(db, v, sb * ((e * av * cv) - lambda * bv));
                    vset(dc, v, sc * ((e * bv * av) - lambda * cv));
                }
                if (!sequential && atomic) {
                    V da;
#pragma unroll
                    for (int v = 0; v < VN; ++v) vset(da, v, vget(an, v) - vget(a0[q], v));
                    if (bulk) {
                        V *sb3 = reinterpret_cast<V *>(buf) + gl * C + q;
                        sb3[0] = da;
                        sb3[R / VN] = db;
                        sb3[2 * (R / VN)] = dc;
                    } else {
                        vatomic_add(arow + q, da);
                        vatomic_add(brow + q, db);
                        vatomic_add(crow + q, dc);
                    }
                } else {
                    V bn, cn;
#pragma unroll
                    for (int v = 0; v < VN; ++v) {
                        vset(bn, v, vget(b[q], v) + vget(db, v));
                        vset(cn, v, vget(c[q], v) + vget(dc, v));
                    }
                    if (!sequential) arow[q] = an;
                    brow[q] = bn;
                    crow[q] = cn;
                }
                a[q] = an;
            }
            if constexpr (std::is_same<T, float>::value) {
                if (bulk) {
                    px::fence_proxy_async_smem();
                    __syncwarp(gmask);
                    if (gl == 0) {
                        px::bulk_reduce_add_f32(U0 + (size_t)r.x * R, buf, R * sizeof(float));
                        px::bulk_reduce_add_f32(U1 + (size_t)r.y * R, buf + R, R * sizeof(float));
                        px::bulk_reduce_add_f32(U2 + (size_t)r.z * R, buf + 2 * R, R * sizeof(float));
                        px::bulk_commit();
                    }
                    ++nstaged;
                }
            }
        }
        if (sequential && arow)
#pragma unroll
            for (int q = 0; q < C; ++q) arow[q] = a[q];
    }
    if (bulk && gl == 0) px::bulk_wait_all();
}

// ---------------------------------------------------------------------
// Hogwild SGD with block-merged updates of the hot rows (FP32,
// sgd_atomic 3).  The most frequent kSgdHot rows of each mode are "hot";
// hot[p] codes the hot slots of nonzero p's three rows (10 bits per mode,
// kSgdCold when the row is not hot).  The block's groups advance in
// lockstep, one nonzero each per step: every group reads its three rows
// from global memory, adds the deltas of cold rows with vector atomics
// as k_sgd does, and adds the deltas of hot rows into the block's
// shared-memory accumulators; after the step the block adds each touched
// hot row's summed delta with one vector atomic per 16 bytes and clears
// it.  The nonzeros of one block step are thus applied as simultaneous
// Hogwild updates (each computed from the rows it read, their sum added),
// and a hot row receives one reduction per block step instead of one per
// nonzero: the same-address reductions queued at the L2 slice that holds
// it, behind which its readers wait, shrink by the number of the block's
// nonzeros that touch it.
// ---------------------------------------------------------------------
constexpr int kSgdHot = 32;          // hot rows per mode
constexpr uint32_t kSgdCold = 1023u; // slot code of a row that is not hot

// 1024-thread blocks for one or two 16-byte slices per lane (at most 64
// registers), 512 for four
template <int R, int C>
__global__ void __launch_bounds__(C <= 2 ? 1024 : 512) k_sgd_hot(const uint4 *__restrict__ rec, const uint32_t *__restrict__ hot,
                                                 uint32_t n, uint32_t tile_len, uint32_t ntiles, float *U0,
                                                 float *U1, float *U2, const float *__restrict__ lr_dev, float lambda,
                                                 uint64_t tile_stride, const float *__restrict__ damp0,
                                                 const float *__restrict__ damp1, const float *__restrict__ damp2,
                                                 const uint32_t *__restrict__ hot_rows)
{
    constexpr int VN = 4;
    constexpr int G = R / (VN * C);
    static_assert(G >= 1 && G <= 32 && (32 % G) == 0 && G * VN * C == R, "unsupported rank / lanes");
    constexpr int GPW = 32 / G;
    constexpr int NV = R / VN;  // float4 per row
    __shared__ __align__(16) float4 acc[3 * kSgdHot * NV];
    // bit s of touched[p][m]: slot s of mode m got a delta in a step of parity p
    __shared__ uint32_t touched[2][3];
    __shared__ uint32_t hrow[3 * kSgdHot];
    const int lane = threadIdx.x & 31;
    const int gl = lane % G;
    const int gw = lane / G;
    for (int i = threadIdx.x; i < 3 * kSgdHot * NV; i += blockDim.x) acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int i = threadIdx.x; i < 3 * kSgdHot; i += blockDim.x) hrow[i] = hot_rows[i];
    if (threadIdx.x < 6) touched[threadIdx.x / 3][threadIdx.x % 3] = 0u;
    __syncthreads();
    const uint64_t ngb = (uint64_t)(blockDim.x >> 5) * GPW;  // groups per block
    const uint64_t group = blockIdx.x * ngb + (uint64_t)(threadIdx.x >> 5) * GPW + gw;
    const uint64_t ngroups = (uint64_t)gridDim.x * ngb;
    const uint64_t rounds = (ntiles + ngroups - 1) / ngroups;
    const float s = *lr_dev;
    uint32_t par = 0;  // parity of the block's step
    for (uint64_t k = 0; k < rounds; ++k) {
        const uint64_t t = group + k * ngroups;
        const bool has_tile = t < ntiles;
        const uint64_t tile = has_tile ? (t * tile_stride) % ntiles : 0;
        const uint64_t start = tile * tile_len;
        const uint64_t end = has_tile ? min(start + tile_len, (uint64_t)n) : start;
        // every group of the block takes tile_len steps per round; the next
        // nonzero's record and hot codes are fetched during this step
        uint4 rn = start < end ? rec[start] : make_uint4(0u, 0u, 0u, 0u);
        uint32_t hn = start < end ? hot[start] : 0u;
        for (uint32_t step = 0; step < tile_len; ++step) {
            const uint64_t p = start + step;
            if (p < end) {
                const uint4 r = rn;
                const uint32_t hc = hn;
                if (p + 1 < end) {
                    rn = rec[p + 1];
                    hn = hot[p + 1];
                }
                const float x = __uint_as_float(r.w);
                float4 *arow = reinterpret_cast<float4 *>(U0 + (size_t)r.x * R) + gl * C;
                float4 *brow = reinterpret_cast<float4 *>(U1 + (size_t)r.y * R) + gl * C;
                float4 *crow = reinterpret_cast<float4 *>(U2 + (size_t)r.z * R) + gl * C;
                float4 a[C], b[C], c[C];
#pragma unroll
                for (int q = 0; q < C; ++q) {
                    a[q] = __ldcg(arow + q);
                    b[q] = __ldcg(brow + q);
                    c[q] = __ldcg(crow + q);
                }
                float part = 0;
#pragma unroll
                for (int q = 0; q < C; ++q)
                    part += a[q].x * b[q].x * c[q].x + a[q].y * b[q].y * c[q].y + a[q].z * b[q].z * c[q].z +
                            a[q].w * b[q].w * c[q].w;
                const uint32_t gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (gw * G));
#pragma unroll
                for (int o = G / 2; o > 0; o >>= 1) part += __shfl_xor_sync(gmask, part, o);
                const float e = x - part;
                float sa = s, sb = s, sc = s;
                if (damp0) {
                    sa *= damp0[r.x];
                    sb *= damp1[r.y];
                    sc *= damp2[r.z];
                }
                const uint32_t slot[3] = {hc & 1023u, (hc >> 10) & 1023u, (hc >> 20) & 1023u};
                float4 *row[3] = {arow, brow, crow};
#pragma unroll
                for (int q = 0; q < C; ++q) {
                    float4 d[3];
                    d[0] = make_float4(sa * (e * b[q].x * c[q].x - lambda * a[q].x),
                                       sa * (e * b[q].y * c[q].y - lambda * a[q].y),
                                       sa * (e * b[q].z * c[q].z - lambda * a[q].z),
                                       sa * (e * b[q].w * c[q].w - lambda * a[q].w));
                    d[1] = make_float4(sb * (e * a[q].x * c[q].x - lambda * b[q].x),
                                       sb * (e * a[q].y * c[q].y - lambda * b[q].y),
                                       sb * (e * a[q].z * c[q].z - lambda * b[q].z),
                                       sb * (e * a[q].w * c[q].w - lambda * b[q].w));
                    d[2] = make_float4(sc * (e * b[q].x * a[q].x - lambda * c[q].x),
                                       sc * (e * b[q].y * a[q].y - lambda * c[q].y),
                                       sc * (e * b[q].z * a[q].z - lambda * c[q].z),
                                       sc * (e * b[q].w * a[q].w - lambda * c[q].w));
#pragma unroll
                    for (int m = 0; m < 3; ++m) {
                        if (slot[m] == kSgdCold) {
                            vatomic_add(row[m] + q, d[m]);
                        } else {
                            float *ac = reinterpret_cast<float *>(&acc[(m * kSgdHot + slot[m]) * NV + gl * C + q]);
                            atomicAdd(ac + 0, d[m].x);
                            atomicAdd(ac + 1, d[m].y);
                            atomicAdd(ac + 2, d[m].z);
                            atomicAdd(ac + 3, d[m].w);
                        }
                    }
                }
                if (gl == 0)
#pragma unroll
                    for (int m = 0; m < 3; ++m)
                        if (slot[m] != kSgdCold) atomicOr(&touched[par][m], 1u << slot[m]);
            }
            __syncthreads();
            // one vector atomic per 16 bytes of every touched hot row; the
            // other parity's marks (the previous step's, read before the
            // barrier above) are cleared for the next step
            if (threadIdx.x < 3) touched[par ^ 1u][threadIdx.x] = 0u;
            for (int i = threadIdx.x; i < 3 * kSgdHot * NV; i += blockDim.x) {
                const int m = i / (kSgdHot * NV), sl = (i / NV) % kSgdHot, v = i % NV;
                if ((touched[par][m] >> sl) & 1u) {
                    const float4 d = acc[i];
                    acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                    float *um = m == 0 ? U0 : (m == 1 ? U1 : U2);
                    vatomic_add(reinterpret_cast<float4 *>(um + (size_t)hrow[m * kSgdHot + sl] * R) + v, d);
                }
            }
            // the accumulators are cleared before the next step adds to them
            __syncthreads();
            par ^= 1u;
        }
    }
}

// hot[p] = the three hot-slot codes of nonzero p (k_sgd_hot), from per-mode
// row -> slot maps (kSgdCold for rows that are not hot)
static __global__ void k_sgd_hot_codes(const uint4 *__restrict__ rec, uint32_t n, const uint16_t *__restrict__ map0,
                                       const uint16_t *__restrict__ map1, const uint16_t *__restrict__ map2,
                                       uint32_t *__restrict__ hot)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint4 r = rec[p];
        hot[p] = (uint32_t)map0[r.x] | ((uint32_t)map1[r.y] << 10) | ((uint32_t)map2[r.z] << 20);
    }
}

// ---------------------------------------------------------------------
// CCD++ (rank-one column updates).  Each mode copy of the training tensor
// is kept as packed 64-bit keys (row | q1 | q2, the row index of the copy's
// mode and the indices of the next two modes) plus a separate residual
// array, 12 bytes per nonzero, in lane-interleaved tile slots (below).  Per
// column f, pack[n][row] holds {current value of column f, final value of
// column f-1, value of column f before its sweeps} for every mode n.
//
// Pass for mode m (k_ccdpp_pass): a warp owns a row-aligned tile; lane l
// walks E consecutive nonzeros, accumulating r*h and h*h per run of equal
// rows (h = product of the other two modes' column f); runs inside a lane
// are finished there, runs crossing lanes are joined by one segmented warp
// scan over the lanes' last runs.  The row's owner writes
// u = sum(r h) / (lambda + sum h^2) into the column and into pack[m].cur.
// FIRST (the first sweep of column f over this copy) also refreshes the
// stored residual:  r <- r - term(f-1, final) + term(f, before sweeps),
// which is the rank-one add-back of f fused with the subtraction of f-1.
// The other two modes' column f (or packs, in FIRST) are gathered from
// shared memory when they fit the block's budget (copied in once per
// persistent block by a bulk async copy), else through L1.  Blocks are
// 512 threads, two per SM, except for a column's first pass when both
// gathered modes' half packs fit one block's shared memory, and for later
// sweeps that stage one sizeable column while gathering the other through
// L1: those run as one 1024-thread block per SM.
// ---------------------------------------------------------------------
struct KeyShape {
    uint32_t s_row, s_q1;   // key >> s_row = row ; (key >> s_q1) & m_q1 = q1
    uint64_t m_q1, m_q2;    // (key >> s_q2) & m_q2 = q2
    uint32_t s_q2;          // 0, or rbits when the residual is packed below the key
    uint32_t rbits;         // packed form: residual bits in the low end of the word
};

__device__ __forceinline__ void unpack_key(uint64_t k, const KeyShape &ks, uint32_t &row, uint32_t &q1,
                                           uint32_t &q2)
{
    row = (uint32_t)(k >> ks.s_row);
    q1 = (uint32_t)((k >> ks.s_q1) & ks.m_q1);
    q2 = (uint32_t)((k >> ks.s_q2) & ks.m_q2);
}

// Packed CCD++ slots (mixed precision): the residual lives in the low
// rbits (16..32) of the key word, as an FP32 value with its low 32 - rbits
// mantissa bits rounded off (round to nearest even): sign, the full 8-bit
// exponent and rbits - 9 mantissa bits.  A finite residual never encodes
// as all ones, so a real entry never equals kPadKey.
__device__ __forceinline__ float packed_res(uint64_t k, uint32_t rbits)
{
    const uint32_t field = (uint32_t)(k & ((1ull << rbits) - 1ull));
    return __uint_as_float(field << (32u - rbits));
}

__device__ __forceinline__ uint64_t with_res(uint64_t k, float r, uint32_t rbits)
{
    uint32_t b = __float_as_uint(r);
    const uint32_t d = 32u - rbits;
    if (d) b = (b + ((1u << (d - 1u)) - 1u) + ((b >> d) & 1u)) >> d;
    const uint64_t mask = (1ull << rbits) - 1ull;
    return (k & ~mask) | ((uint64_t)b & mask);
}

template <typename T>
struct alignas(4 * sizeof(T)) Pack3 {
    T cur, prev, old, pad;
};
// A mode not yet swept in column f (cur == old): {old, final f-1}, half a
// Pack3, so that the first pass of a column can stage both gathered modes
template <typename T>
struct alignas(2 * sizeof(T)) Pack2 {
    T old, prev;
};
template <typename T>
__device__ __forceinline__ T pack_cur(const Pack3<T> &p) { return p.cur; }
template <typename T>
__device__ __forceinline__ T pack_cur(const Pack2<T> &p) { return p.old; }

template <typename T>
__device__ __forceinline__ void ccdpp_finalize(uint32_t row, T nu, T de, T lambda, T *out, Pack3<T> *pkm)
{
    const T u = nu / (lambda + de);
    out[row] = u;
    pkm[row].cur = u;
}

// Tiles of a CCD++ copy are stored in fixed slots of 32*E entries, lane-
// interleaved: entry p of the tile (lane p / E, step p % E) sits at
// slot + (p % E) * 32 + p / E.  Each lane walks its E consecutive entries
// while every load instruction of the warp reads 32 adjacent elements.
// Unused entries of a slot carry kPadKey and a zero residual.
constexpr uint64_t kPadKey = ~0ull;
// pieces of a long row one warp task covers (one slot partial per group)
constexpr int kCcdppGroup = 8;

template <typename T, int E, bool PK>
__device__ __forceinline__ void ccdpp_load_slot(const uint64_t *__restrict__ keys, const T *__restrict__ res,
                                                uint64_t base, int lane, uint32_t rbits, uint64_t (&kv)[E],
                                                T (&rv)[E])
{
#pragma unroll
    for (int e = 0; e < E; ++e) {
        kv[e] = __ldcs(keys + base + 32u * e + lane);
        if constexpr (PK) rv[e] = (T)packed_res(kv[e], rbits);
        else rv[e] = __ldcs(res + base + 32u * e + lane);
    }
}

// FIRST: the refreshed residual of one entry back (into its key word when
// packed)
template <typename T, bool PK>
__device__ __forceinline__ void ccdpp_store_res(uint64_t *keys, T *res, uint64_t at, uint64_t k, T r,
                                                uint32_t rbits)
{
    if constexpr (PK) keys[at] = with_res(k, (float)r, rbits);
    else res[at] = r;
}

template <typename T, int E, bool PK>
__device__ __forceinline__ void ccdpp_store_slot(uint64_t *keys, T *res, uint64_t base, int lane, int cnt,
                                                 const uint64_t (&kv)[E], const T (&rv)[E], uint32_t rbits)
{
#pragma unroll
    for (int e = 0; e < E; ++e)
        if (e < cnt) ccdpp_store_res<T, PK>(keys, res, base + 32u * e + lane, kv[e], rv[e], rbits);
}

// The two gathered modes of a pass.  Non-FIRST passes read column f of each
// (one T per row); FIRST passes read the {cur, prev, old} packs.  A mode
// whose column (or packs) fits the block's shared-memory budget is copied
// there once per block with a bulk async copy and gathered from shared
// memory; the other is gathered through L1 from global memory.
template <typename T>
struct CcdppCols {
    const T *col[2];          // column f of modes m+1, m+2 (global)
    const Pack3<T> *pk[2];    // packs of modes m+1, m+2 (global)
    const Pack2<T> *pk2[2];   // their half packs (the column's first pass)
    uint32_t dim[2];
    int stage[2];             // 1: staged in shared memory
};

template <typename T, bool FIRST, bool FRESH>
__device__ __forceinline__ uint32_t ccdpp_stage_span(const CcdppCols<T> &c, int q, const unsigned char *&src,
                                                     uint32_t &skew)
{
    if constexpr (FIRST && FRESH) {
        src = reinterpret_cast<const unsigned char *>(c.pk2[q]);
        skew = 0;
        return (c.dim[q] * (uint32_t)sizeof(Pack2<T>) + 15u) & ~15u;
    } else if constexpr (FIRST) {
        src = reinterpret_cast<const unsigned char *>(c.pk[q]);
        skew = 0;
        return c.dim[q] * (uint32_t)sizeof(Pack3<T>);
    } else {
        const uintptr_t a = reinterpret_cast<uintptr_t>(c.col[q]);
        skew = (uint32_t)(a & 15u);
        src = reinterpret_cast<const unsigned char *>(a - skew);
        return (skew + c.dim[q] * (uint32_t)sizeof(T) + 15u) & ~15u;
    }
}

// PK: packed slots (residual in the key word, no residual array).  FRESH
// (with FIRST): the column's first pass, where neither gathered mode has
// been swept yet, gathers half packs; it runs as one 1024-thread block per
// SM, whose shared memory holds both gathered modes' half packs.
// BIG: one 1024-thread block per SM (FRESH passes, and later sweeps whose
// staged column would otherwise be held twice per SM, at the cost of the L1
// their other gathers go through)
template <typename T, bool FIRST, int E, bool PK = false, bool FRESH = false, bool BIG = FRESH>
__global__ void __launch_bounds__(BIG ? 1024 : 512, BIG ? 1 : 2)
    k_ccdpp_pass(const int4 *__restrict__ tasks, uint32_t ntasks, uint64_t *__restrict__ keys, T *__restrict__ res,
                 KeyShape ks, Pack3<T> *pkm, CcdppCols<T> cols, T *out, T lambda, T *__restrict__ slot_nu,
                 T *__restrict__ slot_de, const uint4 *__restrict__ heavy, unsigned int *hcnt, int *err,
                 TaskClaim claim)
{
    static_assert(FIRST || !FRESH, "half packs only in a column's first pass");
    using ColT = typename std::conditional<FIRST, typename std::conditional<FRESH, Pack2<T>, Pack3<T>>::type,
                                           T>::type;
    constexpr uint32_t kNone = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char ccdpp_smem[];
    __shared__ __align__(8) uint64_t mbar;
    const int lane = threadIdx.x & 31;

    // ---- stage the gathered columns that fit (one bulk copy each) ----
    const ColT *sc[2] = {nullptr, nullptr};
    if (cols.stage[0] | cols.stage[1]) {
        uint32_t off = 0, total = 0;
        const unsigned char *src[2];
        uint32_t bytes[2] = {0, 0}, dst[2] = {0, 0};
#pragma unroll
        for (int q = 0; q < 2; ++q)
            if (cols.stage[q]) {
                uint32_t skew;
                bytes[q] = ccdpp_stage_span<T, FIRST, FRESH>(cols, q, src[q], skew);
                dst[q] = off;
                sc[q] = reinterpret_cast<const ColT *>(ccdpp_smem + off + skew);
                off += bytes[q];
                total += bytes[q];
            }
        if (threadIdx.x == 0) {
            px::mbar_init(&mbar, 1);
            px::mbar_arrive_expect_tx(&mbar, total);
#pragma unroll
            for (int q = 0; q < 2; ++q)
                for (uint32_t o = 0; o < bytes[q]; o += 32768u)
                    px::bulk_g2s(ccdpp_smem + dst[q] + o, src[q] + o, min(32768u, bytes[q] - o), &mbar);
        }
        __syncthreads();
        const int ok = __syncthreads_and(px::mbar_wait_bounded(px::smem_u32(&mbar), 0) ? 1 : 0);
        if (!ok) {
            // the copy did not complete in time: report, let any copy still
            // in flight land (bounded), and leave the column untouched
            if (threadIdx.x == 0) {
                atomicExch(err, 2);
                px::mbar_wait_bounded(px::smem_u32(&mbar), 0);
            }
            __syncthreads();
            claim.finish(lane);  // every warp still counts itself done
            return;
        }
    }
    auto gat = [&](int q, uint32_t i) -> ColT {
        if constexpr (FIRST && FRESH) return sc[q] ? sc[q][i] : cols.pk2[q][i];
        else if constexpr (FIRST) return sc[q] ? sc[q][i] : cols.pk[q][i];
        else return sc[q] ? sc[q][i] : __ldg(cols.col[q] + i);
    };
    // Later sweeps: the gathers of EC entries e0 .. e0+EC-1 are all issued
    // before any of them is used (h = product of the other two modes'
    // column f); entries past the lane's count, and pads, read index 0 (in
    // bounds) and are skipped by the walk.  First sweeps gather each entry's
    // packs where the walk uses them: holding three products per entry
    // spilled registers there (measured on the 100M workload, tile 256:
    // first sweeps 525-529 us with 1-4 entries ahead against 496 us; later
    // sweeps 268 us with 4 ahead, 354 us with 8, 301 us with none).
    constexpr int EC = FIRST ? 1 : (E < 4 ? E : 4);
    auto gather = [&](int e0, const uint64_t(&kv)[E], int cnt, T(&h)[EC]) {
#pragma unroll
        for (int k = 0; k < EC; ++k) {
            const int e = e0 + k;
            uint32_t row, q1, q2;
            unpack_key(kv[e], ks, row, q1, q2);
            if (e >= cnt || kv[e] == kPadKey) q1 = q2 = 0u;
            if constexpr (!FIRST) h[k] = gat(0, q1) * gat(1, q2);
        }
    };

    // tasks: {tile, len, -1, 0} for a light tile, {first tile, pieces,
    // heavy row, group} for up to kCcdppGroup consecutive pieces of one long
    // row.  A warp takes a fixed-stride share of the tasks, then claims the
    // rest one at a time (TaskClaim, WarpTaskSeq), so warps that drew short
    // tasks take more (a long-row group runs up to kCcdppGroup times a light
    // tile); the task after the current one is known, and its descriptor
    // fetched, while the current one runs.
    const int4 kNoTask = make_int4(0, 0, -1, 0);
    WarpTaskSeq seq(claim, ntasks);
    uint32_t cur_i = seq.next(lane);
    int4 td_cur = cur_i < ntasks ? tasks[cur_i] : kNoTask;
    uint32_t nxt_i = cur_i < ntasks ? seq.next(lane) : ntasks;
    int4 td_nxt = nxt_i < ntasks ? tasks[nxt_i] : kNoTask;
    while (cur_i < ntasks) {
        const int4 td = td_cur;
        // advance first (the task bodies below end with `continue`)
        cur_i = nxt_i;
        td_cur = td_nxt;
        if (cur_i < ntasks) {
            nxt_i = seq.next(lane);
            if (nxt_i < ntasks) td_nxt = tasks[nxt_i];
        }
        uint64_t kv[E];
        T rv[E];
        if (td.z >= 0) {
            // pieces of a long row: per-lane sums over the group's pieces,
            // one warp reduction into the group's slot; the group that
            // arrives last (counter) sums all groups of the row in order and
            // finalises it -- no waiting anywhere
            const uint4 hr = heavy[td.z];
            Pack3<T> pm{};
            if constexpr (FIRST) pm = pkm[hr.x];
            T nu = 0, de = 0;
            for (int j = 0; j < td.y; ++j) {
                const uint64_t base = (uint64_t)(td.x + j) * (uint64_t)(32 * E);
                ccdpp_load_slot<T, E, PK>(keys, res, base, lane, ks.rbits, kv, rv);
#pragma unroll
                for (int e0 = 0; e0 < E; e0 += EC) {
                    T h[EC];
                    gather(e0, kv, E, h);
#pragma unroll
                    for (int k = 0; k < EC; ++k) {
                        const int e = e0 + k;
                        if (kv[e] != kPadKey) {
                            T r = rv[e];
                            T hh;
                            if constexpr (FIRST) {
                                uint32_t rr, q1, q2;
                                unpack_key(kv[e], ks, rr, q1, q2);
                                const ColT ga = gat(0, q1), gb = gat(1, q2);
                                r = r - pm.prev * ga.prev * gb.prev + pm.old * ga.old * gb.old;
                                rv[e] = r;
                                hh = pack_cur<T>(ga) * pack_cur<T>(gb);
                            } else {
                                hh = h[k];
                            }
                            nu += r * hh;
                            de += hh * hh;
                        }
                    }
                }
                if constexpr (FIRST) {
#pragma unroll
                    for (int e = 0; e < E; ++e)
                        if (kv[e] != kPadKey)
                            ccdpp_store_res<T, PK>(keys, res, base + 32u * e + lane, kv[e], rv[e], ks.rbits);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                nu += __shfl_xor_sync(0xffffffffu, nu, o);
                de += __shfl_xor_sync(0xffffffffu, de, o);
            }
            unsigned int last = 0;
            if (lane == 0) {
                slot_nu[td.w] = nu;
                slot_de[td.w] = de;
                __threadfence();
                last = atomicAdd(&hcnt[td.z], 1u) == hr.z - 1 ? 1u : 0u;
            }
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                __threadfence();
                T sn = 0, sd = 0;
                for (uint32_t q = lane; q < hr.z; q += 32) {
                    sn += __ldcg(&slot_nu[hr.y + q]);
                    sd += __ldcg(&slot_de[hr.y + q]);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sn += __shfl_xor_sync(0xffffffffu, sn, o);
                    sd += __shfl_xor_sync(0xffffffffu, sd, o);
                }
                if (lane == 0) {
                    ccdpp_finalize<T>(hr.x, sn, sd, lambda, out, pkm);
                    hcnt[td.z] = 0;
                }
            }
            continue;
        }
        const uint64_t base = (uint64_t)td.x * (uint64_t)(32 * E);
        // valid entries of this lane: the tile's positions lane*E .. +E-1
        const int cnt = max(0, min(E, td.y - lane * E));
        ccdpp_load_slot<T, E, PK>(keys, res, base, lane, ks.rbits, kv, rv);
        // light tile: runs of equal rows inside the lane, then one segmented
        // warp scan joins the runs that cross lanes
        uint32_t hk = kNone, tk = kNone;
        T hn = 0, hd = 0, tn = 0, tdd = 0;
        int nruns = 0;
        Pack3<T> pm{};
#pragma unroll
        for (int e0 = 0; e0 < E; e0 += EC) {
            T h[EC];
            gather(e0, kv, cnt, h);
#pragma unroll
            for (int k = 0; k < EC; ++k) {
                const int e = e0 + k;
                if (e < cnt) {
                    uint32_t row, q1, q2;
                    unpack_key(kv[e], ks, row, q1, q2);
                    if (row != tk) {
                        if (nruns == 1) {
                            hk = tk;
                            hn = tn;
                            hd = tdd;
                        } else if (nruns >= 2) {
                            ccdpp_finalize<T>(tk, tn, tdd, lambda, out, pkm);
                        }
                        tk = row;
                        tn = tdd = 0;
                        ++nruns;
                        if constexpr (FIRST) pm = pkm[row];
                    }
                    T r = rv[e];
                    T hh;
                    if constexpr (FIRST) {
                        const ColT ga = gat(0, q1), gb = gat(1, q2);
                        r = r - pm.prev * ga.prev * gb.prev + pm.old * ga.old * gb.old;
                        rv[e] = r;
                        hh = pack_cur<T>(ga) * pack_cur<T>(gb);
                    } else {
                        hh = h[k];
                    }
                    tn += r * hh;
                    tdd += hh * hh;
                }
            }
        }
        if constexpr (FIRST) ccdpp_store_slot<T, E, PK>(keys, res, base, lane, cnt, kv, rv, ks.rbits);
        const uint32_t in_key = nruns >= 2 ? hk : tk;
        const uint32_t out_key = tk;
        uint32_t prev_out = __shfl_up_sync(0xffffffffu, out_key, 1);
        uint32_t next_in = __shfl_down_sync(0xffffffffu, in_key, 1);
        if (lane == 0) prev_out = kNone;
        if (lane == 31) next_in = kNone;
        int flag = !(nruns == 1 && in_key == prev_out);
        T sn = tn, sd = tdd;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T n2 = __shfl_up_sync(0xffffffffu, sn, d);
            const T d2 = __shfl_up_sync(0xffffffffu, sd, d);
            const int f2 = __shfl_up_sync(0xffffffffu, flag, d);
            if (lane >= d) {
                if (!flag) {
                    sn += n2;
                    sd += d2;
                }
                flag |= f2;
            }
        }
        const T psn = __shfl_up_sync(0xffffffffu, sn, 1);
        const T psd = __shfl_up_sync(0xffffffffu, sd, 1);
        if (nruns >= 2) {
            T n = hn, d = hd;
            if (lane > 0 && hk == prev_out) {
                n += psn;
                d += psd;
            }
            ccdpp_finalize<T>(hk, n, d, lambda, out, pkm);
        }
        if (nruns >= 1 && next_in != out_key) ccdpp_finalize<T>(out_key, sn, sd, lambda, out, pkm);
    }
    claim.finish(lane);
}

// pack[n][row] = {U_n(row, f), U_n(row, f-1) or 0, U_n(row, f), 0} for the
// three modes (column-major factors), before the sweeps of column f, and
// the half pack {U_n(row, f), U_n(row, f-1) or 0} when pk2[n] is given.
struct PackArgs {
    void *pk[3];
    void *pk2[3];
    const void *col[3];   // column f
    const void *pcol[3];  // column f-1 or null
    uint32_t dims[3];
};

template <typename T>
__global__ void k_ccdpp_pack(PackArgs a)
{
    const uint64_t total = (uint64_t)a.dims[0] + a.dims[1] + a.dims[2];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int n = 0;
        uint64_t r = i;
        if (r >= a.dims[0]) {
            r -= a.dims[0];
            n = 1;
            if (r >= a.dims[1]) {
                r -= a.dims[1];
                n = 2;
            }
        }
        const T c = static_cast<const T *>(a.col[n])[r];
        const T p = a.pcol[n] ? static_cast<const T *>(a.pcol[n])[r] : T(0);
        Pack3<T> v;
        v.cur = c;
        v.prev = p;
        v.old = c;
        v.pad = 0;
        static_cast<Pack3<T> *>(a.pk[n])[r] = v;
        if (a.pk2[n]) {
            Pack2<T> h;
            h.old = c;
            h.prev = p;
            static_cast<Pack2<T> *>(a.pk2[n])[r] = h;
        }
    }
}

// indices of the three modes from a key of the mode-m copy
__device__ __forceinline__ void key_modes(uint64_t k, const KeyShape &ks, int m, uint32_t idx[3])
{
    uint32_t row, q1, q2;
    unpack_key(k, ks, row, q1, q2);
    idx[m] = row;
    idx[(m + 1) % 3] = q1;
    idx[(m + 2) % 3] = q2;
}

// res = x - sum_f U0(i0,f) U1(i1,f) U2(i2,f), row-major factors.  A warp
// reads 32 consecutive slots (keys and values) with coalesced loads, then
// walks them with groups of R / VN lanes per slot, lane gl reading the
// 16-byte slice gl of each row (whole rows per warp load), and a butterfly
// sum; unused slot entries (kPadKey) keep their zero residual.
template <typename T, int R, bool PK = false>
__global__ void __launch_bounds__(256) k_ccdpp_init(uint64_t *__restrict__ keys, const T *__restrict__ x,
                                                    T *__restrict__ res, uint32_t n, KeyShape ks, int m,
                                                    const T *__restrict__ U0, const T *__restrict__ U1,
                                                    const T *__restrict__ U2)
{
    using V = typename Vec<T>::type;
    constexpr int VN = Vec<T>::n;
    constexpr int GL = R / VN;
    constexpr int GPW = 32 / GL;
    static_assert(GL >= 1 && 32 % GL == 0, "lanes per slot");
    const int lane = threadIdx.x & 31;
    const int gl = lane % GL, gw = lane / GL;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < n; base += nwarps * 32) {
        const uint64_t mine = base + lane;
        uint64_t key = kPadKey;  // past the end: treated as a pad
        T xv = 0;
        if (mine < n) {
            key = keys[mine];
            xv = x[mine];
        }
#pragma unroll 4
        for (int j = 0; j < GL; ++j) {
            const int src = j * GPW + gw;
            const uint64_t k = __shfl_sync(0xffffffffu, key, src);
            const T xs = __shfl_sync(0xffffffffu, xv, src);
            const bool real = k != kPadKey;
            uint32_t idx[3] = {0u, 0u, 0u};  // row 0 for pads: in bounds, result unused
            if (real) key_modes(k, ks, m, idx);
            const V va = reinterpret_cast<const V *>(U0 + (size_t)idx[0] * R)[gl];
            const V vb = reinterpret_cast<const V *>(U1 + (size_t)idx[1] * R)[gl];
            const V vc = reinterpret_cast<const V *>(U2 + (size_t)idx[2] * R)[gl];
            T p = 0;
#pragma unroll
            for (int v = 0; v < VN; ++v) p += vget(va, v) * vget(vb, v) * vget(vc, v);
#pragma unroll
            for (int o = GL / 2; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
            if (real && gl == 0) ccdpp_store_res<T, PK>(keys, res, base + src, k, xs - p, ks.rbits);
        }
    }
}

// res -= U0(i0,c) U1(i1,c) U2(i2,c) for one column c (column-major
// pointers); optional SSE partials of the new residual.
template <typename T, bool PK = false>
__global__ void __launch_bounds__(256) k_ccdpp_finish(uint64_t *__restrict__ keys, T *__restrict__ res,
                                                      uint32_t n, KeyShape ks, int m, const T *__restrict__ c0,
                                                      const T *__restrict__ c1, const T *__restrict__ c2,
                                                      double *__restrict__ partial)
{
    // four slots per thread per round, every load and gather issued before
    // any residual is formed
    constexpr int U = 4;
    double acc = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint64_t p0 = blockIdx.x * blockDim.x + threadIdx.x; p0 < n; p0 += (uint64_t)U * stride) {
        uint64_t key[U];
        T r0[U], g[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t p = p0 + (uint64_t)u * stride;
            key[u] = p < n ? keys[p] : kPadKey;
            r0[u] = (!PK && p < n) ? res[p] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            g[u] = 0;
            if (key[u] != kPadKey) {
                uint32_t idx[3];
                key_modes(key[u], ks, m, idx);
                g[u] = c0[idx[0]] * c1[idx[1]] * c2[idx[2]];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (key[u] == kPadKey) continue;
            const uint64_t p = p0 + (uint64_t)u * stride;
            const T rb = PK ? (T)packed_res(key[u], ks.rbits) : r0[u];
            const T r = rb - g[u];
            ccdpp_store_res<T, PK>(keys, res, p, key[u], r, ks.rbits);
            // the SSE of the residual as stored
            const T rs = PK ? (T)packed_res(with_res(key[u], (float)r, ks.rbits), ks.rbits) : r;
            acc += (double)rs * (double)rs;
        }
    }
    if (partial) {
        acc = block_sum(acc);
        if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    }
}

// Sum of squares of the residuals held in packed slots (pads skipped).
static __global__ void __launch_bounds__(256) k_ccdpp_res_sumsq(const uint64_t *__restrict__ keys, uint32_t n,
                                                                uint32_t rbits, double *__restrict__ partial)
{
    double acc = 0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint64_t key = keys[p];
        if (key == kPadKey) continue;
        const double r = (double)packed_res(key, rbits);
        acc += r * r;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// column-major (R x d) -> row-major (d x R)
template <typename T>
__global__ void k_col_to_row(const T *__restrict__ col, T *__restrict__ row, uint32_t d, int R)
{
    const uint64_t total = (uint64_t)d * R;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = i / R, f = i % R;
        row[i] = col[f * d + r];
    }
}

// ---------------------------------------------------------------------
// Reference "CCD+" (sgpu/ccd.cu:82-206, 318-348): all columns of a row at
// once, residual with the row's old values, optional per-nonzero
// multiplicity w.  Lane per column (C columns per lane), nonzeros of a tile
// in order; rows absent from the tensor keep their values.
// ---------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(128) k_ccdc_tile(const int4 *__restrict__ tiles, uint32_t ntiles,
                                                   const uint4 *__restrict__ rec,
                                                   const double *__restrict__ v64,
                                                   const T *__restrict__ w, int m, T *Um,
                                                   const T *__restrict__ Ua,
                                                   const T *__restrict__ Ub, T lambda,
                                                   T *__restrict__ slot)
{
    constexpr int C = (R + 31) / 32;
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
    for (uint64_t tile = warp; tile < ntiles; tile += nwarps) {
        const int4 td = tiles[tile];
        const uint32_t start = (uint32_t)td.x, end = start + (uint32_t)td.y;
        const bool heavy = td.z >= 0;
        uint32_t cur = kNoKey;
        T num[C], den[C], arow[C];
        auto flush = [&]() {
            if (cur == kNoKey) return;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int col = lane + 32 * c;
                if (col < R) {
                    if (heavy) {
                        slot[tile * (2 * R) + col] = num[c];
                        slot[tile * (2 * R) + R + col] = den[c];
                    } else {
                        Um[(size_t)cur * R + col] = num[c] / (lambda + den[c]);
                    }
                }
            }
        };
        for (uint32_t p = start; p < end; ++p) {
            const uint4 r = rec[p];
            const uint32_t key = key_of(r, m);
            if (key != cur) {
                flush();
                cur = key;
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const int col = lane + 32 * c;
                    num[c] = den[c] = 0;
                    arow[c] = col < R ? Um[(size_t)key * R + col] : T(0);
                }
            }
            const T wn = w ? w[p] : T(1);
            if (wn == T(0)) continue;
            const uint32_t qa = key_of(r, m1), qb = key_of(r, m2);
            T h[C];
            T dot = 0;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int col = lane + 32 * c;
                h[c] = col < R ? Ua[(size_t)qa * R + col] * Ub[(size_t)qb * R + col] : T(0);
                dot += arow[c] * h[c];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
            const T e = value_of<T>(r, v64, p) - dot;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                den[c] += wn * h[c] * h[c];
                num[c] += wn * h[c] * e;
            }
        }
        flush();
    }
}

template <typename T, int R>
__global__ void __launch_bounds__(128) k_ccdc_fix(const uint4 *__restrict__ heavy, uint32_t nheavy,
                                                  const T *__restrict__ slot, T *Um, T lambda)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t h = warp; h < nheavy; h += nwarps) {
        const uint4 hr = heavy[h];
        for (int col = lane; col < R; col += 32) {
            T nu = 0, de = 0;
            for (uint32_t q = 0; q < hr.z; ++q) {
                nu += slot[(size_t)(hr.y + q) * 2 * R + col];
                de += slot[(size_t)(hr.y + q) * 2 * R + R + col];
            }
            Um[(size_t)hr.x * R + col] = nu / (lambda + de);
        }
    }
}

// ---------------------------------------------------------------------
// ALS (sgpu/als.cu:186-317 + 467-491 + cuSOLVER, restated): per row
//   (sum w h h^T + lambda I) u = sum w x h,  h = Ua(j) o Ub(k).
// Lane layout: L = min(R,32) lanes per nonzero group, NG = 32/L groups
// take consecutive nonzeros of the row, C = R/L Gram columns per lane held
// in registers.  The row's system is solved by its warp in FP64 in shared
// memory: Cholesky, forward/back substitution, one refinement step against
// the register copy of the Gram matrix.  Heavy-row pieces store their
// partial Gram + right-hand side; k_als_sum_pieces sums them in piece order.
// ---------------------------------------------------------------------
template <int R>
struct AlsShape {
    // C Gram columns per lane (lane gl holds columns gl + L*c), L = R / C
    // lanes per nonzero, NG = 32 / L nonzeros per warp step: more columns
    // per lane mean fewer shuffles per nonzero (R / C broadcasts of h)
    static constexpr int C = R <= 8 ? 2 : (R <= 16 ? 4 : 2);
    static constexpr int L = R / C;
    static constexpr int NG = 32 / L;
};

// Batched row solves (the light tiles' rows, and the long rows after their
// pieces are summed): a warp parks the regularised
// systems of NS rows in shared memory and factors them together, one group
// of GS lanes per system (FP64 right-looking Cholesky on the packed lower
// triangle, forward/back substitution, one refinement step against the
// FP32/FP64 Gram as accumulated).  Per system: factor (TRI doubles), b, y,
// u (R doubles each), the Gram (TRI of T); per warp also NS row ids.
// GS = R / 2 below rank 32, 32 from rank 32: few enough parked systems
// that the shared memory of a 4-warp block does not hold the SM below what
// its registers allow (at R = 32, FP32: one 7.4 KB system per warp, 4
// blocks = 16 warps per SM; four systems per warp held it to 1 block, two
// to 3).  Each factor element sees the same operations in the same order
// for any GS, so the choice does not change results.
template <typename T, int R>
struct AlsBatch {
    static constexpr int GS = R >= 32 ? 32 : (R >= 8 ? R / 2 : 2);
    static constexpr int NS = 32 / GS;
    static constexpr int TRI = R * (R + 1) / 2;
    static constexpr int gram_doubles = (TRI * (int)sizeof(T) + 7) / 8;
    // + R doubles: reciprocals of the factor's diagonal
    static constexpr int sys_doubles = TRI + 4 * R + gram_doubles;
    static constexpr int warp_doubles = NS * sys_doubles + (NS + 1) / 2;
};

__device__ __forceinline__ int tri_idx(int i, int k) { return i * (i + 1) / 2 + k; }

// Factor and solve the k (<= NS) parked systems of this warp; writes u into
// the rows' factor rows.  Returns the number of systems whose pivot was not
// positive (diagonal shifted), counted once per system.
template <typename T, int R>
__device__ __forceinline__ int als_solve_parked(double *W, int k, T lambda, T *Um)
{
    using B = AlsBatch<T, R>;
    constexpr int GS = B::GS;
    const int lane = threadIdx.x & 31;
    const int grp = lane / GS, sl = lane % GS;
    const bool act = grp < k;
    double *fac = W + (size_t)(act ? grp : 0) * B::sys_doubles;
    double *bb = fac + B::TRI;
    double *yy = bb + R;
    double *uu = yy + R;
    const T *gram = reinterpret_cast<const T *>(uu + R);
    double *dinv = uu + R + B::gram_doubles;
    const uint32_t *rows = reinterpret_cast<const uint32_t *>(W + (size_t)B::NS * B::sys_doubles);
    int bad = 0;
    for (int j = 0; j < R; ++j) {
        double d = act ? fac[tri_idx(j, j)] : 1.0;
        if (act && !(d > 0.0)) {
            bad = 1;
            d = 1e-300 + fabs(d) + 1e-12 * (double)lambda + 1e-30;
        }
        const double ljj = sqrt(d);
        const double inv = 1.0 / ljj;  // one division per column
        __syncwarp();
        if (act) {
            if (sl == 0) {
                fac[tri_idx(j, j)] = ljj;
                dinv[j] = inv;
            }
            for (int i = j + 1 + sl; i < R; i += GS) fac[tri_idx(i, j)] *= inv;
        }
        __syncwarp();
        // trailing update L(i, k) -= L(i, j) L(k, j), j < k <= i, by columns:
        // lane sl of the group owns the columns k with k mod 2GS equal to sl
        // or 2GS-1-sl, which gives every lane the same number of entries
        if (act)
            for (int c0 = 0; c0 < R; c0 += 2 * GS) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = h == 0 ? c0 + sl : c0 + 2 * GS - 1 - sl;
                    if (k <= j || k >= R) continue;
                    const double lkj = fac[tri_idx(k, j)];
                    int base = k * (k + 1) / 2;  // tri_idx(i, 0) for i = k
                    for (int i = k; i < R; ++i) {
                        fac[base + k] -= fac[base + j] * lkj;
                        base += i + 1;
                    }
                }
            }
        __syncwarp();
    }
    for (int it = 0; it < 2; ++it) {
        for (int i = 0; i < R; ++i) {  // L z = y
            const double zi = act ? yy[i] * dinv[i] : 0.0;
            __syncwarp();
            if (act) {
                if (sl == 0) yy[i] = zi;
                for (int k2 = i + 1 + sl; k2 < R; k2 += GS) yy[k2] -= fac[tri_idx(k2, i)] * zi;
            }
            __syncwarp();
        }
        for (int i = R - 1; i >= 0; --i) {  // L^T v = z
            const double vi = act ? yy[i] * dinv[i] : 0.0;
            __syncwarp();
            if (act) {
                if (sl == 0) yy[i] = vi;
                for (int k2 = sl; k2 < i; k2 += GS) yy[k2] -= fac[tri_idx(i, k2)] * vi;
            }
            __syncwarp();
        }
        if (it == 0) {
            if (act)
                for (int a = sl; a < R; a += GS) uu[a] = yy[a];
            __syncwarp();
            // residual b - (G + lambda I) u with the Gram as accumulated
            if (act)
                for (int a = sl; a < R; a += GS) {
                    double acc = bb[a] - (double)lambda * uu[a];
                    for (int c = 0; c < R; ++c)
                        acc -= (double)gram[a >= c ? tri_idx(a, c) : tri_idx(c, a)] * uu[c];
                    yy[a] = acc;
                }
            __syncwarp();
        } else if (act) {
            T *dst = Um + (size_t)rows[grp] * R;
            for (int a = sl; a < R; a += GS) dst[a] = (T)(uu[a] + yy[a]);
        }
    }
    __syncwarp();
    return (act && sl == 0) ? bad : 0;
}

// Park the row's system (Gram G and right-hand side b as left by
// als_accumulate: lane gl < L holds columns gl + L*c) in slot k.
template <typename T, int R>
__device__ __forceinline__ void als_park(double *W, int k, uint32_t row, const T (&G)[R][AlsShape<R>::C],
                                         const T (&b)[AlsShape<R>::C], T lambda)
{
    using B = AlsBatch<T, R>;
    using Sh = AlsShape<R>;
    constexpr int L = Sh::L, C = Sh::C;
    const int lane = threadIdx.x & 31;
    double *fac = W + (size_t)k * B::sys_doubles;
    double *bb = fac + B::TRI;
    double *yy = bb + R;
    T *gram = reinterpret_cast<T *>(yy + 2 * R);
    // every group of L lanes holds the row's full sums; group g writes the
    // Gram rows a with a % NG == g
    constexpr int NG = Sh::NG;
    const int gl = lane % L, g = lane / L;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const int col = gl + L * c;
#pragma unroll
        for (int a = 0; a < R; ++a)
            if (a % NG == g && a >= col) {
                fac[tri_idx(a, col)] = (double)G[a][c] + (a == col ? (double)lambda : 0.0);
                gram[tri_idx(a, col)] = G[a][c];
            }
        if (g == 0) {
            bb[col] = (double)b[c];
            yy[col] = (double)b[c];
        }
    }
    if (lane == 0) reinterpret_cast<uint32_t *>(W + (size_t)B::NS * B::sys_doubles)[k] = row;
    __syncwarp();
}

template <typename T, int R>
__device__ __forceinline__ void als_accumulate(const uint4 *__restrict__ rec,
                                               const double *__restrict__ v64,
                                               const T *__restrict__ w, int m,
                                               const T *__restrict__ Ua, const T *__restrict__ Ub,
                                               uint32_t s, uint32_t e, T (&G)[R][AlsShape<R>::C],
                                               T (&b)[AlsShape<R>::C])
{
    using Sh = AlsShape<R>;
    constexpr int L = Sh::L, NG = Sh::NG, C = Sh::C;
    const int lane = threadIdx.x & 31;
    const int gl = lane % L, g = lane / L;
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        b[c] = 0;
#pragma unroll
        for (int a = 0; a < R; ++a) G[a][c] = 0;
    }
    // a two-stage pipeline: while step k is multiplied in, the rows of step
    // k + 1 (whose record came a step earlier) and the record of step k + 2
    // are on their way
    const uint4 kZero = make_uint4(0u, 0u, 0u, 0u);
    uint4 r0 = s + g < e ? rec[s + g] : kZero;
    uint4 r1 = s + g + NG < e ? rec[s + g + NG] : kZero;
    T ua[C], ub[C];
#pragma unroll
    for (int c = 0; c < C; ++c) ua[c] = ub[c] = 0;
    if (s + g < e) {
        const T *ra = Ua + (size_t)key_of(r0, m1) * R;
        const T *rb = Ub + (size_t)key_of(r0, m2) * R;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            ua[c] = ra[gl + L * c];
            ub[c] = rb[gl + L * c];
        }
    }
    for (uint32_t base = s; base < e; base += NG) {
        const uint32_t p = base + g;
        const bool valid = p < e;
        T na[C], nb[C];
#pragma unroll
        for (int c = 0; c < C; ++c) na[c] = nb[c] = 0;
        if (p + NG < e) {
            const T *ra = Ua + (size_t)key_of(r1, m1) * R;
            const T *rb = Ub + (size_t)key_of(r1, m2) * R;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                na[c] = ra[gl + L * c];
                nb[c] = rb[gl + L * c];
            }
        }
        const uint4 r2 = p + 2 * NG < e ? rec[p + 2 * NG] : kZero;
        T hc[C], hw[C];
        T wx = 0, wn = 0;
        if (valid) {
            wn = w ? w[p] : T(1);
            wx = wn * value_of<T>(r0, v64, p);
#pragma unroll
            for (int c = 0; c < C; ++c) hc[c] = ua[c] * ub[c];
        } else {
#pragma unroll
            for (int c = 0; c < C; ++c) hc[c] = 0;
        }
        r0 = r1;
        r1 = r2;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            ua[c] = na[c];
            ub[c] = nb[c];
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            b[c] += wx * hc[c];
            hw[c] = wn * hc[c];  // the multiplicity folded into the lane's own columns
        }
#pragma unroll
        for (int a = 0; a < R; ++a) {
            const T ha = __shfl_sync(0xffffffffu, hc[a / L], g * L + (a % L));
#pragma unroll
            for (int c = 0; c < C; ++c) G[a][c] += ha * hw[c];
        }
    }
    if constexpr (NG > 1) {
#pragma unroll
        for (int o = L; o < 32; o <<= 1) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
                b[c] += __shfl_xor_sync(0xffffffffu, b[c], o);
#pragma unroll
                for (int a = 0; a < R; ++a) G[a][c] += __shfl_xor_sync(0xffffffffu, G[a][c], o);
            }
        }
    }
}

// Short rows: a row with k <= KW = R / 2 nonzeros (and no reference
// multiplicities) has a Gram H^T H of rank k, and its system
//     (H^T H + lambda I) u = H^T x            (R x R)
// is solved through the k x k dual (the Woodbury identity)
//     (H H^T + lambda I) y = x,   u = H^T y
// in FP64: H (the row's Khatri-Rao rows, h_i = U_a(q1_i) o U_b(q2_i)
// formed in T as the R x R path forms them) in the warp's free
// parked-system slot, K = H H^T + lambda I by lane per entry, its Cholesky
// factor with lane j owning row j, substitutions with y in registers (lane
// i holds y_i), and one refinement step on the dual residual
// x - H u - lambda y.  Costs k^2 R + k^3 / 6 instead of k R^2 + R^3 / 6.
// Returns 1 when a pivot was not positive (diagonal shifted).
template <typename T, int R>
struct AlsShort {
    static constexpr int KW = R / 2;        // longest row solved this way
    static constexpr int HS = R + 1;        // H row stride (doubles): 2-way banks at most
    static constexpr int KS = KW + 1;       // K row stride
    static constexpr int doubles = KW * HS + KW * KS + KW + R;
    static_assert(doubles <= AlsBatch<T, R>::sys_doubles, "short-row scratch fits one parked-system slot");
    static_assert(KW <= 32, "one lane per dual row");
};

template <typename T, int R>
__device__ __forceinline__ int als_solve_short(const uint4 *__restrict__ rec, const double *__restrict__ v64, int m,
                                               const T *__restrict__ Ua, const T *__restrict__ Ub, uint32_t s,
                                               int k, T lambda, double *scr, T *Um, uint32_t row)
{
    using Sw = AlsShort<T, R>;
    constexpr int HS = Sw::HS, KS = Sw::KS, KW = Sw::KW;
    constexpr int FL = R < 32 ? R : 32;  // lanes per h row
    constexpr int IPS = 32 / FL;         // h rows per step
    const int lane = threadIdx.x & 31;
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
    double *H = scr;                 // k x R
    double *K = H + KW * HS;         // k x k, lower triangle
    double *dinv = K + KW * KS;      // 1 / L(j, j)
    double *u = dinv + KW;           // R
    const double lam = (double)lambda;
    // lane i < k: the record of nonzero i
    uint32_t qa = 0, qb = 0;
    double xi = 0.0;
    if (lane < k) {
        const uint4 r = rec[s + lane];
        qa = key_of(r, m1);
        qb = key_of(r, m2);
        xi = (double)value_of<T>(r, v64, s + lane);
    }
    for (int i0 = 0; i0 < k; i0 += IPS) {
        const int i = i0 + lane / FL;
        const int src = min(i, k - 1);
        const uint32_t a = __shfl_sync(0xffffffffu, qa, src), b = __shfl_sync(0xffffffffu, qb, src);
        if (i < k)
            for (int f = lane % FL; f < R; f += FL) H[i * HS + f] = (double)(Ua[(size_t)a * R + f] * Ub[(size_t)b * R + f]);
    }
    __syncwarp();
    // K = H H^T + lambda I, lower triangle, one lane per entry
    const int npairs = k * (k + 1) / 2;
    for (int p = lane; p < npairs; p += 32) {
        int i = (int)((sqrtf(8.0f * (float)p + 1.0f) - 1.0f) * 0.5f);
        while (i * (i + 1) / 2 > p) --i;
        while ((i + 1) * (i + 2) / 2 <= p) ++i;
        const int j = p - i * (i + 1) / 2;
        double acc = (i == j) ? lam : 0.0;
#pragma unroll 8
        for (int f = 0; f < R; ++f) acc += H[i * HS + f] * H[j * HS + f];
        K[i * KS + j] = acc;
    }
    __syncwarp();
    // Cholesky K = L L^T, right-looking; lane i updates row i
    int bad = 0;
    for (int j = 0; j < k; ++j) {
        if (lane == j) {
            double d = K[j * KS + j];
            if (!(d > 0.0)) {
                bad = 1;
                d = 1e-300 + fabs(d) + 1e-12 * lam + 1e-30;
            }
            const double l = sqrt(d);
            K[j * KS + j] = l;
            dinv[j] = 1.0 / l;
        }
        __syncwarp();
        if (lane > j && lane < k) K[lane * KS + j] *= dinv[j];  // column j of L
        __syncwarp();
        if (lane > j && lane < k) {  // trailing update of row `lane`
            const double lij = K[lane * KS + j];
            for (int c = j + 1; c <= lane; ++c) K[lane * KS + c] -= lij * K[c * KS + j];
        }
        __syncwarp();
    }
    // y = K^-1 x (lane i holds y_i), u = H^T y, then one refinement step
    auto solve = [&](double rhs) -> double {
        double yi = rhs;
        for (int j = 0; j < k; ++j) {  // L z = rhs
            const double yj = __shfl_sync(0xffffffffu, yi, j) * dinv[j];
            if (lane == j) yi = yj;
            else if (lane > j && lane < k) yi -= K[lane * KS + j] * yj;
        }
        for (int j = k - 1; j >= 0; --j) {  // L^T y = z
            const double yj = __shfl_sync(0xffffffffu, yi, j) * dinv[j];
            if (lane == j) yi = yj;
            else if (lane < j) yi -= K[j * KS + lane] * yj;
        }
        return lane < k ? yi : 0.0;
    };
    auto primal = [&](double yi) {  // u = H^T y into shared memory
        double uf[(R + 31) / 32];
#pragma unroll
        for (int t = 0; t < (R + 31) / 32; ++t) uf[t] = 0.0;
        for (int i = 0; i < k; ++i) {
            const double yv = __shfl_sync(0xffffffffu, yi, i);
#pragma unroll
            for (int t = 0; t < (R + 31) / 32; ++t)
                if (lane + 32 * t < R) uf[t] += yv * H[i * HS + lane + 32 * t];
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < (R + 31) / 32; ++t)
            if (lane + 32 * t < R) u[lane + 32 * t] = uf[t];
        __syncwarp();
    };
    double y = solve(xi);
    primal(y);
    // dual residual x_i - h_i . u - lambda y_i (lane i), corrected y
    double res = 0.0;
    if (lane < k) {
        double hu = 0.0;
        for (int f = 0; f < R; ++f) hu += H[lane * HS + f] * u[f];
        res = xi - hu - lam * y;
    }
    y += solve(res);
    primal(y);
    for (int f = lane; f < R; f += 32) Um[(size_t)row * R + f] = (T)u[f];
    const bool any_bad = __any_sync(0xffffffffu, bad != 0);
    __syncwarp();
    return (any_bad && lane == 0) ? 1 : 0;  // once per row, as the parked solves count
}

template <typename T, int R>
__global__ void __launch_bounds__(128) k_als_tile(const int4 *__restrict__ tiles, uint32_t ntiles,
                                                  const uint4 *__restrict__ rec,
                                                  const double *__restrict__ v64,
                                                  const T *__restrict__ w, int m, T *Um,
                                                  const T *__restrict__ Ua,
                                                  const T *__restrict__ Ub, T lambda,
                                                  T *__restrict__ slot,
                                                  unsigned long long *nonspd, int skip_heavy, TaskClaim claim)
{
    using Sh = AlsShape<R>;
    using Bt = AlsBatch<T, R>;
    constexpr int L = Sh::L, C = Sh::C;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    double *W = smem + (size_t)wib * Bt::warp_doubles;
    const int gl = lane % L;
    int bad = 0, parked = 0;
    const bool short_rows = w == nullptr && lambda > T(0);
    T G[R][C];
    T b[C];
    // tiles claimed one at a time (TaskClaim): tiles of many short rows, or
    // pieces that the tensor-core Gram takes, cost very different times
    // (every tile claimed: the grid is larger than the resident blocks, and
    // the fixed-stride sequence's state raised the rank-32 FP32 kernel from
    // 128 to 254 registers, halving its warps per SM)
    for (uint32_t tile = claim.next(lane); tile < ntiles; tile = claim.next(lane)) {
        const int4 td = tiles[tile];
        const uint32_t start = (uint32_t)td.x, end = start + (uint32_t)td.y;
        if (td.z >= 0) {
            if (skip_heavy) continue;  // pieces of long rows go to the tensor-core Gram
            als_accumulate<T, R>(rec, v64, w, m, Ua, Ub, start, end, G, b);
            if (lane < L) {
                T *dst = slot + tile * (size_t)(R * R + R);
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const int col = gl + L * c;
#pragma unroll
                    for (int a = 0; a < R; ++a) dst[a * R + col] = G[a][c];
                    dst[R * R + col] = b[c];
                }
            }
            continue;
        }
        uint32_t s = start;
        while (s < end) {
            // the row's extent: 32 keys at a time, first mismatch by ballot
            const uint32_t key = key_of(rec[s], m);
            uint32_t e = s + 1;
            for (;;) {
                const uint32_t q = e + lane;
                const unsigned same = __ballot_sync(0xffffffffu, q < end && key_of(rec[q], m) == key);
                if (same != 0xffffffffu) {
                    e += __ffs(~same) - 1;
                    break;
                }
                e += 32;
            }
            if (short_rows && e - s <= (uint32_t)AlsShort<T, R>::KW) {
                // the free slot (parked < NS here) holds the short row's scratch
                bad += als_solve_short<T, R>(rec, v64, m, Ua, Ub, s, (int)(e - s), lambda,
                                             W + (size_t)parked * Bt::sys_doubles, Um, key);
                s = e;
                continue;
            }
            als_accumulate<T, R>(rec, v64, w, m, Ua, Ub, s, e, G, b);
            als_park<T, R>(W, parked, key, G, b, lambda);
            if (++parked == Bt::NS) {
                bad += als_solve_parked<T, R>(W, parked, lambda, Um);
                parked = 0;
            }
            s = e;
        }
    }
    if (parked) bad += als_solve_parked<T, R>(W, parked, lambda, Um);
    bad = __reduce_add_sync(0xffffffffu, bad);
    if (lane == 0 && bad) atomicAdd(nonspd, (unsigned long long)bad);
    claim.finish(lane);
}

// Sum of each long row's piece partials, element-parallel: thread per
// (row, slot entry), pieces added in piece order (the order k_als_fix used
// when it summed them itself), the total written into the row's first
// slot.  Coalesced across the threads of a row; every thread touches only
// its own entry.
template <typename T, int R>
__global__ void __launch_bounds__(256) k_als_sum_pieces(const uint4 *__restrict__ heavy, uint32_t nheavy,
                                                        T *__restrict__ slot)
{
    constexpr uint32_t S = R * R + R;
    const uint64_t total = (uint64_t)nheavy * S;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t h = (uint32_t)(i / S), e = (uint32_t)(i % S);
        const uint4 hr = heavy[h];
        const T *src = slot + (size_t)hr.y * S + e;
        T acc = 0;
        for (uint32_t q = 0; q < hr.z; ++q) acc += src[(size_t)q * S];
        slot[(size_t)hr.y * S + e] = acc;
    }
}

// summed != 0: the pieces were already summed into each row's first slot.
// The rows' systems are solved like the light tiles' (parked, packed lower
// triangle, columns owned across the lanes): a row-major system with one
// row per lane put every lane of a column step on the same shared-memory
// bank at rank 32.
template <typename T, int R>
__global__ void __launch_bounds__(128) k_als_fix(const uint4 *__restrict__ heavy, uint32_t nheavy,
                                                 const T *__restrict__ slot, T *Um, T lambda,
                                                 unsigned long long *nonspd, int summed)
{
    using Sh = AlsShape<R>;
    using Bt = AlsBatch<T, R>;
    constexpr int L = Sh::L, C = Sh::C;
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    double *W = smem + (size_t)wib * Bt::warp_doubles;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const int gl = lane % L;
    int bad = 0, parked = 0;
    T G[R][C];
    T b[C];
    for (uint64_t h = warp; h < nheavy; h += nwarps) {
        const uint4 hr = heavy[h];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            b[c] = 0;
#pragma unroll
            for (int a = 0; a < R; ++a) G[a][c] = 0;
        }
        const uint32_t np = summed ? 1u : hr.z;
        for (uint32_t q = 0; q < np; ++q) {
            const T *src = slot + (size_t)(hr.y + q) * (R * R + R);
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const int col = gl + L * c;
#pragma unroll
                for (int a = 0; a < R; ++a) G[a][c] += src[a * R + col];
                b[c] += src[R * R + col];
            }
        }
        als_park<T, R>(W, parked, hr.x, G, b, lambda);
        if (++parked == Bt::NS) {
            bad += als_solve_parked<T, R>(W, parked, lambda, Um);
            parked = 0;
        }
    }
    if (parked) bad += als_solve_parked<T, R>(W, parked, lambda, Um);
    bad = __reduce_add_sync(0xffffffffu, bad);
    if (lane == 0 && bad) atomicAdd(nonspd, (unsigned long long)bad);
}

// ---------------------------------------------------------------------
// Adjoint of 1/2 sum_Omega (x - xhat)^2 + lambda sum ||U||^2 in one pass:
// groups of G = R/VN lanes walk tiles of mode-0-sorted nonzeros, recompute
// the residual, keep the mode-0 gradient row in registers while the row
// does not change, and add the mode-1/2 rows atomically.  G must hold
// 2*lambda*U on entry (k_axpby).
// ---------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(256) k_grad(const uint4 *__restrict__ rec,
                                              const double *__restrict__ v64, uint32_t n,
                                              uint32_t tile_len, uint32_t ntiles,
                                              const T *__restrict__ U0, const T *__restrict__ U1,
                                              const T *__restrict__ U2, T *G0, T *G1, T *G2,
                                              double *__restrict__ partial)
{
    using V = typename Vec<T>::type;
    constexpr int VN = Vec<T>::n;
    constexpr int G = R / VN;
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & 31;
    const int gl = lane % G, gw = lane / G;
    const uint32_t gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (gw * G));
    const uint64_t group = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * GPW + gw;
    const uint64_t ngroups = ((uint64_t)gridDim.x * blockDim.x >> 5) * GPW;
    double obj = 0;
    for (uint64_t tile = group; tile < ntiles; tile += ngroups) {
        const uint64_t start = tile * tile_len;
        const uint64_t end = min(start + tile_len, (uint64_t)n);
        uint32_t cur = kNoKey;
        V ga;
        V *grow = nullptr;
        for (uint64_t p = start; p < end; ++p) {
            const uint4 r = rec[p];
            const T x = value_of<T>(r, v64, p);
            if (r.x != cur) {
                if (grow) vatomic_add(grow, ga);
                cur = r.x;
                grow = reinterpret_cast<V *>(G0 + (size_t)r.x * R) + gl;
#pragma unroll
                for (int v = 0; v < VN; ++v) vset(ga, v, T(0));
            }
            const V a = reinterpret_cast<const V *>(U0 + (size_t)r.x * R)[gl];
            const V b = reinterpret_cast<const V *>(U1 + (size_t)r.y * R)[gl];
            const V c = reinterpret_cast<const V *>(U2 + (size_t)r.z * R)[gl];
            T part = 0;
#pragma unroll
            for (int v = 0; v < VN; ++v) part += vget(a, v) * vget(b, v) * vget(c, v);
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) part += __shfl_xor_sync(gmask, part, o);
            const T e = x - part;
            if (gl == 0) obj += 0.5 * (double)e * (double)e;
            V gb, gc;
#pragma unroll
            for (int v = 0; v < VN; ++v) {
                const T av = vget(a, v), bv = vget(b, v), cv = vget(c, v);
                vset(ga, v, vget(ga, v) - e * bv * cv);
                vset(gb, v, -e * av * cv);
                vset(gc, v, -e * av * bv);
            }
            vatomic_add(reinterpret_cast<V *>(G1 + (size_t)r.y * R) + gl, gb);
            vatomic_add(reinterpret_cast<V *>(G2 + (size_t)r.z * R) + gl, gc);
        }
        if (grow) vatomic_add(grow, ga);
    }
    obj = block_sum(obj);
    if (threadIdx.x == 0) partial[blockIdx.x] = obj;
}

// y = alpha * x (elementwise)
template <typename T>
__global__ void k_scale(const T *__restrict__ x, T *__restrict__ y, uint64_t n, T alpha)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        y[i] = alpha * x[i];
}

// Self-test of the bounded-wait path: one thread waits, with the same
// bounded wait the tensor-core Gram and the CCD++ pass use, on an mbarrier
// that nothing arrives on.  The wait gives up after limit_ns and the kernel
// records `code` in the session's error flag, then returns (no copy is in
// flight, nothing else to release).
static __global__ void k_wait_probe(int *__restrict__ err, int code, uint64_t limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) px::mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0 && !px::mbar_wait_bounded(px::smem_u32(&bar), 0, limit_ns)) atomicExch(err, code);
}

}  // namespace k
}  // namespace ctc
