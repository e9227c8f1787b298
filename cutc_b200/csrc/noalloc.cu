// noalloc.cu -- squared-error sum over device-resident nonzeros that
// allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: a process whose GPU
// memory is fully reserved by another allocator (for example a serving
// stack that pre-allocates one pool for the whole device), or a loop that
// cannot take the device-wide synchronisation and latency of an
// allocation.  ctc_sse_noalloc gives them the residual / RMSE reduction
// with its scratch in a fixed file-scope device array instead.
//
// Scratch: kNoAllocPartials doubles (512 KiB) of static __device__ memory,
// held by every GPU that loads the library until the process exits.  Each
// block reduces a fixed chunk of kNoAllocChunk nonzeros into one slot, so
// at most kNoAllocPartials * kNoAllocChunk = 2^30 nonzeros fit; larger
// inputs are rejected.  Every call overwrites the slots it uses before
// reading them (nothing needs clearing), and all calls share the array:
// calls that overlap on the GPU (different streams, or several host
// threads) race on it.
//
// The device address of the array is looked up once per device, with that
// device current, on the first call made there: that first call should come
// before any stream capture on the device.  With CUDA's lazy module loading
// (the default), the library's device code and this array are loaded onto a
// device by that same first call (or the first launch of any kernel of the
// library there), and loading takes device memory: make the first call, or
// a warm-up call, before another allocator reserves the device's memory.
//
// Inputs are read with 16-byte vector loads: rec, U0, U1 and U2 must be
// 16-byte aligned (out_sse 8-byte aligned), which is checked before any
// launch.  The kernel trusts the indices: each record's i0, i1, i2 must be
// below the row count of U0, U1, U2.
#include "ctc_internal.h"

#include <cuda_runtime.h>

#include <mutex>

namespace {

// block-wide double sum, result in thread 0
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

constexpr int kNoAllocPartials = 65536;
constexpr uint64_t kNoAllocChunk = 16384;  // nonzeros per block
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

std::mutex g_addr_mu;
double *g_addr[kMaxDevices] = {};

// device address of the scratch for the current device (looked up once)
double *scratch_for_current_device(int *err)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *err = CTC_E_CUDA;
        ctc::set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "device ordinal out of range");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p) {
            *err = CTC_E_CUDA;
            ctc::set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "no symbol address");
            return nullptr;
        }
        g_addr[dev] = static_cast<double *>(p);
    }
    return g_addr[dev];
}

// k_sse with a fixed chunk per block: block b sums nonzeros
// [b*chunk, min((b+1)*chunk, n)) into partial[b].
template <int R>
__global__ void __launch_bounds__(kNoAllocThreads) k_sse_chunked(const uint4 *__restrict__ rec, uint64_t n,
                                                               const float *__restrict__ U0,
                                                               const float *__restrict__ U1,
                                                               const float *__restrict__ U2,
                                                               double *__restrict__ partial)
{
    const uint64_t begin = (uint64_t)blockIdx.x * kNoAllocChunk;
    const uint64_t end = min(begin + kNoAllocChunk, n);
    double acc = 0;
    for (uint64_t idx = begin + threadIdx.x; idx < end; idx += blockDim.x) {
        const uint4 r = rec[idx];
        const float4 *a = reinterpret_cast<const float4 *>(U0 + (size_t)r.x * R);
        const float4 *b = reinterpret_cast<const float4 *>(U1 + (size_t)r.y * R);
        const float4 *c = reinterpret_cast<const float4 *>(U2 + (size_t)r.z * R);
        float p = 0;
#pragma unroll
        for (int q = 0; q < R / 4; ++q) {
            const float4 va = a[q], vb = b[q], vc = c[q];
            p += va.x * vb.x * vc.x + va.y * vb.y * vc.y + va.z * vb.z * vc.z + va.w * vb.w * vc.w;
        }
        const float e = __uint_as_float(r.w) - p;
        acc += (double)e * (double)e;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// *out = sum of partial[0..n) in a fixed order (one block)
__global__ void __launch_bounds__(256) k_fold_partials(const double *__restrict__ partial, int n,
                                                       double *__restrict__ out)
{
    double acc = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

}  // namespace

extern "C" int ctc_sse_noalloc(const void *rec, uint64_t n, const float *U0, const float *U1,
                               const float *U2, int rank, double *out_sse, void *stream)
{
    if (!rec || !U0 || !U1 || !U2 || !out_sse) {
        ctc::set_last_error("ctc_sse_noalloc: null pointer argument");
        return CTC_E_ARG;
    }
    if ((reinterpret_cast<uintptr_t>(rec) | reinterpret_cast<uintptr_t>(U0) | reinterpret_cast<uintptr_t>(U1) |
         reinterpret_cast<uintptr_t>(U2)) & 15u) {
        ctc::set_last_error("ctc_sse_noalloc: rec, U0, U1 and U2 must be 16-byte aligned");
        return CTC_E_ARG;
    }
    if (reinterpret_cast<uintptr_t>(out_sse) & 7u) {
        ctc::set_last_error("ctc_sse_noalloc: out_sse must be 8-byte aligned");
        return CTC_E_ARG;
    }
    if (n == 0) {
        ctc::set_last_error("ctc_sse_noalloc: no nonzeros");
        return CTC_E_ARG;
    }
    if (n > (uint64_t)kNoAllocPartials * kNoAllocChunk) {
        ctc::set_last_error("ctc_sse_noalloc: more than 2^30 nonzeros exceeds the fixed scratch "
                            "(65536 partial sums of 16384 nonzeros); use ctc_rmse");
        return CTC_E_ARG;
    }
    if (rank != 8 && rank != 16 && rank != 32 && rank != 64) {
        ctc::set_last_error("ctc_sse_noalloc: rank must be 8, 16, 32 or 64");
        return CTC_E_UNSUP;
    }
    int err = CTC_OK;
    double *scratch = scratch_for_current_device(&err);
    if (!scratch) return err;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const unsigned blocks = (unsigned)((n + kNoAllocChunk - 1) / kNoAllocChunk);
    const uint4 *r = static_cast<const uint4 *>(rec);
    switch (rank) {
    case 8: k_sse_chunked<8><<<blocks, kNoAllocThreads, 0, s>>>(r, n, U0, U1, U2, scratch); break;
    case 16: k_sse_chunked<16><<<blocks, kNoAllocThreads, 0, s>>>(r, n, U0, U1, U2, scratch); break;
    case 32: k_sse_chunked<32><<<blocks, kNoAllocThreads, 0, s>>>(r, n, U0, U1, U2, scratch); break;
    default: k_sse_chunked<64><<<blocks, kNoAllocThreads, 0, s>>>(r, n, U0, U1, U2, scratch); break;
    }
    k_fold_partials<<<1, 256, 0, s>>>(scratch, (int)blocks, out_sse);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctc::set_last_error(cudaGetErrorString(e));
        return CTC_E_CUDA;
    }
    return CTC_OK;
}
