// fo.cuh -- kernels of the first-order (adjoint-driven) training mode:
// the gradient of the masked CP loss
//     f = 1/2 sum_Omega (x - sum_r prod_m U_m(i_m, r))^2 + lambda sum_m ||U_m||^2
// for order-3 and order-4 tensors in one pass over a minibatch (residual
// recomputed, never stored), the dense Adam step on FP32 master factors
// with a BF16 copy for the gathers, and the squared error for evaluation.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "kernels.cuh"

namespace ctc {
namespace fo {

// One 16-byte gather of VE consecutive elements of a factor row,
// converted to the arithmetic type T.
template <typename T, typename GT>
struct Gather;

template <>
struct Gather<float, float> {
    static constexpr int VE = 4;
    __device__ __forceinline__ static void load(const float *p, float (&u)[4])
    {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        u[0] = v.x;
        u[1] = v.y;
        u[2] = v.z;
        u[3] = v.w;
    }
};

// BF16 copies: 8-byte gathers of 4 elements, so that a nonzero takes the
// same R / 4 lanes as in FP32 (fewer nonzeros per warp instruction keep
// fewer colliding reductions on hot rows in one instruction)
template <>
struct Gather<float, __nv_bfloat16> {
    static constexpr int VE = 4;
    __device__ __forceinline__ static void load(const __nv_bfloat16 *p, float (&u)[4])
    {
        const uint2 raw = *reinterpret_cast<const uint2 *>(p);
        // a BF16 value is the high half of the FP32 value with the same bits
        u[0] = __uint_as_float(raw.x << 16);
        u[1] = __uint_as_float(raw.x & 0xffff0000u);
        u[2] = __uint_as_float(raw.y << 16);
        u[3] = __uint_as_float(raw.y & 0xffff0000u);
    }
};

template <>
struct Gather<double, double> {
    static constexpr int VE = 2;
    __device__ __forceinline__ static void load(const double *p, double (&u)[2])
    {
        const double2 v = *reinterpret_cast<const double2 *>(p);
        u[0] = v.x;
        u[1] = v.y;
    }
};

struct FoArgs {
    const uint4 *idx;       // 0-based indices of modes 0..3 (mode 3 unused at order 3)
    const void *val;        // values (T)
    uint64_t begin, end;    // nonzeros [begin, end) of this launch
    const void *U[4];       // gathered factors (GT), row-major dims x R
    void *G[4];             // gradient accumulators (T), row-major dims x R
    uint32_t dims[4];
    int priv[4];            // 1: the mode's gradient rows live in shared memory
    uint32_t priv_off[4];   // their offset in shared memory (elements)
    uint32_t priv_elems;    // total privatised elements
    double scale;           // data-term gradient scale (nonzeros / batch size)
    int bulk;               // 1: gradient rows of the other modes added by bulk row reductions
};

__device__ __forceinline__ void red_add4(float *p, float a, float b, float c, float d)
{
    atomicAdd(reinterpret_cast<float4 *>(p), make_float4(a, b, c, d));
}

// Group of GL = R / VE lanes per nonzero (lane gl holds elements gl*VE ..
// gl*VE+VE-1 of every row); groups stride over [begin, end).  GRAD adds
// -e * prod_{n != m} U_n(i_n, :) * scale into G_m; always accumulates
// 1/2 e^2 into per-block partials (fixed-order reduction).
template <typename T, typename GT, int R, int D, bool GRAD>
__global__ void __launch_bounds__(256) k_fo(FoArgs a, double *__restrict__ partial)
{
    using Gt = Gather<T, GT>;
    constexpr int VE = Gt::VE;
    constexpr int GL = R / VE;
    constexpr int GPW = 32 / GL;
    static_assert(GL >= 1 && 32 % GL == 0, "lanes per nonzero");
    constexpr bool kPriv = GRAD && std::is_same<T, float>::value;
    extern __shared__ __align__(16) float fo_smem[];
    const int lane = threadIdx.x & 31;
    const int gl = lane % GL, gw = lane / GL;
    const uint32_t gmask = (GL == 32) ? 0xffffffffu : (((1u << GL) - 1u) << (gw * GL));
    if constexpr (kPriv) {
        for (uint32_t i = threadIdx.x; i < a.priv_elems; i += blockDim.x) fo_smem[i] = 0.f;
        __syncthreads();
    }
    const uint64_t group = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * GPW + gw;
    const uint64_t ngroups = (((uint64_t)gridDim.x * blockDim.x) >> 5) * GPW;
    const T *vals = static_cast<const T *>(a.val);
    // bulk mode (FP32): a nonzero's gradient rows of the modes not kept in
    // shared memory are staged in the group's slot (two, alternating) and
    // added by one bulk reduction per mode, issued by the group's lane 0;
    // nothing reads G during the pass, so the reductions can land late
    const bool bulk = kPriv && a.bulk;
    float *stage = fo_smem + a.priv_elems +
                   (size_t)((threadIdx.x >> 5) * GPW + gw) * (2 * D * R);
    uint32_t nstaged = 0;
    double obj = 0;
    for (uint64_t p = a.begin + group; p < a.end; p += ngroups) {
        const uint4 ix = a.idx[p];
        const uint32_t row[4] = {ix.x, ix.y, ix.z, ix.w};
        const T x = vals[p];
        T u[D][VE];
#pragma unroll
        for (int m = 0; m < D; ++m)
            Gt::load(static_cast<const GT *>(a.U[m]) + (size_t)row[m] * R + gl * VE, u[m]);
        T part = 0;
#pragma unroll
        for (int v = 0; v < VE; ++v) {
            T pr = u[0][v];
#pragma unroll
            for (int m = 1; m < D; ++m) pr *= u[m][v];
            part += pr;
        }
#pragma unroll
        for (int o = GL / 2; o > 0; o >>= 1) part += __shfl_xor_sync(gmask, part, o);
        const T e = x - part;
        if (gl == 0) obj += 0.5 * (double)e * (double)e;
        if constexpr (GRAD) {
            const T se = -e * (T)a.scale;
            float *buf = stage + (nstaged & 1) * (D * R);
            if (bulk) {
                // the slot staged two nonzeros ago has been read by its reductions
                if (gl == 0) px::bulk_wait_read<1>();
                __syncwarp(gmask);
            }
#pragma unroll
            for (int m = 0; m < D; ++m) {
                T g[VE];
#pragma unroll
                for (int v = 0; v < VE; ++v) {
                    T pr = se;
#pragma unroll
                    for (int n = 0; n < D; ++n)
                        if (n != m) pr *= u[n][v];
                    g[v] = pr;
                }
                const size_t off = (size_t)row[m] * R + gl * VE;
                if constexpr (kPriv) {
                    if (a.priv[m]) {
                        float *s = fo_smem + a.priv_off[m] + off;
#pragma unroll
                        for (int v = 0; v < VE; ++v) atomicAdd(s + v, g[v]);
                        continue;
                    }
                }
                T *dst = static_cast<T *>(a.G[m]) + off;
                if constexpr (std::is_same<T, float>::value) {
                    if (bulk) {
#pragma unroll
                        for (int v = 0; v < VE; v += 4)
                            *reinterpret_cast<float4 *>(buf + m * R + gl * VE + v) =
                                make_float4(g[v], g[v + 1], g[v + 2], g[v + 3]);
                        continue;
                    }
#pragma unroll
                    for (int v = 0; v < VE; v += 4) red_add4(dst + v, g[v], g[v + 1], g[v + 2], g[v + 3]);
                } else {
#pragma unroll
                    for (int v = 0; v < VE; ++v) atomicAdd(dst + v, g[v]);
                }
            }
            if constexpr (kPriv) {
                if (bulk) {
                    px::fence_proxy_async_smem();
                    __syncwarp(gmask);
                    if (gl == 0) {
#pragma unroll
                        for (int m = 0; m < D; ++m)
                            if (!a.priv[m])
                                px::bulk_reduce_add_f32(static_cast<float *>(a.G[m]) + (size_t)row[m] * R,
                                                        buf + m * R, R * sizeof(float));
                        px::bulk_commit();
                    }
                    ++nstaged;
                }
            }
        }
    }
    if (bulk && gl == 0) px::bulk_wait_all();
    obj = k::block_sum(obj);
    if (threadIdx.x == 0) partial[blockIdx.x] = obj;
    if constexpr (kPriv) {
        __syncthreads();
#pragma unroll
        for (int m = 0; m < D; ++m)
            if (a.priv[m]) {
                float *dst = static_cast<float *>(a.G[m]);
                const uint32_t n = a.dims[m] * (uint32_t)R;
                for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                    const float v = fo_smem[a.priv_off[m] + i];
                    if (v != 0.f) atomicAdd(dst + i, v);
                }
            }
    }
}

// Dense Adam step on all factor entries (modes concatenated):
//   g = G + 2 lambda U ; m = b1 m + (1 - b1) g ; v = b2 v + (1 - b2) g^2
//   U -= lr * (m c1) / (sqrt(v c2) + eps)      (c1, c2: bias corrections)
// then G = 0 for the next step and, when Ub is given, Ub = BF16(U).
static __global__ void __launch_bounds__(256) k_fo_adam(float *__restrict__ U, float *__restrict__ M,
                                                 float *__restrict__ Vv, float *__restrict__ G,
                                                 __nv_bfloat16 *__restrict__ Ub, uint64_t n, float lr, float b1,
                                                 float b2, float eps, float c1, float c2, float lam2)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float u = U[i];
        const float g = G[i] + lam2 * u;
        const float m = b1 * M[i] + (1.f - b1) * g;
        const float v = b2 * Vv[i] + (1.f - b2) * g * g;
        const float un = u - lr * (m * c1) / (sqrtf(v * c2) + eps);
        U[i] = un;
        M[i] = m;
        Vv[i] = v;
        G[i] = 0.f;
        if (Ub) Ub[i] = __float2bfloat16_rn(un);
    }
}

// Counter-based shuffle keys: splitmix64 of (seed, i).
static __global__ void k_fo_keys(uint64_t *__restrict__ keys, uint32_t *__restrict__ ids, uint64_t n, uint64_t seed)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        keys[i] = z ^ (z >> 31);
        ids[i] = (uint32_t)i;
    }
}

template <typename T>
__global__ void k_fo_gather(const uint32_t *__restrict__ perm, const uint4 *__restrict__ idx_in,
                            const T *__restrict__ val_in, uint4 *__restrict__ idx_out, T *__restrict__ val_out,
                            uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = perm[i];
        idx_out[i] = idx_in[s];
        val_out[i] = val_in[s];
    }
}

}  // namespace fo
}  // namespace ctc
