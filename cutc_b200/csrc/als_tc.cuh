// als_tc.cuh -- ALS Gram blocks on the 5th-generation tensor cores
// (tcgen05.mma, accumulator in tensor memory), ranks 64 and 32, mixed
// precision.
//
// For one piece of a long row (tile_len nonzeros of one row of the mode's
// sorted copy) the CTA forms
//     G = sum_k h_k h_k^T      (R x R, FP32 in TMEM)
//     b = sum_k x_k h_k        (R, FP32 on the CUDA cores)
// with h_k = U_a(q1) o U_b(q2) read from BF16 copies of the factors, and
// writes them to the piece's slot ({G row-major, b}, the layout the FP64
// fixup solve k_als_fix reads).
//
// The h rows of a chunk of nonzeros are staged in shared memory as BF16,
// 128-byte rows with the 128-byte swizzle (16-byte chunk c of row k stored
// at chunk c ^ (k & 7), 1 KiB aligned).  Read as an MN-major
// operand that tile is both A = H^T (M = 64 x K) and B = H (K x N = 64), so
// each tcgen05.mma (M=64, N=64, K=16, kind::f16, BF16 in, FP32 out)
// accumulates 16 nonzeros of h h^T.  One thread issues the MMAs and commits
// them to an mbarrier; the CTA waits with a bounded spin, then each warp
// reads its quarter of the accumulator (for M = 64, rows 16w..16w+15 live in
// TMEM lanes 32w..32w+15) with tcgen05.ld.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ptx.cuh"

namespace ctc {
namespace tc {

constexpr int kThreads = 128;  // one 128-byte operand row per thread and chunk

using px::smem_u32;
using px::mbar_try_wait;
using px::mbar_wait_bounded;

// UMMA shared-memory descriptor: MN-major, 128-byte swizzle, SM100 version 1
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr)
{
    const uint64_t start = (addr >> 4) & 0x3FFFull;
    const uint64_t lbo = 1ull;                 // one 64-element block along MN: unused
    const uint64_t sbo = (1024u >> 4) & 0x3FFFull;  // 8 rows x 128 B between row groups
    return start | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
}

// instruction descriptor: D F32, A/B BF16, both MN-major, M = 64, N = 64
__host__ __device__ constexpr uint32_t idesc_bf16_m64_n64()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((64u >> 3) << 17) |
           ((64u >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar_addr)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_addr)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld_32x32b_x64(uint32_t taddr, uint32_t (&v)[64])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]),
          "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]),
          "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]),
          "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]),
          "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// Gram + right-hand side of the heavy pieces listed in `pieces` (tile
// indices of the mode's plan), rank R = 64 or 32; slot[t] = {G (R x R
// row-major), b (R)}.  err[0] is set when a bounded wait expires.
//
// Operand rows are 128 bytes, one per thread and chunk.  At R = 64 a row
// is one nonzero's h (a chunk is 128 nonzeros).  At R = 32 a row holds two
// nonzeros, h(c0 + t) in its first 64 bytes and h(c0 + 128 + t) in its
// second: the 64 x 64 product of such rows has the Grams of the two halves
// on its diagonal blocks (the off-diagonal blocks are not read), so a chunk
// is 256 nonzeros in 128 rows and 8 MMAs, and G = block(0,0) + block(1,1),
// added in that order.
//
// Two operand tiles alternate: while the MMAs of one chunk run, the CTA
// gathers the next chunk into the other tile; a tile is rewritten only
// after the MMAs that read it have arrived on its mbarrier.
template <int R>
__global__ void __launch_bounds__(kThreads, R == 64 ? 2 : 4)
    k_als_gram_tc(const int4 *__restrict__ tiles, const uint32_t *__restrict__ pieces, uint32_t npieces,
                  const uint4 *__restrict__ rec, int m, const __nv_bfloat16 *__restrict__ Ua,
                  const __nv_bfloat16 *__restrict__ Ub, float *__restrict__ slot, int *err)
{
    static_assert(R == 64 || R == 32, "tensor-core Gram ranks");
    constexpr int kVec = R / 8;           // 16-byte words of a BF16 factor row
    constexpr int kNz = kThreads * (64 / R);  // nonzeros per chunk: 128 rows of 128 bytes
    constexpr int kRows = kThreads;       // operand rows per chunk
    constexpr int kTile = kRows * 128;    // bytes per operand tile
    constexpr int kLpn = kVec;            // lanes per nonzero in the gathers (one word each)
    constexpr int kNpi = 32 / kLpn;       // nonzeros per warp and gather step
    constexpr int kIt = kNz / 4 / kNpi;   // gather steps per warp and chunk (8)
    extern __shared__ uint8_t dsm[];
    uint8_t *hs0 = dsm + ((1024u - (smem_u32(dsm) & 1023u)) & 1023u);
    __shared__ float rhs_part[kThreads / 32][R];
    __shared__ float gsum[R == 32 ? 32 * 32 : 1];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m1 = (m + 1) % 3, m2 = (m + 2) % 3;
    const uint32_t idesc = idesc_bf16_m64_n64();
    // gathers: warp w takes the chunk's nonzeros w*kNz/4 .. (w+1)*kNz/4 - 1,
    // kNpi per step, lane (word, n) = (lane % kLpn, lane / kLpn)
    const int word = lane % kLpn;
    const int nz0 = warp * (kNz / 4) + lane / kLpn;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "r"(64u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[b])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_d = tmem_base_sh;
    // bit b: the phase tile b's mbarrier completes next / MMAs reading tile b
    // are in flight (bits, not arrays, so they stay in registers)
    uint32_t phases = 0u, pending = 0u;
    uint32_t nchunk = 0;  // chunks issued by this CTA (selects the tile)
    bool ok = true;
    // wait for the MMAs that read tile b (every thread; the outcome is made
    // CTA-uniform so that no thread leaves while others sit at a barrier)
    auto drain = [&](int b) {
        if (!((pending >> b) & 1u) || !ok) return;
        const int got = mbar_wait_bounded(smem_u32(&mbar[b]), (phases >> b) & 1u) ? 1 : 0;
        ok = __syncthreads_and(got) != 0;
        phases ^= 1u << b;
        pending &= ~(1u << b);
    };

    for (uint32_t pi = blockIdx.x; pi < npieces && ok; pi += gridDim.x) {
        const uint32_t tile = pieces[pi];
        const int4 td = tiles[tile];
        const uint32_t start = (uint32_t)td.x, end = start + (uint32_t)td.y;
        // this lane's slice of the right-hand side: columns 8*word .. 8*word+7
        float rhs[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) rhs[e] = 0.f;
        // records of the piece's first chunk; later chunks' records are
        // fetched while the current chunk's rows are gathered
        uint4 rn[kIt];
#pragma unroll
        for (int it = 0; it < kIt; ++it) {
            const uint32_t p = start + nz0 + it * kNpi;
            rn[it] = p < end ? rec[p] : make_uint4(0u, 0u, 0u, 0u);
        }
        for (uint32_t c0 = start; c0 < end && ok; c0 += kNz) {
            const int b = (int)(nchunk & 1u);
            drain(b);
            if (!ok) break;
            uint8_t *hs = hs0 + b * kTile;
            // the group of kLpn lanes of nonzero k = nz0 + it * kNpi loads
            // word `word` of its two factor rows: one L1 wavefront per row
            uint4 va[kIt], vb[kIt];
            float x[kIt];
#pragma unroll
            for (int it = 0; it < kIt; ++it) {
                x[it] = __uint_as_float(rn[it].w);
                if (c0 + nz0 + it * kNpi < end) {
                    const uint32_t q1 = m1 == 0 ? rn[it].x : (m1 == 1 ? rn[it].y : rn[it].z);
                    const uint32_t q2 = m2 == 0 ? rn[it].x : (m2 == 1 ? rn[it].y : rn[it].z);
                    va[it] = reinterpret_cast<const uint4 *>(Ua + (size_t)q1 * R)[word];
                    vb[it] = reinterpret_cast<const uint4 *>(Ub + (size_t)q2 * R)[word];
                }
            }
#pragma unroll
            for (int it = 0; it < kIt; ++it) {
                const uint32_t pn = c0 + kNz + nz0 + it * kNpi;
                rn[it] = pn < end ? rec[pn] : make_uint4(0u, 0u, 0u, 0u);
            }
#pragma unroll
            for (int it = 0; it < kIt; ++it) {
                // nonzero k of the chunk fills segment k / kThreads of operand row k % kThreads
                const int k = nz0 + it * kNpi;
                const int orow = k % kThreads, seg = k / kThreads;
                uint4 out = make_uint4(0u, 0u, 0u, 0u);
                if (c0 + k < end) {
                    const __nv_bfloat162 *pa = reinterpret_cast<const __nv_bfloat162 *>(&va[it]);
                    const __nv_bfloat162 *pb = reinterpret_cast<const __nv_bfloat162 *>(&vb[it]);
                    uint32_t outw[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float2 fa = __bfloat1622float2(pa[q]);
                        const float2 fb = __bfloat1622float2(pb[q]);
                        const float h0 = fa.x * fb.x, h1 = fa.y * fb.y;
                        rhs[2 * q] += x[it] * h0;
                        rhs[2 * q + 1] += x[it] * h1;
                        outw[q] = pack_bf16(h0, h1);
                    }
                    out = make_uint4(outw[0], outw[1], outw[2], outw[3]);
                }
                *reinterpret_cast<uint4 *>(hs + orow * 128 + (((seg * kVec + word) ^ (orow & 7)) << 4)) = out;
            }
            // make the generic-proxy stores visible to the tensor core
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                // rows past the chunk's nonzeros are zero in every segment
                const uint32_t rows = min(end - c0, (uint32_t)kRows);
                const uint32_t nmma = (rows + 15) / 16;
                const uint32_t hs_addr = smem_u32(hs);
                for (uint32_t kk = 0; kk < nmma; ++kk) {
                    const uint64_t d = smem_desc_sw128(hs_addr + kk * 16 * 128);
                    mma_bf16(tmem_d, d, d, idesc, (c0 != start || kk != 0) ? 1u : 0u);
                }
                mma_commit(smem_u32(&mbar[b]));
            }
            pending |= 1u << b;
            ++nchunk;
        }
        // the accumulator is complete once both tiles' MMAs have arrived
        drain(0);
        drain(1);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // right-hand side: sum the slices of the lanes that hold the same
        // word (butterflies over the nonzero bits of the lane), then a
        // fixed-order sum over warps
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            float v = rhs[e];
#pragma unroll
            for (int o = 16; o >= kLpn; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane < kLpn) rhs_part[warp][8 * lane + e] = v;
        }
        // accumulator rows 16w..16w+15 live in TMEM lanes 32w..32w+15
        uint32_t g[64];
        tmem_ld_32x32b_x64(tmem_d + ((uint32_t)(32 * warp) << 16), g);
        float *dst = slot + (size_t)tile * (R * R + R);
        if constexpr (R == 64) {
            if (lane < 16) {
                const int grow = 16 * warp + lane;
                float4 *d4 = reinterpret_cast<float4 *>(dst + grow * R);
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    d4[q] = make_float4(__uint_as_float(g[4 * q]), __uint_as_float(g[4 * q + 1]),
                                        __uint_as_float(g[4 * q + 2]), __uint_as_float(g[4 * q + 3]));
            }
        } else {
            // block (1,1): accumulator rows 32..63, columns 32..63 (warps 2, 3)
            if (warp >= 2 && lane < 16) {
                const int grow = 16 * (warp - 2) + lane;
#pragma unroll
                for (int q = 0; q < 32; ++q) gsum[grow * 32 + q] = __uint_as_float(g[32 + q]);
            }
            __syncthreads();
            // block (0,0): rows 0..31, columns 0..31 (warps 0, 1), plus block (1,1)
            if (warp < 2 && lane < 16) {
                const int grow = 16 * warp + lane;
                float4 *d4 = reinterpret_cast<float4 *>(dst + grow * R);
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    d4[q] = make_float4(__uint_as_float(g[4 * q]) + gsum[grow * 32 + 4 * q],
                                        __uint_as_float(g[4 * q + 1]) + gsum[grow * 32 + 4 * q + 1],
                                        __uint_as_float(g[4 * q + 2]) + gsum[grow * 32 + 4 * q + 2],
                                        __uint_as_float(g[4 * q + 3]) + gsum[grow * 32 + 4 * q + 3]);
            }
        }
        __syncthreads();
        if (tid < R) dst[R * R + tid] = ((rhs_part[0][tid] + rhs_part[1][tid]) + rhs_part[2][tid]) + rhs_part[3][tid];
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (!ok) {
        // report, and give the MMAs in flight one more bounded wait each
        // before the tensor memory they write is released
        if (tid == 0) atomicExch(err, 1);
        for (int b = 0; b < 2; ++b)
            if ((pending >> b) & 1u) mbar_wait_bounded(smem_u32(&mbar[b]), (phases >> b) & 1u);
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(64u));
}

// dynamic shared memory of k_als_gram_tc<R>: two operand tiles of kThreads
// 128-byte rows + alignment
template <int R>
constexpr int gram_smem_bytes()
{
    return 2 * kThreads * 128 + 1024;
}

// FP32 factor rows -> BF16 copies (row-major, same shape)
static __global__ void k_to_bf16(const float *__restrict__ src, __nv_bfloat16 *__restrict__ dst, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

}  // namespace tc
}  // namespace ctc
