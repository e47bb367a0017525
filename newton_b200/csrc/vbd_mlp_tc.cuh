// vbd_mlp_tc.cuh -- inference of the warm-start MLP (64 -> 128 -> 128 -> 3, SiLU) on the 5th-
// generation tensor cores: tcgen05.mma with BF16 operands in shared memory and FP32 accumulators
// in tensor memory (TMEM).  Included by vbd_mlp.cu only.
//
// Work split.  A persistent CTA of 128 threads owns one 128-row tile of samples at a time; thread
// t owns row t (TMEM lane t).  Per tile:
//   1. all threads stage the tile's features as BF16 in shared memory (A1, 128 x 64);
//   2. thread 0 issues layer 1: D1[128 x 128] = A1 W1 (4 MMAs of K = 16) and commits to an
//      mbarrier; every thread waits, reads its row of D1 from TMEM (tcgen05.ld), adds the bias,
//      applies SiLU and writes the BF16 row into A2 (128 x 128);
//   3. layer 2 likewise: D2 = A2 W2 (8 MMAs), epilogue back into A2 (its MMAs have completed);
//   4. layer 3: D3[128 x 16] = A2 W3 (8 MMAs, N padded from 3 to 16, D3 reuses D1's columns);
//      the epilogue adds the bias and stores the 3 outputs.
// Two CTAs run per SM (about 100 KB of shared memory and 256 TMEM columns each), so one CTA's
// MMAs run while the other works through an epilogue.
//
// Shared-memory operand layout: the canonical K-major layout without swizzle.  An operand of R
// rows by K columns is cut into 8 x 8 "core matrices" (8 rows of 16 bytes, 128 contiguous bytes);
// element (r, k) sits at byte ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.  In
// the matrix descriptor, the leading-dimension byte offset (between the two K halves of one
// MMA's K = 16 slice) is (R / 8) * 128 and the stride-dimension byte offset (between 8-row
// groups) is 128; the slice for MMA step s starts at byte s * 2 * (R / 8) * 128.  B operands are
// the weights transposed to [N][K] (K-major), written once per CTA.
//
// Every wait on the mbarrier is bounded: after kTcSpinLimit polls the kernel records a timeout
// (the whole CTA decides together), stops taking tiles, waits (bounded again) for the MMAs it has
// issued, frees its TMEM and returns.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace vbd {
namespace tc {

constexpr int kRows = 128;                   // samples per tile (MMA M, TMEM lanes)
constexpr int kThreads = 128;
constexpr int kN3 = 16;                      // layer-3 MMA N (3 outputs, padded)
constexpr uint32_t kTmemCols = 256;          // D1 [0, 128), D2 [128, 256), D3 reuses [0, 16)
constexpr unsigned kTcSpinLimit = 1u << 26;  // polls of one mbarrier wait before giving up

// shared-memory carve-up (bytes, 1024-aligned blocks)
constexpr int kSzW1 = 128 * 64 * 2;    // B of layer 1: [128][64]
constexpr int kSzW2 = 128 * 128 * 2;   // B of layer 2: [128][128]
constexpr int kSzW3 = kN3 * 128 * 2;   // B of layer 3: [16][128]
constexpr int kSzA1 = kRows * 64 * 2;  // features
constexpr int kSzA2 = kRows * 128 * 2; // hidden activations (layer 1 out, then layer 2 out)
constexpr int kOffW1 = 0;
constexpr int kOffW2 = kOffW1 + kSzW1;
constexpr int kOffW3 = kOffW2 + kSzW2;
constexpr int kOffA1 = kOffW3 + kSzW3;
constexpr int kOffA2 = kOffA1 + kSzA1;
constexpr int kOffBias = kOffA2 + kSzA2;             // b1[128] b2[128] b3[16] (float)
constexpr int kOffBar = kOffBias + (128 + 128 + 16) * 4;  // mbarrier (8 B), TMEM address (4 B)
constexpr int kSmemBytes = kOffBar + 16 + 1024;      // + slack for aligning the base to 1024 B

// byte offset of element (r, k) in an R-row K-major no-swizzle operand
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int R) {
    return static_cast<uint32_t>(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// matrix descriptor: start address, LBO, SBO (all >> 4), version 1 (bits 46-47), no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: D F32, A and B BF16, both K-major, N >> 3, M >> 4
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bar_init(uint32_t bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// one poll of the mbarrier's phase `parity`; true once that phase has completed
__device__ __forceinline__ bool bar_test(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// bounded wait; false after kTcSpinLimit polls
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    for (unsigned k = 0; k < kTcSpinLimit; ++k)
        if (bar_test(bar, parity)) return true;
    return false;
}

// 32 consecutive FP32 columns of this thread's TMEM lane (the load and its wait in one statement,
// so that no use of the registers can be scheduled before the wait)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// SiLU(z) = z * sigmoid(z), sigmoid(z) = 1/2 + tanh(z / 2) / 2 with the hardware tanh approximation
// (relative error ~2^-11, below the BF16 rounding the activations get next)
__device__ __forceinline__ float silu_fast(float z) {
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
    return z * fmaf(0.5f, t, 0.5f);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// bias + SiLU of 32 accumulator columns [c0, c0 + 32) of row r, stored as BF16 into an R = 128 row
// K-major operand (4 stores of 16 bytes)
__device__ __forceinline__ void store_hidden32(unsigned char* A, int r, int c0, const float (&acc)[32],
                                               const float* bias) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint4 w;
        uint32_t* wp = reinterpret_cast<uint32_t*>(&w);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = q * 8 + 2 * j;
            wp[j] = pack_bf16(silu_fast(acc[c] + bias[c0 + c]), silu_fast(acc[c + 1] + bias[c0 + c + 1]));
        }
        *reinterpret_cast<uint4*>(A + kmajor_offset(r, c0 + q * 8, kRows)) = w;
    }
}

struct TcArgs {
    int n;
    const float* params;  // FP32 blob (biases)
    const uint16_t* w16;  // BF16 weights: W1 [64][128] | W2 [128][128] | W3 [128][8]
    const float* X;       // [n][64]
    float* Y;             // [n][3]
    unsigned* status;     // incremented on a wait that gave up (may be NULL)
    int off_b1, off_b2, off_b3;
};

__global__ void __launch_bounds__(kThreads, 2) mlp_infer_tc_kernel(TcArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sW1 = smem + kOffW1;
    unsigned char* sW2 = smem + kOffW2;
    unsigned char* sW3 = smem + kOffW3;
    unsigned char* sA1 = smem + kOffA1;
    unsigned char* sA2 = smem + kOffA2;
    float* sB1 = reinterpret_cast<float*>(smem + kOffBias);
    float* sB2 = sB1 + 128;
    float* sB3 = sB2 + 128;
    uint64_t* bar_p = reinterpret_cast<uint64_t*>(smem + kOffBar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kOffBar + 8);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t bar = smem_u32(bar_p);

    // ---- set-up: weights transposed into the B layouts, biases, mbarrier, TMEM -----------------
    for (int i = tid; i < 64 * 128; i += kThreads) {  // W1[k][n] -> B1[n][k]
        const int k = i / 128, nn = i % 128;
        *reinterpret_cast<uint16_t*>(sW1 + kmajor_offset(nn, k, 128)) = a.w16[i];
    }
    for (int i = tid; i < 128 * 128; i += kThreads) {  // W2[k][n] -> B2[n][k]
        const int k = i / 128, nn = i % 128;
        *reinterpret_cast<uint16_t*>(sW2 + kmajor_offset(nn, k, 128)) = a.w16[64 * 128 + i];
    }
    for (int i = tid; i < kN3 * 128; i += kThreads) {  // W3[k][n] (8 columns) -> B3[n][k], rows 8..15 zero
        const int nn = i / 128, k = i % 128;
        const uint16_t w = nn < 8 ? a.w16[64 * 128 + 128 * 128 + k * 8 + nn] : uint16_t(0);
        *reinterpret_cast<uint16_t*>(sW3 + kmajor_offset(nn, k, kN3)) = w;
    }
    for (int i = tid; i < 128; i += kThreads) {
        sB1[i] = a.params[a.off_b1 + i];
        sB2[i] = a.params[a.off_b2 + i];
    }
    if (tid < kN3) sB3[tid] = tid < 8 ? a.params[a.off_b3 + tid] : 0.f;
    if (tid == 0) {
        bar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t d1 = tmem, d2 = tmem + 128, d3 = tmem;
    const uint32_t lane_base = static_cast<uint32_t>(warp * 32) << 16;  // this warp's TMEM lanes
    const uint32_t idesc128 = instr_desc(128, 128), idesc16 = instr_desc(128, kN3);
    const uint32_t a1 = smem_u32(sA1), a2 = smem_u32(sA2), w1 = smem_u32(sW1), w2 = smem_u32(sW2),
                   w3 = smem_u32(sW3);
    uint32_t phase = 0;
    bool ok = true;
    const int ntiles = (a.n + kRows - 1) / kRows;

    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int row0 = tile * kRows;
        // ---- 1. features -> A1 (BF16), 16 threads per row, coalesced float4 loads ----
        for (int f = tid; f < kRows * 16; f += kThreads) {
            const int r = f >> 4, c4 = f & 15;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (row0 + r < a.n) v = __ldg(reinterpret_cast<const float4*>(a.X + static_cast<size_t>(row0 + r) * 64) + c4);
            uint2 w;
            w.x = pack_bf16(v.x, v.y);
            w.y = pack_bf16(v.z, v.w);
            *reinterpret_cast<uint2*>(sA1 + kmajor_offset(r, 4 * c4, kRows)) = w;
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        // ---- 2. layer 1 ----
        if (tid == 0) {
            fence_after();
#pragma unroll
            for (int s = 0; s < 4; ++s)
                mma_bf16(d1, smem_desc(a1 + s * 2 * 2048, 2048, 128), smem_desc(w1 + s * 2 * 2048, 2048, 128),
                         idesc128, s > 0 ? 1u : 0u);
            mma_commit(bar);
        }
        ok = __syncthreads_and(bar_wait(bar, phase) ? 1 : 0) != 0;  // one decision for the whole CTA
        if (!ok) break;
        phase ^= 1u;
        fence_after();
        {
            const int r = tid;
#pragma unroll 1
            for (int c0 = 0; c0 < 128; c0 += 32) {
                float acc[32];
                tmem_ld32(d1 + lane_base + c0, acc);
                store_hidden32(sA2, r, c0, acc, sB1);
            }
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        // ---- 3. layer 2 ----
        if (tid == 0) {
            fence_after();
#pragma unroll
            for (int s = 0; s < 8; ++s)
                mma_bf16(d2, smem_desc(a2 + s * 2 * 2048, 2048, 128), smem_desc(w2 + s * 2 * 2048, 2048, 128),
                         idesc128, s > 0 ? 1u : 0u);
            mma_commit(bar);
        }
        ok = __syncthreads_and(bar_wait(bar, phase) ? 1 : 0) != 0;  // one decision for the whole CTA
        if (!ok) break;
        phase ^= 1u;
        fence_after();
        {
            const int r = tid;
#pragma unroll 1
            for (int c0 = 0; c0 < 128; c0 += 32) {
                float acc[32];
                tmem_ld32(d2 + lane_base + c0, acc);
                store_hidden32(sA2, r, c0, acc, sB2);  // layer 2's MMAs have completed: A2 is free
            }
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        // ---- 4. layer 3 ----
        if (tid == 0) {
            fence_after();
#pragma unroll
            for (int s = 0; s < 8; ++s)
                mma_bf16(d3, smem_desc(a2 + s * 2 * 2048, 2048, 128), smem_desc(w3 + s * 2 * 256, 256, 128),
                         idesc16, s > 0 ? 1u : 0u);
            mma_commit(bar);
        }
        ok = __syncthreads_and(bar_wait(bar, phase) ? 1 : 0) != 0;  // one decision for the whole CTA
        if (!ok) break;
        phase ^= 1u;
        fence_after();
        {
            float y[16];
            tmem_ld16(d3 + lane_base, y);
            const int r = row0 + tid;
            if (r < a.n) {
                float* out = a.Y + static_cast<size_t>(r) * 3;
                out[0] = y[0] + sB3[0];
                out[1] = y[1] + sB3[1];
                out[2] = y[2] + sB3[2];
            }
        }
        fence_before();
        __syncthreads();  // D1..D3 and A1/A2 are free for the next tile
    }
    if (!ok) {
        // a wait gave up: record it, then wait (bounded) for the MMAs this CTA issued before freeing
        // their TMEM (the last commit tracks all of them)
        if (tid == 0 && a.status) atomicAdd(a.status, 1u);
        bar_wait(bar, phase);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

}  // namespace tc
}  // namespace vbd
