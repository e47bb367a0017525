// vbd_mlp.cu -- learned warm start for the VBD step (no reference counterpart).
//
// A per-vertex MLP 64 -> 128 -> 128 -> 3 with SiLU activations predicts the step's correction
// to the inertia target (x_solved - y) from one-ring features; the Gauss-Seidel iterations then
// start from y + prediction instead of y.  Every product accumulates in FP32 on the tensor cores.
// Inference (vbd_mlp_forward; in the step mode also the features and the start, one launch) runs
// on tcgen05.mma with FP16 operands and TMEM accumulators (vbd_mlp_tc.cuh).  Training is
// hand-written too, on BF16 mma.sync m16n8k16 tiles with FP32 master weights:
//   * mlp_tile_kernel: per warp, 16 samples through the three layers with the activations handed
//     from one layer's accumulator fragments to the next layer's A fragments in registers; in
//     training mode it continues with the backward pass (dY, dH2 = dY W3^T, dZ2, dH1 = dZ2 W2^T,
//     dZ1) and stores the BF16 operands of the weight gradients;
//   * gemm_tn_kernel: dW = A^T B over the sample dimension (split-K, FP32 partials), then a
//     deterministic reduction; column sums give the bias gradients;
//   * adam_kernel: Adam on FP32 master weights, refreshing the BF16 copies.
// Fragment layouts are those of the PTX ISA for mma.m16n8k16 (A row-major, B column-major):
// lane = 4*g + t holds A rows g and g+8 at columns 2t, 2t+1 (+8), B column g at rows 2t, 2t+1
// (+8), and C rows g and g+8 at columns 2t, 2t+1; ldmatrix (with .trans where the stored
// layout is the transpose) produces them from shared memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "vbd_internal.h"
#include "vbd_math.cuh"
#include "vbd_mlp_tc.cuh"

namespace vbd {

namespace {

constexpr int kIn = 64, kHid = 128, kOut = 3, kOutP = 8;
constexpr int kStrideH = kHid + 8;  // bf16 row stride in shared memory (conflict-free ldmatrix)
constexpr int kStrideX = kIn + 8;
constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
// FP32 parameter blob: W1 [64][128] | b1 [128] | W2 [128][128] | b2 [128] | W3 [128][8] | b3 [8]
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kIn * kHid, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kOutP, kParams = kOffB3 + kOutP;
// BF16 weight blob: W1 [64][128] | W2 [128][128] | W3 [128][8]
constexpr int kW16W1 = 0, kW16W2 = kIn * kHid, kW16W3 = kW16W2 + kHid * kHid, kW16 = kW16W3 + kHid * kOutP;
static_assert(kParams == 25864 && kW16 == 25600, "blob layout");

__device__ __forceinline__ unsigned saddr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(saddr(p)));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(saddr(p)));
}
__device__ __forceinline__ void ldsm_x2(unsigned& r0, unsigned& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(saddr(p)));
}
__device__ __forceinline__ void ldsm_x2_t(unsigned& r0, unsigned& r1, const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(saddr(p)));
}
__device__ __forceinline__ void mma16816(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ unsigned pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned*>(&v);
}
__device__ __forceinline__ float2 unpack2(unsigned u) {
    __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162*>(&u);
    return __bfloat1622float2(v);
}
__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.0f + z * (1.0f - s));
}

struct MlpArgs {
    int n;
    const float* params;     // FP32 blob (biases read from it)
    const uint16_t* w16;     // BF16 weight blob
    const float* X;          // [n][64]
    float* Y;                // [n][3] or NULL
    // training
    const float* T;          // [n][3] targets or NULL (inference)
    float grad_scale;        // dL/dY = grad_scale * 2 (y - t)
    float* loss;             // sum of squared errors (monitoring; atomic)
    __nv_bfloat16* Xb;       // [n][64]
    __nv_bfloat16* H1;       // [n][128]
    __nv_bfloat16* H2;       // [n][128]
    __nv_bfloat16* dZ1;      // [n][128]
    __nv_bfloat16* dZ2;      // [n][128]
    __nv_bfloat16* dY;       // [n][8]
};

constexpr size_t kTileSmem = (size_t)(kIn * kStrideH + kHid * kStrideH + kHid * kOutP + kWarps * 16 * kStrideX) * 2 +
                             (size_t)(kHid + kHid + kOutP) * 4;

template <bool kTrain>
__global__ void __launch_bounds__(kThreads) mlp_tile_kernel(MlpArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sW1 = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* sW2 = sW1 + kIn * kStrideH;
    __nv_bfloat16* sW3 = sW2 + kHid * kStrideH;
    __nv_bfloat16* sX = sW3 + kHid * kOutP;
    float* sB1 = reinterpret_cast<float*>(sX + kWarps * 16 * kStrideX);
    float* sB2 = sB1 + kHid;
    float* sB3 = sB2 + kHid;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t4 = lane & 3;
    // weights -> shared (16-byte chunks), biases
    const uint4* gw = reinterpret_cast<const uint4*>(a.w16);
    for (int i = tid; i < kIn * kHid / 8; i += kThreads) {
        const int r = i / (kHid / 8), c = (i % (kHid / 8)) * 8;
        *reinterpret_cast<uint4*>(sW1 + r * kStrideH + c) = gw[(kW16W1 / 8) + i];
    }
    for (int i = tid; i < kHid * kHid / 8; i += kThreads) {
        const int r = i / (kHid / 8), c = (i % (kHid / 8)) * 8;
        *reinterpret_cast<uint4*>(sW2 + r * kStrideH + c) = gw[(kW16W2 / 8) + i];
    }
    for (int i = tid; i < kHid * kOutP / 8; i += kThreads)
        *reinterpret_cast<uint4*>(sW3 + i * 8) = gw[(kW16W3 / 8) + i];
    for (int i = tid; i < kHid; i += kThreads) {
        sB1[i] = a.params[kOffB1 + i];
        sB2[i] = a.params[kOffB2 + i];
    }
    if (tid < kOutP) sB3[tid] = a.params[kOffB3 + tid];
    __syncthreads();
    __nv_bfloat16* myX = sX + warp * 16 * kStrideX;
    const int ntiles = (a.n + 15) / 16;
    const int jj = lane >> 3, rr = lane & 7;  // ldmatrix: matrix index, row inside the matrix
    for (int tile = blockIdx.x * kWarps + warp; tile < ntiles; tile += gridDim.x * kWarps) {
        const int row0 = tile * 16;
        // X rows -> bf16 in shared memory (zeros past n)
        for (int i = lane; i < 16 * kIn / 2; i += 32) {
            const int r = i / (kIn / 2), c = (i % (kIn / 2)) * 2;
            float2 v = make_float2(0.f, 0.f);
            if (row0 + r < a.n) v = *reinterpret_cast<const float2*>(a.X + (size_t)(row0 + r) * kIn + c);
            *reinterpret_cast<unsigned*>(myX + r * kStrideX + c) = pack2(v.x, v.y);
        }
        __syncwarp();
        if (kTrain) {
            for (int i = lane; i < 16 * kIn / 8; i += 32) {
                const int r = i / (kIn / 8), c = (i % (kIn / 8)) * 8;
                if (row0 + r < a.n)
                    *reinterpret_cast<uint4*>(a.Xb + (size_t)(row0 + r) * kIn + c) =
                        *reinterpret_cast<const uint4*>(myX + r * kStrideX + c);
            }
        }
        // ---- layer 1: Z1 = X W1 + b1 ----
        unsigned ax[4][4];
        for (int kt = 0; kt < 4; ++kt) ldsm_x4(ax[kt], myX + (lane & 15) * kStrideX + kt * 16 + (lane >> 4) * 8);
        float acc[16][4];
        for (int nt = 0; nt < 16; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        for (int kt = 0; kt < 4; ++kt)
            for (int np = 0; np < 8; ++np) {
                unsigned b[4];
                ldsm_x4_t(b, sW1 + (kt * 16 + (jj & 1) * 8 + rr) * kStrideH + (2 * np + (jj >> 1)) * 8);
                mma16816(acc[2 * np], ax[kt], b[0], b[1]);
                mma16816(acc[2 * np + 1], ax[kt], b[2], b[3]);
            }
        unsigned z1p[16][2];  // Z1 kept as bf16 pairs for the backward pass
        unsigned ah[8][4];    // H1 as A fragments of layer 2
        for (int nt = 0; nt < 16; ++nt) {
            const int c = nt * 8 + 2 * t4;
            const float z0 = acc[nt][0] + sB1[c], z1 = acc[nt][1] + sB1[c + 1];
            const float z2 = acc[nt][2] + sB1[c], z3 = acc[nt][3] + sB1[c + 1];
            if (kTrain) {
                z1p[nt][0] = pack2(z0, z1);
                z1p[nt][1] = pack2(z2, z3);
            }
            ah[nt >> 1][(nt & 1) * 2 + 0] = pack2(silu(z0), silu(z1));
            ah[nt >> 1][(nt & 1) * 2 + 1] = pack2(silu(z2), silu(z3));
        }
        if (kTrain) {
            for (int nt = 0; nt < 16; ++nt) {
                const int c = nt * 8 + 2 * t4;
                if (row0 + g < a.n)
                    *reinterpret_cast<unsigned*>(a.H1 + (size_t)(row0 + g) * kHid + c) = ah[nt >> 1][(nt & 1) * 2];
                if (row0 + g + 8 < a.n)
                    *reinterpret_cast<unsigned*>(a.H1 + (size_t)(row0 + g + 8) * kHid + c) =
                        ah[nt >> 1][(nt & 1) * 2 + 1];
            }
        }
        // ---- layer 2: Z2 = H1 W2 + b2 ----
        for (int nt = 0; nt < 16; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        for (int kt = 0; kt < 8; ++kt) {
            const unsigned a2[4] = {ah[kt][0], ah[kt][1], ah[kt][2], ah[kt][3]};
            for (int np = 0; np < 8; ++np) {
                unsigned b[4];
                ldsm_x4_t(b, sW2 + (kt * 16 + (jj & 1) * 8 + rr) * kStrideH + (2 * np + (jj >> 1)) * 8);
                mma16816(acc[2 * np], a2, b[0], b[1]);
                mma16816(acc[2 * np + 1], a2, b[2], b[3]);
            }
        }
        unsigned z2p[16][2];  // Z2 kept as bf16 pairs for the backward pass
        for (int nt = 0; nt < 16; ++nt) {
            const int c = nt * 8 + 2 * t4;
            acc[nt][0] += sB2[c];
            acc[nt][1] += sB2[c + 1];
            acc[nt][2] += sB2[c];
            acc[nt][3] += sB2[c + 1];
            if (kTrain) {
                z2p[nt][0] = pack2(acc[nt][0], acc[nt][1]);
                z2p[nt][1] = pack2(acc[nt][2], acc[nt][3]);
            }
            ah[nt >> 1][(nt & 1) * 2 + 0] = pack2(silu(acc[nt][0]), silu(acc[nt][1]));
            ah[nt >> 1][(nt & 1) * 2 + 1] = pack2(silu(acc[nt][2]), silu(acc[nt][3]));
        }
        if (kTrain) {
            for (int nt = 0; nt < 16; ++nt) {
                const int c = nt * 8 + 2 * t4;
                if (row0 + g < a.n)
                    *reinterpret_cast<unsigned*>(a.H2 + (size_t)(row0 + g) * kHid + c) = ah[nt >> 1][(nt & 1) * 2];
                if (row0 + g + 8 < a.n)
                    *reinterpret_cast<unsigned*>(a.H2 + (size_t)(row0 + g + 8) * kHid + c) =
                        ah[nt >> 1][(nt & 1) * 2 + 1];
            }
        }
        // ---- layer 3: Y = H2 W3 + b3 ----
        float y[4] = {0.f, 0.f, 0.f, 0.f};
        for (int kt = 0; kt < 8; ++kt) {
            const unsigned a3[4] = {ah[kt][0], ah[kt][1], ah[kt][2], ah[kt][3]};
            unsigned b0, b1;
            ldsm_x2_t(b0, b1, sW3 + (kt * 16 + (jj & 1) * 8 + rr) * kOutP);
            mma16816(y, a3, b0, b1);
        }
        const int c0 = 2 * t4;
        y[0] += sB3[c0];
        y[1] += sB3[c0 + 1];
        y[2] += sB3[c0];
        y[3] += sB3[c0 + 1];
        if (a.Y) {
            for (int h = 0; h < 2; ++h) {
                const int r = row0 + g + 8 * h;
                if (r >= a.n) continue;
                if (c0 < kOut) a.Y[(size_t)r * kOut + c0] = y[2 * h];
                if (c0 + 1 < kOut) a.Y[(size_t)r * kOut + c0 + 1] = y[2 * h + 1];
            }
        }
        if (!kTrain) continue;
        // ---- backward ----
        float dy[4] = {0.f, 0.f, 0.f, 0.f};
        float se = 0.f;
        for (int h = 0; h < 2; ++h) {
            const int r = row0 + g + 8 * h;
            if (r >= a.n) continue;
            for (int q = 0; q < 2; ++q) {
                const int c = c0 + q;
                if (c >= kOut) continue;
                const float e = y[2 * h + q] - a.T[(size_t)r * kOut + c];
                se += e * e;
                dy[2 * h + q] = a.grad_scale * 2.0f * e;
            }
        }
        for (int off = 16; off > 0; off >>= 1) se += __shfl_xor_sync(0xffffffffu, se, off);
        if (lane == 0 && a.loss) atomicAdd(a.loss, se);
        if (row0 + g < a.n)
            *reinterpret_cast<unsigned*>(a.dY + (size_t)(row0 + g) * kOutP + c0) = pack2(dy[0], dy[1]);
        if (row0 + g + 8 < a.n)
            *reinterpret_cast<unsigned*>(a.dY + (size_t)(row0 + g + 8) * kOutP + c0) = pack2(dy[2], dy[3]);
        // dH2 = dY W3^T   (A = dY padded to K = 16; B[k][n] = W3[n][k])
        const unsigned ady[4] = {pack2(dy[0], dy[1]), pack2(dy[2], dy[3]), 0u, 0u};
        for (int nt = 0; nt < 16; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        for (int np = 0; np < 8; ++np) {
            unsigned b0, b1;  // matrices: rows n of tile 2np, rows n of tile 2np+1 (k 0..7)
            ldsm_x2(b0, b1, sW3 + ((2 * np + (jj & 1)) * 8 + rr) * kOutP);
            mma16816(acc[2 * np], ady, b0, 0u);
            mma16816(acc[2 * np + 1], ady, b1, 0u);
        }
        unsigned adz2[8][4];
        for (int nt = 0; nt < 16; ++nt) {
            const int c = nt * 8 + 2 * t4;
            const float2 za = unpack2(z2p[nt][0]), zb = unpack2(z2p[nt][1]);
            const float d0 = acc[nt][0] * dsilu(za.x), d1 = acc[nt][1] * dsilu(za.y);
            const float d2 = acc[nt][2] * dsilu(zb.x), d3 = acc[nt][3] * dsilu(zb.y);
            adz2[nt >> 1][(nt & 1) * 2 + 0] = pack2(d0, d1);
            adz2[nt >> 1][(nt & 1) * 2 + 1] = pack2(d2, d3);
            if (row0 + g < a.n) *reinterpret_cast<unsigned*>(a.dZ2 + (size_t)(row0 + g) * kHid + c) = pack2(d0, d1);
            if (row0 + g + 8 < a.n)
                *reinterpret_cast<unsigned*>(a.dZ2 + (size_t)(row0 + g + 8) * kHid + c) = pack2(d2, d3);
        }
        // dH1 = dZ2 W2^T  (B[k][n] = W2[n][k]: plain ldmatrix on rows n)
        for (int nt = 0; nt < 16; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
        for (int kt = 0; kt < 8; ++kt) {
            const unsigned a2[4] = {adz2[kt][0], adz2[kt][1], adz2[kt][2], adz2[kt][3]};
            for (int np = 0; np < 8; ++np) {
                unsigned b[4];  // matrices: (tile 2np, k 0-7), (tile 2np, k 8-15), (tile 2np+1, k 0-7), (.., k 8-15)
                ldsm_x4(b, sW2 + ((2 * np + (jj >> 1)) * 8 + rr) * kStrideH + kt * 16 + (jj & 1) * 8);
                mma16816(acc[2 * np], a2, b[0], b[1]);
                mma16816(acc[2 * np + 1], a2, b[2], b[3]);
            }
        }
        for (int nt = 0; nt < 16; ++nt) {
            const int c = nt * 8 + 2 * t4;
            const float2 za = unpack2(z1p[nt][0]), zb = unpack2(z1p[nt][1]);
            const float d0 = acc[nt][0] * dsilu(za.x), d1 = acc[nt][1] * dsilu(za.y);
            const float d2 = acc[nt][2] * dsilu(zb.x), d3 = acc[nt][3] * dsilu(zb.y);
            if (row0 + g < a.n) *reinterpret_cast<unsigned*>(a.dZ1 + (size_t)(row0 + g) * kHid + c) = pack2(d0, d1);
            if (row0 + g + 8 < a.n)
                *reinterpret_cast<unsigned*>(a.dZ1 + (size_t)(row0 + g + 8) * kHid + c) = pack2(d2, d3);
        }
    }
}

// dW[M][N] = sum_s A[s][m] * B[s][n] for s in this split's sample range (FP32 partials).
constexpr int kGemmK = 32;
__global__ void __launch_bounds__(128) gemm_tn_kernel(int S, const __nv_bfloat16* A, int M, const __nv_bfloat16* B,
                                                       int N, int samples_per_split, float* part) {
    __shared__ __align__(16) __nv_bfloat16 sA[kGemmK][64 + 8];
    __shared__ __align__(16) __nv_bfloat16 sB[kGemmK][64 + 8];
    const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64, split = blockIdx.z;
    const int s_begin = split * samples_per_split, s_end = min(S, s_begin + samples_per_split);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t4 = lane & 3, jj = lane >> 3, rr = lane & 7;
    const int nN = min(64, N - n0);
    float acc[8][4];
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    for (int s0 = s_begin; s0 < s_end; s0 += kGemmK) {
        for (int i = tid; i < kGemmK * 8; i += 128) {  // 32 rows x 8 chunks of 8 bf16
            const int r = i >> 3, c = (i & 7) * 8;
            const int s = s0 + r;
            uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
            if (s < s_end) {
                va = *reinterpret_cast<const uint4*>(A + (size_t)s * M + m0 + c);
                if (c < nN) vb = *reinterpret_cast<const uint4*>(B + (size_t)s * N + n0 + c);
            }
            *reinterpret_cast<uint4*>(&sA[r][c]) = va;
            *reinterpret_cast<uint4*>(&sB[r][c]) = vb;
        }
        __syncthreads();
        for (int kt = 0; kt < kGemmK / 16; ++kt) {
            unsigned af[4];
            ldsm_x4_t(af, &sA[kt * 16 + (jj >> 1) * 8 + rr][warp * 16 + (jj & 1) * 8]);
            for (int np = 0; np < 4; ++np) {
                unsigned b[4];
                ldsm_x4_t(b, &sB[kt * 16 + (jj & 1) * 8 + rr][(2 * np + (jj >> 1)) * 8]);
                mma16816(acc[2 * np], af, b[0], b[1]);
                mma16816(acc[2 * np + 1], af, b[2], b[3]);
            }
        }
        __syncthreads();
    }
    float* out = part + (size_t)split * M * N;
    for (int nt = 0; nt < 8; ++nt) {
        const int n = n0 + nt * 8 + 2 * t4;
        if (nt * 8 >= nN) continue;
        const int m = m0 + warp * 16 + g;
        out[(size_t)m * N + n] = acc[nt][0];
        out[(size_t)m * N + n + 1] = acc[nt][1];
        out[(size_t)(m + 8) * N + n] = acc[nt][2];
        out[(size_t)(m + 8) * N + n + 1] = acc[nt][3];
    }
}

// out[i] = sum over splits, in split order (deterministic).
__global__ void reduce_splits_kernel(const float* part, int splits, int count, float* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float s = 0.f;
    for (int k = 0; k < splits; ++k) s += part[(size_t)k * count + i];
    out[i] = s;
}

// column sums of a bf16 [S][C] matrix: per-block partials over row chunks, then reduce_splits
__global__ void colsum_kernel(int S, const __nv_bfloat16* D, int C, int rows_per_block, float* part) {
    const int c = threadIdx.x;
    if (c >= C) return;
    const int r0 = blockIdx.x * rows_per_block, r1 = min(S, r0 + rows_per_block);
    float s = 0.f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(D[(size_t)r * C + c]);
    part[(size_t)blockIdx.x * C + c] = s;
}

__global__ void adam_kernel(float* p, const float* gr, float* m1, float* m2, uint16_t* w16, int n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = gr[i];
    const float a = b1 * m1[i] + (1.0f - b1) * g;
    const float b = b2 * m2[i] + (1.0f - b2) * g * g;
    m1[i] = a;
    m2[i] = b;
    const float v = p[i] - lr * (a * c1) / (sqrtf(b * c2) + eps);
    p[i] = v;
    int widx = -1;
    if (i < kOffB1) widx = kW16W1 + i;
    else if (i >= kOffW2 && i < kOffB2) widx = kW16W2 + (i - kOffW2);
    else if (i >= kOffW3 && i < kOffB3) widx = kW16W3 + (i - kOffW3);
    if (widx >= 0) {
        __nv_bfloat16 h = __float2bfloat16_rn(v);
        w16[widx] = *reinterpret_cast<uint16_t*>(&h);
    }
}

__global__ void to_bf16_kernel(const float* p, uint16_t* w16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    int widx = -1;
    if (i < kOffB1) widx = kW16W1 + i;
    else if (i >= kOffW2 && i < kOffB2) widx = kW16W2 + (i - kOffW2);
    else if (i >= kOffW3 && i < kOffB3) widx = kW16W3 + (i - kOffW3);
    if (widx >= 0) {
        __nv_bfloat16 h = __float2bfloat16_rn(p[i]);
        w16[widx] = *reinterpret_cast<uint16_t*>(&h);
    }
}

std::mutex g_attr_mutex;
bool g_attr_done[64] = {};

// waits of the tensor-core inference kernel that gave up (read by vbd_mlp_timeouts)
__device__ unsigned g_mlp_tc_timeouts;

int ensure_tile_smem() {
    int dev = 0;
    VBD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(VBD_ERR_UNSUPPORTED, "vbd_mlp: device ordinal too large");
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    if (!g_attr_done[dev]) {
        VBD_CUDA_TRY(cudaFuncSetAttribute(mlp_tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(kTileSmem)));
        VBD_CUDA_TRY(cudaFuncSetAttribute(mlp_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(kTileSmem)));
        VBD_CUDA_TRY(cudaFuncSetAttribute(tc::mlp_infer_tc_kernel<tc::kInF32>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes));
        VBD_CUDA_TRY(cudaFuncSetAttribute(tc::mlp_infer_tc_kernel<tc::kInStep>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes));
        g_attr_done[dev] = true;
    }
    return VBD_OK;
}

// persistent grid of the tensor-core inference kernel: one CTA (four tile pipelines) per SM
int tc_grid(int n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (n + tc::kRows - 1) / tc::kRows;
    return std::max(1, std::min(sms, (tiles + tc::kGroups - 1) / tc::kGroups));
}

int tile_grid(int n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int tiles = (n + 15) / 16;
    return std::max(1, std::min(sms * 2, (tiles + kWarps - 1) / kWarps));
}

// ---- features --------------------------------------------------------------------------------
struct FeatArgs {
    int V;
    const int* perm;
    const float4* pinfo;
    const float4* prev;
    const float4* y;
    const int* nbr8;
    const float4* vfeat;
    const int* ccount;
    const float* corr_prev;  // [V][3] model order, may be NULL
    const float* mean;       // [64] or NULL
    const float* inv_std;    // [64] or NULL
    float* out;              // [V][64], row = model index
    int mode;                // VBD_FEATURES_CORRECTIONS or VBD_FEATURES_KINEMATIC
    float3 g_dt2;            // gravity * dt^2 (kinematic set)
    float inv_dt;            // 1 / dt (kinematic set)
};

// Features, 8 lanes per vertex: lane j handles one-ring neighbour j (edge vector, and in the
// corrections set its previous correction), lane 0 the vertex's own terms; the row is assembled in
// shared memory and each lane writes 8 consecutive values (256 contiguous bytes per row), so no
// per-thread 64-value array and no 4-byte stores 256 bytes apart.
//
// Corrections set (VBD_FEATURES_CORRECTIONS), lengths in units of the vertex's mean rest edge L:
//   f[0..2] inertia offset (y - x);  f[3..5] the vertex's previous correction;
//   f[6+3j..8+3j] edge vector to neighbour j;  f[30+3j..32+3j] neighbour j's previous correction;
//   f[54..56] material log-stiffnesses;  f[57] log10 mass;  f[58] contact flag;
//   f[59] one-ring size / 8;  f[60] solvable flag;  f[63] 1
// Kinematic set (VBD_FEATURES_KINEMATIC): the vertex's own motion and its one-ring geometry, no
// solver history:
//   f[0..2] previous step's displacement v dt = (y - x) - g dt^2;  f[3..5] velocity v (m/s);
//   f[6..8] inertia offset (y - x);  f[9+3j..11+3j] edge vector to neighbour j;
//   f[33..35] material log-stiffnesses;  f[36] log10 mass;  f[37] contact flag;
//   f[38] one-ring size / 8;  f[39] solvable flag;  f[63] 1
constexpr int kFeatLanes = 8;
constexpr int kFeatBlock = 128;
constexpr int kFeatRows = kFeatBlock / kFeatLanes;
constexpr int kFeatStride = 68;  // floats per shared row (16-byte aligned, rows 4 banks apart)

__global__ void __launch_bounds__(kFeatBlock) features_kernel(FeatArgs a) {
    __shared__ __align__(16) float rows[kFeatRows * kFeatStride];
    const int t = threadIdx.x, vr = t / kFeatLanes, j = t % kFeatLanes;
    const int i = blockIdx.x * kFeatRows + vr;
    const bool valid = i < a.V;
    float* f = rows + vr * kFeatStride;
#pragma unroll
    for (int k = 0; k < 8; ++k) f[8 * j + k] = 0.f;
    __syncwarp();
    const bool kin = a.mode == VBD_FEATURES_KINEMATIC;
    int nb = -1;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f), vf = make_float4(0.f, 0.f, 0.f, 1.f);
    float3 x = f3(0.f, 0.f, 0.f);
    float invL = 1.f;
    if (valid) {
        pi = a.pinfo[i];
        vf = a.vfeat[i];
        invL = 1.0f / fmaxf(vf.w, 1e-9f);
        x = xyz(a.prev[i]);
        nb = a.nbr8[kFeatLanes * i + j];
        if (nb >= 0) {
            const float3 xn = xyz(a.prev[nb]);
            const int e = kin ? 9 + 3 * j : 6 + 3 * j;
            f[e] = (xn.x - x.x) * invL;
            f[e + 1] = (xn.y - x.y) * invL;
            f[e + 2] = (xn.z - x.z) * invL;
            if (!kin && a.corr_prev) {
                const int on = a.perm[nb];
                f[30 + 3 * j] = a.corr_prev[3 * on] * invL;
                f[31 + 3 * j] = a.corr_prev[3 * on + 1] * invL;
                f[32 + 3 * j] = a.corr_prev[3 * on + 2] * invL;
            }
        }
    }
    // one-ring size: the vertex's 8 lanes are consecutive lanes of one warp
    const unsigned have = __ballot_sync(0xffffffffu, nb >= 0);
    const int nn = __popc((have >> ((t & 31) & ~(kFeatLanes - 1))) & 0xffu);
    if (valid && j == 0) {
        const bool solvable = (__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f;
        const float3 yy = xyz(a.y[i]);
        const float3 off = f3(yy.x - x.x, yy.y - x.y, yy.z - x.z);
        const float mass = pi.x > 0.f ? log10f(pi.x) : 0.f;
        const float contact = (a.ccount && a.ccount[i] > 0) ? 1.f : 0.f;
        if (kin) {
            if (solvable) {
                const float3 vdt = f3(off.x - a.g_dt2.x, off.y - a.g_dt2.y, off.z - a.g_dt2.z);
                f[0] = vdt.x * invL;
                f[1] = vdt.y * invL;
                f[2] = vdt.z * invL;
                f[3] = vdt.x * a.inv_dt;
                f[4] = vdt.y * a.inv_dt;
                f[5] = vdt.z * a.inv_dt;
            }
            f[6] = off.x * invL;
            f[7] = off.y * invL;
            f[8] = off.z * invL;
            f[33] = vf.x;
            f[34] = vf.y;
            f[35] = vf.z;
            f[36] = mass;
            f[37] = contact;
            f[38] = nn * 0.125f;
            f[39] = solvable ? 1.f : 0.f;
        } else {
            f[0] = off.x * invL;
            f[1] = off.y * invL;
            f[2] = off.z * invL;
            if (a.corr_prev) {
                const int o = a.perm[i];
                f[3] = a.corr_prev[3 * o] * invL;
                f[4] = a.corr_prev[3 * o + 1] * invL;
                f[5] = a.corr_prev[3 * o + 2] * invL;
            }
            f[54] = vf.x;
            f[55] = vf.y;
            f[56] = vf.z;
            f[57] = mass;
            f[58] = contact;
            f[59] = nn * 0.125f;
            f[60] = solvable ? 1.f : 0.f;
        }
        f[63] = 1.f;
    }
    __syncwarp();
    if (!valid) return;
    const int row = a.perm[i];
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int c = 8 * j + k;
        v[k] = a.mean ? (f[c] - __ldg(&a.mean[c])) * __ldg(&a.inv_std[c]) : f[c];
    }
    float4* out = reinterpret_cast<float4*>(a.out + static_cast<size_t>(row) * 64 + 8 * j);
    out[0] = make_float4(v[0], v[1], v[2], v[3]);
    out[1] = make_float4(v[4], v[5], v[6], v[7]);
}

// delta = the bounded start (bounded_start) of each solvable vertex, 0 elsewhere, in model order.
// A zero network therefore leaves the solve exactly as plain VBD's.
__global__ void scale_prediction_kernel(int V, const int* perm, const float4* pinfo, const float4* vfeat,
                                        const float* pred, float* delta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const int o = perm[i];
    const float4 pi = pinfo[i];
    const bool solvable = (__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f;
    const float3 m = solvable ? bounded_start(pred[3 * o], pred[3 * o + 1], pred[3 * o + 2], vfeat[i].w)
                              : make_float3(0.f, 0.f, 0.f);
    delta[3 * o] = m.x;
    delta[3 * o + 1] = m.y;
    delta[3 * o + 2] = m.z;
}

}  // namespace

int mlp_features_launch(const VbdModelImpl& m, const float4* prev, const float4* y, const int* ccount,
                        const float* corr_prev, const float* mean, const float* inv_std, float* out, int mode,
                        float dt, cudaStream_t st) {
    if (mode != VBD_FEATURES_CORRECTIONS && mode != VBD_FEATURES_KINEMATIC)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_features: unknown feature set");
    if (mode == VBD_FEATURES_KINEMATIC && !(dt > 0.f))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_features: the kinematic set needs the step's dt (run vbd_forward first)");
    if (reinterpret_cast<uintptr_t>(out) & 15u)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_features: out must be 16-byte aligned");
    if (m.V == 0) return VBD_OK;
    FeatArgs f;
    f.mode = mode;
    f.g_dt2 = make_float3(m.gravity[0] * dt * dt, m.gravity[1] * dt * dt, m.gravity[2] * dt * dt);
    f.inv_dt = dt > 0.f ? 1.0f / dt : 0.f;
    f.V = m.V;
    f.perm = m.perm;
    f.pinfo = m.pinfo;
    f.prev = prev;
    f.y = y;
    f.nbr8 = m.nbr8;
    f.vfeat = m.vfeat;
    f.ccount = ccount;
    f.corr_prev = corr_prev;
    f.mean = mean;
    f.inv_std = inv_std;
    f.out = out;
    features_kernel<<<(m.V + kFeatRows - 1) / kFeatRows, kFeatBlock, 0, st>>>(f);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

int mlp_scale_launch(const VbdModelImpl& m, const float* pred, float* delta, cudaStream_t st) {
    if (m.V == 0) return VBD_OK;
    scale_prediction_kernel<<<(m.V + 255) / 256, 256, 0, st>>>(m.V, m.perm, m.pinfo, m.vfeat, pred, delta);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

}  // namespace vbd

using namespace vbd;

extern "C" int vbd_mlp_sizes(int32_t* params, int32_t* weights16, int32_t* in_features, int32_t* hidden,
                             int32_t* out_features) {
    if (params) *params = kParams;
    if (weights16) *weights16 = kW16;
    if (in_features) *in_features = kIn;
    if (hidden) *hidden = kHid;
    if (out_features) *out_features = kOut;
    return VBD_OK;
}

extern "C" int vbd_mlp_workspace_bytes(int32_t n, int64_t* bytes) {
    if (n < 0 || !bytes) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_workspace_bytes: bad arguments");
    const size_t rows = static_cast<size_t>(n);
    const int splits = 64;
    size_t b = rows * (kIn + 4 * kHid + kOutP) * 2;               // bf16 operands
    b = (b + 255) & ~static_cast<size_t>(255);
    b += static_cast<size_t>(splits) * kHid * kHid * 4;           // GEMM partials (largest)
    b += static_cast<size_t>(1024) * kHid * 4;                    // column-sum partials
    *bytes = static_cast<int64_t>(b);
    return VBD_OK;
}

namespace vbd {
// the tcgen05 inference on FP32 rows (weights: the FP32 blob, rounded to FP16 in the kernel)
static int tc_forward(const float* params, const float* X, int32_t n, float* Y, cudaStream_t st) {
    int rc = ensure_tile_smem();
    if (rc) return rc;
    if (n == 0) return VBD_OK;
    tc::TcArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.params = params;
    a.X = X;
    a.Y = Y;
    unsigned* counter = nullptr;
    VBD_CUDA_TRY(cudaGetSymbolAddress(reinterpret_cast<void**>(&counter), g_mlp_tc_timeouts));
    a.status = counter;
    a.off_w1 = kOffW1;
    a.off_b1 = kOffB1;
    a.off_w2 = kOffW2;
    a.off_b2 = kOffB2;
    a.off_w3 = kOffW3;
    a.off_b3 = kOffB3;
    tc::mlp_infer_tc_kernel<tc::kInF32><<<tc_grid(n), tc::kThreads, tc::kSmemBytes, st>>>(a);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

// The step mode's learned start in one launch: features of every internal vertex computed in the
// tcgen05 kernel, inference, and the bounded start applied to disp / pos (no feature or prediction
// rows in HBM).  Equal, bit for bit, to features -> inference -> scaled start of the staged API.
int mlp_step_start(const VbdModelImpl& m, const float* params, const float4* prev, const float4* y, const int* ccount,
                   const float* corr_prev, const float* mean, const float* inv_std, int mode, float dt, float4* disp,
                   float4* pos, cudaStream_t st) {
    if (mode != VBD_FEATURES_CORRECTIONS && mode != VBD_FEATURES_KINEMATIC)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd warm start: unknown feature set");
    if (mode == VBD_FEATURES_KINEMATIC && !(dt > 0.f))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd warm start: the kinematic set needs the step's dt");
    if (reinterpret_cast<uintptr_t>(m.nbr8) & 15u)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd warm start: misaligned neighbour table");
    int rc = ensure_tile_smem();
    if (rc) return rc;
    if (m.V == 0) return VBD_OK;
    tc::TcArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = m.V;
    a.params = params;
    a.step.pinfo = m.pinfo;
    a.step.prev = prev;
    a.step.y = y;
    a.step.nbr8 = m.nbr8;
    a.step.vfeat = m.vfeat;
    a.step.ccount = ccount;
    a.step.corr_prev = corr_prev;
    a.step.mean = mean;
    a.step.inv_std = inv_std;
    a.step.mode = mode;
    a.step.g_dt2 = make_float3(m.gravity[0] * dt * dt, m.gravity[1] * dt * dt, m.gravity[2] * dt * dt);
    a.step.inv_dt = dt > 0.f ? 1.0f / dt : 0.f;
    a.step.disp = disp;
    a.step.pos = pos;
    unsigned* counter = nullptr;
    VBD_CUDA_TRY(cudaGetSymbolAddress(reinterpret_cast<void**>(&counter), g_mlp_tc_timeouts));
    a.status = counter;
    a.off_w1 = kOffW1;
    a.off_b1 = kOffB1;
    a.off_w2 = kOffW2;
    a.off_b2 = kOffB2;
    a.off_w3 = kOffW3;
    a.off_b3 = kOffB3;
    tc::mlp_infer_tc_kernel<tc::kInStep><<<tc_grid(m.V), tc::kThreads, tc::kSmemBytes, st>>>(a);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}
}  // namespace vbd

extern "C" int vbd_mlp_forward(const float* params, const uint16_t* w16, const float* X, int32_t n, float* Y,
                               void* stream) {
    if (!params || !w16 || (n > 0 && (!X || !Y))) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_forward: NULL argument");
    if ((reinterpret_cast<uintptr_t>(X) & 15u) || (reinterpret_cast<uintptr_t>(w16) & 1u))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_forward: X must be 16-byte aligned");
    return tc_forward(params, X, n, Y, static_cast<cudaStream_t>(stream));
}

extern "C" int vbd_mlp_forward_mma_sync(const float* params, const uint16_t* w16, const float* X, int32_t n, float* Y,
                                        void* stream) {
    if (!params || !w16 || (n > 0 && (!X || !Y)))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_forward_mma_sync: NULL argument");
    int rc = ensure_tile_smem();
    if (rc) return rc;
    if (n == 0) return VBD_OK;
    MlpArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.params = params;
    a.w16 = w16;
    a.X = X;
    a.Y = Y;
    mlp_tile_kernel<false><<<tile_grid(n), kThreads, kTileSmem, static_cast<cudaStream_t>(stream)>>>(a);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_mlp_timeouts(uint32_t* count, int32_t reset) {
    if (!count) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_timeouts: count is NULL");
    VBD_CUDA_TRY(cudaMemcpyFromSymbol(count, g_mlp_tc_timeouts, sizeof(uint32_t)));
    if (reset) {
        const uint32_t zero = 0;
        VBD_CUDA_TRY(cudaMemcpyToSymbol(g_mlp_tc_timeouts, &zero, sizeof(uint32_t)));
    }
    return VBD_OK;
}

extern "C" int vbd_mlp_backward(const float* params, const uint16_t* w16, const float* X, const float* T, int32_t n,
                                float grad_scale, float* grads, float* loss, void* workspace, int64_t workspace_bytes,
                                void* stream) {
    if (!params || !w16 || !X || !T || !grads || !workspace || n <= 0)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_backward: bad arguments");
    int64_t need = 0;
    vbd_mlp_workspace_bytes(n, &need);
    if (workspace_bytes < need) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_backward: workspace too small");
    int rc = ensure_tile_smem();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t rows = static_cast<size_t>(n);
    __nv_bfloat16* base = static_cast<__nv_bfloat16*>(workspace);
    MlpArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.params = params;
    a.w16 = w16;
    a.X = X;
    a.T = T;
    a.grad_scale = grad_scale;
    a.loss = loss;
    a.Xb = base;
    a.H1 = a.Xb + rows * kIn;
    a.H2 = a.H1 + rows * kHid;
    a.dZ1 = a.H2 + rows * kHid;
    a.dZ2 = a.dZ1 + rows * kHid;
    a.dY = a.dZ2 + rows * kHid;
    size_t off = rows * (kIn + 4 * kHid + kOutP) * 2;
    off = (off + 255) & ~static_cast<size_t>(255);
    float* part = reinterpret_cast<float*>(static_cast<unsigned char*>(workspace) + off);
    float* cpart = part + static_cast<size_t>(64) * kHid * kHid;
    mlp_tile_kernel<true><<<tile_grid(n), kThreads, kTileSmem, st>>>(a);
    VBD_CUDA_TRY(cudaGetLastError());
    const int splits = std::min(64, (n + 511) / 512);
    const int per_split = ((n + splits - 1) / splits + kGemmK - 1) / kGemmK * kGemmK;
    auto dW = [&](const __nv_bfloat16* Am, int M, const __nv_bfloat16* Bm, int N, float* out) -> int {
        dim3 grid(M / 64, (N + 63) / 64, splits);
        gemm_tn_kernel<<<grid, 128, 0, st>>>(n, Am, M, Bm, N, per_split, part);
        reduce_splits_kernel<<<(M * N + 255) / 256, 256, 0, st>>>(part, splits, M * N, out);
        VBD_CUDA_TRY(cudaGetLastError());
        return VBD_OK;
    };
    auto db = [&](const __nv_bfloat16* D, int C, float* out) -> int {
        const int blocks = std::min(1024, (n + 255) / 256);
        const int rpb = (n + blocks - 1) / blocks;
        colsum_kernel<<<blocks, 128, 0, st>>>(n, D, C, rpb, cpart);
        reduce_splits_kernel<<<(C + 255) / 256, 256, 0, st>>>(cpart, blocks, C, out);
        VBD_CUDA_TRY(cudaGetLastError());
        return VBD_OK;
    };
    if ((rc = dW(a.Xb, kIn, a.dZ1, kHid, grads + kOffW1))) return rc;
    if ((rc = db(a.dZ1, kHid, grads + kOffB1))) return rc;
    if ((rc = dW(a.H1, kHid, a.dZ2, kHid, grads + kOffW2))) return rc;
    if ((rc = db(a.dZ2, kHid, grads + kOffB2))) return rc;
    if ((rc = dW(a.H2, kHid, a.dY, kOutP, grads + kOffW3))) return rc;
    if ((rc = db(a.dY, kOutP, grads + kOffB3))) return rc;
    return VBD_OK;
}

extern "C" int vbd_mlp_adam(float* params, const float* grads, float* m1, float* m2, uint16_t* w16, int32_t step,
                            float lr, float beta1, float beta2, float eps, void* stream) {
    if (!params || !grads || !m1 || !m2 || !w16 || step < 1)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_adam: bad arguments");
    const float c1 = 1.0f / (1.0f - powf(beta1, static_cast<float>(step)));
    const float c2 = 1.0f / (1.0f - powf(beta2, static_cast<float>(step)));
    adam_kernel<<<(kParams + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grads, m1, m2, w16,
                                                                                       kParams, lr, beta1, beta2,
                                                                                       eps, c1, c2);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_mlp_pack_weights(const float* params, uint16_t* w16, void* stream) {
    if (!params || !w16) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_pack_weights: NULL argument");
    to_bf16_kernel<<<(kParams + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, w16);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}
