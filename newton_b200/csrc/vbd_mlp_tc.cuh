// vbd_mlp_tc.cuh -- inference of the warm-start MLP (64 -> 128 -> 128 -> 3, SiLU) on the 5th-
// generation tensor cores: tcgen05.mma with FP16 operands in shared memory and FP32 accumulators
// in tensor memory (TMEM); bias + SiLU in f16x2 arithmetic.  Included by vbd_mlp.cu only.
//
// Work split.  One persistent CTA of 512 threads per SM runs four independent tile pipelines
// ("groups" of 4 warps) over one shared copy of the weights.  A group owns one 128-row tile of
// samples at a time; its warp q reads TMEM lanes [32 q, 32 q + 32), the rows of those samples, and
// thread 32 q + l owns row 32 q + l.  Per tile, in the group's 32 KB operand buffer and its 128 TMEM
// columns:
//   1. the group stages the tile's features as FP16 (128 x 64, the first 16 KB of the buffer), read
//      from FP32 rows or, in the step mode, computed from the solver's arrays;
//   2. the group's first thread issues layer 1, D[128 x 128] = X W1 (4 MMAs of K = 16), and
//      commits to the group's mbarrier; each thread waits, reads its row of D (tcgen05.ld), adds
//      the bias, applies SiLU and writes the FP16 row into the buffer (X is no longer needed);
//   3. layer 2 likewise: D = H1 W2 (8 MMAs, D's columns reused), epilogue back into the buffer;
//   4. layer 3: D[128 x 16] = H2 W3 (8 MMAs, N padded from 3 to 16); the epilogue adds the bias
//      and stores the 3 outputs (the step mode: applies the start).
// Each step of a tile waits on the previous one (MMA -> epilogue -> MMA); four tiles in flight per
// SM keep the tensor core busy across those waits.
//
// Shared-memory operand layout: the canonical K-major layout without swizzle.  An operand of R
// rows by K columns is cut into 8 x 8 "core matrices" (8 rows of 16 bytes, 128 contiguous bytes);
// element (r, k) sits at byte ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.  In
// the matrix descriptor, the leading-dimension byte offset (between the two K halves of one
// MMA's K = 16 slice) is (R / 8) * 128 and the stride-dimension byte offset (between 8-row
// groups) is 128; the slice for MMA step s starts at byte s * 2 * (R / 8) * 128.  B operands are
// the FP32 weights rounded to FP16 and transposed to [N][K] (K-major), written once per CTA.
// FP16 (11-bit significand) rather than BF16 (8-bit) operands: the values of this network
// (standardized features, activations of a few units, weights below 1) are far inside FP16's
// range, and the rounding of the inputs limits how well the start carries the previous correction
// (measured on the draped cloth: fewer Gauss-Seidel iterations after an FP16 start than after a
// BF16 one; on batched worlds the same).
//
// Every wait on an mbarrier is bounded: after kTcSpinLimit polls the group records a timeout (its
// four warps decide together), stops taking tiles, waits (bounded again) for the MMAs it has
// issued, and the CTA frees its TMEM and returns.
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

namespace vbd {
namespace tc {

constexpr int kRows = 128;                   // samples per tile (MMA M, TMEM lanes)
constexpr int kGroups = 4;                   // tile pipelines per CTA
constexpr int kGroupThreads = 128;           // 4 warps, one per TMEM lane quarter
constexpr int kThreads = kGroups * kGroupThreads;
constexpr uint32_t kTmemCols = 512;          // 128 per group: D of layer 1, then of layer 2, then 3
constexpr unsigned kTcSpinLimit = 1u << 26;  // polls of one mbarrier wait before giving up

// shared-memory carve-up (bytes, 1024-aligned blocks)
constexpr int kSzW1 = 128 * 64 * 2;    // B of layer 1: [128][64]
constexpr int kSzW2 = 128 * 128 * 2;   // B of layer 2: [128][128]
constexpr int kN3 = 16;                 // layer-3 MMA N (3 outputs, padded)
constexpr int kSzW3 = kN3 * 128 * 2;    // B of layer 3: [16][128]
constexpr int kSzBuf = kRows * 128 * 2;  // per group: features (16 KB), then hidden activations (FP16)
constexpr int kOffW1 = 0;
constexpr int kOffW2 = kOffW1 + kSzW1;
constexpr int kOffW3 = kOffW2 + kSzW2;
constexpr int kOffBuf = kOffW3 + kSzW3;
constexpr int kOffBias = kOffBuf + kGroups * kSzBuf;  // b1, b2 as FP16 pairs [64] each, b3[16] float
constexpr int kOffNorm = kOffBias + (128 + 128 + 16) * 4;  // step mode: mean [64], 1 / std [64]
constexpr int kOffBar = kOffNorm + 128 * 4;  // kGroups mbarriers (8 B), TMEM address
constexpr int kSmemBytes = kOffBar + 8 * kGroups + 16 + 1024;  // + slack for aligning the base

// byte offset of element (r, k) in an R-row K-major no-swizzle operand
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int R) {
    return static_cast<uint32_t>(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// matrix descriptor: start address, LBO, SBO (all >> 4), version 1 (bits 46-47), no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: A and B FP16 (type fields 0), both K-major, D FP32 (bit 4
// set) or FP16 (clear), N >> 3, M >> 4
__host__ __device__ constexpr uint32_t instr_desc(int M, int N, bool f32_acc) {
    return (f32_acc ? (1u << 4) : 0u) | (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
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

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// barrier of one group's 128 threads (named barrier 1 + group; 0 is the CTA-wide __syncthreads)
__device__ __forceinline__ void group_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// the group's threads agree: true only if `v` is true in all 128
__device__ __forceinline__ bool group_all(int id, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"(v ? 1u : 0u), "r"(id)
        : "memory");
    return r != 0;
}

// 64 consecutive FP32 columns of this thread's TMEM lane (one load, one wait)
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int j = 0; j < 64; ++j) v[j] = __uint_as_float(r[j]);
}

// two FP32 values rounded to nearest FP16, packed (lo in the low half)
__device__ __forceinline__ uint32_t pack_f16(float lo, float hi) {
    __half2 v = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// SiLU(z + b) of two FP32 accumulator columns: z rounded to FP16 once, then bias add, z / 2, tanh
// (hardware approximation), 1/2 + t / 2 and the product in f16x2 arithmetic, two lanes per
// instruction (each step rounds to FP16, relative 2^-11, the size of the rounding the activation
// gets anyway as the next layer's operand)
__device__ __forceinline__ uint32_t silu2_bias_f16(float z0, float z1, uint32_t bias2) {
    const __half2 half2 = __floats2half2_rn(0.5f, 0.5f);
    uint32_t z2 = pack_f16(z0, z1);
    const __half2 z = __hadd2(*reinterpret_cast<__half2*>(&z2), *reinterpret_cast<__half2*>(&bias2));
    __half2 h = __hmul2(z, half2);
    uint32_t hu = *reinterpret_cast<uint32_t*>(&h), tu;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(tu) : "r"(hu));
    const __half2 sg = __hfma2(*reinterpret_cast<__half2*>(&tu), half2, half2);
    __half2 out = __hmul2(z, sg);
    return *reinterpret_cast<uint32_t*>(&out);
}

// bias + SiLU of 64 accumulator columns [c0, c0 + 64) of row r, stored as FP16 into an R = 128 row
// K-major operand (8 stores of 16 bytes); the bias is read 8 values at a time (a broadcast: every
// thread of the warp reads the same address)
__device__ __forceinline__ void store_hidden64(unsigned char* A, int r, int c0, const float (&acc)[64],
                                               const uint32_t* bias2) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const uint4 b = *reinterpret_cast<const uint4*>(bias2 + (c0 + q * 8) / 2);  // 8 biases, FP16 pairs
        const float* x = acc + q * 8;
        uint4 w;
        w.x = silu2_bias_f16(x[0], x[1], b.x);
        w.y = silu2_bias_f16(x[2], x[3], b.y);
        w.z = silu2_bias_f16(x[4], x[5], b.z);
        w.w = silu2_bias_f16(x[6], x[7], b.w);
        *reinterpret_cast<uint4*>(A + kmajor_offset(r, c0 + q * 8, kRows)) = w;
    }
}

// 16 consecutive FP32 columns of this thread's TMEM lane (one load, one wait)
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

}  // namespace tc

// Largest warm-start move, in characteristic lengths.  Trained corrections are a few hundredths
// of L; a prediction beyond this bound (an input unlike the training data) is shortened to it, so
// that the start cannot fold an element over before the sweeps begin.
constexpr float kMaxPrediction = 0.25f;

// The warm start's move of one vertex: the prediction p (the step's correction x - y in units of
// the vertex's mean rest edge length L) times L, shortened to kMaxPrediction L; 0 for a non-finite
// prediction.  Explicitly rounded operations: every kernel that applies a start gets the same bits.
__device__ __forceinline__ float3 bounded_start(float p0, float p1, float p2, float L) {
    const float n2 = __fmaf_rn(p2, p2, __fmaf_rn(p1, p1, __fmul_rn(p0, p0)));
    if (!isfinite(n2)) return make_float3(0.f, 0.f, 0.f);
    float s = L;
    if (!(n2 <= kMaxPrediction * kMaxPrediction)) s = __fmul_rn(__fmul_rn(s, kMaxPrediction), rsqrtf(n2));
    return make_float3(__fmul_rn(p0, s), __fmul_rn(p1, s), __fmul_rn(p2, s));
}

// the start of solvable internal vertex i: displacement += the bounded move, iterate = x + displacement
__device__ __forceinline__ void apply_start(const float4* pinfo, const float4* vfeat, const float4* prev, float4* disp,
                                            float4* pos, int i, float p0, float p1, float p2) {
    const float4 pi = pinfo[i];
    if (!((__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f)) return;
    const float3 m = bounded_start(p0, p1, p2, vfeat[i].w);
    float4 d = disp[i];
    d = make_float4(__fadd_rn(d.x, m.x), __fadd_rn(d.y, m.y), __fadd_rn(d.z, m.z), 0.f);
    disp[i] = d;
    const float4 p = prev[i];
    pos[i] = make_float4(__fadd_rn(p.x, d.x), __fadd_rn(p.y, d.y), __fadd_rn(p.z, d.z), 0.f);
}

namespace tc {

// Inputs of the step mode (kInput == kInStep): the features of each row are computed from the
// solver's arrays in the kernel (no feature rows in HBM), and the last epilogue applies the bounded
// start to the row's vertex instead of storing the prediction.  Rows are internal vertex ids.
struct TcStep {
    const float4* pinfo;      // [V] mass, flags
    const float4* prev;       // [V] step-start positions x
    const float4* y;          // [V] inertia targets
    const int* nbr8;          // [V][8] one-ring neighbours (16-byte aligned rows)
    const float4* vfeat;      // [V] log-stiffnesses, mean rest edge length L (w)
    const int* ccount;        // [V] contact counts, or NULL
    const float* corr_prev;   // [V][3] previous step's correction (internal order), or NULL
    const float* mean;        // [64] standardization, or NULL
    const float* inv_std;     // [64]
    int mode;                 // VBD_FEATURES_CORRECTIONS or VBD_FEATURES_KINEMATIC
    float3 g_dt2;             // gravity * dt^2 (kinematic set)
    float inv_dt;             // 1 / dt (kinematic set)
    float4* disp;             // [V] displacement from x: += the start
    float4* pos;              // [V] iterate: x + displacement
};

struct TcArgs {
    int n;
    const float* params;  // FP32 blob: weights W1 [64][128], W2 [128][128], W3 [128][8] and biases
    const float* X;       // [n][64] FP32 (kInF32)
    float* Y;             // [n][3] (kInF32)
    TcStep step;          // (kInStep)
    unsigned* status;     // incremented on a wait that gave up (may be NULL)
    int off_w1, off_b1, off_w2, off_b2, off_w3, off_b3;
};

constexpr int kInF32 = 0;   // FP32 feature rows in HBM, prediction rows out
constexpr int kInStep = 1;  // features computed in the kernel, the start applied (TcStep)

// The 64 features of internal vertex i, as the features kernel of vbd_mlp.cu computes them (the
// same expressions in the same order, so the rows are bitwise equal); kKin selects the kinematic
// set.  All indices into f are compile-time constants (f stays in registers).
template <bool kKin>
__device__ __forceinline__ void step_features(const TcStep& s, int i, float (&f)[64]) {
#pragma unroll
    for (int k = 0; k < 64; ++k) f[k] = 0.f;
    const float4 pi = s.pinfo[i];
    const float4 vf = s.vfeat[i];
    const float invL = 1.0f / fmaxf(vf.w, 1e-9f);
    const float4 xp = s.prev[i];
    const float3 x = make_float3(xp.x, xp.y, xp.z);
    const int4 na = __ldg(reinterpret_cast<const int4*>(s.nbr8) + 2 * i);
    const int4 nb4 = __ldg(reinterpret_cast<const int4*>(s.nbr8) + 2 * i + 1);
    const int nb[8] = {na.x, na.y, na.z, na.w, nb4.x, nb4.y, nb4.z, nb4.w};
    int nn = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (nb[j] < 0) continue;
        ++nn;
        const float4 xn = s.prev[nb[j]];
        const int e = kKin ? 9 + 3 * j : 6 + 3 * j;
        f[e] = (xn.x - x.x) * invL;
        f[e + 1] = (xn.y - x.y) * invL;
        f[e + 2] = (xn.z - x.z) * invL;
        if (!kKin && s.corr_prev) {
            f[30 + 3 * j] = s.corr_prev[3 * nb[j]] * invL;
            f[31 + 3 * j] = s.corr_prev[3 * nb[j] + 1] * invL;
            f[32 + 3 * j] = s.corr_prev[3 * nb[j] + 2] * invL;
        }
    }
    const bool solvable = (__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f;
    const float4 yp = s.y[i];
    const float3 off = make_float3(yp.x - x.x, yp.y - x.y, yp.z - x.z);
    const float mass = pi.x > 0.f ? log10f(pi.x) : 0.f;
    const float contact = (s.ccount && s.ccount[i] > 0) ? 1.f : 0.f;
    if (kKin) {
        if (solvable) {
            const float3 vdt = make_float3(off.x - s.g_dt2.x, off.y - s.g_dt2.y, off.z - s.g_dt2.z);
            f[0] = vdt.x * invL;
            f[1] = vdt.y * invL;
            f[2] = vdt.z * invL;
            f[3] = vdt.x * s.inv_dt;
            f[4] = vdt.y * s.inv_dt;
            f[5] = vdt.z * s.inv_dt;
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
        if (s.corr_prev) {
            f[3] = s.corr_prev[3 * i] * invL;
            f[4] = s.corr_prev[3 * i + 1] * invL;
            f[5] = s.corr_prev[3 * i + 2] * invL;
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

// one row of step features, standardized, rounded to FP16 and stored as the row's 8 chunks of
// the K-major A operand (row i >= n: zeros)
template <bool kKin>
__device__ __forceinline__ void stage_step_row(const TcStep& s, int i, int n, const float* mean, const float* inv_std,
                                               unsigned char* A, int r) {
    if (i >= n) {
#pragma unroll
        for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(A + kmajor_offset(r, 8 * c, kRows)) = make_uint4(0u, 0u, 0u, 0u);
        return;
    }
    float f[64];
    step_features<kKin>(s, i, f);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = mean ? (f[8 * c + k] - mean[8 * c + k]) * inv_std[8 * c + k] : f[8 * c + k];
        *reinterpret_cast<uint4*>(A + kmajor_offset(r, 8 * c, kRows)) =
            make_uint4(pack_f16(v[0], v[1]), pack_f16(v[2], v[3]), pack_f16(v[4], v[5]), pack_f16(v[6], v[7]));
    }
}

template <int kInput>
__global__ void __launch_bounds__(kThreads, 1) mlp_infer_tc_kernel(TcArgs a) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sW1 = smem + kOffW1;
    unsigned char* sW2 = smem + kOffW2;
    unsigned char* sW3 = smem + kOffW3;
    uint32_t* sB1 = reinterpret_cast<uint32_t*>(smem + kOffBias);  // FP16 pairs
    uint32_t* sB2 = sB1 + 64;
    float* sB3 = reinterpret_cast<float*>(sB2 + 64);
    float* sMean = reinterpret_cast<float*>(smem + kOffNorm);  // step mode: standardization [64] + [64]
    float* sIstd = sMean + 64;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kOffBar + 8 * kGroups);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int group = warp >> 2, quarter = warp & 3, gtid = tid & (kGroupThreads - 1);
    const int bar_id = 1 + group;
    unsigned char* buf = smem + kOffBuf + group * kSzBuf;
    const uint32_t bar = smem_u32(bars + group);

    // ---- set-up: weights transposed into the B layouts, biases, mbarriers, TMEM ---------------
    // FP32 weights [K][N] -> FP16 B operands [N][K]: a thread gathers 8 consecutive k of one column
    // n (each load instruction reads 32 consecutive n of one row: coalesced) and stores them as one
    // 16-byte chunk of a core matrix (a warp fills 512 contiguous bytes)
    auto transpose_in = [&](unsigned char* dst, const float* src, int K, int N, int ld, int R) {
        for (int i = tid; i < (K / 8) * R; i += kThreads) {
            const int nn = i % R, kg = i / R;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = nn < N ? __ldg(src + (kg * 8 + j) * ld + nn) : 0.f;
            *reinterpret_cast<uint4*>(dst + kmajor_offset(nn, kg * 8, R)) =
                make_uint4(pack_f16(v[0], v[1]), pack_f16(v[2], v[3]), pack_f16(v[4], v[5]), pack_f16(v[6], v[7]));
        }
    };
    transpose_in(sW1, a.params + a.off_w1, 64, 128, 128, 128);
    transpose_in(sW2, a.params + a.off_w2, 128, 128, 128, 128);
    transpose_in(sW3, a.params + a.off_w3, 128, 8, 8, kN3);  // rows 8..15 zero
    for (int i = tid; i < 64; i += kThreads) {
        sB1[i] = pack_f16(a.params[a.off_b1 + 2 * i], a.params[a.off_b1 + 2 * i + 1]);
        sB2[i] = pack_f16(a.params[a.off_b2 + 2 * i], a.params[a.off_b2 + 2 * i + 1]);
    }
    if (tid < kN3) sB3[tid] = tid < 8 ? a.params[a.off_b3 + tid] : 0.f;
    const bool normalize = kInput == kInStep && a.step.mean != nullptr;
    if (normalize && tid < 64) {
        sMean[tid] = a.step.mean[tid];
        sIstd[tid] = a.step.inv_std[tid];
    }
    const bool kinematic = kInput == kInStep && a.step.mode == VBD_FEATURES_KINEMATIC;
    if (tid < kGroups) bar_init(smem_u32(bars + tid), 1);
    if (tid == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t d = *tmem_slot + static_cast<uint32_t>(group * 128);   // this group's columns
    const uint32_t lane_base = static_cast<uint32_t>(quarter * 32) << 16;  // this warp's TMEM lanes
    const uint32_t idesc128 = instr_desc(128, 128, true), idesc16 = instr_desc(128, kN3, true);
    const uint32_t ab = smem_u32(buf), w1 = smem_u32(sW1), w2 = smem_u32(sW2), w3 = smem_u32(sW3);
    const bool issuer = gtid == 0;
    const int r_own = quarter * 32 + lane;  // this thread's row of the tile
    uint32_t phase = 0;
    bool ok = true;
    const int ntiles = (a.n + kRows - 1) / kRows;

    for (int tile = blockIdx.x * kGroups + group; tile < ntiles; tile += gridDim.x * kGroups) {
        const int row0 = tile * kRows;
        // ---- 1. features -> the buffer as FP16.  Warp q stages rows [32 q, 32 q + 32): in pass j
        // a lane takes row 32 q + 8 (j / 4) + lane % 8 and float4 column 4 (j % 4) + lane / 8, so each
        // load reads 8 rows x 64 contiguous bytes and each store fills whole core-matrix rows; the
        // 16 loads are in flight together (the other groups' work covers their latency) ----
        if (kInput == kInStep) {
            // this thread's row: its features from the solver's arrays (one-ring gathers; the other
            // groups' MMAs and epilogues cover their latency)
            if (kinematic)
                stage_step_row<true>(a.step, row0 + r_own, a.n, normalize ? sMean : nullptr, sIstd, buf, r_own);
            else
                stage_step_row<false>(a.step, row0 + r_own, a.n, normalize ? sMean : nullptr, sIstd, buf, r_own);
        } else {
            float4 v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int r = quarter * 32 + 8 * (j >> 2) + (lane & 7);
                const int c4 = 4 * (j & 3) + (lane >> 3);
                v[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (row0 + r < a.n)
                    v[j] = __ldg(reinterpret_cast<const float4*>(a.X + static_cast<size_t>(row0 + r) * 64) + c4);
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int r = quarter * 32 + 8 * (j >> 2) + (lane & 7);
                const int c4 = 4 * (j & 3) + (lane >> 3);
                uint2 w;
                w.x = pack_f16(v[j].x, v[j].y);
                w.y = pack_f16(v[j].z, v[j].w);
                *reinterpret_cast<uint2*>(buf + kmajor_offset(r, 4 * c4, kRows)) = w;
            }
        }
        fence_proxy_async();
        fence_before();
        group_sync(bar_id);
        if (kInput == kInStep) {
            // the group's next tile: its rows' own data toward L2 while this tile runs (a prefetch
            // holds no register; measured 4-5% off the launch at 1.89 M rows)
            const int nxt = (tile + gridDim.x * kGroups) * kRows + r_own;
            if (nxt < a.n) {
                prefetch_l2(a.step.prev + nxt);
                prefetch_l2(a.step.y + nxt);
                prefetch_l2(a.step.pinfo + nxt);
                prefetch_l2(a.step.vfeat + nxt);
                prefetch_l2(a.step.nbr8 + 8 * nxt);
                prefetch_l2(a.step.disp + nxt);
                if (a.step.corr_prev) prefetch_l2(a.step.corr_prev + 3 * nxt);
            }
        }
        // ---- 2. layer 1 ----
        if (issuer) {
            fence_after();
#pragma unroll
            for (int s = 0; s < 4; ++s)
                mma_f16(d, smem_desc(ab + s * 2 * 2048, 2048, 128), smem_desc(w1 + s * 2 * 2048, 2048, 128), idesc128,
                         s > 0 ? 1u : 0u);
            mma_commit(bar);
        }
        ok = group_all(bar_id, bar_wait(bar, phase));  // one decision for the whole group
        if (!ok) break;
        phase ^= 1u;
        fence_after();
#pragma unroll 1
        for (int c0 = 0; c0 < 128; c0 += 64) {
            float acc[64];
            tmem_ld64(d + lane_base + c0, acc);
            store_hidden64(buf, r_own, c0, acc, sB1);  // layer 1's MMAs have completed: X is free
        }
        fence_proxy_async();
        fence_before();
        group_sync(bar_id);
        // ---- 3. layer 2 (D's columns reused: layer 1's epilogue has read them) ----
        if (issuer) {
            fence_after();
#pragma unroll
            for (int s = 0; s < 8; ++s)
                mma_f16(d, smem_desc(ab + s * 2 * 2048, 2048, 128), smem_desc(w2 + s * 2 * 2048, 2048, 128), idesc128,
                         s > 0 ? 1u : 0u);
            mma_commit(bar);
        }
        ok = group_all(bar_id, bar_wait(bar, phase));
        if (!ok) break;
        phase ^= 1u;
        fence_after();
#pragma unroll 1
        for (int c0 = 0; c0 < 128; c0 += 64) {
            float acc[64];
            tmem_ld64(d + lane_base + c0, acc);
            store_hidden64(buf, r_own, c0, acc, sB2);  // layer 2's MMAs have completed: H1 is free
        }
        fence_proxy_async();
        fence_before();
        group_sync(bar_id);
        // ---- 4. layer 3 ----
        if (issuer) {
            fence_after();
#pragma unroll
            for (int s = 0; s < 8; ++s)
                mma_f16(d, smem_desc(ab + s * 2 * 2048, 2048, 128), smem_desc(w3 + s * 2 * 256, 256, 128), idesc16,
                         s > 0 ? 1u : 0u);
            mma_commit(bar);
        }
        ok = group_all(bar_id, bar_wait(bar, phase));
        if (!ok) break;
        phase ^= 1u;
        fence_after();
        {
            float y[16];
            tmem_ld16(d + lane_base, y);
            const int r = row0 + r_own;
            if (r < a.n) {
                const float p0 = y[0] + sB3[0], p1 = y[1] + sB3[1], p2 = y[2] + sB3[2];
                if (kInput == kInStep) {
                    apply_start(a.step.pinfo, a.step.vfeat, a.step.prev, a.step.disp, a.step.pos, r, p0, p1, p2);
                } else {
                    float* out = a.Y + static_cast<size_t>(r) * 3;
                    out[0] = p0;
                    out[1] = p1;
                    out[2] = p2;
                }
            }
        }
        fence_before();
        group_sync(bar_id);  // the buffer and D are free for the group's next tile
    }
    if (!ok) {
        // a wait gave up: record it, then wait (bounded) for the MMAs the group issued before the
        // CTA frees the TMEM (the last commit tracks all of them)
        if (issuer && a.status) atomicAdd(a.status, 1u);
        bar_wait(bar, phase);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(kTmemCols));
    }
}

}  // namespace tc
}  // namespace vbd
