// vbd_solver.cu -- the VBD particle step on B200: forward (inertia) kernel, per-color
// Gauss-Seidel sweep, finalize (velocity) kernel, residual kernel, CUDA-graph replay of a step.
//
// Step structure (SolverVBD.step, solver_vbd.py:1774-1825, particle part only):
//   forward   : _initialize_particles (solver_vbd.py:2065-2100) = forward_step
//               (particle_vbd_kernels.py:1350-1375) + apply_truncation_ts (:2266-2286) with t = 1,
//               max_displacement = inf; also scatters this step's soft-contact records into a
//               per-vertex table (replaces accumulate_particle_body_contact_force_and_hessian's
//               per-color scan over all records, :2289-2401).
//   sweep(c)  : one color of _solve_particle_iteration (solver_vbd.py:2552-2702): contact
//               accumulation, solve_elasticity_tile (:2404-2565) and apply_truncation_ts,
//               fused into one launch over the color's vertices only.
//   finalize  : wp.copy(state_out.q, state_in.q) (solver_vbd.py:2704) + update_velocity
//               (particle_vbd_kernels.py:1468-1471).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "vbd_internal.h"
#include "vbd_math.cuh"
#include "vbd_resident.h"
#include "vbd_self_contact.h"

namespace vbd {

enum StatusSlot { kNonfinite = 0, kSingular = 1, kOverflow = 2, kTimeout = 3, kStatusSlots = 4 };

constexpr int kGateMaxIterations = 100000;  // upper bound of a gated step's iteration cap
constexpr int kGateDefaultRounds = 4;        // sweep mode: check rounds per loop body by default

// Device-side state of the residual gate (vbd_set_residual_gate), one per solver.  The head, up
// to `ref`, is zeroed at the start of every gated step.
// The accumulators of one evaluation are spread over kGateSlots slots, each on its own 128-byte
// line (a sweep's block b adds its block total into slot b mod kGateSlots; the Jacobi evaluation's
// warp w into slot w mod kGateSlots), so that the atomics of a large sweep do not queue on a few
// lines: atomics on one address serialize at the L2.
constexpr int kGateSlots = 256;
constexpr int kSumStride = 16;  // unsigned long long per 128-byte line
constexpr int kMaxStride = 32;  // unsigned per 128-byte line

struct GateState {
    unsigned long long sum[kGateSlots * kSumStride];  // fixed-point sums of the residuals (resid_fixed)
    unsigned maxv[kGateSlots * kMaxStride];  // max residual (float bits; atomicMax target)
    int iters;               // iterations run so far in this step
    unsigned stop;           // 1 once this step's gate has decided: later sweeps of the loop body return
    int pad;
    float ref;               // relative mode: the step's reference residual
    int last_iters;          // iterations of the last finished step
    float last_resid;        // final residual of the last finished step
    float start_resid;       // residual where the last step's iterations started
    unsigned long long steps;     // gated steps finished (since creation or the last reset)
    unsigned long long iter_sum;  // iterations summed over those steps
    unsigned long long capped;    // steps that stopped at the iteration cap above the tolerance
    unsigned long long passes;    // passes of the loop body summed over those steps
};

struct GraphEntry {
    float* q_in;
    const float* qd_in;
    const float* f_ext;
    float* q_out;
    float* qd_out;
    VbdContacts contacts;
    bool has_contacts;
    float dt;
    int iterations;
    int lanes, block;
    int kernels;  // kernel nodes of the captured step
    cudaGraphExec_t exec;
};

struct SolverImpl {
    const VbdModelImpl* m = nullptr;
    int iterations = 10;
    float friction_epsilon = 1e-2f;
    int lanes = 4;  // 0: record-parallel tiles; 1..16: lanes cooperating on one vertex
    int block = 128;
    int K = 4;
    bool use_graph = true;
    long long steps = 0;
    int last_step_kernels = -1;  // kernel launches of the last vbd_step (graph kernel nodes; -1: not a graph)
    int staged_iteration = 0;    // iteration of the staged API (vbd_forward resets, vbd_begin_iteration sets)
    // scratch (allocated once at create)
    float4* pos = nullptr;    // Gauss-Seidel iterate (state_in.particle_q in the reference)
    float4* prev = nullptr;   // particle_q_prev == pos_prev_collision_detection (step start)
    float4* y = nullptr;      // inertia target, .w = mass
    float4* disp = nullptr;   // particle_displacements
    int* ccount = nullptr;    // [V] contacts per vertex (internal order)
    int* cslot = nullptr;     // [V*K] record ids
    float4* ctab = nullptr;   // [V*K][4] the step's contacts per vertex, packed and in record order
    unsigned* status = nullptr;  // [kStatusSlots]
    float* resid_max = nullptr;  // [1] scratch for vbd_residual
    cudaStream_t capture_stream = nullptr;
    std::vector<GraphEntry> graphs;
    // persistent shared-memory-resident step (used by vbd_step when the model fits)
    bool resident_on = false;        // run steps with the resident kernel (when the plan is ready)
    ResidentPlan resident;
    unsigned spin_limit = 1u << 22;  // bound of every wait in the resident kernel
    // learned warm start (vbd_set_warm_start): caller-owned network, solver-owned buffers
    const float* ws_params = nullptr;
    const uint16_t* ws_w16 = nullptr;
    const float* ws_mean = nullptr;
    const float* ws_inv_std = nullptr;
    int ws_iterations = 0;
    float* ws_corr = nullptr;        // [V][3] previous step's correction x_solved - y (internal order)
    int feature_set = VBD_FEATURES_CORRECTIONS;  // vbd_set_feature_set
    float last_dt = 0.f;             // dt of the last vbd_forward (the kinematic features need it)
    // particle self-contact (particle_enable_self_contact)
    SelfContact sc;
    // residual gate (vbd_set_residual_gate): iterate until max_i |f_i| / (m_i |g|) <= tolerance
    float gate_tol = 0.f;            // <= 0: off (fixed iteration count)
    int gate_max = 0;                // iteration cap
    int gate_every = 1;              // iterations between residual checks
    int gate_relative = 0;           // 1: tolerance relative to the residual at the inertia target y
    int gate_mean = 0;               // 1: mean residual over the solved vertices instead of the max
    int gate_sweep = 0;              // 1: the Gauss-Seidel residual the sweeps accumulate (no Jacobi launch)
    int gate_count = 0;              // solved vertices (the mean's divisor)
    int gate_rounds = 4;             // sweep mode: check rounds per body of the device-side loop
    GateState* gate = nullptr;       // device
    cudaStream_t body_stream = nullptr;  // capture stream of the gate's loop body
    // staged sweep (vbd_set_staged_sweep): per color block, the ids of the positions its records
    // read (its patch), and each record's indices into the patch, for one launch shape
    bool stage_on = false;
    bool stage_ready = false;        // built for (stage_lanes, stage_block)
    int stage_lanes = 0, stage_block = 0, stage_max_patch = 0;
    std::vector<int> stage_color_base;  // first patch of each color
    int* patch_off = nullptr;
    int* patch_ids = nullptr;
    uint2* tri_loc = nullptr;
    uint2* edge_loc = nullptr;
    int gate_body_kernels = -1;      // kernel nodes of one loop body (last capture)
    int gate_body_pdl_edges = -1;    // programmatic edges of that body
    bool pdl = true;                 // programmatic dependent launch of the sweeps
};

}  // namespace vbd

struct VbdSolver {
    vbd::SolverImpl s;
};

namespace vbd {

// ---------------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------------
struct ForwardArgs {
    const int* perm;
    const int* inv_perm;
    const float4* pinfo;
    const float* q_in;
    const float* qd_in;
    const float* f_ext;
    float4* pos;
    float4* prev;
    float4* y;
    float4* disp;
    int V;
    float3 g;
    float dt;
    // contact scatter
    const int* c_count;
    const int* c_particle;
    int c_max;
    int* ccount;
    int* cslot;
    int K;
    unsigned* status;
};

__global__ void forward_kernel(ForwardArgs a) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid < a.V) {
        const int i = tid;
        const int o = a.perm[i];
        const float4 pi = a.pinfo[i];
        const int flags = __float_as_int(pi.w);
        const float3 q = f3(a.q_in[3 * o], a.q_in[3 * o + 1], a.q_in[3 * o + 2]);
        float3 yv = q, dv = f3(0.f, 0.f, 0.f);
        if ((flags & VBD_PARTICLE_ACTIVE) && pi.y != 0.0f) {
            const float3 v = f3(a.qd_in[3 * o], a.qd_in[3 * o + 1], a.qd_in[3 * o + 2]);
            float3 fe = f3(0.f, 0.f, 0.f);
            if (a.f_ext) fe = f3(a.f_ext[3 * o], a.f_ext[3 * o + 1], a.f_ext[3 * o + 2]);
            const float3 vn = v + (a.g + fe * pi.y) * a.dt;
            yv = q + vn * a.dt;
            dv = f3(__fmul_rn(vn.x, a.dt), __fmul_rn(vn.y, a.dt), __fmul_rn(vn.z, a.dt));
        }
        a.prev[i] = make_float4(q.x, q.y, q.z, 0.f);
        a.y[i] = make_float4(yv.x, yv.y, yv.z, pi.x);
        a.disp[i] = make_float4(dv.x, dv.y, dv.z, 0.f);
        // the first iterate is x_prev + disp, rounded as two separate operations (no FMA), so that
        // a warm start with a zero offset reproduces it bit for bit
        const float3 p = f3(__fadd_rn(q.x, dv.x), __fadd_rn(q.y, dv.y), __fadd_rn(q.z, dv.z));
        a.pos[i] = make_float4(p.x, p.y, p.z, 0.f);
    }
    if (a.c_count) {
        // the record count lives on the device: grid-stride over it (the grid is sized for the
        // vertices, not for the record capacity V x shapes)
        const int n = min(*a.c_count, a.c_max);
        for (int r = tid; r < n; r += gridDim.x * blockDim.x) {
            const int ip = a.inv_perm[a.c_particle[r]];
            const int k = atomicAdd(&a.ccount[ip], 1);
            if (k < a.K) {
                a.cslot[ip * a.K + k] = r;
            } else {
                atomicAdd(&a.status[kOverflow], 1u);
            }
        }
    }
}

// Per-step packing of the contact table: the scatter above leaves each vertex's record ids in
// arbitrary (atomic) order; this pass sorts them (the reference adds a particle's contacts in
// record order) and gathers what the contact law reads into 4 float4 per contact:
//   (body_pos, ke) (body_vel, kd) (normal, mu) (margin, 0, 0, 0)
// so that every color sweep of the step reads one contiguous entry per contact instead of the
// id -> record -> shape chain.
struct PackArgs {
    const int* ccount;
    const int* cslot;
    int K;
    const int* c_shape;
    const float* c_body_pos;
    const float* c_body_vel;
    const float* c_normal;
    const DevShape* shapes;
    float4* ctab;
    int V;
};

__global__ void pack_contacts_kernel(PackArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.V) return;
    const int n = min(a.ccount[i], a.K);
    if (n <= 0) return;
    // K <= 8: odd-even transposition sort of 8 slots (unused slots hold INT_MAX and sort last);
    // the fixed indices keep the ids in registers
    int ids[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) ids[k] = k < n ? a.cslot[i * a.K + k] : 0x7fffffff;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
#pragma unroll
        for (int k = p & 1; k + 1 < 8; k += 2) {
            const int lo = min(ids[k], ids[k + 1]), hi = max(ids[k], ids[k + 1]);
            ids[k] = lo;
            ids[k + 1] = hi;
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (k < n) {
            const int r = ids[k];
            const float4 sm = a.shapes[a.c_shape[r]].mat;
            float4* e = a.ctab + (static_cast<size_t>(i) * a.K + k) * 4;
            e[0] = make_float4(a.c_body_pos[3 * r], a.c_body_pos[3 * r + 1], a.c_body_pos[3 * r + 2], sm.x);
            e[1] = make_float4(a.c_body_vel[3 * r], a.c_body_vel[3 * r + 1], a.c_body_vel[3 * r + 2], sm.y);
            e[2] = make_float4(a.c_normal[3 * r], a.c_normal[3 * r + 1], a.c_normal[3 * r + 2], sm.z);
            e[3] = make_float4(sm.w, 0.f, 0.f, 0.f);
        }
    }
}

// What a residual check needs besides the state (baked into the step graph).
struct GateParams {
    float tol;
    int max_iters;
    int relative;
    int mean;
    int count;    // solved vertices (the mean's divisor)
    int first;    // 1: the start evaluation; 0: a later one; -1: sweep residuals (first iff iters == 0)
    int set_ref;  // the first evaluation is also the relative mode's reference
    int add;      // iterations since the last check
    int rounds;   // check rounds per pass of the loop body (sweep mode), else 1
};

struct SweepArgs {
    float4* pos;
    const float4* prev;
    const float4* y;
    float4* disp;
    const int4* vadj;
    const float4* pinfo;
    const int4* tri_idx;
    const float4* tri_D;
    const float4* tri_mat;
    const int4* edge_idx;
    const float4* edge_mat;
    // contacts
    const int* ccount;
    const int* cslot;
    int K;
    const int* c_shape;
    const float* c_body_pos;
    const float* c_body_vel;
    const float* c_normal;
    const DevShape* shapes;
    // packed contact table (pack_contacts_kernel); NULL: read the records through cslot instead
    const float4* ctab;
    // self-contact force / Hessian of the vertex (NULL without self-contact)
    const float4* sc_f;
    const float4* sc_h0;
    const float4* sc_h1;
    // constants
    float dt, inv_dt, dt_sqr_recip, eps_u;
    unsigned* status;
    int v_begin, v_end;
    int write_pos;           // 1: commit q = prev + disp in place (conflict-free coloring)
    int prefetch_records;    // 1: prefetch the vertices' element records into L2 (first iteration of a step)
    float* resid_out;        // residual mode: per-vertex residual (original order) or NULL
    float* resid_max;        // residual mode: max residual (float bits, atomicMax)
    unsigned long long* gate_sum;   // residual gate: slotted fixed-point sums (GateState::sum) or NULL
    unsigned* gate_max;      // residual gate: slotted max (GateState::maxv) or NULL
    const int* perm;
    float inv_g;             // 1/|g| (0 when g = 0)
    int no_pdl;              // host side: launch without the programmatic-dependent-launch attribute
    // residual gate, later rounds of an unrolled loop body: return at once when the step's gate
    // has already decided (GateState::stop); NULL otherwise
    const unsigned* gate_stop;
    // staged sweep (vbd_set_staged_sweep): block b of this color reads the positions it needs from
    // shared memory, loaded from patch patch_base + b (its vertices' one-ring, ascending internal
    // ids); the records carry 14/16-bit indices into the patch.  NULL: unstaged.
    const int* patch_off;
    const int* patch_ids;
    const uint2* tri_loc;    // per triangle record: (l0 | l1 << 16, l2 | slot << 16)
    const uint2* edge_loc;   // per hinge record: (o0 | slot << 14 | o1 << 16, v0 | v1 << 16)
    int patch_base;
};

// The staged positions of a block: [patch size] iterate positions, then (damping) [patch size]
// step-start positions.
extern __shared__ float4 s_stage[];

template <bool kDamp>
__device__ __forceinline__ void accumulate_elements(const SweepArgs& a, int i, int lane, int L, int4 adj, float3& f,
                                                    Sym3& h) {
    // the vertex's records are dealt round-robin over one merged list (triangles, then hinges),
    // so every lane gets the same number of records to within one
    const int nt = adj.y - adj.x;
    const int lane_e = (lane - nt % L + L) % L;  // first hinge slot of this lane
    for (int r = adj.x + lane; r < adj.y; r += L) {
        const int4 ti = __ldg(&a.tri_idx[r]);
        const float4 D = __ldg(&a.tri_D[r]);
        const float4 mt = __ldg(&a.tri_mat[r]);
        const float3 x0 = xyz(a.pos[ti.x]), x1 = xyz(a.pos[ti.y]), x2 = xyz(a.pos[ti.z]);
        float3 p0 = x0, p1 = x1, p2 = x2;
        if (kDamp && mt.w > 0.0f) {
            p0 = xyz(__ldg(&a.prev[ti.x]));
            p1 = xyz(__ldg(&a.prev[ti.y]));
            p2 = xyz(__ldg(&a.prev[ti.z]));
        }
        membrane_eval<kDamp>(ti.w, x0, x1, x2, p0, p1, p2, D, mt, a.inv_dt, f, h);
    }
    for (int r = adj.z + lane_e; r < adj.w; r += L) {
        const int4 ei = __ldg(&a.edge_idx[r]);
        const float4 em = __ldg(&a.edge_mat[r]);
        const int order = static_cast<int>(static_cast<unsigned>(ei.x) >> 30);
        const int o0 = ei.x & 0x3fffffff;
        const float3 x0 = xyz(a.pos[o0]), x1 = xyz(a.pos[ei.y]), x2 = xyz(a.pos[ei.z]), x3 = xyz(a.pos[ei.w]);
        float3 p0 = x0, p1 = x1, p2 = x2, p3 = x3;
        if (kDamp && em.w > 0.0f) {
            p0 = xyz(__ldg(&a.prev[o0]));
            p1 = xyz(__ldg(&a.prev[ei.y]));
            p2 = xyz(__ldg(&a.prev[ei.z]));
            p3 = xyz(__ldg(&a.prev[ei.w]));
        }
        bending_eval<kDamp>(order, x0, x1, x2, x3, p0, p1, p2, p3, em, a.inv_dt, f, h);
    }
}

// The staged walk: the same records and the same math, with every position read from the block's
// shared-memory patch (s_pos, and s_prev for damping) through the record's local indices.
template <bool kDamp>
__device__ __forceinline__ void accumulate_elements_staged(const SweepArgs& a, int lane, int L, int4 adj,
                                                           const float4* s_pos, const float4* s_prev, float3& f,
                                                           Sym3& h) {
    const int nt = adj.y - adj.x;
    const int lane_e = (lane - nt % L + L) % L;
    for (int r = adj.x + lane; r < adj.y; r += L) {
        const uint2 tl = __ldg(&a.tri_loc[r]);
        const float4 D = __ldg(&a.tri_D[r]);
        const float4 mt = __ldg(&a.tri_mat[r]);
        const int l0 = tl.x & 0xffff, l1 = tl.x >> 16, l2 = tl.y & 0xffff, slot = tl.y >> 16;
        const float3 x0 = xyz(s_pos[l0]), x1 = xyz(s_pos[l1]), x2 = xyz(s_pos[l2]);
        float3 p0 = x0, p1 = x1, p2 = x2;
        if (kDamp && mt.w > 0.0f) {
            p0 = xyz(s_prev[l0]);
            p1 = xyz(s_prev[l1]);
            p2 = xyz(s_prev[l2]);
        }
        membrane_eval<kDamp>(slot, x0, x1, x2, p0, p1, p2, D, mt, a.inv_dt, f, h);
    }
    for (int r = adj.z + lane_e; r < adj.w; r += L) {
        const uint2 el = __ldg(&a.edge_loc[r]);
        const float4 em = __ldg(&a.edge_mat[r]);
        const int o0 = el.x & 0x3fff, order = (el.x >> 14) & 3, o1 = el.x >> 16, v0 = el.y & 0xffff, v1 = el.y >> 16;
        const float3 x0 = xyz(s_pos[o0]), x1 = xyz(s_pos[o1]), x2 = xyz(s_pos[v0]), x3 = xyz(s_pos[v1]);
        float3 p0 = x0, p1 = x1, p2 = x2, p3 = x3;
        if (kDamp && em.w > 0.0f) {
            p0 = xyz(s_prev[o0]);
            p1 = xyz(s_prev[o1]);
            p2 = xyz(s_prev[v0]);
            p3 = xyz(s_prev[v1]);
        }
        bending_eval<kDamp>(order, x0, x1, x2, x3, p0, p1, p2, p3, em, a.inv_dt, f, h);
    }
}

// The staged walk with two records in flight per lane: accumulate_elements_x2's order and math,
// positions from the patch (used where the unstaged sweep uses the two-record walk, so that both
// give the same bits).
template <bool kDamp>
__device__ __forceinline__ void accumulate_elements_staged_x2(const SweepArgs& a, int lane, int L, int4 adj,
                                                              const float4* s_pos, const float4* s_prev, float3& f,
                                                              Sym3& h) {
    const int nt = adj.y - adj.x;
    const int lane_e = (lane - nt % L + L) % L;
    for (int r = adj.x + lane; r < adj.y; r += 2 * L) {
        const bool two = r + L < adj.y;
        const int rb = two ? r + L : r;
        const uint2 ta = __ldg(&a.tri_loc[r]), tb = __ldg(&a.tri_loc[rb]);
        const float4 Da = __ldg(&a.tri_D[r]), Db = __ldg(&a.tri_D[rb]);
        const float4 ma = __ldg(&a.tri_mat[r]), mb = __ldg(&a.tri_mat[rb]);
        const int a0 = ta.x & 0xffff, a1 = ta.x >> 16, a2 = ta.y & 0xffff, sa = ta.y >> 16;
        const int b0 = tb.x & 0xffff, b1 = tb.x >> 16, b2 = tb.y & 0xffff, sb = tb.y >> 16;
        const float3 xa0 = xyz(s_pos[a0]), xa1 = xyz(s_pos[a1]), xa2 = xyz(s_pos[a2]);
        const float3 xb0 = xyz(s_pos[b0]), xb1 = xyz(s_pos[b1]), xb2 = xyz(s_pos[b2]);
        float3 pa0 = xa0, pa1 = xa1, pa2 = xa2, pb0 = xb0, pb1 = xb1, pb2 = xb2;
        if (kDamp && (ma.w > 0.0f || mb.w > 0.0f)) {
            pa0 = xyz(s_prev[a0]);
            pa1 = xyz(s_prev[a1]);
            pa2 = xyz(s_prev[a2]);
            pb0 = xyz(s_prev[b0]);
            pb1 = xyz(s_prev[b1]);
            pb2 = xyz(s_prev[b2]);
        }
        float3 fa = f3(0.f, 0.f, 0.f), fb = fa;
        Sym3 ha = zero_sym(), hb = zero_sym();
        membrane_eval<kDamp>(sa, xa0, xa1, xa2, pa0, pa1, pa2, Da, ma, a.inv_dt, fa, ha);
        membrane_eval<kDamp>(sb, xb0, xb1, xb2, pb0, pb1, pb2, Db, mb, a.inv_dt, fb, hb);
        f = f + fa;
        add(h, ha);
        if (two) {
            f = f + fb;
            add(h, hb);
        }
    }
    for (int r = adj.z + lane_e; r < adj.w; r += 2 * L) {
        const bool two = r + L < adj.w;
        const int rb = two ? r + L : r;
        const uint2 ea = __ldg(&a.edge_loc[r]), eb = __ldg(&a.edge_loc[rb]);
        const float4 ma = __ldg(&a.edge_mat[r]), mb = __ldg(&a.edge_mat[rb]);
        const int oa = (ea.x >> 14) & 3, ob = (eb.x >> 14) & 3;
        const int a0 = ea.x & 0x3fff, a1 = ea.x >> 16, a2 = ea.y & 0xffff, a3 = ea.y >> 16;
        const int b0 = eb.x & 0x3fff, b1 = eb.x >> 16, b2 = eb.y & 0xffff, b3 = eb.y >> 16;
        const float3 xa0 = xyz(s_pos[a0]), xa1 = xyz(s_pos[a1]), xa2 = xyz(s_pos[a2]), xa3 = xyz(s_pos[a3]);
        const float3 xb0 = xyz(s_pos[b0]), xb1 = xyz(s_pos[b1]), xb2 = xyz(s_pos[b2]), xb3 = xyz(s_pos[b3]);
        float3 pa0 = xa0, pa1 = xa1, pa2 = xa2, pa3 = xa3, pb0 = xb0, pb1 = xb1, pb2 = xb2, pb3 = xb3;
        if (kDamp && (ma.w > 0.0f || mb.w > 0.0f)) {
            pa0 = xyz(s_prev[a0]);
            pa1 = xyz(s_prev[a1]);
            pa2 = xyz(s_prev[a2]);
            pa3 = xyz(s_prev[a3]);
            pb0 = xyz(s_prev[b0]);
            pb1 = xyz(s_prev[b1]);
            pb2 = xyz(s_prev[b2]);
            pb3 = xyz(s_prev[b3]);
        }
        float3 fa = f3(0.f, 0.f, 0.f), fb = fa;
        Sym3 ha = zero_sym(), hb = zero_sym();
        bending_eval<kDamp, true>(oa, xa0, xa1, xa2, xa3, pa0, pa1, pa2, pa3, ma, a.inv_dt, fa, ha);
        bending_eval<kDamp, true>(ob, xb0, xb1, xb2, xb3, pb0, pb1, pb2, pb3, mb, a.inv_dt, fb, hb);
        f = f + fa;
        add(h, ha);
        if (two) {
            f = f + fb;
            add(h, hb);
        }
    }
}

// The same walk with two records in flight per lane: records r and r + L are loaded and evaluated
// as two independent chains (zero-started partial sums, added in record order), so the latency of
// one record's loads and math overlaps the other's.  Used where the launch leaves registers for
// it (few lanes per vertex, uncapped build).  A lane with an odd count evaluates its last record
// twice and keeps one result.
template <bool kDamp>
__device__ __forceinline__ void accumulate_elements_x2(const SweepArgs& a, int lane, int L, int4 adj, float3& f,
                                                       Sym3& h) {
    const int nt = adj.y - adj.x;
    const int lane_e = (lane - nt % L + L) % L;
    for (int r = adj.x + lane; r < adj.y; r += 2 * L) {
        const bool two = r + L < adj.y;
        const int rb = two ? r + L : r;
        const int4 ta = __ldg(&a.tri_idx[r]), tb = __ldg(&a.tri_idx[rb]);
        const float4 Da = __ldg(&a.tri_D[r]), Db = __ldg(&a.tri_D[rb]);
        const float4 ma = __ldg(&a.tri_mat[r]), mb = __ldg(&a.tri_mat[rb]);
        const float3 xa0 = xyz(a.pos[ta.x]), xa1 = xyz(a.pos[ta.y]), xa2 = xyz(a.pos[ta.z]);
        const float3 xb0 = xyz(a.pos[tb.x]), xb1 = xyz(a.pos[tb.y]), xb2 = xyz(a.pos[tb.z]);
        float3 pa0 = xa0, pa1 = xa1, pa2 = xa2, pb0 = xb0, pb1 = xb1, pb2 = xb2;
        if (kDamp && (ma.w > 0.0f || mb.w > 0.0f)) {
            pa0 = xyz(__ldg(&a.prev[ta.x]));
            pa1 = xyz(__ldg(&a.prev[ta.y]));
            pa2 = xyz(__ldg(&a.prev[ta.z]));
            pb0 = xyz(__ldg(&a.prev[tb.x]));
            pb1 = xyz(__ldg(&a.prev[tb.y]));
            pb2 = xyz(__ldg(&a.prev[tb.z]));
        }
        float3 fa = f3(0.f, 0.f, 0.f), fb = fa;
        Sym3 ha = zero_sym(), hb = zero_sym();
        membrane_eval<kDamp>(ta.w, xa0, xa1, xa2, pa0, pa1, pa2, Da, ma, a.inv_dt, fa, ha);
        membrane_eval<kDamp>(tb.w, xb0, xb1, xb2, pb0, pb1, pb2, Db, mb, a.inv_dt, fb, hb);
        f = f + fa;
        add(h, ha);
        if (two) {
            f = f + fb;
            add(h, hb);
        }
    }
    for (int r = adj.z + lane_e; r < adj.w; r += 2 * L) {
        const bool two = r + L < adj.w;
        const int rb = two ? r + L : r;
        const int4 ea = __ldg(&a.edge_idx[r]), eb = __ldg(&a.edge_idx[rb]);
        const float4 ma = __ldg(&a.edge_mat[r]), mb = __ldg(&a.edge_mat[rb]);
        const int oa = static_cast<int>(static_cast<unsigned>(ea.x) >> 30), ob = static_cast<int>(static_cast<unsigned>(eb.x) >> 30);
        const int a0 = ea.x & 0x3fffffff, b0 = eb.x & 0x3fffffff;
        const float3 xa0 = xyz(a.pos[a0]), xa1 = xyz(a.pos[ea.y]), xa2 = xyz(a.pos[ea.z]), xa3 = xyz(a.pos[ea.w]);
        const float3 xb0 = xyz(a.pos[b0]), xb1 = xyz(a.pos[eb.y]), xb2 = xyz(a.pos[eb.z]), xb3 = xyz(a.pos[eb.w]);
        float3 pa0 = xa0, pa1 = xa1, pa2 = xa2, pa3 = xa3, pb0 = xb0, pb1 = xb1, pb2 = xb2, pb3 = xb3;
        if (kDamp && (ma.w > 0.0f || mb.w > 0.0f)) {
            pa0 = xyz(__ldg(&a.prev[a0]));
            pa1 = xyz(__ldg(&a.prev[ea.y]));
            pa2 = xyz(__ldg(&a.prev[ea.z]));
            pa3 = xyz(__ldg(&a.prev[ea.w]));
            pb0 = xyz(__ldg(&a.prev[b0]));
            pb1 = xyz(__ldg(&a.prev[eb.y]));
            pb2 = xyz(__ldg(&a.prev[eb.z]));
            pb3 = xyz(__ldg(&a.prev[eb.w]));
        }
        float3 fa = f3(0.f, 0.f, 0.f), fb = fa;
        Sym3 ha = zero_sym(), hb = zero_sym();
        bending_eval<kDamp, true>(oa, xa0, xa1, xa2, xa3, pa0, pa1, pa2, pa3, ma, a.inv_dt, fa, ha);
        bending_eval<kDamp, true>(ob, xb0, xb1, xb2, xb3, pb0, pb1, pb2, pb3, mb, a.inv_dt, fb, hb);
        f = f + fa;
        add(h, ha);
        if (two) {
            f = f + fb;
            add(h, hb);
        }
    }
}

__device__ __forceinline__ void accumulate_contacts(const SweepArgs& a, int i, float3 x, float3 xp, float radius,
                                                    float3& f, Sym3& h) {
    const DevShape* shapes = a.shapes;
    vertex_contacts(a.ccount, a.cslot, a.K, i, a.c_shape, a.c_body_pos, a.c_body_vel, a.c_normal,
                    [shapes](int s) { return shapes[s].mat; }, x, xp, radius, a.dt, a.eps_u, f, h);
}

__device__ __forceinline__ void add_self_contact(const SweepArgs& a, int i, float3& f, Sym3& h) {
    const float4 sf = a.sc_f[i], h0 = a.sc_h0[i], h1 = a.sc_h1[i];
    f = f + xyz(sf);
    h.xx += h0.x;
    h.xy += h0.y;
    h.xz += h0.z;
    h.yy += h0.w;
    h.yz += h1.x;
    h.zz += h1.y;
}

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// L2 prefetch of the 128-byte lines holding records [b, e) of a 16-byte-per-record array, the
// lines dealt round-robin over the vertex's L lanes
__device__ __forceinline__ void prefetch_rows_l2(const void* base, int b, int e, int lane, int L) {
    if (e <= b) return;
    const char* p = static_cast<const char*>(base);
    const uintptr_t first = reinterpret_cast<uintptr_t>(p + 16 * static_cast<size_t>(b)) & ~uintptr_t(127);
    const uintptr_t last = reinterpret_cast<uintptr_t>(p + 16 * static_cast<size_t>(e) - 1) & ~uintptr_t(127);
    for (uintptr_t line = first + 128 * static_cast<uintptr_t>(lane); line <= last; line += 128 * static_cast<uintptr_t>(L))
        prefetch_l2(reinterpret_cast<const void*>(line));
}

__device__ __forceinline__ float warp_sum(float v, int L) {
    for (int off = L >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// Contacts (packed table or records), self-contact, and inertia added to a vertex's summed
// elastic force / Hessian, in the reference's order: elastic + inertia + contact
// (solve_elasticity_tile, particle_vbd_kernels.py:2546-2565).
__device__ __forceinline__ void add_vertex_terms(const SweepArgs& a, int i, float4 pi, float4 pv, float3 x, float4 yv,
                                                 float3& f, Sym3& h) {
    const float mass = yv.w;
    float3 fc = f3(0.f, 0.f, 0.f);
    Sym3 hc = zero_sym();
    if (a.ctab) {
        // the step's packed contacts, already in record order
        const int nc = min(a.ccount[i], a.K);
        const float4* e = a.ctab + static_cast<size_t>(i) * a.K * 4;
        for (int k = 0; k < nc; ++k, e += 4) {
            const float4 e0 = e[0], e1 = e[1], e2 = e[2], e3 = e[3];
            contact_eval(x, xyz(pv), xyz(e0), xyz(e1), xyz(e2), pi.z, make_float4(e0.w, e1.w, e2.w, e3.x), a.dt,
                         a.eps_u, fc, hc);
        }
    } else if (a.ccount) {
        accumulate_contacts(a, i, x, xyz(pv), pi.z, fc, hc);
    }
    if (a.sc_f) {
        const float4 s0 = a.sc_f[i], s1 = a.sc_h0[i], s2 = a.sc_h1[i];
        fc = fc + xyz(s0);
        hc.xx += s1.x;
        hc.xy += s1.y;
        hc.xz += s1.z;
        hc.yy += s1.w;
        hc.yz += s2.x;
        hc.zz += s2.y;
    }
    // h_total = h_elastic + m/dt^2 I + h_contact ; f_total = f_elastic + m (y - x)/dt^2 + f_contact
    add_diag(h, mass * a.dt_sqr_recip);
    add(h, hc);
    const float3 fi = (mass * (xyz(yv) - x)) * a.dt_sqr_recip;
    f = f + fi + fc;
}

// The vertex's Newton step on its 3x3 block: disp += H^-1 f when |det H| > 1e-8 and the result is
// finite (else counted and skipped, as the reference skips it), then q = prev + disp when the
// color commits in place (solve_elasticity(_tile) + apply_truncation_ts without self-contact).
__device__ __forceinline__ void solve_and_commit(const SweepArgs& a, int i, float4 pv, const Sym3& h, float3 f) {
    float3 dx;
    float4 d = a.disp[i];
    if (solve3(h, f, dx)) {
        if (isfinite(dx.x) && isfinite(dx.y) && isfinite(dx.z)) {
            d = make_float4(d.x + dx.x, d.y + dx.y, d.z + dx.z, 0.f);
            a.disp[i] = d;
        } else {
            atomicAdd(&a.status[kNonfinite], 1u);
        }
    } else {
        atomicAdd(&a.status[kSingular], 1u);
    }
    if (a.write_pos) a.pos[i] = make_float4(pv.x + d.x, pv.y + d.y, pv.z + d.z, 0.f);
}

// Fixed-point scale of the residual sums (units of m|g|): r is rounded to 1/256 and clamped at
// kResidSumClamp, so 2^64 holds the sum of ~7e7 clamped residuals
constexpr float kResidSumScale = 256.0f;
constexpr float kResidSumClamp = 1.0e9f;

__device__ __forceinline__ unsigned long long resid_fixed(float r) {
    // NaN and values beyond the clamp count as the clamp
    const float c = (r <= kResidSumClamp) ? r : kResidSumClamp;
    return static_cast<unsigned long long>(c * kResidSumScale + 0.5f);
}

// Warp-collective (one full warp): the gate's residual norm of the current evaluation -- the max,
// or the sum over the solved vertices divided by their number -- from the slots, which are
// cleared for the next evaluation.  Every lane returns the norm.
__device__ __forceinline__ float gate_take_warp(GateState* g, int mean, int count) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned long long sum = 0ull;
    unsigned mx0 = 0u;
#pragma unroll
    for (int k = lane; k < kGateSlots; k += 32) {
        sum += g->sum[k * kSumStride];
        mx0 = max(mx0, g->maxv[k * kMaxStride]);
        g->sum[k * kSumStride] = 0ull;
        g->maxv[k * kMaxStride] = 0u;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(full, sum, off);
    const unsigned mx = __reduce_max_sync(full, mx0);
    if (!mean) return __uint_as_float(mx);
    if (count <= 0) return 0.0f;
    return static_cast<float>(static_cast<double>(sum) / kResidSumScale / static_cast<double>(count));
}

// One thread: record the check of residual norm r and set the while node's condition.
__device__ __forceinline__ void gate_decide(GateState* g, cudaGraphConditionalHandle handle, float r,
                                            const GateParams& p) {
    const bool is_first = p.first == 1 || (p.first == -1 && g->iters == 0);
    if (is_first) {
        g->start_resid = r;
        if (p.set_ref) g->ref = r;
    }
    if (p.first != 1) g->iters += p.add;
    const float thresh = p.relative ? p.tol * g->ref : p.tol;
    const bool more = (r > thresh) && (g->iters < p.max_iters);
    if (!more) {
        g->stop = 1u;
        g->last_iters = g->iters;
        g->last_resid = r;
        g->steps += 1ull;
        g->iter_sum += static_cast<unsigned long long>(g->iters);
        if (r > thresh) g->capped += 1ull;
        if (p.first != 1) {
            const int checks = p.add > 0 ? (g->iters + p.add - 1) / p.add : 0;
            g->passes += static_cast<unsigned long long>((checks + p.rounds - 1) / p.rounds);
        }
    }
    // the condition keeps its value between loop passes: write it only where it changes (the
    // start evaluation of Jacobi mode, whose default is 0; the stop)
    if (!more || p.first == 1) cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// Warp-collective: every thread of the warp calls it (r = 0 and counted = false where the thread
// holds no vertex).  Max (float bits as unsigned: exact for r >= 0; NaN bits exceed +inf) and the
// fixed-point sum go to the accumulators with one atomic each per warp: the single max of
// vbd_residual, and the residual gate's slots (slot = global warp index mod kGateSlots).
__device__ __forceinline__ void reduce_residual(const SweepArgs& a, float r, bool counted) {
    const unsigned full = 0xffffffffu;
    const unsigned mx = __reduce_max_sync(full, __float_as_uint(r));
    const bool any = __any_sync(full, counted);
    unsigned long long sum = 0ull;
    if (a.gate_sum) {
        sum = counted ? resid_fixed(r) : 0ull;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(full, sum, off);
    }
    if ((threadIdx.x & 31) == 0 && any) {
        const int slot = static_cast<int>(((blockIdx.x * blockDim.x + threadIdx.x) >> 5) & (kGateSlots - 1));
        if (a.resid_max) atomicMax(reinterpret_cast<unsigned*>(a.resid_max), mx);
        if (a.gate_max) atomicMax(a.gate_max + slot * kMaxStride, mx);
        if (a.gate_sum) atomicAdd(a.gate_sum + slot * kSumStride, sum);
    }
}

// Warp-collective (every thread of the warp calls it): the same reduction for a sweep whose
// vertices are held by lanes 0, L, 2L, ... of each warp (the others pass r = 0): the warp's values
// are combined over those lanes only and lane 0 adds the warp's sum (and max, in max mode) to slot
// (global warp index mod kGateSlots).  Integer sums: the result does not depend on the order.
template <int L>
__device__ __forceinline__ void reduce_residual_lanes(const SweepArgs& a, float r, bool counted) {
    const unsigned full = 0xffffffffu;
    const bool want_max = a.gate_max != nullptr;
    unsigned mx = __float_as_uint(r);
    unsigned long long sum = counted ? resid_fixed(r) : 0ull;
#pragma unroll
    for (int off = 16; off >= L; off >>= 1) {
        sum += __shfl_xor_sync(full, sum, off);
        if (want_max) mx = max(mx, __shfl_xor_sync(full, mx, off));
    }
    // one atomic per warp, spread over the slots by global warp index: no block barrier at the
    // end of the sweep (a block-level reduction before one atomic per block cost 0.7 us per
    // iteration at 65,536 vertices and 8 us at 1.89 M)
    if ((threadIdx.x & 31) == 0) {
        const int slot = static_cast<int>(((blockIdx.x * blockDim.x + threadIdx.x) >> 5) & (kGateSlots - 1));
        if (want_max) atomicMax(a.gate_max + slot * kMaxStride, mx);
        if (a.gate_sum && sum) atomicAdd(a.gate_sum + slot * kSumStride, sum);
    }
}

// One Gauss-Seidel color (kResidual = false) or a Jacobi residual evaluation over a vertex range
// (kResidual = true).  L lanes cooperate on one vertex: each lane takes every L-th element record
// (triangles, then hinges, as the reference's 16-thread tile does), then the partial force and
// Hessian are summed across the L lanes with xor shuffles and lane 0 adds the contacts and solves.
// kCap: the same kernel limited to 64 registers per thread (4 blocks of 256 per SM), used when the
// uncapped kernel would need more than one wave of blocks (large colors, many lanes per vertex)
template <int L, bool kDamp, bool kResidual, bool kCap, bool kGate, bool kStaged = false>
__device__ __forceinline__ void sweep_body(const SweepArgs& a) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = a.v_begin + tid / L;
    const int lane = tid & (L - 1);
    const bool valid = i < a.v_end;
    float3 f = f3(0.f, 0.f, 0.f);
    Sym3 h = zero_sym();
    bool solve = false;
    float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
    int4 adj = make_int4(0, 0, 0, 0);
    if (valid) {
        // vertex info and record ranges never change during a step: read them before waiting on
        // the previous kernel (programmatic dependent launch; a no-op in an ordinary launch)
        pi = __ldg(&a.pinfo[i]);
        adj = __ldg(&a.vadj[i]);
        solve = (__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f;
        if (solve && !kResidual && !kCap && a.prefetch_records) {
            // the vertex's element records are static too: start bringing them into L2 while the
            // previous color still runs (asked for on the first iteration of a step, after the
            // records may have left L2; the register-capped build, used for grids of several
            // waves, runs slower with it)
            prefetch_rows_l2(a.tri_idx, adj.x, adj.y, lane, L);
            prefetch_rows_l2(a.tri_D, adj.x, adj.y, lane, L);
            prefetch_rows_l2(a.tri_mat, adj.x, adj.y, lane, L);
            prefetch_rows_l2(a.edge_idx, adj.z, adj.w, lane, L);
            prefetch_rows_l2(a.edge_mat, adj.z, adj.w, lane, L);
        }
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;");
    // a round of the gate's loop body after the decision: nothing to do (the flag was written by
    // an earlier kernel of the stream and is the same for every thread of the grid)
    if (a.gate_stop && *reinterpret_cast<const volatile unsigned*>(a.gate_stop) != 0u) return;
    const float4* s_pos = s_stage;
    const float4* s_prev = s_stage;
    if (kStaged) {
        // the block's one-ring: one coalesced pass over the patch ids, one gather per position
        // (the previous kernel's writes are visible after griddepcontrol.wait), then every record
        // of the block reads its positions from shared memory
        const int p = a.patch_base + static_cast<int>(blockIdx.x);
        const int b0 = __ldg(&a.patch_off[p]), n = __ldg(&a.patch_off[p + 1]) - b0;
        float4* sp = s_stage;
        float4* sq = s_stage + n;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int g = __ldg(&a.patch_ids[b0 + j]);
            sp[j] = a.pos[g];
            if (kDamp) sq[j] = __ldg(&a.prev[g]);
        }
        s_prev = sq;
        __syncthreads();
    }
    if (valid && solve && lane == 0) {
        // Warm L1 with what lane 0 reads after the element walk (the vertex's own state, its
        // contact count, its self-contact terms): a prefetch holds no register, so the walk keeps
        // the register budget at which two color grids fit on an SM together and the next color's
        // launch overlaps this one.  (The packed contacts themselves are not prefetched: most
        // vertices have none, and their unused entries would be fetched from DRAM.)
        prefetch_l1(&a.prev[i]);
        prefetch_l1(&a.pos[i]);
        prefetch_l1(&a.y[i]);
        prefetch_l1(&a.disp[i]);
        if (a.ctab) prefetch_l1(&a.ccount[i]);
        if (a.sc_f) {
            prefetch_l1(&a.sc_f[i]);
            prefetch_l1(&a.sc_h0[i]);
            prefetch_l1(&a.sc_h1[i]);
        }
    }
    if (valid && solve) {
        if (kStaged && L <= 2 && !kCap) accumulate_elements_staged_x2<kDamp>(a, lane, L, adj, s_pos, s_prev, f, h);
        else if (kStaged) accumulate_elements_staged<kDamp>(a, lane, L, adj, s_pos, s_prev, f, h);
        else if (L <= 2 && !kCap) accumulate_elements_x2<kDamp>(a, lane, L, adj, f, h);
        else accumulate_elements<kDamp>(a, i, lane, L, adj, f, h);
    }
    if (L > 1) {
        f.x = warp_sum(f.x, L);
        f.y = warp_sum(f.y, L);
        f.z = warp_sum(f.z, L);
        if (!kResidual) {
            // the Jacobi residual reads the force only: without these reductions the compiler
            // drops the Hessian arithmetic of every element evaluation from that instantiation
            h.xx = warp_sum(h.xx, L);
            h.xy = warp_sum(h.xy, L);
            h.xz = warp_sum(h.xz, L);
            h.yy = warp_sum(h.yy, L);
            h.yz = warp_sum(h.yz, L);
            h.zz = warp_sum(h.zz, L);
        }
    }
    if (kResidual) {
        // Jacobi residual: lane 0 of each vertex forms r_i, then the warp reduces max, sum and
        // count before one atomic per warp (fixed shuffle tree + integer atomics: deterministic)
        float r = 0.0f;
        bool counted = false;
        if (valid && lane == 0) {
            if (solve) {
                const float4 pv = a.prev[i];
                const float4 yv = a.y[i];
                add_vertex_terms(a, i, pi, pv, xyz(a.pos[i]), yv, f, h);
                r = length(f) / yv.w * a.inv_g;
                counted = true;
            }
            if (a.resid_out) a.resid_out[a.perm[i]] = r;
        }
        reduce_residual(a, r, counted);
        return;
    }
    if (kGate) {
        // the same update, and the vertex's force norm before it (the Gauss-Seidel residual of
        // the sweep) reduced per block into the residual gate's accumulators
        float rg = 0.0f;
        bool counted = false;
        if (valid && lane == 0) {
            const float4 pv = a.prev[i];
            if (!solve) {
                a.disp[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (a.write_pos) a.pos[i] = pv;
            } else {
                const float4 yv = a.y[i];
                add_vertex_terms(a, i, pi, pv, xyz(a.pos[i]), yv, f, h);
                rg = length(f) / yv.w * a.inv_g;
                counted = true;
                solve_and_commit(a, i, pv, h, f);
            }
        }
        reduce_residual_lanes<L>(a, rg, counted);
        return;
    }
    if (!valid || lane != 0) return;
    const float4 pv = a.prev[i];
    if (!solve) {
        a.disp[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a.write_pos) a.pos[i] = pv;
        return;
    }
    add_vertex_terms(a, i, pi, pv, xyz(a.pos[i]), a.y[i], f, h);
    solve_and_commit(a, i, pv, h, f);
}

template <int L, bool kDamp, bool kResidual, bool kCap, bool kGate = false, bool kStaged = false>
__global__ void __launch_bounds__(256, kCap ? 4 : 1) sweep_kernel(SweepArgs a) {
    sweep_body<L, kDamp, kResidual, kCap, kGate, kStaged>(a);
}

// The gate's accumulating sweep with 4 or more lanes per vertex, held to the 72 registers of the
// plain sweep: at 74 (what the compiler picks for the extra reduction) the allocation rounds up
// to 80 registers per thread, two color grids no longer fit on an SM together, and each launch
// loses its overlap with the previous one.
template <int L, bool kDamp, bool kStaged = false>
__global__ void __maxnreg__(72) sweep_gate_kernel(SweepArgs a) {
    sweep_body<L, kDamp, false, false, true, kStaged>(a);
}

// The staged sweep at 4 or more lanes, held to the same 72 registers (unbounded, the damping
// build takes 79).
template <int L, bool kDamp>
__global__ void __maxnreg__(72) sweep_staged_kernel(SweepArgs a) {
    sweep_body<L, kDamp, false, false, false, true>(a);
}

// Record-parallel variant of the same color update (lanes_per_vertex == 0).  A block owns
// VT = TB/16 consecutive vertices of the color and the contiguous runs of element records they
// own.  Every thread evaluates one record at a time (all triangles of the tile, then all hinges),
// writing its force/Hessian contribution to shared memory; then 9 reducer threads per vertex --
// one per component -- add the vertex's contributions in record order, starting from the
// inertia term.  That is the summation order of the reference's serial path
// (solve_elasticity, particle_vbd_kernels.py:2568-2706): inertia, triangles in CSR order, hinges
// in CSR order, then the accumulated contact force and Hessian.  The order never depends on
// thread scheduling, so results are deterministic.
template <int TB, bool kDamp, bool kResidual>
__global__ void __launch_bounds__(TB) tile_kernel(SweepArgs a) {
    constexpr int VT = TB / 16;
    constexpr int MAXR = 2 * TB;
    constexpr int STRIDE = MAXR + 1;  // odd row stride: the 9 reducers of a vertex hit 9 banks
    static_assert(VT * 9 <= TB, "one reducer thread per vertex component");
    __shared__ float s_c[9 * STRIDE];
    __shared__ int4 s_adj[VT];
    __shared__ float s_sum[VT][9];
    const int vb = a.v_begin + blockIdx.x * VT;
    const int nv = min(VT, a.v_end - vb);
    const int t = threadIdx.x;
    if (t < nv) s_adj[t] = __ldg(&a.vadj[vb + t]);
    __syncthreads();
    const int rv = t / 9;
    const int rc = t - 9 * rv;
    const bool reducer = rv < nv;
    float acc = 0.0f;
    if (reducer) {
        // inertia: f = m (y - x) / dt^2, H = m / dt^2 I  (zero for vertices that own no records)
        const int4 ad = s_adj[rv];
        if (ad.y > ad.x || ad.w > ad.z) {
            const float4 yv = __ldg(&a.y[vb + rv]);
            const float4 xv = a.pos[vb + rv];
            const float m = yv.w;
            if (rc < 3) {
                const float d = rc == 0 ? yv.x - xv.x : (rc == 1 ? yv.y - xv.y : yv.z - xv.z);
                acc = (m * d) * a.dt_sqr_recip;
            } else if (rc == 3 || rc == 6 || rc == 8) {
                acc = m * a.dt_sqr_recip;
            }
        }
    }
    // One merged list per tile: the tile's triangle records, then its hinge records.  Component
    // order in shared memory: f.x f.y f.z h.xx h.xy h.xz h.yy h.yz h.zz.
    const int tb = s_adj[0].x, nt = s_adj[nv - 1].y - tb;
    const int eb = s_adj[0].z, ne = s_adj[nv - 1].w - eb;
    const int ntot = nt + ne;
    for (int base = 0; base < ntot; base += MAXR) {
        const int n = min(MAXR, ntot - base);
        for (int r = t; r < n; r += TB) {
            float3 f = f3(0.f, 0.f, 0.f);
            Sym3 h = zero_sym();
            const int k = base + r;
            if (k < nt) {
                const int rec = tb + k;
                const int4 ti = __ldg(&a.tri_idx[rec]);
                const float4 D = __ldg(&a.tri_D[rec]);
                const float4 mt = __ldg(&a.tri_mat[rec]);
                const float3 x0 = xyz(a.pos[ti.x]), x1 = xyz(a.pos[ti.y]), x2 = xyz(a.pos[ti.z]);
                float3 p0 = x0, p1 = x1, p2 = x2;
                if (kDamp && mt.w > 0.0f) {
                    p0 = xyz(__ldg(&a.prev[ti.x]));
                    p1 = xyz(__ldg(&a.prev[ti.y]));
                    p2 = xyz(__ldg(&a.prev[ti.z]));
                }
                membrane_eval<kDamp>(ti.w, x0, x1, x2, p0, p1, p2, D, mt, a.inv_dt, f, h);
            } else {
                const int rec = eb + (k - nt);
                const int4 ei = __ldg(&a.edge_idx[rec]);
                const float4 em = __ldg(&a.edge_mat[rec]);
                const int order = static_cast<int>(static_cast<unsigned>(ei.x) >> 30);
                const int o0 = ei.x & 0x3fffffff;
                const float3 x0 = xyz(a.pos[o0]), x1 = xyz(a.pos[ei.y]), x2 = xyz(a.pos[ei.z]),
                             x3 = xyz(a.pos[ei.w]);
                float3 p0 = x0, p1 = x1, p2 = x2, p3 = x3;
                if (kDamp && em.w > 0.0f) {
                    p0 = xyz(__ldg(&a.prev[o0]));
                    p1 = xyz(__ldg(&a.prev[ei.y]));
                    p2 = xyz(__ldg(&a.prev[ei.z]));
                    p3 = xyz(__ldg(&a.prev[ei.w]));
                }
                bending_eval<kDamp>(order, x0, x1, x2, x3, p0, p1, p2, p3, em, a.inv_dt, f, h);
            }
            s_c[0 * STRIDE + r] = f.x;
            s_c[1 * STRIDE + r] = f.y;
            s_c[2 * STRIDE + r] = f.z;
            s_c[3 * STRIDE + r] = h.xx;
            s_c[4 * STRIDE + r] = h.xy;
            s_c[5 * STRIDE + r] = h.xz;
            s_c[6 * STRIDE + r] = h.yy;
            s_c[7 * STRIDE + r] = h.yz;
            s_c[8 * STRIDE + r] = h.zz;
        }
        __syncthreads();
        if (reducer) {
            // this vertex's triangles, then its hinges, in record order
            const int4 ad = s_adj[rv];
            const float* row = s_c + rc * STRIDE - base;
            int lo = max(ad.x - tb, base), hi = min(ad.y - tb, base + n);
            for (int r = lo; r < hi; ++r) acc += row[r];
            lo = max(nt + ad.z - eb, base);
            hi = min(nt + ad.w - eb, base + n);
            for (int r = lo; r < hi; ++r) acc += row[r];
        }
        __syncthreads();
    }
    if (reducer) s_sum[rv][rc] = acc;
    __syncthreads();
    if (t >= nv) return;
    const int i = vb + t;
    const float4 pv = a.prev[i];
    const int4 ad = s_adj[t];
    const float4 pi = __ldg(&a.pinfo[i]);
    const bool solve = (__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f;
    if (!solve) {
        if (kResidual) {
            if (a.resid_out) a.resid_out[a.perm[i]] = 0.0f;
        } else {
            a.disp[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (a.write_pos) a.pos[i] = pv;
        }
        return;
    }
    float3 f;
    Sym3 h;
    if (ad.y > ad.x || ad.w > ad.z) {
        f = f3(s_sum[t][0], s_sum[t][1], s_sum[t][2]);
        h.xx = s_sum[t][3];
        h.xy = s_sum[t][4];
        h.xz = s_sum[t][5];
        h.yy = s_sum[t][6];
        h.yz = s_sum[t][7];
        h.zz = s_sum[t][8];
    } else {
        // a solvable vertex without elements: inertia only
        const float4 yv = __ldg(&a.y[i]);
        const float4 xv = a.pos[i];
        f = (yv.w * (xyz(yv) - xyz(xv))) * a.dt_sqr_recip;
        h = zero_sym();
        add_diag(h, yv.w * a.dt_sqr_recip);
    }
    float3 fc = f3(0.f, 0.f, 0.f);
    Sym3 hc = zero_sym();
    if (a.ccount) accumulate_contacts(a, i, xyz(a.pos[i]), xyz(pv), pi.z, fc, hc);
    if (a.sc_f) add_self_contact(a, i, fc, hc);
    add(h, hc);
    f = f + fc;
    if (kResidual) {
        const float r = length(f) / pi.x * a.inv_g;
        if (a.resid_out) a.resid_out[a.perm[i]] = r;
        // one vertex per thread here: plain per-vertex atomics (integer, so still deterministic)
        if (a.resid_max) atomicMax(reinterpret_cast<unsigned*>(a.resid_max), __float_as_uint(r));
        const int slot = static_cast<int>(i & (kGateSlots - 1));
        if (a.gate_max) atomicMax(a.gate_max + slot * kMaxStride, __float_as_uint(r));
        if (a.gate_sum) atomicAdd(a.gate_sum + slot * kSumStride, resid_fixed(r));
        return;
    }
    float3 dx;
    float4 d = a.disp[i];
    if (solve3(h, f, dx)) {
        if (isfinite(dx.x) && isfinite(dx.y) && isfinite(dx.z)) {
            d = make_float4(d.x + dx.x, d.y + dx.y, d.z + dx.z, 0.f);
            a.disp[i] = d;
        } else {
            atomicAdd(&a.status[kNonfinite], 1u);
        }
    } else {
        atomicAdd(&a.status[kSingular], 1u);
    }
    if (a.write_pos) a.pos[i] = make_float4(pv.x + d.x, pv.y + d.y, pv.z + d.z, 0.f);
}

// Commit of a color when the coloring is not conflict-free for every element stencil: the
// sweep then leaves positions untouched (Jacobi within the color, as the reference's separate
// apply_truncation_ts launch does) and this pass writes q = prev + disp.
__global__ void commit_kernel(float4* pos, const float4* prev, const float4* disp, int b, int e) {
    const int i = b + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    const float4 p = prev[i], d = disp[i];
    pos[i] = make_float4(p.x + d.x, p.y + d.y, p.z + d.z, 0.f);
}

struct FinalizeArgs {
    const int* perm;
    const float4* pos;
    const float4* prev;
    float* q_in;
    float* q_out;
    float* qd_out;
    int* ccount;
    // learned warm start: the step's correction x_solved - y, internal order (NULL: not kept)
    const float4* pinfo;
    const float4* y;
    float* corr;
    int V;
    float dt;
};

__global__ void finalize_kernel(FinalizeArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.V) return;
    const int o = a.perm[i];
    const float4 p = a.pos[i], pv = a.prev[i];
    if (a.q_in) {
        a.q_in[3 * o] = p.x;
        a.q_in[3 * o + 1] = p.y;
        a.q_in[3 * o + 2] = p.z;
    }
    if (a.q_out) {
        a.q_out[3 * o] = p.x;
        a.q_out[3 * o + 1] = p.y;
        a.q_out[3 * o + 2] = p.z;
    }
    if (a.qd_out) {
        a.qd_out[3 * o] = (p.x - pv.x) / a.dt;
        a.qd_out[3 * o + 1] = (p.y - pv.y) / a.dt;
        a.qd_out[3 * o + 2] = (p.z - pv.z) / a.dt;
    }
    if (a.ccount) a.ccount[i] = 0;
    if (a.corr) {
        const float4 pi = a.pinfo[i];
        const bool solvable = (__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f;
        const float4 yy = a.y[i];
        a.corr[3 * i] = solvable ? p.x - yy.x : 0.f;
        a.corr[3 * i + 1] = solvable ? p.y - yy.y : 0.f;
        a.corr[3 * i + 2] = solvable ? p.z - yy.z : 0.f;
    }
}

// Warm start: the initial Gauss-Seidel iterate becomes inertia target + delta for every vertex the
// sweep solves (pinned / massless vertices keep their position).
__global__ void warm_start_kernel(const int* perm, const float4* pinfo, const float4* prev, float4* disp, float4* pos,
                                  const float* delta, int V, int internal = 0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const float4 pi = pinfo[i];
    if (!((__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f)) return;
    const int o = internal ? i : perm[i];  // row of delta
    float4 d = disp[i];
    d = make_float4(d.x + delta[3 * o], d.y + delta[3 * o + 1], d.z + delta[3 * o + 2], 0.f);
    disp[i] = d;
    const float4 p = prev[i];
    pos[i] = make_float4(__fadd_rn(p.x, d.x), __fadd_rn(p.y, d.y), __fadd_rn(p.z, d.z), 0.f);
}

// out[3 i + k] = in[3 perm[i] + k]: a [V,3] model-order array into the internal order
__global__ void gather_rows3_kernel(const int* perm, const float* in, float* out, int V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const int o = perm[i];
    out[3 * i] = in[3 * o];
    out[3 * i + 1] = in[3 * o + 1];
    out[3 * i + 2] = in[3 * o + 2];
}

__global__ void gather_positions_kernel(const int* perm, const float4* pos, float* q, int V) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= V) return;
    const int o = perm[i];
    const float4 p = pos[i];
    q[3 * o] = p.x;
    q[3 * o + 1] = p.y;
    q[3 * o + 2] = p.z;
}

// Residual gate: after an evaluation of the residual (a Jacobi evaluation, a kResidual sweep over
// every solved vertex; or the Gauss-Seidel residual the last round's sweeps accumulated) decide
// whether the loop runs another round.  One warp.
__global__ void gate_check_kernel(GateState* g, cudaGraphConditionalHandle handle, GateParams p) {
    // launched as a programmatic dependent of the round's last sweep: wait for that grid (its
    // accumulators), then let the next sweep start its prologue (it waits for this grid in turn)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;");
    if (p.first != 1 && g->stop) return;  // a later round of a loop body that has already decided
    const float r = gate_take_warp(g, p.mean, p.count);
    if (threadIdx.x == 0) gate_decide(g, handle, r, p);
}

// relative mode with a warm start: the residual at the plain start y becomes the reference
__global__ void gate_ref_kernel(GateState* g, int mean, int count) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;");
    const float r = gate_take_warp(g, mean, count);
    if (threadIdx.x == 0) g->ref = r;
}

// ---------------------------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------------------------
static SweepArgs make_sweep_args(const SolverImpl& s, const VbdContacts* c, float dt) {
    const VbdModelImpl& m = *s.m;
    SweepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.pos = s.pos;
    a.prev = s.prev;
    a.y = s.y;
    a.disp = s.disp;
    a.vadj = m.vadj;
    a.pinfo = m.pinfo;
    a.tri_idx = m.tri_idx;
    a.tri_D = m.tri_D;
    a.tri_mat = m.tri_mat;
    a.edge_idx = m.edge_idx;
    a.edge_mat = m.edge_mat;
    a.K = s.K;
    if (c && m.S > 0) {
        a.ccount = s.ccount;
        a.cslot = s.cslot;
        a.c_shape = c->soft_contact_shape;
        a.c_body_pos = c->soft_contact_body_pos;
        a.c_body_vel = c->soft_contact_body_vel;
        a.c_normal = c->soft_contact_normal;
        a.shapes = m.shapes;
        a.ctab = s.ctab;
    }
    a.dt = dt;
    a.inv_dt = 1.0f / dt;
    a.dt_sqr_recip = 1.0f / (dt * dt);
    a.eps_u = s.friction_epsilon * dt;
    a.status = s.status;
    a.write_pos = m.fused_commit ? 1 : 0;
    if (s.sc.on) {
        // positions are written by the truncation pass after the color (pos = cd + disp)
        a.sc_f = s.sc.sc_f;
        a.sc_h0 = s.sc.sc_h0;
        a.sc_h1 = s.sc.sc_h1;
        a.write_pos = 0;
    }
    a.perm = m.perm;
    a.inv_g = m.gravity_norm > 0.f ? 1.0f / m.gravity_norm : 0.f;
    a.no_pdl = s.pdl ? 0 : 1;
    return a;
}

static GateParams gate_params(const SolverImpl& s, int first, int set_ref, int add) {
    GateParams p;
    p.tol = s.gate_tol;
    p.max_iters = s.gate_max;
    p.relative = s.gate_relative;
    p.mean = s.gate_mean;
    p.count = s.gate_count;
    p.first = first;
    p.set_ref = set_ref;
    p.add = add;
    p.rounds = (s.gate_sweep && s.lanes > 0) ? s.gate_rounds : 1;
    return p;
}

// blocks of `kernel` resident on the whole device at `block` threads (cached per kernel / block)
static long long resident_blocks(const void* kernel, int block, size_t smem = 0) {
    static std::mutex mu;
    static std::map<std::pair<const void*, long long>, long long> cache;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(kernel, static_cast<long long>(block) | (static_cast<long long>(smem) << 16));
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
    const long long n = static_cast<long long>(std::max(per_sm, 1)) * std::max(sms, 1);
    cache[key] = n;
    return n;
}

// Sweeps are launched as programmatic dependents of the previous kernel on the stream: their
// blocks may start while that kernel drains and wait (griddepcontrol.wait) before reading any
// position, so consecutive colors overlap launch latency instead of serialising it.
template <typename Kernel>
static void launch_dependent(Kernel kernel, int grid, int block, cudaStream_t st, const SweepArgs& a,
                             size_t smem = 0) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = a.no_pdl ? 0 : 1;
    cudaLaunchKernelEx(&cfg, kernel, a);
}

// a one-warp gate kernel as a programmatic dependent of the kernel before it (pdl), so that its
// launch overlaps that kernel's tail instead of following its completion
template <typename... Args>
static void launch_gate(void (*kernel)(Args...), cudaStream_t st, bool pdl, Args... args) {
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(32);
    cfg.stream = st;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

// the staged instantiations: the same choice between the uncapped (or 72-register gate) kernel
// and the 64-register one, with the patch's shared memory counted in the occupancy
template <int L, bool kDamp, bool kGate>
static void launch_staged_LDG(const SweepArgs& a, int grid, int block, cudaStream_t st, size_t smem) {
    if constexpr (kGate && L >= 4) {
        if (grid > resident_blocks(reinterpret_cast<const void*>(&sweep_gate_kernel<L, kDamp, true>), block, smem))
            launch_dependent(sweep_kernel<L, kDamp, false, true, kGate, true>, grid, block, st, a, smem);
        else
            launch_dependent(sweep_gate_kernel<L, kDamp, true>, grid, block, st, a, smem);
    } else if constexpr (kGate || L <= 2) {
        // (at 1-2 lanes the two-record walk needs more than 72 registers, as unstaged)
        const void* uncapped = reinterpret_cast<const void*>(&sweep_kernel<L, kDamp, false, false, kGate, true>);
        if (grid > resident_blocks(uncapped, block, smem))
            launch_dependent(sweep_kernel<L, kDamp, false, true, kGate, true>, grid, block, st, a, smem);
        else
            launch_dependent(sweep_kernel<L, kDamp, false, false, kGate, true>, grid, block, st, a, smem);
    } else {
        if (grid > resident_blocks(reinterpret_cast<const void*>(&sweep_staged_kernel<L, kDamp>), block, smem))
            launch_dependent(sweep_kernel<L, kDamp, false, true, false, true>, grid, block, st, a, smem);
        else
            launch_dependent(sweep_staged_kernel<L, kDamp>, grid, block, st, a, smem);
    }
}

template <int L>
static void prime_staged_occupancy_L(int block, size_t smem) {
    if constexpr (L >= 4) {
        resident_blocks(reinterpret_cast<const void*>(&sweep_staged_kernel<L, true>), block, smem);
        resident_blocks(reinterpret_cast<const void*>(&sweep_staged_kernel<L, false>), block, smem);
    } else {
        resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, true, false, false, false, true>), block, smem);
        resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, false, false, false, false, true>), block, smem);
    }
    if constexpr (L >= 4) {
        resident_blocks(reinterpret_cast<const void*>(&sweep_gate_kernel<L, true, true>), block, smem);
        resident_blocks(reinterpret_cast<const void*>(&sweep_gate_kernel<L, false, true>), block, smem);
    } else {
        resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, true, false, false, true, true>), block, smem);
        resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, false, false, false, true, true>), block, smem);
    }
}

template <int L, bool kDamp, bool kResidual, bool kGate = false>
static void launch_sweep_LDR(const SweepArgs& a, int grid, int block, cudaStream_t st, size_t smem = 0) {
    if constexpr (!kResidual) {
        if (a.patch_off) {
            launch_staged_LDG<L, kDamp, kGate>(a, grid, block, st, smem);
            return;
        }
    }
    if constexpr (kGate && !kResidual && L >= 4) {
        if (grid > resident_blocks(reinterpret_cast<const void*>(&sweep_gate_kernel<L, kDamp>), block))
            launch_dependent(sweep_kernel<L, kDamp, kResidual, true, kGate>, grid, block, st, a);
        else
            launch_dependent(sweep_gate_kernel<L, kDamp>, grid, block, st, a);
    } else {
        const void* uncapped = reinterpret_cast<const void*>(&sweep_kernel<L, kDamp, kResidual, false, kGate>);
        if (grid > resident_blocks(uncapped, block))
            launch_dependent(sweep_kernel<L, kDamp, kResidual, true, kGate>, grid, block, st, a);
        else
            launch_dependent(sweep_kernel<L, kDamp, kResidual, false, kGate>, grid, block, st, a);
    }
}

// occupancy queries happen here, outside any stream capture (solver creation, vbd_set_launch)
template <int L>
static void prime_occupancy_L(int block) {
    resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, true, true, false>), block);
    resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, false, true, false>), block);
    resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, true, false, false>), block);
    resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, false, false, false>), block);
    resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, true, false, false, true>), block);
    resident_blocks(reinterpret_cast<const void*>(&sweep_kernel<L, false, false, false, true>), block);
    if constexpr (L >= 4) {
        resident_blocks(reinterpret_cast<const void*>(&sweep_gate_kernel<L, true>), block);
        resident_blocks(reinterpret_cast<const void*>(&sweep_gate_kernel<L, false>), block);
    }
}

static void prime_occupancy(int lanes, int block) {
    switch (lanes) {
        case 1: prime_occupancy_L<1>(block); break;
        case 2: prime_occupancy_L<2>(block); break;
        case 4: prime_occupancy_L<4>(block); break;
        case 8: prime_occupancy_L<8>(block); break;
        case 16: prime_occupancy_L<16>(block); break;
        default: break;
    }
}

template <int L>
static void launch_sweep_L(const SweepArgs& a, bool damp, bool residual, int block, cudaStream_t st, bool gate,
                           size_t smem) {
    const long long threads = static_cast<long long>(a.v_end - a.v_begin) * L;
    const int grid = static_cast<int>((threads + block - 1) / block);
    if (grid <= 0) return;
    if (gate && !residual) {
        if (damp) launch_sweep_LDR<L, true, false, true>(a, grid, block, st, smem);
        else launch_sweep_LDR<L, false, false, true>(a, grid, block, st, smem);
        return;
    }
    if (residual) {
        if (damp) launch_sweep_LDR<L, true, true>(a, grid, block, st);
        else launch_sweep_LDR<L, false, true>(a, grid, block, st);
    } else {
        if (damp) launch_sweep_LDR<L, true, false>(a, grid, block, st, smem);
        else launch_sweep_LDR<L, false, false>(a, grid, block, st, smem);
    }
}

template <int TB>
static void launch_tile_TB(const SweepArgs& a, bool damp, bool residual, cudaStream_t st) {
    constexpr int VT = TB / 16;
    const int grid = (a.v_end - a.v_begin + VT - 1) / VT;
    if (grid <= 0) return;
    if (residual) {
        if (damp) tile_kernel<TB, true, true><<<grid, TB, 0, st>>>(a);
        else tile_kernel<TB, false, true><<<grid, TB, 0, st>>>(a);
    } else {
        if (damp) tile_kernel<TB, true, false><<<grid, TB, 0, st>>>(a);
        else tile_kernel<TB, false, false><<<grid, TB, 0, st>>>(a);
    }
}

// gate: a Gauss-Seidel color that also accumulates its residual into a.resid_* (lanes > 0 only)
static void launch_sweep(const SweepArgs& a, int lanes, bool damp, bool residual, int block, cudaStream_t st,
                         bool gate = false, size_t smem = 0) {
    if (lanes == 0) {
        if (block <= 64) launch_tile_TB<64>(a, damp, residual, st);
        else if (block <= 128) launch_tile_TB<128>(a, damp, residual, st);
        else launch_tile_TB<256>(a, damp, residual, st);
        return;
    }
    switch (lanes) {
        case 1: launch_sweep_L<1>(a, damp, residual, block, st, gate, smem); break;
        case 2: launch_sweep_L<2>(a, damp, residual, block, st, gate, smem); break;
        case 8: launch_sweep_L<8>(a, damp, residual, block, st, gate, smem); break;
        case 16: launch_sweep_L<16>(a, damp, residual, block, st, gate, smem); break;
        default: launch_sweep_L<4>(a, damp, residual, block, st, gate, smem); break;
    }
}

static int enqueue_forward(SolverImpl& s, const float* q_in, const float* qd_in, const float* f_ext,
                           const VbdContacts* c, float dt, cudaStream_t st) {
    const VbdModelImpl& m = *s.m;
    s.last_dt = dt;
    ForwardArgs a;
    std::memset(&a, 0, sizeof(a));
    a.perm = m.perm;
    a.inv_perm = m.inv_perm;
    a.pinfo = m.pinfo;
    a.q_in = q_in;
    a.qd_in = qd_in;
    a.f_ext = f_ext;
    a.pos = s.pos;
    a.prev = s.prev;
    a.y = s.y;
    a.disp = s.disp;
    a.V = m.V;
    a.g = make_float3(m.gravity[0], m.gravity[1], m.gravity[2]);
    a.dt = dt;
    a.K = s.K;
    a.ccount = s.ccount;
    a.cslot = s.cslot;
    a.status = s.status;
    int n = m.V;
    if (c && m.S > 0 && c->soft_contact_count) {
        a.c_count = c->soft_contact_count;
        a.c_particle = c->soft_contact_particle;
        a.c_max = c->soft_contact_max;
        n = std::max(n, std::min(c->soft_contact_max, 148 * 2048));
        // the scatter counts into ccount: start it from zero here rather than trusting the previous
        // step's finalize (a staged sequence -- forward and sweeps without finalize, as the launch
        // autotuner runs -- leaves it set)
        VBD_CUDA_TRY(cudaMemsetAsync(s.ccount, 0, sizeof(int) * static_cast<size_t>(m.V), st));
    }
    const int block = 256;
    if (n > 0) forward_kernel<<<(n + block - 1) / block, block, 0, st>>>(a);
    if (a.c_count && s.ctab && m.V > 0) {
        PackArgs p;
        p.ccount = s.ccount;
        p.cslot = s.cslot;
        p.K = s.K;
        p.c_shape = c->soft_contact_shape;
        p.c_body_pos = c->soft_contact_body_pos;
        p.c_body_vel = c->soft_contact_body_vel;
        p.c_normal = c->soft_contact_normal;
        p.shapes = m.shapes;
        p.ctab = s.ctab;
        p.V = m.V;
        pack_contacts_kernel<<<(m.V + block - 1) / block, block, 0, st>>>(p);
    }
    return VBD_OK;
}

// gate: also accumulate the color's Gauss-Seidel residual into the residual gate (sweep mode);
// skip_when_decided: return at once once the step's gate has decided (later rounds of a loop body)
static void enqueue_color(SolverImpl& s, int color, const VbdContacts* c, float dt, cudaStream_t st,
                          bool first_iteration = true, bool gate = false, bool skip_when_decided = false) {
    const VbdModelImpl& m = *s.m;
    SweepArgs a = make_sweep_args(s, c, dt);
    a.prefetch_records = first_iteration ? 1 : 0;
    if (skip_when_decided) a.gate_stop = &s.gate->stop;
    if (gate) {
        a.gate_max = s.gate_mean ? nullptr : s.gate->maxv;
        a.gate_sum = s.gate_mean ? s.gate->sum : nullptr;
    }
    a.v_begin = m.color_start[color];
    a.v_end = m.color_start[color + 1];
    if (a.v_end <= a.v_begin) return;
    size_t smem = 0;
    const bool damp = m.any_tri_damping || m.any_edge_damping;
    if (s.stage_on && s.stage_ready && !s.sc.on && s.lanes == s.stage_lanes && s.block == s.stage_block) {
        a.patch_off = s.patch_off;
        a.patch_ids = s.patch_ids;
        a.tri_loc = s.tri_loc;
        a.edge_loc = s.edge_loc;
        a.patch_base = s.stage_color_base[color];
        smem = static_cast<size_t>(s.stage_max_patch) * sizeof(float4) * (damp ? 2 : 1);
    }
    if (s.sc.on) {
        self_contact_accumulate(m, s.sc, s.pos, s.prev, color, dt, s.friction_epsilon, st);
        launch_sweep(a, s.lanes, m.any_tri_damping || m.any_edge_damping, false, s.block, st);
        self_contact_truncate(m, s.sc, s.pos, s.disp, st);
        return;
    }
    launch_sweep(a, s.lanes, damp, false, s.block, st, gate, smem);
    if (!m.fused_commit) {
        const int n = a.v_end - a.v_begin;
        commit_kernel<<<(n + 255) / 256, 256, 0, st>>>(s.pos, s.prev, s.disp, a.v_begin, a.v_end);
    }
}

static void enqueue_finalize(SolverImpl& s, float* q_in, float* q_out, float* qd_out, float dt, cudaStream_t st,
                             float* corr = nullptr) {
    const VbdModelImpl& m = *s.m;
    FinalizeArgs a;
    a.perm = m.perm;
    a.pinfo = m.pinfo;
    a.y = s.y;
    a.corr = corr;
    a.pos = s.pos;
    a.prev = s.prev;
    a.q_in = q_in;
    a.q_out = q_out;
    a.qd_out = qd_out;
    a.ccount = s.ccount;
    a.V = m.V;
    a.dt = dt;
    if (m.V > 0) finalize_kernel<<<(m.V + 255) / 256, 256, 0, st>>>(a);
}

// Self-contact at the step start, after the forward pass: detection at the step's input
// positions (x_prev, which becomes pos_prev_collision_detection) and the first truncation of the
// forward displacement (solver_vbd.py:2065-2100).
static int self_contact_start(SolverImpl& s, cudaStream_t st) {
    int rc = self_contact_detect(*s.m, s.sc, s.prev, s.disp, false, st);
    if (!rc) rc = self_contact_truncate(*s.m, s.sc, s.pos, s.disp, st);
    return rc;
}

// kernel nodes of a captured graph (memset and other nodes excluded); -1 if it cannot be read.
// The type query of a conditional node fails on this runtime (cudaErrorUnknown) even though the
// graph instantiates and runs: such nodes are skipped, and the error the failed query leaves in
// the runtime's last-error slot is cleared so that it is not reported by an unrelated later call.
static int kernel_nodes(cudaGraph_t graph) {
    size_t n = 0;
    if (cudaGraphGetNodes(graph, nullptr, &n) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    std::vector<cudaGraphNode_t> nodes(n);
    if (n > 0 && cudaGraphGetNodes(graph, nodes.data(), &n) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int k = 0;
    for (size_t j = 0; j < n; ++j) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[j], &t) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (t == cudaGraphNodeTypeKernel) ++k;
    }
    return k;
}

// programmatic (PDL) edges of a captured graph; -1 if they cannot be read
static int programmatic_edges(cudaGraph_t graph) {
    size_t n = 0;
    if (cudaGraphGetEdges_v2(graph, nullptr, nullptr, nullptr, &n) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    std::vector<cudaGraphNode_t> from(n), to(n);
    std::vector<cudaGraphEdgeData> data(n);
    if (n > 0 && cudaGraphGetEdges_v2(graph, from.data(), to.data(), data.data(), &n) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    int k = 0;
    for (size_t j = 0; j < n; ++j) k += data[j].type == cudaGraphDependencyTypeProgrammatic ? 1 : 0;
    return k;
}

// Jacobi residual of the current iterate into the gate's accumulator
static void enqueue_gate_residual(SolverImpl& s, const VbdContacts* c, float dt, cudaStream_t st) {
    const VbdModelImpl& m = *s.m;
    SweepArgs a = make_sweep_args(s, c, dt);
    a.v_begin = 0;
    a.v_end = m.swept;
    a.resid_out = nullptr;
    a.gate_max = s.gate_mean ? nullptr : s.gate->maxv;
    a.gate_sum = s.gate_mean ? s.gate->sum : nullptr;
    launch_sweep(a, s.lanes, m.any_tri_damping || m.any_edge_damping, true, s.block, st);
}

// The gated iterations of one step, recorded into the graph that `st` is capturing:
//   residual at the start -> check (sets the condition) -> while (condition) {
//       gate_every iterations of all colors -> residual -> check }
// The loop is a conditional WHILE node; its body is captured on the solver's body stream into
// the node's body graph.  Only valid while `st` is capturing.
static int enqueue_gated_iterations(SolverImpl& s, const VbdContacts* c, float dt, cudaStream_t st, bool set_ref) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    VBD_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps));
    if (cs != cudaStreamCaptureStatusActive || !graph)
        return fail(VBD_ERR_UNSUPPORTED, "residual-gated step: the stream is not capturing");
    // sweep residuals need the lane-parallel sweep; the record-parallel one is checked by Jacobi
    const bool sweep = s.gate_sweep && s.lanes > 0;
    cudaGraphConditionalHandle handle;
    // the loop runs at least once in sweep mode (its first check follows the first iteration)
    const unsigned enter = (sweep && s.gate_max > 0) ? 1u : 0u;
    VBD_CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, graph, enter, cudaGraphCondAssignDefault));
    if (!sweep || s.gate_max == 0) {
        // the Jacobi residual at the start iterate (in sweep mode only when no iteration may run,
        // so that the step is still recorded)
        enqueue_gate_residual(s, c, dt, st);
        gate_check_kernel<<<1, 32, 0, st>>>(s.gate, handle, gate_params(s, 1, set_ref ? 1 : 0, 0));
        VBD_CUDA_TRY(cudaGetLastError());
        VBD_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps));
    }
    cudaGraphNodeParams params = {cudaGraphNodeTypeConditional};  // the union has no default constructor
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    VBD_CUDA_TRY(cudaGraphAddNode(&node, graph, deps, ndeps, &params));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    VBD_CUDA_TRY(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    VBD_CUDA_TRY(cudaStreamBeginCaptureToGraph(s.body_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    // sweep mode: the body holds gate_rounds rounds; the last iteration of a round accumulates
    // the sweep residuals and a one-warp check kernel after it decides; once decided, the rest
    // of the body returns at once.  (A decision taken by the round's last sweep itself -- its last
    // block to finish, found by an election over atomic counters -- cost 14 us more per round at
    // 1.89 M vertices: every block of that sweep had to take part.)
    const int rounds = sweep ? s.gate_rounds : 1;
    for (int u = 0; u < rounds; ++u) {
        for (int k = 0; k < s.gate_every; ++k) {
            const bool last = k == s.gate_every - 1;
            for (int color = 0; color < s.m->C; ++color)
                enqueue_color(s, color, c, dt, s.body_stream, false, sweep && last, u > 0);
            if (sweep && last)
                launch_gate(gate_check_kernel, s.body_stream, s.pdl, s.gate, handle,
                            gate_params(s, -1, set_ref ? 1 : 0, s.gate_every));
        }
    }
    if (!sweep) {
        enqueue_gate_residual(s, c, dt, s.body_stream);
        launch_gate(gate_check_kernel, s.body_stream, s.pdl, s.gate, handle, gate_params(s, 0, 0, s.gate_every));
    }
    const cudaError_t e1 = cudaGetLastError();
    cudaGraph_t captured = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s.body_stream, &captured);
    if (e1 != cudaSuccess) return cuda_fail(e1, "residual-gated loop body");
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture (residual-gated loop body)");
    s.gate_body_kernels = kernel_nodes(body);
    s.gate_body_pdl_edges = programmatic_edges(body);
    return VBD_OK;
}

static int enqueue_step(SolverImpl& s, float* q_in, const float* qd_in, const float* f_ext, float* q_out,
                        float* qd_out, const VbdContacts* c, float dt, int iterations, cudaStream_t st) {
    enqueue_forward(s, q_in, qd_in, f_ext, c, dt, st);
    if (s.ws_params) {
        // learned warm start: features -> MLP -> iterate from y + prediction
        const bool gated = s.gate_tol > 0.f;
        if (gated) {
            VBD_CUDA_TRY(cudaMemsetAsync(s.gate, 0, offsetof(GateState, pad), st));
            if (s.gate_relative) {
                // the relative tolerance refers to the plain start y, before the warm start moves it
                enqueue_gate_residual(s, c, dt, st);
                launch_gate(gate_ref_kernel, st, s.pdl, s.gate, s.gate_mean, s.gate_count);
            }
        }
        // features, inference and the bounded start in one tcgen05 launch over the internal rows
        const int rc = mlp_step_start(*s.m, s.ws_params, s.prev, s.y, c ? s.ccount : nullptr, s.ws_corr, s.ws_mean,
                                      s.ws_inv_std, s.feature_set, dt, s.disp, s.pos, st);
        if (rc) return rc;
        if (gated) {
            const int rg = enqueue_gated_iterations(s, c, dt, st, false);
            if (rg) return rg;
        } else {
            for (int it = 0; it < s.ws_iterations; ++it)
                for (int color = 0; color < s.m->C; ++color) enqueue_color(s, color, c, dt, st, it == 0);
        }
        enqueue_finalize(s, q_in, q_out, qd_out, dt, st, s.ws_corr);  // and the correction kept
        return VBD_OK;
    }
    if (s.resident_on && s.resident.ready && iterations > 0 && !(s.gate_tol > 0.f)) {
        const VbdModelImpl& m = *s.m;
        ResidentLaunch L;
        std::memset(&L, 0, sizeof(L));
        L.pos = s.pos;
        L.prev = s.prev;
        L.y = s.y;
        L.disp = s.disp;
        if (c && m.S > 0) {
            L.ccount = s.ccount;
            L.cslot = s.cslot;
            L.c_shape = c->soft_contact_shape;
            L.c_body_pos = c->soft_contact_body_pos;
            L.c_body_vel = c->soft_contact_body_vel;
            L.c_normal = c->soft_contact_normal;
        }
        L.K = s.K;
        L.status = s.status;
        L.q_in = q_in;
        L.q_out = q_out;
        L.qd_out = qd_out;
        L.ccount_clear = s.ccount;
        L.dt = dt;
        L.friction_epsilon = s.friction_epsilon;
        L.iterations = iterations;
        L.spin_limit = s.spin_limit;
        return resident_enqueue(m, s.resident, L, st);
    }
    if (s.sc.on) {
        int rc = self_contact_start(s, st);
        for (int it = 0; it < iterations && !rc; ++it) {
            if (self_contact_detect_now(s.sc, it)) rc = self_contact_detect(*s.m, s.sc, s.pos, s.disp, true, st);
            for (int color = 0; color < s.m->C; ++color) enqueue_color(s, color, c, dt, st, it == 0);
        }
        if (rc) return rc;
        enqueue_finalize(s, q_in, q_out, qd_out, dt, st);
        return VBD_OK;
    }
    if (s.gate_tol > 0.f) {
        VBD_CUDA_TRY(cudaMemsetAsync(s.gate, 0, offsetof(GateState, pad), st));
        // relative mode: the reference is the Jacobi residual at the plain start y -- the Jacobi
        // check at the start iterate when the gate evaluates one anyway, else one evaluation here
        const bool sweep = s.gate_sweep && s.lanes > 0;
        if (s.gate_relative && sweep) {
            enqueue_gate_residual(s, c, dt, st);
            launch_gate(gate_ref_kernel, st, s.pdl, s.gate, s.gate_mean, s.gate_count);
        }
        const int rc = enqueue_gated_iterations(s, c, dt, st, !sweep);
        if (rc) return rc;
        enqueue_finalize(s, q_in, q_out, qd_out, dt, st);
        return VBD_OK;
    }
    for (int it = 0; it < iterations; ++it)
        for (int color = 0; color < s.m->C; ++color) enqueue_color(s, color, c, dt, st, it == 0);
    enqueue_finalize(s, q_in, q_out, qd_out, dt, st);
    return VBD_OK;
}

static void free_solver(SolverImpl& s) {
    resident_free(s.resident);
    self_contact_free(s.sc);
    cudaFree(s.patch_off);
    cudaFree(s.patch_ids);
    cudaFree(s.tri_loc);
    cudaFree(s.edge_loc);
    s.patch_off = s.patch_ids = nullptr;
    s.tri_loc = s.edge_loc = nullptr;
    if (s.ws_corr) cudaFree(s.ws_corr);
    s.ws_corr = nullptr;
    for (auto& g : s.graphs) cudaGraphExecDestroy(g.exec);
    s.graphs.clear();
    void* ptrs[] = {s.pos, s.prev, s.y, s.disp, s.ccount, s.cslot, s.ctab, s.status, s.resid_max};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s.capture_stream) cudaStreamDestroy(s.capture_stream);
    if (s.body_stream) cudaStreamDestroy(s.body_stream);
    if (s.gate) cudaFree(s.gate);
    s.gate = nullptr;
    s.body_stream = nullptr;
    s.pos = s.prev = s.y = s.disp = nullptr;
    s.ccount = s.cslot = nullptr;
    s.ctab = nullptr;
    s.status = nullptr;
    s.resid_max = nullptr;
    s.capture_stream = nullptr;
}

// nullptr when (lanes, block) is a supported sweep launch shape, else the reason
static const char* launch_shape_error(int lanes, int block) {
    if (lanes == 0) {
        if (block != 64 && block != 128 && block != 256)
            return "block_size must be 64, 128 or 256 for the record-parallel sweep (lanes_per_vertex 0)";
        return nullptr;
    }
    if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16)
        return "lanes_per_vertex must be 0 (record-parallel), 1, 2, 4, 8 or 16";
    if (block < 32 || block > 256 || (block % 32) != 0) return "block_size must be a multiple of 32 in [32, 256]";
    return nullptr;
}

static bool same_contacts(const VbdContacts& a, const VbdContacts& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

static int check_state_args(const char* fn, const float* a, const float* b) {
    if (!a || !b) return fail(VBD_ERR_INVALID_ARGUMENT, std::string(fn) + ": required state array is NULL");
    return VBD_OK;
}

}  // namespace vbd

using namespace vbd;

extern "C" int vbd_solver_create(const VbdModel* model, const VbdSolverOptions* options, VbdSolver** out) {
    if (!out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_solver_create: out is NULL");
    *out = nullptr;
    if (!model) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_solver_create: model is NULL");
    const VbdModelImpl& m = model->m;
    VbdSolver* h = new VbdSolver();
    SolverImpl& s = h->s;
    s.m = &m;
    if (options) {
        if (options->iterations < 0) {
            delete h;
            return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_solver_create: iterations must be >= 0");
        }
        s.iterations = options->iterations;
        s.friction_epsilon = options->friction_epsilon;
        if (options->lanes_per_vertex > 0) s.lanes = options->lanes_per_vertex;
        if (options->lanes_per_vertex < 0) s.lanes = 0;
        if (options->block_size) s.block = options->block_size;
        if (options->contacts_per_vertex) s.K = options->contacts_per_vertex;
        s.use_graph = options->use_graph != 0;
        s.resident_on = options->step_kernel == 1;
        if (options->self_contact && s.resident_on) {
            delete h;
            return fail(VBD_ERR_UNSUPPORTED, "vbd_solver_create: the resident step kernel has no self-contact");
        }
    }
    if (const char* why = launch_shape_error(s.lanes, s.block)) {
        delete h;
        return fail(VBD_ERR_INVALID_ARGUMENT, std::string("vbd_solver_create: ") + why);
    }
    if (s.K < 1 || s.K > 8) {
        delete h;
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_solver_create: contacts_per_vertex must be in [1, 8]");
    }
    auto alloc = [&](void** p, size_t bytes) -> int {
        if (bytes == 0) bytes = 16;
        VBD_CUDA_TRY(cudaMalloc(p, bytes));
        VBD_CUDA_TRY(cudaMemset(*p, 0, bytes));
        return VBD_OK;
    };
    const size_t V = static_cast<size_t>(m.V);
    int rc = VBD_OK;
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.pos), V * sizeof(float4));
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.prev), V * sizeof(float4));
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.y), V * sizeof(float4));
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.disp), V * sizeof(float4));
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.ccount), V * sizeof(int));
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.cslot), V * s.K * sizeof(int));
    if (!rc && m.S > 0) rc = alloc(reinterpret_cast<void**>(&s.ctab), V * s.K * 4 * sizeof(float4));
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.status), kStatusSlots * sizeof(unsigned));
    if (!rc) rc = alloc(reinterpret_cast<void**>(&s.resid_max), sizeof(float));
    if (!rc) {
        cudaError_t e = cudaStreamCreateWithFlags(&s.capture_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamCreateWithFlags");
    }
    if (!rc) prime_occupancy(s.lanes, s.block);
    if (!rc && s.resident_on) rc = resident_build(m, s.resident);
    if (!rc && options && options->self_contact && m.V > 0) {
        SelfContactParams p;
        p.radius = options->self_contact_radius;
        p.margin = options->self_contact_margin;
        p.relaxation = options->conservative_bound_relaxation;
        p.edge_parallel_epsilon = options->edge_parallel_epsilon;
        p.rest_exclusion_radius = options->rest_exclusion_radius;
        p.vertex_buffer = options->vertex_contact_buffer_size;
        p.edge_buffer = options->edge_contact_buffer_size;
        p.interval = options->collision_detection_interval;
        p.filter_threshold = options->topological_filter_threshold;
        if (options->vertex_filter_offsets) {
            p.vertex_filter_off.assign(options->vertex_filter_offsets, options->vertex_filter_offsets + m.V + 1);
            if (options->vertex_filter_triangles)
                p.vertex_filter.assign(options->vertex_filter_triangles,
                                       options->vertex_filter_triangles + p.vertex_filter_off[m.V]);
        }
        if (options->edge_filter_offsets) {
            p.edge_filter_off.assign(options->edge_filter_offsets, options->edge_filter_offsets + m.E + 1);
            if (options->edge_filter_edges)
                p.edge_filter.assign(options->edge_filter_edges, options->edge_filter_edges + p.edge_filter_off[m.E]);
        }
        rc = self_contact_create(m, p, s.sc);
    }
    if (rc) {
        free_solver(s);
        delete h;
        return rc;
    }
    *out = h;
    return VBD_OK;
}

extern "C" int vbd_solver_destroy(VbdSolver* solver) {
    if (!solver) return VBD_OK;
    free_solver(solver->s);
    delete solver;
    return VBD_OK;
}

extern "C" int vbd_step(VbdSolver* solver, float* q_in, const float* qd_in, const float* f_ext, float* q_out,
                        float* qd_out, const VbdContacts* contacts, float dt, int32_t iterations, void* stream) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step: solver is NULL");
    SolverImpl& s = solver->s;
    if (s.m->V == 0) return VBD_OK;
    int rc = check_state_args("vbd_step", q_in, qd_in);
    if (rc) return rc;
    if (!q_out || !qd_out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step: state_out arrays are NULL");
    if (!(dt > 0.0f)) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step: dt must be > 0");
    const int iters = iterations < 0 ? s.iterations : iterations;
    if (contacts && !contacts->soft_contact_count) contacts = nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    s.steps++;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    VBD_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
    const bool gated = s.gate_tol > 0.f;
    if ((!s.use_graph && !gated) || cs != cudaStreamCaptureStatusNone) {
        // plain launches (also the path taken inside a caller's own stream capture, where a
        // residual-gated step adds its conditional loop to the caller's graph); a gated step
        // outside a capture always runs from a graph, since its loop is a conditional graph node
        s.last_step_kernels = -1;
        rc = enqueue_step(s, q_in, qd_in, f_ext, q_out, qd_out, contacts, dt, iters, st);
        if (rc) return rc;
        VBD_CUDA_TRY(cudaGetLastError());
        return VBD_OK;
    }
    VbdContacts ckey;
    std::memset(&ckey, 0, sizeof(ckey));
    if (contacts) ckey = *contacts;
    for (auto& g : s.graphs) {
        if (g.q_in == q_in && g.qd_in == qd_in && g.f_ext == f_ext && g.q_out == q_out && g.qd_out == qd_out &&
            g.has_contacts == (contacts != nullptr) && same_contacts(g.contacts, ckey) && g.dt == dt &&
            g.iterations == iters && g.lanes == s.lanes && g.block == s.block) {
            s.last_step_kernels = g.kernels;
            VBD_CUDA_TRY(cudaGraphLaunch(g.exec, st));
            return VBD_OK;
        }
    }
    // capture the step on the private stream, instantiate, replay on the caller's stream; if the
    // resident kernel cannot be captured on this driver, fall back to per-color launches; if a
    // gated loop body with programmatic dependent launches does not instantiate, fall back to
    // plain launches inside the loop
    cudaGraphExec_t exec = nullptr;
    int kernels = -1;
    for (int attempt = 0; attempt < 2 && !exec; ++attempt) {
        VBD_CUDA_TRY(cudaStreamBeginCapture(s.capture_stream, cudaStreamCaptureModeThreadLocal));
        const int erc = enqueue_step(s, q_in, qd_in, f_ext, q_out, qd_out, contacts, dt, iters, s.capture_stream);
        cudaGraph_t graph = nullptr;
        cudaError_t e1 = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(s.capture_stream, &graph);
        cudaError_t e3 = cudaErrorUnknown;
        if (erc == VBD_OK && e1 == cudaSuccess && e2 == cudaSuccess && graph) e3 = cudaGraphInstantiate(&exec, graph, 0);
        if (e3 == cudaSuccess) kernels = kernel_nodes(graph);
        if (graph) cudaGraphDestroy(graph);
        if (e3 == cudaSuccess) break;
        exec = nullptr;
        cudaGetLastError();
        if (gated && s.pdl && !erc) {
            s.pdl = false;  // retry the gated step without programmatic dependent launch
            continue;
        }
        if (!s.resident.ready || !s.resident_on) {
            if (erc) return erc;
            return cuda_fail(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3), "vbd_step graph capture");
        }
        s.resident_on = false;  // retry with one launch per color
    }
    if (!exec) return fail(VBD_ERR_CUDA, "vbd_step: the step graph could not be instantiated");
    if (s.graphs.size() >= 8) {
        cudaGraphExecDestroy(s.graphs.front().exec);
        s.graphs.erase(s.graphs.begin());
    }
    GraphEntry g;
    g.q_in = q_in;
    g.qd_in = qd_in;
    g.f_ext = f_ext;
    g.q_out = q_out;
    g.qd_out = qd_out;
    g.contacts = ckey;
    g.has_contacts = contacts != nullptr;
    g.dt = dt;
    g.iterations = iters;
    g.lanes = s.lanes;
    g.block = s.block;
    g.kernels = kernels;
    g.exec = exec;
    s.graphs.push_back(g);
    s.last_step_kernels = kernels;
    VBD_CUDA_TRY(cudaGraphLaunch(exec, st));
    return VBD_OK;
}

extern "C" int vbd_batch_step(VbdSolver* const* solvers, int32_t count, float* const* q_in, const float* const* qd_in,
                              const float* const* f_ext, float* const* q_out, float* const* qd_out,
                              const VbdContacts* const* contacts, float dt, const int32_t* iterations,
                              void* stream) {
    if (count < 0) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_batch_step: count must be >= 0");
    if (count == 0) return VBD_OK;
    if (!solvers || !q_in || !qd_in || !q_out || !qd_out)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_batch_step: solvers and state array lists must not be NULL");
    for (int b = 0; b < count; ++b) {
        const int rc = vbd_step(solvers[b], q_in[b], qd_in[b], f_ext ? f_ext[b] : nullptr, q_out[b], qd_out[b],
                                contacts ? contacts[b] : nullptr, dt, iterations ? iterations[b] : -1, stream);
        if (rc) return fail(rc, "vbd_batch_step: solver " + std::to_string(b) + ": " + vbd_last_error());
    }
    return VBD_OK;
}

extern "C" int vbd_forward(VbdSolver* solver, const float* q_in, const float* qd_in, const float* f_ext,
                           const VbdContacts* contacts, float dt, void* stream) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_forward: solver is NULL");
    SolverImpl& s = solver->s;
    if (s.m->V == 0) return VBD_OK;
    int rc = check_state_args("vbd_forward", q_in, qd_in);
    if (rc) return rc;
    if (!(dt > 0.0f)) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_forward: dt must be > 0");
    if (contacts && !contacts->soft_contact_count) contacts = nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // a staged sequence starts from an empty contact table
    VBD_CUDA_TRY(cudaMemsetAsync(s.ccount, 0, sizeof(int) * static_cast<size_t>(s.m->V), st));
    s.staged_iteration = 0;
    enqueue_forward(s, q_in, qd_in, f_ext, contacts, dt, st);
    VBD_CUDA_TRY(cudaGetLastError());
    if (s.sc.on) return self_contact_start(s, st);
    return VBD_OK;
}

extern "C" int vbd_begin_iteration(VbdSolver* solver, int32_t iteration, void* stream) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_begin_iteration: solver is NULL");
    SolverImpl& s = solver->s;
    if (iteration < 0) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_begin_iteration: iteration must be >= 0");
    s.staged_iteration = iteration;
    if (s.m->V == 0 || !self_contact_detect_now(s.sc, iteration)) return VBD_OK;
    return self_contact_detect(*s.m, s.sc, s.pos, s.disp, true, static_cast<cudaStream_t>(stream));
}

extern "C" int vbd_self_contact_detect(VbdSolver* solver, const float* particle_q, void* stream) {
    if (!solver || !particle_q) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_self_contact_detect: NULL argument");
    SolverImpl& s = solver->s;
    if (!s.sc.on) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_self_contact_detect: self-contact is not enabled");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = self_contact_load_positions(*s.m, s.sc, particle_q, st);
    if (!rc) rc = self_contact_detect(*s.m, s.sc, s.sc.cd, nullptr, false, st);
    return rc;
}

extern "C" int vbd_self_contact_lists(VbdSolver* solver, int32_t* vt_counts, int32_t* vt_lists, int32_t* ee_counts,
                                      int32_t* ee_lists) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_self_contact_lists: solver is NULL");
    SolverImpl& s = solver->s;
    if (!s.sc.on) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_self_contact_lists: self-contact is not enabled");
    const VbdModelImpl& m = *s.m;
    const int V = m.V, E = m.E, vb = s.sc.p.vertex_buffer, eb = s.sc.p.edge_buffer;
    VBD_CUDA_TRY(cudaDeviceSynchronize());
    std::vector<int> vc(V), vl(static_cast<size_t>(V) * vb), ec(E), el(static_cast<size_t>(E) * eb);
    if (V) VBD_CUDA_TRY(cudaMemcpy(vc.data(), s.sc.vt_count, vc.size() * sizeof(int), cudaMemcpyDeviceToHost));
    if (V) VBD_CUDA_TRY(cudaMemcpy(vl.data(), s.sc.vt_list, vl.size() * sizeof(int), cudaMemcpyDeviceToHost));
    if (E) VBD_CUDA_TRY(cudaMemcpy(ec.data(), s.sc.ee_count, ec.size() * sizeof(int), cudaMemcpyDeviceToHost));
    if (E) VBD_CUDA_TRY(cudaMemcpy(el.data(), s.sc.ee_list, el.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < V; ++i) {
        const int o = m.perm_host[i];
        if (vt_counts) vt_counts[o] = vc[i];
        if (vt_lists)
            for (int k = 0; k < vb; ++k) vt_lists[static_cast<size_t>(o) * vb + k] = k < vc[i] ? vl[static_cast<size_t>(i) * vb + k] : -1;
    }
    for (int e = 0; e < E; ++e) {
        if (ee_counts) ee_counts[e] = ec[e];
        if (ee_lists)
            for (int k = 0; k < eb; ++k) ee_lists[static_cast<size_t>(e) * eb + k] = k < ec[e] ? el[static_cast<size_t>(e) * eb + k] : -1;
    }
    return VBD_OK;
}

extern "C" int vbd_sweep_color(VbdSolver* solver, int32_t color, const VbdContacts* contacts, float dt,
                               void* stream) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_sweep_color: solver is NULL");
    SolverImpl& s = solver->s;
    if (color < 0 || color >= s.m->C) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_sweep_color: color out of range");
    if (!(dt > 0.0f)) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_sweep_color: dt must be > 0");
    if (contacts && !contacts->soft_contact_count) contacts = nullptr;
    enqueue_color(s, color, contacts, dt, static_cast<cudaStream_t>(stream), s.staged_iteration == 0);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_finalize(VbdSolver* solver, float* q_in, float* q_out, float* qd_out, float dt, void* stream) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_finalize: solver is NULL");
    if (!(dt > 0.0f)) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_finalize: dt must be > 0");
    enqueue_finalize(solver->s, q_in, q_out, qd_out, dt, static_cast<cudaStream_t>(stream));
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_warm_start(VbdSolver* solver, const float* delta, void* stream) {
    if (!solver || !delta) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_warm_start: NULL argument");
    SolverImpl& s = solver->s;
    if (s.m->V == 0) return VBD_OK;
    warm_start_kernel<<<(s.m->V + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        s.m->perm, s.m->pinfo, s.prev, s.disp, s.pos, delta, s.m->V);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_mlp_features(VbdSolver* solver, const float* corr_prev, const float* mean, const float* inv_std,
                                float* out, void* stream) {
    if (!solver || !out || ((mean == nullptr) != (inv_std == nullptr)))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_features: bad arguments");
    SolverImpl& s = solver->s;
    return mlp_features_launch(*s.m, s.prev, s.y, s.ccount, corr_prev, mean, inv_std, out, s.feature_set, s.last_dt,
                               static_cast<cudaStream_t>(stream));
}

extern "C" int vbd_set_feature_set(VbdSolver* solver, int32_t feature_set) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_feature_set: solver is NULL");
    if (feature_set != VBD_FEATURES_CORRECTIONS && feature_set != VBD_FEATURES_KINEMATIC)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_feature_set: unknown feature set");
    SolverImpl& s = solver->s;
    if (s.feature_set != feature_set) {
        for (auto& g : s.graphs) cudaGraphExecDestroy(g.exec);  // captured steps change
        s.graphs.clear();
    }
    s.feature_set = feature_set;
    return VBD_OK;
}

extern "C" int vbd_set_warm_start(VbdSolver* solver, const float* params, const uint16_t* w16, const float* mean,
                                  const float* inv_std, int32_t iterations) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_warm_start: solver is NULL");
    SolverImpl& s = solver->s;
    for (auto& g : s.graphs) cudaGraphExecDestroy(g.exec);  // captured steps change
    s.graphs.clear();
    if (!params) {
        s.ws_params = nullptr;
        s.ws_w16 = nullptr;
        return VBD_OK;
    }
    if (!w16 || iterations < 0 || ((mean == nullptr) != (inv_std == nullptr)))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_warm_start: bad arguments");
    if (s.sc.on) return fail(VBD_ERR_UNSUPPORTED, "vbd_set_warm_start: not available with self-contact");
    const size_t V = static_cast<size_t>(s.m->V);
    if (!s.ws_corr) {
        VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&s.ws_corr), std::max<size_t>(V, 1) * 3 * sizeof(float)));
    }
    VBD_CUDA_TRY(cudaMemset(s.ws_corr, 0, std::max<size_t>(V, 1) * 3 * sizeof(float)));
    // make the MLP kernel's shared-memory opt-in outside any later stream capture
    int rc = vbd_mlp_forward(params, w16, nullptr, 0, nullptr, nullptr);
    if (rc) return rc;
    s.ws_params = params;
    s.ws_w16 = w16;
    s.ws_mean = mean;
    s.ws_inv_std = inv_std;
    s.ws_iterations = iterations;
    return VBD_OK;
}

extern "C" int vbd_set_warm_start_correction(VbdSolver* solver, const float* corr, void* stream) {
    if (!solver || !corr) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_warm_start_correction: NULL argument");
    SolverImpl& s = solver->s;
    if (!s.ws_corr) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_warm_start_correction: the warm start is off");
    const int V = s.m->V;
    if (V == 0) return VBD_OK;
    // the step mode keeps it in the internal vertex order
    gather_rows3_kernel<<<(V + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(s.m->perm, corr, s.ws_corr, V);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_mlp_warm_start(VbdSolver* solver, const float* params, const uint16_t* w16, const float* corr_prev,
                                  const float* mean, const float* inv_std, float* workspace, int64_t workspace_floats,
                                  void* stream) {
    if (!solver || !params || !w16 || !workspace || ((mean == nullptr) != (inv_std == nullptr)))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_warm_start: bad arguments");
    SolverImpl& s = solver->s;
    const int V = s.m->V;
    if (workspace_floats < static_cast<int64_t>(V) * (64 + 3 + 3))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_mlp_warm_start: workspace must hold V*70 floats");
    if (V == 0) return VBD_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float* feats = workspace;
    float* pred = feats + static_cast<size_t>(V) * 64;
    float* delta = pred + static_cast<size_t>(V) * 3;
    int rc = mlp_features_launch(*s.m, s.prev, s.y, s.ccount, corr_prev, mean, inv_std, feats, s.feature_set,
                                 s.last_dt, st);
    if (rc) return rc;
    rc = vbd_mlp_forward(params, w16, feats, V, pred, stream);
    if (rc) return rc;
    rc = mlp_scale_launch(*s.m, pred, delta, st);
    if (rc) return rc;
    return vbd_warm_start(solver, delta, stream);
}

extern "C" int vbd_get_positions(const VbdSolver* solver, float* q_out, void* stream) {
    if (!solver || !q_out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_get_positions: NULL argument");
    const SolverImpl& s = solver->s;
    if (s.m->V == 0) return VBD_OK;
    gather_positions_kernel<<<(s.m->V + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(s.m->perm, s.pos,
                                                                                                   q_out, s.m->V);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_residual(VbdSolver* solver, const VbdContacts* contacts, float dt, float* per_vertex_out,
                            float* max_out, void* stream) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_residual: solver is NULL");
    if (!(dt > 0.0f)) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_residual: dt must be > 0");
    SolverImpl& s = solver->s;
    const VbdModelImpl& m = *s.m;
    if (contacts && !contacts->soft_contact_count) contacts = nullptr;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float* mx = max_out ? max_out : s.resid_max;
    VBD_CUDA_TRY(cudaMemsetAsync(mx, 0, sizeof(float), st));
    if (per_vertex_out && m.V > m.swept) VBD_CUDA_TRY(cudaMemsetAsync(per_vertex_out, 0, sizeof(float) * m.V, st));
    if (s.sc.on) {
        const int rc = self_contact_accumulate(m, s.sc, s.pos, s.prev, -1, dt, s.friction_epsilon, st);
        if (rc) return rc;
    }
    SweepArgs a = make_sweep_args(s, contacts, dt);
    a.v_begin = 0;
    a.v_end = m.swept;
    a.resid_out = per_vertex_out;
    a.resid_max = mx;
    launch_sweep(a, s.lanes, m.any_tri_damping || m.any_edge_damping, true, s.block, st);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_set_residual_gate(VbdSolver* solver, float tolerance, int32_t max_iterations, int32_t check_every,
                                     int32_t mode) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_residual_gate: solver is NULL");
    SolverImpl& s = solver->s;
    if (!(tolerance > 0.f)) {
        s.gate_tol = 0.f;  // off: back to the fixed iteration count
    } else {
        // the cap bounds the device-side loop: every step ends after at most max_iterations
        if (max_iterations < 0 || max_iterations > kGateMaxIterations || check_every < 1 || check_every > 64)
            return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_residual_gate: max_iterations must be in [0, " +
                                                      std::to_string(kGateMaxIterations) +
                                                      "] and check_every in [1, 64]");
        if (s.sc.on) return fail(VBD_ERR_UNSUPPORTED, "vbd_set_residual_gate: not available with self-contact");
        if (!(s.m->gravity_norm > 0.f))
            return fail(VBD_ERR_UNSUPPORTED, "vbd_set_residual_gate: the residual is in units of m|g|; gravity is zero");
        if (!s.gate) {
            VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&s.gate), sizeof(GateState)));
            VBD_CUDA_TRY(cudaMemset(s.gate, 0, sizeof(GateState)));
        }
        if (!s.body_stream) VBD_CUDA_TRY(cudaStreamCreateWithFlags(&s.body_stream, cudaStreamNonBlocking));
        s.gate_tol = tolerance;
        s.gate_max = max_iterations;
        s.gate_every = check_every;
        if (mode & ~(VBD_GATE_RELATIVE | VBD_GATE_MEAN | VBD_GATE_SWEEP | VBD_GATE_ROUNDS_MASK))
            return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_residual_gate: unknown mode bits");
        const int rounds = (mode & VBD_GATE_ROUNDS_MASK) >> VBD_GATE_ROUNDS_SHIFT;
        s.gate_rounds = rounds > 0 ? rounds : kGateDefaultRounds;
        s.gate_relative = (mode & VBD_GATE_RELATIVE) ? 1 : 0;
        s.gate_mean = (mode & VBD_GATE_MEAN) ? 1 : 0;
        s.gate_sweep = (mode & VBD_GATE_SWEEP) ? 1 : 0;
        // every vertex a color solves is counted once per evaluation
        int count = 0;
        for (int i = 0; i < s.m->swept; ++i) {
            const float4 pi = s.m->pinfo_h[i];
            int flags = 0;
            std::memcpy(&flags, &pi.w, sizeof(flags));
            if ((flags & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f) ++count;
        }
        s.gate_count = count;
    }
    for (auto& g : s.graphs) cudaGraphExecDestroy(g.exec);  // captured steps change
    s.graphs.clear();
    return VBD_OK;
}

extern "C" int vbd_gate_stats(VbdSolver* solver, VbdGateStats* out, int32_t reset) {
    if (!solver || !out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_gate_stats: NULL argument");
    SolverImpl& s = solver->s;
    std::memset(out, 0, sizeof(*out));
    out->body_kernels = s.gate_body_kernels;
    out->body_programmatic_edges = s.pdl ? s.gate_body_pdl_edges : 0;
    if (!s.gate) return VBD_OK;
    GateState g;
    VBD_CUDA_TRY(cudaDeviceSynchronize());
    VBD_CUDA_TRY(cudaMemcpy(&g, s.gate, sizeof(g), cudaMemcpyDeviceToHost));
    out->steps = static_cast<int64_t>(g.steps);
    out->iterations = static_cast<int64_t>(g.iter_sum);
    out->capped_steps = static_cast<int64_t>(g.capped);
    out->last_iterations = g.last_iters;
    out->last_residual = g.last_resid;
    out->last_start_residual = g.start_resid;
    out->last_reference_residual = g.ref;
    out->body_passes = static_cast<int64_t>(g.passes);
    if (reset) {
        g.steps = g.iter_sum = g.capped = g.passes = 0ull;
        VBD_CUDA_TRY(cudaMemcpy(s.gate, &g, sizeof(g), cudaMemcpyHostToDevice));
    }
    return VBD_OK;
}

extern "C" int vbd_status(VbdSolver* solver, VbdStatus* out, int32_t reset) {
    if (!solver || !out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_status: NULL argument");
    SolverImpl& s = solver->s;
    unsigned h[kStatusSlots];
    VBD_CUDA_TRY(cudaDeviceSynchronize());
    VBD_CUDA_TRY(cudaMemcpy(h, s.status, sizeof(h), cudaMemcpyDeviceToHost));
    out->steps = s.steps;
    out->nonfinite_updates = static_cast<int32_t>(h[kNonfinite]);
    out->singular_blocks = static_cast<int32_t>(h[kSingular]);
    out->contact_overflow = static_cast<int32_t>(h[kOverflow]);
    out->timeouts = static_cast<int32_t>(h[kTimeout]);
    out->self_contact_overflow = 0;
    out->reserved = 0;
    if (s.sc.on) {
        unsigned c[kScCounters];
        VBD_CUDA_TRY(cudaMemcpy(c, s.sc.counters, sizeof(c), cudaMemcpyDeviceToHost));
        for (unsigned v : c) out->self_contact_overflow += static_cast<int32_t>(v);
    }
    if (reset) {
        VBD_CUDA_TRY(cudaMemset(s.status, 0, sizeof(h)));
        if (s.sc.on) VBD_CUDA_TRY(cudaMemset(s.sc.counters, 0, kScCounters * sizeof(unsigned)));
        s.steps = 0;
    }
    return VBD_OK;
}

extern "C" int vbd_solver_info(const VbdSolver* solver, int32_t* color_count, int32_t* lanes_per_vertex,
                               int32_t* block_size) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_solver_info: solver is NULL");
    if (color_count) *color_count = solver->s.m->C;
    if (lanes_per_vertex) *lanes_per_vertex = solver->s.lanes;
    if (block_size) *block_size = solver->s.block;
    return VBD_OK;
}

// ---- staged sweep ---------------------------------------------------------------------------
constexpr int kMaxPatch = 1536;  // patch entries: local indices fit 14 bits; 2 x 16 B x 1536 = 48 KB

static void free_staged(SolverImpl& s) {
    cudaFree(s.patch_off);
    cudaFree(s.patch_ids);
    cudaFree(s.tri_loc);
    cudaFree(s.edge_loc);
    s.patch_off = s.patch_ids = nullptr;
    s.tri_loc = s.edge_loc = nullptr;
    s.stage_ready = false;
    s.stage_max_patch = 0;
    s.stage_color_base.clear();
}

// Patches of the staged sweep for the solver's launch shape: color c's block b (the vertices
// [color_start[c] + b V_B, + V_B), V_B = block / lanes, as the sweep's grid maps them) gets the
// sorted ids of every position its vertices' records read; each record's ids become indices into
// its vertex's patch.  Built on the host's cores.  Leaves stage_ready false (unstaged sweeps) for
// the record-parallel shape or when a patch would exceed kMaxPatch entries.
static int build_staged(SolverImpl& s) {
    free_staged(s);
    const VbdModelImpl& m = *s.m;
    if (s.lanes < 1 || m.C == 0) return VBD_OK;
    const int VB = s.block / s.lanes;
    std::vector<int> base(static_cast<size_t>(m.C) + 1, 0);
    for (int c = 0; c < m.C; ++c) base[c + 1] = base[c] + (m.color_start[c + 1] - m.color_start[c] + VB - 1) / VB;
    const int P = base[m.C];
    std::vector<std::vector<int>> ids(P);
    std::vector<uint2> tri_loc(std::max(m.n_tri_rec, 1)), edge_loc(std::max(m.n_edge_rec, 1));
    std::atomic<bool> too_big{false};
    parallel_chunks(
        P,
        [&](int pb, int pe) {
            std::vector<int> buf;
            for (int p = pb; p < pe; ++p) {
                const int c = static_cast<int>(std::upper_bound(base.begin(), base.end(), p) - base.begin()) - 1;
                const int v0 = m.color_start[c] + (p - base[c]) * VB;
                const int v1 = std::min(v0 + VB, m.color_start[c + 1]);
                buf.clear();
                for (int i = v0; i < v1; ++i) {
                    const int4 ad = m.vadj_h[i];
                    for (int r = ad.x; r < ad.y; ++r) {
                        const int4 t = m.tri_idx_h[r];
                        buf.insert(buf.end(), {t.x, t.y, t.z});
                    }
                    for (int r = ad.z; r < ad.w; ++r) {
                        const int4 e = m.edge_idx_h[r];
                        buf.insert(buf.end(), {e.x & 0x3fffffff, e.y, e.z, e.w});
                    }
                }
                std::sort(buf.begin(), buf.end());
                buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
                if (static_cast<int>(buf.size()) > kMaxPatch) {
                    too_big = true;
                    continue;
                }
                auto loc = [&buf](int g) {
                    return static_cast<unsigned>(std::lower_bound(buf.begin(), buf.end(), g) - buf.begin());
                };
                for (int i = v0; i < v1; ++i) {
                    const int4 ad = m.vadj_h[i];
                    for (int r = ad.x; r < ad.y; ++r) {
                        const int4 t = m.tri_idx_h[r];
                        tri_loc[r] = make_uint2(loc(t.x) | (loc(t.y) << 16), loc(t.z) | (static_cast<unsigned>(t.w) << 16));
                    }
                    for (int r = ad.z; r < ad.w; ++r) {
                        const int4 e = m.edge_idx_h[r];
                        const unsigned slot = static_cast<unsigned>(e.x) >> 30;
                        edge_loc[r] = make_uint2(loc(e.x & 0x3fffffff) | (slot << 14) | (loc(e.y) << 16),
                                                 loc(e.z) | (loc(e.w) << 16));
                    }
                }
                ids[p] = buf;
            }
        },
        64);
    if (too_big) return VBD_OK;
    std::vector<int> off(static_cast<size_t>(P) + 1, 0);
    int maxp = 0;
    for (int p = 0; p < P; ++p) {
        off[p + 1] = off[p] + static_cast<int>(ids[p].size());
        maxp = std::max(maxp, static_cast<int>(ids[p].size()));
    }
    std::vector<int> flat(std::max(off[P], 1));
    for (int p = 0; p < P; ++p) std::copy(ids[p].begin(), ids[p].end(), flat.begin() + off[p]);
    VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&s.patch_off), off.size() * sizeof(int)));
    VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&s.patch_ids), flat.size() * sizeof(int)));
    VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&s.tri_loc), tri_loc.size() * sizeof(uint2)));
    VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&s.edge_loc), edge_loc.size() * sizeof(uint2)));
    VBD_CUDA_TRY(cudaMemcpy(s.patch_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
    VBD_CUDA_TRY(cudaMemcpy(s.patch_ids, flat.data(), flat.size() * sizeof(int), cudaMemcpyHostToDevice));
    VBD_CUDA_TRY(cudaMemcpy(s.tri_loc, tri_loc.data(), tri_loc.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    VBD_CUDA_TRY(cudaMemcpy(s.edge_loc, edge_loc.data(), edge_loc.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    s.stage_color_base = base;
    s.stage_max_patch = maxp;
    s.stage_lanes = s.lanes;
    s.stage_block = s.block;
    s.stage_ready = true;
    // occupancy of the staged kernels with their shared memory, queried outside any capture
    const bool damp = m.any_tri_damping || m.any_edge_damping;
    const size_t smem = static_cast<size_t>(maxp) * sizeof(float4) * (damp ? 2 : 1);
    switch (s.lanes) {
        case 1: prime_staged_occupancy_L<1>(s.block, smem); break;
        case 2: prime_staged_occupancy_L<2>(s.block, smem); break;
        case 4: prime_staged_occupancy_L<4>(s.block, smem); break;
        case 8: prime_staged_occupancy_L<8>(s.block, smem); break;
        case 16: prime_staged_occupancy_L<16>(s.block, smem); break;
        default: break;
    }
    return VBD_OK;
}

extern "C" int vbd_set_staged_sweep(VbdSolver* solver, int32_t on) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_staged_sweep: solver is NULL");
    SolverImpl& s = solver->s;
    for (auto& g : s.graphs) cudaGraphExecDestroy(g.exec);  // captured steps change
    s.graphs.clear();
    s.stage_on = on != 0;
    if (s.stage_on && !(s.stage_ready && s.stage_lanes == s.lanes && s.stage_block == s.block)) return build_staged(s);
    return VBD_OK;
}

extern "C" int vbd_staged_sweep_info(const VbdSolver* solver, int32_t* active, int32_t* max_patch,
                                     int64_t* patch_entries) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_staged_sweep_info: solver is NULL");
    const SolverImpl& s = solver->s;
    const bool act = s.stage_on && s.stage_ready && !s.sc.on && s.lanes == s.stage_lanes && s.block == s.stage_block;
    if (active) *active = act ? 1 : 0;
    if (max_patch) *max_patch = s.stage_ready ? s.stage_max_patch : 0;
    if (patch_entries) {
        *patch_entries = 0;
        if (s.stage_ready && !s.stage_color_base.empty()) {
            int last = 0;
            cudaMemcpy(&last, s.patch_off + s.stage_color_base.back(), sizeof(int), cudaMemcpyDeviceToHost);
            *patch_entries = last;
        }
    }
    return VBD_OK;
}

extern "C" int vbd_set_launch(VbdSolver* solver, int32_t lanes_per_vertex, int32_t block_size) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_launch: solver is NULL");
    if (const char* why = launch_shape_error(lanes_per_vertex, block_size))
        return fail(VBD_ERR_INVALID_ARGUMENT, std::string("vbd_set_launch: ") + why);
    solver->s.lanes = lanes_per_vertex;
    solver->s.block = block_size;
    prime_occupancy(lanes_per_vertex, block_size);
    if (solver->s.stage_on) return build_staged(solver->s);
    return VBD_OK;
}

extern "C" int vbd_solver_step_kernel(const VbdSolver* solver, int32_t* resident, int32_t* patches,
                                      int32_t* smem_bytes) {
    if (!solver) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_solver_step_kernel: solver is NULL");
    const SolverImpl& s = solver->s;
    const bool on = s.resident_on && s.resident.ready;
    if (resident) *resident = on ? 1 : 0;
    if (patches) *patches = on ? s.resident.patches : 0;
    if (smem_bytes) *smem_bytes = on ? s.resident.smem_bytes : 0;
    return VBD_OK;
}

extern "C" int vbd_step_kernel_count(const VbdSolver* solver, int32_t* kernels) {
    if (!solver || !kernels) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_kernel_count: NULL argument");
    *kernels = solver->s.last_step_kernels;
    return VBD_OK;
}

extern "C" int vbd_set_spin_limit(VbdSolver* solver, uint32_t spins) {
    if (!solver || spins == 0) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_set_spin_limit: NULL solver or zero limit");
    solver->s.spin_limit = spins;
    for (auto& g : solver->s.graphs) cudaGraphExecDestroy(g.exec);  // the limit is baked into captured steps
    solver->s.graphs.clear();
    return VBD_OK;
}

extern "C" const char* vbd_version(void) { return "vbd_b200 0.2 (sm_100a)"; }

// ---------------------------------------------------------------------------------------------
// Allocation-free step: vbd_step_static.
//
// Some callers cannot call cudaMalloc: code that runs while a stream is being captured into a
// CUDA graph (allocation is not a capturable operation), host callbacks and real-time loops
// where an allocation could block or implicitly synchronize the device, and embedders whose
// device memory is owned by a framework allocator that forbids raw cudaMalloc (an ML framework's
// custom-call / FFI handler, for instance).  vbd_solver_create allocates the step's scratch, so
// those callers cannot create a VbdSolver.  vbd_step_static runs the same step without a solver:
// its scratch (Gauss-Seidel iterate, step-start positions, inertia targets, displacements, the
// per-vertex contact slots and the packed contact table) lives in the file-scope device array
// below, sized for at most kStaticMaxParticles particles (~5.3 MiB, held by every GPU that loads
// the library until the process exits).
// ---------------------------------------------------------------------------------------------
namespace vbd {
namespace {

constexpr int kStaticMaxParticles = 16384;
constexpr int kStaticContactsPerVertex = 4;
constexpr size_t kStaticVec4Bytes = static_cast<size_t>(kStaticMaxParticles) * sizeof(float4);
constexpr size_t kStaticCountBytes = static_cast<size_t>(kStaticMaxParticles) * sizeof(int);
constexpr size_t kStaticSlotBytes = static_cast<size_t>(kStaticMaxParticles) * kStaticContactsPerVertex * sizeof(int);
constexpr size_t kStaticTableBytes = static_cast<size_t>(kStaticMaxParticles) * kStaticContactsPerVertex * 4 * sizeof(float4);
constexpr size_t kStaticStatusBytes = 256;
constexpr size_t kStaticScratchBytes =
    4 * kStaticVec4Bytes + kStaticCountBytes + kStaticSlotBytes + kStaticTableBytes + kStaticStatusBytes;
constexpr size_t kStaticTableOffset = 4 * kStaticVec4Bytes + kStaticCountBytes + kStaticSlotBytes;
constexpr size_t kStaticStatusOffset = kStaticTableOffset + kStaticTableBytes;
static_assert(kStaticTableOffset % 16 == 0 && kStaticStatusOffset % 16 == 0, "16-byte aligned sections");

static __device__ __align__(256) unsigned char g_step_scratch[kStaticScratchBytes];

constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mutex;
unsigned char* g_static_scratch_ptr[kStaticMaxDevices] = {};

// Device address of g_step_scratch on the current device (host code cannot use the symbol's
// name as an address).  Looked up once per device, on that device's first call.  `dev_out`
// receives the current device ordinal.
int static_scratch(unsigned char** out, int* dev_out) {
    int dev = 0;
    VBD_CUDA_TRY(cudaGetDevice(&dev));
    *dev_out = dev;
    if (dev < 0 || dev >= kStaticMaxDevices) return fail(VBD_ERR_UNSUPPORTED, "vbd_step_static: device ordinal too large");
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_step_scratch)");
        g_static_scratch_ptr[dev] = static_cast<unsigned char*>(p);
        prime_occupancy(4, 128);  // the launch shape of the static step, queried before any capture
    }
    *out = g_static_scratch_ptr[dev];
    return VBD_OK;
}

}  // namespace
}  // namespace vbd

extern "C" int vbd_step_static(const VbdModel* model, float* q_in, const float* qd_in, const float* f_ext,
                               float* q_out, float* qd_out, const VbdContacts* contacts, float dt, int32_t iterations,
                               float friction_epsilon, void* stream) {
    using namespace vbd;
    if (!model) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_static: model is NULL");
    const VbdModelImpl& m = model->m;
    if (m.V > kStaticMaxParticles)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_static: the model has " + std::to_string(m.V) +
                                                  " particles; the static scratch holds at most " +
                                                  std::to_string(kStaticMaxParticles) + " (use vbd_solver_create + vbd_step)");
    if (m.V == 0) return VBD_OK;
    int rc = check_state_args("vbd_step_static", q_in, qd_in);
    if (rc) return rc;
    if (!q_out || !qd_out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_static: state_out arrays are NULL");
    if (!(dt > 0.0f)) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_static: dt must be > 0");
    if (iterations < 0) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_static: iterations must be >= 0");
    if (contacts && !contacts->soft_contact_count) contacts = nullptr;
    unsigned char* base = nullptr;
    int dev = -1;
    rc = static_scratch(&base, &dev);
    if (rc) return rc;
    if (dev != m.device)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_static: the current device is " + std::to_string(dev) +
                                                  " but the model lives on device " + std::to_string(m.device) +
                                                  "; make the model's device current");
    SolverImpl s;  // host-side view of the static scratch; owns nothing
    s.m = &m;
    s.iterations = iterations;
    s.friction_epsilon = friction_epsilon;
    s.lanes = 4;
    s.block = 128;
    s.K = kStaticContactsPerVertex;
    s.use_graph = false;
    s.pos = reinterpret_cast<float4*>(base);
    s.prev = reinterpret_cast<float4*>(base + kStaticVec4Bytes);
    s.y = reinterpret_cast<float4*>(base + 2 * kStaticVec4Bytes);
    s.disp = reinterpret_cast<float4*>(base + 3 * kStaticVec4Bytes);
    s.ccount = reinterpret_cast<int*>(base + 4 * kStaticVec4Bytes);
    s.cslot = reinterpret_cast<int*>(base + 4 * kStaticVec4Bytes + kStaticCountBytes);
    if (m.S > 0) s.ctab = reinterpret_cast<float4*>(base + kStaticTableOffset);
    s.status = reinterpret_cast<unsigned*>(base + kStaticStatusOffset);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: the contact slot counts and the status
    // counters must start at zero (the packed table is rewritten for every slot that is read)
    VBD_CUDA_TRY(cudaMemsetAsync(s.ccount, 0, sizeof(int) * static_cast<size_t>(m.V), st));
    VBD_CUDA_TRY(cudaMemsetAsync(s.status, 0, kStaticStatusBytes, st));
    rc = enqueue_step(s, q_in, qd_in, f_ext, q_out, qd_out, contacts, dt, iterations, st);
    if (rc) return rc;
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}

extern "C" int vbd_step_static_status(VbdStatus* out) {
    using namespace vbd;
    if (!out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_step_static_status: out is NULL");
    unsigned h[kStatusSlots];
    // a copy from the symbol: no address lookup and no allocation
    VBD_CUDA_TRY(cudaMemcpyFromSymbol(h, g_step_scratch, sizeof(h), kStaticStatusOffset, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->nonfinite_updates = static_cast<int32_t>(h[kNonfinite]);
    out->singular_blocks = static_cast<int32_t>(h[kSingular]);
    out->contact_overflow = static_cast<int32_t>(h[kOverflow]);
    out->timeouts = static_cast<int32_t>(h[kTimeout]);
    return VBD_OK;
}
