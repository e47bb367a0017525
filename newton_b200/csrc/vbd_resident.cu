// vbd_resident.cu -- one persistent, shared-memory-resident kernel for all Gauss-Seidel colors of
// all iterations of a VBD step.
//
// The per-color path (vbd_solver.cu) pays one launch per color and re-gathers every record and
// position from L2 at every color; on a 65k-vertex cloth a color is only ~16k vertices, so each
// launch is a short latency chain.  Here the model is cut once into compact patches, one per CTA
// (all co-resident: cooperative launch).  A CTA keeps its patch in shared memory for the whole
// step: its owned vertices and their halo (every vertex any owned vertex's elements touch), the
// triangles and hinges of its owned vertices (deduplicated, 16-bit local vertex ids), and each
// owned vertex's list of (element, slot) references in the reference's CSR order.  The static
// part is one contiguous image per patch, brought into shared memory by one bulk asynchronous
// copy per CTA (cp.async.bulk, global to shared, this CTA only) at kernel start.
//
// Ordering without a grid barrier.  Step t = iteration * C + color.  A patch starts step t only
// after every neighbour patch (owner of one of its halo vertices; the relation is symmetric) has
// published progress >= t, i.e. finished step t-1.  Then (1) every halo value of a color that
// precedes `color` in this iteration is final -- it was refreshed right after its own step -- and
// (2) no halo value of a later color has been touched yet, since a neighbour cannot start step t+1
// before this patch finishes step t.  The color being solved never appears in the stencil of its
// own vertices (the coloring is conflict-free for every element), so each vertex sees exactly the
// values a global color-by-color sweep would give it: results are bitwise identical to the
// per-color launches with 4 lanes per vertex (same lane split, same reduction order, same math).
//
// Publication: owned vertices' new positions are stored to global memory, the CTA barriers, then
// thread 0 issues a gpu-scope fence and a release store of its progress counter; readers spin on
// an acquire load (bounded: on timeout the status word counts it and the CTA stops) and read halo
// positions with L2-coherent loads (ld.global.cg).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "vbd_math.cuh"
#include "vbd_resident.h"

namespace vbd {

namespace {

constexpr int kLanes = 4;
constexpr unsigned kTmaChunk = 32768;
// Bound of the wait for the CTA's own bulk copies (independent of the tunable neighbour-wait
// limit: a CTA never leaves while a copy into its shared memory may still be in flight).
constexpr unsigned kTmaWaitLimit = 1u << 24;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fence_acquire_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ float lane_sum(float v) {
    for (int off = kLanes >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

struct ResidentKernelArgs {
    const PatchMeta* meta;
    const unsigned char* blob;
    const int* l2g;
    const int* nbr;
    int* progress;
    const int* perm;
    const float4* pinfo;
    const DevShape* shapes;
    int colors;
    ResidentLaunch L;
};

template <bool kDamp>
__global__ void __launch_bounds__(kResidentThreads, 1) resident_kernel(ResidentKernelArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ PatchMeta M;
    __shared__ int s_abort;
    const int t = threadIdx.x;
    const int p = blockIdx.x;
    const ResidentLaunch& a = A.L;
    if (t == 0) {
        M = A.meta[p];
        s_abort = 0;
    }
    __syncthreads();

    // static image (element data, references) by TMA bulk copies completing on one mbarrier
    if (t == 0 && M.blob_bytes > 0) {
        mbar_init(&s_bar, 1);
        mbar_arrive_expect_tx(&s_bar, static_cast<unsigned>(M.blob_bytes));
        for (unsigned off = 0; off < static_cast<unsigned>(M.blob_bytes); off += kTmaChunk) {
            const unsigned n = min(kTmaChunk, static_cast<unsigned>(M.blob_bytes) - off);
            tma_bulk_load(smem + off, A.blob + M.blob_offset + off, n, &s_bar);
        }
    }
    const int* l2g = A.l2g + M.l2g_offset;
    float4* s_pos = reinterpret_cast<float4*>(smem + M.off_pos);
    float4* s_y = reinterpret_cast<float4*>(smem + M.off_y);
    float4* s_prev = reinterpret_cast<float4*>(smem + M.off_prev);
    float4* s_disp = reinterpret_cast<float4*>(smem + M.off_disp);
    for (int l = t; l < M.n_local; l += kResidentThreads) {
        const int g = l2g[l];
        s_pos[l] = __ldcg(&a.pos[g]);
        s_prev[l] = __ldcg(&a.prev[g]);
    }
    float4* s_pinfo = reinterpret_cast<float4*>(smem + M.off_pinfo);
    int* s_ccount = reinterpret_cast<int*>(smem + M.off_ccount);
    for (int l = t; l < M.n_owned; l += kResidentThreads) {
        const int g = l2g[l];
        s_y[l] = __ldcg(&a.y[g]);
        s_disp[l] = __ldcg(&a.disp[g]);
        s_pinfo[l] = __ldg(&A.pinfo[g]);
        s_ccount[l] = a.ccount ? __ldcg(&a.ccount[g]) : 0;
    }
    if (t == 0 && M.blob_bytes > 0) {
        unsigned spins = 0;
        while (!mbar_try_wait(&s_bar, 0)) {
            if (++spins > kTmaWaitLimit) {
                atomicAdd(&a.status[3], 1u);
                s_abort = 1;
                // the copies are still in flight: wait for them (again bounded) before leaving
                unsigned drain = 0;
                while (!mbar_try_wait(&s_bar, 0) && ++drain < kTmaWaitLimit) __nanosleep(256);
                break;
            }
            __nanosleep(32);
        }
    }
    __syncthreads();

    const int4* s_vr = reinterpret_cast<const int4*>(smem);
    const unsigned* s_refs = reinterpret_cast<const unsigned*>(smem + M.off_refs);
    const ushort4* s_tri_idx = reinterpret_cast<const ushort4*>(smem + M.off_tri_idx);
    const float4* s_tri_D = reinterpret_cast<const float4*>(smem + M.off_tri_D);
    const float4* s_tri_mat = reinterpret_cast<const float4*>(smem + M.off_tri_mat);
    const ushort4* s_hinge_idx = reinterpret_cast<const ushort4*>(smem + M.off_hinge_idx);
    const float4* s_hinge_mat = reinterpret_cast<const float4*>(smem + M.off_hinge_mat);
    const float inv_dt = 1.0f / a.dt;
    const float dtsr = 1.0f / (a.dt * a.dt);
    const float eps_u = a.friction_epsilon * a.dt;
    const DevShape* shapes = A.shapes;
    auto shape_mat = [shapes](int s) { return shapes[s].mat; };
    const int C = A.colors;
    const int steps = s_abort ? 0 : a.iterations * C;

    // Solves owned vertices [vb, ve) of the current color (4 lanes per vertex).
    auto solve_range = [&](int vb, int ve) {
        const int nthreads = (ve - vb) * kLanes;
        for (int base = 0; base < nthreads; base += kResidentThreads) {
            const int idx = base + t;
            const bool valid = idx < nthreads;
            const int v = vb + idx / kLanes;
            const int lane = idx & (kLanes - 1);
            float3 f = f3(0.f, 0.f, 0.f);
            Sym3 h = zero_sym();
            if (valid) {
                const int4 vr = s_vr[v];
                for (int r = vr.x + lane; r < vr.y; r += kLanes) {
                    const unsigned ref = s_refs[r];
                    const int e = static_cast<int>(ref >> 2);
                    const ushort4 ti = s_tri_idx[e];
                    const float4 mt = s_tri_mat[e];
                    const float3 x0 = xyz(s_pos[ti.x]), x1 = xyz(s_pos[ti.y]), x2 = xyz(s_pos[ti.z]);
                    float3 p0 = x0, p1 = x1, p2 = x2;
                    if (kDamp && mt.w > 0.0f) {
                        p0 = xyz(s_prev[ti.x]);
                        p1 = xyz(s_prev[ti.y]);
                        p2 = xyz(s_prev[ti.z]);
                    }
                    membrane_eval<kDamp>(static_cast<int>(ref & 3u), x0, x1, x2, p0, p1, p2, s_tri_D[e], mt, inv_dt,
                                         f, h);
                }
                // hinges continue the round-robin deal of the merged record list
                const int lane_e = (lane - (vr.y - vr.x) % kLanes + kLanes) % kLanes;
                for (int r = vr.z + lane_e; r < vr.w; r += kLanes) {
                    const unsigned ref = s_refs[r];
                    const int e = static_cast<int>(ref >> 2);
                    const ushort4 hi = s_hinge_idx[e];
                    const float4 em = s_hinge_mat[e];
                    const float3 x0 = xyz(s_pos[hi.x]), x1 = xyz(s_pos[hi.y]), x2 = xyz(s_pos[hi.z]),
                                 x3 = xyz(s_pos[hi.w]);
                    float3 p0 = x0, p1 = x1, p2 = x2, p3 = x3;
                    if (kDamp && em.w > 0.0f) {
                        p0 = xyz(s_prev[hi.x]);
                        p1 = xyz(s_prev[hi.y]);
                        p2 = xyz(s_prev[hi.z]);
                        p3 = xyz(s_prev[hi.w]);
                    }
                    bending_eval<kDamp>(static_cast<int>(ref & 3u), x0, x1, x2, x3, p0, p1, p2, p3, em, inv_dt, f, h);
                }
            }
            f.x = lane_sum(f.x);
            f.y = lane_sum(f.y);
            f.z = lane_sum(f.z);
            h.xx = lane_sum(h.xx);
            h.xy = lane_sum(h.xy);
            h.xz = lane_sum(h.xz);
            h.yy = lane_sum(h.yy);
            h.yz = lane_sum(h.yz);
            h.zz = lane_sum(h.zz);
            if (valid && lane == 0) {
                const int g = l2g[v];
                const float4 pi = s_pinfo[v];
                const float4 pv = s_prev[v];
                const bool solve = (__float_as_int(pi.w) & VBD_PARTICLE_ACTIVE) && pi.x != 0.0f;
                float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
                if (solve) {
                    const float3 x = xyz(s_pos[v]);
                    const float4 yv = s_y[v];
                    const float mass = yv.w;
                    float3 fc = f3(0.f, 0.f, 0.f);
                    Sym3 hc = zero_sym();
                    if (s_ccount[v] > 0)
                        vertex_contacts(a.ccount, a.cslot, a.K, g, a.c_shape, a.c_body_pos, a.c_body_vel, a.c_normal,
                                        shape_mat, x, xyz(pv), pi.z, a.dt, eps_u, fc, hc);
                    add_diag(h, mass * dtsr);
                    add(h, hc);
                    const float3 fi = (mass * (xyz(yv) - x)) * dtsr;
                    f = f + fi + fc;
                    float3 dx;
                    d = s_disp[v];
                    if (solve3(h, f, dx)) {
                        if (isfinite(dx.x) && isfinite(dx.y) && isfinite(dx.z)) {
                            d = make_float4(d.x + dx.x, d.y + dx.y, d.z + dx.z, 0.f);
                        } else {
                            atomicAdd(&a.status[0], 1u);
                        }
                    } else {
                        atomicAdd(&a.status[1], 1u);
                    }
                }
                const float4 np = make_float4(pv.x + d.x, pv.y + d.y, pv.z + d.z, 0.f);
                s_disp[v] = d;
                s_pos[v] = np;
                a.pos[g] = np;  // published to the neighbours at the end of the step
            }
        }
    };

    const int* nb = A.nbr + M.nbr_offset;
    for (int step = 0; step < steps; ++step) {
        const int c = step % C;
        // one thread per neighbour issues a relaxed read of its progress now; the read's latency
        // overlaps the interior vertices, which read owned positions only and need no wait
        int seen = step;
        if (step > 0 && t < M.n_nbr) seen = ld_relaxed(A.progress + nb[t]);
        solve_range(M.own_color_start[c], M.own_color_mid[c]);
        if (step > 0) {
            if (t < M.n_nbr) {
                unsigned spins = 0;
                while (seen < step) {
                    if (++spins > a.spin_limit || *static_cast<volatile int*>(&s_abort)) {
                        atomicAdd(&a.status[3], 1u);
                        s_abort = 1;
                        break;
                    }
                    __nanosleep(20);
                    seen = ld_relaxed(A.progress + nb[t]);
                }
                fence_acquire_gpu();  // acquire: the neighbour's published positions are visible
            }
            for (int k = t + kResidentThreads; k < M.n_nbr; k += kResidentThreads) {  // > 512 neighbours
                unsigned spins = 0;
                while (ld_relaxed(A.progress + nb[k]) < step) {
                    if (++spins > a.spin_limit || *static_cast<volatile int*>(&s_abort)) {
                        atomicAdd(&a.status[3], 1u);
                        s_abort = 1;
                        break;
                    }
                    __nanosleep(20);
                }
                fence_acquire_gpu();
            }
            __syncthreads();
            if (s_abort) break;
            const int cp = (c + C - 1) % C;
            for (int l = M.halo_color_start[cp] + t; l < M.halo_color_start[cp + 1]; l += kResidentThreads)
                s_pos[l] = __ldcg(&a.pos[l2g[l]]);
            __syncthreads();
        }
        solve_range(M.own_color_mid[c], M.own_color_start[c + 1]);
        __syncthreads();
        // release: every position stored by this CTA before the barrier is visible before the
        // new progress value is
        if (t == 0) st_release(A.progress + p, step + 1);
    }
    __syncthreads();
    // finalize: state_in.q (the GS iterate), state_out.q, state_out.qd = (x - x_prev) / dt
    for (int l = t; l < M.n_owned; l += kResidentThreads) {
        const int g = l2g[l];
        const int o = A.perm[g];
        const float4 x = s_pos[l], pv = s_prev[l];
        a.pos[g] = x;
        a.disp[g] = s_disp[l];
        if (a.q_in) {
            a.q_in[3 * o] = x.x;
            a.q_in[3 * o + 1] = x.y;
            a.q_in[3 * o + 2] = x.z;
        }
        if (a.q_out) {
            a.q_out[3 * o] = x.x;
            a.q_out[3 * o + 1] = x.y;
            a.q_out[3 * o + 2] = x.z;
        }
        if (a.qd_out) {
            a.qd_out[3 * o] = (x.x - pv.x) / a.dt;
            a.qd_out[3 * o + 1] = (x.y - pv.y) / a.dt;
            a.qd_out[3 * o + 2] = (x.z - pv.z) / a.dt;
        }
        if (a.ccount_clear) a.ccount_clear[g] = 0;
    }
}

// ---- host: patch decomposition -----------------------------------------------------------
struct DSU {
    std::vector<int> p;
    explicit DSU(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
    int find(int x) {
        while (p[x] != x) x = p[x] = p[p[x]];
        return x;
    }
    void unite(int a, int b) {
        a = find(a);
        b = find(b);
        if (a != b) p[std::max(a, b)] = std::min(a, b);
    }
};

// recursive coordinate bisection of `v` into k parts (by rest position; BFS-free fallback keeps order)
void rcb(std::vector<int>& v, int lo, int hi, int k, const std::vector<float>& q, std::vector<std::vector<int>>& out) {
    if (k <= 1 || hi - lo <= 1) {
        out.emplace_back(v.begin() + lo, v.begin() + hi);
        return;
    }
    int axis = 0;
    if (!q.empty()) {
        float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
        for (int i = lo; i < hi; ++i)
            for (int d = 0; d < 3; ++d) {
                mn[d] = std::min(mn[d], q[3 * v[i] + d]);
                mx[d] = std::max(mx[d], q[3 * v[i] + d]);
            }
        for (int d = 1; d < 3; ++d)
            if (mx[d] - mn[d] > mx[axis] - mn[axis]) axis = d;
    }
    const int k1 = k / 2;
    const int mid = lo + static_cast<int>((static_cast<long long>(hi - lo) * k1) / k);
    if (!q.empty())
        std::nth_element(v.begin() + lo, v.begin() + mid, v.begin() + hi,
                         [&](int a, int b) { return q[3 * a + axis] < q[3 * b + axis] || (q[3 * a + axis] == q[3 * b + axis] && a < b); });
    rcb(v, lo, mid, k1, q, out);
    rcb(v, mid, hi, k - k1, q, out);
}

int align16(int x) { return (x + 15) & ~15; }

template <bool kDamp>
int set_smem(int bytes) {
    cudaError_t e = cudaFuncSetAttribute(resident_kernel<kDamp>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e == cudaSuccess ? VBD_OK : cuda_fail(e, "cudaFuncSetAttribute(resident_kernel)");
}

}  // namespace

void resident_free(ResidentPlan& plan) {
    void* ptrs[] = {plan.meta, plan.blob, plan.l2g, plan.nbr, plan.progress};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    plan = ResidentPlan();
}

int resident_build(const VbdModelImpl& m, ResidentPlan& plan) {
    resident_free(plan);
    const int V = m.V, C = m.C;
    if (V == 0 || C == 0 || C > kResidentMaxColors || !m.fused_commit || m.swept != V) return VBD_OK;
    int dev = 0, sms = 0, smem_optin = 0;
    VBD_CUDA_TRY(cudaGetDevice(&dev));
    VBD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    VBD_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const int smem_limit = smem_optin - 1024;  // static shared (mbarrier, meta, flags)
    std::vector<int> color(V);
    for (int c = 0; c < C; ++c)
        for (int i = m.color_start[c]; i < m.color_start[c + 1]; ++i) color[i] = c;

    // connected components over element stencils
    DSU dsu(V);
    for (const int4& r : m.tri_idx_h) {
        dsu.unite(r.x, r.y);
        dsu.unite(r.x, r.z);
    }
    for (const int4& r : m.edge_idx_h) {
        const int o0 = r.x & 0x3fffffff;
        dsu.unite(o0, r.y);
        dsu.unite(o0, r.z);
        dsu.unite(o0, r.w);
    }
    std::vector<std::vector<int>> comps;
    {
        std::vector<int> id(V, -1);
        for (int i = 0; i < V; ++i) {
            const int r = dsu.find(i);
            if (id[r] < 0) {
                id[r] = static_cast<int>(comps.size());
                comps.emplace_back();
            }
            comps[id[r]].push_back(i);
        }
    }
    // target patch size: enough patches to fill the SMs, but at least ~96 vertices per color
    const int target = std::max((V + sms - 1) / sms, 96 * C);
    std::vector<std::vector<int>> patches;
    std::vector<std::vector<int>> small;
    for (auto& cv : comps) {
        if (static_cast<int>(cv.size()) > target) {
            const int k = (static_cast<int>(cv.size()) + target - 1) / target;
            rcb(cv, 0, static_cast<int>(cv.size()), k, m.rest_q_h, patches);
        } else {
            small.push_back(std::move(cv));
        }
    }
    // pack whole small components first-fit decreasing
    std::sort(small.begin(), small.end(), [](const std::vector<int>& a, const std::vector<int>& b) { return a.size() > b.size(); });
    const size_t first_small = patches.size();
    for (auto& cv : small) {
        bool placed = false;
        for (size_t b = first_small; b < patches.size(); ++b) {
            if (patches[b].size() + cv.size() <= static_cast<size_t>(target)) {
                patches[b].insert(patches[b].end(), cv.begin(), cv.end());
                placed = true;
                break;
            }
        }
        if (!placed) patches.push_back(cv);
    }
    const int P = static_cast<int>(patches.size());
    if (P > sms) return VBD_OK;  // one CTA per SM, all co-resident
    std::vector<int> patch_of(V, -1);
    for (int p = 0; p < P; ++p) {
        std::sort(patches[p].begin(), patches[p].end());  // internal order == color-major
        for (int v : patches[p]) patch_of[v] = p;
    }

    std::vector<PatchMeta> meta(P);
    std::vector<unsigned char> blob;
    std::vector<int> l2g_all, nbr_all;
    std::vector<int> local_of(V, -1), tri_local(m.T > 0 ? m.T : 1, -1), hinge_local(m.E > 0 ? m.E : 1, -1);
    int smem_max = 0, max_owned_color = 0;
    for (int p = 0; p < P; ++p) {
        const std::vector<int>& own = patches[p];
        PatchMeta& M = meta[p];
        std::memset(&M, 0, sizeof(M));
        M.n_owned = static_cast<int>(own.size());
        for (int l = 0; l < M.n_owned; ++l) local_of[own[l]] = l;
        // halo: vertices of owned vertices' elements that this patch does not own
        std::vector<int> halo;
        auto touch = [&](int g) {
            if (local_of[g] == -1) {
                local_of[g] = -2;
                halo.push_back(g);
            }
        };
        std::vector<int> tris, hinges;  // record index of the first occurrence of each element
        for (int v : own) {
            const int4 ad = m.vadj_h[v];
            for (int r = ad.x; r < ad.y; ++r) {
                const int4 ti = m.tri_idx_h[r];
                touch(ti.x);
                touch(ti.y);
                touch(ti.z);
                const int e = m.tri_elem_h[r];
                if (tri_local[e] == -1) {
                    tri_local[e] = static_cast<int>(tris.size());
                    tris.push_back(r);
                }
            }
            for (int r = ad.z; r < ad.w; ++r) {
                const int4 hi = m.edge_idx_h[r];
                touch(hi.x & 0x3fffffff);
                touch(hi.y);
                touch(hi.z);
                touch(hi.w);
                const int e = m.edge_elem_h[r];
                if (hinge_local[e] == -1) {
                    hinge_local[e] = static_cast<int>(hinges.size());
                    hinges.push_back(r);
                }
            }
        }
        std::sort(halo.begin(), halo.end());  // internal order: by color, then index
        // inside each color, interior vertices (whole stencil owned) first, then boundary ones
        std::vector<int> own_sorted = own;
        {
            auto is_boundary = [&](int v) {
                const int4 ad = m.vadj_h[v];
                for (int r = ad.x; r < ad.y; ++r) {
                    const int4 ti = m.tri_idx_h[r];
                    if (local_of[ti.x] < 0 || local_of[ti.y] < 0 || local_of[ti.z] < 0) return true;
                }
                for (int r = ad.z; r < ad.w; ++r) {
                    const int4 hi = m.edge_idx_h[r];
                    if (local_of[hi.x & 0x3fffffff] < 0 || local_of[hi.y] < 0 || local_of[hi.z] < 0 ||
                        local_of[hi.w] < 0)
                        return true;
                }
                return false;
            };
            std::vector<char> bnd(own.size());
            for (size_t k = 0; k < own.size(); ++k) bnd[k] = is_boundary(own[k]) ? 1 : 0;
            std::vector<int> order(own.size());
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
                const int cx = color[own[x]], cy = color[own[y]];
                if (cx != cy) return cx < cy;
                return bnd[x] < bnd[y];
            });
            for (size_t k = 0; k < own.size(); ++k) own_sorted[k] = own[order[k]];
            for (int c = 0, k = 0; c < C; ++c) {
                while (k < static_cast<int>(own.size()) && color[own[order[k]]] < c) ++k;
                int j = k;
                while (j < static_cast<int>(own.size()) && color[own[order[j]]] == c && !bnd[order[j]]) ++j;
                M.own_color_mid[c] = j;
            }
        }
        for (int l = 0; l < M.n_owned; ++l) local_of[own_sorted[l]] = l;
        M.n_local = M.n_owned + static_cast<int>(halo.size());
        for (size_t k = 0; k < halo.size(); ++k) local_of[halo[k]] = M.n_owned + static_cast<int>(k);
        M.n_tri = static_cast<int>(tris.size());
        M.n_hinge = static_cast<int>(hinges.size());
        bool fits = M.n_local <= 65535 && M.n_tri < (1 << 29) && M.n_hinge < (1 << 29);
        // per-color ranges
        for (int c = 0, l = 0; c <= C; ++c) {
            while (l < M.n_owned && color[own_sorted[l]] < c) ++l;
            M.own_color_start[c] = l;
        }
        for (int c = 0, k = 0; c <= C; ++c) {
            while (k < static_cast<int>(halo.size()) && color[halo[k]] < c) ++k;
            M.halo_color_start[c] = M.n_owned + k;
        }
        for (int c = 0; c < C; ++c)
            max_owned_color = std::max(max_owned_color, M.own_color_start[c + 1] - M.own_color_start[c]);
        // references per owned vertex
        std::vector<int4> vr(M.n_owned);
        std::vector<unsigned> refs;
        for (int l = 0; l < M.n_owned; ++l) {
            const int4 ad = m.vadj_h[own_sorted[l]];
            int4 rr;
            rr.x = static_cast<int>(refs.size());
            for (int r = ad.x; r < ad.y; ++r)
                refs.push_back((static_cast<unsigned>(tri_local[m.tri_elem_h[r]]) << 2) |
                               static_cast<unsigned>(m.tri_idx_h[r].w));
            rr.y = static_cast<int>(refs.size());
            rr.z = rr.y;
            for (int r = ad.z; r < ad.w; ++r)
                refs.push_back((static_cast<unsigned>(hinge_local[m.edge_elem_h[r]]) << 2) |
                               (static_cast<unsigned>(m.edge_idx_h[r].x) >> 30));
            rr.w = static_cast<int>(refs.size());
            vr[l] = rr;
        }
        M.n_refs = static_cast<int>(refs.size());
        // shared-memory image layout
        int off = align16(M.n_owned * 16);
        M.off_refs = off;
        off = align16(off + M.n_refs * 4);
        M.off_tri_idx = off;
        off = align16(off + M.n_tri * 8);
        M.off_tri_D = off;
        off = align16(off + M.n_tri * 16);
        M.off_tri_mat = off;
        off = align16(off + M.n_tri * 16);
        M.off_hinge_idx = off;
        off = align16(off + M.n_hinge * 8);
        M.off_hinge_mat = off;
        off = align16(off + M.n_hinge * 16);
        M.blob_bytes = off;
        M.off_pos = off;
        off = align16(off + M.n_local * 16);
        M.off_prev = off;
        off += M.n_local * 16;
        M.off_y = off;
        off += M.n_owned * 16;
        M.off_disp = off;
        off += M.n_owned * 16;
        M.off_pinfo = off;
        off += M.n_owned * 16;
        M.off_ccount = off;
        off = align16(off + M.n_owned * 4);
        if (off > smem_limit || !fits) {
            // does not fit: leave the plan unusable (per-color launches)
            for (int g : own) local_of[g] = -1;
            for (int g : halo) local_of[g] = -1;
            for (int r : tris) tri_local[m.tri_elem_h[r]] = -1;
            for (int r : hinges) hinge_local[m.edge_elem_h[r]] = -1;
            return VBD_OK;
        }
        smem_max = std::max(smem_max, off);
        M.blob_offset = static_cast<int>(blob.size());
        blob.resize(blob.size() + M.blob_bytes, 0);
        unsigned char* B = blob.data() + M.blob_offset;
        std::memcpy(B, vr.data(), vr.size() * sizeof(int4));
        if (!refs.empty()) std::memcpy(B + M.off_refs, refs.data(), refs.size() * 4);
        for (int k = 0; k < M.n_tri; ++k) {
            const int r = tris[k];
            const int4 ti = m.tri_idx_h[r];
            const unsigned short idx[4] = {static_cast<unsigned short>(local_of[ti.x]),
                                           static_cast<unsigned short>(local_of[ti.y]),
                                           static_cast<unsigned short>(local_of[ti.z]), 0};
            std::memcpy(B + M.off_tri_idx + 8 * k, idx, 8);
            std::memcpy(B + M.off_tri_D + 16 * k, &m.tri_D_h[r], 16);
            std::memcpy(B + M.off_tri_mat + 16 * k, &m.tri_mat_h[r], 16);
        }
        for (int k = 0; k < M.n_hinge; ++k) {
            const int r = hinges[k];
            const int4 hi = m.edge_idx_h[r];
            const unsigned short idx[4] = {static_cast<unsigned short>(local_of[hi.x & 0x3fffffff]),
                                           static_cast<unsigned short>(local_of[hi.y]),
                                           static_cast<unsigned short>(local_of[hi.z]),
                                           static_cast<unsigned short>(local_of[hi.w])};
            std::memcpy(B + M.off_hinge_idx + 8 * k, idx, 8);
            std::memcpy(B + M.off_hinge_mat + 16 * k, &m.edge_mat_h[r], 16);
        }
        M.l2g_offset = static_cast<int>(l2g_all.size());
        l2g_all.insert(l2g_all.end(), own_sorted.begin(), own_sorted.end());
        l2g_all.insert(l2g_all.end(), halo.begin(), halo.end());
        std::vector<int> nb;
        for (int g : halo) nb.push_back(patch_of[g]);
        std::sort(nb.begin(), nb.end());
        nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
        M.nbr_offset = static_cast<int>(nbr_all.size());
        M.n_nbr = static_cast<int>(nb.size());
        nbr_all.insert(nbr_all.end(), nb.begin(), nb.end());
        // reset the scratch maps touched by this patch
        for (int g : own) local_of[g] = -1;
        for (int g : halo) local_of[g] = -1;
        for (int r : tris) tri_local[m.tri_elem_h[r]] = -1;
        for (int r : hinges) hinge_local[m.edge_elem_h[r]] = -1;
    }
    // occupancy: one CTA per SM must fit
    int rc;
    if ((rc = set_smem<false>(smem_max))) return rc;
    if ((rc = set_smem<true>(smem_max))) return rc;
    int per_sm = 0;
    VBD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, resident_kernel<true>, kResidentThreads, smem_max));
    if (per_sm < 1) return VBD_OK;

    if (nbr_all.empty()) nbr_all.push_back(0);
    auto up = [](auto** dst, const auto& src) -> int {
        using T = typename std::remove_reference<decltype(src)>::type::value_type;
        VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), src.size() * sizeof(T)));
        VBD_CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
        return VBD_OK;
    };
    if ((rc = up(&plan.meta, meta))) return rc;
    if ((rc = up(&plan.blob, blob))) return rc;
    if ((rc = up(&plan.l2g, l2g_all))) return rc;
    if ((rc = up(&plan.nbr, nbr_all))) return rc;
    VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&plan.progress), sizeof(int) * P));
    VBD_CUDA_TRY(cudaMemset(plan.progress, 0, sizeof(int) * P));
    plan.meta_h = std::move(meta);
    plan.patches = P;
    plan.smem_bytes = smem_max;
    plan.max_owned_per_color = max_owned_color;
    plan.ready = true;
    return VBD_OK;
}

int resident_enqueue(const VbdModelImpl& m, const ResidentPlan& plan, const ResidentLaunch& L, cudaStream_t st) {
    VBD_CUDA_TRY(cudaMemsetAsync(plan.progress, 0, sizeof(int) * plan.patches, st));
    ResidentKernelArgs A;
    A.meta = plan.meta;
    A.blob = plan.blob;
    A.l2g = plan.l2g;
    A.nbr = plan.nbr;
    A.progress = plan.progress;
    A.perm = m.perm;
    A.pinfo = m.pinfo;
    A.shapes = m.shapes;
    A.colors = m.C;
    A.L = L;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(plan.patches);
    cfg.blockDim = dim3(kResidentThreads);
    cfg.dynamicSmemBytes = static_cast<size_t>(plan.smem_bytes);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const bool damp = m.any_tri_damping || m.any_edge_damping;
    cudaError_t e = damp ? cudaLaunchKernelEx(&cfg, resident_kernel<true>, A) : cudaLaunchKernelEx(&cfg, resident_kernel<false>, A);
    if (e != cudaSuccess) return cuda_fail(e, "cudaLaunchKernelEx(resident_kernel)");
    return VBD_OK;
}

}  // namespace vbd
