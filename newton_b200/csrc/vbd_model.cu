// vbd_model.cu -- device model construction (vbd_model_create) and soft-contact generation
// (vbd_collide).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "vbd_internal.h"
#include "vbd_math.cuh"

namespace vbd {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
int cuda_fail(cudaError_t err, const char* what) {
    g_last_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(err);
    return err == cudaErrorMemoryAllocation ? VBD_ERR_OUT_OF_MEMORY : VBD_ERR_CUDA;
}

template <typename T>
static int upload(T** dst, const std::vector<T>& src) {
    *dst = nullptr;
    if (src.empty()) return VBD_OK;
    VBD_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), src.size() * sizeof(T)));
    VBD_CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return VBD_OK;
}

static void free_model(VbdModelImpl& m) {
    void* ptrs[] = {m.perm,       m.inv_perm, m.pinfo,          m.vadj,
                    m.tri_idx,    m.tri_D,    m.tri_mat,        m.edge_idx,
                    m.edge_mat,   m.shapes,   m.particle_world, m.particle_flags_orig,
                    m.particle_radius_orig, m.nbr8, m.vfeat, m.world_shape_offsets, m.world_shapes};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    m.perm = m.inv_perm = nullptr;
    m.pinfo = nullptr;
    m.vadj = nullptr;
    m.tri_idx = nullptr;
    m.tri_D = m.tri_mat = nullptr;
    m.edge_idx = nullptr;
    m.edge_mat = nullptr;
    m.shapes = nullptr;
    m.particle_world = m.particle_flags_orig = nullptr;
    m.particle_radius_orig = nullptr;
    m.nbr8 = nullptr;
    m.vfeat = nullptr;
    m.world_shape_offsets = m.world_shapes = nullptr;
}

static int build_model(const VbdModelDesc* d, VbdModelImpl& m) {
    if (!d) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: desc is NULL");
    const int V = d->particle_count, T = d->tri_count, E = d->edge_count, S = d->shape_count, C = d->color_count;
    if (V < 0 || T < 0 || E < 0 || S < 0 || C < 0)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: negative element count");
    if (V >= (1 << 30)) return fail(VBD_ERR_UNSUPPORTED, "vbd_model_create: more than 2^30 particles");
    if (V > 0 && (!d->particle_mass || !d->particle_inv_mass || !d->particle_flags || !d->particle_radius))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: particle arrays missing");
    if (T > 0 && (!d->tri_indices || !d->tri_poses || !d->tri_materials || !d->tri_areas || !d->v_adj_tris_offsets ||
                  !d->v_adj_tris))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: triangle arrays or adjacency missing");
    if (E > 0 && (!d->edge_indices || !d->edge_rest_angle || !d->edge_rest_length || !d->edge_bending_properties ||
                  !d->v_adj_edges_offsets || !d->v_adj_edges))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: edge arrays or adjacency missing");
    if (V > 0 && C == 0)
        return fail(VBD_ERR_INVALID_ARGUMENT,
                    "model.particle_color_groups is empty! Call ModelBuilder.color() or set_coloring() before "
                    "finalize()");
    if (C > 0 && (!d->color_group_offsets || !d->color_group_particles))
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: color groups missing");
    if (S > 0 && !d->shapes) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: shapes missing");
    VBD_CUDA_TRY(cudaGetDevice(&m.device));
    m.V = V;
    m.T = T;
    m.E = E;
    m.S = S;
    m.C = C;
    for (int k = 0; k < 3; ++k) m.gravity[k] = d->gravity[k];
    m.gravity_norm = std::sqrt(m.gravity[0] * m.gravity[0] + m.gravity[1] * m.gravity[1] + m.gravity[2] * m.gravity[2]);

    // ---- color-major renumbering -------------------------------------------------------
    std::vector<int> color_of(V, -1);
    m.color_start.assign(C + 1, 0);
    std::vector<int> perm;
    perm.reserve(V);
    for (int c = 0; c < C; ++c) {
        const int b = d->color_group_offsets[c], e = d->color_group_offsets[c + 1];
        if (b < 0 || e < b) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: bad color_group_offsets");
        std::vector<int> grp(d->color_group_particles + b, d->color_group_particles + e);
        std::sort(grp.begin(), grp.end());
        m.color_start[c] = static_cast<int>(perm.size());
        for (int v : grp) {
            if (v < 0 || v >= V) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: color group index out of range");
            if (color_of[v] != -1)
                return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: particle appears in two color groups");
            color_of[v] = c;
            perm.push_back(v);
        }
    }
    m.color_start[C] = static_cast<int>(perm.size());
    m.swept = static_cast<int>(perm.size());
    for (int v = 0; v < V; ++v)
        if (color_of[v] == -1) perm.push_back(v);  // never swept: moves with its inertia target
    std::vector<int> inv(V);
    for (int i = 0; i < V; ++i) inv[perm[i]] = i;
    m.perm_host = perm;

    // ---- conflict check: may a color's update be written in place? ---------------------
    m.fused_commit = true;
    for (int t = 0; t < T && m.fused_commit; ++t) {
        const int* ti = d->tri_indices + 3 * t;
        const int a = ti[0], b = ti[1], c = ti[2];
        if (color_of[a] >= 0 && (color_of[a] == color_of[b] || color_of[a] == color_of[c])) m.fused_commit = false;
        if (color_of[b] >= 0 && color_of[b] == color_of[c]) m.fused_commit = false;
    }
    for (int e = 0; e < E && m.fused_commit; ++e) {
        const int* ei = d->edge_indices + 4 * e;
        if (ei[0] < 0 || ei[1] < 0 || !(d->edge_bending_properties[2 * e] > 0.0f)) continue;
        for (int x = 0; x < 4; ++x)
            for (int y = x + 1; y < 4; ++y)
                if (color_of[ei[x]] >= 0 && color_of[ei[x]] == color_of[ei[y]]) m.fused_commit = false;
    }

    // ---- per-vertex element records ----------------------------------------------------
    // Two passes over the vertices, each split over the host's cores: count the records each
    // vertex keeps, then (after a prefix sum) write them at their offsets.  The record order is
    // the serial one: vertices in internal order, a vertex's records in its CSR order.
    std::vector<float4> pinfo(V);
    std::vector<int4> vadj(V);
    std::vector<int> n_tri_keep(static_cast<size_t>(V) + 1, 0), n_edge_keep(static_cast<size_t>(V) + 1, 0);
    std::atomic<int> bad_record{-1};  // smallest internal vertex with an invalid record, or -1
    auto solvable_of = [&](int o) {
        return (d->particle_flags[o] & VBD_PARTICLE_ACTIVE) && d->particle_mass[o] != 0.0f;
    };
    auto tri_kept = [&](int t) {
        const float* mat = d->tri_materials + 5 * t;
        return mat[0] > 0.0f || mat[1] > 0.0f;  // the reference skips the others
    };
    auto edge_kept = [&](int ed) {
        const int* ei = d->edge_indices + 4 * ed;
        // ke <= 0: not evaluated by the reference; boundary hinge: exact zero in the reference
        return d->edge_bending_properties[2 * ed] > 0.0f && ei[0] != -1 && ei[1] != -1;
    };
    auto note_bad = [&](int i) {
        int cur = bad_record.load();
        while ((cur == -1 || i < cur) && !bad_record.compare_exchange_weak(cur, i)) {
        }
    };
    parallel_chunks(V, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            const int o = perm[i];
            // pinned / massless vertices are never solved (solve_elasticity returns early for
            // them), so they own no element records
            if (!solvable_of(o)) continue;
            int nt = 0, ne = 0;
            if (T > 0) {
                for (int k = d->v_adj_tris_offsets[o]; k < d->v_adj_tris_offsets[o + 1]; k += 2) {
                    const int t = d->v_adj_tris[k], slot = d->v_adj_tris[k + 1];
                    if (t < 0 || t >= T || slot < 0 || slot > 2) {
                        note_bad(i);
                        break;
                    }
                    nt += tri_kept(t) ? 1 : 0;
                }
            }
            if (E > 0) {
                for (int k = d->v_adj_edges_offsets[o]; k < d->v_adj_edges_offsets[o + 1]; k += 2) {
                    const int ed = d->v_adj_edges[k], slot = d->v_adj_edges[k + 1];
                    if (ed < 0 || ed >= E || slot < 0 || slot > 3) {
                        note_bad(i);
                        break;
                    }
                    ne += edge_kept(ed) ? 1 : 0;
                }
            }
            n_tri_keep[i + 1] = nt;
            n_edge_keep[i + 1] = ne;
        }
    });
    if (bad_record.load() >= 0) {
        // report the first invalid record the serial walk would meet
        const int o = perm[bad_record.load()];
        bool tri_bad = false;
        if (T > 0)
            for (int k = d->v_adj_tris_offsets[o]; k < d->v_adj_tris_offsets[o + 1]; k += 2) {
                const int t = d->v_adj_tris[k], slot = d->v_adj_tris[k + 1];
                tri_bad |= t < 0 || t >= T || slot < 0 || slot > 2;
            }
        return fail(VBD_ERR_INVALID_ARGUMENT, tri_bad ? "vbd_model_create: bad triangle adjacency record"
                                                      : "vbd_model_create: bad edge adjacency record");
    }
    for (int i = 0; i < V; ++i) {
        n_tri_keep[i + 1] += n_tri_keep[i];
        n_edge_keep[i + 1] += n_edge_keep[i];
    }
    const size_t n_tri_rec = static_cast<size_t>(n_tri_keep[V]), n_edge_rec = static_cast<size_t>(n_edge_keep[V]);
    std::vector<int4> tri_idx(n_tri_rec);
    std::vector<float4> tri_D(n_tri_rec), tri_mat(n_tri_rec);
    std::vector<int4> edge_idx(n_edge_rec);
    std::vector<float4> edge_mat(n_edge_rec);
    m.tri_elem_h.assign(n_tri_rec, 0);
    m.edge_elem_h.assign(n_edge_rec, 0);
    std::atomic<bool> any_tri_damp{false}, any_edge_damp{false};
    parallel_chunks(V, [&](int b, int e) {
        bool tdamp = false, edamp = false;
        for (int i = b; i < e; ++i) {
            const int o = perm[i];
            int flags = d->particle_flags[o];
            float fl;
            std::memcpy(&fl, &flags, sizeof(float));
            pinfo[i] = make_float4(d->particle_mass[o], d->particle_inv_mass[o], d->particle_radius[o], fl);
            vadj[i] = make_int4(n_tri_keep[i], n_tri_keep[i + 1], n_edge_keep[i], n_edge_keep[i + 1]);
            if (!solvable_of(o)) continue;
            int r = n_tri_keep[i];
            if (T > 0) {
                for (int k = d->v_adj_tris_offsets[o]; k < d->v_adj_tris_offsets[o + 1]; k += 2) {
                    const int t = d->v_adj_tris[k], slot = d->v_adj_tris[k + 1];
                    if (!tri_kept(t)) continue;
                    const float* mat = d->tri_materials + 5 * t;
                    const int* ti = d->tri_indices + 3 * t;
                    tri_idx[r] = make_int4(inv[ti[0]], inv[ti[1]], inv[ti[2]], slot);
                    m.tri_elem_h[r] = t;
                    const float* P = d->tri_poses + 4 * t;
                    tri_D[r] = make_float4(P[0], P[1], P[2], P[3]);
                    // (area*mu, area*lambda_nh, alpha, area*kd) with lambda_nh = lambda + mu and
                    // alpha = 1 + mu / lambda_nh (particle_vbd_kernels.py:561-565), in float32
                    const float area = d->tri_areas[t], mu = mat[0], lnh = mat[1] + mat[0];
                    const float lsafe = (lnh < 0.0f ? -1.0f : 1.0f) * std::max(std::fabs(lnh), 1.0e-6f);
                    const float alpha = 1.0f + mu / lsafe;
                    tri_mat[r] = make_float4(area * mu, area * lnh, alpha, area * mat[2]);
                    tdamp |= mat[2] > 0.0f;
                    ++r;
                }
            }
            r = n_edge_keep[i];
            if (E > 0) {
                for (int k = d->v_adj_edges_offsets[o]; k < d->v_adj_edges_offsets[o + 1]; k += 2) {
                    const int ed = d->v_adj_edges[k], slot = d->v_adj_edges[k + 1];
                    if (!edge_kept(ed)) continue;
                    const int* ei = d->edge_indices + 4 * ed;
                    const float ke = d->edge_bending_properties[2 * ed], kd = d->edge_bending_properties[2 * ed + 1];
                    edge_idx[r] = make_int4(inv[ei[0]] | (slot << 30), inv[ei[1]], inv[ei[2]], inv[ei[3]]);
                    m.edge_elem_h[r] = ed;
                    edge_mat[r] = make_float4(d->edge_rest_angle[ed], d->edge_rest_length[ed], ke, kd);
                    edamp |= kd > 0.0f;
                    ++r;
                }
            }
        }
        if (tdamp) any_tri_damp = true;
        if (edamp) any_edge_damp = true;
    });
    m.any_tri_damping = any_tri_damp.load();
    m.any_edge_damping = any_edge_damp.load();
    m.n_tri_rec = static_cast<int>(tri_idx.size());
    m.n_edge_rec = static_cast<int>(edge_idx.size());

    // ---- shapes ---------------------------------------------------------------------------
    m.shapes_host.resize(S);
    for (int s = 0; s < S; ++s) {
        const VbdShape& sh = d->shapes[s];
        if (sh.geo_type != VBD_GEO_PLANE && sh.geo_type != VBD_GEO_SPHERE && sh.geo_type != VBD_GEO_BOX)
            return fail(VBD_ERR_UNSUPPORTED, "vbd_model_create: only static plane, sphere and box shapes are supported");
        DevShape ds;
        std::memset(&ds, 0, sizeof(ds));
        // init_body_particle_contacts / _average_contact_material, in float32 like the reference
        const float ke = 0.5f * (d->soft_contact_ke + sh.material_ke);
        const float kd = 0.5f * (d->soft_contact_kd + sh.material_kd);
        const float mu = std::sqrt(d->soft_contact_mu * sh.material_mu);
        ds.mat = make_float4(ke, kd, mu, sh.margin);
        ds.pos = make_float4(sh.xform[0], sh.xform[1], sh.xform[2], static_cast<float>(sh.geo_type));
        ds.rot = make_float4(sh.xform[3], sh.xform[4], sh.xform[5], sh.xform[6]);
        ds.scale = make_float4(sh.scale[0], sh.scale[1], sh.scale[2], static_cast<float>(sh.flags));
        ds.world = sh.world;
        m.shapes_host[s] = ds;
    }

    // learned-warm-start inputs: one-ring neighbours and material features per vertex
    std::vector<int> nbr8(static_cast<size_t>(V) * 8, -1);
    std::vector<float4> vfeat(V);
    parallel_chunks(V, [&](int ib, int ie) {
        for (int i = ib; i < ie; ++i) {
            const int o = perm[i];
            int nn = 0;
            double lke = 0, lka = 0, larea = 0, lek = 0;
            int nt = 0, ne = 0;
            if (T > 0) {
                for (int k = d->v_adj_tris_offsets[o]; k < d->v_adj_tris_offsets[o + 1]; k += 2) {
                    const int t = d->v_adj_tris[k];
                    if (t < 0 || t >= T) continue;  // (records of unsolved vertices are not validated above)
                    const int* ti = d->tri_indices + 3 * t;
                    const float* mat = d->tri_materials + 5 * t;
                    lke += std::log10(std::max(mat[0], 1e-12f));
                    lka += std::log10(std::max(mat[1], 1e-12f));
                    larea += std::sqrt(2.0 * std::max(d->tri_areas[t], 0.0f));
                    ++nt;
                    for (int c = 0; c < 3; ++c) {
                        const int nb = inv[ti[c]];
                        if (ti[c] == o || nn >= 8) continue;
                        bool seen = false;
                        for (int q = 0; q < nn; ++q) seen |= nbr8[8 * i + q] == nb;
                        if (!seen) nbr8[8 * i + nn++] = nb;
                    }
                }
            }
            if (E > 0) {
                for (int k = d->v_adj_edges_offsets[o]; k < d->v_adj_edges_offsets[o + 1]; k += 2) {
                    const int e = d->v_adj_edges[k];
                    if (e < 0 || e >= E) continue;
                    lek += std::log10(std::max(d->edge_bending_properties[2 * e], 1e-12f));
                    ++ne;
                }
            }
            vfeat[i] = make_float4(nt ? float(lke / nt) : 0.f, nt ? float(lka / nt) : 0.f, ne ? float(lek / ne) : 0.f,
                                   nt ? float(larea / nt) : 1.f);
        }
    });

    std::vector<int> pworld(V, -1), pflags(V);
    std::vector<float> pradius(V);
    int W = 0;
    for (int v = 0; v < V; ++v) {
        pworld[v] = d->particle_world ? d->particle_world[v] : -1;
        pflags[v] = d->particle_flags[v];
        pradius[v] = d->particle_radius[v];
        W = std::max(W, pworld[v] + 1);
    }
    for (int s = 0; s < S; ++s) W = std::max(W, d->shapes[s].world + 1);
    // candidate shapes per particle world, in ascending shape id (the record order per particle)
    std::vector<int> wso(static_cast<size_t>(W) + 2, 0), wsl;
    for (int w = 0; w <= W; ++w) {
        for (int s = 0; s < S; ++s) {
            const int sw = d->shapes[s].world;
            if (w == W || sw == -1 || sw == w) wsl.push_back(s);
        }
        wso[w + 1] = static_cast<int>(wsl.size());
    }
    m.n_worlds = W;

    if (d->particle_q) {
        m.rest_q_h.resize(3 * static_cast<size_t>(V));
        for (int i = 0; i < V; ++i)
            for (int k = 0; k < 3; ++k) m.rest_q_h[3 * i + k] = d->particle_q[3 * perm[i] + k];
    }
    int rc;
    if ((rc = upload(&m.perm, perm))) return rc;
    if ((rc = upload(&m.inv_perm, inv))) return rc;
    if ((rc = upload(&m.pinfo, pinfo))) return rc;
    if ((rc = upload(&m.vadj, vadj))) return rc;
    if ((rc = upload(&m.tri_idx, tri_idx))) return rc;
    if ((rc = upload(&m.tri_D, tri_D))) return rc;
    if ((rc = upload(&m.tri_mat, tri_mat))) return rc;
    if ((rc = upload(&m.edge_idx, edge_idx))) return rc;
    if ((rc = upload(&m.edge_mat, edge_mat))) return rc;
    if ((rc = upload(&m.shapes, m.shapes_host))) return rc;
    if ((rc = upload(&m.particle_world, pworld))) return rc;
    if ((rc = upload(&m.particle_flags_orig, pflags))) return rc;
    if ((rc = upload(&m.particle_radius_orig, pradius))) return rc;
    if ((rc = upload(&m.world_shape_offsets, wso))) return rc;
    if ((rc = upload(&m.world_shapes, wsl))) return rc;
    if ((rc = upload(&m.nbr8, nbr8))) return rc;
    if ((rc = upload(&m.vfeat, vfeat))) return rc;
    m.tri_raw_h.assign(d->tri_indices, d->tri_indices + 3 * static_cast<size_t>(T));
    m.edge_raw_h.assign(d->edge_indices, d->edge_indices + 4 * static_cast<size_t>(E));
    if (T > 0) {
        m.adj_t_off_h.assign(d->v_adj_tris_offsets, d->v_adj_tris_offsets + V + 1);
        m.adj_t_h.assign(d->v_adj_tris, d->v_adj_tris + m.adj_t_off_h[V]);
    } else {
        m.adj_t_off_h.assign(V + 1, 0);
    }
    if (E > 0) {
        m.adj_e_off_h.assign(d->v_adj_edges_offsets, d->v_adj_edges_offsets + V + 1);
        m.adj_e_h.assign(d->v_adj_edges, d->v_adj_edges + m.adj_e_off_h[V]);
    } else {
        m.adj_e_off_h.assign(V + 1, 0);
    }
    m.pworld_h = pworld;
    m.soft_ke = d->soft_contact_ke;
    m.soft_kd = d->soft_contact_kd;
    m.soft_mu = d->soft_contact_mu;
    m.pinfo_h = std::move(pinfo);
    m.vadj_h = std::move(vadj);
    m.tri_idx_h = std::move(tri_idx);
    m.tri_D_h = std::move(tri_D);
    m.tri_mat_h = std::move(tri_mat);
    m.edge_idx_h = std::move(edge_idx);
    m.edge_mat_h = std::move(edge_mat);
    return VBD_OK;
}

// ---------------------------------------------------------------------------------------------
// Soft contacts against static shapes: restates create_soft_contacts (geometry/kernels.py:1020-1184)
// for PLANE, SPHERE and BOX with the SDFs of geometry/kernels.py:181-274 and :584-620.
// One thread per particle, shapes in model order; a particle's records are reserved as one block
// (warp-aggregated), so the records of a particle are consecutive and in shape order.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float3 quat_rotate(float4 q, float3 v) {
    const float3 u = f3(q.x, q.y, q.z);
    const float s = q.w;
    return v * (2.0f * s * s - 1.0f) + cross(u, v) * (2.0f * s) + u * (2.0f * dot(u, v));
}
__device__ __forceinline__ float sgn(float x) { return x < 0.0f ? -1.0f : 1.0f; }

__device__ __forceinline__ bool shape_sdf(const DevShape& sh, float3 x, float& d, float3& n) {
    const int type = static_cast<int>(sh.pos.w);
    if (type == VBD_GEO_SPHERE) {
        const float r = sh.scale.x;
        const float len = length(x);
        d = len - r;
        n = len > 1.0e-8f ? x * (1.0f / len) : f3(0.f, 0.f, 1.f);
        return true;
    }
    if (type == VBD_GEO_BOX) {
        const float hx = sh.scale.x, hy = sh.scale.y, hz = sh.scale.z;
        const float qx = fabsf(x.x) - hx, qy = fabsf(x.y) - hy, qz = fabsf(x.z) - hz;
        const float3 e = f3(fmaxf(qx, 0.f), fmaxf(qy, 0.f), fmaxf(qz, 0.f));
        d = length(e) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
        if (qx > 0.0f || qy > 0.0f || qz > 0.0f) {
            const float3 c = f3(fminf(fmaxf(x.x, -hx), hx), fminf(fmaxf(x.y, -hy), hy), fminf(fmaxf(x.z, -hz), hz));
            const float3 dv = x - c;
            const float l = length(dv);
            n = l > 0.0f ? dv * (1.0f / l) : f3(0.f, 0.f, 0.f);
        } else if ((qx > qy && qx > qz) || (qy == 0.0f && qz == 0.0f)) {
            n = f3(sgn(x.x), 0.f, 0.f);
        } else if ((qy > qx && qy > qz) || (qx == 0.0f && qz == 0.0f)) {
            n = f3(0.f, sgn(x.y), 0.f);
        } else {
            n = f3(0.f, 0.f, sgn(x.z));
        }
        return true;
    }
    if (type == VBD_GEO_PLANE) {
        const float w = sh.scale.x * 0.5f, l = sh.scale.y * 0.5f;
        if (w > 0.0f && l > 0.0f) {
            d = fmaxf(fmaxf(fabsf(x.x) - w, fabsf(x.y) - l), fabsf(x.z));
        } else {
            d = x.z;
        }
        n = f3(0.f, 0.f, 1.f);
        return true;
    }
    return false;
}

struct CollideArgs {
    const DevShape* shapes;
    const int* world_shape_offsets;
    const int* world_shapes;
    int S, V, W;
    const float* q;
    const float* radius;
    const int* flags;
    const int* world;
    float margin;
    VbdContacts c;
};

__device__ __forceinline__ bool shape_test(const CollideArgs& a, int s, int pw, float3 px, float radius,
                                           float3& bpos, float3& wn) {
    const DevShape sh = a.shapes[s];
    const int sflags = static_cast<int>(sh.scale.w);
    if ((sflags & VBD_SHAPE_COLLIDE_PARTICLES) == 0) return false;
    if (pw != -1 && sh.world != -1 && pw != sh.world) return false;
    const float4 q = sh.rot;
    const float4 qi = make_float4(-q.x, -q.y, -q.z, q.w);
    const float3 p = xyz(sh.pos);
    const float3 xl = quat_rotate(qi, px) + quat_rotate(qi, -p);
    float d = 1.0e6f;
    float3 n = f3(0.f, 0.f, 0.f);
    shape_sdf(sh, xl, d, n);
    if (!(d < a.margin + sh.mat.w + radius)) return false;
    bpos = quat_rotate(q, xl - n * d) + p;
    wn = quat_rotate(q, n);
    return true;
}

__global__ void collide_kernel(CollideArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < a.V;
    int n = 0;
    float3 px = f3(0.f, 0.f, 0.f);
    float radius = 0.f;
    int pw = -1;
    bool active = false;
    if (valid) {
        active = (a.flags[p] & VBD_PARTICLE_ACTIVE) != 0;
        if (active) {
            px = f3(a.q[3 * p], a.q[3 * p + 1], a.q[3 * p + 2]);
            radius = a.radius[p];
            pw = a.world ? a.world[p] : -1;
            const int row = (pw >= 0 && pw < a.W) ? pw : a.W;
            for (int k = a.world_shape_offsets[row]; k < a.world_shape_offsets[row + 1]; ++k) {
                float3 bp, wn;
                if (shape_test(a, a.world_shapes[k], pw, px, radius, bp, wn)) ++n;
            }
        }
    }
    // warp-aggregated reservation of n consecutive record slots per particle
    const unsigned lane = threadIdx.x & 31u;
    int incl = n;
    for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= static_cast<unsigned>(off)) incl += t;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(a.c.soft_contact_count, total);
    base = __shfl_sync(0xffffffffu, base, 31) + incl - n;
    if (n == 0) return;
    int k = 0;
    const int row = (pw >= 0 && pw < a.W) ? pw : a.W;
    for (int j = a.world_shape_offsets[row]; j < a.world_shape_offsets[row + 1]; ++j) {
        const int s = a.world_shapes[j];
        float3 bp, wn;
        if (!shape_test(a, s, pw, px, radius, bp, wn)) continue;
        const int idx = base + k++;
        if (idx >= a.c.soft_contact_max) continue;
        a.c.soft_contact_shape[idx] = s;
        a.c.soft_contact_body_pos[3 * idx] = bp.x;
        a.c.soft_contact_body_pos[3 * idx + 1] = bp.y;
        a.c.soft_contact_body_pos[3 * idx + 2] = bp.z;
        a.c.soft_contact_body_vel[3 * idx] = 0.f;
        a.c.soft_contact_body_vel[3 * idx + 1] = 0.f;
        a.c.soft_contact_body_vel[3 * idx + 2] = 0.f;
        a.c.soft_contact_particle[idx] = p;
        if (a.c.soft_contact_indices) {
            a.c.soft_contact_indices[3 * idx] = p;
            a.c.soft_contact_indices[3 * idx + 1] = -1;
            a.c.soft_contact_indices[3 * idx + 2] = -1;
        }
        if (a.c.soft_contact_barycentric) {
            a.c.soft_contact_barycentric[3 * idx] = 1.f;
            a.c.soft_contact_barycentric[3 * idx + 1] = 0.f;
            a.c.soft_contact_barycentric[3 * idx + 2] = 0.f;
        }
        a.c.soft_contact_normal[3 * idx] = wn.x;
        a.c.soft_contact_normal[3 * idx + 1] = wn.y;
        a.c.soft_contact_normal[3 * idx + 2] = wn.z;
    }
}

}  // namespace vbd

using namespace vbd;

extern "C" const char* vbd_last_error(void) { return g_last_error.c_str(); }

extern "C" int vbd_model_create(const VbdModelDesc* desc, VbdModel** out) {
    if (!out) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_model_create: out is NULL");
    *out = nullptr;
    VbdModel* h = new VbdModel();
    const int rc = build_model(desc, h->m);
    if (rc != VBD_OK) {
        free_model(h->m);
        delete h;
        return rc;
    }
    *out = h;
    return VBD_OK;
}

extern "C" int vbd_model_destroy(VbdModel* model) {
    if (!model) return VBD_OK;
    free_model(model->m);
    delete model;
    return VBD_OK;
}

extern "C" int vbd_collide(const VbdModel* model, const float* particle_q, float soft_contact_margin,
                           const VbdContacts* contacts, void* stream) {
    if (!model || !contacts) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_collide: NULL model or contacts");
    const VbdModelImpl& m = model->m;
    if (!contacts->soft_contact_count) return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_collide: soft_contact_count is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    VBD_CUDA_TRY(cudaMemsetAsync(contacts->soft_contact_count, 0, sizeof(int), s));
    if (m.V == 0 || m.S == 0 || contacts->soft_contact_max <= 0) return VBD_OK;
    if (!particle_q || !contacts->soft_contact_particle || !contacts->soft_contact_shape ||
        !contacts->soft_contact_body_pos || !contacts->soft_contact_body_vel || !contacts->soft_contact_normal)
        return fail(VBD_ERR_INVALID_ARGUMENT, "vbd_collide: contact record arrays missing");
    CollideArgs a;
    a.shapes = m.shapes;
    a.world_shape_offsets = m.world_shape_offsets;
    a.world_shapes = m.world_shapes;
    a.W = m.n_worlds;
    a.S = m.S;
    a.V = m.V;
    a.q = particle_q;
    a.radius = m.particle_radius_orig;
    a.flags = m.particle_flags_orig;
    a.world = m.particle_world;
    a.margin = soft_contact_margin;
    a.c = *contacts;
    const int block = 256;
    collide_kernel<<<(m.V + block - 1) / block, block, 0, s>>>(a);
    VBD_CUDA_TRY(cudaGetLastError());
    return VBD_OK;
}
