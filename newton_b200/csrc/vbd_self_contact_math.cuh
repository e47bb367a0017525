// vbd_self_contact_math.cuh -- device math of cloth self-contact (vertex-triangle and
// edge-edge), restating the reference's particle self-contact functions:
//   triangle_closest_point                 geometry/kernels.py:80-145
//   closest points of two segments         Warp builtin closest_point_edge_edge (not in the tree),
//                                          restated after Ericson, Real-Time Collision Detection 5.1.9
//   orthonormal_basis                      math/__init__.py:236-275
//   evaluate_self_contact_force_norm       solvers/vbd/particle_vbd_kernels.py:819-845
//   damp_collision                         :846-858
//   evaluate_edge_edge_contact_2_vertices  :990-1106
//   evaluate_vertex_triangle_collision_force_hessian_4_vertices  :1195-1313
//   compute_friction                       :1316-1345
//   segment_plane_intersects, the vertex-triangle / edge-edge division planes,
//   robust_edge_pair_normal, planar_truncation_t   :1864-2130
// Hessians are symmetric (outer products and T (f1 I) T^T), kept as Sym3.
#pragma once

#include "vbd_math.cuh"

namespace vbd {

__device__ __forceinline__ float clamp01f(float x) { return x < 0.f ? 0.f : (x > 1.f ? 1.f : x); }

__device__ __forceinline__ float3 triangle_closest_point(float3 a, float3 b, float3 c, float3 p, float3& bary) {
    const float3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) {
        bary = f3(1.f, 0.f, 0.f);
        return a;
    }
    const float3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.f && d4 <= d3) {
        bary = f3(0.f, 1.f, 0.f);
        return b;
    }
    const float3 cp = p - c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.f && d5 <= d6) {
        bary = f3(0.f, 0.f, 1.f);
        return c;
    }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = d1 / (d1 - d3);
        bary = f3(1.f - v, v, 0.f);
        return a + v * ab;
    }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float v = d2 / (d2 - d6);
        bary = f3(1.f - v, 0.f, v);
        return a + v * ac;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        bary = f3(0.f, 1.f - v, v);
        return b + v * (c - b);
    }
    const float denom = 1.f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    bary = f3(1.f - v - w, v, w);
    return a + v * ab + w * ac;
}

__device__ __forceinline__ void closest_edge_edge(float3 p1, float3 q1, float3 p2, float3 q2, float eps, float& s,
                                                  float& t, float& dist) {
    const float3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    if (a <= eps && e <= eps) {
        s = t = 0.f;
    } else if (a <= eps) {
        s = 0.f;
        t = clamp01f(f / e);
    } else {
        const float c = dot(d1, r);
        if (e <= eps) {
            t = 0.f;
            s = clamp01f(-c / a);
        } else {
            const float b = dot(d1, d2);
            const float denom = a * e - b * b;
            s = denom != 0.f ? clamp01f((b * f - c * e) / denom) : 0.f;
            t = (b * s + f) / e;
            if (t < 0.f) {
                t = 0.f;
                s = clamp01f(-c / a);
            } else if (t > 1.f) {
                t = 1.f;
                s = clamp01f((b - c) / a);
            }
        }
    }
    dist = length((p1 + d1 * s) - (p2 + d2 * t));
}

__device__ __forceinline__ void orthonormal_basis(float3 n, float3& b1, float3& b2) {
    if (n.z < 0.f) {
        const float a = 1.f / (1.f - n.z);
        const float b = n.x * n.y * a;
        b1 = f3(1.f - n.x * n.x * a, -b, n.x);
        b2 = f3(b, n.y * n.y * a - 1.f, -n.y);
    } else {
        const float a = 1.f / (1.f + n.z);
        const float b = -n.x * n.y * a;
        b1 = f3(1.f - n.x * n.x * a, b, -n.x);
        b2 = f3(b, 1.f - n.y * n.y * a, -n.y);
    }
}

__device__ __forceinline__ void self_contact_norm(float dis, float r, float k, float& dEdD, float& d2E) {
    const float pen = r - dis;
    const float tau = r * 0.5f;
    const float d_min = 1.0e-5f;
    if (tau > dis && dis > d_min) {
        const float k2 = tau * tau * k;
        dEdD = -k2 / dis;
        d2E = k2 / (dis * dis);
    } else if (dis <= d_min) {
        const float k2 = tau * tau * k;
        const float d_min_sq = d_min * d_min;
        dEdD = k2 * (dis - 2.f * d_min) / d_min_sq;
        d2E = k2 / d_min_sq;
    } else {
        dEdD = -k * pen;
        d2E = k;
    }
}

__device__ __forceinline__ void ipc_friction(float mu, float fn, float3 b1, float3 b2, float u0, float u1,
                                             float eps_u, float3& f, Sym3& H) {
    f = f3(0.f, 0.f, 0.f);
    H = zero_sym();
    const float un = sqrtf(u0 * u0 + u1 * u1);
    if (!(un > 0.f)) return;
    const float f1 = un > eps_u ? 1.f / un : (-un / eps_u + 2.f) / eps_u;
    const float sf = -mu * fn;
    const float w0 = f1 * u0, w1 = f1 * u1;
    f = f3((sf * b1.x) * w0 + (sf * b2.x) * w1, (sf * b1.y) * w0 + (sf * b2.y) * w1,
           (sf * b1.z) * w0 + (sf * b2.z) * w1);
    const float sh = mu * fn;
    const float t0[3] = {b1.x, b1.y, b1.z}, t1[3] = {b2.x, b2.y, b2.z};
    auto hij = [&](int i, int j) { return ((sh * t0[i]) * f1) * t0[j] + ((sh * t1[i]) * f1) * t1[j]; };
    H.xx = hij(0, 0);
    H.xy = hij(0, 1);
    H.xz = hij(0, 2);
    H.yy = hij(1, 1);
    H.yz = hij(1, 2);
    H.zz = hij(2, 2);
}

// adds the slot's share of one contact: f += cf b + damping(b) + b ff, H += b b ch + damping + b b fh
__device__ __forceinline__ void add_slot(float b, float3 cf, float d2E, float3 n, float gap_rate, float kd, float dt,
                                         float3 ff, const Sym3& fh, float3& f, Sym3& H) {
    float3 fk = cf * b;
    Sym3 hk = zero_sym();
    add_outer(hk, b * (b * d2E), n);
    float3 df = f3(0.f, 0.f, 0.f);
    float dh = 0.f;
    if (gap_rate < -1.0e-6f) {
        df = ((-kd * gap_rate) * b) * n;
        dh = ((kd / dt) * b) * b;
    }
    fk = fk + (df + b * ff);
    Sym3 extra = fh;
    scale(extra, b * b);
    add_outer(extra, dh, n);
    add(hk, extra);
    f = f + fk;
    add(H, hk);
}

// vertex p against triangle (a, b, c): adds the force / Hessian share of participant `slot`
// (0, 1, 2 = a, b, c; 3 = p).  Returns false when the pair is not within the radius.
__device__ __forceinline__ bool vt_contact_slot(float3 a, float3 b, float3 c, float3 p, float3 a0, float3 b0,
                                                float3 c0, float3 p0, int slot, float r, float ke, float kd, float mu,
                                                float eps_u, float dt, float3& f, Sym3& H) {
    float3 bary;
    const float3 cp = triangle_closest_point(a, b, c, p, bary);
    const float3 diff = p - cp;
    const float dis = length(diff);
    if (!(0.f < dis && dis < r)) return false;
    const float3 n = f3(diff.x / dis, diff.y / dis, diff.z / dis);
    float dEdD, d2E;
    self_contact_norm(dis, r, ke, dEdD, d2E);
    const float3 cf = (-dEdD) * n;
    const float3 cprev = bary.x * a0 + bary.y * b0 + bary.z * c0;
    const float3 dx = (p - p0) - (cp - cprev);
    float3 b1, b2;
    orthonormal_basis(n, b1, b2);
    float3 ff;
    Sym3 fh;
    ipc_friction(mu, -dEdD, b1, b2, dot(b1, dx), dot(b2, dx), eps_u, ff, fh);
    const float gap_rate = dot(n, dx) / dt;
    const float bs = slot == 0 ? -bary.x : (slot == 1 ? -bary.y : (slot == 2 ? -bary.z : 1.f));
    add_slot(bs, cf, d2E, n, gap_rate, kd, dt, ff, fh, f, H);
    return true;
}

// edge (e0, e1) against edge (g0, g1): adds the share of endpoint `slot` (0 = e0, 1 = e1)
__device__ __forceinline__ bool ee_contact_slot(float3 e0, float3 e1, float3 g0, float3 g1, float3 e0a, float3 e1a,
                                                float3 g0a, float3 g1a, int slot, float r, float ke, float kd, float mu,
                                                float eps_u, float dt, float par_eps, float3& f, Sym3& H) {
    float s, t, dis;
    closest_edge_edge(e0, e1, g0, g1, par_eps, s, t, dis);
    if (!(0.f < dis && dis < r)) return false;
    const float3 c1 = e0 + (e1 - e0) * s, c2 = g0 + (g1 - g0) * t;
    const float3 diff = c1 - c2;
    const float3 n = f3(diff.x / dis, diff.y / dis, diff.z / dis);
    float dEdD, d2E;
    self_contact_norm(dis, r, ke, dEdD, d2E);
    const float3 cf = (-dEdD) * n;
    const float3 c1p = e0a + (e1a - e0a) * s, c2p = g0a + (g1a - g0a) * t;
    const float3 dx = (c1 - c1p) - (c2 - c2p);
    float3 b1, b2;
    orthonormal_basis(n, b1, b2);
    float3 ff;
    Sym3 fh;
    ipc_friction(mu, -dEdD, b1, b2, dot(b1, dx), dot(b2, dx), eps_u, ff, fh);
    const float gap_rate = dot(n, dx) / dt;
    add_slot(slot == 0 ? 1.f - s : s, cf, d2E, n, gap_rate, kd, dt, ff, fh, f, H);
    return true;
}

__device__ __forceinline__ bool segment_plane_intersects(float3 v, float3 dv, float3 n, float3 d, float eps_par,
                                                         float eps_near, float eps_far) {
    const float nv = dot(n, dv);
    const float num = -dot(n, v - d);
    if (fabsf(nv) < eps_par) return false;
    const float t = num / nv;
    return t >= eps_near && t <= 1.f + eps_far;
}

__device__ __forceinline__ float3 normalized3(float3 a) {
    const float l = length(a);
    return f3(a.x / l, a.y / l, a.z / l);
}

// vertex-triangle division plane; dummy bits: 1 = v, 2 = t1, 4 = t2, 8 = t3
__device__ __forceinline__ int vt_plane(float3 v, float3 dv, float3 t1, float3 dt1, float3 t2, float3 dt2, float3 t3,
                                        float3 dt3, float3& n, float3& d) {
    float3 bary;
    const float3 cp = triangle_closest_point(t1, t2, t3, v, bary);
    const float3 nh = v - cp;
    if (length(nh) < 1e-12f) {
        n = f3(0.f, 0.f, 0.f);
        d = v;
        return 0;
    }
    n = normalized3(nh);
    const float dvn = fmaxf(-dot(n, dv), 0.f);
    const float dtn = fmaxf(fmaxf(dot(n, dt1), dot(n, dt2)), fmaxf(dot(n, dt3), 0.f));
    if (dtn + dvn == 0.f) {
        d = cp + 0.5f * nh;
    } else {
        float l = dtn / (dtn + dvn);
        l = l < 0.05f ? 0.05f : (l > 0.95f ? 0.95f : l);
        d = cp + l * nh;
    }
    int dummy = 0;
    if (dvn == 0.f || !segment_plane_intersects(v, dv, n, d, 1e-6f, -1e-8f, 1e-8f)) dummy |= 1;
    if (dtn == 0.f) {
        dummy |= 2 | 4 | 8;
    } else {
        if (!segment_plane_intersects(t1, dt1, n, d, 1e-6f, -1e-8f, 1e-8f)) dummy |= 2;
        if (!segment_plane_intersects(t2, dt2, n, d, 1e-6f, -1e-8f, 1e-8f)) dummy |= 4;
        if (!segment_plane_intersects(t3, dt3, n, d, 1e-6f, -1e-8f, 1e-8f)) dummy |= 8;
    }
    return dummy;
}

__device__ __forceinline__ float3 robust_edge_pair_normal(float3 a0, float3 a1, float3 b0, float3 b1) {
    const float eps = 1.0e-6f;
    float3 d0 = a1 - a0, d1 = b1 - b0;
    const float l0 = length(d0), l1 = length(d1);
    d0 = l0 > eps ? f3(d0.x / l0, d0.y / l0, d0.z / l0) : f3(0.f, 0.f, 0.f);
    d1 = l1 > eps ? f3(d1.x / l1, d1.y / l1, d1.z / l1) : f3(0.f, 0.f, 0.f);
    float3 n = cross(d0, d1);
    float ln = length(n);
    if (ln > eps) return f3(n.x / ln, n.y / ln, n.z / ln);
    float3 ref = d0;
    if (length(ref) <= eps) ref = d1;
    if (length(ref) <= eps) return f3(1.f, 0.f, 0.f);
    const float3 bridge = 0.5f * ((b0 + b1) - (a0 + a1));
    const float bl = length(bridge);
    if (bl > eps) {
        n = cross(ref, f3(bridge.x / bl, bridge.y / bl, bridge.z / bl));
        ln = length(n);
        if (ln > eps) return f3(n.x / ln, n.y / ln, n.z / ln);
    }
    float3 axis = f3(1.f, 0.f, 0.f);
    if (fabsf(dot(ref, axis)) > 0.9f) axis = f3(0.f, 1.f, 0.f);
    n = cross(ref, axis);
    ln = length(n);
    if (ln > eps) return f3(n.x / ln, n.y / ln, n.z / ln);
    n = cross(ref, f3(0.f, 0.f, 1.f));
    ln = length(n);
    if (ln > eps) return f3(n.x / ln, n.y / ln, n.z / ln);
    return f3(1.f, 0.f, 0.f);
}

// edge-edge division plane; dummy bits: 1 = a0, 2 = a1, 4 = b0, 8 = b1
__device__ __forceinline__ int ee_plane(float3 a0, float3 da0, float3 a1, float3 da1, float3 b0, float3 db0, float3 b1,
                                        float3 db1, float3& n, float3& d) {
    float s, t, dist;
    closest_edge_edge(a0, a1, b0, b1, 1e-6f, s, t, dist);
    const float3 c1 = a0 + (a1 - a0) * s, c2 = b0 + (b1 - b0) * t;
    const float3 nh = c1 - c2;
    if (length(nh) < 1e-12f) {
        n = robust_edge_pair_normal(a0, a1, b0, b1);
        d = c1 * 0.5f + c2 * 0.5f;
        return 0;
    }
    n = normalized3(nh);
    const float de0 = fmaxf(fmaxf(-dot(n, da0), -dot(n, da1)), 0.f);
    const float de1 = fmaxf(fmaxf(dot(n, db0), dot(n, db1)), 0.f);
    if (de0 + de1 == 0.f) {
        d = c2 + 0.5f * nh;
    } else {
        float l = de1 / (de1 + de0);
        l = l < 0.05f ? 0.05f : (l > 0.95f ? 0.95f : l);
        d = c2 + l * nh;
    }
    int dummy = 0;
    if (de0 == 0.f) {
        dummy |= 1 | 2;
    } else {
        if (!segment_plane_intersects(a0, da0, n, d, 1e-6f, -1e-8f, 1e-6f)) dummy |= 1;
        if (!segment_plane_intersects(a1, da1, n, d, 1e-6f, -1e-8f, 1e-6f)) dummy |= 2;
    }
    if (de1 == 0.f) {
        dummy |= 4 | 8;
    } else {
        if (!segment_plane_intersects(b0, db0, n, d, 1e-6f, -1e-8f, 1e-6f)) dummy |= 4;
        if (!segment_plane_intersects(b1, db1, n, d, 1e-6f, -1e-8f, 1e-6f)) dummy |= 8;
    }
    return dummy;
}

__device__ __forceinline__ float planar_truncation_t(float3 v, float3 dv, float3 n, float3 d, float eps, float gamma) {
    const float denom = dot(n, dv);
    if (fabsf(denom) < eps) return 1.f;
    float t = dot(n, d - v) / denom;
    if (t < 0.f) return 1.f;
    t = fminf(t * gamma, t - 1e-3f);
    return clamp01f(t);
}

}  // namespace vbd
