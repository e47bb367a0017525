// vbd_math.cuh -- per-element force/Hessian math of the VBD cloth sweep (device code, FP32).
//
// Each function restates one reference function of newton/_src/solvers/vbd:
//   membrane_eval      evaluate_neo_hookean_membrane_force_hessian (particle_vbd_kernels.py:502-632)
//   bending_eval       evaluate_dihedral_angle_based_bending_force_hessian (:664-816)
//   contact_eval       _eval_body_particle_contact (rigid_vbd_kernels.py:1366-1440) for a static
//                      shape, _compute_body_particle_contact_force (:1332-1362) and
//                      compute_projected_isotropic_friction (:1604-1645)
//   solve3             `if |det H| > 1e-8: disp += inverse(H) * f` (particle_vbd_kernels.py:2558-2565)
//
// Hessians are accumulated as the 6 unique entries of a symmetric 3x3 block
// (xx, xy, xz, yy, yz, zz): every term the reference adds is symmetric (identity, outer
// products v v^T), so the dropped lower triangle is bit-identical to the upper one.
//
// The bending angle derivative is evaluated only for the vertex being solved.  The reference
// forms all four dtheta/dx (each from two 3x3x3 products) and keeps one through 0/1 masks; here
// the kept one is written as
//     dtheta/dx = T2(cos (e x n1) - sin n1) + T1(-cos (e x n2) - sin n2),
//     Tj(y)     = sigma_j / |nj| * ((y - nj (nj . y)) x u_j),
// which is the same expression after expanding skew(a)^T y = y x a and the projector
// (I - n n^T) / |n|.  It is algebraically identical; results differ from the matrix form only
// by FP32 rounding.
#pragma once

#include <cuda_runtime.h>

namespace vbd {

struct Sym3 {
    float xx, xy, xz, yy, yz, zz;
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 xyz(const float4& a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }

__device__ __forceinline__ void add_outer(Sym3& h, float s, float3 a) {
    // h += s * a a^T
    const float sx = s * a.x, sy = s * a.y, sz = s * a.z;
    h.xx += sx * a.x; h.xy += sx * a.y; h.xz += sx * a.z;
    h.yy += sy * a.y; h.yz += sy * a.z; h.zz += sz * a.z;
}
__device__ __forceinline__ void add_diag(Sym3& h, float s) { h.xx += s; h.yy += s; h.zz += s; }
__device__ __forceinline__ void add(Sym3& h, const Sym3& o) {
    h.xx += o.xx; h.xy += o.xy; h.xz += o.xz; h.yy += o.yy; h.yz += o.yz; h.zz += o.zz;
}
__device__ __forceinline__ void scale(Sym3& h, float s) {
    h.xx *= s; h.xy *= s; h.xz *= s; h.yy *= s; h.yz *= s; h.zz *= s;
}
__device__ __forceinline__ float3 mul(const Sym3& h, float3 v) {
    return f3(h.xx * v.x + h.xy * v.y + h.xz * v.z,
              h.xy * v.x + h.yy * v.y + h.yz * v.z,
              h.xz * v.x + h.yz * v.y + h.zz * v.z);
}
__device__ __forceinline__ Sym3 zero_sym() { Sym3 h = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}; return h; }

// ---------------------------------------------------------------------------------------------
// Stable Neo-Hookean membrane of one triangle, force and Hessian block of vertex `order`.
// D = DmInv (row-major 00, 01, 10, 11).  mat = (area*mu, area*(lambda+mu), alpha, area*kd) with
// alpha = 1 + mu / lambda_nh, precomputed per record at model build: every term of the
// reference's force and Hessian is linear in (mu, lambda_nh, kd), so folding the final
// `* area` (particle_vbd_kernels.py:629-630) into the moduli is the same expression.
// Restates particle_vbd_kernels.py:502-632 otherwise term by term.
// ---------------------------------------------------------------------------------------------
template <bool kDamping>
__device__ __forceinline__ void membrane_eval(int order, float3 x0, float3 x1, float3 x2, float3 a0,
                                              float3 a1, float3 a2, float4 D, float4 mat, float inv_dt,
                                              float3& f, Sym3& h) {
    const float mu = mat.x, lnh = mat.y, alpha = mat.z, kd = mat.w;
    const float3 x01 = x1 - x0;
    const float3 x02 = x2 - x0;
    const float3 F0 = x01 * D.x + x02 * D.z;
    const float3 F1 = x01 * D.y + x02 * D.w;
    const float c00 = dot(F0, F0), c11 = dot(F1, F1), c01 = dot(F0, F1);
    const float js2 = fmaxf(c00 * c11 - c01 * c01, 1.0e-20f);
    const float inv_js = rsqrtf(js2);
    const float js = js2 * inv_js;
    const float3 g0 = inv_js * (c11 * F0 - c01 * F1);
    const float3 g1 = inv_js * (c00 * F1 - c01 * F0);
    const float s = lnh * (js - alpha);
    const float3 P0 = mu * F0 + s * g0;
    const float3 P1 = mu * F1 + s * g1;
    // dF/dx of the selected vertex: vertex 0 -> -(D row 0 + D row 1), vertex 1 -> D row 0, vertex 2 -> D row 1
    const float d0 = order == 0 ? -(D.x + D.z) : (order == 1 ? D.x : D.z);
    const float d1 = order == 0 ? -(D.y + D.w) : (order == 1 ? D.y : D.w);
    f = f - (P0 * d0 + P1 * d1);

    const float r = fmaxf(0.0f, s) * inv_js;
    const float cJ = lnh - r;
    const float3 dJ = g0 * d0 + g1 * d1;
    const float3 w = F1 * d0 - F0 * d1;
    const float icoef = mu * (d0 * d0 + d1 * d1) + r * (d0 * d0 * c11 + d1 * d1 * c00 - 2.0f * d0 * d1 * c01);
    add_diag(h, icoef);
    add_outer(h, cJ, dJ);
    add_outer(h, -r, w);

    if (kDamping && kd > 0.0f) {
        const float3 p01 = a1 - a0;
        const float3 p02 = a2 - a0;
        const float3 F0p = p01 * D.x + p02 * D.z;
        const float3 F1p = p01 * D.y + p02 * D.w;
        const float r00 = (c00 - dot(F0p, F0p)) * inv_dt;
        const float r01 = (c01 - dot(F0p, F1p)) * inv_dt;
        const float r11 = (c11 - dot(F1p, F1p)) * inv_dt;
        const float3 e00 = (2.0f * d0) * F0;
        const float3 e01 = d0 * F1 + d1 * F0;
        const float3 e11 = (2.0f * d1) * F1;
        const float3 fd = r00 * e00 + (2.0f * r01) * e01 + r11 * e11;
        f = f + (-kd) * fd;
        const float kdt = kd * inv_dt;
        add_outer(h, kdt, e00);
        add_outer(h, 2.0f * kdt, e01);
        add_outer(h, kdt, e11);
    }
}

// atan2 from the arctangent approximation of Abramowitz & Stegun, Handbook of Mathematical
// Functions, eq. 4.4.49 (C. Hastings): atan(x) = x (1 + a2 x^2 + ... + a16 x^16), 0 <= x <= 1,
// |error| <= 2e-8, extended to the full circle by the usual octant reduction.
__device__ __forceinline__ float atan2_as(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    if (!(mx > 0.0f)) return 0.0f;
    const float z = __fdividef(mn, mx);
    const float z2 = z * z;
    float p = 0.0028662257f;
    p = fmaf(p, z2, -0.0161657367f);
    p = fmaf(p, z2, 0.0429096138f);
    p = fmaf(p, z2, -0.0752896400f);
    p = fmaf(p, z2, 0.1065626393f);
    p = fmaf(p, z2, -0.1420889944f);
    p = fmaf(p, z2, 0.1999355085f);
    p = fmaf(p, z2, -0.3333314528f);
    p = fmaf(p, z2, 1.0f);
    float a = z * p;
    if (ay > ax) a = 1.57079632679489662f - a;
    if (x < 0.0f) a = 3.14159265358979324f - a;
    return y < 0.0f ? -a : a;
}

// ---------------------------------------------------------------------------------------------
// Dihedral-angle bending of one hinge (o0, o1, v0, v1) = (x0, x1, x2, x3); `order` selects the
// vertex.  em = (rest_angle, rest_length, ke, kd).  Restates particle_vbd_kernels.py:664-816.
// The caller has already dropped boundary hinges (o0 or o1 == -1, which the reference returns
// as exact zero) and hinges with ke <= 0 (which the reference never evaluates).
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float3 project_cross(float inv_len, float3 nh, float3 y, float3 u) {
    // (1/|n|) (I - nh nh^T) y  x  u
    const float3 p = (y - nh * dot(nh, y)) * inv_len;
    return cross(p, u);
}

// kSelect: form both projections for every order and select the result afterwards (straight-line
// code, so that the caller can interleave the evaluation of independent hinges); otherwise branch
// on the order (fewer live registers).  Both compute the same operations for a given order, so
// they give the same bits.
template <bool kDamping, bool kSelect = false>
__device__ __forceinline__ void bending_eval(int order, float3 x0, float3 x1, float3 x2, float3 x3, float3 a0,
                                             float3 a1, float3 a2, float3 a3, float4 em, float inv_dt, float3& f,
                                             Sym3& h) {
    const float eps = 1.0e-6f;
    const float3 x02 = x2 - x0;
    const float3 x03 = x3 - x0;
    const float3 x13 = x3 - x1;
    const float3 x12 = x2 - x1;
    const float3 e = x3 - x2;
    const float3 n1 = cross(x02, x03);
    const float3 n2 = cross(x13, x12);
    // |n| < eps  <=>  |n|^2 < eps^2; the unit vectors use the hardware reciprocal square root
    const float d1 = dot(n1, n1), d2 = dot(n2, n2), de = dot(e, e);
    if (d1 < eps * eps || d2 < eps * eps || de < eps * eps) return;
    const float i1 = rsqrtf(d1), i2 = rsqrtf(d2), ie = rsqrtf(de);
    const float3 n1h = n1 * i1;
    const float3 n2h = n2 * i2;
    const float3 eh = e * ie;
    const float sin_t = dot(cross(n1h, n2h), eh);
    const float cos_t = dot(n1h, n2h);
    const float theta = atan2_as(sin_t, cos_t);
    const float k = em.z * em.y;
    const float dE = k * (theta - em.x);

    // Selected dtheta/dx (see header comment).
    float3 g;
    if (kSelect) {
        //   order 0:  T1(y1) x e            order 2:  T2(y2) x x13 - T1(y1) x x03
        //   order 1: -T2(y2) x e            order 3:  T1(y1) x x02 - T2(y2) x x12
        const float3 y1 = -cos_t * cross(eh, n2h) - sin_t * n2h;
        const float3 y2 = cos_t * cross(eh, n1h) - sin_t * n1h;
        const float3 u1 = order == 0 ? e : (order == 2 ? x03 : x02);
        const float3 u2 = order == 1 ? e : (order == 2 ? x13 : x12);
        const float3 t1 = project_cross(i1, n1h, y1, u1);
        const float3 t2 = project_cross(i2, n2h, y2, u2);
        const float3 d12 = t1 - t2;
        g = order == 0 ? t1 : (order == 1 ? -t2 : (order == 2 ? -d12 : d12));
    } else if (order == 0) {
        const float3 y1 = -cos_t * cross(eh, n2h) - sin_t * n2h;
        g = project_cross(i1, n1h, y1, e);
    } else if (order == 1) {
        const float3 y2 = cos_t * cross(eh, n1h) - sin_t * n1h;
        g = -project_cross(i2, n2h, y2, e);
    } else if (order == 2) {
        const float3 y1 = -cos_t * cross(eh, n2h) - sin_t * n2h;
        const float3 y2 = cos_t * cross(eh, n1h) - sin_t * n1h;
        g = project_cross(i2, n2h, y2, x13) - project_cross(i1, n1h, y1, x03);
    } else {
        const float3 y1 = -cos_t * cross(eh, n2h) - sin_t * n2h;
        const float3 y2 = cos_t * cross(eh, n1h) - sin_t * n1h;
        g = project_cross(i1, n1h, y1, x02) - project_cross(i2, n2h, y2, x12);
    }
    f = f + (-dE) * g;
    add_outer(h, k, g);

    if (kDamping && em.w > 0.0f) {
        const float3 p02 = a2 - a0;
        const float3 p03 = a3 - a0;
        const float3 p13 = a3 - a1;
        const float3 p12 = a2 - a1;
        const float3 pe = a3 - a2;
        const float3 q1 = cross(p02, p03);
        const float3 q2 = cross(p13, p12);
        const float s1 = dot(q1, q1), s2 = dot(q2, q2), se = dot(pe, pe);
        if (s1 < eps * eps || s2 < eps * eps || se < eps * eps) return;
        const float3 q1h = q1 * rsqrtf(s1);
        const float3 q2h = q2 * rsqrtf(s2);
        const float3 qeh = pe * rsqrtf(se);
        const float theta_prev = atan2_as(dot(cross(q1h, q2h), qeh), dot(q1h, q2h));
        float dth = theta - theta_prev;
        if (dth > 3.141592653589793f) {
            dth = dth - 6.283185307179586f;
        } else if (dth < -3.141592653589793f) {
            dth = dth + 6.283185307179586f;
        }
        const float rate = dth * inv_dt;
        const float kdl = em.w * em.y;
        f = f + (-kdl * rate) * g;
        add_outer(h, kdl * inv_dt, g);
    }
}

// ---------------------------------------------------------------------------------------------
// Particle vs static-shape contact (one record).  sm = (ke, kd, mu, shape margin) of the
// shape, already mixed with the particle material as init_body_particle_contacts does
// (rigid_vbd_kernels.py:3277-3321): ke, kd arithmetic mean, mu geometric mean.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void contact_eval(float3 x, float3 x_prev, float3 bx, float3 bv, float3 n, float radius,
                                             float4 sm, float dt, float eps_u, float3& f, Sym3& h) {
    const float pen = -(dot(n, x - bx) - radius - sm.w);
    if (!(pen > 0.0f)) return;
    const float3 rel = (x - x_prev) - bv * dt;
    const float fn = pen * sm.x;
    float3 force = n * fn;
    Sym3 H = zero_sym();
    add_outer(H, sm.x, n);
    if (dot(n, rel) < 0.0f) {
        Sym3 Hd = zero_sym();
        add_outer(Hd, sm.y / dt, n);
        force = force - mul(Hd, rel);
        add(H, Hd);
    }
    // projected isotropic friction (IPC-style smoothing below eps_u)
    const float dnu = dot(n, rel);
    const float3 ut = rel - n * dnu;
    const float un = length(ut);
    if (un > 0.0f) {
        const float f1 = un > eps_u ? 1.0f / un : (-un / eps_u + 2.0f) / eps_u;
        const float sc = sm.z * fn * f1;
        force = force - sc * ut;
        add_diag(H, sc);
        add_outer(H, -sc, n);
    }
    f = f + force;
    add(h, H);
}

// Contacts of one vertex (internal index i), summed in record order: the per-vertex table holds
// up to K record ids written in arbitrary order by the scatter, so the few ids are sorted first
// (the reference's serial launch adds a particle's records in record order).
// `shape_mat(s)` returns the shape's mixed (ke, kd, mu, margin).
template <typename ShapeMat>
__device__ __forceinline__ void vertex_contacts(const int* ccount, const int* cslot, int K, int i, const int* c_shape,
                                                const float* c_body_pos, const float* c_body_vel, const float* c_normal,
                                                ShapeMat shape_mat, float3 x, float3 xp, float radius, float dt,
                                                float eps_u, float3& f, Sym3& h) {
    const int n = min(ccount[i], K);
    if (n <= 0) return;
    int ids[8];
    const int nn = min(n, 8);
    for (int k = 0; k < nn; ++k) ids[k] = cslot[i * K + k];
    for (int p = 1; p < nn; ++p) {
        const int v = ids[p];
        int q = p - 1;
        while (q >= 0 && ids[q] > v) {
            ids[q + 1] = ids[q];
            --q;
        }
        ids[q + 1] = v;
    }
    for (int k = 0; k < nn; ++k) {
        const int r = ids[k];
        const float4 sm = shape_mat(c_shape[r]);
        const float3 bx = f3(c_body_pos[3 * r], c_body_pos[3 * r + 1], c_body_pos[3 * r + 2]);
        const float3 bv = f3(c_body_vel[3 * r], c_body_vel[3 * r + 1], c_body_vel[3 * r + 2]);
        const float3 nrm = f3(c_normal[3 * r], c_normal[3 * r + 1], c_normal[3 * r + 2]);
        contact_eval(x, xp, bx, bv, nrm, radius, sm, dt, eps_u, f, h);
    }
}

// |det H| > 1e-8 -> dx = H^-1 f by adjugate / determinant; returns false when singular.
__device__ __forceinline__ bool solve3(const Sym3& H, float3 f, float3& dx) {
    const float c00 = H.yy * H.zz - H.yz * H.yz;
    const float c01 = H.yz * H.xz - H.xy * H.zz;
    const float c02 = H.xy * H.yz - H.yy * H.xz;
    const float det = H.xx * c00 + H.xy * c01 + H.xz * c02;
    if (!(fabsf(det) > 1.0e-8f)) return false;
    const float c11 = H.xx * H.zz - H.xz * H.xz;
    const float c12 = H.xz * H.xy - H.xx * H.yz;
    const float c22 = H.xx * H.yy - H.xy * H.xy;
    const float inv = 1.0f / det;
    dx = f3((c00 * f.x + c01 * f.y + c02 * f.z) * inv,
            (c01 * f.x + c11 * f.y + c12 * f.z) * inv,
            (c02 * f.x + c12 * f.y + c22 * f.z) * inv);
    return true;
}

}  // namespace vbd
