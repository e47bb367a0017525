// vbd_oracle.cpp -- CPU restatement of Newton's particle VBD cloth step.  TEST INFRASTRUCTURE:
// used only by tests/, the smoke check and bench.py's CPU-baseline leg, as the checker of the
// CUDA library -- never as the product path.
//
// It follows the reference's *serial* CPU path (the one Warp's CPU device runs,
// particle_enable_tile_solve is ignored on CPU, solver_vbd.py:565-568), function by function:
//   forward_step                particle_vbd_kernels.py:1350-1375
//   apply_truncation_ts         particle_vbd_kernels.py:2266-2286 (no self-contact: t = 1, max = inf)
//   solve_elasticity            particle_vbd_kernels.py:2568-2706 (inertia, triangles in CSR order,
//                               hinges in CSR order, + accumulated contact force/Hessian, det check)
//   membrane                    evaluate_neo_hookean_membrane_force_hessian :502-632
//   bending                     evaluate_dihedral_angle_based_bending_force_hessian :635-816, forming
//                               all four dtheta/dx and selecting one with 0/1 masks, as the reference does
//   contact accumulation        accumulate_particle_body_contact_force_and_hessian :2289-2401 (serial
//                               over records, in record order, only records of the current color)
//   contact law                 rigid_vbd_kernels.py:1332-1362, :1366-1440, :1604-1645
//   contact material            init_body_particle_contacts rigid_vbd_kernels.py:3277-3321 (+ :799-815)
//   update_velocity             particle_vbd_kernels.py:1468-1471
//   step orchestration          solver_vbd.py:1774-1825, :2065-2100, :2516-2704, :3158-3169
//   soft-contact generation     create_soft_contacts geometry/kernels.py:1020-1184 (plane, sphere, box)
// The 3x3 inverse (Warp's wp.inverse, third-party) is restated as adjugate / determinant.
//
// Templated on the scalar: the float instantiation is the FP32 oracle, the double one is the
// "FP64 re-evaluation" of the same step.  Compiled with -ffp-contract=off so the FP32 result
// does not depend on whether the host compiler fuses multiply-adds.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

struct OracleShape {
    int32_t geo_type, flags, world, reserved;
    float xform[7];
    float scale[3];
    float margin, material_ke, material_kd, material_mu;
};

struct OracleModelDesc {
    int32_t particle_count, tri_count, edge_count, shape_count, color_count, reserved;
    const float* particle_mass;
    const float* particle_inv_mass;
    const float* particle_radius;
    const int32_t* particle_flags;
    const int32_t* particle_world;
    const int32_t* tri_indices;
    const float* tri_poses;
    const float* tri_materials;
    const float* tri_areas;
    const int32_t* edge_indices;
    const float* edge_rest_angle;
    const float* edge_rest_length;
    const float* edge_bending_properties;
    const int32_t* v_adj_tris_offsets;
    const int32_t* v_adj_tris;
    const int32_t* v_adj_edges_offsets;
    const int32_t* v_adj_edges;
    const int32_t* color_group_offsets;
    const int32_t* color_group_particles;
    float gravity[3];
    float soft_contact_ke, soft_contact_kd, soft_contact_mu;
    const OracleShape* shapes;
};

}  // extern "C"

namespace {

template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T>
V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T>
V3<T> operator+(V3<T> a, V3<T> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T>
V3<T> operator-(V3<T> a, V3<T> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T>
V3<T> operator-(V3<T> a) { return v3(-a.x, -a.y, -a.z); }
template <typename T>
V3<T> operator*(V3<T> a, T s) { return v3(a.x * s, a.y * s, a.z * s); }
template <typename T>
V3<T> operator*(T s, V3<T> a) { return v3(s * a.x, s * a.y, s * a.z); }
template <typename T>
V3<T> operator/(V3<T> a, T s) { return v3(a.x / s, a.y / s, a.z / s); }
template <typename T>
T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
V3<T> cross(V3<T> a, V3<T> b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
template <typename T>
T len(V3<T> a) { return std::sqrt(dot(a, a)); }

template <typename T>
struct M3 {
    T m[3][3];
};
template <typename T>
M3<T> zero3() {
    M3<T> r;
    std::memset(&r, 0, sizeof(r));
    return r;
}
template <typename T>
M3<T> eye3() {
    M3<T> r = zero3<T>();
    r.m[0][0] = r.m[1][1] = r.m[2][2] = T(1);
    return r;
}
template <typename T>
M3<T> operator+(const M3<T>& a, const M3<T>& b) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] + b.m[i][j];
    return r;
}
template <typename T>
M3<T> operator-(const M3<T>& a, const M3<T>& b) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] - b.m[i][j];
    return r;
}
template <typename T>
M3<T> operator*(T s, const M3<T>& a) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = s * a.m[i][j];
    return r;
}
template <typename T>
M3<T> operator*(const M3<T>& a, const M3<T>& b) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}
template <typename T>
V3<T> operator*(const M3<T>& a, V3<T> v) {
    return v3(a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z, a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
              a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z);
}
template <typename T>
M3<T> transpose(const M3<T>& a) {
    M3<T> r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
    return r;
}
template <typename T>
M3<T> outer(V3<T> a, V3<T> b) {
    M3<T> r;
    const T av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = av[i] * bv[j];
    return r;
}
template <typename T>
M3<T> skew(V3<T> a) {
    M3<T> r = zero3<T>();
    r.m[0][1] = -a.z;
    r.m[0][2] = a.y;
    r.m[1][0] = a.z;
    r.m[1][2] = -a.x;
    r.m[2][0] = -a.y;
    r.m[2][1] = a.x;
    return r;
}
template <typename T>
T det3(const M3<T>& a) {
    return a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
           a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
           a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
}
// textbook inverse: adjugate / determinant
template <typename T>
M3<T> inverse3(const M3<T>& a) {
    const T d = det3(a);
    M3<T> adj;
    adj.m[0][0] = a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1];
    adj.m[0][1] = a.m[0][2] * a.m[2][1] - a.m[0][1] * a.m[2][2];
    adj.m[0][2] = a.m[0][1] * a.m[1][2] - a.m[0][2] * a.m[1][1];
    adj.m[1][0] = a.m[1][2] * a.m[2][0] - a.m[1][0] * a.m[2][2];
    adj.m[1][1] = a.m[0][0] * a.m[2][2] - a.m[0][2] * a.m[2][0];
    adj.m[1][2] = a.m[0][2] * a.m[1][0] - a.m[0][0] * a.m[1][2];
    adj.m[2][0] = a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0];
    adj.m[2][1] = a.m[0][1] * a.m[2][0] - a.m[0][0] * a.m[2][1];
    adj.m[2][2] = a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0];
    return (T(1) / d) * adj;
}

template <typename T>
V3<T> load3(const T* p, int i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
template <typename T>
void store3(T* p, int i, V3<T> v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
template <typename T>
T sign(T x) { return x < T(0) ? T(-1) : T(1); }

// ---- element laws ------------------------------------------------------------------------
template <typename T>
void membrane(int face, int v_order, const T* pos, const T* anchor, const int32_t* tri, const T* pose, T area, T mu,
              T lmbd, T damping, T dt, V3<T>& force, M3<T>& hessian) {
    const int v0 = tri[3 * face], v1 = tri[3 * face + 1], v2 = tri[3 * face + 2];
    const V3<T> x0 = load3(pos, v0);
    const V3<T> x01 = load3(pos, v1) - x0;
    const V3<T> x02 = load3(pos, v2) - x0;
    const T D00 = pose[0], D01 = pose[1], D10 = pose[2], D11 = pose[3];
    const V3<T> f0 = x01 * D00 + x02 * D10;
    const V3<T> f1 = x01 * D01 + x02 * D11;
    const T a = dot(f0, f0), b = dot(f1, f1), c = dot(f0, f1);
    T js2 = a * b - c * c;
    js2 = std::max(js2, T(1.0e-20));
    const T js = std::sqrt(js2);
    const T inv_js = T(1) / js;
    const T mu_nh = mu;
    const T l_nh = lmbd + mu;
    const T l_safe = sign(l_nh) * std::max(std::fabs(l_nh), T(1.0e-6));
    const T alpha = T(1) + mu_nh / l_safe;
    const V3<T> g0 = inv_js * (b * f0 - c * f1);
    const V3<T> g1 = inv_js * (a * f1 - c * f0);
    const T s = l_nh * (js - alpha);
    const V3<T> P0 = mu_nh * f0 + s * g0;
    const V3<T> P1 = mu_nh * f1 + s * g1;
    const T m0 = v_order == 0 ? T(1) : T(0), m1 = v_order == 1 ? T(1) : T(0), m2 = v_order == 2 ? T(1) : T(0);
    const T df0 = D00 * (m1 - m0) + D10 * (m2 - m0);
    const T df1 = D01 * (m1 - m0) + D11 * (m2 - m0);
    force = -(P0 * df0 + P1 * df1);
    const T r = std::max(T(0), s) * inv_js;
    const T c1 = l_nh - r;
    const V3<T> dJ = g0 * df0 + g1 * df1;
    const V3<T> w = f1 * df0 - f0 * df1;
    const T icoef = mu_nh * (df0 * df0 + df1 * df1) + r * (df0 * df0 * b + df1 * df1 * a - T(2) * df0 * df1 * c);
    hessian = (icoef * eye3<T>() + c1 * outer(dJ, dJ)) - r * outer(w, w);
    if (damping > T(0)) {
        const T inv_dt = T(1) / dt;
        const V3<T> p0 = load3(anchor, v0);
        const V3<T> p01 = load3(anchor, v1) - p0;
        const V3<T> p02 = load3(anchor, v2) - p0;
        const V3<T> f0p = p01 * D00 + p02 * D10;
        const V3<T> f1p = p01 * D01 + p02 * D11;
        const T r00 = (a - dot(f0p, f0p)) * inv_dt;
        const T r01 = (c - dot(f0p, f1p)) * inv_dt;
        const T r11 = (b - dot(f1p, f1p)) * inv_dt;
        const V3<T> e00 = (T(2) * df0) * f0;
        const V3<T> e01 = df0 * f1 + df1 * f0;
        const V3<T> e11 = (T(2) * df1) * f1;
        const V3<T> fd = (r00 * e00 + (T(2) * r01) * e01) + r11 * e11;
        force = force + (-damping) * fd;
        hessian = hessian + (damping * inv_dt) * ((outer(e00, e00) + T(2) * outer(e01, e01)) + outer(e11, e11));
    }
    force = force * area;
    hessian = area * hessian;
}

template <typename T>
M3<T> norm_vec_derivative(T n_len, V3<T> n_hat, const M3<T>& dn) {
    return ((T(1) / n_len) * (eye3<T>() - outer(n_hat, n_hat))) * dn;
}

template <typename T>
V3<T> angle_derivative(V3<T> n1h, V3<T> n2h, V3<T> eh, const M3<T>& dn1, const M3<T>& dn2, T sin_t, T cos_t,
                       const M3<T>& sk1, const M3<T>& sk2) {
    const V3<T> dsin = transpose(sk1 * dn2 - sk2 * dn1) * eh;
    const V3<T> dcos = transpose(dn1) * n2h + transpose(dn2) * n1h;
    return dsin * cos_t - dcos * sin_t;
}

template <typename T>
void bending(int e, int v_order, const T* pos, const T* anchor, const int32_t* ei, const T* rest_angle,
             const T* rest_length, T stiffness, T damping, T dt, V3<T>& force, M3<T>& hessian) {
    force = v3(T(0), T(0), T(0));
    hessian = zero3<T>();
    if (ei[4 * e] == -1 || ei[4 * e + 1] == -1) return;
    const T eps = T(1.0e-6);
    const int i0 = ei[4 * e], i1 = ei[4 * e + 1], i2 = ei[4 * e + 2], i3 = ei[4 * e + 3];
    const V3<T> x0 = load3(pos, i0), x1 = load3(pos, i1), x2 = load3(pos, i2), x3 = load3(pos, i3);
    const V3<T> x02 = x2 - x0, x03 = x3 - x0, x13 = x3 - x1, x12 = x2 - x1, ev = x3 - x2;
    const V3<T> n1 = cross(x02, x03), n2 = cross(x13, x12);
    const T n1n = len(n1), n2n = len(n2), en = len(ev);
    if (n1n < eps || n2n < eps || en < eps) return;
    const V3<T> n1h = n1 / n1n, n2h = n2 / n2n, eh = ev / en;
    const T sin_t = dot(cross(n1h, n2h), eh);
    const T cos_t = dot(n1h, n2h);
    const T theta = std::atan2(sin_t, cos_t);
    const T k = stiffness * rest_length[e];
    const T dE = k * (theta - rest_angle[e]);
    const M3<T> sk_e = skew(ev), sk_x03 = skew(x03), sk_x02 = skew(x02), sk_x13 = skew(x13), sk_x12 = skew(x12);
    const M3<T> sk1 = skew(n1h), sk2 = skew(n2h);
    const M3<T> Z = zero3<T>();
    const M3<T> dn1_0 = norm_vec_derivative(n1n, n1h, sk_e), dn2_0 = Z;
    const M3<T> dn1_1 = Z, dn2_1 = norm_vec_derivative(n2n, n2h, T(-1) * sk_e);
    const M3<T> dn1_2 = norm_vec_derivative(n1n, n1h, T(-1) * sk_x03), dn2_2 = norm_vec_derivative(n2n, n2h, sk_x13);
    const M3<T> dn1_3 = norm_vec_derivative(n1n, n1h, sk_x02), dn2_3 = norm_vec_derivative(n2n, n2h, T(-1) * sk_x12);
    const V3<T> d0 = angle_derivative(n1h, n2h, eh, dn1_0, dn2_0, sin_t, cos_t, sk1, sk2);
    const V3<T> d1 = angle_derivative(n1h, n2h, eh, dn1_1, dn2_1, sin_t, cos_t, sk1, sk2);
    const V3<T> d2 = angle_derivative(n1h, n2h, eh, dn1_2, dn2_2, sin_t, cos_t, sk1, sk2);
    const V3<T> d3 = angle_derivative(n1h, n2h, eh, dn1_3, dn2_3, sin_t, cos_t, sk1, sk2);
    const T m0 = v_order == 0 ? T(1) : T(0), m1 = v_order == 1 ? T(1) : T(0);
    const T m2 = v_order == 2 ? T(1) : T(0), m3 = v_order == 3 ? T(1) : T(0);
    const V3<T> g = ((d0 * m0 + d1 * m1) + d2 * m2) + d3 * m3;
    force = (-dE) * g;
    hessian = k * outer(g, g);
    if (damping > T(0)) {
        const T inv_dt = T(1) / dt;
        const V3<T> a0 = load3(anchor, i0), a1 = load3(anchor, i1), a2 = load3(anchor, i2), a3 = load3(anchor, i3);
        const V3<T> p02 = a2 - a0, p03 = a3 - a0, p13 = a3 - a1, p12 = a2 - a1, pe = a3 - a2;
        const V3<T> q1 = cross(p02, p03), q2 = cross(p13, p12);
        const T q1n = len(q1), q2n = len(q2), qen = len(pe);
        if (q1n < eps || q2n < eps || qen < eps) return;
        const V3<T> q1h = q1 / q1n, q2h = q2 / q2n, qeh = pe / qen;
        const T theta_prev = std::atan2(dot(cross(q1h, q2h), qeh), dot(q1h, q2h));
        T dth = theta - theta_prev;
        if (dth > T(3.141592653589793)) {
            dth = dth - T(6.283185307179586);
        } else if (dth < T(-3.141592653589793)) {
            dth = dth + T(6.283185307179586);
        }
        const T rate = dth * inv_dt;
        const T L0 = rest_length[e];
        force = force + ((-damping) * L0 * rate) * g;
        hessian = hessian + (damping * L0 * inv_dt) * outer(g, g);
    }
}

// _compute_body_particle_contact_force + compute_projected_isotropic_friction
template <typename T>
void contact_force(T pen, V3<T> n, V3<T> rel, T ke, T kd, T mu, T friction_eps, T dt, V3<T>& f, M3<T>& H) {
    const T fn = pen * ke;
    f = n * fn;
    H = ke * outer(n, n);
    if (dot(n, rel) < T(0)) {
        const M3<T> Hd = (kd / dt) * outer(n, n);
        H = H + Hd;
        f = f - Hd * rel;
    }
    const T eps_u = friction_eps * dt;
    const T dnu = dot(n, rel);
    const V3<T> ut = rel - n * dnu;
    const T un = len(ut);
    if (un > T(0)) {
        const T f1 = un > eps_u ? T(1) / un : (-un / eps_u + T(2)) / eps_u;
        const T sc = mu * fn * f1;
        f = f + (-(sc * ut));
        H = H + sc * (eye3<T>() - outer(n, n));
    }
}

// _eval_body_particle_contact for a static shape (body = -1, no body_q_prev).
template <typename T>
void contact(V3<T> x, V3<T> xp, V3<T> bpos, V3<T> bvel, V3<T> n, T radius, T margin, T ke, T kd, T mu, T feps, T dt,
             V3<T>& f, M3<T>& H) {
    f = v3(T(0), T(0), T(0));
    H = zero3<T>();
    const V3<T> bx = bpos;
    const T pen = -(dot(n, x - bx) - radius - margin);
    if (pen > T(0)) {
        const V3<T> dx = x - xp;
        const V3<T> bv = bvel;
        const V3<T> rel = dx - bv * dt;
        contact_force(pen, n, rel, ke, kd, mu, feps, dt, f, H);
    }
}

// ---- soft contact generation (static plane / sphere / box) -------------------------------
template <typename T>
V3<T> quat_rotate(const T q[4], V3<T> v) {
    const V3<T> u = v3(q[0], q[1], q[2]);
    const T s = q[3];
    return (v * (T(2) * s * s - T(1)) + cross(u, v) * (T(2) * s)) + u * (T(2) * dot(u, v));
}

template <typename T>
bool sdf_test(const OracleShape& sh, V3<T> px, T radius, T margin, V3<T>& bpos, V3<T>& wn) {
    const T q[4] = {T(sh.xform[3]), T(sh.xform[4]), T(sh.xform[5]), T(sh.xform[6])};
    const T qi[4] = {-q[0], -q[1], -q[2], q[3]};
    const V3<T> p = v3(T(sh.xform[0]), T(sh.xform[1]), T(sh.xform[2]));
    const V3<T> x = quat_rotate(qi, px) + quat_rotate(qi, -p);
    T d = T(1.0e6);
    V3<T> n = v3(T(0), T(0), T(0));
    if (sh.geo_type == 3) {
        const T r = T(sh.scale[0]);
        const T l = len(x);
        d = l - r;
        n = l > T(1.0e-8) ? x / l : v3(T(0), T(0), T(1));
    } else if (sh.geo_type == 7) {
        const T hx = sh.scale[0], hy = sh.scale[1], hz = sh.scale[2];
        const T qx = std::fabs(x.x) - hx, qy = std::fabs(x.y) - hy, qz = std::fabs(x.z) - hz;
        const V3<T> e = v3(std::max(qx, T(0)), std::max(qy, T(0)), std::max(qz, T(0)));
        d = len(e) + std::min(std::max(qx, std::max(qy, qz)), T(0));
        if (qx > T(0) || qy > T(0) || qz > T(0)) {
            const V3<T> c = v3(std::min(std::max(x.x, -hx), hx), std::min(std::max(x.y, -hy), hy),
                               std::min(std::max(x.z, -hz), hz));
            const V3<T> dv = x - c;
            const T l = len(dv);
            n = l > T(0) ? dv / l : v3(T(0), T(0), T(0));
        } else if ((qx > qy && qx > qz) || (qy == T(0) && qz == T(0))) {
            n = v3(sign(x.x), T(0), T(0));
        } else if ((qy > qx && qy > qz) || (qx == T(0) && qz == T(0))) {
            n = v3(T(0), sign(x.y), T(0));
        } else {
            n = v3(T(0), T(0), sign(x.z));
        }
    } else if (sh.geo_type == 1) {
        const T w = T(sh.scale[0]) * T(0.5), l = T(sh.scale[1]) * T(0.5);
        if (w > T(0) && l > T(0)) {
            d = std::max(std::max(std::fabs(x.x) - w, std::fabs(x.y) - l), std::fabs(x.z));
        } else {
            d = x.z;
        }
        n = v3(T(0), T(0), T(1));
    } else {
        return false;
    }
    if (!(d < margin + T(sh.margin) + radius)) return false;
    bpos = quat_rotate(q, x - n * d) + p;
    wn = quat_rotate(q, n);
    return true;
}

// ---- solver state ------------------------------------------------------------------------
template <typename T>
struct Oracle {
    int V = 0, Tn = 0, E = 0, S = 0, C = 0;
    std::vector<T> mass, inv_mass, radius;
    std::vector<int32_t> flags, world, tri, adj_t, adj_t_off, edges, adj_e, adj_e_off, color_off, color_par, colors;
    std::vector<T> poses, tri_mat, areas, rest_angle, rest_len, bend;
    std::vector<OracleShape> shapes;
    std::vector<T> shape_ke, shape_kd, shape_mu;  // mixed per shape (init_body_particle_contacts)
    T g[3] = {0, 0, 0};
    T friction_eps = T(1e-2);
    // scratch
    std::vector<T> q, q_prev, inertia, disp, pos_prev_cd, pf, ph;
    // contacts (reference record layout, per step)
    int ncontacts = 0;
    std::vector<int32_t> c_particle, c_shape;
    std::vector<T> c_body_pos, c_body_vel, c_normal;
    int threads = 1;
};

template <typename T>
void init_oracle(Oracle<T>& o, const OracleModelDesc* d) {
    o.V = d->particle_count;
    o.Tn = d->tri_count;
    o.E = d->edge_count;
    o.S = d->shape_count;
    o.C = d->color_count;
    const int V = o.V;
    o.mass.assign(d->particle_mass, d->particle_mass + V);
    o.inv_mass.assign(d->particle_inv_mass, d->particle_inv_mass + V);
    o.radius.assign(d->particle_radius, d->particle_radius + V);
    o.flags.assign(d->particle_flags, d->particle_flags + V);
    o.world.assign(V, -1);
    if (d->particle_world) o.world.assign(d->particle_world, d->particle_world + V);
    o.tri.assign(d->tri_indices, d->tri_indices + 3 * o.Tn);
    o.poses.assign(d->tri_poses, d->tri_poses + 4 * o.Tn);
    o.tri_mat.assign(d->tri_materials, d->tri_materials + 5 * o.Tn);
    o.areas.assign(d->tri_areas, d->tri_areas + o.Tn);
    o.edges.assign(d->edge_indices, d->edge_indices + 4 * o.E);
    o.rest_angle.assign(d->edge_rest_angle, d->edge_rest_angle + o.E);
    o.rest_len.assign(d->edge_rest_length, d->edge_rest_length + o.E);
    o.bend.assign(d->edge_bending_properties, d->edge_bending_properties + 2 * o.E);
    if (o.Tn > 0) {
        o.adj_t_off.assign(d->v_adj_tris_offsets, d->v_adj_tris_offsets + V + 1);
        o.adj_t.assign(d->v_adj_tris, d->v_adj_tris + o.adj_t_off[V]);
    } else {
        o.adj_t_off.assign(V + 1, 0);
    }
    if (o.E > 0) {
        o.adj_e_off.assign(d->v_adj_edges_offsets, d->v_adj_edges_offsets + V + 1);
        o.adj_e.assign(d->v_adj_edges, d->v_adj_edges + o.adj_e_off[V]);
    } else {
        o.adj_e_off.assign(V + 1, 0);
    }
    o.color_off.assign(d->color_group_offsets, d->color_group_offsets + o.C + 1);
    o.color_par.assign(d->color_group_particles, d->color_group_particles + o.color_off[o.C]);
    o.colors.assign(V, -1);
    for (int c = 0; c < o.C; ++c)
        for (int k = o.color_off[c]; k < o.color_off[c + 1]; ++k) o.colors[o.color_par[k]] = c;
    o.shapes.assign(d->shapes, d->shapes + o.S);
    o.shape_ke.resize(o.S);
    o.shape_kd.resize(o.S);
    o.shape_mu.resize(o.S);
    for (int s = 0; s < o.S; ++s) {
        // _average_contact_material in float32, as the reference kernel computes it
        const float ke = 0.5f * (d->soft_contact_ke + o.shapes[s].material_ke);
        const float kd = 0.5f * (d->soft_contact_kd + o.shapes[s].material_kd);
        const float mu = std::sqrt(d->soft_contact_mu * o.shapes[s].material_mu);
        o.shape_ke[s] = T(ke);
        o.shape_kd[s] = T(kd);
        o.shape_mu[s] = T(mu);
    }
    for (int k = 0; k < 3; ++k) o.g[k] = T(d->gravity[k]);
    o.q.assign(3 * V, T(0));
    o.q_prev = o.q;
    o.inertia = o.q;
    o.disp = o.q;
    o.pos_prev_cd = o.q;
    o.pf = o.q;
    o.ph.assign(9 * V, T(0));
}

template <typename T>
void forward(Oracle<T>& o, const float* q_in, const float* qd_in, const float* f_ext, T dt) {
    const int V = o.V;
    for (int i = 0; i < 3 * V; ++i) o.q[i] = T(q_in[i]);
    o.pos_prev_cd = o.q;                       // pos_prev_collision_detection.assign(state_in.q)
    std::fill(o.disp.begin(), o.disp.end(), T(0));
    for (int p = 0; p < V; ++p) {              // forward_step
        const V3<T> x = load3(o.q.data(), p);
        store3(o.q_prev.data(), p, x);
        if (!(o.flags[p] & 1) || o.inv_mass[p] == T(0)) {
            store3(o.inertia.data(), p, x);
            store3(o.disp.data(), p, v3(T(0), T(0), T(0)));
            continue;
        }
        const V3<T> v = v3(T(qd_in[3 * p]), T(qd_in[3 * p + 1]), T(qd_in[3 * p + 2]));
        V3<T> fe = v3(T(0), T(0), T(0));
        if (f_ext) fe = v3(T(f_ext[3 * p]), T(f_ext[3 * p + 1]), T(f_ext[3 * p + 2]));
        const V3<T> vn = v + (v3(o.g[0], o.g[1], o.g[2]) + fe * o.inv_mass[p]) * dt;
        store3(o.inertia.data(), p, x + vn * dt);
        store3(o.disp.data(), p, vn * dt);
    }
    for (int p = 0; p < V; ++p)                // apply_truncation_ts (t = 1, max = inf)
        store3(o.q.data(), p, load3(o.pos_prev_cd.data(), p) + load3(o.disp.data(), p));
}

template <typename T>
void accumulate_contacts(Oracle<T>& o, int color, T dt) {
    for (int r = 0; r < o.ncontacts; ++r) {
        const int p = o.c_particle[r];
        if (o.colors[p] != color) continue;
        const int s = o.c_shape[r];
        V3<T> f;
        M3<T> H;
        contact(load3(o.q.data(), p), load3(o.q_prev.data(), p), load3(o.c_body_pos.data(), r),
                load3(o.c_body_vel.data(), r), load3(o.c_normal.data(), r), o.radius[p], T(o.shapes[s].margin),
                o.shape_ke[s], o.shape_kd[s], o.shape_mu[s], o.friction_eps, dt, f, H);
        store3(o.pf.data(), p, load3(o.pf.data(), p) + f);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) o.ph[9 * p + 3 * a + b] += H.m[a][b];
    }
}

// solve_elasticity for one vertex; returns the total force and Hessian (before the solve)
template <typename T>
void vertex_force(const Oracle<T>& o, int p, T dt, V3<T>& f, M3<T>& h) {
    const T dtsr = T(1) / (dt * dt);
    const V3<T> x = load3(o.q.data(), p);
    f = (o.mass[p] * (load3(o.inertia.data(), p) - x)) * dtsr;
    h = (o.mass[p] * dtsr) * eye3<T>();
    if (o.Tn > 0) {
        for (int k = o.adj_t_off[p]; k < o.adj_t_off[p + 1]; k += 2) {
            const int t = o.adj_t[k], slot = o.adj_t[k + 1];
            const T* mat = o.tri_mat.data() + 5 * t;
            if (mat[0] > T(0) || mat[1] > T(0)) {
                V3<T> ft;
                M3<T> ht;
                membrane(t, slot, o.q.data(), o.q_prev.data(), o.tri.data(), o.poses.data() + 4 * t, o.areas[t], mat[0],
                         mat[1], mat[2], dt, ft, ht);
                f = f + ft;
                h = h + ht;
            }
        }
    }
    if (o.E > 0) {
        for (int k = o.adj_e_off[p]; k < o.adj_e_off[p + 1]; k += 2) {
            const int e = o.adj_e[k], slot = o.adj_e[k + 1];
            if (o.bend[2 * e] > T(0)) {
                V3<T> fe;
                M3<T> he;
                bending(e, slot, o.q.data(), o.q_prev.data(), o.edges.data(), o.rest_angle.data(), o.rest_len.data(),
                        o.bend[2 * e], o.bend[2 * e + 1], dt, fe, he);
                f = f + fe;
                h = h + he;
            }
        }
    }
    M3<T> pc;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) pc.m[a][b] = o.ph[9 * p + 3 * a + b];
    h = h + pc;
    f = f + load3(o.pf.data(), p);
}

template <typename T>
void sweep_color(Oracle<T>& o, int color, T dt) {
    accumulate_contacts(o, color, dt);
    const int b = o.color_off[color], e = o.color_off[color + 1];
#pragma omp parallel for schedule(static) num_threads(o.threads) if (o.threads > 1)
    for (int k = b; k < e; ++k) {
        const int p = o.color_par[k];
        if (!(o.flags[p] & 1) || o.mass[p] == T(0)) {
            store3(o.disp.data(), p, v3(T(0), T(0), T(0)));
            continue;
        }
        V3<T> f;
        M3<T> h;
        vertex_force(o, p, dt, f, h);
        if (std::fabs(det3(h)) > T(1.0e-8)) {
            const M3<T> hi = inverse3(h);
            store3(o.disp.data(), p, load3(o.disp.data(), p) + hi * f);
        }
    }
    // apply_truncation_ts over all particles
#pragma omp parallel for schedule(static) num_threads(o.threads) if (o.threads > 1)
    for (int p = 0; p < o.V; ++p) store3(o.q.data(), p, load3(o.pos_prev_cd.data(), p) + load3(o.disp.data(), p));
}

template <typename T>
void begin_iteration(Oracle<T>& o) {
    std::fill(o.pf.begin(), o.pf.end(), T(0));
    std::fill(o.ph.begin(), o.ph.end(), T(0));
}

template <typename T>
void finalize(Oracle<T>& o, float* q_in, float* q_out, float* qd_out, T dt) {
    for (int p = 0; p < o.V; ++p) {
        const V3<T> x = load3(o.q.data(), p);
        const V3<T> v = (x - load3(o.q_prev.data(), p)) / dt;
        for (int k = 0; k < 3; ++k) {
            const T xv = k == 0 ? x.x : (k == 1 ? x.y : x.z);
            const T vv = k == 0 ? v.x : (k == 1 ? v.y : v.z);
            if (q_in) q_in[3 * p + k] = float(xv);
            if (q_out) q_out[3 * p + k] = float(xv);
            if (qd_out) qd_out[3 * p + k] = float(vv);
        }
    }
}

template <typename T>
void set_contacts(Oracle<T>& o, int count, const int32_t* particle, const int32_t* shape, const float* body_pos,
                  const float* body_vel, const float* normal) {
    o.ncontacts = count;
    o.c_particle.assign(particle, particle + count);
    o.c_shape.assign(shape, shape + count);
    o.c_body_pos.resize(3 * count);
    o.c_body_vel.resize(3 * count);
    o.c_normal.resize(3 * count);
    for (int i = 0; i < 3 * count; ++i) {
        o.c_body_pos[i] = T(body_pos[i]);
        o.c_body_vel[i] = T(body_vel[i]);
        o.c_normal[i] = T(normal[i]);
    }
}

template <typename T>
void residual(Oracle<T>& o, T dt, float* per_vertex) {
    // contact forces at the current iterate for every vertex (all colors at once)
    std::fill(o.pf.begin(), o.pf.end(), T(0));
    std::fill(o.ph.begin(), o.ph.end(), T(0));
    for (int c = 0; c < o.C; ++c) accumulate_contacts(o, c, dt);
    const T gn = std::sqrt(o.g[0] * o.g[0] + o.g[1] * o.g[1] + o.g[2] * o.g[2]);
#pragma omp parallel for schedule(static) num_threads(o.threads) if (o.threads > 1)
    for (int p = 0; p < o.V; ++p) {
        if (!(o.flags[p] & 1) || o.mass[p] == T(0) || o.colors[p] < 0) {
            per_vertex[p] = 0.f;
            continue;
        }
        V3<T> f;
        M3<T> h;
        vertex_force(o, p, dt, f, h);
        per_vertex[p] = float(len(f) / (o.mass[p] * gn));
    }
}

}  // namespace

// ---- C ABI (ctypes) ----------------------------------------------------------------------
extern "C" {

struct OracleHandle {
    int is_double;
    void* impl;
};

OracleHandle* oracle_create(const OracleModelDesc* d, int is_double, float friction_epsilon, int threads) {
    OracleHandle* h = new OracleHandle();
    h->is_double = is_double;
    if (is_double) {
        auto* o = new Oracle<double>();
        init_oracle(*o, d);
        o->friction_eps = friction_epsilon;
        o->threads = threads;
        h->impl = o;
    } else {
        auto* o = new Oracle<float>();
        init_oracle(*o, d);
        o->friction_eps = friction_epsilon;
        o->threads = threads;
        h->impl = o;
    }
    return h;
}

void oracle_destroy(OracleHandle* h) {
    if (!h) return;
    if (h->is_double) delete static_cast<Oracle<double>*>(h->impl);
    else delete static_cast<Oracle<float>*>(h->impl);
    delete h;
}

#define ORACLE_DISPATCH(h, call)                                   \
    do {                                                           \
        if ((h)->is_double) {                                      \
            auto& o = *static_cast<Oracle<double>*>((h)->impl);    \
            using T = double;                                      \
            (void)sizeof(T);                                       \
            call;                                                  \
        } else {                                                   \
            auto& o = *static_cast<Oracle<float>*>((h)->impl);     \
            using T = float;                                       \
            (void)sizeof(T);                                       \
            call;                                                  \
        }                                                          \
    } while (0)

void oracle_set_threads(OracleHandle* h, int threads) { ORACLE_DISPATCH(h, o.threads = threads); }

void oracle_set_contacts(OracleHandle* h, int count, const int32_t* particle, const int32_t* shape,
                         const float* body_pos, const float* body_vel, const float* normal) {
    ORACLE_DISPATCH(h, set_contacts(o, count, particle, shape, body_pos, body_vel, normal));
}

void oracle_forward(OracleHandle* h, const float* q_in, const float* qd_in, const float* f_ext, float dt) {
    ORACLE_DISPATCH(h, forward(o, q_in, qd_in, f_ext, T(dt)));
}

void oracle_begin_iteration(OracleHandle* h) { ORACLE_DISPATCH(h, begin_iteration(o)); }

void oracle_sweep_color(OracleHandle* h, int color, float dt) { ORACLE_DISPATCH(h, sweep_color(o, color, T(dt))); }

void oracle_finalize(OracleHandle* h, float* q_in, float* q_out, float* qd_out, float dt) {
    ORACLE_DISPATCH(h, finalize(o, q_in, q_out, qd_out, T(dt)));
}

// SolverVBD.step: forward, `iterations` x (zero contact accumulators, all colors), finalize.
void oracle_step(OracleHandle* h, float* q_in, const float* qd_in, const float* f_ext, float* q_out, float* qd_out,
                 float dt, int iterations) {
    ORACLE_DISPATCH(h, {
        forward(o, q_in, qd_in, f_ext, T(dt));
        for (int it = 0; it < iterations; ++it) {
            begin_iteration(o);
            for (int c = 0; c < o.C; ++c) sweep_color(o, c, T(dt));
        }
        finalize(o, q_in, q_out, qd_out, T(dt));
    });
}

void oracle_get_positions(OracleHandle* h, double* out) {
    ORACLE_DISPATCH(h, {
        for (int i = 0; i < 3 * o.V; ++i) out[i] = double(o.q[i]);
    });
}

// Overwrite the current Gauss-Seidel iterate (e.g. with another implementation's positions).
void oracle_set_positions(OracleHandle* h, const float* q) {
    ORACLE_DISPATCH(h, {
        for (int i = 0; i < 3 * o.V; ++i) o.q[i] = T(q[i]);
    });
}

void oracle_residual(OracleHandle* h, float dt, float* per_vertex) { ORACLE_DISPATCH(h, residual(o, T(dt), per_vertex)); }

// Element-level entry points (used by the known-answer tests).
void oracle_membrane(int is_double, int face, int v_order, const double* pos, const double* anchor,
                     const int32_t* tri, const double* pose, double area, double mu, double lmbd, double damping,
                     double dt, int npos, double* f_out, double* h_out) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        std::vector<T> p(pos, pos + 3 * npos), a(anchor, anchor + 3 * npos);
        const T ps[4] = {T(pose[0]), T(pose[1]), T(pose[2]), T(pose[3])};
        V3<T> f;
        M3<T> H;
        membrane<T>(face, v_order, p.data(), a.data(), tri, ps, T(area), T(mu), T(lmbd), T(damping), T(dt), f, H);
        f_out[0] = f.x;
        f_out[1] = f.y;
        f_out[2] = f.z;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) h_out[3 * i + j] = H.m[i][j];
    };
    if (is_double) run(double(0));
    else run(float(0));
}

void oracle_bending(int is_double, int edge, int v_order, const double* pos, const double* anchor, const int32_t* ei,
                    double rest_angle, double rest_length, double ke, double kd, double dt, int npos, double* f_out,
                    double* h_out) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        std::vector<T> p(pos, pos + 3 * npos), a(anchor, anchor + 3 * npos);
        std::vector<T> ra(edge + 1, T(rest_angle)), rl(edge + 1, T(rest_length));
        V3<T> f;
        M3<T> H;
        bending<T>(edge, v_order, p.data(), a.data(), ei, ra.data(), rl.data(), T(ke), T(kd), T(dt), f, H);
        f_out[0] = f.x;
        f_out[1] = f.y;
        f_out[2] = f.z;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) h_out[3 * i + j] = H.m[i][j];
    };
    if (is_double) run(double(0));
    else run(float(0));
}

void oracle_contact(int is_double, const double* x, const double* xp, const double* bpos, const double* bvel,
                    const double* n, double radius, double margin, double ke, double kd, double mu, double feps,
                    double dt, double* f_out, double* h_out) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        V3<T> f;
        M3<T> H;
        contact<T>(v3(T(x[0]), T(x[1]), T(x[2])), v3(T(xp[0]), T(xp[1]), T(xp[2])),
                   v3(T(bpos[0]), T(bpos[1]), T(bpos[2])), v3(T(bvel[0]), T(bvel[1]), T(bvel[2])),
                   v3(T(n[0]), T(n[1]), T(n[2])), T(radius), T(margin), T(ke), T(kd), T(mu), T(feps), T(dt), f, H);
        f_out[0] = f.x;
        f_out[1] = f.y;
        f_out[2] = f.z;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) h_out[3 * i + j] = H.m[i][j];
    };
    if (is_double) run(double(0));
    else run(float(0));
}

// create_soft_contacts over static shapes, serial in (particle, shape) order: returns the number
// of records written (records of one particle consecutive, in shape order).
int oracle_collide(int V, const float* q, const float* radius, const int32_t* flags, const int32_t* world, int S,
                   const OracleShape* shapes, float margin, int max_out, int32_t* particle, int32_t* shape,
                   float* body_pos, float* body_vel, float* normal) {
    int n = 0;
    for (int p = 0; p < V; ++p) {
        if (!(flags[p] & 1)) continue;
        const V3<float> px = v3(q[3 * p], q[3 * p + 1], q[3 * p + 2]);
        const int pw = world ? world[p] : -1;
        for (int s = 0; s < S; ++s) {
            if (!(shapes[s].flags & 4)) continue;
            if (pw != -1 && shapes[s].world != -1 && pw != shapes[s].world) continue;
            V3<float> bp, wn;
            if (!sdf_test<float>(shapes[s], px, radius[p], margin, bp, wn)) continue;
            if (n < max_out) {
                particle[n] = p;
                shape[n] = s;
                body_pos[3 * n] = bp.x;
                body_pos[3 * n + 1] = bp.y;
                body_pos[3 * n + 2] = bp.z;
                body_vel[3 * n] = body_vel[3 * n + 1] = body_vel[3 * n + 2] = 0.f;
                normal[3 * n] = wn.x;
                normal[3 * n + 1] = wn.y;
                normal[3 * n + 2] = wn.z;
            }
            ++n;
        }
    }
    return n;
}

}  // extern "C"
