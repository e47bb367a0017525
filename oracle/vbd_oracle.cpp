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
//   self-contact (optional)     detection: vertex_triangle_collision_detection_kernel geometry/kernels.py:1328,
//                               edge_colliding_edges_detection_kernel :1499, n-ring filters
//                               solvers/vbd/tri_mesh_collision.py:123-233 (brute force here, all pairs);
//                               forces: evaluate_self_contact_force_norm particle_vbd_kernels.py:819,
//                               damp_collision :846, evaluate_edge_edge_contact_2_vertices :990,
//                               evaluate_vertex_triangle_collision_force_hessian_4_vertices :1195,
//                               compute_friction :1316; truncation: :1864-2286
//                               (apply_planar_truncation_parallel_by_collision + apply_truncation_ts);
//                               orchestration solver_vbd.py:2003-2063, :2540-2545, :3221-3237;
//                               triangle_closest_point geometry/kernels.py:80-145;
//                               orthonormal_basis math/__init__.py:236-275.  Warp's builtin
//                               closest_point_edge_edge (not in the tree) is restated after Ericson,
//                               Real-Time Collision Detection, 5.1.9.  Per vertex the self-contact
//                               terms are summed in a fixed order (own vertex-triangle pairs, then
//                               incident triangles' pairs, then incident edges' pairs); the reference
//                               adds them with atomics in no fixed order.
// The 3x3 inverse (Warp's wp.inverse, third-party) is restated as adjugate / determinant.
//
// Templated on the scalar: the float instantiation is the FP32 oracle, the double one is the
// "FP64 re-evaluation" of the same step.  Compiled with -ffp-contract=off so the FP32 result
// does not depend on whether the host compiler fuses multiply-adds.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <tuple>
#include <queue>

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

struct OracleSelfContact {
    int32_t enabled;
    float radius, margin, relaxation;
    int32_t vertex_buffer, edge_buffer, interval;
    float edge_parallel_epsilon;
    int32_t filter_threshold;
    float rest_exclusion_radius;
    const float* rest_q;  // [3V] rest positions (the exclusion radius is measured there); may be NULL
    // external filter maps as CSR (ascending rows; may be NULL): vertex -> triangles, edge -> edges
    const int32_t* vertex_filter_offsets;
    const int32_t* vertex_filter_triangles;
    const int32_t* edge_filter_offsets;
    const int32_t* edge_filter_edges;
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
    float soft_ke = 0.f, soft_kd = 0.f, soft_mu = 0.f;  // model.soft_contact_* (self-contact material)
    // scratch
    std::vector<T> q, q_prev, inertia, disp, pos_prev_cd, pf, ph;
    // Gauss-Seidel residual of the last sweep of each vertex: |f| / (m |g|) at its visit
    std::vector<float> gs_r;
    // contacts (reference record layout, per step)
    int ncontacts = 0;
    std::vector<int32_t> c_particle, c_shape;
    std::vector<T> c_body_pos, c_body_vel, c_normal;
    int threads = 1;
    int iteration = 0;  // iterations begun since the last forward
    // self-contact
    OracleSelfContact sc{};
    std::vector<T> rest_q;
    std::vector<int32_t> near_off, near;        // vertices within (threshold-1) rings, sorted, self excluded
    std::vector<int32_t> vt_count, vt_list;     // per vertex: colliding triangles (ascending), stride vertex_buffer
    std::vector<int32_t> ee_count, ee_list;     // per edge: colliding edges (ascending), stride edge_buffer
    std::vector<std::vector<int32_t>> tri_vs;   // per triangle: vertices that collide with it (ascending)
    std::vector<int32_t> vfilt_off, vfilt, efilt_off, efilt;  // external filter maps (CSR)
    long long sc_overflow = 0;
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
    o.soft_ke = d->soft_contact_ke;
    o.soft_kd = d->soft_contact_kd;
    o.soft_mu = d->soft_contact_mu;
    o.q.assign(3 * V, T(0));
    o.q_prev = o.q;
    o.inertia = o.q;
    o.disp = o.q;
    o.pos_prev_cd = o.q;
    o.pf = o.q;
    o.gs_r.assign(static_cast<size_t>(o.V), 0.f);
    o.ph.assign(9 * V, T(0));
}

// ---- self-contact --------------------------------------------------------------------------
template <typename T>
T clamp01(T x) { return x < T(0) ? T(0) : (x > T(1) ? T(1) : x); }

// triangle_closest_point (geometry/kernels.py:80-145): closest point of triangle abc to p and
// its barycentric coordinates (Ericson's Voronoi-region walk).
template <typename T>
V3<T> triangle_closest_point(V3<T> a, V3<T> b, V3<T> c, V3<T> p, V3<T>& bary) {
    const V3<T> ab = b - a, ac = c - a, ap = p - a;
    const T d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= T(0) && d2 <= T(0)) {
        bary = v3(T(1), T(0), T(0));
        return a;
    }
    const V3<T> bp = p - b;
    const T d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= T(0) && d4 <= d3) {
        bary = v3(T(0), T(1), T(0));
        return b;
    }
    const V3<T> cp = p - c;
    const T d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= T(0) && d5 <= d6) {
        bary = v3(T(0), T(0), T(1));
        return c;
    }
    const T vc = d1 * d4 - d3 * d2;
    if (vc <= T(0) && d1 >= T(0) && d3 <= T(0)) {
        const T v = d1 / (d1 - d3);
        bary = v3(T(1) - v, v, T(0));
        return a + v * ab;
    }
    const T vb = d5 * d2 - d1 * d6;
    if (vb <= T(0) && d2 >= T(0) && d6 <= T(0)) {
        const T v = d2 / (d2 - d6);
        bary = v3(T(1) - v, T(0), v);
        return a + v * ac;
    }
    const T va = d3 * d6 - d5 * d4;
    if (va <= T(0) && (d4 - d3) >= T(0) && (d5 - d6) >= T(0)) {
        const T v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        bary = v3(T(0), T(1) - v, v);
        return b + v * (c - b);
    }
    const T denom = T(1) / (va + vb + vc);
    const T v = vb * denom, w = vc * denom;
    bary = v3(T(1) - v - w, v, w);
    return a + v * ab + w * ac;
}

// Closest points of segments p1q1 and p2q2 (Ericson, Real-Time Collision Detection, 5.1.9):
// s, t along the segments and the distance between the two points.  eps bounds degenerate
// (point-like) segments; parallel segments (zero denominator) take s = 0.
template <typename T>
void closest_edge_edge(V3<T> p1, V3<T> q1, V3<T> p2, V3<T> q2, T eps, T& s, T& t, T& dist) {
    const V3<T> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const T a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    if (a <= eps && e <= eps) {
        s = t = T(0);
    } else if (a <= eps) {
        s = T(0);
        t = clamp01(f / e);
    } else {
        const T c = dot(d1, r);
        if (e <= eps) {
            t = T(0);
            s = clamp01(-c / a);
        } else {
            const T b = dot(d1, d2);
            const T denom = a * e - b * b;
            s = denom != T(0) ? clamp01((b * f - c * e) / denom) : T(0);
            t = (b * s + f) / e;
            if (t < T(0)) {
                t = T(0);
                s = clamp01(-c / a);
            } else if (t > T(1)) {
                t = T(1);
                s = clamp01((b - c) / a);
            }
        }
    }
    dist = len((p1 + d1 * s) - (p2 + d2 * t));
}

// orthonormal_basis (math/__init__.py:236-275)
template <typename T>
void orthonormal_basis(V3<T> n, V3<T>& b1, V3<T>& b2) {
    if (n.z < T(0)) {
        const T a = T(1) / (T(1) - n.z);
        const T b = n.x * n.y * a;
        b1 = v3(T(1) - n.x * n.x * a, -b, n.x);
        b2 = v3(b, n.y * n.y * a - T(1), -n.y);
    } else {
        const T a = T(1) / (T(1) + n.z);
        const T b = -n.x * n.y * a;
        b1 = v3(T(1) - n.x * n.x * a, b, -n.x);
        b2 = v3(b, T(1) - n.y * n.y * a, -n.y);
    }
}

// evaluate_self_contact_force_norm (particle_vbd_kernels.py:819-845): linear penalty for
// d in [tau, r), log barrier in (1e-5, tau), its quadratic Taylor extension below 1e-5.
template <typename T>
void self_contact_norm(T dis, T r, T k, T& dEdD, T& d2E) {
    const T pen = r - dis;
    const T tau = r * T(0.5);
    const T d_min = T(1.0e-5);
    if (tau > dis && dis > d_min) {
        const T k2 = tau * tau * k;
        dEdD = -k2 / dis;
        d2E = k2 / (dis * dis);
    } else if (dis <= d_min) {
        const T k2 = tau * tau * k;
        const T d_min_sq = d_min * d_min;
        dEdD = k2 * (dis - T(2) * d_min) / d_min_sq;
        d2E = k2 / d_min_sq;
    } else {
        dEdD = -k * pen;
        d2E = k;
    }
}

// compute_friction (:1316-1345): IPC-smoothed friction in the tangent frame T = [b1 b2]
template <typename T>
void ipc_friction(T mu, T fn, V3<T> b1, V3<T> b2, T u0, T u1, T eps_u, V3<T>& f, M3<T>& H) {
    const T un = std::sqrt(u0 * u0 + u1 * u1);
    f = v3(T(0), T(0), T(0));
    H = zero3<T>();
    if (!(un > T(0))) return;
    const T f1 = un > eps_u ? T(1) / un : (-un / eps_u + T(2)) / eps_u;
    const T sf = -mu * fn;
    const T w0 = f1 * u0, w1 = f1 * u1;
    const T Tm[3][2] = {{b1.x, b2.x}, {b1.y, b2.y}, {b1.z, b2.z}};
    T fv[3];
    for (int i = 0; i < 3; ++i) fv[i] = (sf * Tm[i][0]) * w0 + (sf * Tm[i][1]) * w1;
    f = v3(fv[0], fv[1], fv[2]);
    const T sh = mu * fn;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) H.m[i][j] = ((sh * Tm[i][0]) * f1) * Tm[j][0] + ((sh * Tm[i][1]) * f1) * Tm[j][1];
}

// damp_collision (:846-858): damping on the contact's gap rate, only while the gap closes
template <typename T>
void damp_collision(T gap_rate, T b, V3<T> n, T kd, T dt, V3<T>& f, M3<T>& H) {
    if (gap_rate < T(-1.0e-6)) {
        f = ((-kd * gap_rate) * b) * n;
        H = (((kd / dt) * b) * b) * outer(n, n);
    } else {
        f = v3(T(0), T(0), T(0));
        H = zero3<T>();
    }
}

// evaluate_vertex_triangle_collision_force_hessian_4_vertices (:1195-1313): vertex p against
// triangle (a, b, c); outputs for a, b, c, p (indices 0..3).
template <typename T>
bool vt_contact(V3<T> a, V3<T> b, V3<T> c, V3<T> p, V3<T> a0, V3<T> b0, V3<T> c0, V3<T> p0, T r, T ke, T kd, T mu,
                T feps, T dt, V3<T> F[4], M3<T> H[4]) {
    V3<T> bary;
    const V3<T> cp = triangle_closest_point(a, b, c, p, bary);
    const V3<T> diff = p - cp;
    const T dis = len(diff);
    const V3<T> n = diff / dis;
    if (!(T(0) < dis && dis < r)) return false;
    const T bs[4] = {-bary.x, -bary.y, -bary.z, T(1)};
    T dEdD, d2E;
    self_contact_norm(dis, r, ke, dEdD, d2E);
    const V3<T> cf = (-dEdD) * n;
    const M3<T> ch = d2E * outer(n, n);
    const V3<T> dxv = p - p0;
    const V3<T> cprev = bary.x * a0 + bary.y * b0 + bary.z * c0;
    const V3<T> dx = dxv - (cp - cprev);
    V3<T> b1, b2;
    orthonormal_basis(n, b1, b2);
    V3<T> ff;
    M3<T> fh;
    ipc_friction(mu, -dEdD, b1, b2, dot(b1, dx), dot(b2, dx), feps * dt, ff, fh);
    const T gap_rate = dot(n, dx) / dt;
    for (int k = 0; k < 4; ++k) {
        F[k] = cf * bs[k];
        H[k] = bs[k] * (bs[k] * ch);
        V3<T> df;
        M3<T> dh;
        damp_collision(gap_rate, bs[k], n, kd, dt, df, dh);
        F[k] = F[k] + (df + bs[k] * ff);
        H[k] = H[k] + (dh + (bs[k] * bs[k]) * fh);
    }
    return true;
}

// evaluate_edge_edge_contact_2_vertices (:990-1106): edge (e0, e1) against edge (f0, f1);
// outputs for e0, e1.
template <typename T>
bool ee_contact(V3<T> e0, V3<T> e1, V3<T> f0, V3<T> f1, V3<T> e0a, V3<T> e1a, V3<T> f0a, V3<T> f1a, T r, T ke, T kd,
                T mu, T feps, T dt, T par_eps, V3<T> F[2], M3<T> H[2]) {
    T s, t, dis;
    closest_edge_edge(e0, e1, f0, f1, par_eps, s, t, dis);
    const V3<T> c1 = e0 + (e1 - e0) * s, c2 = f0 + (f1 - f0) * t;
    const V3<T> n = (c1 - c2) / dis;
    if (!(T(0) < dis && dis < r)) return false;
    const T bs[2] = {T(1) - s, s};
    T dEdD, d2E;
    self_contact_norm(dis, r, ke, dEdD, d2E);
    const V3<T> cf = (-dEdD) * n;
    const M3<T> ch = d2E * outer(n, n);
    const V3<T> c1p = e0a + (e1a - e0a) * s, c2p = f0a + (f1a - f0a) * t;
    const V3<T> dx = (c1 - c1p) - (c2 - c2p);
    V3<T> b1, b2;
    orthonormal_basis(n, b1, b2);
    V3<T> ff;
    M3<T> fh;
    ipc_friction(mu, -dEdD, b1, b2, dot(b1, dx), dot(b2, dx), feps * dt, ff, fh);
    const T gap_rate = dot(n, dx) / dt;
    for (int k = 0; k < 2; ++k) {
        F[k] = cf * bs[k];
        H[k] = bs[k] * (bs[k] * ch);
        V3<T> df;
        M3<T> dh;
        damp_collision(gap_rate, bs[k], n, kd, dt, df, dh);
        F[k] = F[k] + (df + bs[k] * ff);
        H[k] = H[k] + (dh + (bs[k] * bs[k]) * fh);
    }
    return true;
}

// segment_plane_intersects (:1865-1887)
template <typename T>
bool segment_plane_intersects(V3<T> v, V3<T> dv, V3<T> n, V3<T> d, T eps_par, T eps_near, T eps_far) {
    const T nv = dot(n, dv);
    const T num = -dot(n, v - d);
    if (std::fabs(nv) < eps_par) return false;
    const T t = num / nv;
    return t >= eps_near && t <= T(1) + eps_far;
}

template <typename T>
V3<T> normalized(V3<T> a) {
    return a / len(a);
}

// create_vertex_triangle_division_plane_closest_pt (:1890-1947): plane n.(x - d) = 0 between
// vertex v and triangle t, n towards the vertex; dummy[k] marks a participant the plane does not
// stop (order v, t1, t2, t3).  Returns false for a degenerate (touching) pair.
template <typename T>
void vt_plane(V3<T> v, V3<T> dv, V3<T> t1, V3<T> dt1, V3<T> t2, V3<T> dt2, V3<T> t3, V3<T> dt3, bool dummy[4],
              V3<T>& n, V3<T>& d) {
    V3<T> bary;
    const V3<T> cp = triangle_closest_point(t1, t2, t3, v, bary);
    const V3<T> nh = v - cp;
    if (len(nh) < T(1e-12)) {
        for (int k = 0; k < 4; ++k) dummy[k] = false;
        n = v3(T(0), T(0), T(0));
        d = v;
        return;
    }
    n = normalized(nh);
    const T dvn = std::max(-dot(n, dv), T(0));
    const T dtn = std::max(std::max(dot(n, dt1), dot(n, dt2)), std::max(dot(n, dt3), T(0)));
    if (dtn + dvn == T(0)) {
        d = cp + T(0.5) * nh;
    } else {
        T l = dtn / (dtn + dvn);
        l = l < T(0.05) ? T(0.05) : (l > T(0.95) ? T(0.95) : l);
        d = cp + l * nh;
    }
    dummy[0] = dvn == T(0) ? true : !segment_plane_intersects(v, dv, n, d, T(1e-6), T(-1e-8), T(1e-8));
    if (dtn == T(0)) {
        dummy[1] = dummy[2] = dummy[3] = true;
    } else {
        dummy[1] = !segment_plane_intersects(t1, dt1, n, d, T(1e-6), T(-1e-8), T(1e-8));
        dummy[2] = !segment_plane_intersects(t2, dt2, n, d, T(1e-6), T(-1e-8), T(1e-8));
        dummy[3] = !segment_plane_intersects(t3, dt3, n, d, T(1e-6), T(-1e-8), T(1e-8));
    }
}

// robust_edge_pair_normal (:1951-2016)
template <typename T>
V3<T> robust_edge_pair_normal(V3<T> a0, V3<T> a1, V3<T> b0, V3<T> b1) {
    const T eps = T(1.0e-6);
    V3<T> d0 = a1 - a0, d1 = b1 - b0;
    const T l0 = len(d0), l1 = len(d1);
    d0 = l0 > eps ? d0 / l0 : v3(T(0), T(0), T(0));
    d1 = l1 > eps ? d1 / l1 : v3(T(0), T(0), T(0));
    V3<T> n = cross(d0, d1);
    T ln = len(n);
    if (ln > eps) return n / ln;
    V3<T> ref = d0;
    if (len(ref) <= eps) ref = d1;
    if (len(ref) <= eps) return v3(T(1), T(0), T(0));
    const V3<T> bridge = T(0.5) * ((b0 + b1) - (a0 + a1));
    const T bl = len(bridge);
    if (bl > eps) {
        n = cross(ref, bridge / bl);
        ln = len(n);
        if (ln > eps) return n / ln;
    }
    V3<T> axis = v3(T(1), T(0), T(0));
    if (std::fabs(dot(ref, axis)) > T(0.9)) axis = v3(T(0), T(1), T(0));
    n = cross(ref, axis);
    ln = len(n);
    if (ln > eps) return n / ln;
    n = cross(ref, v3(T(0), T(0), T(1)));
    ln = len(n);
    if (ln > eps) return n / ln;
    return v3(T(1), T(0), T(0));
}

// create_edge_edge_division_plane_closest_pt (:2020-2090); order e0v0, e0v1, e1v0, e1v1
template <typename T>
void ee_plane(V3<T> a0, V3<T> da0, V3<T> a1, V3<T> da1, V3<T> b0, V3<T> db0, V3<T> b1, V3<T> db1, bool dummy[4],
              V3<T>& n, V3<T>& d) {
    T s, t, dist;
    closest_edge_edge(a0, a1, b0, b1, T(1e-6), s, t, dist);
    const V3<T> c1 = a0 + (a1 - a0) * s, c2 = b0 + (b1 - b0) * t;
    const V3<T> nh = c1 - c2;
    if (len(nh) < T(1e-12)) {
        for (int k = 0; k < 4; ++k) dummy[k] = false;
        n = robust_edge_pair_normal(a0, a1, b0, b1);
        d = c1 * T(0.5) + c2 * T(0.5);
        return;
    }
    n = normalized(nh);
    const T de0 = std::max(std::max(-dot(n, da0), -dot(n, da1)), T(0));
    const T de1 = std::max(std::max(dot(n, db0), dot(n, db1)), T(0));
    if (de0 + de1 == T(0)) {
        d = c2 + T(0.5) * nh;
    } else {
        T l = de1 / (de1 + de0);
        l = l < T(0.05) ? T(0.05) : (l > T(0.95) ? T(0.95) : l);
        d = c2 + l * nh;
    }
    if (de0 == T(0)) {
        dummy[0] = dummy[1] = true;
    } else {
        dummy[0] = !segment_plane_intersects(a0, da0, n, d, T(1e-6), T(-1e-8), T(1e-6));
        dummy[1] = !segment_plane_intersects(a1, da1, n, d, T(1e-6), T(-1e-8), T(1e-6));
    }
    if (de1 == T(0)) {
        dummy[2] = dummy[3] = true;
    } else {
        dummy[2] = !segment_plane_intersects(b0, db0, n, d, T(1e-6), T(-1e-8), T(1e-6));
        dummy[3] = !segment_plane_intersects(b1, db1, n, d, T(1e-6), T(-1e-8), T(1e-6));
    }
}

// planar_truncation_t (:2114-2130)
template <typename T>
T planar_truncation_t(V3<T> v, V3<T> dv, V3<T> n, V3<T> d, T eps, T gamma) {
    const T denom = dot(n, dv);
    if (std::fabs(denom) < eps) return T(1);
    T t = dot(n, d - v) / denom;
    if (t < T(0)) return T(1);
    t = std::min(t * gamma, t - T(1e-3));
    return clamp01(t);
}

template <typename T>
bool sorted_contains(const int32_t* b, const int32_t* e, int32_t x) {
    const int32_t* it = std::lower_bound(b, e, x);
    return it != e && *it == x;
}

// vertices within (threshold - 1) edge rings of each vertex, itself excluded (the n-ring filter,
// tri_mesh_collision.py:123-233): a triangle with a vertex in that set, or an edge with an
// endpoint in the union of its endpoints' sets, is not a contact candidate.
template <typename T>
void build_near_sets(Oracle<T>& o) {
    const int V = o.V;
    std::vector<std::vector<int32_t>> ring1(V);
    for (int e = 0; e < o.E; ++e) {
        const int a = o.edges[4 * e + 2], b = o.edges[4 * e + 3];
        ring1[a].push_back(b);
        ring1[b].push_back(a);
    }
    for (auto& r : ring1) {
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
    }
    const int depth = o.sc.filter_threshold - 1;
    o.near_off.assign(V + 1, 0);
    o.near.clear();
    for (int v = 0; v < V; ++v) {
        std::vector<int32_t> seen{v}, frontier{v};
        for (int k = 0; k < depth; ++k) {
            std::vector<int32_t> next;
            for (int u : frontier)
                for (int w : ring1[u])
                    if (std::find(seen.begin(), seen.end(), w) == seen.end()) {
                        seen.push_back(w);
                        next.push_back(w);
                    }
            frontier.swap(next);
            if (frontier.empty()) break;
        }
        std::sort(seen.begin(), seen.end());
        for (int w : seen)
            if (w != v) o.near.push_back(w);
        o.near_off[v + 1] = static_cast<int32_t>(o.near.size());
    }
}

template <typename T>
bool near_contains(const Oracle<T>& o, int v, int x) {
    if (o.sc.filter_threshold < 2) return false;
    return sorted_contains<T>(o.near.data() + o.near_off[v], o.near.data() + o.near_off[v + 1], x);
}

// vertex-triangle and edge-edge candidates within the margin at positions q (all pairs)
template <typename T>
void detect_self_contacts(Oracle<T>& o, const std::vector<T>& q) {
    const int V = o.V, Tn = o.Tn, E = o.E;
    const int vb = o.sc.vertex_buffer, eb = o.sc.edge_buffer;
    const T margin = T(o.sc.margin);
    const T excl = T(o.sc.rest_exclusion_radius);
    const bool use_rest = excl > T(0) && !o.rest_q.empty();
    o.vt_count.assign(V, 0);
    o.vt_list.assign(static_cast<size_t>(V) * vb, -1);
    o.ee_count.assign(E, 0);
    o.ee_list.assign(static_cast<size_t>(E) * eb, -1);
    o.tri_vs.assign(Tn, {});
#pragma omp parallel for schedule(dynamic, 64) num_threads(o.threads) if (o.threads > 1)
    for (int v = 0; v < V; ++v) {
        const V3<T> p = load3(q.data(), v);
        const int wv = o.world[v];
        int n = 0;
        long long over = 0;
        for (int t = 0; t < Tn; ++t) {
            const int a = o.tri[3 * t], b = o.tri[3 * t + 1], c = o.tri[3 * t + 2];
            if (a == v || b == v || c == v) continue;
            const int wt = o.world[a];
            if (wv >= 0 && wt >= 0 && wv != wt) continue;
            if (near_contains(o, v, a) || near_contains(o, v, b) || near_contains(o, v, c)) continue;
            if (!o.vfilt_off.empty() &&
                sorted_contains<T>(o.vfilt.data() + o.vfilt_off[v], o.vfilt.data() + o.vfilt_off[v + 1], t))
                continue;
            V3<T> bary;
            const T dist = len(triangle_closest_point(load3(q.data(), a), load3(q.data(), b), load3(q.data(), c), p, bary) - p);
            if (use_rest) {
                const T dr = len(triangle_closest_point(load3(o.rest_q.data(), a), load3(o.rest_q.data(), b),
                                                        load3(o.rest_q.data(), c), load3(o.rest_q.data(), v), bary) -
                                 load3(o.rest_q.data(), v));
                if (dr < excl) continue;
            }
            if (dist < margin) {
                if (n < vb) o.vt_list[static_cast<size_t>(v) * vb + n] = t;
                else ++over;
                ++n;
            }
        }
        o.vt_count[v] = std::min(n, vb);
        if (over) {
#pragma omp atomic
            o.sc_overflow += over;
        }
    }
#pragma omp parallel for schedule(dynamic, 64) num_threads(o.threads) if (o.threads > 1)
    for (int e = 0; e < E; ++e) {
        const int a0 = o.edges[4 * e + 2], a1 = o.edges[4 * e + 3];
        const V3<T> pa0 = load3(q.data(), a0), pa1 = load3(q.data(), a1);
        const int we = o.world[a0];
        int n = 0;
        long long over = 0;
        for (int f = 0; f < E; ++f) {
            const int b0 = o.edges[4 * f + 2], b1 = o.edges[4 * f + 3];
            if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) continue;
            const int wf = o.world[b0];
            if (we >= 0 && wf >= 0 && we != wf) continue;
            if (near_contains(o, a0, b0) || near_contains(o, a0, b1) || near_contains(o, a1, b0) ||
                near_contains(o, a1, b1))
                continue;
            if (!o.efilt_off.empty() &&
                sorted_contains<T>(o.efilt.data() + o.efilt_off[e], o.efilt.data() + o.efilt_off[e + 1], f))
                continue;
            T s, t, dist;
            closest_edge_edge(pa0, pa1, load3(q.data(), b0), load3(q.data(), b1), T(o.sc.edge_parallel_epsilon), s, t,
                              dist);
            if (use_rest) {
                T sr, tr, dr;
                closest_edge_edge(load3(o.rest_q.data(), a0), load3(o.rest_q.data(), a1), load3(o.rest_q.data(), b0),
                                  load3(o.rest_q.data(), b1), T(o.sc.edge_parallel_epsilon), sr, tr, dr);
                if (dr < excl) continue;
            }
            if (dist < margin) {
                if (n < eb) o.ee_list[static_cast<size_t>(e) * eb + n] = f;
                else ++over;
                ++n;
            }
        }
        o.ee_count[e] = std::min(n, eb);
        if (over) {
#pragma omp atomic
            o.sc_overflow += over;
        }
    }
    for (int v = 0; v < V; ++v)
        for (int k = 0; k < o.vt_count[v]; ++k) o.tri_vs[o.vt_list[static_cast<size_t>(v) * o.sc.vertex_buffer + k]].push_back(v);
}

// self-contact force and Hessian of vertex v (fixed order: own vertex-triangle pairs, then the
// pairs of each incident triangle in CSR order, then each incident edge's edge-edge pairs)
template <typename T>
void self_contact_vertex(const Oracle<T>& o, int v, T ke, T kd, T mu, T dt, V3<T>& f, M3<T>& H) {
    f = v3(T(0), T(0), T(0));
    H = zero3<T>();
    const T r = T(o.sc.radius);
    const T* q = o.q.data();
    const T* qa = o.q_prev.data();
    V3<T> F[4];
    M3<T> Hk[4];
    auto vt = [&](int p, int t, int slot) {
        const int a = o.tri[3 * t], b = o.tri[3 * t + 1], c = o.tri[3 * t + 2];
        if (vt_contact(load3(q, a), load3(q, b), load3(q, c), load3(q, p), load3(qa, a), load3(qa, b), load3(qa, c),
                       load3(qa, p), r, ke, kd, mu, o.friction_eps, dt, F, Hk)) {
            f = f + F[slot];
            H = H + Hk[slot];
        }
    };
    const size_t vb = o.sc.vertex_buffer;
    for (int k = 0; k < o.vt_count[v]; ++k) vt(v, o.vt_list[v * vb + k], 3);
    if (o.Tn > 0)
        for (int k = o.adj_t_off[v]; k < o.adj_t_off[v + 1]; k += 2) {
            const int t = o.adj_t[k], slot = o.adj_t[k + 1];
            for (int p : o.tri_vs[t]) vt(p, t, slot);
        }
    if (o.E > 0)
        for (int k = o.adj_e_off[v]; k < o.adj_e_off[v + 1]; k += 2) {
            const int e = o.adj_e[k], slot = o.adj_e[k + 1];
            if (slot < 2) continue;
            const int a0 = o.edges[4 * e + 2], a1 = o.edges[4 * e + 3];
            const size_t eb = o.sc.edge_buffer;
            for (int j = 0; j < o.ee_count[e]; ++j) {
                const int g = o.ee_list[e * eb + j];
                const int b0 = o.edges[4 * g + 2], b1 = o.edges[4 * g + 3];
                if (ee_contact(load3(q, a0), load3(q, a1), load3(q, b0), load3(q, b1), load3(qa, a0), load3(qa, a1),
                               load3(qa, b0), load3(qa, b1), r, ke, kd, mu, o.friction_eps, dt,
                               T(o.sc.edge_parallel_epsilon), F, Hk)) {
                    f = f + F[slot - 2];
                    H = H + Hk[slot - 2];
                }
            }
        }
}

// _penetration_free_truncation with self-contact (solver_vbd.py:2026-2063): per-vertex t from
// every contact's division plane (minimum), then disp *= t, |disp| <= margin * relaxation / 2,
// q = pos_prev_cd + disp for all particles.
template <typename T>
void planar_truncate(Oracle<T>& o) {
    const int V = o.V;
    std::vector<T> ts(V, T(1));
    const T eps = T(o.sc.edge_parallel_epsilon), gamma = T(o.sc.relaxation);
    const T* x = o.pos_prev_cd.data();
    const T* dx = o.disp.data();
    auto upd = [&](int i, V3<T> n, V3<T> d) {
        const T t = planar_truncation_t(load3(x, i), load3(dx, i), n, d, eps, gamma);
        if (t < ts[i]) ts[i] = t;
    };
    const size_t vb = o.sc.vertex_buffer, eb = o.sc.edge_buffer;
    for (int v = 0; v < V; ++v)
        for (int k = 0; k < o.vt_count[v]; ++k) {
            const int t = o.vt_list[v * vb + k];
            const int a = o.tri[3 * t], b = o.tri[3 * t + 1], c = o.tri[3 * t + 2];
            bool dummy[4];
            V3<T> n, d;
            vt_plane(load3(x, v), load3(dx, v), load3(x, a), load3(dx, a), load3(x, b), load3(dx, b), load3(x, c),
                     load3(dx, c), dummy, n, d);
            if (!dummy[0]) upd(v, n, d);
            if (!dummy[1]) upd(a, n, d);
            if (!dummy[2]) upd(b, n, d);
            if (!dummy[3]) upd(c, n, d);
        }
    for (int e = 0; e < o.E; ++e)
        for (int j = 0; j < o.ee_count[e]; ++j) {
            const int g = o.ee_list[e * eb + j];
            const int a0 = o.edges[4 * e + 2], a1 = o.edges[4 * e + 3];
            const int b0 = o.edges[4 * g + 2], b1 = o.edges[4 * g + 3];
            bool dummy[4];
            V3<T> n, d;
            ee_plane(load3(x, a0), load3(dx, a0), load3(x, a1), load3(dx, a1), load3(x, b0), load3(dx, b0),
                     load3(x, b1), load3(dx, b1), dummy, n, d);
            if (!dummy[0]) upd(a0, n, d);
            if (!dummy[1]) upd(a1, n, d);
            if (!dummy[2]) upd(b0, n, d);
            if (!dummy[3]) upd(b1, n, d);
        }
    const T maxd = T(static_cast<float>(double(o.sc.margin) * double(o.sc.relaxation) * 0.5));
    for (int p = 0; p < V; ++p) {
        V3<T> d = load3(o.disp.data(), p) * ts[p];
        const T l = len(d);
        if (l > maxd) d = d * maxd / l;
        store3(o.disp.data(), p, d);
        store3(o.q.data(), p, load3(o.pos_prev_cd.data(), p) + d);
    }
}

// _collision_detection_penetration_free (solver_vbd.py:3221-3237)
template <typename T>
void collision_detection_penetration_free(Oracle<T>& o) {
    o.pos_prev_cd = o.q;
    std::fill(o.disp.begin(), o.disp.end(), T(0));
    detect_self_contacts(o, o.q);
}

template <typename T>
void forward(Oracle<T>& o, const float* q_in, const float* qd_in, const float* f_ext, T dt) {
    const int V = o.V;
    for (int i = 0; i < 3 * V; ++i) o.q[i] = T(q_in[i]);
    o.iteration = 0;
    if (o.sc.enabled) {
        collision_detection_penetration_free(o);
    } else {
        o.pos_prev_cd = o.q;                   // pos_prev_collision_detection.assign(state_in.q)
        std::fill(o.disp.begin(), o.disp.end(), T(0));
    }
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
    if (o.sc.enabled) {
        planar_truncate(o);
        return;
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
    if (o.sc.enabled) {
        const T ke = T(o.soft_ke), kd = T(o.soft_kd), mu = T(o.soft_mu);
#pragma omp parallel for schedule(static) num_threads(o.threads) if (o.threads > 1)
        for (int k = b; k < e; ++k) {
            const int p = o.color_par[k];
            V3<T> f;
            M3<T> H;
            self_contact_vertex(o, p, ke, kd, mu, dt, f, H);
            store3(o.pf.data(), p, load3(o.pf.data(), p) + f);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) o.ph[9 * p + 3 * i + j] += H.m[i][j];
        }
    }
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
        const T gn = std::sqrt(o.g[0] * o.g[0] + o.g[1] * o.g[1] + o.g[2] * o.g[2]);
        o.gs_r[p] = float(len(f) / (o.mass[p] * gn));
        if (std::fabs(det3(h)) > T(1.0e-8)) {
            const M3<T> hi = inverse3(h);
            store3(o.disp.data(), p, load3(o.disp.data(), p) + hi * f);
        }
    }
    if (o.sc.enabled) {
        planar_truncate(o);
        return;
    }
    // apply_truncation_ts over all particles
#pragma omp parallel for schedule(static) num_threads(o.threads) if (o.threads > 1)
    for (int p = 0; p < o.V; ++p) store3(o.q.data(), p, load3(o.pos_prev_cd.data(), p) + load3(o.disp.data(), p));
}

template <typename T>
void begin_iteration(Oracle<T>& o) {
    // self-contact detection at iteration 0 (interval 0) or every `interval` iterations (:2540-2545)
    const int it = o.iteration++;
    if (o.sc.enabled && ((o.sc.interval == 0 && it == 0) || (o.sc.interval >= 1 && it % o.sc.interval == 0)))
        collision_detection_penetration_free(o);
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
    if (o.sc.enabled) {
        for (int p = 0; p < o.V; ++p) {
            V3<T> f;
            M3<T> H;
            self_contact_vertex(o, p, T(o.soft_ke), T(o.soft_kd), T(o.soft_mu), dt, f, H);
            store3(o.pf.data(), p, load3(o.pf.data(), p) + f);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) o.ph[9 * p + 3 * i + j] += H.m[i][j];
        }
    }
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

// Gauss-Seidel residual of each vertex's last sweep (0 for vertices never solved): the residual
// the library's sweep-residual gate accumulates
void oracle_sweep_residual(OracleHandle* h, float* per_vertex) {
    ORACLE_DISPATCH(h, std::copy(o.gs_r.begin(), o.gs_r.end(), per_vertex));
}

// Self-contact (particle_enable_self_contact=True path): parameters, and detection alone.
void oracle_set_self_contact(OracleHandle* h, const OracleSelfContact* p) {
    ORACLE_DISPATCH(h, {
        o.sc = *p;
        o.sc.rest_q = nullptr;
        o.rest_q.clear();
        if (p->rest_q) o.rest_q.assign(p->rest_q, p->rest_q + 3 * o.V);
        o.vt_count.assign(o.V, 0);
        o.vt_list.assign(static_cast<size_t>(o.V) * std::max(1, p->vertex_buffer), -1);
        o.ee_count.assign(o.E, 0);
        o.ee_list.assign(static_cast<size_t>(o.E) * std::max(1, p->edge_buffer), -1);
        o.tri_vs.assign(o.Tn, {});
        if (p->enabled && p->filter_threshold >= 2) build_near_sets(o);
        o.vfilt_off.clear();
        o.vfilt.clear();
        o.efilt_off.clear();
        o.efilt.clear();
        if (p->vertex_filter_offsets) {
            o.vfilt_off.assign(p->vertex_filter_offsets, p->vertex_filter_offsets + o.V + 1);
            o.vfilt.assign(p->vertex_filter_triangles, p->vertex_filter_triangles + o.vfilt_off[o.V]);
        }
        if (p->edge_filter_offsets) {
            o.efilt_off.assign(p->edge_filter_offsets, p->edge_filter_offsets + o.E + 1);
            o.efilt.assign(p->edge_filter_edges, p->edge_filter_edges + o.efilt_off[o.E]);
        }
        o.sc.vertex_filter_offsets = o.sc.vertex_filter_triangles = nullptr;
        o.sc.edge_filter_offsets = o.sc.edge_filter_edges = nullptr;
    });
}

// Detection at positions q (model order): per-vertex colliding triangles and per-edge colliding
// edges (ascending, -1 padded, strides vertex_buffer / edge_buffer).  Returns the number of
// candidates dropped because a buffer was full.
long long oracle_self_contact_detect(OracleHandle* h, const float* q, int32_t* vt_counts, int32_t* vt_lists,
                                     int32_t* ee_counts, int32_t* ee_lists) {
    long long over = 0;
    ORACLE_DISPATCH(h, {
        std::vector<T> qq(q, q + 3 * o.V);
        o.sc_overflow = 0;
        detect_self_contacts(o, qq);
        over = o.sc_overflow;
        std::copy(o.vt_count.begin(), o.vt_count.end(), vt_counts);
        std::copy(o.vt_list.begin(), o.vt_list.end(), vt_lists);
        std::copy(o.ee_count.begin(), o.ee_count.end(), ee_counts);
        std::copy(o.ee_list.begin(), o.ee_list.end(), ee_lists);
    });
    return over;
}

// Element-level self-contact functions (known-answer tests).
void oracle_self_contact_norm(int is_double, double dis, double r, double k, double* out) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        T a, b;
        self_contact_norm<T>(T(dis), T(r), T(k), a, b);
        out[0] = a;
        out[1] = b;
    };
    if (is_double) run(double(0));
    else run(float(0));
}

// pos / anchor: a, b, c, p (12 values each); outputs for a, b, c, p
int oracle_vt_contact(int is_double, const double* pos, const double* anchor, double r, double ke, double kd,
                      double mu, double feps, double dt, double* f_out, double* h_out) {
    int has = 0;
    auto run = [&](auto tag) {
        using T = decltype(tag);
        V3<T> x[4], a[4], F[4];
        M3<T> H[4];
        for (int k = 0; k < 4; ++k) {
            x[k] = v3(T(pos[3 * k]), T(pos[3 * k + 1]), T(pos[3 * k + 2]));
            a[k] = v3(T(anchor[3 * k]), T(anchor[3 * k + 1]), T(anchor[3 * k + 2]));
        }
        has = vt_contact<T>(x[0], x[1], x[2], x[3], a[0], a[1], a[2], a[3], T(r), T(ke), T(kd), T(mu), T(feps), T(dt),
                            F, H);
        for (int k = 0; k < 4; ++k) {
            f_out[3 * k] = has ? double(F[k].x) : 0.0;
            f_out[3 * k + 1] = has ? double(F[k].y) : 0.0;
            f_out[3 * k + 2] = has ? double(F[k].z) : 0.0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) h_out[9 * k + 3 * i + j] = has ? double(H[k].m[i][j]) : 0.0;
        }
    };
    if (is_double) run(double(0));
    else run(float(0));
    return has;
}

// pos / anchor: e0, e1, f0, f1 (12 values each); outputs for e0, e1
int oracle_ee_contact(int is_double, const double* pos, const double* anchor, double r, double ke, double kd,
                      double mu, double feps, double dt, double par_eps, double* f_out, double* h_out) {
    int has = 0;
    auto run = [&](auto tag) {
        using T = decltype(tag);
        V3<T> x[4], a[4], F[2];
        M3<T> H[2];
        for (int k = 0; k < 4; ++k) {
            x[k] = v3(T(pos[3 * k]), T(pos[3 * k + 1]), T(pos[3 * k + 2]));
            a[k] = v3(T(anchor[3 * k]), T(anchor[3 * k + 1]), T(anchor[3 * k + 2]));
        }
        has = ee_contact<T>(x[0], x[1], x[2], x[3], a[0], a[1], a[2], a[3], T(r), T(ke), T(kd), T(mu), T(feps), T(dt),
                            T(par_eps), F, H);
        for (int k = 0; k < 2; ++k) {
            f_out[3 * k] = has ? double(F[k].x) : 0.0;
            f_out[3 * k + 1] = has ? double(F[k].y) : 0.0;
            f_out[3 * k + 2] = has ? double(F[k].z) : 0.0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) h_out[9 * k + 3 * i + j] = has ? double(H[k].m[i][j]) : 0.0;
        }
    };
    if (is_double) run(double(0));
    else run(float(0));
    return has;
}

// p1 q1 p2 q2 (12 values) -> s, t, distance
void oracle_closest_edge_edge(const double* pts, double eps, double* out) {
    V3<double> p[4];
    for (int k = 0; k < 4; ++k) p[k] = v3(pts[3 * k], pts[3 * k + 1], pts[3 * k + 2]);
    closest_edge_edge<double>(p[0], p[1], p[2], p[3], eps, out[0], out[1], out[2]);
}

// a b c p (12 values) -> closest point (3) and barycentric coordinates (3)
void oracle_triangle_closest_point(const double* pts, double* out) {
    V3<double> p[4];
    for (int k = 0; k < 4; ++k) p[k] = v3(pts[3 * k], pts[3 * k + 1], pts[3 * k + 2]);
    V3<double> bary;
    const V3<double> c = triangle_closest_point<double>(p[0], p[1], p[2], p[3], bary);
    out[0] = c.x;
    out[1] = c.y;
    out[2] = c.z;
    out[3] = bary.x;
    out[4] = bary.y;
    out[5] = bary.z;
}

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

// ---------------------------------------------------------------------------------------------
// Model set-up restated for the checker (independent of the library's host code): the bending-
// edge table and the conflict-graph coloring.  Used by oracle/setup.py to build scenes without the
// CUDA library (the CPU-baseline leg) and to cross-check the library's set-up tables.
// ---------------------------------------------------------------------------------------------

// Edge table [o0, o1, v0, v1] of MeshAdjacency._compute_edge_adjacency (utils/mesh.py:465-531),
// by sorting: every triangle slot (t, k) names the undirected edge {tris[t][k], tris[t][k+1]}
// with opposite vertex tris[t][k+2]; slots are sorted by (edge key, slot index), each group is one
// edge whose first slot fills [o0, -1, v0, v1] and whose second fills o1 (later ones are ignored,
// as the reference does for non-manifold edges); edges are numbered in the order of their first
// slot.  edges_out holds room for 3 nt rows; returns the edge count.
int oracle_edge_table(const int32_t* tris, int nt, int32_t* edges_out) {
    const int64_t ns = 3 * static_cast<int64_t>(nt);
    std::vector<int64_t> slot(ns);
    std::vector<uint64_t> key(ns);
    for (int64_t j = 0; j < ns; ++j) {
        const int64_t t = j / 3;
        const int k = static_cast<int>(j % 3);
        const uint32_t a = static_cast<uint32_t>(tris[3 * t + k]), b = static_cast<uint32_t>(tris[3 * t + (k + 1) % 3]);
        key[j] = (static_cast<uint64_t>(std::min(a, b)) << 32) | std::max(a, b);
        slot[j] = j;
    }
    std::sort(slot.begin(), slot.end(), [&](int64_t x, int64_t y) { return key[x] != key[y] ? key[x] < key[y] : x < y; });
    // groups: (first slot, second slot or -1)
    std::vector<std::pair<int64_t, int64_t>> groups;
    for (int64_t i = 0; i < ns;) {
        int64_t j = i + 1;
        while (j < ns && key[slot[j]] == key[slot[i]]) ++j;
        groups.push_back({slot[i], j - i > 1 ? slot[i + 1] : -1});
        i = j;
    }
    std::sort(groups.begin(), groups.end());
    for (size_t e = 0; e < groups.size(); ++e) {
        const int64_t f = groups[e].first, g = groups[e].second;
        const int64_t t = f / 3;
        const int k = static_cast<int>(f % 3);
        int32_t* row = edges_out + 4 * e;
        row[0] = tris[3 * t + (k + 2) % 3];
        row[1] = -1;
        row[2] = tris[3 * t + k];
        row[3] = tris[3 * t + (k + 1) % 3];
        if (g >= 0) row[1] = tris[3 * (g / 3) + (g % 3 + 2) % 3];
    }
    return static_cast<int>(groups.size());
}

// Coloring of a canonical edge list (unique (min, max) pairs in lexicographic order), the
// algorithm the library states: an ordering, first-fit colors in that order, then balancing.
//   algorithm 0 (MCS, Pereira & Palsberg 2005): repeatedly take the unvisited vertex with the
//     most visited neighbours; ties go to the vertex whose count was raised last (initially
//     vertex 0 first, then 1, 2, ...).  Restated here with a priority queue keyed by (count,
//     time of the last raise).
//   algorithm 1 (GREEDY): decreasing degree, ties by index.
//   balance: while max/min color size > target, move the lowest-index vertices of the largest
//     color that have no neighbour in the smallest color into it; stop when a pass moves nothing
//     (or after 64 passes per color).
// Neighbour lists are in edge-list order.  Returns the number of colors (before balancing).
int oracle_color_graph(int n, int64_t m, const int32_t* edges, int algorithm, int do_balance, float target,
                       int32_t* colors) {
    std::vector<std::vector<int>> nb(n);
    for (int64_t e = 0; e < m; ++e) {
        const int a = edges[2 * e], b = edges[2 * e + 1];
        if (a == b) continue;
        nb[a].push_back(b);
        nb[b].push_back(a);
    }
    std::vector<int> order;
    order.reserve(n);
    if (algorithm == 0) {
        using Entry = std::tuple<int, int64_t, int>;  // (count, raise time, vertex)
        std::priority_queue<Entry> pq;
        std::vector<int> count(n, 0);
        std::vector<char> done(n, 0);
        int64_t clock = 0;
        for (int v = n - 1; v >= 0; --v) pq.emplace(0, clock++, v);
        while (!pq.empty()) {
            const auto [c, tm, v] = pq.top();
            pq.pop();
            if (done[v] || c != count[v]) continue;
            done[v] = 1;
            order.push_back(v);
            for (int u : nb[v]) {
                if (done[u]) continue;
                pq.emplace(++count[u], clock++, u);
            }
        }
    } else {
        for (int v = 0; v < n; ++v) order.push_back(v);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return nb[a].size() > nb[b].size(); });
    }
    std::vector<int> col(n, -1);
    int nc = 0;
    for (int v : order) {
        std::vector<char> used(nb[v].size() + 1, 0);
        for (int u : nb[v])
            if (col[u] >= 0 && col[u] <= static_cast<int>(nb[v].size())) used[col[u]] = 1;
        int c = 0;
        while (used[c]) ++c;
        col[v] = c;
        nc = std::max(nc, c + 1);
    }
    if (do_balance && nc >= 2) {
        std::vector<int64_t> size(nc, 0);
        for (int v = 0; v < n; ++v) size[col[v]]++;
        auto ratio_ok = [&](int hi, int lo) { return size[lo] > 0 && double(size[hi]) / double(size[lo]) <= target; };
        for (int pass = 0; pass < 64 * nc; ++pass) {
            const int hi = static_cast<int>(std::max_element(size.begin(), size.end()) - size.begin());
            const int lo = static_cast<int>(std::min_element(size.begin(), size.end()) - size.begin());
            if (ratio_ok(hi, lo)) break;
            bool moved = false;
            for (int v = 0; v < n && size[hi] > size[lo] + 1; ++v) {
                if (col[v] != hi) continue;
                if (std::any_of(nb[v].begin(), nb[v].end(), [&](int u) { return col[u] == lo; })) continue;
                col[v] = lo;
                size[hi]--;
                size[lo]++;
                moved = true;
                if (ratio_ok(hi, lo)) break;
            }
            if (!moved) break;
        }
    }
    for (int v = 0; v < n; ++v) colors[v] = col[v];
    return nc;
}

}  // extern "C"

