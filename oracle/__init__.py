"""CPU oracle of Newton's particle VBD cloth step -- TEST INFRASTRUCTURE ONLY.

A C++ restatement (``vbd_oracle.cpp``) of the reference's serial CPU path, FP32 and FP64, with a
ctypes wrapper.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
use it, as the checker of the CUDA library; the product path never calls it.

Parity pinning: the reference (Python + Warp) cannot run in this environment (``warp-lang`` is
not installed), so the oracle is pinned against the known-answer tests of the reference's own
test suite (``newton/tests/test_solver_vbd.py``), restated in ``tests/test_oracle_kat.py``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from .build_oracle import OUT, build

_lib = None

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)


class OracleShape(ctypes.Structure):
    _fields_ = [
        ("geo_type", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("world", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("xform", ctypes.c_float * 7),
        ("scale", ctypes.c_float * 3),
        ("margin", ctypes.c_float),
        ("material_ke", ctypes.c_float),
        ("material_kd", ctypes.c_float),
        ("material_mu", ctypes.c_float),
    ]


class OracleModelDesc(ctypes.Structure):
    _fields_ = [
        ("particle_count", ctypes.c_int32),
        ("tri_count", ctypes.c_int32),
        ("edge_count", ctypes.c_int32),
        ("shape_count", ctypes.c_int32),
        ("color_count", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("particle_mass", c_float_p),
        ("particle_inv_mass", c_float_p),
        ("particle_radius", c_float_p),
        ("particle_flags", c_int32_p),
        ("particle_world", c_int32_p),
        ("tri_indices", c_int32_p),
        ("tri_poses", c_float_p),
        ("tri_materials", c_float_p),
        ("tri_areas", c_float_p),
        ("edge_indices", c_int32_p),
        ("edge_rest_angle", c_float_p),
        ("edge_rest_length", c_float_p),
        ("edge_bending_properties", c_float_p),
        ("v_adj_tris_offsets", c_int32_p),
        ("v_adj_tris", c_int32_p),
        ("v_adj_edges_offsets", c_int32_p),
        ("v_adj_edges", c_int32_p),
        ("color_group_offsets", c_int32_p),
        ("color_group_particles", c_int32_p),
        ("gravity", ctypes.c_float * 3),
        ("soft_contact_ke", ctypes.c_float),
        ("soft_contact_kd", ctypes.c_float),
        ("soft_contact_mu", ctypes.c_float),
        ("shapes", ctypes.POINTER(OracleShape)),
    ]


class OracleSelfContact(ctypes.Structure):
    _fields_ = [
        ("enabled", ctypes.c_int32),
        ("radius", ctypes.c_float),
        ("margin", ctypes.c_float),
        ("relaxation", ctypes.c_float),
        ("vertex_buffer", ctypes.c_int32),
        ("edge_buffer", ctypes.c_int32),
        ("interval", ctypes.c_int32),
        ("edge_parallel_epsilon", ctypes.c_float),
        ("filter_threshold", ctypes.c_int32),
        ("rest_exclusion_radius", ctypes.c_float),
        ("rest_q", ctypes.POINTER(ctypes.c_float)),
        ("vertex_filter_offsets", ctypes.POINTER(ctypes.c_int32)),
        ("vertex_filter_triangles", ctypes.POINTER(ctypes.c_int32)),
        ("edge_filter_offsets", ctypes.POINTER(ctypes.c_int32)),
        ("edge_filter_edges", ctypes.POINTER(ctypes.c_int32)),
    ]


def filter_map_csr(mapping, rows: int):
    """{row: iterable of ids} -> (offsets [rows+1], ascending ids) int32 arrays, or (None, None)."""
    if not mapping:
        return None, None
    lists = [sorted({int(x) for x in mapping.get(r, ())}) for r in range(rows)]
    off = np.zeros(rows + 1, np.int32)
    off[1:] = np.cumsum([len(l) for l in lists])
    flat = np.array([x for l in lists for x in l], dtype=np.int32)
    return off, flat


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(OUT))
        vp = ctypes.c_void_p
        lib.oracle_create.restype = vp
        lib.oracle_create.argtypes = [ctypes.POINTER(OracleModelDesc), ctypes.c_int, ctypes.c_float, ctypes.c_int]
        lib.oracle_destroy.argtypes = [vp]
        lib.oracle_set_threads.argtypes = [vp, ctypes.c_int]
        lib.oracle_set_contacts.argtypes = [vp, ctypes.c_int, c_int32_p, c_int32_p, c_float_p, c_float_p, c_float_p]
        lib.oracle_forward.argtypes = [vp, c_float_p, c_float_p, c_float_p, ctypes.c_float]
        lib.oracle_begin_iteration.argtypes = [vp]
        lib.oracle_sweep_color.argtypes = [vp, ctypes.c_int, ctypes.c_float]
        lib.oracle_finalize.argtypes = [vp, c_float_p, c_float_p, c_float_p, ctypes.c_float]
        lib.oracle_step.argtypes = [vp, c_float_p, c_float_p, c_float_p, c_float_p, c_float_p, ctypes.c_float, ctypes.c_int]
        lib.oracle_get_positions.argtypes = [vp, c_double_p]
        lib.oracle_residual.argtypes = [vp, ctypes.c_float, c_float_p]
        lib.oracle_set_positions.argtypes = [vp, c_float_p]
        lib.oracle_sweep_residual.argtypes = [vp, c_float_p]
        d = ctypes.c_double
        lib.oracle_membrane.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p, c_int32_p,
                                        c_double_p, d, d, d, d, d, ctypes.c_int, c_double_p, c_double_p]
        lib.oracle_bending.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p, c_int32_p, d, d,
                                       d, d, d, ctypes.c_int, c_double_p, c_double_p]
        lib.oracle_contact.argtypes = [ctypes.c_int, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p, d, d, d,
                                       d, d, d, d, c_double_p, c_double_p]
        lib.oracle_collide.restype = ctypes.c_int
        lib.oracle_collide.argtypes = [ctypes.c_int, c_float_p, c_float_p, c_int32_p, c_int32_p, ctypes.c_int,
                                       ctypes.POINTER(OracleShape), ctypes.c_float, ctypes.c_int, c_int32_p, c_int32_p,
                                       c_float_p, c_float_p, c_float_p]
        lib.oracle_set_self_contact.argtypes = [vp, ctypes.POINTER(OracleSelfContact)]
        lib.oracle_self_contact_detect.restype = ctypes.c_longlong
        lib.oracle_self_contact_detect.argtypes = [vp, c_float_p, c_int32_p, c_int32_p, c_int32_p, c_int32_p]
        lib.oracle_self_contact_norm.argtypes = [ctypes.c_int, d, d, d, c_double_p]
        lib.oracle_vt_contact.restype = ctypes.c_int
        lib.oracle_vt_contact.argtypes = [ctypes.c_int, c_double_p, c_double_p, d, d, d, d, d, d, c_double_p,
                                          c_double_p]
        lib.oracle_ee_contact.restype = ctypes.c_int
        lib.oracle_ee_contact.argtypes = [ctypes.c_int, c_double_p, c_double_p, d, d, d, d, d, d, d, c_double_p,
                                          c_double_p]
        lib.oracle_closest_edge_edge.argtypes = [c_double_p, d, c_double_p]
        lib.oracle_triangle_closest_point.argtypes = [c_double_p, c_double_p]
        _lib = lib
    return _lib


def _f32(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    return a, a.ctypes.data_as(c_float_p)


def _i32(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    return a, a.ctypes.data_as(c_int32_p)


def _f64(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a, a.ctypes.data_as(c_double_p)


def _shapes(model):
    S = model.shape_count
    arr = (OracleShape * max(S, 1))()
    for s in range(S):
        sh = arr[s]
        sh.geo_type = int(model.shape_type[s])
        sh.flags = int(model.shape_flags[s])
        sh.world = int(model.shape_world[s])
        for k in range(7):
            sh.xform[k] = float(model.shape_transform[s, k])
        for k in range(3):
            sh.scale[k] = float(model.shape_scale[s, k])
        sh.margin = float(model.shape_margin[s])
        sh.material_ke = float(model.shape_material_ke[s])
        sh.material_kd = float(model.shape_material_kd[s])
        sh.material_mu = float(model.shape_material_mu[s])
    return arr


class VBDOracle:
    """Stateful CPU oracle of one SolverVBD (particle path) on a finalized ``newton_b200.Model``."""

    def __init__(self, model, precision: str = "f32", friction_epsilon: float = 1e-2, threads: int = 1):
        lib = load()
        self.model = model
        self.V = model.particle_count
        keep = []

        def f(a):
            arr, p = _f32(a)
            keep.append(arr)
            return p if arr.size else None

        def i(a):
            arr, p = _i32(a)
            keep.append(arr)
            return p if arr.size else None

        d = OracleModelDesc()
        d.particle_count = model.particle_count
        d.tri_count = model.tri_count
        d.edge_count = model.edge_count
        d.shape_count = model.shape_count
        d.color_count = len(model.particle_color_groups)
        d.particle_mass = f(model.particle_mass)
        d.particle_inv_mass = f(model.particle_inv_mass)
        d.particle_radius = f(model.particle_radius)
        d.particle_flags = i(model.particle_flags)
        d.particle_world = i(model.particle_world)
        d.tri_indices = i(model.tri_indices)
        d.tri_poses = f(model.tri_poses)
        d.tri_materials = f(model.tri_materials)
        d.tri_areas = f(model.tri_areas)
        d.edge_indices = i(model.edge_indices)
        d.edge_rest_angle = f(model.edge_rest_angle)
        d.edge_rest_length = f(model.edge_rest_length)
        d.edge_bending_properties = f(model.edge_bending_properties)
        adj = model.soft_mesh_adjacency
        d.v_adj_tris_offsets = i(adj.v_adj_tris_offsets)
        d.v_adj_tris = i(adj.v_adj_tris)
        d.v_adj_edges_offsets = i(adj.v_adj_edges_offsets)
        d.v_adj_edges = i(adj.v_adj_edges)
        offs, flat = model.color_group_csr()
        d.color_group_offsets = i(offs)
        d.color_group_particles = i(flat)
        g = np.asarray(model.gravity, dtype=np.float32).reshape(-1, 3)[0]
        for k in range(3):
            d.gravity[k] = float(g[k])
        d.soft_contact_ke = float(np.float32(model.soft_contact_ke))
        d.soft_contact_kd = float(np.float32(model.soft_contact_kd))
        d.soft_contact_mu = float(np.float32(model.soft_contact_mu))
        self._shapes = _shapes(model)
        d.shapes = ctypes.cast(self._shapes, ctypes.POINTER(OracleShape))
        self.precision = precision
        self._h = lib.oracle_create(ctypes.byref(d), 1 if precision == "f64" else 0, friction_epsilon, threads)
        self._lib = lib

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.oracle_destroy(self._h)
            self._h = None

    def set_self_contact(self, radius: float, margin: float, relaxation: float = 0.85, vertex_buffer: int = 32,
                         edge_buffer: int = 64, interval: int = 0, edge_parallel_epsilon: float = 1e-5,
                         filter_threshold: int = 2, rest_exclusion_radius: float = 0.0, rest_q=None,
                         enabled: bool = True, vertex_filter_map=None, edge_filter_map=None) -> None:
        """SolverVBD's particle self-contact settings (solver_vbd.py:231-241)."""
        p = OracleSelfContact()
        p.enabled = 1 if enabled else 0
        p.radius, p.margin, p.relaxation = radius, margin, relaxation
        p.vertex_buffer, p.edge_buffer, p.interval = vertex_buffer, edge_buffer, interval
        p.edge_parallel_epsilon = edge_parallel_epsilon
        p.filter_threshold = filter_threshold
        p.rest_exclusion_radius = rest_exclusion_radius
        rq = None
        if rest_q is not None:
            rq, p.rest_q = _f32(np.asarray(rest_q).reshape(-1, 3))
        keep = []
        vo, vl = filter_map_csr(vertex_filter_map, self.V)
        if vo is not None:
            keep += [vo, vl]
            p.vertex_filter_offsets = vo.ctypes.data_as(c_int32_p)
            p.vertex_filter_triangles = vl.ctypes.data_as(c_int32_p)
        eo, el = filter_map_csr(edge_filter_map, self.model.edge_count)
        if eo is not None:
            keep += [eo, el]
            p.edge_filter_offsets = eo.ctypes.data_as(c_int32_p)
            p.edge_filter_edges = el.ctypes.data_as(c_int32_p)
        self.sc_buffers = (vertex_buffer, edge_buffer)
        self._lib.oracle_set_self_contact(self._h, ctypes.byref(p))

    def self_contact_detect(self, q):
        """Vertex-triangle and edge-edge candidates at q: (vt_counts, vt_lists, ee_counts, ee_lists, dropped)."""
        vb, eb = self.sc_buffers
        E = self.model.edge_count
        vc = np.zeros(self.V, np.int32)
        vl = np.zeros((self.V, vb), np.int32)
        ec = np.zeros(E, np.int32)
        el = np.zeros((max(E, 1), eb), np.int32)
        qa, pq = _f32(np.asarray(q).reshape(-1, 3))
        dropped = self._lib.oracle_self_contact_detect(self._h, pq, vc.ctypes.data_as(c_int32_p),
                                                       vl.ctypes.data_as(c_int32_p), ec.ctypes.data_as(c_int32_p),
                                                       el.ctypes.data_as(c_int32_p))
        return vc, vl, ec, el[:E], int(dropped)

    def set_threads(self, n: int) -> None:
        self._lib.oracle_set_threads(self._h, int(n))

    def set_contacts(self, particle, shape, body_pos, body_vel, normal) -> None:
        n = len(particle)
        a, pa = _i32(particle)
        b, pb = _i32(shape)
        c, pc = _f32(np.asarray(body_pos).reshape(-1, 3))
        e, pe = _f32(np.asarray(body_vel).reshape(-1, 3))
        g, pg = _f32(np.asarray(normal).reshape(-1, 3))
        self._lib.oracle_set_contacts(self._h, n, pa, pb, pc, pe, pg)

    def clear_contacts(self) -> None:
        z = np.zeros(0)
        self.set_contacts(np.zeros(0, np.int32), np.zeros(0, np.int32), z, z, z)

    def step(self, q_in: np.ndarray, qd_in: np.ndarray, f_ext: np.ndarray | None, dt: float, iterations: int):
        """One SolverVBD.step; returns (q_in_after, q_out, qd_out) as float32 [V,3] arrays."""
        q, pq = _f32(np.array(q_in, dtype=np.float32).reshape(-1, 3))
        qd, pqd = _f32(qd_in)
        fe, pfe = _f32(f_ext) if f_ext is not None else (None, None)
        q_out = np.zeros((self.V, 3), np.float32)
        qd_out = np.zeros((self.V, 3), np.float32)
        self._lib.oracle_step(self._h, pq, pqd, pfe, q_out.ctypes.data_as(c_float_p), qd_out.ctypes.data_as(c_float_p),
                              float(dt), int(iterations))
        return q, q_out, qd_out

    def forward(self, q_in, qd_in, f_ext, dt: float) -> None:
        q, pq = _f32(q_in)
        qd, pqd = _f32(qd_in)
        fe, pfe = _f32(f_ext) if f_ext is not None else (None, None)
        self._lib.oracle_forward(self._h, pq, pqd, pfe, float(dt))

    def begin_iteration(self) -> None:
        self._lib.oracle_begin_iteration(self._h)

    def sweep_color(self, color: int, dt: float) -> None:
        self._lib.oracle_sweep_color(self._h, int(color), float(dt))

    def finalize(self, dt: float):
        q_in = np.zeros((self.V, 3), np.float32)
        q_out = np.zeros((self.V, 3), np.float32)
        qd_out = np.zeros((self.V, 3), np.float32)
        self._lib.oracle_finalize(self._h, q_in.ctypes.data_as(c_float_p), q_out.ctypes.data_as(c_float_p),
                                  qd_out.ctypes.data_as(c_float_p), float(dt))
        return q_in, q_out, qd_out

    def positions(self) -> np.ndarray:
        out = np.zeros((self.V, 3), np.float64)
        self._lib.oracle_get_positions(self._h, out.ctypes.data_as(c_double_p))
        return out

    def set_positions(self, q) -> None:
        a, p = _f32(np.asarray(q).reshape(-1, 3))
        self._lib.oracle_set_positions(self._h, p)

    def residual(self, dt: float) -> np.ndarray:
        out = np.zeros(self.V, np.float32)
        self._lib.oracle_residual(self._h, float(dt), out.ctypes.data_as(c_float_p))
        return out

    def sweep_residual(self) -> np.ndarray:
        """|f_i| / (m_i |g|) of every vertex at its last Gauss-Seidel visit (0 if never solved)."""
        out = np.zeros(self.V, np.float32)
        self._lib.oracle_sweep_residual(self._h, out.ctypes.data_as(c_float_p))
        return out

    @staticmethod
    def _norm(pv, norm):
        if norm == "max":
            return float(pv.max()) if pv.size else 0.0
        fixed = np.floor(np.minimum(pv, np.float32(1e9)) * np.float32(256.0) + np.float32(0.5))
        return float(np.float32(float(fixed.astype(np.uint64).sum()) / 256.0 / max(pv.size, 1)))

    def gated_step(self, q_in, qd_in, f_ext, dt: float, tolerance: float, max_iterations: int,
                   check_every: int = 1, norm: str = "mean", relative: bool = False):
        """The residual gate with sweep residuals (the library's VBD_GATE_SWEEP): forward, then
        iterations until the norm of the last iteration's Gauss-Seidel residuals is <= tolerance
        (``relative``: tolerance x the norm of the Jacobi residual at the inertia target y),
        checked every ``check_every`` iterations, at least one iteration, at most
        ``max_iterations`` rounded up to a multiple of ``check_every``.  Returns
        (q_in_after, q_out, qd_out, iterations, final norm)."""
        self.forward(q_in, qd_in, f_ext, dt)
        m = self.model
        solvable = ((np.asarray(m.particle_flags) & 1) != 0) & (np.asarray(m.particle_mass) != 0)
        thresh = float(np.float32(tolerance))
        if relative:
            thresh = float(np.float32(tolerance) * np.float32(self._norm(self.residual(dt)[solvable], norm)))
        k, r = 0, 0.0
        while max_iterations > 0:
            for _ in range(check_every):
                self.begin_iteration()
                for c in range(len(m.particle_color_groups)):
                    self.sweep_color(c, dt)
            k += check_every
            r = self._norm(self.sweep_residual()[solvable], norm)
            if r <= thresh or k >= max_iterations:
                break
        q_in_after, q_out, qd_out = self.finalize(dt)
        return q_in_after, q_out, qd_out, k, r


def collide(model, q: np.ndarray, margin: float):
    """create_soft_contacts over the model's static shapes; returns record arrays (shape order per particle)."""
    lib = load()
    V, S = model.particle_count, model.shape_count
    mx = V * S
    particle = np.zeros(max(mx, 1), np.int32)
    shape = np.zeros(max(mx, 1), np.int32)
    bpos = np.zeros((max(mx, 1), 3), np.float32)
    bvel = np.zeros((max(mx, 1), 3), np.float32)
    nrm = np.zeros((max(mx, 1), 3), np.float32)
    qa, pq = _f32(np.asarray(q).reshape(-1, 3))
    ra, pr = _f32(model.particle_radius)
    fa, pf = _i32(model.particle_flags)
    wa, pw = _i32(model.particle_world)
    shapes = _shapes(model)
    n = lib.oracle_collide(V, pq, pr, pf, pw, S, ctypes.cast(shapes, ctypes.POINTER(OracleShape)), float(margin), mx,
                           particle.ctypes.data_as(c_int32_p), shape.ctypes.data_as(c_int32_p),
                           bpos.ctypes.data_as(c_float_p), bvel.ctypes.data_as(c_float_p), nrm.ctypes.data_as(c_float_p))
    n = min(n, mx)
    return particle[:n], shape[:n], bpos[:n], bvel[:n], nrm[:n]


def _elem(fn, is_double, *args):
    f = np.zeros(3, np.float64)
    h = np.zeros(9, np.float64)
    fn(is_double, *args, f.ctypes.data_as(c_double_p), h.ctypes.data_as(c_double_p))
    return f, h.reshape(3, 3)


def membrane(face, v_order, pos, anchor, tri_indices, pose, area, mu, lmbd, damping, dt, precision="f32"):
    lib = load()
    p, pp = _f64(np.asarray(pos).reshape(-1, 3))
    a, pa = _f64(np.asarray(anchor).reshape(-1, 3))
    t, pt = _i32(np.asarray(tri_indices).reshape(-1, 3))
    ps, pps = _f64(np.asarray(pose).reshape(4))
    return _elem(lib.oracle_membrane, 1 if precision == "f64" else 0, int(face), int(v_order), pp, pa, pt, pps,
                 float(area), float(mu), float(lmbd), float(damping), float(dt), p.shape[0])


def bending(edge, v_order, pos, anchor, edge_indices, rest_angle, rest_length, ke, kd, dt, precision="f32"):
    lib = load()
    p, pp = _f64(np.asarray(pos).reshape(-1, 3))
    a, pa = _f64(np.asarray(anchor).reshape(-1, 3))
    e, pe = _i32(np.asarray(edge_indices).reshape(-1, 4))
    return _elem(lib.oracle_bending, 1 if precision == "f64" else 0, int(edge), int(v_order), pp, pa, pe,
                 float(rest_angle), float(rest_length), float(ke), float(kd), float(dt), p.shape[0])


def contact(x, x_prev, body_pos, body_vel, normal, radius, margin, ke, kd, mu, friction_epsilon, dt, precision="f32"):
    lib = load()
    arrs = [_f64(np.asarray(v).reshape(3)) for v in (x, x_prev, body_pos, body_vel, normal)]
    return _elem(lib.oracle_contact, 1 if precision == "f64" else 0, *[p for _, p in arrs], float(radius), float(margin),
                 float(ke), float(kd), float(mu), float(friction_epsilon), float(dt))


def self_contact_norm(dis, radius, k, precision="f32"):
    out = np.zeros(2, np.float64)
    load().oracle_self_contact_norm(1 if precision == "f64" else 0, float(dis), float(radius), float(k),
                                    out.ctypes.data_as(c_double_p))
    return out[0], out[1]


def vt_contact(pos, anchor, radius, ke, kd, mu, friction_epsilon, dt, precision="f32"):
    """Vertex-triangle self-contact; pos/anchor rows a, b, c, p.  Returns (has, F[4,3], H[4,3,3])."""
    p, pp = _f64(np.asarray(pos).reshape(4, 3))
    a, pa = _f64(np.asarray(anchor).reshape(4, 3))
    f = np.zeros(12, np.float64)
    h = np.zeros(36, np.float64)
    has = load().oracle_vt_contact(1 if precision == "f64" else 0, pp, pa, float(radius), float(ke), float(kd),
                                   float(mu), float(friction_epsilon), float(dt), f.ctypes.data_as(c_double_p),
                                   h.ctypes.data_as(c_double_p))
    return bool(has), f.reshape(4, 3), h.reshape(4, 3, 3)


def ee_contact(pos, anchor, radius, ke, kd, mu, friction_epsilon, dt, parallel_epsilon=1e-5, precision="f32"):
    """Edge-edge self-contact; pos/anchor rows e0, e1, f0, f1.  Returns (has, F[2,3], H[2,3,3]) for e0, e1."""
    p, pp = _f64(np.asarray(pos).reshape(4, 3))
    a, pa = _f64(np.asarray(anchor).reshape(4, 3))
    f = np.zeros(6, np.float64)
    h = np.zeros(18, np.float64)
    has = load().oracle_ee_contact(1 if precision == "f64" else 0, pp, pa, float(radius), float(ke), float(kd),
                                   float(mu), float(friction_epsilon), float(dt), float(parallel_epsilon),
                                   f.ctypes.data_as(c_double_p), h.ctypes.data_as(c_double_p))
    return bool(has), f.reshape(2, 3), h.reshape(2, 3, 3)


def closest_edge_edge(p1, q1, p2, q2, eps=1e-5):
    pts, pp = _f64(np.stack([p1, q1, p2, q2]).reshape(12))
    out = np.zeros(3, np.float64)
    load().oracle_closest_edge_edge(pp, float(eps), out.ctypes.data_as(c_double_p))
    return out[0], out[1], out[2]


def triangle_closest_point(a, b, c, p):
    pts, pp = _f64(np.stack([a, b, c, p]).reshape(12))
    out = np.zeros(6, np.float64)
    load().oracle_triangle_closest_point(pp, out.ctypes.data_as(c_double_p))
    return out[:3], out[3:]
