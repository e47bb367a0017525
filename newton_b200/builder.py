"""ModelBuilder for the VBD cloth path (particles, triangles, bending hinges, static shapes).

Restates the cloth part of ``newton.ModelBuilder`` (``newton/_src/sim/builder.py``):

* ``add_particles``         builder.py:8340   (flags ACTIVE, world = current world)
* ``add_triangles``         builder.py:8543-8655: rest frame ``R = [e1, e2]`` from the first edge and
                            the normal, ``D = R^T [x1-x0, x2-x0]``, ``DmInv = D^-1``,
                            ``area = det(D)/2``; triangles with area <= 0 are dropped
* ``add_edges``             builder.py:8798-8880: rest angle ``atan2((n1 x n2).e, clip(n1.n2))``,
                            rest length ``|x_v1 - x_v0|``
* ``add_cloth_mesh``        builder.py:9071-9219: lumped mass ``+= density * area / 3`` per triangle
                            corner, one bending hinge per interior/boundary edge
* ``add_cloth_grid``        builder.py:8944-9069: grid triangulation, then per-particle ``mass`` and
                            pinned borders (flag cleared, mass 0) overwrite the lumped masses
* ``add_shape_plane/ground_plane/sphere/box``  builder.py:6599-6830 (static shapes only)
* ``color`` / ``set_coloring``                  builder.py:10130-10226
* ``add_builder``           merges a builder as a new world; color groups of independent worlds are
                            combined by size pairing (builder.py:2925-2937)
* ``finalize``              builder.py:10962-11070, :11796-11832 (inverse mass, adjacency CSR)

Builder math runs in float64 (numpy) and the model arrays are float32, as in the reference.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass, replace

import numpy as np

from .coloring import (
    ColoringAlgorithm,
    color_graph,
    combine_independent_coloring_plan,
    construct_trimesh_graph_edges,
)
from .mesh import MeshAdjacency
from .model import GeoType, Model, ParticleFlags, ShapeFlags


def _normalized(a: np.ndarray) -> np.ndarray:
    n = np.linalg.norm(a, axis=-1, keepdims=True)
    n[n == 0] = 1.0
    return a / n


def quat_to_matrix(q) -> np.ndarray:
    """Rotation matrix of a unit quaternion (x, y, z, w), evaluated in float32."""
    x, y, z, w = (np.float32(c) for c in q)
    one, two = np.float32(1.0), np.float32(2.0)
    return np.array(
        [
            [one - two * (y * y + z * z), two * (x * y - z * w), two * (x * z + y * w)],
            [two * (x * y + z * w), one - two * (x * x + z * z), two * (y * z - x * w)],
            [two * (x * z - y * w), two * (y * z + x * w), one - two * (x * x + y * y)],
        ],
        dtype=np.float32,
    )


def quat_between_vectors(a, b) -> tuple[float, float, float, float]:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    a = a / np.linalg.norm(a)
    b = b / np.linalg.norm(b)
    d = float(np.dot(a, b))
    if d > 1.0 - 1e-12:
        return (0.0, 0.0, 0.0, 1.0)
    if d < -1.0 + 1e-12:
        axis = np.cross(a, [1.0, 0.0, 0.0])
        if np.linalg.norm(axis) < 1e-6:
            axis = np.cross(a, [0.0, 1.0, 0.0])
        axis /= np.linalg.norm(axis)
        return (float(axis[0]), float(axis[1]), float(axis[2]), 0.0)
    c = np.cross(a, b)
    q = np.array([c[0], c[1], c[2], 1.0 + d])
    q /= np.linalg.norm(q)
    return tuple(float(v) for v in q)


class _Chunked:
    """A builder array kept as a list of appended chunks and concatenated on first read, so that
    appending many worlds stays linear in the total size."""

    def __set_name__(self, owner, name):
        self.key = "_chunks_" + name

    def __get__(self, obj, objtype=None):
        if obj is None:
            return self
        chunks = obj.__dict__[self.key]
        if len(chunks) > 1:
            chunks[:] = [np.concatenate(chunks)]
        return chunks[0]

    def __set__(self, obj, value):
        obj.__dict__[self.key] = [value]


class ModelBuilder:
    """Host-side construction of a cloth Model."""

    tri_indices = _Chunked()
    tri_poses = _Chunked()
    tri_materials = _Chunked()
    tri_areas = _Chunked()
    edge_indices = _Chunked()
    edge_rest_angle = _Chunked()
    edge_rest_length = _Chunked()
    edge_bending_properties = _Chunked()

    @dataclass
    class ShapeConfig:
        """``ModelBuilder.ShapeConfig`` defaults (builder.py:452-560) used by particle contact."""

        ke: float = 2.5e3
        kd: float = 100.0
        mu: float = 1.0
        margin: float = 0.0
        collide_particles: bool = True

        def copy(self):
            return replace(self)

    def __init__(self, up_axis: str = "Z", gravity: float = -9.81):
        axes = {"X": (1.0, 0.0, 0.0), "Y": (0.0, 1.0, 0.0), "Z": (0.0, 0.0, 1.0)}
        self.up_vector = axes[up_axis.upper()]
        self.gravity = gravity
        self.default_shape_cfg = ModelBuilder.ShapeConfig()
        self.default_particle_radius = 0.1
        self.default_tri_ke = 100.0
        self.default_tri_ka = 100.0
        self.default_tri_kd = 10.0
        self.default_tri_drag = 0.0
        self.default_tri_lift = 0.0
        self.default_edge_ke = 100.0
        self.default_edge_kd = 0.0
        self.current_world = -1
        self.world_count = 0
        # particles
        self._pq: list[np.ndarray] = []
        self._pqd: list[np.ndarray] = []
        self._pmass: list[np.ndarray] = []
        self._pradius: list[np.ndarray] = []
        self._pflags: list[np.ndarray] = []
        self._pworld: list[np.ndarray] = []
        self._pcache = None
        # triangles
        self.tri_indices = np.empty((0, 3), dtype=np.int32)
        self.tri_poses = np.empty((0, 2, 2), dtype=np.float64)
        self.tri_materials = np.empty((0, 5), dtype=np.float64)
        self.tri_areas = np.empty(0, dtype=np.float64)
        # bending hinges
        self.edge_indices = np.empty((0, 4), dtype=np.int32)
        self.edge_rest_angle = np.empty(0, dtype=np.float64)
        self.edge_rest_length = np.empty(0, dtype=np.float64)
        self.edge_bending_properties = np.empty((0, 2), dtype=np.float64)
        # shapes
        self.shape_type: list[int] = []
        self.shape_transform: list[tuple] = []
        self.shape_scale: list[tuple] = []
        self.shape_margin: list[float] = []
        self.shape_material_ke: list[float] = []
        self.shape_material_kd: list[float] = []
        self.shape_material_mu: list[float] = []
        self.shape_flags: list[int] = []
        self.shape_world: list[int] = []
        self.shape_body: list[int] = []
        # color groups as a merge plan: [(size, [(group, index offset), ...]), ...]
        self._color_plan: list = []

    def _append(self, name: str, arr: np.ndarray) -> None:
        self.__dict__["_chunks_" + name].append(arr)

    def _count(self, name: str) -> int:
        return int(sum(c.shape[0] for c in self.__dict__["_chunks_" + name]))

    @property
    def particle_color_groups(self) -> list[np.ndarray]:
        groups = [
            np.concatenate([np.asarray(g, dtype=np.int64) + off for g, off in chunks]).astype(np.int32)
            for _, chunks in self._color_plan
        ]
        self._color_plan = [(len(g), [(g, 0)]) for g in groups]
        return groups

    @particle_color_groups.setter
    def particle_color_groups(self, groups) -> None:
        self._color_plan = [(len(g), [(np.asarray(g, dtype=np.int32), 0)]) for g in groups]

    # ---------------------------------------------------------------- particles
    def _flush_particles(self):
        if self._pcache is None or len(self._pq) > 1:
            if self._pq:
                cat = {
                    "q": np.concatenate(self._pq),
                    "qd": np.concatenate(self._pqd),
                    "mass": np.concatenate(self._pmass),
                    "radius": np.concatenate(self._pradius),
                    "flags": np.concatenate(self._pflags),
                    "world": np.concatenate(self._pworld),
                }
            else:
                cat = {
                    "q": np.empty((0, 3)),
                    "qd": np.empty((0, 3)),
                    "mass": np.empty(0),
                    "radius": np.empty(0),
                    "flags": np.empty(0, np.int32),
                    "world": np.empty(0, np.int32),
                }
            self._pq, self._pqd, self._pmass = [cat["q"]], [cat["qd"]], [cat["mass"]]
            self._pradius, self._pflags, self._pworld = [cat["radius"]], [cat["flags"]], [cat["world"]]
            self._pcache = cat
        return self._pcache

    @property
    def particle_count(self) -> int:
        return int(sum(len(a) for a in self._pmass))

    @property
    def particle_q(self) -> np.ndarray:
        return self._flush_particles()["q"]

    @property
    def particle_qd(self) -> np.ndarray:
        return self._flush_particles()["qd"]

    @property
    def particle_mass(self) -> np.ndarray:
        return self._flush_particles()["mass"]

    @property
    def particle_radius(self) -> np.ndarray:
        return self._flush_particles()["radius"]

    @property
    def particle_flags(self) -> np.ndarray:
        return self._flush_particles()["flags"]

    @property
    def particle_world(self) -> np.ndarray:
        return self._flush_particles()["world"]

    @property
    def tri_count(self) -> int:
        return self._count("tri_indices")

    @property
    def edge_count(self) -> int:
        return self._count("edge_indices")

    @property
    def shape_count(self) -> int:
        return len(self.shape_type)

    def add_particles(self, pos, vel, mass, radius=None, flags=None) -> None:
        pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
        n = pos.shape[0]
        vel = np.broadcast_to(np.asarray(vel, dtype=np.float64).reshape(-1, 3), (n, 3)).copy()
        mass = np.broadcast_to(np.asarray(mass, dtype=np.float64).reshape(-1), (n,)).copy()
        if radius is None:
            radius = self.default_particle_radius
        radius = np.broadcast_to(np.asarray(radius, dtype=np.float64).reshape(-1), (n,)).copy()
        if flags is None:
            flags = ParticleFlags.ACTIVE
        flags = np.broadcast_to(np.asarray(flags, dtype=np.int32).reshape(-1), (n,)).copy()
        self._pq.append(pos)
        self._pqd.append(vel)
        self._pmass.append(mass)
        self._pradius.append(radius)
        self._pflags.append(flags)
        self._pworld.append(np.full(n, self.current_world, dtype=np.int32))
        self._pcache = None

    def add_particle(self, pos, vel, mass, radius=None, flags=None) -> int:
        idx = self.particle_count
        self.add_particles([pos], [vel], [mass], None if radius is None else [radius], None if flags is None else [flags])
        return idx

    def set_particle_mass(self, indices, mass) -> None:
        self._flush_particles()["mass"][np.asarray(indices)] = mass

    def set_particle_flags(self, indices, flags) -> None:
        self._flush_particles()["flags"][np.asarray(indices)] = flags

    # ---------------------------------------------------------------- triangles / hinges
    def add_triangles(self, i, j, k, tri_ke=None, tri_ka=None, tri_kd=None, tri_drag=None, tri_lift=None) -> np.ndarray:
        """Rest pose, area and material per triangle; returns all areas (0 for dropped ones)."""
        q = self.particle_q
        i = np.asarray(i, dtype=np.int64)
        j = np.asarray(j, dtype=np.int64)
        k = np.asarray(k, dtype=np.int64)
        p, qq, r = q[i], q[j], q[k]
        qp = qq - p
        rp = r - p
        n = _normalized(np.cross(qp, rp))
        e1 = _normalized(qp)
        e2 = _normalized(np.cross(n, e1))
        R = np.concatenate((e1[..., None], e2[..., None]), axis=-1)
        M = np.concatenate((qp[..., None], rp[..., None]), axis=-1)
        D = np.matmul(R.transpose(0, 2, 1), M)
        areas = np.linalg.det(D) / 2.0
        areas[areas < 0.0] = 0.0
        valid = np.flatnonzero(areas > 0.0)
        if len(valid) < len(areas):
            warnings.warn("inverted or degenerate triangle elements", stacklevel=2)
        D[areas == 0.0] = np.eye(2)[None, ...]
        inv_D = np.linalg.inv(D)
        nt = len(areas)

        def col(v, d):
            v = d if v is None else v
            return np.broadcast_to(np.asarray(v, dtype=np.float64).reshape(-1), (nt,))

        mats = np.stack(
            [
                col(tri_ke, self.default_tri_ke),
                col(tri_ka, self.default_tri_ka),
                col(tri_kd, self.default_tri_kd),
                col(tri_drag, self.default_tri_drag),
                col(tri_lift, self.default_tri_lift),
            ],
            axis=1,
        )
        inds = np.stack([i[valid], j[valid], k[valid]], axis=1).astype(np.int32)
        self._append("tri_indices", inds)
        self._append("tri_poses", inv_D[valid])
        self._append("tri_materials", mats[valid])
        self._append("tri_areas", areas[valid])
        return areas

    def add_edges(self, i, j, k, l, rest=None, edge_ke=None, edge_kd=None) -> None:
        """Bending hinges ``[o0, o1, v0, v1]``; triangles (o0, v0, v1) and (o1, v1, v0)."""
        i_ = np.asarray(i, dtype=np.int64)
        j_ = np.asarray(j, dtype=np.int64)
        k_ = np.asarray(k, dtype=np.int64)
        l_ = np.asarray(l, dtype=np.int64)
        q = self.particle_q
        x3, x4 = q[k_], q[l_]
        if rest is None:
            rest = np.zeros(len(i_), dtype=np.float64)
            valid = (i_ != -1) & (j_ != -1)
            x1, x2 = q[i_[valid]], q[j_[valid]]
            n1 = _normalized(np.cross(x3[valid] - x1, x4[valid] - x1))
            n2 = _normalized(np.cross(x4[valid] - x2, x3[valid] - x2))
            e = _normalized(x4[valid] - x3[valid])
            cos_t = np.clip((n1 * n2).sum(-1), -1.0, 1.0)
            sin_t = (np.cross(n1, n2) * e).sum(-1)
            rest[valid] = np.arctan2(sin_t, cos_t)
        ne = len(i_)

        def col(v, d):
            v = d if v is None else v
            return np.broadcast_to(np.asarray(v, dtype=np.float64).reshape(-1), (ne,))

        self._append("edge_indices", np.stack([i_, j_, k_, l_], axis=1).astype(np.int32))
        self._append("edge_rest_angle", np.asarray(rest, dtype=np.float64))
        self._append("edge_rest_length", np.linalg.norm(x4 - x3, axis=1))
        props = np.stack([col(edge_ke, self.default_edge_ke), col(edge_kd, self.default_edge_kd)], axis=1)
        self._append("edge_bending_properties", props)

    def add_cloth_mesh(self, *, pos, rot, scale, vel, vertices, indices, density, tri_ke=None, tri_ka=None,
                       tri_kd=None, tri_drag=None, tri_lift=None, edge_ke=None, edge_kd=None, particle_radius=None,
                       add_springs=False) -> None:
        if add_springs:
            raise NotImplementedError("springs are not part of the VBD cloth path built here")
        tri_ke = self.default_tri_ke if tri_ke is None else tri_ke
        tri_ka = self.default_tri_ka if tri_ka is None else tri_ka
        tri_kd = self.default_tri_kd if tri_kd is None else tri_kd
        tri_drag = self.default_tri_drag if tri_drag is None else tri_drag
        tri_lift = self.default_tri_lift if tri_lift is None else tri_lift
        edge_ke = self.default_edge_ke if edge_ke is None else edge_ke
        edge_kd = self.default_edge_kd if edge_kd is None else edge_kd
        particle_radius = self.default_particle_radius if particle_radius is None else particle_radius
        verts = np.asarray(vertices, dtype=np.float64).reshape(-1, 3) * scale
        rmat = quat_to_matrix(rot)
        verts3 = np.dot(verts, rmat.T) + np.asarray(pos, dtype=np.float64)
        nv = verts3.shape[0]
        start_vertex = self.particle_count
        start_tri = self.tri_count
        self.add_particles(verts3, np.tile(np.asarray(vel, dtype=np.float64), (nv, 1)), np.zeros(nv), particle_radius)
        inds = (start_vertex + np.asarray(indices, dtype=np.int64)).reshape(-1, 3)
        areas = self.add_triangles(inds[:, 0], inds[:, 1], inds[:, 2], tri_ke, tri_ka, tri_kd, tri_drag, tri_lift)
        mass = self._flush_particles()["mass"]
        np.add.at(mass, inds.reshape(-1), np.repeat(density * areas / 3.0, 3))
        end_tri = self.tri_count
        if end_tri > start_tri:
            e = self._edge_table(self.tri_indices[start_tri:end_tri])
            if e.shape[0]:
                self.add_edges(e[:, 0], e[:, 1], e[:, 2], e[:, 3], edge_ke=edge_ke, edge_kd=edge_kd)

    @staticmethod
    def grid_mesh(dim_x: int, dim_y: int, cell_x: float, cell_y: float, reverse_winding: bool = False):
        """Vertices and triangle indices of ``add_cloth_grid``'s planar grid (builder.py:9010-9029)."""
        ys, xs = np.meshgrid(np.arange(dim_y + 1), np.arange(dim_x + 1), indexing="ij")
        vertices = np.stack([xs.reshape(-1) * cell_x, ys.reshape(-1) * cell_y, np.zeros(xs.size)], axis=1)
        yy, xx = np.meshgrid(np.arange(1, dim_y + 1), np.arange(1, dim_x + 1), indexing="ij")
        xx, yy = xx.reshape(-1), yy.reshape(-1)
        w = dim_x + 1
        v0 = (yy - 1) * w + (xx - 1)
        v1 = (yy - 1) * w + xx
        v2 = yy * w + xx
        v3 = yy * w + (xx - 1)
        if reverse_winding:
            tris = np.stack([v0, v1, v2, v0, v2, v3], axis=1)
        else:
            tris = np.stack([v0, v1, v3, v1, v2, v3], axis=1)
        return vertices, tris.reshape(-1).astype(np.int64)

    def add_cloth_grid(self, *, pos, rot, vel, dim_x, dim_y, cell_x, cell_y, mass, reverse_winding=False,
                       fix_left=False, fix_right=False, fix_top=False, fix_bottom=False, tri_ke=None, tri_ka=None,
                       tri_kd=None, tri_drag=None, tri_lift=None, edge_ke=None, edge_kd=None, particle_radius=None):
        vertices, indices = self.grid_mesh(dim_x, dim_y, cell_x, cell_y, reverse_winding)
        start_vertex = self.particle_count
        total_mass = mass * (dim_x + 1) * (dim_x + 1)
        total_area = cell_x * cell_y * dim_x * dim_y
        self.add_cloth_mesh(pos=pos, rot=rot, scale=1.0, vel=vel, vertices=vertices, indices=indices,
                            density=total_mass / total_area, tri_ke=tri_ke, tri_ka=tri_ka, tri_kd=tri_kd,
                            tri_drag=tri_drag, tri_lift=tri_lift, edge_ke=edge_ke, edge_kd=edge_kd,
                            particle_radius=particle_radius)
        ys, xs = np.meshgrid(np.arange(dim_y + 1), np.arange(dim_x + 1), indexing="ij")
        xs, ys = xs.reshape(-1), ys.reshape(-1)
        fixed = (fix_left & (xs == 0)) | (fix_right & (xs == dim_x)) | (fix_bottom & (ys == 0)) | (fix_top & (ys == dim_y))
        cache = self._flush_particles()
        sl = slice(start_vertex, start_vertex + len(xs))
        cache["mass"][sl] = np.where(fixed, 0.0, mass)
        cache["flags"][sl] = np.where(fixed, cache["flags"][sl] & ~ParticleFlags.ACTIVE, ParticleFlags.ACTIVE)

    # ---------------------------------------------------------------- shapes
    def _add_shape(self, geo_type, xform, scale, cfg, body=-1) -> int:
        if body != -1:
            raise NotImplementedError("only static shapes (body = -1) are supported on the VBD cloth path")
        cfg = self.default_shape_cfg if cfg is None else cfg
        p = tuple(float(v) for v in xform[0])
        q = tuple(float(v) for v in xform[1])
        self.shape_type.append(int(geo_type))
        self.shape_transform.append(p + q)
        self.shape_scale.append(tuple(float(v) for v in scale))
        self.shape_margin.append(float(cfg.margin))
        self.shape_material_ke.append(float(cfg.ke))
        self.shape_material_kd.append(float(cfg.kd))
        self.shape_material_mu.append(float(cfg.mu))
        flags = ShapeFlags.VISIBLE | ShapeFlags.COLLIDE_SHAPES
        if cfg.collide_particles:
            flags |= ShapeFlags.COLLIDE_PARTICLES
        self.shape_flags.append(int(flags))
        self.shape_world.append(self.current_world)
        self.shape_body.append(body)
        return len(self.shape_type) - 1

    def add_shape_plane(self, plane=(0.0, 0.0, 1.0, 0.0), *, xform=None, width=10.0, length=10.0, body=-1, cfg=None) -> int:
        if xform is None:
            normal = np.array(plane[:3], dtype=np.float64)
            norm = np.linalg.norm(normal)
            normal /= norm
            d = plane[3] / norm
            pos = -d * normal
            xform = (tuple(pos), quat_between_vectors((0.0, 0.0, 1.0), normal))
        return self._add_shape(GeoType.PLANE, xform, (width, length, 0.0), cfg, body)

    def add_ground_plane(self, *, height: float = 0.0, cfg=None) -> int:
        return self.add_shape_plane(plane=(*self.up_vector, -height), width=0.0, length=0.0, cfg=cfg)

    def add_shape_sphere(self, body: int = -1, *, xform=None, radius: float = 1.0, cfg=None) -> int:
        xform = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 1.0)) if xform is None else xform
        return self._add_shape(GeoType.SPHERE, xform, (radius, 0.0, 0.0), cfg, body)

    def add_shape_box(self, body: int = -1, *, xform=None, hx: float = 0.5, hy: float = 0.5, hz: float = 0.5, cfg=None) -> int:
        xform = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 1.0)) if xform is None else xform
        return self._add_shape(GeoType.BOX, xform, (hx, hy, hz), cfg, body)

    # ---------------------------------------------------------------- connectivity and coloring
    # The four steps below run in the library's native code (mesh.py, coloring.py): the first three
    # on the GPU for large meshes (``setup_device``), the coloring on the host.  They are methods so
    # that a subclass can supply the same tables another way; the model data the rest of the
    # builder produces does not depend on how.

    # Where the edge table, vertex CSR and conflict edges are computed: "auto" (the current CUDA
    # device, when one is available, for meshes of at least SETUP_DEVICE_MIN_ELEMENTS elements;
    # otherwise the host), None (always the host) or a CUDA device.  The tables are the same.
    setup_device = "auto"
    SETUP_DEVICE_MIN_ELEMENTS = 1 << 16

    def _setup_dev(self, elements: int):
        d = self.setup_device
        if d != "auto":
            return d
        if elements < self.SETUP_DEVICE_MIN_ELEMENTS:
            return None
        import torch

        return torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None

    def _edge_table(self, tri_indices) -> np.ndarray:
        """Bending-edge table ``[o0, o1, v0, v1]`` of one mesh (``utils/mesh.py:465-531``)."""
        return MeshAdjacency(tri_indices, device=self._setup_dev(len(tri_indices))).edge_indices

    def _vertex_adjacency(self, tri_indices, edge_indices, particle_count: int) -> MeshAdjacency:
        """Per-vertex element CSR of the finalized model (``utils/mesh.py:595-926``)."""
        dev = self._setup_dev(len(tri_indices) + len(edge_indices))
        return MeshAdjacency(tri_indices, edge_indices, device=dev).init_vertex_adjacency(particle_count)

    def _conflict_edges(self, tri_indices, tri_mask, bend_indices, bend_mask) -> np.ndarray:
        """Canonical conflict-graph edges (``graph_coloring.py:99-197``)."""
        n = (0 if tri_indices is None else len(tri_indices)) + (0 if bend_indices is None else len(bend_indices))
        return construct_trimesh_graph_edges(tri_indices, tri_mask, bend_indices, bend_mask, device=self._setup_dev(n))

    def _color_graph(self, num_nodes, edges, balance_colors, target_ratio, algorithm) -> list[np.ndarray]:
        """Color groups of the conflict graph (``graph_coloring.py:243-311``)."""
        return color_graph(num_nodes, edges, balance_colors, target_ratio, algorithm)

    def set_coloring(self, particle_color_groups) -> None:
        self.particle_color_groups = [np.asarray(g, dtype=np.int32) for g in particle_color_groups]

    def coloring_graph_edges(self, include_bending: bool = False) -> np.ndarray:
        tri_mask = None
        if self.tri_count:
            tri_mask = self.tri_materials[:, 0] * self.tri_materials[:, 1]
        bend, bend_mask = None, None
        if include_bending and self.edge_count:
            bend = self.edge_indices
            props = self.edge_bending_properties
            bend_mask = (props[:, 0] != 0.0) | (props[:, 1] != 0.0)
        return self._conflict_edges(self.tri_indices if self.tri_count else None, tri_mask, bend, bend_mask)

    def color(self, include_bending: bool = False, balance_colors: bool = True, target_max_min_color_ratio: float = 1.1,
              coloring_algorithm: ColoringAlgorithm = ColoringAlgorithm.MCS) -> None:
        if self.particle_count == 0:
            self.particle_color_groups = []
            return
        edges = self.coloring_graph_edges(include_bending)
        if len(edges) > 0:
            self.particle_color_groups = self._color_graph(self.particle_count, edges, balance_colors,
                                                     target_max_min_color_ratio, coloring_algorithm)
        else:
            self.particle_color_groups = [np.arange(self.particle_count, dtype=np.int32)]

    # ---------------------------------------------------------------- worlds
    def begin_world(self) -> None:
        self.current_world = self.world_count
        self.world_count += 1

    def end_world(self) -> None:
        self.current_world = -1

    def add_builder(self, builder: "ModelBuilder", world: int | None = None) -> None:
        """Append ``builder`` (as world ``world``; a new world when None) with index offsets."""
        if world is None:
            world = self.world_count
            self.world_count += 1
        else:
            self.world_count = max(self.world_count, world + 1)
        start = self.particle_count
        src = builder._flush_particles()
        if len(src["mass"]):
            self._pq.append(src["q"].copy())
            self._pqd.append(src["qd"].copy())
            self._pmass.append(src["mass"].copy())
            self._pradius.append(src["radius"].copy())
            self._pflags.append(src["flags"].copy())
            self._pworld.append(np.full(len(src["mass"]), world, dtype=np.int32))
            self._pcache = None
        self._append("tri_indices", builder.tri_indices + start)
        self._append("tri_poses", builder.tri_poses)
        self._append("tri_materials", builder.tri_materials)
        self._append("tri_areas", builder.tri_areas)
        e = builder.edge_indices.copy()
        e[e >= 0] += start
        self._append("edge_indices", e)
        self._append("edge_rest_angle", builder.edge_rest_angle)
        self._append("edge_rest_length", builder.edge_rest_length)
        self._append("edge_bending_properties", builder.edge_bending_properties)
        for s in range(builder.shape_count):
            self.shape_type.append(builder.shape_type[s])
            self.shape_transform.append(builder.shape_transform[s])
            self.shape_scale.append(builder.shape_scale[s])
            self.shape_margin.append(builder.shape_margin[s])
            self.shape_material_ke.append(builder.shape_material_ke[s])
            self.shape_material_kd.append(builder.shape_material_kd[s])
            self.shape_material_mu.append(builder.shape_material_mu[s])
            self.shape_flags.append(builder.shape_flags[s])
            self.shape_world.append(world if builder.shape_world[s] == -1 else builder.shape_world[s])
            self.shape_body.append(builder.shape_body[s])
        if builder._color_plan:
            other = [(size, [(g, off + start) for g, off in chunks]) for size, chunks in builder._color_plan]
            self._color_plan = combine_independent_coloring_plan(self._color_plan, other)

    def add_world(self, builder: "ModelBuilder") -> None:
        """``ModelBuilder.add_world`` (``builder.py:4016``): append ``builder`` as a new world."""
        self.add_builder(builder, world=None)

    # ---------------------------------------------------------------- finalize
    def finalize(self, device="cuda:0", requires_grad: bool = False) -> Model:
        p = self._flush_particles()
        m = Model(device)
        V = len(p["mass"])
        m.world_count = max(self.world_count, 1)
        m.particle_count = V
        m.particle_q = p["q"].astype(np.float32)
        m.particle_qd = p["qd"].astype(np.float32)
        ms = p["mass"].astype(np.float32)
        m.particle_mass = ms
        m.particle_inv_mass = np.divide(np.float32(1.0), ms, out=np.zeros_like(ms), where=ms != 0.0).astype(np.float32)
        m.particle_radius = p["radius"].astype(np.float32)
        m.particle_flags = p["flags"].astype(np.int32)
        m.particle_world = p["world"].astype(np.int32)
        m.particle_color_groups = [np.asarray(g, dtype=np.int32) for g in self.particle_color_groups]
        colors = np.full(V, -1, dtype=np.int32)
        for c, g in enumerate(m.particle_color_groups):
            colors[g] = c
        m.particle_colors = colors
        m.tri_count = self.tri_count
        m.tri_indices = self.tri_indices.astype(np.int32).reshape(-1, 3)
        m.tri_poses = self.tri_poses.astype(np.float32).reshape(-1, 2, 2)
        m.tri_materials = self.tri_materials.astype(np.float32).reshape(-1, 5)
        m.tri_areas = self.tri_areas.astype(np.float32)
        m.edge_count = self.edge_count
        m.edge_indices = self.edge_indices.astype(np.int32).reshape(-1, 4)
        m.edge_rest_angle = self.edge_rest_angle.astype(np.float32)
        m.edge_rest_length = self.edge_rest_length.astype(np.float32)
        m.edge_bending_properties = self.edge_bending_properties.astype(np.float32).reshape(-1, 2)
        m.soft_mesh_adjacency = self._vertex_adjacency(m.tri_indices, m.edge_indices, V)
        S = self.shape_count
        m.shape_count = S
        m.shape_type = np.asarray(self.shape_type, dtype=np.int32)
        m.shape_transform = np.asarray(self.shape_transform, dtype=np.float32).reshape(S, 7)
        m.shape_scale = np.asarray(self.shape_scale, dtype=np.float32).reshape(S, 3)
        m.shape_margin = np.asarray(self.shape_margin, dtype=np.float32)
        m.shape_material_ke = np.asarray(self.shape_material_ke, dtype=np.float32)
        m.shape_material_kd = np.asarray(self.shape_material_kd, dtype=np.float32)
        m.shape_material_mu = np.asarray(self.shape_material_mu, dtype=np.float32)
        m.shape_flags = np.asarray(self.shape_flags, dtype=np.int32)
        m.shape_world = np.asarray(self.shape_world, dtype=np.int32)
        m.shape_body = np.asarray(self.shape_body, dtype=np.int32)
        g = np.asarray(self.up_vector, dtype=np.float64) * self.gravity
        m.gravity = np.tile(g.astype(np.float32), (m.world_count, 1))
        return m
