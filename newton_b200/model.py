"""Data containers of the VBD cloth path: Model, State, Control, Contacts.

Mirrors the particle/cloth part of ``newton.Model`` (``newton/_src/sim/model.py:298``),
``newton.State`` (``state.py:57``), ``newton.Control`` and the soft-contact part of
``newton.Contacts`` (``contacts.py:327-345``).  Host arrays are numpy (the layout and dtypes of
the reference's ``wp.array``s); state and contact buffers are torch tensors on the model device.
"""

from __future__ import annotations

import ctypes

from enum import IntEnum

import numpy as np
import torch

from . import _lib


class ModelFlags(IntEnum):
    """Which parts of a Model changed (``newton.ModelFlags``, ``sim/enums.py:8-57``), for
    ``SolverBase.notify_model_changed``."""

    JOINT_PROPERTIES = 1 << 0
    JOINT_DOF_PROPERTIES = 1 << 1
    BODY_PROPERTIES = 1 << 2
    BODY_INERTIAL_PROPERTIES = 1 << 3
    SHAPE_PROPERTIES = 1 << 4
    MODEL_PROPERTIES = 1 << 5
    CONSTRAINT_PROPERTIES = 1 << 6
    TENDON_PROPERTIES = 1 << 7
    ACTUATOR_PROPERTIES = 1 << 8
    ALL = (1 << 9) - 1


class ParticleFlags:
    """``newton.ParticleFlags`` (``geometry/flags.py:8``)."""

    ACTIVE = 1 << 0
    PROXY = 1 << 1


class ShapeFlags:
    """``newton.ShapeFlags`` (``geometry/flags.py:27``)."""

    VISIBLE = 1 << 0
    COLLIDE_SHAPES = 1 << 1
    COLLIDE_PARTICLES = 1 << 2
    SITE = 1 << 3


class GeoType:
    """``newton.GeoType`` values (``geometry/types.py:70``) of the supported static shapes."""

    PLANE = 1
    SPHERE = 3
    BOX = 7


class State:
    """Time-varying particle state (``state.py:57``)."""

    def __init__(self):
        self.particle_q: torch.Tensor | None = None
        self.particle_qd: torch.Tensor | None = None
        self.particle_f: torch.Tensor | None = None
        self.body_q = None
        self.body_qd = None

    @property
    def particle_count(self) -> int:
        return 0 if self.particle_q is None else int(self.particle_q.shape[0])

    def clear_forces(self) -> None:
        """``State.clear_forces`` (``state.py:189``)."""
        if self.particle_f is not None:
            self.particle_f.zero_()

    def assign(self, other: "State") -> None:
        """``State.assign`` (``state.py:202``): copy another state's arrays into this one."""
        for name in ("particle_q", "particle_qd", "particle_f"):
            src, dst = getattr(other, name), getattr(self, name)
            if src is not None and dst is not None:
                dst.copy_(src)


class Control:
    """``newton.Control``; the particle path reads nothing from it."""


class Contacts:
    """Soft-contact records in the reference layout (``contacts.py:327-345``)."""

    def __init__(self, soft_contact_max: int, device):
        n = max(int(soft_contact_max), 0)
        self.soft_contact_max = n
        dev = torch.device(device)
        self.soft_contact_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.soft_contact_particle = torch.zeros(n, dtype=torch.int32, device=dev)
        self.soft_contact_indices = torch.full((n, 3), -1, dtype=torch.int32, device=dev)
        self.soft_contact_barycentric = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.soft_contact_shape = torch.zeros(n, dtype=torch.int32, device=dev)
        self.soft_contact_body_pos = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.soft_contact_body_vel = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.soft_contact_normal = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self._c = None

    def c_struct(self) -> _lib.VbdContacts:
        if self._c is None:
            c = _lib.VbdContacts()
            c.soft_contact_max = self.soft_contact_max
            c.soft_contact_count = self.soft_contact_count.data_ptr()
            c.soft_contact_particle = self.soft_contact_particle.data_ptr()
            c.soft_contact_indices = self.soft_contact_indices.data_ptr()
            c.soft_contact_barycentric = self.soft_contact_barycentric.data_ptr()
            c.soft_contact_shape = self.soft_contact_shape.data_ptr()
            c.soft_contact_body_pos = self.soft_contact_body_pos.data_ptr()
            c.soft_contact_body_vel = self.soft_contact_body_vel.data_ptr()
            c.soft_contact_normal = self.soft_contact_normal.data_ptr()
            self._c = c
        return self._c

    def count(self) -> int:
        return min(int(self.soft_contact_count.item()), self.soft_contact_max)


class DeviceModel:
    """Owner of a ``VbdModel*`` (``vbd_model_create``) built from a finalized Model."""

    def __init__(self, model: "Model"):
        lib = _lib.load()
        self._keep = []
        d = _lib.VbdModelDesc()

        def f32(a, shape=None):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
            self._keep.append(a)
            return _lib.as_f32p(a) if a.size else None

        def i32(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
            self._keep.append(a)
            return _lib.as_i32p(a) if a.size else None

        d.particle_count = model.particle_count
        d.tri_count = model.tri_count
        d.edge_count = model.edge_count
        d.shape_count = model.shape_count
        d.color_count = len(model.particle_color_groups)
        d.particle_mass = f32(model.particle_mass)
        d.particle_inv_mass = f32(model.particle_inv_mass)
        d.particle_radius = f32(model.particle_radius)
        d.particle_flags = i32(model.particle_flags)
        d.particle_world = i32(model.particle_world)
        d.tri_indices = i32(model.tri_indices)
        d.tri_poses = f32(model.tri_poses)
        d.tri_materials = f32(model.tri_materials)
        d.tri_areas = f32(model.tri_areas)
        d.edge_indices = i32(model.edge_indices)
        d.edge_rest_angle = f32(model.edge_rest_angle)
        d.edge_rest_length = f32(model.edge_rest_length)
        d.edge_bending_properties = f32(model.edge_bending_properties)
        adj = model.soft_mesh_adjacency
        d.v_adj_tris_offsets = i32(adj.v_adj_tris_offsets)
        d.v_adj_tris = i32(adj.v_adj_tris)
        d.v_adj_edges_offsets = i32(adj.v_adj_edges_offsets)
        d.v_adj_edges = i32(adj.v_adj_edges)
        offs, flat = model.color_group_csr()
        d.color_group_offsets = i32(offs)
        d.color_group_particles = i32(flat)
        g = np.asarray(model.gravity, dtype=np.float32).reshape(-1, 3)[0]
        for k in range(3):
            d.gravity[k] = float(g[k])
        d.soft_contact_ke = float(np.float32(model.soft_contact_ke))
        d.soft_contact_kd = float(np.float32(model.soft_contact_kd))
        d.soft_contact_mu = float(np.float32(model.soft_contact_mu))
        shapes = (_lib.VbdShape * max(model.shape_count, 1))()
        for s in range(model.shape_count):
            sh = shapes[s]
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
        self._keep.append(shapes)
        d.shapes = ctypes.cast(shapes, ctypes.POINTER(_lib.VbdShape))
        d.particle_q = f32(model.particle_q)
        handle = ctypes.c_void_p()
        with torch.cuda.device(model.device):
            _lib.check(lib.vbd_model_create(ctypes.byref(d), ctypes.byref(handle)))
        self.handle = handle
        self._lib = lib
        self._keep = None  # arrays were copied by vbd_model_create

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.vbd_model_destroy(h)
            except Exception:
                pass
            self.handle = None


class Model:
    """Finalized particle/cloth model (``model.py:298``) -- produced by ``ModelBuilder.finalize``."""

    def __init__(self, device="cuda:0"):
        self.device = torch.device(device)
        self.requires_grad = False
        self.world_count = 1
        self.particle_count = 0
        self.tri_count = 0
        self.edge_count = 0
        self.shape_count = 0
        self.body_count = 0
        self.soft_contact_ke = 1.0e3
        self.soft_contact_kd = 10.0
        self.soft_contact_mu = 0.5
        self.particle_color_groups: list[np.ndarray] = []
        self._device_model = None

    # -- state factories -------------------------------------------------------------------
    def state(self, requires_grad: bool | None = None) -> State:
        """``Model.state`` (``model.py:1828``): a fresh State with copies of the initial arrays."""
        s = State()
        s.particle_q = torch.tensor(self.particle_q, dtype=torch.float32, device=self.device).reshape(-1, 3)
        s.particle_qd = torch.tensor(self.particle_qd, dtype=torch.float32, device=self.device).reshape(-1, 3)
        s.particle_f = torch.zeros_like(s.particle_q)
        return s

    def control(self, clone_variables: bool = True) -> Control:
        return Control()

    def contacts(self, soft_contact_max: int | None = None) -> Contacts:
        n = self.particle_count * self.shape_count if soft_contact_max is None else soft_contact_max
        return Contacts(n, self.device)

    # -- helpers ---------------------------------------------------------------------------
    def color_group_csr(self) -> tuple[np.ndarray, np.ndarray]:
        groups = [np.asarray(g, dtype=np.int32).reshape(-1) for g in self.particle_color_groups]
        offs = np.zeros(len(groups) + 1, dtype=np.int32)
        if groups:
            offs[1:] = np.cumsum([len(g) for g in groups])
            flat = np.concatenate(groups).astype(np.int32)
        else:
            flat = np.empty(0, dtype=np.int32)
        return offs, flat

    def device_model(self) -> DeviceModel:
        if self._device_model is None:
            if self.device.type != "cuda":
                raise RuntimeError("the VBD CUDA library needs a model on a CUDA device")
            self._device_model = DeviceModel(self)
        return self._device_model

    def set_gravity(self, gravity, world: int | None = None) -> None:
        """``Model.set_gravity`` (``model.py:1958-1991``): one vector for every world, a per-world
        [world_count, 3] array, or one world's vector.  As in the reference, call the solver's
        ``notify_model_changed(ModelFlags.MODEL_PROPERTIES)`` afterwards when a solver exists (the
        device copy of the model is rebuilt on its next use either way)."""
        g = np.asarray(gravity, dtype=np.float32)
        cur = np.array(np.asarray(self.gravity, dtype=np.float32).reshape(-1, 3))
        if world is not None:
            if g.shape != (3,):
                raise ValueError("Expected single gravity vector (3,) when world is specified")
            if world < 0 or world >= self.world_count:
                raise IndexError(f"world {world} out of range [0, {self.world_count})")
            cur[world] = g
        elif g.ndim == 1:
            cur[:] = g
        else:
            if len(g) != self.world_count:
                raise ValueError(f"Expected {self.world_count} gravity vectors, got {len(g)}")
            cur = g.reshape(-1, 3).copy()
        self.gravity = cur
        self._device_model = None

    def notify_model_changed(self) -> None:
        """Drop the device copy so the next solver/pipeline use rebuilds it from the host arrays."""
        self._device_model = None
