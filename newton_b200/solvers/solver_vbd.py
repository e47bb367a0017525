"""``SolverVBD`` for particles/cloth on B200, behind the reference's solver interface.

Drop-in for the particle path of ``newton.solvers.SolverVBD``
(``newton/_src/solvers/vbd/solver_vbd.py:92``): same constructor keywords for the particle path,
same ``step(state_in, state_out, control, contacts, dt)`` contract, same state aliasing --
``state_in.particle_q`` is overwritten with the solved positions (the reference keeps its
Gauss-Seidel iterate there, ``solver_vbd.py:2100``/``:2702``) and ``state_out.particle_q``/
``particle_qd`` receive the result (``:2704``, ``:3158-3169``).

Every step runs in ``libvbd_b200.so`` (``vbd_step``): one forward kernel, ``iterations x colors``
sweep kernels and one finalize kernel, replayed from a cached CUDA graph.  There is no CPU or
eager fallback: without the library or a CUDA device the constructor raises.
"""

from __future__ import annotations

import ctypes
import warnings

import numpy as np
import torch

from .. import _lib
from ..model import Contacts, Control, Model, ModelFlags, State
from .solver import SolverBase


class SolverVBD(SolverBase):
    def __init__(
        self,
        model: Model,
        *,
        iterations: int = 10,
        friction_epsilon: float = 1e-2,
        integrate_with_external_rigid_solver: bool = False,
        particle_enable_self_contact: bool = False,
        particle_self_contact_radius: float = 0.2,
        particle_self_contact_margin: float = 0.2,
        particle_conservative_bound_relaxation: float = 0.85,
        particle_vertex_contact_buffer_size: int = 32,
        particle_edge_contact_buffer_size: int = 64,
        particle_collision_detection_interval: int = 0,
        particle_edge_parallel_epsilon: float = 1e-5,
        particle_enable_tile_solve: bool = True,
        particle_topological_contact_filter_threshold: int = 2,
        particle_rest_shape_contact_exclusion_radius: float = 0.0,
        particle_external_vertex_contact_filtering_map: dict | None = None,
        particle_external_edge_contact_filtering_map: dict | None = None,
        lanes_per_vertex: int = 0,
        block_size: int = 0,
        contacts_per_vertex: int = 4,
        use_cuda_graph: bool = True,
        resident_step: bool = False,
    ):
        super().__init__(model)
        self.iterations = int(iterations)
        self.friction_epsilon = float(friction_epsilon)
        self.integrate_with_external_rigid_solver = integrate_with_external_rigid_solver
        self.particle_enable_self_contact = particle_enable_self_contact
        self.particle_self_contact_radius = particle_self_contact_radius
        self.particle_self_contact_margin = particle_self_contact_margin
        self.particle_enable_tile_solve = particle_enable_tile_solve
        self.particle_conservative_bound_relaxation = particle_conservative_bound_relaxation
        self.particle_collision_detection_interval = particle_collision_detection_interval
        self.particle_topological_contact_filter_threshold = particle_topological_contact_filter_threshold
        self.particle_rest_shape_contact_exclusion_radius = particle_rest_shape_contact_exclusion_radius
        self._sc_buffers = (int(particle_vertex_contact_buffer_size), int(particle_edge_contact_buffer_size))
        self._iteration = 0
        self._handle = None
        if model.particle_count == 0:
            return
        if particle_enable_self_contact:
            if particle_self_contact_margin < particle_self_contact_radius:
                raise ValueError(
                    "particle_self_contact_margin is smaller than particle_self_contact_radius, this will result in "
                    "missing contacts and cause instability.\nIt is advisable to make particle_self_contact_margin "
                    "1.5-2 times larger than particle_self_contact_radius."
                )

        if len(model.particle_color_groups) == 0:
            raise ValueError(
                "model.particle_color_groups is empty! When using the SolverVBD you must call ModelBuilder.color() "
                "or ModelBuilder.set_coloring() before calling ModelBuilder.finalize()."
            )
        if model.soft_mesh_adjacency is None:
            raise ValueError("model.soft_mesh_adjacency is missing; finalize the model with ModelBuilder.")
        self._lib = _lib.load()
        opts = _lib.VbdSolverOptions()
        opts.iterations = self.iterations
        opts.friction_epsilon = self.friction_epsilon
        opts.lanes_per_vertex = int(lanes_per_vertex)
        opts.block_size = int(block_size)
        opts.contacts_per_vertex = int(contacts_per_vertex)
        opts.use_graph = 1 if use_cuda_graph else 0
        opts.step_kernel = 1 if resident_step else 0
        if particle_enable_self_contact:
            opts.self_contact = 1
            opts.self_contact_radius = float(particle_self_contact_radius)
            opts.self_contact_margin = float(particle_self_contact_margin)
            opts.conservative_bound_relaxation = float(particle_conservative_bound_relaxation)
            opts.vertex_contact_buffer_size = int(particle_vertex_contact_buffer_size)
            opts.edge_contact_buffer_size = int(particle_edge_contact_buffer_size)
            opts.collision_detection_interval = int(particle_collision_detection_interval)
            opts.edge_parallel_epsilon = float(particle_edge_parallel_epsilon)
            opts.topological_filter_threshold = int(particle_topological_contact_filter_threshold)
            opts.rest_exclusion_radius = float(particle_rest_shape_contact_exclusion_radius)
            self._filters = []  # keeps the CSR arrays alive while the library copies them
            for mapping, rows, off_name, list_name in (
                (particle_external_vertex_contact_filtering_map, model.particle_count, "vertex_filter_offsets",
                 "vertex_filter_triangles"),
                (particle_external_edge_contact_filtering_map, model.edge_count, "edge_filter_offsets",
                 "edge_filter_edges"),
            ):
                if not mapping:
                    continue
                lists = [sorted({int(x) for x in mapping.get(r, ())}) for r in range(rows)]
                off = np.zeros(rows + 1, np.int32)
                off[1:] = np.cumsum([len(l) for l in lists])
                flat = np.array([x for l in lists for x in l] or [0], dtype=np.int32)
                self._filters += [off, flat]
                setattr(opts, off_name, off.ctypes.data)
                setattr(opts, list_name, flat.ctypes.data)
        self._opts = opts
        self._warm = None
        self._gate = None
        self._feature_set = "corrections"
        self._staged = False
        self._create()

    def _create(self) -> None:
        dm = self.model.device_model()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.model.device):
            _lib.check(self._lib.vbd_solver_create(dm.handle, ctypes.byref(self._opts), ctypes.byref(h)))
        self._handle = h
        self._dm = dm  # keeps the device model alive as long as the solver

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                self._lib.vbd_solver_destroy(h)
            except Exception:
                pass
            self._handle = None

    # -----------------------------------------------------------------------------------
    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(torch.cuda.current_stream(self.model.device).cuda_stream)

    @staticmethod
    def _check_state(state: State, name: str, V: int, device) -> None:
        for attr in ("particle_q", "particle_qd"):
            t = getattr(state, attr)
            if t is None:
                raise ValueError(f"{name}.{attr} is None")
            if t.dtype != torch.float32 or t.device != device or not t.is_contiguous() or t.numel() != 3 * V:
                raise ValueError(f"{name}.{attr} must be a contiguous float32 [{V},3] tensor on {device}")

    def _contacts(self, contacts: Contacts | None):
        if contacts is None or self.model.shape_count == 0:
            return None
        return ctypes.byref(contacts.c_struct())

    def step(self, state_in: State, state_out: State, control: Control | None, contacts: Contacts | None,
             dt: float) -> None:
        if self.model.particle_count == 0:
            return
        V = self.model.particle_count
        dev = self.model.device
        self._check_state(state_in, "state_in", V, dev)
        self._check_state(state_out, "state_out", V, dev)
        f = state_in.particle_f
        _lib.check(
            self._lib.vbd_step(
                self._handle,
                _lib.ptr(state_in.particle_q),
                _lib.ptr(state_in.particle_qd),
                _lib.ptr(f),
                _lib.ptr(state_out.particle_q),
                _lib.ptr(state_out.particle_qd),
                self._contacts(contacts),
                ctypes.c_float(dt),
                self.iterations,
                self._stream(),
            )
        )

    @staticmethod
    def step_batch(solvers: list["SolverVBD"], states_in: list[State], states_out: list[State],
                   contacts: list[Contacts | None] | None, dt: float) -> None:
        """``step`` of several independent solvers in one library call (``vbd_batch_step``): the
        same results as calling ``solvers[b].step(states_in[b], states_out[b], None, contacts[b],
        dt)`` in order, enqueued on the current stream.  All solvers must live on one device; each
        uses its own ``iterations``."""
        n = len(solvers)
        if not (len(states_in) == len(states_out) == n) or (contacts is not None and len(contacts) != n):
            raise ValueError("step_batch: solvers, states_in, states_out and contacts must have the same length")
        if contacts is None:
            contacts = [None] * n
        # models without particles have nothing to step (as in ``step``)
        keep = [b for b in range(n) if solvers[b].model.particle_count > 0]
        if not keep:
            return
        dev = solvers[keep[0]].model.device
        for b in keep:
            s = solvers[b]
            if s.model.device != dev:
                raise ValueError("step_batch: all solvers must be on one device")
            V = s.model.particle_count
            s._check_state(states_in[b], f"states_in[{b}]", V, dev)
            s._check_state(states_out[b], f"states_out[{b}]", V, dev)

        def addr(t):
            p = _lib.ptr(t)
            return None if p is None else p.value

        m = len(keep)
        arr = ctypes.c_void_p * m
        handles = arr(*[solvers[b]._handle.value for b in keep])
        q_in = arr(*[addr(states_in[b].particle_q) for b in keep])
        qd_in = arr(*[addr(states_in[b].particle_qd) for b in keep])
        f_ext = arr(*[addr(states_in[b].particle_f) for b in keep])
        q_out = arr(*[addr(states_out[b].particle_q) for b in keep])
        qd_out = arr(*[addr(states_out[b].particle_qd) for b in keep])
        cp = ctypes.POINTER(_lib.VbdContacts)
        cptrs = (cp * m)(*[cp(contacts[b].c_struct()) if (contacts[b] is not None and solvers[b].model.shape_count > 0)
                           else cp() for b in keep])
        iters = (ctypes.c_int32 * m)(*[solvers[b].iterations for b in keep])
        s0 = solvers[keep[0]]
        _lib.check(s0._lib.vbd_batch_step(handles, m, q_in, qd_in, f_ext, q_out, qd_out, cptrs, ctypes.c_float(dt),
                                          iters, s0._stream()))

    # ---- staged pieces (parity tests, residual-gated loops) ------------------------------
    def forward(self, state_in: State, contacts: Contacts | None, dt: float) -> None:
        self._iteration = 0
        _lib.check(
            self._lib.vbd_forward(
                self._handle,
                _lib.ptr(state_in.particle_q),
                _lib.ptr(state_in.particle_qd),
                _lib.ptr(state_in.particle_f),
                self._contacts(contacts),
                ctypes.c_float(dt),
                self._stream(),
            )
        )

    def sweep_color(self, color: int, contacts: Contacts | None, dt: float) -> None:
        _lib.check(self._lib.vbd_sweep_color(self._handle, int(color), self._contacts(contacts), ctypes.c_float(dt),
                                             self._stream()))

    def begin_iteration(self) -> None:
        """Start the next iteration of a staged step (self-contact detection when it is scheduled)."""
        _lib.check(self._lib.vbd_begin_iteration(self._handle, self._iteration, self._stream()))
        self._iteration += 1

    def iterate(self, contacts: Contacts | None, dt: float, iterations: int = 1) -> None:
        for _ in range(iterations):
            self.begin_iteration()
            for c in range(len(self.model.particle_color_groups)):
                self.sweep_color(c, contacts, dt)

    def self_contact_detect(self, particle_q: torch.Tensor):
        """Self-contact candidates at ``particle_q``: (vt_counts [V], vt_lists [V, vertex buffer],
        ee_counts [E], ee_lists [E, edge buffer]) as numpy arrays, ids ascending, -1 padded."""
        V, E = self.model.particle_count, self.model.edge_count
        vb, eb = self._sc_buffers
        _lib.check(self._lib.vbd_self_contact_detect(self._handle, _lib.ptr(particle_q), self._stream()))
        vc = np.zeros(V, np.int32)
        vl = np.zeros((V, vb), np.int32)
        ec = np.zeros(max(E, 1), np.int32)
        el = np.zeros((max(E, 1), eb), np.int32)
        _lib.check(self._lib.vbd_self_contact_lists(self._handle, vc.ctypes.data, vl.ctypes.data, ec.ctypes.data,
                                                    el.ctypes.data))
        return vc, vl, ec[:E], el[:E]

    def finalize(self, state_in: State, state_out: State, dt: float) -> None:
        _lib.check(
            self._lib.vbd_finalize(
                self._handle,
                _lib.ptr(state_in.particle_q),
                _lib.ptr(state_out.particle_q),
                _lib.ptr(state_out.particle_qd),
                ctypes.c_float(dt),
                self._stream(),
            )
        )

    def warm_start(self, delta: torch.Tensor) -> None:
        """After ``forward``: start the iterations from inertia target + ``delta`` ([V,3], model order)."""
        if delta.dtype != torch.float32 or not delta.is_contiguous() or delta.numel() != 3 * self.model.particle_count:
            raise ValueError("delta must be a contiguous float32 [V,3] tensor")
        _lib.check(self._lib.vbd_warm_start(self._handle, _lib.ptr(delta), self._stream()))

    def positions(self) -> torch.Tensor:
        out = torch.empty((self.model.particle_count, 3), dtype=torch.float32, device=self.model.device)
        _lib.check(self._lib.vbd_get_positions(self._handle, _lib.ptr(out), self._stream()))
        return out

    def residual(self, contacts: Contacts | None, dt: float, per_vertex: bool = False):
        """Max (and optionally per-vertex) force residual / (m |g|) at the current iterate."""
        mx = torch.zeros(1, dtype=torch.float32, device=self.model.device)
        pv = torch.zeros(self.model.particle_count, dtype=torch.float32, device=self.model.device) if per_vertex else None
        _lib.check(self._lib.vbd_residual(self._handle, self._contacts(contacts), ctypes.c_float(dt), _lib.ptr(pv),
                                          _lib.ptr(mx), self._stream()))
        return (mx, pv) if per_vertex else mx

    def status(self, reset: bool = False) -> dict:
        st = _lib.VbdStatus()
        _lib.check(self._lib.vbd_status(self._handle, ctypes.byref(st), 1 if reset else 0))
        return {
            "steps": st.steps,
            "nonfinite_updates": st.nonfinite_updates,
            "singular_blocks": st.singular_blocks,
            "contact_overflow": st.contact_overflow,
            "timeouts": st.timeouts,
            "self_contact_overflow": st.self_contact_overflow,
        }

    def set_launch(self, lanes_per_vertex: int, block_size: int) -> None:
        _lib.check(self._lib.vbd_set_launch(self._handle, int(lanes_per_vertex), int(block_size)))

    def set_staged_sweep(self, on: bool = True) -> None:
        """Sweeps read the one-ring positions from a per-block shared-memory patch
        (``vbd_set_staged_sweep``); bit-identical results."""
        self._staged = bool(on)
        _lib.check(self._lib.vbd_set_staged_sweep(self._handle, 1 if on else 0))

    def staged_sweep_info(self) -> dict:
        a, mp, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        _lib.check(self._lib.vbd_staged_sweep_info(self._handle, ctypes.byref(a), ctypes.byref(mp), ctypes.byref(n)))
        return {"active": bool(a.value), "max_patch": mp.value, "patch_entries": n.value}

    def launch_info(self) -> dict:
        c, l, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.vbd_solver_info(self._handle, ctypes.byref(c), ctypes.byref(l), ctypes.byref(b)))
        return {"colors": c.value, "lanes_per_vertex": l.value, "block_size": b.value}

    def step_kernel_info(self) -> dict:
        r, p, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self._lib.vbd_solver_step_kernel(self._handle, ctypes.byref(r), ctypes.byref(p), ctypes.byref(b)))
        return {"resident": bool(r.value), "patches": p.value, "smem_bytes": b.value}

    def step_kernel_count(self) -> int:
        """Kernel launches of the most recent ``step`` (kernel nodes of the CUDA graph it replayed;
        -1 when it ran as plain launches)."""
        k = ctypes.c_int32()
        _lib.check(self._lib.vbd_step_kernel_count(self._handle, ctypes.byref(k)))
        return k.value

    def set_warm_start_correction(self, corr: torch.Tensor) -> None:
        """The previous step's correction ``x_solved - y`` ([V,3] model order, device) the warm-start
        step mode feeds to the next step's features (``vbd_set_warm_start_correction``)."""
        corr = corr.contiguous()
        _lib.check(self._lib.vbd_set_warm_start_correction(self._handle, _lib.ptr(corr), self._stream()))

    FEATURE_SETS = {"corrections": 0, "kinematic": 1}

    def set_feature_set(self, name: str) -> None:
        """Input features of the learned warm start (``vbd_set_feature_set``): ``"corrections"``
        (the previous step's solver correction of the vertex and its one-ring, the default) or
        ``"kinematic"`` (previous displacement, velocity and inertia offset only)."""
        if name not in self.FEATURE_SETS:
            raise ValueError(f"feature set must be one of {sorted(self.FEATURE_SETS)}")
        self._feature_set = name
        _lib.check(self._lib.vbd_set_feature_set(self._handle, self.FEATURE_SETS[name]))

    def set_warm_start(self, mlp, iterations: int) -> None:
        """Learned warm start as the step mode: every ``step`` runs forward, the MLP's prediction,
        ``iterations`` colour sweeps and finalize (``mlp=None`` turns it off).  The solver takes
        the network's feature set (``mlp.feature_set``)."""
        self._warm = mlp  # keeps the network's buffers alive while the solver points at them
        self._warm_iterations = int(iterations)
        if mlp is None:
            _lib.check(self._lib.vbd_set_warm_start(self._handle, None, None, None, None, 0))
            return
        self.set_feature_set(getattr(mlp, "feature_set", "corrections"))
        _lib.check(self._lib.vbd_set_warm_start(self._handle, _lib.ptr(mlp.params), _lib.ptr(mlp.w16),
                                                _lib.ptr(mlp.mean), _lib.ptr(mlp.inv_std), int(iterations)))

    def set_residual_gate(self, tolerance: float | None, max_iterations: int = 100, check_every: int = 1,
                          relative: bool = False, norm: str = "max", residual: str = "jacobi",
                          rounds_per_body: int = 0) -> None:
        """Residual-gated steps (no reference counterpart; the reference runs a fixed iteration count,
        ``solver_vbd.py:1817-1819``): each ``step`` iterates until the Jacobi force residual norm --
        ``max_i |f_i| / (m_i |g|)`` (``norm="max"``) or its mean over the solved vertices
        (``norm="mean"``) -- is at most ``tolerance`` (relative to the norm at the inertia target
        when ``relative``), checked every ``check_every`` iterations, at most ``max_iterations``.
        ``residual="jacobi"`` evaluates the residual at the current iterate (one extra sweep-sized
        launch per check); ``residual="sweep"`` uses the Gauss-Seidel residual the sweeps form
        anyway (each vertex's force when its color is solved; no extra launch).  The loop runs on
        the device (a conditional node of the step's CUDA graph); with ``residual="sweep"`` one
        pass of its body runs ``rounds_per_body`` check rounds (0: the library's default, 4), the
        rounds after the decision returning at once.  ``tolerance=None`` turns the gate off."""
        if norm not in ("max", "mean"):
            raise ValueError("norm must be 'max' or 'mean'")
        if residual not in ("jacobi", "sweep"):
            raise ValueError("residual must be 'jacobi' or 'sweep'")
        if not 0 <= int(rounds_per_body) <= 15:
            raise ValueError("rounds_per_body must be in [0, 15]")
        self._gate = None if tolerance is None else (float(tolerance), int(max_iterations), int(check_every),
                                                     bool(relative), norm, residual, int(rounds_per_body))
        tol = 0.0 if tolerance is None else float(tolerance)
        mode = ((1 if relative else 0) | (2 if norm == "mean" else 0) | (4 if residual == "sweep" else 0)
                | (int(rounds_per_body) << 8))
        _lib.check(self._lib.vbd_set_residual_gate(self._handle, ctypes.c_float(tol), int(max_iterations),
                                                   int(check_every), mode))

    def gate_stats(self, reset: bool = False) -> dict:
        """Iterations and residuals of the gated steps since the gate was enabled (or last reset)."""
        g = _lib.VbdGateStats()
        _lib.check(self._lib.vbd_gate_stats(self._handle, ctypes.byref(g), 1 if reset else 0))
        return {
            "steps": g.steps,
            "iterations": g.iterations,
            "mean_iterations": (g.iterations / g.steps) if g.steps else None,
            "capped_steps": g.capped_steps,
            "last_iterations": g.last_iterations,
            "body_kernels": g.body_kernels,
            "last_residual": g.last_residual,
            "last_start_residual": g.last_start_residual,
            "last_reference_residual": g.last_reference_residual,
            "body_programmatic_edges": g.body_programmatic_edges,
            "body_passes": g.body_passes,
        }

    def set_spin_limit(self, spins: int) -> None:
        _lib.check(self._lib.vbd_set_spin_limit(self._handle, int(spins)))

    def reset(self, state: State, world_mask=None, flags=None) -> None:
        warnings.warn(
            "SolverVBD.reset() does not support particle resets; particle solver history is unchanged.", stacklevel=2
        )

    def notify_model_changed(self, flags: int) -> None:
        """``SolverBase.notify_model_changed`` (``solver.py:375``).  The reference's particle path
        reads gravity, shapes and contact materials from the model at every step; here they live
        in the device copy of the model, so MODEL_PROPERTIES or SHAPE_PROPERTIES rebuild that copy
        and the native solver (same options, learned warm start kept).  Other flags concern rigid
        bodies, joints and actuators and change nothing on the particle path."""
        if self._handle is None:
            return
        if not int(flags) & (ModelFlags.MODEL_PROPERTIES | ModelFlags.SHAPE_PROPERTIES):
            return
        old = self._handle
        self.model.notify_model_changed()
        self._create()
        self._lib.vbd_solver_destroy(old)
        if self._feature_set != "corrections":
            self.set_feature_set(self._feature_set)
        if self._staged:
            self.set_staged_sweep(True)
        if self._warm is not None:
            self.set_warm_start(self._warm, self._warm_iterations)
        if getattr(self, "_gate", None) is not None:
            self.set_residual_gate(*self._gate)

    def rebuild_bvh(self, state: State) -> None:
        """``SolverVBD.rebuild_bvh`` (``solver_vbd.py:3239``): the reference rebuilds its self-contact
        BVHs from ``state``.  Self-contact detection here rebuilds its hash grid from the current
        positions at every detection, so there is nothing to rebuild."""
        return None
