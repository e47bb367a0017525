"""Learned warm start for the VBD step.

A per-vertex MLP (64 -> 128 -> 128 -> 3, SiLU; trained with FP32 master weights on BF16 mma.sync
tiles with FP32 accumulation, run for inference on tcgen05 with FP16 operands and FP32
accumulation) predicts the correction ``x_solved - y`` that the coming step applies to the inertia
target ``y``, in units of the vertex's characteristic element length, from one-ring features
(``vbd_mlp_features``).  Two feature sets: ``"corrections"`` (default) -- the inertia offset, the
previous step's correction of the vertex and of 8 one-ring neighbours, the 8 one-ring edge
vectors, log-stiffnesses, mass, contact and pin flags; ``"kinematic"`` -- previous step's
displacement, velocity and inertia offset with the same geometry, material and flags, no solver
history.  The Gauss-Seidel iterations then start from ``y + prediction``; a zero network is
plain VBD bit for bit.  What decides whether the warm start pays is the residual-gated step
(``SolverVBD.set_residual_gate``): from the same state, the learned and the plain solver iterate
until the same force residual, and the iterations they need are compared (``gated_steps``).

The previous correction is a feature and never the start itself: starting from
``y + (x_prev_solved - y_prev)`` counts the previous step's acceleration twice (it is already in
the velocity that ``y`` extrapolates), and a trajectory advanced that way gains energy and
diverges within a few hundred steps on the draped cloth even at 10 iterations.

Everything numeric runs in ``libvbd_b200.so``: features, inference, the backward pass, the
weight-gradient GEMMs and Adam (``vbd_mlp_*``).  Torch tensors are only the buffers.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib

IN, HID, OUT, OUTP = 64, 128, 3, 8
OFF_W1, OFF_B1 = 0, IN * HID
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + HID * OUTP
N_PARAMS = OFF_B3 + OUTP
N_W16 = IN * HID + HID * HID + HID * OUTP


def characteristic_length(model) -> np.ndarray:
    """Per-vertex mean of sqrt(2 * area) over incident triangles (the library's feature scale)."""
    V = model.particle_count
    tris = model.tri_indices.reshape(-1, 3)
    s = np.sqrt(2.0 * np.maximum(model.tri_areas.astype(np.float64), 0.0))
    acc = np.zeros(V)
    cnt = np.zeros(V)
    for k in range(3):
        np.add.at(acc, tris[:, k], s)
        np.add.at(cnt, tris[:, k], 1.0)
    return np.where(cnt > 0, acc / np.maximum(cnt, 1), 1.0).astype(np.float32)


class WarmStartMLP:
    """Parameters, optimiser state and feature standardisation of the warm-start network."""

    def __init__(self, device, seed: int = 0, feature_set: str = "corrections"):
        self.device = torch.device(device)
        self.feature_set = feature_set  # the solver's feature set this network reads
        self.lib = _lib.load()
        sizes = [ctypes.c_int32() for _ in range(5)]
        _lib.check(self.lib.vbd_mlp_sizes(*[ctypes.byref(v) for v in sizes]))
        assert sizes[0].value == N_PARAMS and sizes[1].value == N_W16
        g = torch.Generator(device="cpu").manual_seed(seed)
        p = torch.zeros(N_PARAMS, dtype=torch.float32)
        p[OFF_W1:OFF_B1] = torch.randn(IN * HID, generator=g) * math.sqrt(2.0 / IN)
        p[OFF_W2:OFF_B2] = torch.randn(HID * HID, generator=g) * math.sqrt(2.0 / HID)
        w3 = torch.zeros(HID, OUTP)
        w3[:, :OUT] = torch.randn(HID, OUT, generator=g) * math.sqrt(1.0 / HID) * 0.1
        p[OFF_W3:OFF_B3] = w3.reshape(-1)
        self.params = p.to(self.device)
        self.w16 = torch.zeros(N_W16, dtype=torch.int16, device=self.device)
        self.m1 = torch.zeros_like(self.params)
        self.m2 = torch.zeros_like(self.params)
        self.grads = torch.zeros_like(self.params)
        self.mean = torch.zeros(IN, dtype=torch.float32, device=self.device)
        self.inv_std = torch.ones(IN, dtype=torch.float32, device=self.device)
        self.step_count = 0
        self._ws = None
        self.pack()

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def pack(self) -> None:
        _lib.check(self.lib.vbd_mlp_pack_weights(_lib.ptr(self.params), _lib.ptr(self.w16), self._stream()))

    def set_standardization(self, X: torch.Tensor) -> None:
        """Feature mean / inverse std from raw features (constant features keep std 1)."""
        m = X.double().mean(0)
        sd = X.double().std(0)
        sd = torch.where(sd > 1e-6, sd, torch.ones_like(sd))
        self.mean.copy_(m.float())
        self.inv_std.copy_((1.0 / sd).float())

    def standardize(self, X: torch.Tensor) -> torch.Tensor:
        return (X - self.mean) * self.inv_std

    def forward(self, X: torch.Tensor) -> torch.Tensor:
        X = X.contiguous()
        Y = torch.empty((X.shape[0], OUT), dtype=torch.float32, device=self.device)
        _lib.check(self.lib.vbd_mlp_forward(_lib.ptr(self.params), _lib.ptr(self.w16), _lib.ptr(X), X.shape[0],
                                            _lib.ptr(Y), self._stream()))
        return Y

    def _workspace(self, n: int) -> torch.Tensor:
        b = ctypes.c_int64()
        _lib.check(self.lib.vbd_mlp_workspace_bytes(n, ctypes.byref(b)))
        if self._ws is None or self._ws.numel() < b.value:
            self._ws = torch.empty(b.value, dtype=torch.uint8, device=self.device)
        return self._ws

    def gradients(self, X: torch.Tensor, T: torch.Tensor) -> float:
        """Fills self.grads with d/dparams of mean |MLP(X) - T|^2; returns that loss."""
        X, T = X.contiguous(), T.contiguous()
        n = X.shape[0]
        ws = self._workspace(n)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        _lib.check(self.lib.vbd_mlp_backward(_lib.ptr(self.params), _lib.ptr(self.w16), _lib.ptr(X), _lib.ptr(T), n,
                                             ctypes.c_float(1.0 / n), _lib.ptr(self.grads), _lib.ptr(loss), _lib.ptr(ws),
                                             ws.numel(), self._stream()))
        return loss

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step_count += 1
        _lib.check(self.lib.vbd_mlp_adam(_lib.ptr(self.params), _lib.ptr(self.grads), _lib.ptr(self.m1),
                                         _lib.ptr(self.m2), _lib.ptr(self.w16), self.step_count, ctypes.c_float(lr),
                                         ctypes.c_float(beta1), ctypes.c_float(beta2), ctypes.c_float(eps),
                                         self._stream()))

    def train(self, X: torch.Tensor, T: torch.Tensor, epochs: int = 20, batch: int = 32768, lr: float = 2e-3,
              seed: int = 0, log=None) -> list[float]:
        """Mini-batch Adam over (standardised X, T); cosine learning-rate decay."""
        n = X.shape[0]
        gen = torch.Generator(device=self.device).manual_seed(seed)
        steps = epochs * max(1, n // batch)
        k = 0
        history = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen, device=self.device)
            tot = torch.zeros((), device=self.device)
            for b0 in range(0, n - batch + 1 if n >= batch else 1, batch):
                idx = perm[b0:b0 + batch]
                tot += self.gradients(X[idx], T[idx])[0]
                self.adam(lr * 0.5 * (1.0 + math.cos(math.pi * k / max(steps, 1))))
                k += 1
            history.append(float(tot.item()) / n)
            if log:
                log(f"epoch {ep}: mse {history[-1]:.4g}")
        return history

    def state_dict(self) -> dict:
        return {"params": self.params.cpu().numpy(), "mean": self.mean.cpu().numpy(),
                "inv_std": self.inv_std.cpu().numpy(), "feature_set": self.feature_set}

    def load_state_dict(self, d: dict) -> None:
        self.feature_set = str(d.get("feature_set", "corrections"))
        self.params.copy_(torch.as_tensor(np.asarray(d["params"]), device=self.device))
        self.mean.copy_(torch.as_tensor(np.asarray(d["mean"]), device=self.device))
        self.inv_std.copy_(torch.as_tensor(np.asarray(d["inv_std"]), device=self.device))
        self.pack()


def inertia_target(model, state, dt: float) -> torch.Tensor:
    """y = x + (v + g dt) dt for active massive particles, x otherwise (forward_step)."""
    g = torch.tensor(np.asarray(model.gravity, dtype=np.float32).reshape(-1, 3)[0], device=state.particle_q.device)
    solvable = torch.from_numpy(((model.particle_flags & 1) != 0) & (model.particle_inv_mass != 0)).to(g.device)
    y = state.particle_q + (state.particle_qd + g * dt) * dt
    return torch.where(solvable[:, None], y, state.particle_q)


def generate_dataset(model, q0, solver, pipe, steps: int, dt: float, target_iterations: int = 20,
                     samples_per_step: int = 1024, seed: int = 0, trajectory_iterations: int | None = None,
                     feature_set: str | tuple = "corrections", record_every: int = 1):
    """Features and targets from a VBD trajectory.

    At every ``record_every``-th step: collide, forward, features of ``feature_set`` (with the
    previous step's correction), then ``target_iterations`` sweeps give the target correction
    (x - y) / L.  The trajectory advances every step with ``trajectory_iterations`` plain sweeps
    from y (default: the target solve itself).  Returns raw (unstandardised) features [N,64] and
    targets [N,3]; with a tuple of feature sets, the features are a dict {set: [N,64]} of the
    same samples."""
    sets = (feature_set,) if isinstance(feature_set, str) else tuple(feature_set)
    dev = model.device
    L = torch.from_numpy(characteristic_length(model)).to(dev)
    solvable = torch.from_numpy(((model.particle_flags & 1) != 0) & (model.particle_inv_mass != 0)).to(dev)
    cand = torch.nonzero(solvable).reshape(-1)
    gen = torch.Generator(device=dev).manual_seed(seed)
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.as_tensor(q0, device=dev))
    c = pipe.contacts() if pipe is not None else None
    corr = torch.zeros_like(s0.particle_q)
    feats = {fs: torch.empty((model.particle_count, IN), dtype=torch.float32, device=dev) for fs in sets}
    lib = _lib.load()
    Xs, Ts = {fs: [] for fs in sets}, []
    it_traj = target_iterations if trajectory_iterations is None else trajectory_iterations
    for step in range(steps):
        if pipe is not None:
            pipe.collide(s0, c)
        y = inertia_target(model, s0, dt)
        solver.forward(s0, c, dt)
        record = step % max(1, record_every) == 0
        if record:
            for fs in sets:
                solver.set_feature_set(fs)
                _lib.check(lib.vbd_mlp_features(solver._handle, _lib.ptr(corr), None, None, _lib.ptr(feats[fs]),
                                                solver._stream()))
            solver.iterate(c, dt, target_iterations)
            x = solver.positions()
            T = (x - y) / L[:, None]
            idx = cand[torch.randint(0, cand.numel(), (min(samples_per_step, cand.numel()),), generator=gen,
                                     device=dev)]
            for fs in sets:
                Xs[fs].append(feats[fs][idx].clone())
            Ts.append(T[idx].clone())
        if not record or it_traj != target_iterations:  # advance with the trajectory's own count
            if record:
                solver.forward(s0, c, dt)
            solver.iterate(c, dt, it_traj)
        solver.finalize(s0, s1, dt)
        corr = s1.particle_q - y
        s0, s1 = s1, s0
    X = {fs: torch.cat(Xs[fs]) for fs in sets}
    return (X[sets[0]] if isinstance(feature_set, str) else X), torch.cat(Ts)


def record_plain_states(model, q_start, qd_start, pipe, gate: dict, steps: int, dt: float,
                        launch: dict | None = None) -> list:
    """The state before each of ``steps`` residual-gated plain-VBD steps from (q_start, qd_start):
    [(particle_q, particle_qd)] as device tensors."""
    from .solvers import SolverVBD

    dev = model.device
    solver = SolverVBD(model, iterations=10)
    if launch is not None:
        solver.set_launch(launch["lanes_per_vertex"], launch["block_size"])
    solver.set_residual_gate(**gate)
    c = pipe.contacts() if pipe is not None else None
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.as_tensor(q_start, device=dev))
    s0.particle_qd.copy_(torch.as_tensor(qd_start, device=dev))
    states = []
    for _ in range(steps):
        states.append((s0.particle_q.clone(), s0.particle_qd.clone()))
        if pipe is not None:
            pipe.collide(s0, c)
        solver.step(s0, s1, None, c, dt)
        s0, s1 = s1, s0
    torch.cuda.synchronize(dev)
    return states


def teacher_forced_steps(model, states: list, pipe, gate: dict, dt: float, mlp: WarmStartMLP | None = None,
                         launch: dict | None = None, warm: int = 0, timer=None, history: bool = True) -> dict:
    """One residual-gated step from every recorded state of a plain trajectory, by plain VBD
    (``mlp=None``) or by the learned step mode.  Both arms start each step from the same state,
    hence the same inertia target y and -- the gate being relative to the residual at y -- the same
    absolute tolerance: the iterations they need are counted to the same force residual.  With
    ``history`` the learned solver's previous-correction feature is the recorded trajectory's own
    (x_k - y_(k-1), set before each step), as it is for a solver on its own trajectory; otherwise it
    carries over from the learned solver's previous step from the previous recorded state.  The
    first ``warm`` states are stepped but not counted.  ``timer`` (optional) has ``before()`` /
    ``after()``, called around each counted collide + step.  Returns the gate statistics of the
    counted steps and the solver status."""
    from .solvers import SolverVBD

    solver = SolverVBD(model, iterations=10)
    if launch is not None:
        solver.set_launch(launch["lanes_per_vertex"], launch["block_size"])
    if mlp is not None:
        solver.set_warm_start(mlp, 10)
    solver.set_residual_gate(**gate)
    c = pipe.contacts() if pipe is not None else None
    s0, s1 = model.state(), model.state()
    for k, (q, qd) in enumerate(states):
        if k == warm:
            solver.gate_stats(reset=True)
            solver.status(reset=True)
        if mlp is not None and history and k > 0:
            # the recorded trajectory's correction of step k-1: its solved positions (state k)
            # minus the inertia target of state k-1
            s0.particle_q.copy_(states[k - 1][0])
            s0.particle_qd.copy_(states[k - 1][1])
            solver.set_warm_start_correction(q - inertia_target(model, s0, dt))
        s0.particle_q.copy_(q)
        s0.particle_qd.copy_(qd)
        counted = k >= warm and timer is not None
        if counted:
            timer.before()
        if pipe is not None:
            pipe.collide(s0, c)
        solver.step(s0, s1, None, c, dt)
        if counted:
            timer.after()
    torch.cuda.synchronize(model.device)
    out = solver.gate_stats()
    out["status"] = solver.status()
    return out


def gated_steps(model, q_start, qd_start, pipe, gate: dict, steps: int, dt: float, mlp: WarmStartMLP | None = None,
                launch: dict | None = None) -> dict:
    """``steps`` residual-gated steps (``SolverVBD.set_residual_gate(**gate)``) from the state
    (q_start, qd_start): plain VBD (``mlp=None``) or the learned step mode.  Returns the gate
    statistics (mean iterations, capped steps, residuals), the solver status and the end state."""
    from .solvers import SolverVBD

    dev = model.device
    solver = SolverVBD(model, iterations=10)
    if launch is not None:
        solver.set_launch(launch["lanes_per_vertex"], launch["block_size"])
    if mlp is not None:
        solver.set_warm_start(mlp, 10)
    solver.set_residual_gate(**gate)
    c = pipe.contacts() if pipe is not None else None
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.as_tensor(q_start, device=dev))
    s0.particle_qd.copy_(torch.as_tensor(qd_start, device=dev))
    for _ in range(steps):
        if pipe is not None:
            pipe.collide(s0, c)
        solver.step(s0, s1, None, c, dt)
        s0, s1 = s1, s0
    torch.cuda.synchronize(dev)
    out = solver.gate_stats()
    out["status"] = solver.status()
    out["q"] = s0.particle_q.clone()
    return out
