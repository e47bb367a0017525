"""Learned warm start for the VBD step.

A per-vertex MLP (64 -> 128 -> 128 -> 3, SiLU, BF16 weights, FP32 accumulation on the tensor
cores) predicts the correction ``x_solved - y`` that the coming step applies to the inertia
target ``y``, in units of the vertex's characteristic element length, from one-ring features
(``vbd_mlp_features``): inertia offset, the previous step's correction of the vertex and of 8
one-ring neighbours, the 8 one-ring edge vectors, log-stiffnesses, mass, contact and pin flags.
The Gauss-Seidel iterations then start from ``y + prediction``; a zero network is plain VBD bit
for bit.  The force residual after the iterations, against plain VBD's on the same state, is
what decides whether the warm start pays (``calibrate_iterations``).

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

    def __init__(self, device, seed: int = 0):
        self.device = torch.device(device)
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
                "inv_std": self.inv_std.cpu().numpy()}

    def load_state_dict(self, d: dict) -> None:
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
                     samples_per_step: int = 1024, seed: int = 0, trajectory_iterations: int | None = None):
    """Features and targets from a VBD trajectory.

    At every step: collide, forward, features (with the previous step's correction), then
    ``target_iterations`` sweeps give the target correction (x - y) / L.  The trajectory advances
    with ``trajectory_iterations`` plain sweeps from y (default: the target solve itself).
    Returns raw (unstandardised) features [N,64] and targets [N,3]."""
    dev = model.device
    L = torch.from_numpy(characteristic_length(model)).to(dev)
    solvable = torch.from_numpy(((model.particle_flags & 1) != 0) & (model.particle_inv_mass != 0)).to(dev)
    cand = torch.nonzero(solvable).reshape(-1)
    gen = torch.Generator(device=dev).manual_seed(seed)
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.as_tensor(q0, device=dev))
    c = pipe.contacts() if pipe is not None else None
    corr = torch.zeros_like(s0.particle_q)
    feats = torch.empty((model.particle_count, IN), dtype=torch.float32, device=dev)
    lib = _lib.load()
    Xs, Ts = [], []
    it_traj = target_iterations if trajectory_iterations is None else trajectory_iterations
    for _ in range(steps):
        if pipe is not None:
            pipe.collide(s0, c)
        y = inertia_target(model, s0, dt)
        solver.forward(s0, c, dt)
        _lib.check(lib.vbd_mlp_features(solver._handle, _lib.ptr(corr), None, None, _lib.ptr(feats), solver._stream()))
        solver.iterate(c, dt, target_iterations)
        x = solver.positions()
        T = (x - y) / L[:, None]
        idx = cand[torch.randint(0, cand.numel(), (min(samples_per_step, cand.numel()),), generator=gen, device=dev)]
        Xs.append(feats[idx].clone())
        Ts.append(T[idx].clone())
        if it_traj != target_iterations:  # advance with the trajectory's own iteration count
            solver.forward(s0, c, dt)
            solver.iterate(c, dt, it_traj)
        solver.finalize(s0, s1, dt)
        corr = s1.particle_q - y
        s0, s1 = s1, s0
    return torch.cat(Xs), torch.cat(Ts)


def mean_residual(solver, contacts, dt: float) -> float:
    """Mean over solved vertices of |f_i| / (m_i |g|) at the current iterate."""
    _, pv = solver.residual(contacts, dt, per_vertex=True)
    m = solver.model
    solvable = torch.from_numpy(((m.particle_flags & 1) != 0) & (m.particle_inv_mass != 0)).to(pv.device)
    return float(pv[solvable].mean().item())


def calibrate_iterations(model, q0, solver, pipe, mlp: WarmStartMLP, steps: int, dt: float,
                         plain_iterations: int = 10, max_iterations: int = 10, check_every: int = 10,
                         advance: str = "learned"):
    """At every ``check_every``-th step, find the fewest warm-started iterations whose mean
    residual matches plain VBD's after ``plain_iterations`` on the same step (same state).  The
    trajectory advances with the learned solver (``advance="learned"``) or with plain VBD
    (``advance="plain"``: teacher forcing, which isolates the per-step effect of the start from
    the stability of a trajectory driven by it).  Returns (iterations, per-check records)."""
    dev = model.device
    lib = _lib.load()
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.as_tensor(q0, device=dev))
    c = pipe.contacts() if pipe is not None else None
    corr = torch.zeros_like(s0.particle_q)
    work = torch.empty(model.particle_count * 70, dtype=torch.float32, device=dev)
    need = []
    records = []
    for step in range(steps):
        if pipe is not None:
            pipe.collide(s0, c)
        y = inertia_target(model, s0, dt)
        if step % check_every == 0:
            solver.forward(s0, c, dt)
            r_plain_k = []
            for k in range(1, plain_iterations + 1):
                solver.iterate(c, dt, 1)
                r_plain_k.append(mean_residual(solver, c, dt))
            r_plain = r_plain_k[-1]
            solver.forward(s0, c, dt)
            _lib.check(lib.vbd_mlp_warm_start(solver._handle, _lib.ptr(mlp.params), _lib.ptr(mlp.w16), _lib.ptr(corr),
                                              _lib.ptr(mlp.mean), _lib.ptr(mlp.inv_std), _lib.ptr(work), work.numel(),
                                              solver._stream()))
            r_k = []
            k_hit = max_iterations + 1
            for k in range(1, max_iterations + 1):
                solver.iterate(c, dt, 1)
                r = mean_residual(solver, c, dt)
                r_k.append(r)
                if r <= r_plain and k_hit > max_iterations:
                    k_hit = k
            # the same start without the network: previous correction only
            solver.forward(s0, c, dt)
            solver.warm_start(corr.contiguous())
            k_prev = max_iterations + 1
            for k in range(1, max_iterations + 1):
                solver.iterate(c, dt, 1)
                if mean_residual(solver, c, dt) <= r_plain:
                    k_prev = k
                    break
            need.append(k_hit)
            records.append({"step": step, "plain": r_plain, "plain_curve": r_plain_k, "warm": r_k, "k": k_hit,
                            "k_previous_correction": k_prev})
        solver.forward(s0, c, dt)
        if advance == "plain":
            solver.iterate(c, dt, plain_iterations)
        else:  # the learned solver at the current working point
            _lib.check(lib.vbd_mlp_warm_start(solver._handle, _lib.ptr(mlp.params), _lib.ptr(mlp.w16), _lib.ptr(corr),
                                              _lib.ptr(mlp.mean), _lib.ptr(mlp.inv_std), _lib.ptr(work), work.numel(),
                                              solver._stream()))
            solver.iterate(c, dt, max(1, int(np.percentile(need, 90))) if need else plain_iterations)
        solver.finalize(s0, s1, dt)
        corr = s1.particle_q - y
        s0, s1 = s1, s0
    return int(np.ceil(np.percentile(need, 90))), records
