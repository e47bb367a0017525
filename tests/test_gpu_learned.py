"""GPU tests of the learned warm start: the tensor-core MLP kernels against an FP64 CPU
restatement (forward, gradients), training, the zero-network identity with plain VBD, and the
A/B measurement against plain VBD at equal residual."""

import numpy as np
import pytest
import torch

from newton_b200 import CollisionPipeline, scenes
from newton_b200 import learned as L
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu


def _np_params(mlp):
    p = mlp.params.cpu().double().numpy()
    bf = lambda a: torch.tensor(a, dtype=torch.float32).bfloat16().double().numpy()  # noqa: E731
    W1 = bf(p[L.OFF_W1:L.OFF_B1].reshape(L.IN, L.HID))
    W2 = bf(p[L.OFF_W2:L.OFF_B2].reshape(L.HID, L.HID))
    W3 = bf(p[L.OFF_W3:L.OFF_B3].reshape(L.HID, L.OUTP))[:, :L.OUT]
    return W1, p[L.OFF_B1:L.OFF_W2], W2, p[L.OFF_B2:L.OFF_W3], W3, p[L.OFF_B3:L.OFF_B3 + L.OUT]


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _reference(mlp, X, T):
    """FP64 forward / backward of mean |y - t|^2 with BF16-rounded weights and inputs."""
    W1, b1, W2, b2, W3, b3 = _np_params(mlp)
    bf = lambda a: torch.tensor(a, dtype=torch.float32).bfloat16().double().numpy()  # noqa: E731
    x = bf(X)
    z1 = x @ W1 + b1
    h1 = _silu(z1)
    z2 = h1 @ W2 + b2
    h2 = _silu(z2)
    y = h2 @ W3 + b3
    n = X.shape[0]
    dy = 2.0 * (y - T) / n
    s2 = 1 / (1 + np.exp(-z2))
    dz2 = (dy @ W3.T) * s2 * (1 + z2 * (1 - s2))
    s1 = 1 / (1 + np.exp(-z1))
    dz1 = (dz2 @ W2.T) * s1 * (1 + z1 * (1 - s1))
    g = {"W1": x.T @ dz1, "b1": dz1.sum(0), "W2": h1.T @ dz2, "b2": dz2.sum(0), "W3": h2.T @ dy, "b3": dy.sum(0)}
    return y, g


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-12))


def test_mlp_forward_matches_fp64_reference():
    mlp = L.WarmStartMLP("cuda:0", seed=1)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(1000, L.IN)).astype(np.float32)
    y = mlp.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    y_ref, _ = _reference(mlp, X, np.zeros((1000, 3)))
    assert _rel(y, y_ref) < 2e-2


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 4097, 300000])
def test_tcgen05_inference_matches_the_mma_sync_path_and_fp64(n):
    """The tcgen05 inference kernel (TMEM accumulators) against the mma.sync one and the FP64
    restatement: partial tiles, one tile, many tiles per CTA; no wait gave up."""
    import ctypes

    from newton_b200 import _lib

    lib = _lib.load()
    cnt = ctypes.c_uint32()
    _lib.check(lib.vbd_mlp_timeouts(ctypes.byref(cnt), 1))
    mlp = L.WarmStartMLP("cuda:0", seed=7)
    rng = np.random.default_rng(n)
    X = torch.from_numpy(rng.normal(size=(n, L.IN)).astype(np.float32)).cuda()
    y_tc = mlp.forward(X)
    y_ms = torch.empty_like(y_tc)
    _lib.check(lib.vbd_mlp_forward_mma_sync(_lib.ptr(mlp.params), _lib.ptr(mlp.w16), _lib.ptr(X), n, _lib.ptr(y_ms),
                                            mlp._stream()))
    torch.cuda.synchronize()
    a, b = y_tc.cpu().numpy(), y_ms.cpu().numpy()
    assert np.isfinite(a).all()
    # both round the activations to BF16; SiLU differs (hardware tanh vs exact), ~1e-3 relative
    assert _rel(a, b) < 2e-2, _rel(a, b)
    if n <= 4097:
        y_ref, _ = _reference(mlp, X.cpu().numpy(), np.zeros((n, 3)))
        assert _rel(a, y_ref) < 2e-2
    _lib.check(lib.vbd_mlp_timeouts(ctypes.byref(cnt), 0))
    assert cnt.value == 0


def test_mlp_gradients_match_fp64_reference():
    mlp = L.WarmStartMLP("cuda:0", seed=2)
    rng = np.random.default_rng(1)
    n = 3000  # not a multiple of the tile sizes
    X = rng.normal(size=(n, L.IN)).astype(np.float32)
    T = rng.normal(size=(n, 3)).astype(np.float32)
    loss = mlp.gradients(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    torch.cuda.synchronize()
    y_ref, g = _reference(mlp, X, T)
    assert abs(float(loss.item()) / n - float(((y_ref - T) ** 2).sum(1).mean())) < 2e-2 * float(((y_ref - T) ** 2).sum(1).mean())
    gr = mlp.grads.cpu().double().numpy()
    assert _rel(gr[L.OFF_W1:L.OFF_B1].reshape(L.IN, L.HID), g["W1"]) < 5e-2
    assert _rel(gr[L.OFF_B1:L.OFF_W2], g["b1"]) < 5e-2
    assert _rel(gr[L.OFF_W2:L.OFF_B2].reshape(L.HID, L.HID), g["W2"]) < 5e-2
    assert _rel(gr[L.OFF_B2:L.OFF_W3], g["b2"]) < 5e-2
    assert _rel(gr[L.OFF_W3:L.OFF_B3].reshape(L.HID, L.OUTP)[:, :3], g["W3"]) < 5e-2
    assert _rel(gr[L.OFF_B3:L.OFF_B3 + 3], g["b3"]) < 5e-2
    assert np.all(gr[L.OFF_W3:L.OFF_B3].reshape(L.HID, L.OUTP)[:, 3:] == 0)


def test_training_fits_a_smooth_function():
    mlp = L.WarmStartMLP("cuda:0", seed=3)
    rng = np.random.default_rng(2)
    X = torch.from_numpy(rng.normal(size=(65536, L.IN)).astype(np.float32)).cuda()
    T = torch.stack([torch.sin(X[:, 0]), X[:, 1] * X[:, 2] * 0.5, torch.tanh(X[:, 3] + X[:, 4])], 1)
    hist = mlp.train(X, T, epochs=30, batch=8192, lr=3e-3)
    assert hist[-1] < 0.1 * hist[0]


def test_zero_network_warm_start_is_plain_vbd():
    """The learned step mode with a network whose output is zero reproduces plain VBD bit for bit
    (same start y, same sweeps), contacts included."""
    dt = 1.0 / 600.0
    out = []
    for learned in (False, True):
        model, q0 = scenes.single_cloth(n=24, side=1.0, seed=5, pin_top_corners=False, ground=0.0,
                                        sphere=((0.0, 0.0, 0.5), 0.4), height=0.95)
        solver = SolverVBD(model, iterations=6)
        if learned:
            mlp = L.WarmStartMLP("cuda:0", seed=6)
            mlp.params.zero_()
            mlp.pack()
            solver.set_warm_start(mlp, 6)
        pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
        c = pipe.contacts()
        a, b = model.state(), model.state()
        a.particle_q.copy_(torch.from_numpy(q0).cuda())
        for _ in range(40):
            pipe.collide(a, c)
            solver.step(a, b, None, c, dt)
            a, b = b, a
        torch.cuda.synchronize()
        out.append((a.particle_q.clone(), a.particle_qd.clone()))
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])


def test_learned_warm_start_ab_measurement():
    """A/B of the learned start against plain VBD on a held-out drape: the network trains, and the
    calibration reports, per checked step, plain VBD's 10-iteration mean residual and the fewest
    warm-started iterations that match it (11 = not reached within 10)."""
    dt = 1.0 / 600.0
    model, q0 = scenes.single_cloth(n=48, side=1.0, seed=30, pin_top_corners=False, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.95, z_noise=0.0)
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    X, T = L.generate_dataset(model, q0, solver, pipe, steps=300, dt=dt, target_iterations=20, samples_per_step=1024,
                              trajectory_iterations=10)
    mlp = L.WarmStartMLP("cuda:0", seed=4)
    mlp.set_standardization(X)
    hist = mlp.train(mlp.standardize(X), T, epochs=40, batch=8192, lr=2e-3)
    assert hist[-1] < hist[0]
    model, q_test = scenes.single_cloth(n=48, side=1.0, seed=31, pin_top_corners=False, ground=0.0,
                                        sphere=((0.1, 0.05, 0.5), 0.4), height=0.95, z_noise=0.0)
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    k, records = L.calibrate_iterations(model, q_test, solver, pipe, mlp, steps=100, dt=dt, check_every=20)
    print("iterations to reach plain-10 residual (learned):", [r["k"] for r in records])
    print("iterations to reach plain-10 residual (previous correction only):", [r["k_previous_correction"] for r in records])
    assert len(records) == 5
    for r in records:
        assert np.isfinite(r["plain"]) and len(r["plain_curve"]) == 10
        assert 1 <= r["k"] <= 11 and 1 <= r["k_previous_correction"] <= 11
    assert 1 <= k <= 11
