"""Known-answer tests that pin the CPU oracle.

The reference cannot run here (its kernels need Warp), so the oracle is pinned against the
known answers of the reference's own VBD tests (``newton/tests/test_solver_vbd.py``), restated
on the same inputs, plus mathematical identities every correct implementation satisfies
(rest state is force-free, forces are minus the energy gradient, Hessians are symmetric).
"""

import math

import numpy as np
import pytest

import oracle

PRECISIONS = ["f32", "f64"]


# ---- inputs of the reference tests -------------------------------------------------------
def _rotations_from_quaternions(quat):
    x, y, z, w = quat[:, 0], quat[:, 1], quat[:, 2], quat[:, 3]
    r = np.empty((quat.shape[0], 3, 3), dtype=np.float32)
    r[:, 0, 0] = 1.0 - 2.0 * (y * y + z * z)
    r[:, 0, 1] = 2.0 * (x * y - z * w)
    r[:, 0, 2] = 2.0 * (x * z + y * w)
    r[:, 1, 0] = 2.0 * (x * y + z * w)
    r[:, 1, 1] = 1.0 - 2.0 * (x * x + z * z)
    r[:, 1, 2] = 2.0 * (y * z - x * w)
    r[:, 2, 0] = 2.0 * (x * z - y * w)
    r[:, 2, 1] = 2.0 * (y * z + x * w)
    r[:, 2, 2] = 1.0 - 2.0 * (x * x + y * y)
    return r


def _seeded_rigid_motions(count, seed):
    """Rotations and translations drawn as in test_solver_vbd.py:62-66, :172-196 (seed 17)."""
    rng = np.random.default_rng(seed)
    quat = rng.normal(size=(count, 4))
    quat /= np.linalg.norm(quat, axis=1, keepdims=True)
    rot = _rotations_from_quaternions(quat)
    trans = np.random.default_rng(seed + 1).uniform(-1.0, 1.0, size=(count, 3)).astype(np.float32)
    return rot, trans


# rest points of test_solver_vbd.py:173-181
REST = np.array([[0.0, 0.0, 0.0], [1.2, 0.1, 0.0], [0.2, 1.1, 0.1], [0.1, 0.2, 1.3]], dtype=np.float32)


def _tri_rest_pose(rest):
    qp, rp = rest[1] - rest[0], rest[2] - rest[0]
    n = np.cross(qp, rp)
    n /= np.linalg.norm(n)
    e1 = qp / np.linalg.norm(qp)
    e2 = np.cross(n, e1)
    e2 /= np.linalg.norm(e2)
    D = np.array((e1, e2), dtype=np.float32) @ np.array((qp, rp), dtype=np.float32).T
    return np.linalg.inv(D).astype(np.float32), np.float32(np.linalg.det(D) * 0.5)


def _hinge_rest(rest):
    x1, x2, x3, x4 = rest
    n1 = np.cross(x3 - x1, x4 - x1)
    n1 /= np.linalg.norm(n1)
    n2 = np.cross(x4 - x2, x3 - x2)
    n2 /= np.linalg.norm(n2)
    e = (x4 - x3) / np.linalg.norm(x4 - x3)
    return np.float32(math.atan2(np.dot(np.cross(n1, n2), e), np.dot(n1, n2))), np.float32(np.linalg.norm(x4 - x3))


@pytest.mark.parametrize("precision", PRECISIONS)
def test_elastic_damping_ignores_rigid_motion(precision):
    """test_solver_vbd.py:1593-1646: membrane and bending damping vanish under rigid motion (atol 1e-4)."""
    rot, trans = _seeded_rigid_motions(100, 17)
    pose, area = _tri_rest_pose(REST)
    rest_angle, rest_len = _hinge_rest(REST)
    dt, damping = 0.1, 20.0
    tri_max, bend_max = 0.0, 0.0
    for s in range(100):
        pos = (REST @ rot[s].T + trans[s]).astype(np.float32)
        for v in range(3):
            f, _ = oracle.membrane(0, v, pos, REST, [[0, 1, 2]], pose.reshape(4), area, 0.0, 1.0, damping, dt, precision)
            tri_max = max(tri_max, float(np.linalg.norm(f)))
        for v in range(4):
            f, _ = oracle.bending(0, v, pos, REST, [[0, 1, 2, 3]], rest_angle, rest_len, 0.0, damping, dt, precision)
            bend_max = max(bend_max, float(np.linalg.norm(f)))
    assert tri_max <= 1e-4
    assert bend_max <= 1e-4


@pytest.mark.parametrize("precision", PRECISIONS)
def test_bending_damping_handles_degenerate_anchor(precision):
    """test_solver_vbd.py:1560-1590: collapsed previous-step geometry gives exactly zero."""
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [1.0, 1.0, 0.1]])
    anchor = np.zeros((4, 3))
    for v in range(4):
        f, h = oracle.bending(0, v, pos, anchor, [[0, 1, 2, 3]], 0.0, 1.0, 0.0, 20.0, 0.1, precision)
        norm = np.linalg.norm(f) + sum(np.linalg.norm(h[r]) for r in range(3))
        assert np.isfinite(norm)
        assert norm <= 1e-6


@pytest.mark.parametrize("precision", PRECISIONS)
def test_body_particle_contact_damping_is_absolute(precision):
    """test_solver_vbd.py:1333-1374: damping contribution is (0, 0, 2) whatever the stiffness."""
    forces = []
    for i in range(4):
        ke = 400.0 if i < 2 else 100.0
        kd = 20.0 if (i & 1) == 0 else 0.0
        f, _ = oracle.contact([0.0, 0.0, 0.04], [0.0, 0.0, 0.05], [0, 0, 0], [0, 0, 0], [0.0, 0.0, 1.0], 0.1, 0.0, ke,
                              kd, 0.0, 0.01, 0.1, precision)
        forces.append(f)
    low, high = forces[0] - forces[1], forces[2] - forces[3]
    np.testing.assert_allclose(low, high, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(low, [0.0, 0.0, 2.0], rtol=1e-6, atol=1e-6)


# ---- identities ----------------------------------------------------------------------------
@pytest.mark.parametrize("precision", PRECISIONS)
def test_membrane_rest_state_is_force_free(precision):
    rest = REST.astype(np.float64)
    qp, rp = rest[1] - rest[0], rest[2] - rest[0]
    n = np.cross(qp, rp) / np.linalg.norm(np.cross(qp, rp))
    e1 = qp / np.linalg.norm(qp)
    e2 = np.cross(n, e1)
    D = np.array((e1, e2)) @ np.array((qp, rp)).T
    pose, area = np.linalg.inv(D), 0.5 * np.linalg.det(D)
    rng = np.random.default_rng(3)
    for _ in range(10):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        R = _rotations_from_quaternions(q[None, :].astype(np.float64)).astype(np.float64)[0]
        U, _, Vt = np.linalg.svd(R)
        R = U @ Vt
        pos = rest @ R.T + rng.uniform(-1, 1, size=3)
        for v in range(3):
            f, h = oracle.membrane(0, v, pos, pos, [[0, 1, 2]], pose.reshape(4), area, 1e4, 1e4, 0.0, 1e-3, precision)
            tol = 5e-2 if precision == "f32" else 1e-7
            assert np.linalg.norm(f) <= tol
            np.testing.assert_allclose(h, h.T, rtol=1e-6, atol=1e-6 * np.abs(h).max())


def _membrane_energy(pos, pose, area, mu, lmbd):
    x01, x02 = pos[1] - pos[0], pos[2] - pos[0]
    D = pose.reshape(2, 2).astype(np.float64)
    f0 = x01 * D[0, 0] + x02 * D[1, 0]
    f1 = x01 * D[0, 1] + x02 * D[1, 1]
    a, b, c = f0 @ f0, f1 @ f1, f0 @ f1
    js = math.sqrt(max(a * b - c * c, 1e-20))
    lnh = lmbd + mu
    alpha = 1.0 + mu / lnh
    return area * (0.5 * mu * (a + b - 2.0) + 0.5 * lnh * (js - alpha) ** 2)


def test_membrane_force_is_minus_energy_gradient():
    pose, area = _tri_rest_pose(REST)
    rng = np.random.default_rng(5)
    mu, lmbd = 3.0, 7.0
    for _ in range(5):
        pos = REST[:3].astype(np.float64) * rng.uniform(0.8, 1.25) + rng.normal(scale=0.05, size=(3, 3))
        for v in range(3):
            f, _ = oracle.membrane(0, v, pos, pos, [[0, 1, 2]], pose.reshape(4), area, mu, lmbd, 0.0, 1e-3, "f64")
            g = np.zeros(3)
            h = 1e-6
            for k in range(3):
                p1, p2 = pos.copy(), pos.copy()
                p1[v, k] += h
                p2[v, k] -= h
                g[k] = (_membrane_energy(p1, pose, area, mu, lmbd) - _membrane_energy(p2, pose, area, mu, lmbd)) / (2 * h)
            np.testing.assert_allclose(f, -g, rtol=1e-6, atol=1e-8)


def _dihedral(pos):
    x0, x1, x2, x3 = pos
    n1 = np.cross(x2 - x0, x3 - x0)
    n2 = np.cross(x3 - x1, x2 - x1)
    e = x3 - x2
    n1 /= np.linalg.norm(n1)
    n2 /= np.linalg.norm(n2)
    e /= np.linalg.norm(e)
    return math.atan2(np.dot(np.cross(n1, n2), e), np.dot(n1, n2))


def test_bending_force_is_minus_energy_gradient():
    """E = (ke L0 / 2)(theta - theta0)^2: force and Gauss-Newton Hessian k g g^T for all four vertices."""
    rng = np.random.default_rng(11)
    ke, L0, theta0 = 0.7, 1.3, 0.2
    for _ in range(5):
        pos = REST.astype(np.float64) + rng.normal(scale=0.1, size=(4, 3))
        theta = _dihedral(pos)
        for v in range(4):
            f, H = oracle.bending(0, v, pos, pos, [[0, 1, 2, 3]], theta0, L0, ke, 0.0, 1e-3, "f64")
            g = np.zeros(3)
            h = 1e-6
            for k in range(3):
                p1, p2 = pos.copy(), pos.copy()
                p1[v, k] += h
                p2[v, k] -= h
                g[k] = (_dihedral(p1) - _dihedral(p2)) / (2 * h)
            k_eff = ke * L0
            np.testing.assert_allclose(f, -k_eff * (theta - theta0) * g, rtol=1e-5, atol=1e-8)
            np.testing.assert_allclose(H, k_eff * np.outer(g, g), rtol=1e-5, atol=1e-8)


def test_boundary_hinge_is_zero():
    pos = REST.astype(np.float64)
    for v in range(4):
        f, h = oracle.bending(0, v, pos, pos, [[-1, 1, 2, 3]], 0.0, 1.0, 1.0, 1.0, 1e-3, "f32")
        assert np.all(f == 0) and np.all(h == 0)


def test_contact_friction_regimes():
    """IPC friction: linear ramp below eps_u, 1/|u| above (rigid_vbd_kernels.py:1604-1645)."""
    dt, feps, mu, ke = 0.01, 0.01, 0.5, 100.0
    eps_u = feps * dt
    n = np.array([0.0, 0.0, 1.0])
    for slip in (0.3 * eps_u, 3.0 * eps_u):
        x = np.array([slip, 0.0, -0.01])
        xp = np.array([0.0, 0.0, -0.01])
        f, H = oracle.contact(x, xp, [0, 0, 0], [0, 0, 0], n, 0.0, 0.0, ke, 0.0, mu, feps, dt, "f64")
        fn = 0.01 * ke
        f1 = 1.0 / slip if slip > eps_u else (-slip / eps_u + 2.0) / eps_u
        np.testing.assert_allclose(f, [-mu * fn * f1 * slip, 0.0, fn], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(H, ke * np.outer(n, n) + mu * fn * f1 * (np.eye(3) - np.outer(n, n)), rtol=1e-12)
