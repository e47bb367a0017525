"""The oracle's restatement of the sweep-residual gate (CPU): bounds and the fixed-count identity."""

import numpy as np

import oracle
from newton_b200 import scenes

DT = 1.0 / 600.0


def test_oracle_gated_step_bounds_and_identity():
    model, q0 = scenes.hanging_cloth(seed=3, device="cpu")
    qd = np.zeros_like(q0)
    orc = oracle.VBDOracle(model, "f32", threads=4)
    # a tolerance every residual meets: one iteration; one no residual meets: the cap
    _, q1, _, k1, _ = orc.gated_step(q0, qd, None, DT, 1e30, 20)
    _, q7, _, k7, r7 = orc.gated_step(q0, qd, None, DT, 0.0, 7)
    assert k1 == 1 and k7 == 7 and r7 > 0
    _, f1, _ = orc.step(q0, qd, None, DT, 1)
    _, f7, _ = orc.step(q0, qd, None, DT, 7)
    np.testing.assert_array_equal(q1, f1)
    np.testing.assert_array_equal(q7, f7)
    # check every 3: the cap is rounded up to a multiple of 3
    _, _, _, k3, _ = orc.gated_step(q0, qd, None, DT, 0.0, 7, check_every=3)
    assert k3 == 9
    # the sweep residual of the last iteration is each vertex's force norm at its visit
    r = orc.sweep_residual()
    solvable = ((model.particle_flags & 1) != 0) & (model.particle_mass != 0)
    assert (r[~solvable] == 0).all() and (r[solvable] > 0).all()


def test_oracle_relative_gate_refers_to_the_residual_at_the_inertia_target():
    model, q0 = scenes.hanging_cloth(seed=4, device="cpu")
    qd = np.zeros_like(q0)
    orc = oracle.VBDOracle(model, "f32", threads=4)
    orc.forward(q0, qd, None, DT)
    solvable = ((model.particle_flags & 1) != 0) & (model.particle_mass != 0)
    r_y = orc._norm(orc.residual(DT)[solvable], "mean")
    _, _, _, k, r = orc.gated_step(q0, qd, None, DT, 0.5, 200, relative=True)
    assert r <= np.float32(0.5) * np.float32(r_y) or k == 200
    # one iteration earlier the tolerance was not met
    if k > 1:
        _, _, _, k2, r2 = orc.gated_step(q0, qd, None, DT, 1e-30, k - 1, relative=True)
        assert k2 == k - 1 and r2 > np.float32(0.5) * np.float32(r_y)
