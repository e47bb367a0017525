"""notify_model_changed: gravity and shape edits take effect on the next step (the reference reads
them from the model at every step); unrelated flags change nothing."""

import numpy as np
import pytest
import torch

import oracle
from newton_b200 import CollisionPipeline, ModelFlags, scenes
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0


def test_gravity_change_applies_after_notify():
    model, q0 = scenes.hanging_cloth(seed=8)
    solver = SolverVBD(model, iterations=10)
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q0).cuda())
    for _ in range(3):
        solver.step(a, b, None, None, DT)
        a, b = b, a
    model.gravity = np.array([[1.5, 0.0, -3.0]], np.float32)
    solver.notify_model_changed(ModelFlags.BODY_PROPERTIES)  # no particle effect
    solver.notify_model_changed(ModelFlags.MODEL_PROPERTIES)
    q_in, qd_in = a.particle_q.cpu().numpy().copy(), a.particle_qd.cpu().numpy().copy()
    solver.step(a, b, None, None, DT)
    orc = oracle.VBDOracle(model, "f32")
    _, q_ref, _ = orc.step(q_in, qd_in, None, DT, 10)
    assert np.abs(b.particle_q.cpu().numpy() - q_ref).max() <= 1e-5


def test_moved_shape_applies_after_notify():
    model, q0 = scenes.single_cloth(n=24, side=1.0, seed=9, pin_top_corners=False, ground=None,
                                    sphere=((0.0, 0.0, -0.39), 0.4), height=0.0)
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    a = model.state()
    a.particle_q.copy_(torch.from_numpy(q0).cuda())
    pipe.collide(a, c)
    n_before = c.count()
    assert n_before > 0
    tf = model.shape_transform.copy()
    tf[0, 2] = -2.0  # the sphere drops out of reach
    model.shape_transform = tf
    solver.notify_model_changed(ModelFlags.SHAPE_PROPERTIES)
    pipe.collide(a, c)
    assert c.count() == 0
    b = model.state()
    q_in = a.particle_q.cpu().numpy().copy()
    solver.step(a, b, None, c, DT)
    orc = oracle.VBDOracle(model, "f32")
    orc.set_contacts(*oracle.collide(model, q_in, 5e-3))
    _, q_ref, _ = orc.step(q_in, np.zeros_like(q_in), None, DT, 10)
    assert np.abs(b.particle_q.cpu().numpy() - q_ref).max() <= 1e-5
