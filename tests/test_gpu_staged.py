"""GPU tests of the staged sweep (``SolverVBD.set_staged_sweep`` / ``vbd_set_staged_sweep``): each
block reads its one-ring positions from a shared-memory patch; the math and its order are the
unstaged sweep's, so every result must be bit-identical to it, for every launch shape, with
contacts, with damping, in batched worlds and under the residual gate."""

import numpy as np
import pytest
import torch

from newton_b200 import CollisionPipeline, scenes
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu
DT = 1.0 / 600.0


def _run(model, q0, steps, staged, launch=None, gate=None, margin=5e-3, **kw):
    solver = SolverVBD(model, iterations=10, **kw)
    if launch is not None:
        solver.set_launch(*launch)
    if staged:
        solver.set_staged_sweep(True)
    if gate is not None:
        solver.set_residual_gate(**gate)
    pipe = CollisionPipeline(model, soft_contact_margin=margin) if model.shape_count else None
    c = pipe.contacts() if pipe is not None else None
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q0).cuda())
    for _ in range(steps):
        if pipe is not None:
            pipe.collide(a, c)
        solver.step(a, b, None, c, DT)
        a, b = b, a
    torch.cuda.synchronize()
    info = solver.staged_sweep_info()
    stats = solver.gate_stats() if gate is not None else None
    return a.particle_q.clone(), a.particle_qd.clone(), info, stats


@pytest.mark.parametrize("launch", [(4, 128), (4, 64), (1, 128), (2, 128), (8, 256), (16, 256), (1, 256)])
def test_staged_sweep_is_bit_identical_on_the_hanging_cloth(launch):
    model, q0 = scenes.hanging_cloth(seed=2)   # triangle damping on: the staged step-start positions
    qa, va, info, _ = _run(model, q0, 30, True, launch)
    qb, vb, _, _ = _run(model, q0, 30, False, launch)
    assert info["active"] and 0 < info["max_patch"] <= 1536
    assert torch.equal(qa, qb) and torch.equal(va, vb)


def test_staged_sweep_is_bit_identical_with_contacts_and_in_batched_worlds():
    model, q0 = scenes.draped_cloth(n=64, seed=3, height=0.9)
    qa, va, info, _ = _run(model, q0, 40, True)
    qb, vb, _, _ = _run(model, q0, 40, False)
    assert info["active"] and torch.equal(qa, qb) and torch.equal(va, vb)
    model, q0 = scenes.batched_worlds(24, seed=5)
    for launch in ((2, 128), (4, 128)):
        qa, va, info, _ = _run(model, q0, 12, True, launch)
        qb, vb, _, _ = _run(model, q0, 12, False, launch)
        assert info["active"] and torch.equal(qa, qb) and torch.equal(va, vb)


def test_staged_sweep_under_the_residual_gate():
    model, q0 = scenes.draped_cloth(n=64, seed=4, height=0.9)
    gate = {"tolerance": 0.9, "max_iterations": 40, "relative": True, "norm": "mean", "residual": "sweep"}
    qa, va, _, sa = _run(model, q0, 25, True, gate=gate)
    qb, vb, _, sb = _run(model, q0, 25, False, gate=gate)
    assert sa["iterations"] == sb["iterations"] and sa["last_residual"] == sb["last_residual"]
    assert torch.equal(qa, qb) and torch.equal(va, vb)


def test_staged_sweep_follows_the_launch_shape_and_stays_off_with_self_contact():
    model, q0 = scenes.hanging_cloth(seed=0)
    s = SolverVBD(model, iterations=4)
    assert not s.staged_sweep_info()["active"]
    s.set_staged_sweep(True)
    first = s.staged_sweep_info()
    s.set_launch(1, 256)                       # patches rebuilt for 256 vertices per block
    second = s.staged_sweep_info()
    assert first["active"] and second["active"] and second["max_patch"] > first["max_patch"]
    s.set_launch(0, 128)                       # record-parallel shape: not staged
    assert not s.staged_sweep_info()["active"]
    s.set_staged_sweep(False)
    assert not s.staged_sweep_info()["active"]
    sc = SolverVBD(model, iterations=4, particle_enable_self_contact=True, particle_self_contact_radius=0.002,
                   particle_self_contact_margin=0.003)
    sc.set_staged_sweep(True)
    assert not sc.staged_sweep_info()["active"]
