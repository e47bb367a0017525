"""Edge cases of the CUDA step: an empty model, particles without elements, zero iterations, a
fully pinned cloth and uneven world sizes -- each against the oracle or the exact expectation."""

import numpy as np
import pytest
import torch

import oracle
from newton_b200 import ModelBuilder, scenes
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0


def _step(model, q0, iterations=10, steps=1):
    solver = SolverVBD(model, iterations=iterations)
    a, b = model.state(), model.state()
    if q0 is not None:
        a.particle_q.copy_(torch.from_numpy(q0).cuda())
    for _ in range(steps):
        solver.step(a, b, None, None, DT)
        a, b = b, a
    torch.cuda.synchronize()
    return a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy(), solver


def test_empty_model_steps_as_a_no_op():
    b = ModelBuilder()
    m = b.finalize("cuda:0")
    solver = SolverVBD(m)
    s0, s1 = m.state(), m.state()
    solver.step(s0, s1, None, None, DT)
    assert s0.particle_q.numel() == 0


def test_free_particles_without_elements_fall_like_the_oracle():
    b = ModelBuilder()
    rng = np.random.default_rng(0)
    for k in range(37):
        b.add_particle(tuple(rng.uniform(-1, 1, 3)), (0.0, 0.0, 0.0), float(rng.uniform(0.01, 1.0)))
    b.add_particle((0.0, 0.0, 2.0), (0.0, 0.0, 0.0), 0.0)  # massless: stays
    b.color()
    m = b.finalize("cuda:0")
    q, qd, _ = _step(m, None, steps=3)
    orc = oracle.VBDOracle(m, "f32")
    x, v = m.particle_q.copy(), np.zeros_like(m.particle_q)
    for _ in range(3):
        _, x, v = orc.step(x, v, None, DT, 10)
    assert np.abs(q - x).max() <= 1e-6
    np.testing.assert_array_equal(q[-1], m.particle_q[-1])


def test_zero_iterations_is_the_inertia_step():
    model, q0 = scenes.hanging_cloth(seed=4)
    q, qd, _ = _step(model, q0, iterations=0)
    g = np.array([0.0, 0.0, -9.81], np.float32)
    solvable = ((model.particle_flags & 1) != 0) & (model.particle_inv_mass != 0)
    expect = q0 + (g * np.float32(DT)) * np.float32(DT)
    np.testing.assert_allclose(q[solvable], expect[solvable], atol=1e-7)
    np.testing.assert_array_equal(q[~solvable], q0[~solvable])


def test_fully_pinned_cloth_does_not_move():
    b = ModelBuilder()
    verts, tris = ModelBuilder.grid_mesh(7, 7, 0.1, 0.1)
    b.add_cloth_mesh(pos=(0.0, 0.0, 1.0), rot=(0.0, 0.0, 0.0, 1.0), scale=1.0, vel=(0.0, 0.0, 0.0), vertices=verts,
                     indices=tris, density=0.1, tri_ke=1e4, tri_ka=1e4, tri_kd=1e-3, edge_ke=1e-2)
    b.set_particle_mass(np.arange(b.particle_count), 0.0)
    b.color(include_bending=True)
    m = b.finalize("cuda:0")
    q, qd, solver = _step(m, None, steps=5)
    np.testing.assert_array_equal(q, m.particle_q)
    assert np.all(qd == 0.0)
    assert solver.status()["nonfinite_updates"] == 0


def test_uneven_worlds_with_single_vertex_colors_match_the_oracle():
    model, q0 = scenes.batched_worlds(num_worlds=9, seed=21, n_range=(2, 6))
    q, qd, _ = _step(model, q0, steps=2)
    orc = oracle.VBDOracle(model, "f32")
    x, v = q0.copy(), np.zeros_like(q0)
    for _ in range(2):
        _, x, v = orc.step(x, v, None, DT, 10)
    assert np.abs(q - x).max() <= 1e-5
