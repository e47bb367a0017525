"""The reference's own cloth checks (``newton/tests/test_cloth.py``, VBD list ``:1220-1231``, and the
``cloth_hanging`` example check ``test_examples.py:498-506``) on the CUDA path, through
``SolverVBD.step`` with the reference's set-ups and tolerances (``tests/cloth_experiments.py``).

These exercise the membrane and bending stiffness, the PSD-projected membrane Hessian, damping,
particle-shape contact and self-contact over whole trajectories.  ``test_cloth_stitching`` is not
restated: it needs springs, which the VBD cloth path built here does not carry.
"""

import pytest

import cloth_experiments as X

pytestmark = pytest.mark.gpu

DEVICE = "cuda:0"


def test_cloth_sagging():
    spec = X.sagging(DEVICE)
    X.check_sagging(spec, X.run(spec, "gpu"))


def test_cloth_bending():
    spec = X.bending(DEVICE)
    X.check_stable_and_moved(spec, X.run(spec, "gpu"))


def test_cloth_collision():
    spec = X.collision(DEVICE)
    r = X.run(spec, "gpu")
    X.check_velocity_died_out(spec, r)
    assert (r.init_pos != r.q0).any()


def test_cloth_bending_consistent_angle_computation():
    spec = X.complex_rest_angles(DEVICE, tri_ke=1e2, tri_kd=0.0, edge_ke=1e-1, edge_kd=0.0, fixed=[1],
                                 use_gravity=False)
    diff = X.check_angles(spec, X.run(spec, "gpu"), 0.01)
    print(f"max |angle - rest angle| = {diff:.2e} rad (limit 0.01)")


def test_cloth_bending_non_zero_rest_angle_bending():
    spec = X.cylinder(DEVICE)
    X.check_stable_and_moved(spec, X.run(spec, "gpu"), absolute=True)


def test_cloth_bending_with_complex_rest_angles():
    spec = X.complex_rest_angles(DEVICE, tri_ke=1e3, tri_kd=0.0, edge_ke=1e3, edge_kd=1e0, fixed=[1])
    r = X.run(spec, "gpu")
    X.check_stable_and_moved(spec, r, absolute=True)
    diff = X.check_angles(spec, r, 0.1)
    print(f"max |angle - rest angle| = {diff:.3f} rad (limit 0.1)")


def test_cloth_free_fall_with_internal_forces_and_damping():
    spec = X.complex_rest_angles(DEVICE, tri_ke=5e1, tri_kd=5e0, edge_ke=1e1, edge_kd=1e0)
    diff, off = X.check_free_fall_internal_forces(spec, X.run(spec, "gpu"))
    print(f"max angle change {diff:.3f} rad (limit 0.1), max non-gravitational displacement {off:.2e} (limit 0.02)")


def test_cloth_free_fall():
    spec = X.free_fall(DEVICE)
    X.check_free_fall(spec, X.run(spec, "gpu"))


def test_cloth_body_collision():
    spec = X.body_collision(DEVICE)
    X.check_body_collision(spec, X.run(spec, "gpu"))


def test_example_cloth_hanging():
    """The example test's default (CUDA) options: 64 x 32 grid, 100 frames, self-contact on."""
    spec = X.example_cloth_hanging(DEVICE)
    X.check_example_hanging(spec, X.run(spec, "gpu"), width=64)
