"""The reference's own cloth checks (``newton/tests/test_cloth.py``, VBD list ``:1220-1231``, and the
``cloth_hanging`` example check ``test_examples.py:498-506``) run on the CPU oracle.

These are the reference-held checks that exercise the membrane and bending stiffness, the PSD
projection of the membrane Hessian and the contact law end to end: a sheet sagging from two pins,
bending sheets, hinges returning to non-zero rest angles, free fall with and without internal
forces and damping, a sheet settling on a box, a triangle falling onto a fixed sheet with
self-contact.  The same experiments run on the GPU in ``test_gpu_reference_cloth.py``; here
they pin the oracle that the GPU parity tests compare against.  ``test_cloth_stitching`` is not
restated: it needs springs, which the VBD cloth path built here does not carry.
"""

import cloth_experiments as X

DEVICE = "cpu"


def test_cloth_sagging_oracle():
    spec = X.sagging(DEVICE)
    X.check_sagging(spec, X.run(spec, "oracle"))


def test_cloth_bending_oracle():
    spec = X.bending(DEVICE)
    X.check_stable_and_moved(spec, X.run(spec, "oracle"))


def test_cloth_collision_oracle():
    spec = X.collision(DEVICE)
    r = X.run(spec, "oracle")
    X.check_velocity_died_out(spec, r)
    assert (r.init_pos != r.q0).any()


def test_cloth_bending_consistent_angle_computation_oracle():
    spec = X.complex_rest_angles(DEVICE, tri_ke=1e2, tri_kd=0.0, edge_ke=1e-1, edge_kd=0.0, fixed=[1],
                                 use_gravity=False)
    X.check_angles(spec, X.run(spec, "oracle"), 0.01)


def test_cloth_bending_non_zero_rest_angle_oracle():
    spec = X.cylinder(DEVICE)
    X.check_stable_and_moved(spec, X.run(spec, "oracle"), absolute=True)


def test_cloth_bending_with_complex_rest_angles_oracle():
    spec = X.complex_rest_angles(DEVICE, tri_ke=1e3, tri_kd=0.0, edge_ke=1e3, edge_kd=1e0, fixed=[1])
    r = X.run(spec, "oracle")
    X.check_stable_and_moved(spec, r, absolute=True)
    X.check_angles(spec, r, 0.1)


def test_cloth_free_fall_with_internal_forces_and_damping_oracle():
    spec = X.complex_rest_angles(DEVICE, tri_ke=5e1, tri_kd=5e0, edge_ke=1e1, edge_kd=1e0)
    X.check_free_fall_internal_forces(spec, X.run(spec, "oracle"))


def test_cloth_free_fall_oracle():
    spec = X.free_fall(DEVICE)
    X.check_free_fall(spec, X.run(spec, "oracle"))


def test_cloth_body_collision_oracle():
    spec = X.body_collision(DEVICE)
    X.check_body_collision(spec, X.run(spec, "oracle"))


def test_example_cloth_hanging_oracle():
    """The example test's CPU options: 32 x 16 grid, 10 frames."""
    spec = X.example_cloth_hanging(DEVICE, width=32, height=16, frames=10)
    X.check_example_hanging(spec, X.run(spec, "oracle"), width=32)
