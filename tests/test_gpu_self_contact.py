"""Cloth self-contact on the GPU against the CPU oracle.

The scene is a square cloth folded over itself: the right half is mirrored onto the left half
and lifted by 3 mm, so vertex-triangle and edge-edge pairs are inside the contact radius
(4 mm) from the first step.  Detection must find exactly the oracle's candidate lists; a step
from identical states must agree with the oracle within 1e-5 m per coordinate; repeated runs
are bit-identical; and over a longer run the two layers never pass through each other.
"""

import numpy as np
import pytest
import torch

import oracle
from newton_b200 import CollisionPipeline, scenes
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0
RADIUS, MARGIN = 0.004, 0.006
TOL = 1e-5


def _folded(n=24, side=0.5, gap=0.003, ground=None):
    model, q0 = scenes.single_cloth(n=n, side=side, seed=0, pin_top_corners=False, ground=ground, z_noise=0.0)
    q = q0.astype(np.float64).copy()
    right = q[:, 0] > 0.0
    q[right, 0] = -q[right, 0]
    q[right, 2] += gap
    model.soft_contact_ke = 1.0e3
    model.soft_contact_kd = 1.0e-2
    model.soft_contact_mu = 0.2
    return model, q.astype(np.float32), right


def _solver(model, iterations=5, **kw):
    return SolverVBD(model, iterations=iterations, particle_enable_self_contact=True,
                     particle_self_contact_radius=RADIUS, particle_self_contact_margin=MARGIN, **kw)


def _oracle(model, iterations_kw=None, vb=32, eb=64):
    orc = oracle.VBDOracle(model, "f32")
    orc.set_self_contact(radius=RADIUS, margin=MARGIN, vertex_buffer=vb, edge_buffer=eb, rest_q=model.particle_q)
    return orc


def test_detection_matches_oracle():
    model, q, _ = _folded()
    solver = _solver(model, particle_vertex_contact_buffer_size=64, particle_edge_contact_buffer_size=128)
    vc, vl, ec, el = solver.self_contact_detect(torch.from_numpy(q).cuda())
    orc = _oracle(model, vb=64, eb=128)
    ovc, ovl, oec, oel, dropped = orc.self_contact_detect(q)
    assert dropped == 0
    assert vc.sum() > 0 and ec.sum() > 0
    np.testing.assert_array_equal(vc, ovc)
    np.testing.assert_array_equal(vl, ovl)
    np.testing.assert_array_equal(ec, oec)
    np.testing.assert_array_equal(el, oel)
    assert solver.status()["self_contact_overflow"] == 0


@pytest.mark.parametrize("interval", [0, -1, 2])
def test_step_matches_oracle(interval):
    model, q, _ = _folded()
    solver = _solver(model, particle_collision_detection_interval=interval)
    orc = _oracle(model)
    orc.set_self_contact(radius=RADIUS, margin=MARGIN, interval=interval, rest_q=model.particle_q)
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q).cuda())
    worst = 0.0
    for _ in range(6):
        q_in = a.particle_q.cpu().numpy().copy()
        qd_in = a.particle_qd.cpu().numpy().copy()
        solver.step(a, b, None, None, DT)
        _, q_ref, qd_ref = orc.step(q_in, qd_in, None, DT, 5)
        q_gpu = b.particle_q.cpu().numpy()
        worst = max(worst, float(np.abs(q_gpu - q_ref).max()))
        a, b = b, a
    st = solver.status()
    assert st["nonfinite_updates"] == 0 and st["self_contact_overflow"] == 0
    print(f"self-contact step parity (interval {interval}): max |dx| = {worst:.3e} m over 6 steps")
    assert worst <= TOL, worst


def test_detection_with_external_filter_maps_matches_oracle():
    model, q, _ = _folded()
    orc = _oracle(model, vb=64, eb=128)
    ovc, ovl, oec, oel, _ = orc.self_contact_detect(q)
    rng = np.random.default_rng(5)
    vmap = {int(v): set(ovl[v, :ovc[v]][: 2].tolist()) for v in rng.choice(np.flatnonzero(ovc), 20, replace=False)}
    emap = {int(e): set(oel[e, :oec[e]][::2].tolist()) for e in rng.choice(np.flatnonzero(oec), 40, replace=False)}
    orc.set_self_contact(radius=RADIUS, margin=MARGIN, vertex_buffer=64, edge_buffer=128, rest_q=model.particle_q,
                         vertex_filter_map=vmap, edge_filter_map=emap)
    ovc, ovl, oec, oel, _ = orc.self_contact_detect(q)
    solver = _solver(model, particle_vertex_contact_buffer_size=64, particle_edge_contact_buffer_size=128,
                     particle_external_vertex_contact_filtering_map=vmap,
                     particle_external_edge_contact_filtering_map=emap)
    vc, vl, ec, el = solver.self_contact_detect(torch.from_numpy(q).cuda())
    np.testing.assert_array_equal(vc, ovc)
    np.testing.assert_array_equal(vl, ovl)
    np.testing.assert_array_equal(ec, oec)
    np.testing.assert_array_equal(el, oel)


def test_step_with_body_contacts_matches_oracle():
    """Self-contact and particle-shape contact in the same step: the lower layer lies in the
    ground plane's contact band (plane 4 mm below, particle radius 5 mm, margin 5 mm)."""
    model, q, _ = _folded(ground=-0.004)
    solver = _solver(model)
    orc = _oracle(model)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q).cuda())
    worst = 0.0
    n_contacts = 0
    for _ in range(4):
        q_in = a.particle_q.cpu().numpy().copy()
        qd_in = a.particle_qd.cpu().numpy().copy()
        pipe.collide(a, c)
        n_contacts = max(n_contacts, c.count())
        solver.step(a, b, None, c, DT)
        orc.set_contacts(*oracle.collide(model, q_in, 5e-3))
        _, q_ref, _ = orc.step(q_in, qd_in, None, DT, 5)
        worst = max(worst, float(np.abs(b.particle_q.cpu().numpy() - q_ref).max()))
        a, b = b, a
    print(f"self-contact + ground contact parity: max |dx| = {worst:.3e} m, {n_contacts} ground contacts")
    assert n_contacts > 0
    assert solver.status()["nonfinite_updates"] == 0
    assert worst <= TOL, worst


def test_cloth_on_boxes_small_matches_oracle():
    """The config-5 scene shape at 48 x 48 (4 m side scaled to 0.5 m): self-contact and box / ground
    contacts together, per step from identical states over the first folds."""
    model, q0 = scenes.cloth_on_boxes(n=48, side=0.5, boxes=4, seed=3, height=0.12)
    solver = _solver(model, iterations=10)
    orc = _oracle(model)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q0).cuda())
    worst, steps_checked = 0.0, 0
    for step in range(150):
        check = step % 30 == 29
        if check:
            q_in = a.particle_q.cpu().numpy().copy()
            qd_in = a.particle_qd.cpu().numpy().copy()
        pipe.collide(a, c)
        solver.step(a, b, None, c, DT)
        if check:
            orc.set_contacts(*oracle.collide(model, q_in, 5e-3))
            _, q_ref, _ = orc.step(q_in, qd_in, None, DT, 10)
            worst = max(worst, float(np.abs(b.particle_q.cpu().numpy() - q_ref).max()))
            steps_checked += 1
        a, b = b, a
    vc, _, ec, _ = solver.self_contact_detect(a.particle_q)
    print(f"cloth on boxes 48x48: max |dx| = {worst:.3e} m over {steps_checked} checked steps; "
          f"{int(vc.sum())} vertex-triangle and {int(ec.sum())} edge-edge pairs at the end")
    st = solver.status()
    assert st["nonfinite_updates"] == 0 and st["self_contact_overflow"] == 0
    assert worst <= TOL, worst


def test_staged_step_matches_step():
    model, q, _ = _folded()
    out = []
    for staged in (False, True):
        solver = _solver(model, use_cuda_graph=False)
        a, b = model.state(), model.state()
        a.particle_q.copy_(torch.from_numpy(q).cuda())
        for _ in range(3):
            if staged:
                solver.forward(a, None, DT)
                solver.iterate(None, DT, 5)
                solver.finalize(a, b, DT)
            else:
                solver.step(a, b, None, None, DT)
            a, b = b, a
        torch.cuda.synchronize()
        out.append(a.particle_q.clone())
    assert torch.equal(out[0], out[1])


def test_layers_do_not_pass_through_and_runs_are_deterministic():
    model, q, right = _folded()
    runs = []
    for _ in range(2):
        solver = _solver(model, iterations=10)
        a, b = model.state(), model.state()
        a.particle_q.copy_(torch.from_numpy(q).cuda())
        for _ in range(120):
            solver.step(a, b, None, None, DT)
            a, b = b, a
        torch.cuda.synchronize()
        st = solver.status()
        assert st["nonfinite_updates"] == 0 and st["self_contact_overflow"] == 0
        runs.append(a.particle_q.cpu().numpy())
    assert np.array_equal(runs[0], runs[1])
    x = runs[0]
    assert np.isfinite(x).all()
    # every lifted (right-half) vertex is still above the lower layer near it
    lower = x[~right]
    for p in x[right]:
        d = np.linalg.norm(lower[:, :2] - p[:2], axis=1)
        k = np.argsort(d)[:3]
        assert p[2] > lower[k, 2].min() - 1e-4


def test_full_size_cloth_on_boxes_is_deterministic_and_clean():
    """The benchmark's self-contact workload at full size (1024 x 1024 = 1,048,576 vertices on 16
    boxes): two independent solvers stepped 150 times from the same state end bit-identical,
    finite, with no dropped contact, singular block or non-finite update."""
    model, q0 = scenes.cloth_on_boxes(n=1024)
    runs = []
    for _ in range(2):
        solver = SolverVBD(model, iterations=10, particle_enable_self_contact=True,
                           particle_self_contact_radius=0.002, particle_self_contact_margin=0.003)
        pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
        c = pipe.contacts()
        s0, s1 = model.state(), model.state()
        s0.particle_q.copy_(torch.from_numpy(q0).cuda())
        for _ in range(150):
            pipe.collide(s0, c)
            solver.step(s0, s1, None, c, 1.0 / 600.0)
            s0, s1 = s1, s0
        torch.cuda.synchronize()
        runs.append(s0.particle_q.cpu().numpy())
        st = solver.status()
        assert st["nonfinite_updates"] == 0 and st["singular_blocks"] == 0
        assert st["contact_overflow"] == 0 and st["self_contact_overflow"] == 0
        assert c.count() > 0
        del solver, pipe, c, s0, s1
        torch.cuda.empty_cache()
    assert np.isfinite(runs[0]).all()
    assert np.array_equal(runs[0], runs[1])
