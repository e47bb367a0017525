"""GPU parity of the VBD cloth step against the CPU oracle (FP32 and FP64).

Parity criterion (per step, from identical states): max |x_gpu - x_oracle| <= 1e-5 m after one
``SolverVBD.step`` with the same inputs, against the FP32 oracle and against the FP64
re-evaluation of the same step (both asserted).  Every parity result also states the force
residual of the GPU's result, max_i |f_i| / (m_i |g|) and its mean, evaluated by the FP64 oracle
at the GPU positions with the step's inertia targets and contacts.  All calls go through the
C-ABI library (``libvbd_b200.so``).
"""

import numpy as np
import pytest
import torch

import oracle
from newton_b200 import CollisionPipeline, scenes
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

TOL_STEP = 1.0e-5  # m, per step from identical states
DT = 1.0 / 600.0


def _gpu_step(model, solver, q, qd, pipe, dt, iterations=None):
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.from_numpy(np.ascontiguousarray(q)).to(s0.particle_q.device))
    s0.particle_qd.copy_(torch.from_numpy(np.ascontiguousarray(qd)).to(s0.particle_q.device))
    contacts = None
    if pipe is not None:
        contacts = pipe.contacts()
        pipe.collide(s0, contacts)
    if iterations is not None:
        solver.iterations = iterations
    solver.step(s0, s1, None, contacts, dt)
    torch.cuda.synchronize()
    return s0.particle_q.cpu().numpy(), s1.particle_q.cpu().numpy(), s1.particle_qd.cpu().numpy(), contacts


def _oracle_step(model, orc, q, qd, margin, dt, iterations):
    if model.shape_count:
        orc.set_contacts(*oracle.collide(model, q, margin))
    return orc.step(q, qd, None, dt, iterations)


def _residual_of(orc64, q_gpu):
    """Force residual (max, mean over solvable vertices; units of m|g|) of the GPU's positions,
    evaluated by the FP64 oracle right after its own step from the same state (same inertia
    targets, anchors and contacts)."""
    orc64.set_positions(q_gpu)
    r = orc64.residual(DT)
    m = orc64.model
    solvable = ((m.particle_flags & 1) != 0) & (m.particle_mass != 0)
    return float(r.max()), float(r[solvable].mean()) if solvable.any() else 0.0


def _report(name, err, err64, resid):
    print(f"{name}: max |dx| vs FP32 oracle {err:.3e} m, vs FP64 {err64:.3e} m; "
          f"force residual of the GPU result max {resid[0]:.4g} / mean {resid[1]:.4g} m|g|")


def _trajectory_parity(model, q0, steps, iterations, margin=5e-3, check_every=1):
    orc32 = oracle.VBDOracle(model, "f32", threads=8)
    orc64 = oracle.VBDOracle(model, "f64", threads=8)
    solver = SolverVBD(model, iterations=iterations)
    pipe = CollisionPipeline(model, soft_contact_margin=margin) if model.shape_count else None
    q, qd = q0.astype(np.float32), np.zeros_like(q0, dtype=np.float32)
    worst, worst64, resid = 0.0, 0.0, (0.0, 0.0)
    for k in range(steps):
        qin_o, q_o, qd_o = _oracle_step(model, orc32, q, qd, margin, DT, iterations)
        if k % check_every == 0:
            qin_g, q_g, qd_g, _ = _gpu_step(model, solver, q, qd, pipe, DT)
            _, q_64, _ = _oracle_step(model, orc64, q, qd, margin, DT, iterations)
            err = float(np.abs(q_g - q_o).max())
            err64 = float(np.abs(q_g - q_64).max())
            r = _residual_of(orc64, q_g)
            resid = max(resid, r)
            # aliasing: state_in.particle_q holds the solved positions, like the reference
            assert np.array_equal(qin_g, q_g)
            assert np.abs(qd_g - qd_o).max() <= 2.0 * TOL_STEP / DT
            worst, worst64 = max(worst, err), max(worst64, err64)
            assert err <= TOL_STEP, f"step {k}: max |dx| = {err:.3e} m vs FP32 oracle"
            assert err64 <= TOL_STEP, f"step {k}: max |dx| = {err64:.3e} m vs FP64 re-evaluation"
            assert np.isfinite(r[0])
        q, qd = q_o, qd_o
    return worst, worst64, resid


def test_hanging_cloth_single_step():
    model, q0 = scenes.hanging_cloth(seed=0)
    _report("hanging 32x32, 1 step", *_trajectory_parity(model, q0, steps=1, iterations=10))


def test_hanging_cloth_trajectory_per_step():
    """30 substeps (3 frames): every step from the oracle's own state stays within 1e-5 m."""
    model, q0 = scenes.hanging_cloth(seed=1)
    _report("hanging 32x32, 30 steps", *_trajectory_parity(model, q0, steps=30, iterations=10, check_every=3))


def test_draped_cloth_contacts_per_step():
    """Sphere + ground contacts: cloth released just above the sphere so contacts are active."""
    model, q0 = scenes.single_cloth(n=48, side=1.0, seed=2, pin_top_corners=False, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.905)
    _report("draped 48x48 on sphere + ground, 12 steps",
            *_trajectory_parity(model, q0, steps=12, iterations=10, check_every=2))


def test_collide_matches_oracle():
    model, q0 = scenes.single_cloth(n=40, side=1.0, seed=3, pin_top_corners=False, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.902)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    s = model.state()
    s.particle_q.copy_(torch.from_numpy(q0).cuda())
    pipe.collide(s, c)
    n = c.count()
    assert n > 0
    part = c.soft_contact_particle[:n].cpu().numpy()
    shp = c.soft_contact_shape[:n].cpu().numpy()
    order = np.lexsort((shp, part))
    op, osh, obp, obv, onr = oracle.collide(model, q0, 5e-3)
    assert n == len(op)
    np.testing.assert_array_equal(part[order], op)
    np.testing.assert_array_equal(shp[order], osh)
    np.testing.assert_allclose(c.soft_contact_body_pos[:n].cpu().numpy()[order], obp, atol=1e-6)
    np.testing.assert_allclose(c.soft_contact_normal[:n].cpu().numpy()[order], onr, atol=1e-6)
    # records of one particle are consecutive and in shape order
    for p in np.unique(part):
        idx = np.flatnonzero(part == p)
        assert np.all(np.diff(idx) == 1) and np.all(np.diff(shp[idx]) > 0)


def test_staged_api_matches_step_and_oracle_per_color():
    model, q0 = scenes.hanging_cloth(seed=4)
    V = model.particle_count
    qd = np.zeros((V, 3), np.float32)
    solver = SolverVBD(model, iterations=2)
    orc = oracle.VBDOracle(model, "f32")
    s0 = model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).cuda())
    solver.forward(s0, None, DT)
    orc.forward(q0, qd, None, DT)
    np.testing.assert_allclose(solver.positions().cpu().numpy(), orc.positions(), atol=1e-7)
    for it in range(2):
        orc.begin_iteration()
        for c in range(len(model.particle_color_groups)):
            solver.sweep_color(c, None, DT)
            orc.sweep_color(c, DT)
            err = np.abs(solver.positions().cpu().numpy() - orc.positions()).max()
            assert err <= TOL_STEP, f"iteration {it} color {c}: {err:.3e}"
    s1 = model.state()
    solver.finalize(s0, s1, DT)
    staged = s1.particle_q.cpu().numpy()
    _, full, _, _ = _gpu_step(model, solver, q0, qd, None, DT)
    np.testing.assert_array_equal(staged, full)


def test_graph_replay_and_plain_launches_are_bitwise_equal_and_deterministic():
    model, q0 = scenes.single_cloth(n=48, side=1.0, seed=5, pin_top_corners=False, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.905)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    outs = []
    for use_graph in (True, True, False):
        solver = SolverVBD(model, iterations=5, use_cuda_graph=use_graph)
        s0, s1 = model.state(), model.state()
        s0.particle_q.copy_(torch.from_numpy(q0).cuda())
        c = pipe.contacts()
        for _ in range(6):
            pipe.collide(s0, c)
            solver.step(s0, s1, None, c, DT)
            s0, s1 = s1, s0
        torch.cuda.synchronize()
        outs.append(s0.particle_q.cpu().numpy())
        st = solver.status()
        assert st["nonfinite_updates"] == 0 and st["contact_overflow"] == 0
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])


@pytest.mark.parametrize("lanes", [0, 1, 2, 4, 8, 16])
def test_launch_shapes_agree(lanes):
    model, q0 = scenes.hanging_cloth(seed=6)
    qd = np.zeros_like(q0)
    ref = None
    for block in (64, 128, 256):
        solver = SolverVBD(model, iterations=4, lanes_per_vertex=lanes, block_size=block)
        _, q, _, _ = _gpu_step(model, solver, q0, qd, None, DT)
        if ref is None:
            ref = q
        np.testing.assert_array_equal(q, ref)  # block size never changes the arithmetic
    orc = oracle.VBDOracle(model, "f32")
    _, q_o, _ = orc.step(q0, qd, None, DT, 4)
    assert np.abs(ref - q_o).max() <= TOL_STEP


def test_residual_matches_oracle():
    """Jacobi force residual at the GPU's own iterate, GPU (FP32) vs oracle (FP64)."""
    model, q0 = scenes.hanging_cloth(seed=7)
    V = model.particle_count
    qd = np.zeros((V, 3), np.float32)
    solver = SolverVBD(model, iterations=3)
    orc = oracle.VBDOracle(model, "f64")
    s0 = model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).cuda())
    solver.forward(s0, None, DT)
    solver.iterate(None, DT, 3)
    orc.forward(q0, qd, None, DT)
    orc.set_positions(solver.positions().cpu().numpy())
    mx, pv = solver.residual(None, DT, per_vertex=True)
    r_gpu = pv.cpu().numpy()
    r_orc = orc.residual(DT)
    assert abs(float(mx.item()) - r_gpu.max()) <= 1e-6 * max(1.0, r_gpu.max())
    assert r_orc.max() > 0
    np.testing.assert_allclose(r_gpu, r_orc, rtol=1e-3, atol=1e-3 * max(1.0, r_orc.max()))


def test_batched_worlds_per_step():
    model, q0 = scenes.batched_worlds(num_worlds=6, seed=8, n_range=(8, 20))
    _report("batched 6 worlds, 4 steps", *_trajectory_parity(model, q0, steps=4, iterations=10, check_every=1))


def test_invalid_state_is_rejected():
    model, q0 = scenes.hanging_cloth(seed=9)
    solver = SolverVBD(model, iterations=1)
    s0, s1 = model.state(), model.state()
    s0.particle_q = s0.particle_q.double()
    with pytest.raises(ValueError):
        solver.step(s0, s1, None, None, DT)


def test_step_kernel_count_matches_the_step_structure():
    """The step graph holds forward (+ the contact pack when contacts are given), one sweep per
    color and iteration, and finalize; a plain (non-graph) step reports -1."""
    model, q0 = scenes.single_cloth(n=16, side=0.5, seed=3, pin_top_corners=False, ground=0.0,
                                    sphere=((0.0, 0.0, -0.2), 0.2), height=0.002)
    colors = len(model.particle_color_groups)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    for contacts in (None, pipe.contacts()):
        solver = SolverVBD(model, iterations=3)
        s0, s1 = model.state(), model.state()
        s0.particle_q.copy_(torch.from_numpy(q0).cuda())
        if contacts is not None:
            pipe.collide(s0, contacts)
        solver.step(s0, s1, None, contacts, DT)
        torch.cuda.synchronize()
        expect = 1 + (1 if contacts is not None else 0) + 3 * colors + 1
        assert solver.step_kernel_count() == expect
    solver = SolverVBD(model, iterations=3, use_cuda_graph=False)
    s0, s1 = model.state(), model.state()
    solver.step(s0, s1, None, None, DT)
    assert solver.step_kernel_count() == -1


def test_batch_step_equals_individual_steps():
    """vbd_batch_step over independent solvers (different meshes, with and without contacts, their
    own iteration counts) gives bit-identical results to one step call per solver."""
    specs = [
        scenes.single_cloth(n=12, side=0.5, seed=4, pin_top_corners=True, ground=0.0,
                            sphere=((0.0, 0.0, -0.2), 0.2), height=0.002),
        scenes.hanging_cloth(seed=8),
        scenes.single_cloth(n=20, side=0.8, seed=9, pin_top_corners=False, ground=0.0,
                            sphere=((0.0, 0.0, 0.3), 0.3), height=0.61),
    ]
    iters = [3, 5, 4]

    def setup():
        out = []
        for (model, q0), it in zip(specs, iters):
            solver = SolverVBD(model, iterations=it)
            pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
            c = pipe.contacts() if model.shape_count > 0 else None
            s0, s1 = model.state(), model.state()
            s0.particle_q.copy_(torch.from_numpy(q0).cuda())
            out.append((solver, pipe, c, s0, s1))
        return out

    single, batch = setup(), setup()
    for _ in range(3):
        for solver, pipe, c, s0, s1 in single:
            if c is not None:
                pipe.collide(s0, c)
            solver.step(s0, s1, None, c, DT)
            s0.assign(s1)
        for solver, pipe, c, s0, s1 in batch:
            if c is not None:
                pipe.collide(s0, c)
        SolverVBD.step_batch([b[0] for b in batch], [b[3] for b in batch], [b[4] for b in batch],
                             [b[2] for b in batch], DT)
        for b in batch:
            b[3].assign(b[4])
    torch.cuda.synchronize()
    for a, b in zip(single, batch):
        assert torch.equal(a[4].particle_q, b[4].particle_q)
        assert torch.equal(a[4].particle_qd, b[4].particle_qd)
    with pytest.raises(ValueError):
        SolverVBD.step_batch([single[0][0]], [], [], None, DT)


def test_full_size_draped_cloth_step_matches_oracle():
    """The benchmark's draped cloth at its full size (256 x 256, 65,536 vertices, sphere + ground):
    drape it on the GPU until it rests on the sphere, then one GPU step and one FP32 oracle step
    from that same state agree to TOL_STEP, contacts included."""
    import os

    model, q0 = scenes.draped_cloth(n=256, seed=0)
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).cuda())
    for _ in range(300):  # 0.5 s: the cloth lands on the sphere after ~0.2 s
        pipe.collide(s0, c)
        solver.step(s0, s1, None, c, DT)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    q = s0.particle_q.cpu().numpy()
    qd = s0.particle_qd.cpu().numpy()
    assert np.isfinite(q).all()
    _, q_g, qd_g, contacts = _gpu_step(model, solver, q, qd, pipe, DT)
    assert contacts.count() > 1000, "the cloth should rest on the sphere"
    orc = oracle.VBDOracle(model, "f32", threads=os.cpu_count() or 1)
    _, q_o, qd_o = _oracle_step(model, orc, q, qd, 5e-3, DT, 10)
    orc64 = oracle.VBDOracle(model, "f64", threads=os.cpu_count() or 1)
    _, q_64, _ = _oracle_step(model, orc64, q, qd, 5e-3, DT, 10)
    err = float(np.abs(q_g - q_o).max())
    err64 = float(np.abs(q_g - q_64).max())
    _report(f"full-size draped cloth 256x256, {contacts.count()} contacts", err, err64, _residual_of(orc64, q_g))
    assert err <= TOL_STEP and err64 <= TOL_STEP
    assert np.abs(qd_g - qd_o).max() <= 2.0 * TOL_STEP / DT


def test_full_size_batched_worlds_step_matches_oracle():
    """The 512-world batch at its full size (1.89 M vertices, one ground plane per world): after 260
    GPU steps (the cloths, released 0.5 m up, are on the ground by then), one GPU step and one FP32
    oracle step from that state agree to TOL_STEP, ground contacts included."""
    import os

    model, q0 = scenes.batched_worlds(512, seed=0)
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).cuda())
    for _ in range(260):
        pipe.collide(s0, c)
        solver.step(s0, s1, None, c, DT)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    q = s0.particle_q.cpu().numpy()
    qd = s0.particle_qd.cpu().numpy()
    assert np.isfinite(q).all()
    _, q_g, _, contacts = _gpu_step(model, solver, q, qd, pipe, DT)
    assert contacts.count() > 10000, "the cloths should lie on their ground planes"
    orc = oracle.VBDOracle(model, "f32", threads=os.cpu_count() or 1)
    _, q_o, _ = _oracle_step(model, orc, q, qd, 5e-3, DT, 10)
    del orc
    orc64 = oracle.VBDOracle(model, "f64", threads=os.cpu_count() or 1)
    _, q_64, _ = _oracle_step(model, orc64, q, qd, 5e-3, DT, 10)
    err = float(np.abs(q_g - q_o).max())
    err64 = float(np.abs(q_g - q_64).max())
    _report(f"full-size batched worlds ({model.particle_count} vertices, {contacts.count()} contacts)", err, err64,
            _residual_of(orc64, q_g))
    assert err <= TOL_STEP and err64 <= TOL_STEP


def test_step_after_an_unfinished_staged_sequence_is_unaffected():
    """A staged forward + sweeps without finalize (what the launch autotuner runs) must not leave
    contact-table state behind: the next step equals a fresh solver's step bit for bit."""
    model, q0 = scenes.single_cloth(n=32, side=1.0, seed=12, pin_top_corners=False, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.903)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    outs = []
    for staged_first in (False, True):
        solver = SolverVBD(model, iterations=5)
        c = pipe.contacts()
        s0, s1 = model.state(), model.state()
        s0.particle_q.copy_(torch.from_numpy(q0).cuda())
        pipe.collide(s0, c)
        assert c.count() > 0
        if staged_first:
            solver.forward(s0, c, DT)
            solver.iterate(c, DT, 2)
        solver.step(s0, s1, None, c, DT)
        torch.cuda.synchronize()
        outs.append(s1.particle_q.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
