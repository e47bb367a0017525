"""GPU tests of the residual-gated step (``SolverVBD.set_residual_gate`` / ``vbd_set_residual_gate``).

The reference runs a fixed number of Gauss-Seidel iterations per step (``solver_vbd.py:1817-1819``);
the gate replaces that loop by "iterate until max_i |f_i| / (m_i |g|) <= tolerance", evaluated on
the device inside the step's CUDA graph (a conditional while node).  Checked here:

* a gated step equals the fixed-count step with the iteration count the gate chose, bit for bit,
  and that count is the first at which the Jacobi residual meets the tolerance;
* the oracle's restatement of the gate (same residual definition, same loop) chooses the same
  count and lands within the step tolerance;
* the cap, relative tolerances, checks every k iterations, the gate inside a caller's own CUDA
  graph capture, and a zero warm-start network under the gate.
"""

import numpy as np
import pytest
import torch

import oracle
from newton_b200 import CollisionPipeline, scenes
from newton_b200 import learned as L
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0
TOL_STEP = 1.0e-5  # m, per step from identical states


def _hanging_state(steps=60, seed=1):
    """A hanging cloth advanced by the FP32 oracle (deformed, non-trivial residual)."""
    model, q0 = scenes.hanging_cloth(seed=seed)
    orc = oracle.VBDOracle(model, "f32", threads=8)
    q, qd = q0.astype(np.float32), np.zeros_like(q0, dtype=np.float32)
    for _ in range(steps):
        orc.set_contacts(*oracle.collide(model, q, 5e-3))
        _, q, qd = orc.step(q, qd, None, DT, 10)
    return model, q, qd


def _run(model, solver, q, qd, iterations=None, pipe=None):
    pipe = pipe or CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(q).cuda())
    a.particle_qd.copy_(torch.from_numpy(qd).cuda())
    pipe.collide(a, c)
    solver.step(a, b, None, c, DT)
    torch.cuda.synchronize()
    return b.particle_q.cpu().numpy(), b.particle_qd.cpu().numpy(), a.particle_q.cpu().numpy()


def _gate_mean(pv, solvable):
    """The gate's mean norm from per-vertex residuals: fixed-point sum (1/256, clamped at 1e9) / count."""
    r = np.minimum(pv[solvable].astype(np.float32), np.float32(1e9))
    fixed = np.floor(r * np.float32(256.0) + np.float32(0.5)).astype(np.uint64)
    return float(np.float32(float(fixed.sum()) / 256.0 / len(r)))


def _jacobi_residuals(model, q, qd, kmax, norm="max"):
    """Residual norm after 0..kmax plain iterations (staged API, same kernels as the step)."""
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    a = model.state()
    a.particle_q.copy_(torch.from_numpy(q).cuda())
    a.particle_qd.copy_(torch.from_numpy(qd).cuda())
    pipe.collide(a, c)
    solver.forward(a, c, DT)
    solvable = ((model.particle_flags & 1) != 0) & (model.particle_mass != 0)

    def value():
        mx, pv = solver.residual(c, DT, per_vertex=True)
        return float(mx.item()) if norm == "max" else _gate_mean(pv.cpu().numpy(), solvable)

    out = [value()]
    for _ in range(kmax):
        solver.iterate(c, DT, 1)
        out.append(value())
    return out


def _clear_drop(curve, start=3, gap=0.97):
    """First k >= start whose residual is clearly below every earlier one, and a tolerance in that gap."""
    for k in range(start, len(curve)):
        prior = min(curve[:k])
        if curve[k] < gap * prior:
            return k, float(np.float32(0.5 * (curve[k] + prior)))
    raise AssertionError(f"no clear drop in {curve}")


def _first_at_or_below(curve, thresh, step=1):
    return min(i for i in range(0, len(curve), step) if curve[i] <= thresh)


def _oracle_gated(model, q, qd, tol, cap, norm="max"):
    """The gate restated on the oracle: forward, then iterate while the residual norm > tol."""
    orc = oracle.VBDOracle(model, "f32", threads=8)
    orc.set_contacts(*oracle.collide(model, q, 5e-3))
    orc.forward(q, qd, None, DT)
    solvable = ((model.particle_flags & 1) != 0) & (model.particle_mass != 0)

    def value():
        pv = orc.residual(DT)
        return float(pv.max()) if norm == "max" else _gate_mean(pv, solvable)

    k = 0
    r = value()
    while r > tol and k < cap:
        orc.begin_iteration()
        for color in range(len(model.particle_color_groups)):
            orc.sweep_color(color, DT)
        k += 1
        r = value()
    _, q_out, qd_out = orc.finalize(DT)
    return k, r, q_out, qd_out


@pytest.mark.parametrize("norm", ["max", "mean"])
def test_gate_stops_at_the_first_iterate_that_meets_the_tolerance(norm):
    model, q, qd = _hanging_state()
    curve = _jacobi_residuals(model, q, qd, 40, norm=norm)
    # a tolerance in a clear gap of the (not always monotone) residual curve, so that the
    # oracle's slightly different FP32 rounding decides the same way
    kd, tol = _clear_drop(curve, start=2 if norm == "max" else 6, gap=0.99 if norm == "max" else 0.9995)
    solver = SolverVBD(model, iterations=10)
    solver.set_residual_gate(tol, max_iterations=40, norm=norm)
    qg, qdg, qing = _run(model, solver, q, qd)
    st = solver.gate_stats()
    k = st["last_iterations"]
    assert st["steps"] == 1 and st["capped_steps"] == 0
    assert k == kd == _first_at_or_below(curve, tol), (k, kd, curve[:16], tol)
    assert st["last_residual"] == curve[k] and st["last_start_residual"] == curve[0]
    print(f"gated step ({norm} norm): {k} iterations to residual {st['last_residual']:.5g} m|g| "
          f"(start {st['last_start_residual']:.5g}, tolerance {tol:.5g})")
    # the same as the fixed-count step with that many iterations, bit for bit
    qf, qdf, qinf = _run(model, SolverVBD(model, iterations=k), q, qd)
    assert np.array_equal(qg, qf) and np.array_equal(qdg, qdf) and np.array_equal(qing, qinf)
    # the oracle's gate picks the same count, and the step agrees within the step tolerance
    ko, ro, qo, qdo = _oracle_gated(model, q, qd, tol, 40, norm=norm)
    assert ko == k, (ko, k)
    err = float(np.abs(qg - qo).max())
    assert err <= TOL_STEP, err
    print(f"oracle gate: {ko} iterations, residual {ro:.5g}; max |dx| GPU vs oracle {err:.3e} m")


def test_gate_cap_and_turning_it_off():
    model, q, qd = _hanging_state(steps=30, seed=2)
    solver = SolverVBD(model, iterations=10)
    solver.set_residual_gate(1.0e-3, max_iterations=7)  # far below what 7 iterations reach
    qg, qdg, _ = _run(model, solver, q, qd)
    st = solver.gate_stats()
    assert st["last_iterations"] == 7 and st["capped_steps"] == 1 and st["last_residual"] > 1.0e-3
    qf, qdf, _ = _run(model, SolverVBD(model, iterations=7), q, qd)
    assert np.array_equal(qg, qf) and np.array_equal(qdg, qdf)
    # off again: the fixed iteration count applies
    solver.set_residual_gate(None)
    q10, _, _ = _run(model, solver, q, qd)
    qf10, _, _ = _run(model, SolverVBD(model, iterations=10), q, qd)
    assert np.array_equal(q10, qf10)
    # iteration cap 0: the step is the forward prediction
    solver.set_residual_gate(1.0e-3, max_iterations=0)
    q0g, _, _ = _run(model, solver, q, qd)
    q0f, _, _ = _run(model, SolverVBD(model, iterations=0), q, qd)
    assert np.array_equal(q0g, q0f)


def test_gate_relative_tolerance_and_check_interval():
    model, q, qd = _hanging_state(steps=45, seed=3)
    for norm in ("max", "mean"):
        curve = _jacobi_residuals(model, q, qd, 60, norm=norm)
        rho = 0.9 if norm == "max" else 0.97
        thresh = float(np.float32(rho) * np.float32(curve[0]))
        solver = SolverVBD(model, iterations=10)
        solver.set_residual_gate(rho, max_iterations=60, relative=True, norm=norm)
        qg, _, _ = _run(model, solver, q, qd)
        st = solver.gate_stats(reset=True)
        k = st["last_iterations"]
        assert st["last_reference_residual"] == pytest.approx(curve[0], rel=1e-6)
        assert k == _first_at_or_below(curve, thresh), (norm, k, curve[:12])
        assert st["capped_steps"] == 0
        qf, _, _ = _run(model, SolverVBD(model, iterations=k), q, qd)
        assert np.array_equal(qg, qf)
        # checks every 4 iterations: the first multiple of 4 at which the tolerance holds
        solver.set_residual_gate(rho, max_iterations=60, check_every=4, relative=True, norm=norm)
        qg4, _, _ = _run(model, solver, q, qd)
        k4 = solver.gate_stats()["last_iterations"]
        assert k4 % 4 == 0 and k4 == _first_at_or_below(curve, thresh, step=4)
        qf4, _, _ = _run(model, SolverVBD(model, iterations=k4), q, qd)
        assert np.array_equal(qg4, qf4)
        print(f"{norm} norm: relative {rho}: {k} iterations (every 4: {k4}); curve {curve[:k + 1]}")


def test_gate_inside_a_callers_graph_capture():
    """A gated step recorded into the caller's own CUDA graph (as Warp's ScopedCapture does in the
    reference's tests) adds its device-side loop to that graph; replays match the cached-graph path."""
    model, q, qd = _hanging_state(steps=30, seed=4)
    curve = _jacobi_residuals(model, q, qd, 30)
    kd, tol = _clear_drop(curve, start=2, gap=0.99)
    ref_solver = SolverVBD(model, iterations=10)
    ref_solver.set_residual_gate(tol, max_iterations=30)
    q_ref, qd_ref, _ = _run(model, ref_solver, q, qd)
    assert ref_solver.gate_stats()["last_iterations"] == kd

    solver = SolverVBD(model, iterations=10)
    solver.set_residual_gate(tol, max_iterations=30)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            pipe.collide(a, c)
            solver.step(a, b, None, c, DT)
    for _ in range(2):
        a.particle_q.copy_(torch.from_numpy(q).cuda())
        a.particle_qd.copy_(torch.from_numpy(qd).cuda())
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(b.particle_q.cpu().numpy(), q_ref)
        assert np.array_equal(b.particle_qd.cpu().numpy(), qd_ref)
    st = solver.gate_stats()
    assert st["steps"] == 2 and st["last_iterations"] == kd


def test_zero_network_warm_start_under_the_gate_is_plain_gated_vbd():
    model, q, qd = _hanging_state(steps=30, seed=5)
    plain = SolverVBD(model, iterations=10)
    plain.set_residual_gate(0.8, max_iterations=50, relative=True, norm="mean")
    qp, qdp, _ = _run(model, plain, q, qd)
    learned = SolverVBD(model, iterations=10)
    mlp = L.WarmStartMLP("cuda:0", seed=6)
    mlp.params.zero_()
    mlp.pack()
    learned.set_warm_start(mlp, 10)
    learned.set_residual_gate(0.8, max_iterations=50, relative=True, norm="mean")
    ql, qdl, _ = _run(model, learned, q, qd)
    sp, sl = plain.gate_stats(), learned.gate_stats()
    assert sp["last_iterations"] == sl["last_iterations"]
    assert sp["last_reference_residual"] == sl["last_reference_residual"]
    assert np.array_equal(qp, ql) and np.array_equal(qdp, qdl)


def test_gate_rejects_self_contact_and_bad_arguments():
    from newton_b200._lib import VbdError

    model, q0 = scenes.single_cloth(n=12, side=0.5, seed=1, pin_top_corners=False, ground=None, z_noise=0.0)
    solver = SolverVBD(model, iterations=4, particle_enable_self_contact=True, particle_self_contact_radius=0.002,
                       particle_self_contact_margin=0.003)
    with pytest.raises(VbdError, match="self-contact"):
        solver.set_residual_gate(1.0, max_iterations=10)
    plain = SolverVBD(model, iterations=4)
    with pytest.raises(VbdError, match="check_every"):
        plain.set_residual_gate(1.0, max_iterations=10, check_every=0)


@pytest.mark.parametrize("norm", ["mean", "max"])
def test_sweep_residual_gate(norm):
    """residual="sweep": the check after iteration k reads the Gauss-Seidel residual R_k the
    sweeps of iteration k accumulated (each vertex's force when its color was solved); the step
    stops at the first k with R_k <= tolerance and equals the fixed-count step with k iterations."""
    model, q, qd = _hanging_state()
    solver = SolverVBD(model, iterations=10)
    curve = [float("inf")]  # R_k for k = 1..16, each from a step capped at k
    for k in range(1, 17):
        solver.set_residual_gate(1e-30, max_iterations=k, norm=norm, residual="sweep")
        _run(model, solver, q, qd)
        st = solver.gate_stats(reset=True)
        assert st["last_iterations"] == k and st["capped_steps"] == 1
        curve.append(st["last_residual"])
    # one pass of the loop body is 4 check rounds: the colors' sweeps and a one-warp check kernel
    assert all(np.isfinite(curve[1:])) and st["body_kernels"] == 4 * (len(model.particle_color_groups) + 1)
    kd, tol = _clear_drop(curve, start=3, gap=0.99 if norm == "max" else 0.9995)
    solver.set_residual_gate(tol, max_iterations=40, norm=norm, residual="sweep")
    qg, qdg, _ = _run(model, solver, q, qd)
    st = solver.gate_stats()
    assert st["last_iterations"] == kd and st["last_residual"] == curve[kd] and st["capped_steps"] == 0
    qf, qdf, _ = _run(model, SolverVBD(model, iterations=kd), q, qd)
    assert np.array_equal(qg, qf) and np.array_equal(qdg, qdf)
    # the oracle's restatement of the sweep gate picks the same count
    orc = oracle.VBDOracle(model, "f32", threads=8)
    orc.set_contacts(*oracle.collide(model, q, 5e-3))
    _, qo, _, ko, ro = orc.gated_step(q, qd, None, DT, tol, 40, norm=norm)
    assert ko == kd, (ko, kd)
    assert float(np.abs(qg - qo).max()) <= TOL_STEP
    # every 2 iterations: the first even k whose R_k meets the tolerance
    solver.set_residual_gate(tol, max_iterations=40, check_every=2, norm=norm, residual="sweep")
    _run(model, solver, q, qd)
    k2 = solver.gate_stats()["last_iterations"]
    assert k2 == min(k for k in range(2, 17, 2) if curve[k] <= tol)
    print(f"sweep residual ({norm}): R_1..R_6 {[round(x, 3) for x in curve[1:7]]}, tolerance {tol:.5g} -> "
          f"{kd} iterations (every 2: {k2})")


def test_sweep_gate_rounds_per_body_do_not_change_the_step():
    """The rounds per pass of the device-side loop body only change how the loop is launched: the
    same stop, the same bits, ceil(iterations / rounds) passes, and the sweeps after the decision
    change nothing."""
    model, q, qd = _hanging_state(steps=45, seed=3)
    colors = len(model.particle_color_groups)
    qf, qdf, _ = _run(model, SolverVBD(model, iterations=5), q, qd)
    for tol, cap in ((1e-30, 5), (0.9, 40)):  # stopped by the cap mid-body; by the tolerance
        out = {}
        for rounds in (1, 3, 4, 7):
            solver = SolverVBD(model, iterations=10)
            solver.set_residual_gate(tol, max_iterations=cap, relative=True, norm="mean", residual="sweep",
                                     rounds_per_body=rounds)
            qg, qdg, _ = _run(model, solver, q, qd)
            st = solver.gate_stats()
            k = st["last_iterations"]
            assert st["steps"] == 1 and st["body_kernels"] == rounds * (colors + 1)
            assert st["body_passes"] == -(-k // rounds)
            out[rounds] = (k, qg, qdg, st["last_residual"])
        k1, q1, qd1, r1 = out[1]
        for rounds, (k, qg, qdg, r) in out.items():
            assert k == k1 and r == r1 and np.array_equal(qg, q1) and np.array_equal(qdg, qd1), rounds
        if cap == 5:
            assert k1 == 5 and np.array_equal(q1, qf) and np.array_equal(qd1, qdf)
    with pytest.raises(ValueError):
        SolverVBD(model, iterations=10).set_residual_gate(0.9, residual="sweep", rounds_per_body=16)


def test_relative_sweep_gate_refers_to_the_jacobi_residual_at_y():
    """Relative sweep mode (the benchmark's gate): the reference is the mean Jacobi residual at the
    inertia target y, the stop is the first k whose mean sweep residual R_k <= rho x reference."""
    model, q, qd = _hanging_state(steps=45, seed=3)
    jac = _jacobi_residuals(model, q, qd, 0, norm="mean")
    solver = SolverVBD(model, iterations=10)
    curve = [float("inf")]
    for k in range(1, 13):
        solver.set_residual_gate(1e-30, max_iterations=k, relative=True, norm="mean", residual="sweep")
        _run(model, solver, q, qd)
        st = solver.gate_stats(reset=True)
        assert st["last_reference_residual"] == jac[0]
        curve.append(st["last_residual"])
    kd, _ = _clear_drop(curve, start=3, gap=0.9995)
    rho = float(np.float32(0.5 * (curve[kd] + min(curve[:kd])) / jac[0]))
    thresh = float(np.float32(rho) * np.float32(jac[0]))
    expect = _first_at_or_below(curve, thresh)
    solver.set_residual_gate(rho, max_iterations=40, relative=True, norm="mean", residual="sweep")
    qg, _, _ = _run(model, solver, q, qd)
    assert solver.gate_stats()["last_iterations"] == expect
    qf, _, _ = _run(model, SolverVBD(model, iterations=expect), q, qd)
    assert np.array_equal(qg, qf)
    orc = oracle.VBDOracle(model, "f32", threads=8)
    orc.set_contacts(*oracle.collide(model, q, 5e-3))
    _, qo, _, ko, _ = orc.gated_step(q, qd, None, DT, rho, 40, norm="mean", relative=True)
    assert ko == expect and float(np.abs(qg - qo).max()) <= TOL_STEP
