"""GPU tests of the persistent shared-memory-resident step kernel.

The resident kernel runs every color of every iteration in one cooperative launch, with
neighbour-only synchronisation between patches.  It must give the same positions as the
per-color launches (4 lanes per vertex, the same arithmetic and summation order), stay within the
parity tolerance of the CPU oracle, and return (never hang) when its waits run out.
"""

import numpy as np
import pytest
import torch

import oracle
from newton_b200 import CollisionPipeline, scenes
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0


def _run(model, q0, resident, steps=3, iterations=10, margin=5e-3, spin_limit=None):
    dev = model.device
    solver = SolverVBD(model, iterations=iterations, lanes_per_vertex=4, block_size=128, resident_step=resident)
    if spin_limit is not None:
        solver.set_spin_limit(spin_limit)
    pipe = CollisionPipeline(model, soft_contact_margin=margin) if model.shape_count else None
    c = pipe.contacts() if pipe else None
    s0, s1 = model.state(), model.state()
    s0.particle_q.copy_(torch.from_numpy(q0).to(dev))
    for _ in range(steps):
        if pipe:
            pipe.collide(s0, c)
        solver.step(s0, s1, None, c, DT)
        s0, s1 = s1, s0
    torch.cuda.synchronize()
    return solver, s0.particle_q.cpu().numpy(), s0.particle_qd.cpu().numpy()


SCENES = {
    "hanging_32": lambda: scenes.hanging_cloth(seed=20),
    "draped_48_contacts": lambda: scenes.single_cloth(n=48, side=1.0, seed=21, pin_top_corners=False, ground=0.0,
                                                      sphere=((0.0, 0.0, 0.5), 0.4), height=0.905),
    "draped_256": lambda: scenes.draped_cloth(n=256, seed=22),
    "batched_8_worlds": lambda: scenes.batched_worlds(num_worlds=8, seed=23, n_range=(10, 30)),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_resident_matches_per_color_launches(name):
    model, q0 = SCENES[name]()
    solver_r, q_r, v_r = _run(model, q0, resident=True)
    info = solver_r.step_kernel_info()
    assert info["resident"], f"{name}: the resident kernel should be used ({info})"
    _, q_c, v_c = _run(model, q0, resident=False)
    err = float(np.abs(q_r - q_c).max())
    print(f"{name}: patches={info['patches']} smem={info['smem_bytes']} B, max |dx| resident vs per-color {err:.3e}")
    assert err <= 1e-6
    st = solver_r.status()
    assert st["timeouts"] == 0 and st["nonfinite_updates"] == 0


def test_resident_step_matches_oracle():
    model, q0 = scenes.single_cloth(n=64, side=1.0, seed=24, pin_top_corners=True, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.903)
    solver, q_r, _ = _run(model, q0, resident=True, steps=1)
    assert solver.step_kernel_info()["resident"]
    orc = oracle.VBDOracle(model, "f32", threads=8)
    orc.set_contacts(*oracle.collide(model, q0, 5e-3))
    _, q_o, _ = orc.step(q0, np.zeros_like(q0), None, DT, 10)
    assert np.abs(q_r - q_o).max() <= 1e-5


def test_resident_waits_are_bounded():
    """A one-poll wait limit makes neighbour waits run out: the kernel returns, counts timeouts, and
    the context stays usable for a normal step afterwards."""
    model, q0 = scenes.draped_cloth(n=128, seed=25)
    solver, q_bad, _ = _run(model, q0, resident=True, steps=1, spin_limit=1)
    assert solver.step_kernel_info()["patches"] > 1
    st = solver.status()
    assert st["timeouts"] > 0
    solver.set_spin_limit(1 << 22)
    _, q_ok, _ = _run(model, q0, resident=True, steps=1)
    _, q_ref, _ = _run(model, q0, resident=False, steps=1)
    assert np.abs(q_ok - q_ref).max() <= 1e-6
