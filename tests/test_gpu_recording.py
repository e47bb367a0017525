"""A recorded simulation reloads into a model that reproduces it: steps resumed from a recorded
frame with the recorded model are bit-identical to the original run."""

import pytest
import torch

from newton_b200 import CollisionPipeline, Model, scenes
from newton_b200.recording import RecorderFile
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0


def _run(model, state, steps, rec=None):
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    other = model.state()
    for _ in range(steps):
        pipe.collide(state, c)
        solver.step(state, other, None, c, DT)
        state, other = other, state
        if rec is not None:
            rec.log_state(state)
    torch.cuda.synchronize()
    return state


def test_resume_from_recording_is_bit_identical(tmp_path):
    model, q0 = scenes.single_cloth(n=24, side=1.0, seed=3, pin_top_corners=False, ground=0.0,
                                    sphere=((0.0, 0.0, 0.5), 0.4), height=0.95)
    rec = RecorderFile(str(tmp_path / "drape.json"), auto_save=False)
    rec.set_model(model)
    s = model.state()
    s.particle_q.copy_(torch.from_numpy(q0).cuda())
    ref = _run(model, s, 5, rec)
    rec.save_recording()

    back = RecorderFile(str(tmp_path / "drape.json"))
    back.load_recording()
    m2 = Model("cuda:0")
    back.load_model(m2)
    s2 = m2.state()
    back.load_state(s2, 1)  # state after step 2
    out = _run(m2, s2, 3)
    assert torch.equal(out.particle_q, ref.particle_q)
    assert torch.equal(out.particle_qd, ref.particle_qd)
