"""Sharded batched worlds on the GPU: every shard's CUDA step reproduces the full model's step
for its worlds bit for bit (ranks emulated one after another on one GPU; no collective is on
the data path, so nothing waits on another rank)."""

import numpy as np
import pytest
import torch

from newton_b200 import CollisionPipeline, scenes
from newton_b200.sharding import extract_worlds, partition_worlds, world_vertex_counts
from newton_b200.solvers import SolverVBD

pytestmark = pytest.mark.gpu

DT = 1.0 / 600.0


def _run(model, q0, steps):
    solver = SolverVBD(model, iterations=10)
    pipe = CollisionPipeline(model, soft_contact_margin=5e-3)
    c = pipe.contacts()
    a, b = model.state(), model.state()
    a.particle_q.copy_(torch.from_numpy(np.ascontiguousarray(q0)).cuda())
    for _ in range(steps):
        pipe.collide(a, c)
        solver.step(a, b, None, c, DT)
        a, b = b, a
    torch.cuda.synchronize()
    assert solver.status()["nonfinite_updates"] == 0
    return a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy()


@pytest.mark.parametrize("ranks", [2, 3])
def test_shards_reproduce_the_full_model(ranks):
    model, q0 = scenes.batched_worlds(num_worlds=24, seed=5, n_range=(8, 24))
    q0 = q0.copy()
    q0[:, 2] -= 0.497
    q_full, qd_full = _run(model, q0, 20)
    q_sh = np.zeros_like(q_full)
    qd_sh = np.zeros_like(qd_full)
    for ids in partition_worlds(world_vertex_counts(model), ranks):
        sub, pidx = extract_worlds(model, ids)
        q, qd = _run(sub, q0[pidx], 20)
        q_sh[pidx] = q
        qd_sh[pidx] = qd
    assert np.array_equal(q_sh, q_full)
    assert np.array_equal(qd_sh, qd_full)
