"""Batched worlds sharded over ranks (host logic, CPU): partition, extraction, and a
world_size-2 gloo run whose gathered result equals the unsharded run bit for bit (the CPU
oracle steps each shard here; the CUDA path is covered by the GPU sharding test)."""

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from newton_b200 import scenes
from newton_b200.sharding import extract_worlds, gather_particles, partition_worlds, world_vertex_counts

DT = 1.0 / 600.0
MARGIN = 5.0e-3


def _model():
    model, q0 = scenes.batched_worlds(num_worlds=7, seed=11, n_range=(6, 11), device="cpu")
    q0 = q0.copy()
    q0[:, 2] -= 0.497  # cloths start 3 mm above their ground planes: contacts from the first step
    return model, q0


def _run_oracle(model, q0, steps=3):
    orc = oracle.VBDOracle(model, "f32")
    q = np.asarray(q0, np.float32).copy()
    qd = np.zeros_like(q)
    for _ in range(steps):
        orc.set_contacts(*oracle.collide(model, q, MARGIN))
        _, q, qd = orc.step(q, qd, None, DT, 10)
    return q, qd


def test_partition_covers_every_world_once_and_balances():
    rng = np.random.default_rng(0)
    counts = rng.integers(16 * 16, 96 * 96, size=512)
    for n in (1, 2, 3, 8):
        parts = partition_worlds(counts, n)
        allw = np.sort(np.concatenate(parts))
        assert np.array_equal(allw, np.arange(512))
        loads = np.array([counts[p].sum() for p in parts])
        assert loads.max() - loads.min() <= counts.max()
        assert all(np.all(np.diff(p) > 0) for p in parts)


def test_extract_keeps_each_worlds_order_and_colors():
    model, _ = _model()
    counts = world_vertex_counts(model)
    assert counts.sum() == model.particle_count
    for ids in partition_worlds(counts, 3):
        sub, pidx = extract_worlds(model, ids)
        assert sub.particle_count == len(pidx) == counts[ids].sum()
        assert np.array_equal(sub.particle_q, model.particle_q[pidx])
        assert np.all(np.diff(pidx) > 0)
        # triangles map back to full-model triangles, in order
        full_tris = {tuple(t) for t in model.tri_indices.tolist()}
        assert all(tuple(t) in full_tris for t in pidx[sub.tri_indices].tolist())
        # every world meets its vertices in the same color sequence as in the full model
        full_color = model.particle_colors[pidx]
        assert np.array_equal(np.argsort(sub.particle_colors, kind="stable"),
                              np.argsort(full_color, kind="stable"))
        assert set(np.unique(sub.shape_world)) <= set(range(len(ids))) | {-1}


def test_extract_rejects_global_particles():
    model, _ = _model()
    model.particle_world = model.particle_world.copy()
    model.particle_world[0] = -1
    with pytest.raises(ValueError):
        extract_worlds(model, [0])


def _rank_main(rank, world_size, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        model, q0 = _model()
        ids = partition_worlds(world_vertex_counts(model), world_size)[rank]
        sub, pidx = extract_worlds(model, ids)
        q, qd = _run_oracle(sub, q0[pidx])
        q_full = gather_particles(q, pidx, model.particle_count)
        qd_full = gather_particles(qd, pidx, model.particle_count)
        if rank == 0:
            np.save(os.path.join(out_dir, "q.npy"), q_full)
            np.save(os.path.join(out_dir, "qd.npy"), qd_full)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_sharded_run_equals_unsharded(tmp_path):
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    model, q0 = _model()
    q_ref, qd_ref = _run_oracle(model, q0)
    assert np.array_equal(np.load(tmp_path / "q.npy"), q_ref)
    assert np.array_equal(np.load(tmp_path / "qd.npy"), qd_ref)
