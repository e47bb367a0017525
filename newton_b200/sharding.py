"""Batched cloth worlds sharded across ranks (one process per GPU).

Worlds never interact: a particle only meets triangles, hinges and shapes of its own world (or
global shapes, world -1), and the step has no global reduction.  So a rank steps the worlds it
owns with no collective on the data path; results are gathered only when a caller asks for them.

* ``partition_worlds`` assigns worlds to ranks by vertex count, largest first, each to the rank
  with the smallest load so far (ties: the lowest world id, then the lowest rank).
* ``extract_worlds`` cuts a shard out of the full model and keeps the relative order of
  particles, triangles, hinges, shapes and of every color group.  Each world therefore sees the
  same color sequence and the same per-vertex element order as in the full model, and a shard's
  step reproduces the full model's step for its worlds bit for bit.
* ``gather_particles`` collects the shards' per-particle arrays on rank 0 in full-model order
  (``torch.distributed``, any backend that supports object gathers).

The reference batches worlds inside one model (``ModelBuilder.add_builder``/``add_world``,
``builder.py:2925-2937``; coloring merge ``graph_coloring.py:382-410``); sharding them over
GPUs is this library's own layer above that.
"""

from __future__ import annotations

import numpy as np

from .mesh import MeshAdjacency
from .model import Model


def world_vertex_counts(model) -> np.ndarray:
    """Particles per world (worlds 0 .. world_count-1)."""
    w = np.asarray(model.particle_world, dtype=np.int64)
    return np.bincount(w[w >= 0], minlength=int(model.world_count)).astype(np.int64)


def partition_worlds(counts, n_ranks: int) -> list[np.ndarray]:
    """World ids per rank (ascending), balancing the summed vertex counts greedily."""
    counts = np.asarray(counts, dtype=np.int64)
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = np.lexsort((np.arange(len(counts)), -counts))
    loads = np.zeros(n_ranks, dtype=np.int64)
    owned: list[list[int]] = [[] for _ in range(n_ranks)]
    for w in order:
        r = int(np.argmin(loads))
        owned[r].append(int(w))
        loads[r] += counts[w]
    return [np.asarray(sorted(o), dtype=np.int64) for o in owned]


def extract_worlds(model, world_ids, device=None) -> tuple[Model, np.ndarray]:
    """Sub-model holding only ``world_ids`` (renumbered 0..k-1 in ascending order of their ids).

    Returns (shard, particle_index): ``particle_index[i]`` is the full-model index of the shard's
    particle i.  Global particles (world -1) cannot be split between shards and are rejected."""
    pw = np.asarray(model.particle_world, dtype=np.int64)
    if np.any(pw < 0):
        raise ValueError("extract_worlds: the model has global (world -1) particles")
    world_ids = np.unique(np.asarray(world_ids, dtype=np.int64))
    if world_ids.size and (world_ids[0] < 0 or world_ids[-1] >= model.world_count):
        raise ValueError("extract_worlds: world id out of range")
    world_new = np.full(int(model.world_count), -1, dtype=np.int64)
    world_new[world_ids] = np.arange(world_ids.size)
    keep = world_new[pw] >= 0
    pidx = np.flatnonzero(keep)
    remap = np.full(model.particle_count, -1, dtype=np.int64)
    remap[pidx] = np.arange(pidx.size)

    m = Model(model.device if device is None else device)
    m.requires_grad = model.requires_grad
    m.world_count = max(int(world_ids.size), 1)
    m.particle_count = int(pidx.size)
    for name in ("particle_q", "particle_qd", "particle_mass", "particle_inv_mass", "particle_radius",
                 "particle_flags"):
        setattr(m, name, np.ascontiguousarray(getattr(model, name)[pidx]))
    m.particle_world = world_new[pw[pidx]].astype(np.int32)

    tri = np.asarray(model.tri_indices, dtype=np.int64).reshape(-1, 3)
    tkeep = keep[tri].all(axis=1) if tri.size else np.zeros(0, dtype=bool)
    if tri.size and np.any(keep[tri].any(axis=1) & ~tkeep):
        raise ValueError("extract_worlds: a triangle spans worlds")
    m.tri_count = int(tkeep.sum())
    m.tri_indices = remap[tri[tkeep]].astype(np.int32).reshape(-1, 3)
    m.tri_poses = np.ascontiguousarray(model.tri_poses[tkeep])
    m.tri_materials = np.ascontiguousarray(model.tri_materials[tkeep])
    m.tri_areas = np.ascontiguousarray(model.tri_areas[tkeep])

    e = np.asarray(model.edge_indices, dtype=np.int64).reshape(-1, 4)
    ekeep = keep[e[:, 2]] if e.size else np.zeros(0, dtype=bool)
    es = e[ekeep].copy()
    es[es >= 0] = remap[es[es >= 0]]
    m.edge_count = int(ekeep.sum())
    m.edge_indices = es.astype(np.int32).reshape(-1, 4)
    m.edge_rest_angle = np.ascontiguousarray(model.edge_rest_angle[ekeep])
    m.edge_rest_length = np.ascontiguousarray(model.edge_rest_length[ekeep])
    m.edge_bending_properties = np.ascontiguousarray(model.edge_bending_properties[ekeep])

    groups = []
    for g in model.particle_color_groups:
        g = np.asarray(g, dtype=np.int64)
        g = remap[g[keep[g]]]
        if g.size:
            groups.append(g.astype(np.int32))
    m.particle_color_groups = groups
    colors = np.full(m.particle_count, -1, dtype=np.int32)
    for c, g in enumerate(groups):
        colors[g] = c
    m.particle_colors = colors

    adj = MeshAdjacency(m.tri_indices, m.edge_indices)
    adj.init_vertex_adjacency(m.particle_count)
    m.soft_mesh_adjacency = adj

    sw = np.asarray(model.shape_world, dtype=np.int64)
    skeep = (sw < 0) | (world_new[np.clip(sw, 0, None)] >= 0) if sw.size else np.zeros(0, dtype=bool)
    m.shape_count = int(skeep.sum())
    for name in ("shape_type", "shape_transform", "shape_scale", "shape_margin", "shape_material_ke",
                 "shape_material_kd", "shape_material_mu", "shape_flags", "shape_body"):
        setattr(m, name, np.ascontiguousarray(np.asarray(getattr(model, name))[skeep]))
    m.shape_world = np.where(sw[skeep] < 0, -1, world_new[np.clip(sw[skeep], 0, None)]).astype(np.int32)

    grav = np.asarray(model.gravity, dtype=np.float32).reshape(-1, 3)
    m.gravity = np.ascontiguousarray(grav[world_ids] if world_ids.size else grav[:1])
    m.soft_contact_ke = model.soft_contact_ke
    m.soft_contact_kd = model.soft_contact_kd
    m.soft_contact_mu = model.soft_contact_mu
    return m, pidx


def gather_particles(values: np.ndarray, particle_index: np.ndarray, particle_count: int, group=None):
    """Rank 0 receives the full-model array assembled from every rank's shard rows (others: None)."""
    import torch.distributed as dist

    values = np.asarray(values)
    payload = (np.asarray(particle_index, dtype=np.int64), values)
    rank = dist.get_rank(group)
    out = [None] * dist.get_world_size(group) if rank == 0 else None
    dist.gather_object(payload, out, dst=0, group=group)
    if rank != 0:
        return None
    full = np.zeros((particle_count,) + values.shape[1:], dtype=values.dtype)
    seen = np.zeros(particle_count, dtype=bool)
    for idx, v in out:
        if np.any(seen[idx]):
            raise RuntimeError("gather_particles: a particle is owned by two ranks")
        seen[idx] = True
        full[idx] = v
    if not seen.all():
        raise RuntimeError("gather_particles: some particles are owned by no rank")
    return full
