"""Soft-mesh connectivity: bending-edge table and per-vertex CSR adjacency.

Restates the connectivity that Newton's VBD cloth path consumes
(``newton/_src/utils/mesh.py``):

* ``compute_edge_adjacency`` follows ``MeshAdjacency._compute_edge_adjacency``
  (``utils/mesh.py:465-531``): every triangle contributes three local edge slots
  ``(v0,v1|v2)``, ``(v1,v2|v0)``, ``(v2,v0|v1)``; undirected edges are numbered in
  first-occurrence order of that traversal; the first triangle to touch an edge
  fills ``[o0, -, v0, v1]`` and the second fills ``o1``.
* ``vertex_adjacency`` follows ``init_vertex_adjacency`` and the serial
  count/fill kernels (``utils/mesh.py:595-655``, ``:675-772``): per-vertex records
  are ``(element_id, local_slot)`` pairs in element-id order.  For a bending edge
  the fill order per element is endpoint ``v0`` (slot 2), endpoint ``v1`` (slot 3),
  opposite ``o0`` (slot 0), opposite ``o1`` (slot 1).  The order of these records
  fixes the floating-point summation order of the sweep, so it is kept exactly.

Everything here is vectorised numpy: the reference runs the count/fill passes as
single-threaded loops, which is the slow part of building large scenes.
"""

from __future__ import annotations

import warnings

import numpy as np


def compute_edge_adjacency(tri_indices) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Edge table ``[o0, o1, v0, v1]``, edge->triangle map and triangle->edge map.

    Mirrors ``MeshAdjacency._compute_edge_adjacency`` (``utils/mesh.py:465-531``).
    """
    tris = np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
    nt = tris.shape[0]
    if nt == 0:
        return (
            np.empty((0, 4), np.int32),
            np.empty((0, 2), np.int32),
            np.empty((0, 3), np.int32),
        )
    a = tris.reshape(-1)                                   # slot k starts at vertex k
    b = np.roll(tris, -1, axis=1).reshape(-1)              # ... ends at vertex k+1
    opp = np.roll(tris, -2, axis=1).reshape(-1)            # ... opposite is vertex k+2
    entry_tri = np.repeat(np.arange(nt, dtype=np.int64), 3)
    entry_slot = np.tile(np.arange(3, dtype=np.int64), nt)

    lo = np.minimum(a, b).astype(np.int64)
    hi = np.maximum(a, b).astype(np.int64)
    key = lo * (int(hi.max()) + 1) + hi
    # stable sort groups equal keys while keeping traversal order inside each group
    order = np.argsort(key, kind="stable")
    skey = key[order]
    is_first = np.ones(len(skey), dtype=bool)
    is_first[1:] = skey[1:] != skey[:-1]
    group_id_sorted = np.cumsum(is_first) - 1
    group_first_entry = order[is_first]                    # first entry of each group
    # number groups by the position of their first entry (first-occurrence order)
    rank = np.empty(len(group_first_entry), dtype=np.int64)
    rank[np.argsort(group_first_entry, kind="stable")] = np.arange(len(group_first_entry))
    entry_edge = np.empty(len(key), dtype=np.int64)
    entry_edge[order] = rank[group_id_sorted]
    # position of each entry inside its group (0 = first side, 1 = second side, ...)
    group_start = np.flatnonzero(is_first)
    pos_in_group_sorted = np.arange(len(skey)) - np.repeat(group_start, np.diff(np.append(group_start, len(skey))))
    side = np.empty(len(key), dtype=np.int64)
    side[order] = pos_in_group_sorted

    ne = len(group_first_entry)
    edge_indices = np.full((ne, 4), -1, dtype=np.int32)
    edge_tri = np.full((ne, 2), -1, dtype=np.int32)
    tri_edge = np.full((nt, 3), -1, dtype=np.int32)
    tri_edge[entry_tri, entry_slot] = entry_edge

    s0 = side == 0
    edge_indices[entry_edge[s0], 0] = opp[s0]
    edge_indices[entry_edge[s0], 2] = a[s0]
    edge_indices[entry_edge[s0], 3] = b[s0]
    edge_tri[entry_edge[s0], 0] = entry_tri[s0]
    s1 = side == 1
    edge_indices[entry_edge[s1], 1] = opp[s1]
    edge_tri[entry_edge[s1], 1] = entry_tri[s1]
    if np.any(side > 1):
        warnings.warn("Detected non-manifold edge", stacklevel=2)
    return edge_indices, edge_tri, tri_edge


def _csr(vertex_ids: np.ndarray, element_ids: np.ndarray, slots: np.ndarray, particle_count: int):
    """Build an ``(element, slot)`` CSR ordered by (vertex, entry order given)."""
    counts = np.bincount(vertex_ids, minlength=particle_count).astype(np.int64)
    offsets = np.zeros(particle_count + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(2 * counts)
    order = np.argsort(vertex_ids, kind="stable")
    values = np.empty(2 * len(vertex_ids), dtype=np.int32)
    values[0::2] = element_ids[order]
    values[1::2] = slots[order]
    return values, offsets.astype(np.int32)


def vertex_adjacency_tris(tri_indices, particle_count: int):
    """Per-vertex triangle CSR (``utils/mesh.py:692-772`` fill order)."""
    tris = np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
    nt = tris.shape[0]
    if nt == 0:
        return np.empty(0, np.int32), np.zeros(particle_count + 1, np.int32)
    vid = tris.reshape(-1).astype(np.int64)
    eid = np.repeat(np.arange(nt, dtype=np.int32), 3)
    slot = np.tile(np.arange(3, dtype=np.int32), nt)
    return _csr(vid, eid, slot, particle_count)


def vertex_adjacency_edges(edge_indices, particle_count: int):
    """Per-vertex bending-edge CSR (``utils/mesh.py:692-725`` fill order v0, v1, o0, o1)."""
    edges = np.asarray(edge_indices, dtype=np.int32).reshape(-1, 4)
    ne = edges.shape[0]
    if ne == 0:
        return np.empty(0, np.int32), np.zeros(particle_count + 1, np.int32)
    # per element the entries are emitted in the order v0(slot 2), v1(slot 3), o0(slot 0), o1(slot 1)
    vid = np.stack([edges[:, 2], edges[:, 3], edges[:, 0], edges[:, 1]], axis=1).reshape(-1)
    slot = np.tile(np.array([2, 3, 0, 1], dtype=np.int32), ne)
    eid = np.repeat(np.arange(ne, dtype=np.int32), 4)
    keep = vid != -1
    return _csr(vid[keep].astype(np.int64), eid[keep], slot[keep], particle_count)


class MeshAdjacency:
    """Connectivity tables of a soft triangle mesh (``utils/mesh.py:247``).

    ``edge_indices`` rows are ``[o0, o1, v0, v1]``; ``v_adj_tris``/``v_adj_edges`` are
    flat ``(element_id, local_slot)`` pairs with ``*_offsets`` of length
    ``particle_count + 1`` counting int32 values (two per record), as in the reference.
    """

    def __init__(self, tri_indices=None, edge_indices=None):
        self.indices = None if tri_indices is None else np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
        if edge_indices is not None:
            self.edge_indices = np.asarray(edge_indices, dtype=np.int32).reshape(-1, 4)
            self.edge_tri_indices = None
            self.tri_edge_indices = None
        elif self.indices is not None:
            self.edge_indices, self.edge_tri_indices, self.tri_edge_indices = compute_edge_adjacency(self.indices)
        else:
            self.edge_indices = np.empty((0, 4), np.int32)
            self.edge_tri_indices = np.empty((0, 2), np.int32)
            self.tri_edge_indices = np.empty((0, 3), np.int32)
        self.v_adj_tris = None
        self.v_adj_tris_offsets = None
        self.v_adj_edges = None
        self.v_adj_edges_offsets = None
        self.vertex_adjacency_initialized = False

    def init_vertex_adjacency(self, particle_count: int) -> "MeshAdjacency":
        if self.vertex_adjacency_initialized:
            return self
        tris = self.indices if self.indices is not None else np.empty((0, 3), np.int32)
        self.v_adj_tris, self.v_adj_tris_offsets = vertex_adjacency_tris(tris, particle_count)
        self.v_adj_edges, self.v_adj_edges_offsets = vertex_adjacency_edges(self.edge_indices, particle_count)
        self.vertex_adjacency_initialized = True
        return self
