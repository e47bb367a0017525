"""Soft-mesh connectivity: bending-edge table and per-vertex CSR adjacency.

Restates the connectivity that Newton's VBD cloth path consumes
(``newton/_src/utils/mesh.py``), computed by the library's host functions
(``vbd_mesh_edge_adjacency``, ``vbd_mesh_vertex_csr``) or, given a CUDA ``device``, by their
GPU counterparts (``*_device``), which produce the same tables:

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
"""

from __future__ import annotations

import warnings

import numpy as np

from . import _lib


def compute_edge_adjacency(tri_indices, device=None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Edge table ``[o0, o1, v0, v1]``, edge->triangle map and triangle->edge map.

    Mirrors ``MeshAdjacency._compute_edge_adjacency`` (``utils/mesh.py:465-531``).
    """
    if device is not None:
        edges, edge_tri, tri_edge, nonmanifold = _lib.mesh_edge_adjacency_device(tri_indices, device)
    else:
        edges, edge_tri, tri_edge, nonmanifold = _lib.mesh_edge_adjacency(tri_indices)
    if nonmanifold:
        warnings.warn("Detected non-manifold edge", stacklevel=2)
    return edges, edge_tri, tri_edge


def _csr(entries, slots, particle_count: int, device):
    if device is not None:
        return _lib.mesh_vertex_csr_device(entries, slots, particle_count, device)
    return _lib.mesh_vertex_csr(entries, slots, particle_count)


def vertex_adjacency_tris(tri_indices, particle_count: int, device=None):
    """Per-vertex triangle CSR (``utils/mesh.py:692-772`` fill order)."""
    tris = np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
    if tris.shape[0] == 0:
        return np.empty(0, np.int32), np.zeros(particle_count + 1, np.int32)
    return _csr(tris, (0, 1, 2), particle_count, device)


def vertex_adjacency_edges(edge_indices, particle_count: int, device=None):
    """Per-vertex bending-edge CSR (``utils/mesh.py:692-725`` fill order v0, v1, o0, o1)."""
    edges = np.asarray(edge_indices, dtype=np.int32).reshape(-1, 4)
    if edges.shape[0] == 0:
        return np.empty(0, np.int32), np.zeros(particle_count + 1, np.int32)
    # per element the entries are emitted in the order v0 (slot 2), v1 (slot 3), o0 (slot 0), o1 (slot 1)
    return _csr(np.ascontiguousarray(edges[:, [2, 3, 0, 1]]), (2, 3, 0, 1), particle_count, device)


class MeshAdjacency:
    """Connectivity tables of a soft triangle mesh (``utils/mesh.py:247``).

    ``edge_indices`` rows are ``[o0, o1, v0, v1]``; ``v_adj_tris``/``v_adj_edges`` are
    flat ``(element_id, local_slot)`` pairs with ``*_offsets`` of length
    ``particle_count + 1`` counting int32 values (two per record), as in the reference.
    """

    def __init__(self, tri_indices=None, edge_indices=None, device=None):
        self.device = device  # a CUDA device: the tables are computed there
        self.indices = None if tri_indices is None else np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
        if edge_indices is not None:
            self.edge_indices = np.asarray(edge_indices, dtype=np.int32).reshape(-1, 4)
            self.edge_tri_indices = None
            self.tri_edge_indices = None
        elif self.indices is not None:
            self.edge_indices, self.edge_tri_indices, self.tri_edge_indices = compute_edge_adjacency(self.indices,
                                                                                                    device)
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
        self.v_adj_tris, self.v_adj_tris_offsets = vertex_adjacency_tris(tris, particle_count, self.device)
        self.v_adj_edges, self.v_adj_edges_offsets = vertex_adjacency_edges(self.edge_indices, particle_count,
                                                                            self.device)
        self.vertex_adjacency_initialized = True
        return self
