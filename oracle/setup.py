"""Model set-up restated for the checker -- TEST INFRASTRUCTURE ONLY.

``OracleModelBuilder`` is the package's ``ModelBuilder`` with its four connectivity / coloring
steps replaced by independent restatements, so that a scene can be built without loading the CUDA
library (the CPU-baseline leg of ``bench.py``) and so that the library's set-up tables can be
checked against a second implementation (``tests/test_oracle_setup.py``):

* bending-edge table (``utils/mesh.py:465-531``): ``oracle_edge_table``, a sort of the triangle
  slots by edge key (``vbd_oracle.cpp``);
* per-vertex element CSR (``utils/mesh.py:595-772``): a stable argsort of the element slots by
  vertex, so each vertex lists its (element, slot) records in element order;
* conflict-graph edges (``graph_coloring.py:99-197``): the unique sorted (min, max) pairs of every
  active triangle's 3 and every active hinge's 6 vertex pairs (numpy);
* coloring (``graph_coloring.py:243-311``; the library's MCS / greedy + balance):
  ``oracle_color_graph``, MCS with a priority queue (``vbd_oracle.cpp``).
"""

from __future__ import annotations

import ctypes

import numpy as np

from newton_b200.builder import ModelBuilder
from newton_b200.coloring import ColoringAlgorithm, convert_to_color_groups

from . import load

_i32p = ctypes.POINTER(ctypes.c_int32)


def _setup_lib():
    lib = load()
    if not getattr(lib, "_setup_ready", False):
        lib.oracle_edge_table.restype = ctypes.c_int
        lib.oracle_edge_table.argtypes = [_i32p, ctypes.c_int, _i32p]
        lib.oracle_color_graph.restype = ctypes.c_int
        lib.oracle_color_graph.argtypes = [ctypes.c_int, ctypes.c_int64, _i32p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_float, _i32p]
        lib._setup_ready = True
    return lib


def edge_table(tri_indices) -> np.ndarray:
    tris = np.ascontiguousarray(np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3))
    out = np.zeros((max(3 * len(tris), 1), 4), np.int32)
    ne = _setup_lib().oracle_edge_table(tris.ctypes.data_as(_i32p), len(tris), out.ctypes.data_as(_i32p))
    return out[:ne].copy()


def vertex_csr(elements: np.ndarray, slots, particle_count: int):
    """(values, offsets) of (element, slot) records per vertex, element order within a vertex;
    ``elements`` lists per element its vertex ids in the emission order ``slots``; -1 is skipped."""
    elements = np.asarray(elements, dtype=np.int64).reshape(len(elements), -1)
    vid = elements.reshape(-1)
    eid = np.repeat(np.arange(len(elements), dtype=np.int64), elements.shape[1])
    sid = np.tile(np.asarray(slots, dtype=np.int64), len(elements))
    keep = vid >= 0
    vid, eid, sid = vid[keep], eid[keep], sid[keep]
    order = np.argsort(vid, kind="stable")
    values = np.stack([eid[order], sid[order]], axis=1).reshape(-1).astype(np.int32)
    counts = np.bincount(vid, minlength=particle_count)
    offsets = np.zeros(particle_count + 1, np.int32)
    offsets[1:] = 2 * np.cumsum(counts)
    return values, offsets


class _Adjacency:
    """The attributes of ``MeshAdjacency`` the model and the solvers read."""

    def __init__(self, tri_indices, edge_indices, particle_count):
        self.indices = np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
        self.edge_indices = np.asarray(edge_indices, dtype=np.int32).reshape(-1, 4)
        self.v_adj_tris, self.v_adj_tris_offsets = vertex_csr(self.indices, (0, 1, 2), particle_count)
        self.v_adj_edges, self.v_adj_edges_offsets = vertex_csr(self.edge_indices[:, [2, 3, 0, 1]], (2, 3, 0, 1),
                                                                particle_count)
        self.vertex_adjacency_initialized = True


def conflict_edges(tri_indices, tri_mask, bend_indices, bend_mask) -> np.ndarray:
    pairs = []
    if tri_indices is not None:
        t = np.asarray(tri_indices, dtype=np.int64).reshape(-1, 3)
        if tri_mask is not None:
            t = t[np.broadcast_to(np.asarray(tri_mask).astype(bool), (len(t),))]
        pairs += [t[:, [0, 1]], t[:, [0, 2]], t[:, [1, 2]]]
    if bend_indices is not None:
        b = np.asarray(bend_indices, dtype=np.int64).reshape(-1, 4)
        if bend_mask is not None:
            b = b[np.broadcast_to(np.asarray(bend_mask).astype(bool), (len(b),))]
        for i in range(4):
            for j in range(i + 1, 4):
                pairs.append(b[:, [i, j]])
    if not pairs:
        return np.empty((0, 2), np.int32)
    p = np.concatenate(pairs)
    p = p[(p[:, 0] >= 0) & (p[:, 1] >= 0) & (p[:, 0] != p[:, 1])]
    if len(p) == 0:
        return np.empty((0, 2), np.int32)
    return np.unique(np.sort(p, axis=1), axis=0).astype(np.int32)


def color(num_nodes, edges, balance_colors, target_ratio, algorithm) -> list[np.ndarray]:
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1, 2))
    colors = np.zeros(num_nodes, np.int32)
    alg = algorithm.value if isinstance(algorithm, ColoringAlgorithm) else int(algorithm)
    nc = _setup_lib().oracle_color_graph(num_nodes, len(e), e.ctypes.data_as(_i32p), alg, 1 if balance_colors else 0,
                                         float(target_ratio), colors.ctypes.data_as(_i32p))
    return convert_to_color_groups(nc, colors)


class OracleModelBuilder(ModelBuilder):
    """``ModelBuilder`` whose connectivity and coloring come from the restatements above."""

    def _edge_table(self, tri_indices):
        return edge_table(tri_indices)

    def _vertex_adjacency(self, tri_indices, edge_indices, particle_count):
        return _Adjacency(tri_indices, edge_indices, particle_count)

    def _conflict_edges(self, tri_indices, tri_mask, bend_indices, bend_mask):
        return conflict_edges(tri_indices, tri_mask, bend_indices, bend_mask)

    def _color_graph(self, num_nodes, edges, balance_colors, target_ratio, algorithm):
        return color(num_nodes, edges, balance_colors, target_ratio, algorithm)
