"""Particle conflict graph and color groups for the Gauss-Seidel sweep.

* ``construct_trimesh_graph_edges`` restates ``graph_coloring.py:99-197``: every active triangle
  contributes its three sides; with bending, every active hinge contributes all six pairs of its
  four vertices (negative ids skipped); pairs are canonicalised (sorted, unique).
* ``color_graph`` restates ``graph_coloring.py:243-311`` on top of the library's host coloring
  (``vbd_color_graph``: MCS or degree-ordered greedy, then balancing).
* ``combine_independent_coloring_plan`` restates ``graph_coloring.py:382-410``: the colorings of
  independent worlds are merged by pairing the smallest groups of one with the largest of the
  other.
"""

from __future__ import annotations

from enum import Enum

import numpy as np

from . import _lib


class ColoringAlgorithm(Enum):
    MCS = 0
    GREEDY = 1


def _canonicalize_edges(edges: np.ndarray) -> np.ndarray:
    """Unique (min, max) pairs without self-pairs, lexicographic (native counting sort)."""
    if edges.size == 0:
        return np.empty((0, 2), dtype=np.int32)
    return _lib.canonical_edges(int(edges.max()) + 1, edges)


def construct_trimesh_graph_edges(tri_indices, tri_active_mask=None, bending_edge_indices=None,
                                  bending_edge_active_mask=None, device=None) -> np.ndarray:
    """The canonical conflict-graph edges; ``device`` (a CUDA device) computes the same edges on
    the GPU (``vbd_trimesh_graph_edges_device``), None on the host."""
    tris = np.empty((0, 3), np.int32)
    bend = np.empty((0, 4), np.int32)
    if tri_indices is not None:
        tris = np.asarray(tri_indices, dtype=np.int32).reshape(-1, 3)
        if tri_active_mask is not None:
            m = np.asarray(tri_active_mask).astype(bool)
            tris = tris if m.ndim == 0 and m else (tris[:0] if m.ndim == 0 else tris[m])
    if bending_edge_indices is not None:
        bend = np.asarray(bending_edge_indices, dtype=np.int32).reshape(-1, 4)
        if bending_edge_active_mask is not None:
            m = np.asarray(bending_edge_active_mask).astype(bool)
            bend = bend if m.ndim == 0 and m else (bend[:0] if m.ndim == 0 else bend[m])
    if tris.size == 0 and bend.size == 0:
        return np.empty((0, 2), dtype=np.int32)
    num_nodes = int(max(tris.max() if tris.size else -1, bend.max() if bend.size else -1)) + 1
    # the pairs are generated and canonicalised natively (no [3 nt + 6 nb, 2] intermediate)
    if device is not None:
        return _lib.trimesh_graph_edges_device(num_nodes, tris, bend, device)
    return _lib.trimesh_graph_edges(num_nodes, tris, bend)


def convert_to_color_groups(num_colors: int, particle_colors: np.ndarray) -> list[np.ndarray]:
    order = np.argsort(particle_colors, kind="stable")
    counts = np.bincount(particle_colors, minlength=num_colors)
    splits = np.cumsum(counts)[:-1]
    return [g.astype(np.int32) for g in np.split(order, splits)]


def color_graph(num_nodes: int, graph_edge_indices: np.ndarray, balance_colors: bool = True,
                target_max_min_color_ratio: float = 1.1,
                algorithm: ColoringAlgorithm = ColoringAlgorithm.MCS) -> list[np.ndarray]:
    if num_nodes == 0:
        return []
    edges = np.asarray(graph_edge_indices)
    if edges.ndim != 2:
        raise ValueError(f"graph_edge_indices must be a 2 dimensional array! The provided one is {edges.ndim} dimensional.")
    colors, nc = _lib.color_graph(num_nodes, edges, algorithm.value, balance_colors, target_max_min_color_ratio)
    return convert_to_color_groups(nc, colors)


def validate_coloring(graph_edges: np.ndarray, color_groups: list[np.ndarray], num_nodes: int) -> bool:
    """True when no graph edge joins two vertices of the same color (and every vertex has one)."""
    colors = np.full(num_nodes, -1, dtype=np.int64)
    for c, g in enumerate(color_groups):
        colors[np.asarray(g)] = c
    if np.any(colors < 0):
        return False
    e = np.asarray(graph_edges).reshape(-1, 2)
    return bool(np.all(colors[e[:, 0]] != colors[e[:, 1]])) if e.size else True


def combine_independent_coloring_plan(sized_groups_1: list, sized_groups_2: list) -> list:
    """Pair (size, chunks) groups of two independent colorings, smallest with largest."""
    if len(sized_groups_1) == 0:
        return sized_groups_2
    if len(sized_groups_2) == 0:
        return sized_groups_1
    if len(sized_groups_1) < len(sized_groups_2):
        sized_groups_1, sized_groups_2 = sized_groups_2, sized_groups_1
    g1 = sorted(sized_groups_1, key=lambda g: g[0])
    g2 = sorted(sized_groups_2, key=lambda g: -g[0])
    out = []
    for i, (s1, c1) in enumerate(g1):
        if i < len(g2):
            s2, c2 = g2[i]
            out.append((s1 + s2, c1 + c2))
        else:
            out.append((s1, c1))
    return out
