"""The library's model set-up tables against the checker's independent restatement (CPU only).

``oracle/setup.py`` restates the bending-edge table (``utils/mesh.py:465-531``), the per-vertex
element CSR (``:595-772``), the conflict graph (``graph_coloring.py:99-197``) and the coloring
(the library's MCS / greedy + balance) with different algorithms (sorting instead of hashing, a
priority queue instead of buckets, numpy instead of native code).  The scenes built both ways must
be identical array for array, which is also what lets ``bench.py``'s CPU-baseline leg build the
benchmark scene without loading the CUDA library.
"""

import warnings

import numpy as np
import pytest

from newton_b200 import scenes
from newton_b200.coloring import ColoringAlgorithm, color_graph, construct_trimesh_graph_edges
from newton_b200.mesh import compute_edge_adjacency, vertex_adjacency_edges, vertex_adjacency_tris
from oracle import setup as S

FIELDS = ("particle_q", "particle_mass", "particle_flags", "tri_indices", "tri_poses", "tri_materials", "tri_areas",
          "edge_indices", "edge_rest_angle", "edge_rest_length", "edge_bending_properties", "shape_world")


def _same_model(a, b):
    for f in FIELDS:
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)
    assert len(a.particle_color_groups) == len(b.particle_color_groups)
    for ga, gb in zip(a.particle_color_groups, b.particle_color_groups):
        np.testing.assert_array_equal(ga, gb)
    for f in ("v_adj_tris", "v_adj_tris_offsets", "v_adj_edges", "v_adj_edges_offsets"):
        np.testing.assert_array_equal(getattr(a.soft_mesh_adjacency, f), getattr(b.soft_mesh_adjacency, f), err_msg=f)


@pytest.mark.parametrize("make", [
    lambda cls: scenes.hanging_cloth(seed=0, device="cpu", builder_cls=cls),
    lambda cls: scenes.draped_cloth(n=64, device="cpu", builder_cls=cls),
    lambda cls: scenes.single_cloth(n=40, include_bending=False, device="cpu", builder_cls=cls),
    lambda cls: scenes.batched_worlds(num_worlds=16, seed=3, n_range=(8, 30), device="cpu", builder_cls=cls),
    lambda cls: scenes.cloth_on_boxes(n=48, side=1.0, device="cpu", builder_cls=cls),
])
def test_scenes_built_with_the_restated_setup_are_identical(make):
    a, qa = make(scenes.ModelBuilder)
    b, qb = make(S.OracleModelBuilder)
    np.testing.assert_array_equal(qa, qb)
    _same_model(a, b)


def test_benchmark_scene_is_identical():
    """The draped-cloth benchmark scene at full size (65,536 vertices)."""
    a, _ = scenes.draped_cloth(n=256, device="cpu")
    b, _ = scenes.draped_cloth(n=256, device="cpu", builder_cls=S.OracleModelBuilder)
    _same_model(a, b)


def test_edge_tables_and_csr_on_random_soups():
    """Non-manifold soups: first-occurrence numbering, the second triangle fills o1, later ones
    are ignored."""
    rng = np.random.default_rng(5)
    for _ in range(40):
        nv = int(rng.integers(3, 30))
        nt = int(rng.integers(1, 120))
        tris = np.stack([rng.choice(nv, 3, replace=False) for _ in range(nt)]).astype(np.int32)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            lib_edges = compute_edge_adjacency(tris)[0]
        np.testing.assert_array_equal(S.edge_table(tris), lib_edges)
        vt, ot = vertex_adjacency_tris(tris, nv + 2)
        np.testing.assert_array_equal(S.vertex_csr(tris, (0, 1, 2), nv + 2)[0], vt)
        np.testing.assert_array_equal(S.vertex_csr(tris, (0, 1, 2), nv + 2)[1], ot)
        ve, oe = vertex_adjacency_edges(lib_edges, nv + 2)
        rv, ro = S.vertex_csr(lib_edges[:, [2, 3, 0, 1]], (2, 3, 0, 1), nv + 2)
        np.testing.assert_array_equal(rv, ve)
        np.testing.assert_array_equal(ro, oe)
        mask = rng.random(nt) > 0.3
        bmask = rng.random(len(lib_edges)) > 0.3
        np.testing.assert_array_equal(S.conflict_edges(tris, mask, lib_edges, bmask),
                                      construct_trimesh_graph_edges(tris, mask, lib_edges, bmask))


@pytest.mark.parametrize("algorithm", [ColoringAlgorithm.MCS, ColoringAlgorithm.GREEDY])
def test_coloring_on_random_graphs(algorithm):
    rng = np.random.default_rng(7)
    for _ in range(30):
        n = int(rng.integers(2, 200))
        m = int(rng.integers(1, 4 * n))
        e = rng.integers(0, n, size=(m, 2))
        e = e[e[:, 0] != e[:, 1]]
        if len(e) == 0:
            continue
        edges = np.unique(np.sort(e, axis=1), axis=0).astype(np.int32)
        for balance in (False, True):
            lib = color_graph(n, edges, balance, 1.1, algorithm)
            ora = S.color(n, edges, balance, 1.1, algorithm)
            assert len(lib) == len(ora)
            for ga, gb in zip(lib, ora):
                np.testing.assert_array_equal(ga, gb)
