"""GPU tests of the set-up tables on the device (``vbd_*_device``): the same edge table, vertex
CSR and conflict-graph edges as the host functions, element for element, on grids, shuffled
grids, non-manifold soups with masks and boundary hinges, and a whole scene built either way."""

import time
import warnings

import numpy as np
import pytest
import torch

from newton_b200 import _lib, scenes
from newton_b200.builder import ModelBuilder
from newton_b200.coloring import construct_trimesh_graph_edges
from newton_b200.mesh import MeshAdjacency, compute_edge_adjacency

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _check_tables(tris, V, rng):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # soups have non-manifold edges
        host = _lib.mesh_edge_adjacency(tris)
    dev = _lib.mesh_edge_adjacency_device(tris, DEV)
    for h, d in zip(host, dev):
        np.testing.assert_array_equal(np.asarray(h), np.asarray(d))
    edges = host[0]
    for entries, slots in ((tris, (0, 1, 2)), (np.ascontiguousarray(edges[:, [2, 3, 0, 1]]), (2, 3, 0, 1))):
        hv, ho = _lib.mesh_vertex_csr(entries, slots, V)
        dv, do = _lib.mesh_vertex_csr_device(entries, slots, V, DEV)
        np.testing.assert_array_equal(hv, dv)
        np.testing.assert_array_equal(ho, do)
    tmask = rng.random(len(tris)) > 0.25
    bmask = rng.random(len(edges)) > 0.25
    for args in ((tris, tmask, edges, bmask), (tris, None, edges, None), (tris, None, None, None)):
        h = construct_trimesh_graph_edges(*args)
        d = construct_trimesh_graph_edges(*args, device=DEV)
        np.testing.assert_array_equal(h, d)
    return edges


def test_device_tables_match_the_host_on_grids_and_soups():
    rng = np.random.default_rng(3)
    for nx, ny in ((1, 1), (7, 5), (64, 48), (300, 200)):
        verts, tris = ModelBuilder.grid_mesh(nx, ny, 0.1, 0.1)
        tris = tris.reshape(-1, 3).astype(np.int32)
        _check_tables(tris, verts.shape[0], rng)
        _check_tables(np.ascontiguousarray(tris[rng.permutation(len(tris))]), verts.shape[0], rng)
    for _ in range(10):
        nv = int(rng.integers(3, 60))
        nt = int(rng.integers(1, 400))
        tris = np.stack([rng.choice(nv, 3, replace=False) for _ in range(nt)]).astype(np.int32)
        _check_tables(tris, nv + 3, rng)  # trailing isolated vertices


def test_device_tables_reject_out_of_range_ids():
    tris = np.array([[0, 1, 2], [1, 2, 7]], np.int32)
    with pytest.raises(_lib.VbdError, match="out of range"):
        _lib.mesh_vertex_csr_device(tris, (0, 1, 2), 5, DEV)
    with pytest.raises(_lib.VbdError, match="out of range"):
        _lib.trimesh_graph_edges_device(5, tris, None, DEV)
    bend = np.array([[0, 9, 1, 2]], np.int32)
    with pytest.raises(_lib.VbdError, match="hinge vertex out of range"):
        _lib.trimesh_graph_edges_device(5, tris[:1], bend, DEV)


def test_scene_built_on_the_device_equals_the_host_build():
    """The 1024 x 1024 cloth on boxes (1,048,576 vertices): colors, adjacency and device-model
    tables identical with the set-up tables computed on the GPU and on the host."""

    class HostBuilder(ModelBuilder):
        setup_device = None

    class DeviceBuilder(ModelBuilder):
        setup_device = DEV

    out = {}
    for name, cls in (("host", HostBuilder), ("device", DeviceBuilder)):
        t = time.perf_counter()
        m, q0 = scenes.cloth_on_boxes(n=1024, device=DEV, builder_cls=cls)
        adj = m.soft_mesh_adjacency
        out[name] = (m, q0, adj, time.perf_counter() - t)
    mh, qh, ah, th = out["host"]
    md, qd, ad, td = out["device"]
    print(f"1M-vertex scene: host tables {th:.2f} s, device tables {td:.2f} s")
    np.testing.assert_array_equal(qh, qd)
    np.testing.assert_array_equal(mh.edge_indices, md.edge_indices)
    assert len(mh.particle_color_groups) == len(md.particle_color_groups)
    for a, b in zip(mh.particle_color_groups, md.particle_color_groups):
        np.testing.assert_array_equal(a, b)
    for k in ("v_adj_tris", "v_adj_tris_offsets", "v_adj_edges", "v_adj_edges_offsets"):
        np.testing.assert_array_equal(getattr(ah, k), getattr(ad, k))
    torch.cuda.synchronize()
