"""CPU tests: C-ABI exports, host model building, adjacency order, coloring, oracle properties."""

import ctypes
import re
from pathlib import Path

import warnings

import numpy as np
import pytest

import oracle
from newton_b200 import ModelBuilder, _lib, scenes
from newton_b200.coloring import construct_trimesh_graph_edges, validate_coloring
from newton_b200.mesh import MeshAdjacency, compute_edge_adjacency

ROOT = Path(__file__).resolve().parent.parent


# ---- C ABI ---------------------------------------------------------------------------------
def _declared_symbols():
    text = (ROOT / "include" / "vbd_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(vbd_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures must cover exactly the header"
    assert b"sm_100a" in lib.vbd_version()


def test_c_abi_rejects_invalid_arguments_without_a_gpu():
    lib = _lib.load()
    out = ctypes.c_void_p()
    assert lib.vbd_model_create(None, ctypes.byref(out)) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert b"NULL" in lib.vbd_last_error()
    d = _lib.VbdModelDesc()
    d.particle_count = 4
    assert lib.vbd_model_create(ctypes.byref(d), ctypes.byref(out)) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert lib.vbd_step(None, None, None, None, None, None, None, ctypes.c_float(0.01), 10, None) != 0
    assert lib.vbd_solver_create(None, None, ctypes.byref(out)) == _lib.VBD_ERR_INVALID_ARGUMENT
    colors = np.zeros(3, np.int32)
    nc = ctypes.c_int32()
    bad = np.array([[0, 5]], np.int32)
    assert lib.vbd_color_graph(3, 1, _lib.as_i32p(bad), 0, 1, ctypes.c_float(1.1), _lib.as_i32p(colors),
                               ctypes.byref(nc)) == _lib.VBD_ERR_INVALID_ARGUMENT
    # host setup functions: NULL outputs and out-of-range vertex ids are errors, not crashes
    tri = np.array([[0, 1, 2]], np.int32)
    n32 = ctypes.c_int32()
    assert lib.vbd_mesh_edge_adjacency(_lib.as_i32p(tri), 1, None, None, None, ctypes.byref(n32),
                                       None) == _lib.VBD_ERR_INVALID_ARGUMENT
    vals = np.zeros(8, np.int32)
    offs = np.zeros(3, np.int32)
    slots = np.array([0, 1, 2], np.int32)
    assert lib.vbd_mesh_vertex_csr(_lib.as_i32p(tri), 1, 3, _lib.as_i32p(slots), 2, _lib.as_i32p(vals),
                                   _lib.as_i32p(offs)) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert b"out of range" in lib.vbd_last_error()
    out = np.zeros((3, 2), np.int32)
    n64 = ctypes.c_int64()
    assert lib.vbd_trimesh_graph_edges(2, _lib.as_i32p(tri), 1, None, 0, _lib.as_i32p(out),
                                       ctypes.byref(n64)) == _lib.VBD_ERR_INVALID_ARGUMENT
    assert lib.vbd_trimesh_graph_edges(3, _lib.as_i32p(tri), 1, None, 0, _lib.as_i32p(out), ctypes.byref(n64)) == 0
    assert n64.value == 3 and out.tolist() == [[0, 1], [0, 2], [1, 2]]


# ---- adjacency -----------------------------------------------------------------------------
def _edge_adjacency_loop(tris, with_maps=False):
    """Loop restatement of MeshAdjacency._compute_edge_adjacency (utils/mesh.py:465-531)."""
    edges = {}
    order = []
    rows = []
    edge_tri = []
    tri_edge = []
    seen = []
    for t, (a, b, c) in enumerate(tris):
        te = []
        for v0, v1, o in ((a, b, c), (b, c, a), (c, a, b)):
            key = (min(v0, v1), max(v0, v1))
            if key not in edges:
                edges[key] = len(order)
                order.append(key)
                rows.append([o, -1, v0, v1])
                edge_tri.append([t, -1])
                seen.append(1)
            else:
                e = edges[key]
                if seen[e] == 1:  # the second side fills o1; a third or later one is non-manifold
                    rows[e][1] = o
                    edge_tri[e][1] = t
                seen[e] += 1
            te.append(edges[key])
        tri_edge.append(te)
    if with_maps:
        return (np.array(rows, dtype=np.int32).reshape(-1, 4), np.array(edge_tri, dtype=np.int32).reshape(-1, 2),
                np.array(tri_edge, dtype=np.int32).reshape(-1, 3))
    return np.array(rows, dtype=np.int32)


def _csr_loop(elems, V, slot_order):
    """Loop restatement of the serial count/fill kernels (utils/mesh.py:675-772)."""
    lists = [[] for _ in range(V)]
    for e, row in enumerate(elems):
        for slot in slot_order:
            v = row[slot]
            if v != -1:
                lists[v] += [e, slot]
    offs = np.zeros(V + 1, np.int32)
    offs[1:] = np.cumsum([len(x) for x in lists])
    return np.array([x for l in lists for x in l], np.int32), offs


def test_edge_and_vertex_adjacency_follow_reference_order():
    rng = np.random.default_rng(0)
    verts, tris = ModelBuilder.grid_mesh(7, 5, 0.1, 0.1)
    tris = tris.reshape(-1, 3)
    tris = tris[rng.permutation(len(tris))]  # arbitrary triangle order
    e, _, _ = compute_edge_adjacency(tris)
    np.testing.assert_array_equal(e, _edge_adjacency_loop(tris.tolist()))
    V = verts.shape[0]
    adj = MeshAdjacency(tris, e).init_vertex_adjacency(V)
    vt, ot = _csr_loop(tris.tolist(), V, [0, 1, 2])
    np.testing.assert_array_equal(adj.v_adj_tris, vt)
    np.testing.assert_array_equal(adj.v_adj_tris_offsets, ot)
    ve, oe = _csr_loop(e.tolist(), V, [2, 3, 0, 1])
    np.testing.assert_array_equal(adj.v_adj_edges, ve)
    np.testing.assert_array_equal(adj.v_adj_edges_offsets, oe)


def test_edge_adjacency_of_non_manifold_soups_matches_the_reference_rules():
    """Random triangle soups (edges shared by 3+ triangles, isolated vertices): the second side
    fills o1 / tri1, later sides only warn, as in utils/mesh.py:510-525; the per-vertex CSRs keep
    element order and skip -1 (boundary) opposites."""
    import warnings

    rng = np.random.default_rng(7)
    for _ in range(20):
        nv = int(rng.integers(3, 40))
        nt = int(rng.integers(1, 200))
        tris = np.stack([rng.choice(nv, 3, replace=False) for _ in range(nt)]).astype(np.int32)
        with warnings.catch_warnings(record=True) as w:
            warnings.simplefilter("always")
            e, et, te = compute_edge_adjacency(tris)
        re, ret, rte = _edge_adjacency_loop(tris.tolist(), with_maps=True)
        np.testing.assert_array_equal(e, re)
        np.testing.assert_array_equal(et, ret)
        np.testing.assert_array_equal(te, rte)
        counts = np.unique(np.sort(np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]]), axis=1),
                           axis=0, return_counts=True)[1]
        assert any("non-manifold" in str(x.message) for x in w) == bool((counts > 2).any())
        adj = MeshAdjacency(tris, e).init_vertex_adjacency(nv + 3)  # trailing isolated vertices
        vt, ot = _csr_loop(tris.tolist(), nv + 3, [0, 1, 2])
        np.testing.assert_array_equal(adj.v_adj_tris, vt)
        np.testing.assert_array_equal(adj.v_adj_tris_offsets, ot)
        ve, oe = _csr_loop(e.tolist(), nv + 3, [2, 3, 0, 1])
        np.testing.assert_array_equal(adj.v_adj_edges, ve)
        np.testing.assert_array_equal(adj.v_adj_edges_offsets, oe)


# ---- builder -------------------------------------------------------------------------------
def test_cloth_grid_counts_masses_and_rest_data():
    model, q0 = scenes.hanging_cloth(seed=0, device="cpu")
    assert (model.particle_count, model.tri_count, model.edge_count) == (1024, 1922, 2945)
    area = (1.0 / 31) ** 2 / 2
    np.testing.assert_allclose(model.tri_areas, area, rtol=1e-6)
    # lumped mass: density * area / 3 per incident triangle, pinned corners zeroed
    counts = np.bincount(model.tri_indices.reshape(-1), minlength=1024)
    expect = 0.1 * area / 3.0 * counts
    pinned = np.flatnonzero((model.particle_flags & 1) == 0)
    assert len(pinned) == 2
    expect[pinned] = 0.0
    np.testing.assert_allclose(model.particle_mass, expect, rtol=1e-6)
    assert np.all(model.particle_inv_mass[pinned] == 0)
    np.testing.assert_allclose(model.edge_rest_angle, 0.0, atol=1e-7)  # flat rest shape
    interior = (model.edge_indices[:, 0] >= 0) & (model.edge_indices[:, 1] >= 0)
    assert interior.sum() == 2945 - 4 * 31
    # hanging in the XZ plane from the two top corners, noise only normal to the cloth (y)
    np.testing.assert_allclose(model.particle_q[:, 1], 0.0, atol=1e-7)
    assert abs(model.particle_q[:, 2].max() - 0.05) < 1e-6 and abs(model.particle_q[:, 2].min() + 0.95) < 1e-6
    np.testing.assert_allclose(model.particle_q[pinned, 2], 0.05, atol=1e-6)
    assert np.abs(q0[:, 1]).max() <= 1e-3 and np.abs(q0[:, 1]).max() > 0
    np.testing.assert_array_equal(q0[:, [0, 2]], model.particle_q[:, [0, 2]])
    # DmInv maps the rest edges to the 2D rest frame: D * DmInv = I
    t = model.tri_indices[0]
    x = model.particle_q[t].astype(np.float64)
    e1 = (x[1] - x[0]) / np.linalg.norm(x[1] - x[0])
    n = np.cross(x[1] - x[0], x[2] - x[0])
    e2 = np.cross(n / np.linalg.norm(n), e1)
    D = np.array([e1, e2]) @ np.array([x[1] - x[0], x[2] - x[0]]).T
    np.testing.assert_allclose(D @ model.tri_poses[0], np.eye(2), atol=1e-5)


def _graph_edges_loop(tris, bend):
    """Set restatement of construct_trimesh_graph_edges (graph_coloring.py:99-197)."""
    pairs = set()
    for a, b, c in tris:
        for u, v in ((a, b), (a, c), (b, c)):
            if u != v:
                pairs.add((min(u, v), max(u, v)))
    for row in bend:
        for i in range(4):
            for j in range(i + 1, 4):
                u, v = row[i], row[j]
                if u >= 0 and v >= 0 and u != v:
                    pairs.add((min(u, v), max(u, v)))
    return np.array(sorted(pairs), dtype=np.int32).reshape(-1, 2)


def test_conflict_graph_edges_match_a_set_restatement():
    rng = np.random.default_rng(11)
    for k in range(25):
        nv = int(rng.integers(3, 40))
        nt = int(rng.integers(1, 150))
        tris = np.stack([rng.choice(nv, 3, replace=False) for _ in range(nt)]).astype(np.int32)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")  # random soups have non-manifold edges
            bend = compute_edge_adjacency(tris)[0]
        tmask = rng.random(nt) > 0.25
        bmask = rng.random(len(bend)) > 0.25
        got = construct_trimesh_graph_edges(tris, tmask, bend, bmask)
        np.testing.assert_array_equal(got, _graph_edges_loop(tris[tmask].tolist(), bend[bmask].tolist()))
        got = construct_trimesh_graph_edges(tris, None, None, None)
        np.testing.assert_array_equal(got, _graph_edges_loop(tris.tolist(), []))
    assert construct_trimesh_graph_edges(None, None, None, None).shape == (0, 2)


def test_coloring_valid_and_balanced():
    for include_bending in (False, True):
        model, _ = scenes.single_cloth(n=40, include_bending=include_bending, device="cpu")
        b = ModelBuilder()
        edges = construct_trimesh_graph_edges(model.tri_indices, None,
                                              model.edge_indices if include_bending else None, None)
        assert validate_coloring(edges, model.particle_color_groups, model.particle_count)
        sizes = [len(g) for g in model.particle_color_groups]
        assert max(sizes) / min(sizes) <= 1.1 + 1e-9
        del b


def test_batched_worlds_merge_colorings():
    model, _ = scenes.batched_worlds(num_worlds=12, seed=1, device="cpu")
    edges = construct_trimesh_graph_edges(model.tri_indices, None, model.edge_indices, None)
    assert validate_coloring(edges, model.particle_color_groups, model.particle_count)
    worlds = model.particle_world
    assert set(np.unique(worlds)) == set(range(12))
    # each world's ground plane belongs to that world
    assert list(model.shape_world) == list(range(12))


# ---- oracle properties ---------------------------------------------------------------------
def test_oracle_thread_count_does_not_change_results():
    model, q0 = scenes.hanging_cloth(seed=2, device="cpu")
    qd = np.zeros_like(q0)
    a = oracle.VBDOracle(model, "f32", threads=1).step(q0, qd, None, 1 / 600, 5)[1]
    b = oracle.VBDOracle(model, "f32", threads=4).step(q0, qd, None, 1 / 600, 5)[1]
    np.testing.assert_array_equal(a, b)


def test_oracle_fp32_tracks_fp64():
    model, q0 = scenes.hanging_cloth(seed=3, device="cpu")
    qd = np.zeros_like(q0)
    o32 = oracle.VBDOracle(model, "f32", threads=4)
    o64 = oracle.VBDOracle(model, "f64", threads=4)
    q32, q64, v32, v64 = q0, q0, qd, qd
    for _ in range(10):
        _, q32, v32 = o32.step(q32, v32, None, 1 / 600, 10)
        _, q64, v64 = o64.step(q64, v64, None, 1 / 600, 10)
    assert np.abs(q32 - q64).max() <= 1e-5
    # pinned corners do not move; free vertices fall
    pinned = np.flatnonzero((model.particle_flags & 1) == 0)
    np.testing.assert_array_equal(q32[pinned], q0[pinned])
    assert q32[:, 2].mean() < q0[:, 2].mean()


def test_free_fall_matches_ballistic_motion():
    """test_cloth.py:1116-1137: an unconstrained cloth free-falls by g t^2 / 2 (implicit Euler)."""
    model, q0 = scenes.single_cloth(n=8, pin_top_corners=False, ground=None, device="cpu")
    qd = np.zeros_like(q0)
    orc = oracle.VBDOracle(model, "f64")
    q, v = q0, qd
    dt, n = 1 / 600, 60
    for _ in range(n):
        _, q, v = orc.step(q, v, None, dt, 5)
    drop = (q0[:, 2] - q[:, 2]).mean()
    t = n * dt
    # implicit Euler falls g dt^2 n(n+1)/2
    np.testing.assert_allclose(drop, 9.81 * dt * dt * n * (n + 1) / 2, rtol=1e-3)
    assert abs(drop - 0.5 * 9.81 * t * t) < 0.2


def test_solver_requires_coloring():
    from newton_b200.solvers import SolverVBD

    b = ModelBuilder()
    verts, tris = ModelBuilder.grid_mesh(3, 3, 0.1, 0.1)
    b.add_cloth_mesh(pos=(0, 0, 0), rot=(0, 0, 0, 1), scale=1.0, vel=(0, 0, 0), vertices=verts, indices=tris,
                     density=0.1)
    m = b.finalize(device="cpu")
    with pytest.raises(ValueError, match="particle_color_groups is empty"):
        SolverVBD(m)
