"""Known-answer tests of the oracle's self-contact restatement (CPU).

Inputs and expected properties follow the reference's own tests in
``newton/tests/test_solver_vbd.py``: barrier continuity (:745, :788), uniform-motion damping
(:1734) and rigid-motion damping of vertex-triangle contacts (seed 29, :95-170, :1649).  The
geometric helpers (closest points) are checked against dense sampling, and detection against a
direct evaluation of the n-ring filter and the distance test over all pairs.
"""

import numpy as np
import pytest

import oracle
from newton_b200 import scenes

PRECISIONS = ["f32", "f64"]


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("where", ["tau", "d_min"])
def test_barrier_is_c2_continuous(precision, where):
    r, k = 0.02, 1.0e3
    d0 = r * 0.5 if where == "tau" else 1.0e-5
    eps = d0 * 1e-5
    a = oracle.self_contact_norm(d0 - eps, r, k, precision)
    b = oracle.self_contact_norm(d0 + eps, r, k, precision)
    np.testing.assert_allclose(a[0], b[0], rtol=1e-3)
    np.testing.assert_allclose(a[1], b[1], rtol=1e-3)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_self_contact_damping_uses_relative_gap_rate(precision):
    pos = np.array([[-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 0.05]], np.float32)
    prev = pos + np.array([0.0, 0.0, 0.01], np.float32)
    out = []
    for kd in (0.0, 50.0):
        has, F, H = oracle.vt_contact(pos, prev, 0.1, 100.0, kd, 0.0, 0.01, 0.1, precision)
        assert has
        out.append((F[3], H[3]))
    np.testing.assert_allclose(out[1][0], out[0][0], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(out[1][1], out[0][1], rtol=1e-6, atol=1e-6)


def _rigid_motions_seed29(count=100, seed=29):
    rng = np.random.default_rng(seed)
    quat = rng.normal(size=(count, 4)).astype(np.float32)
    quat /= np.linalg.norm(quat, axis=1, keepdims=True)
    x, y, z, w = quat[:, 0], quat[:, 1], quat[:, 2], quat[:, 3]
    R = np.empty((count, 3, 3), np.float32)
    R[:, 0, 0] = 1.0 - 2.0 * (y * y + z * z)
    R[:, 0, 1] = 2.0 * (x * y - z * w)
    R[:, 0, 2] = 2.0 * (x * z + y * w)
    R[:, 1, 0] = 2.0 * (x * y + z * w)
    R[:, 1, 1] = 1.0 - 2.0 * (x * x + z * z)
    R[:, 1, 2] = 2.0 * (y * z - x * w)
    R[:, 2, 0] = 2.0 * (x * z - y * w)
    R[:, 2, 1] = 2.0 * (y * z + x * w)
    R[:, 2, 2] = 1.0 - 2.0 * (x * x + y * y)
    t = np.random.default_rng(seed + 1).uniform(-1.0, 1.0, size=(count, 3)).astype(np.float32)
    return R, t


@pytest.mark.parametrize("precision", PRECISIONS)
def test_vertex_triangle_damping_ignores_rigid_motion(precision):
    soft_rest = np.array([[-0.6, -0.5, 0.0], [0.7, -0.4, 0.0], [0.1, 0.8, 0.0], [0.05, 0.1, 0.04]], np.float32)
    R, t = _rigid_motions_seed29()
    worst = 0.0
    for s in range(len(R)):
        pos = soft_rest @ R[s].T + t[s]
        _, Fd, _ = oracle.vt_contact(pos, soft_rest, 0.1, 100.0, 20.0, 0.0, 0.01, 0.1, precision)
        _, Fu, _ = oracle.vt_contact(pos, soft_rest, 0.1, 100.0, 0.0, 0.0, 0.01, 0.1, precision)
        worst = max(worst, float(np.linalg.norm(Fd - Fu, axis=1).max()))
    assert worst <= 1e-4


def test_closest_points_match_dense_sampling():
    rng = np.random.default_rng(3)
    for _ in range(200):
        a, b, c, p = rng.normal(size=(4, 3))
        cp, bary = oracle.triangle_closest_point(a, b, c, p)
        np.testing.assert_allclose(bary.sum(), 1.0, atol=1e-12)
        assert np.all(bary >= -1e-12)
        np.testing.assert_allclose(cp, bary[0] * a + bary[1] * b + bary[2] * c, atol=1e-12)
        u, v = np.meshgrid(np.linspace(0, 1, 61), np.linspace(0, 1, 61))
        m = (u + v) <= 1.0
        pts = a + u[m, None] * (b - a) + v[m, None] * (c - a)
        assert np.linalg.norm(cp - p) <= np.linalg.norm(pts - p, axis=1).min() + 1e-12
        p1, q1, p2, q2 = rng.normal(size=(4, 3))
        s, t, d = oracle.closest_edge_edge(p1, q1, p2, q2)
        assert 0.0 <= s <= 1.0 and 0.0 <= t <= 1.0
        np.testing.assert_allclose(d, np.linalg.norm((p1 + s * (q1 - p1)) - (p2 + t * (q2 - p2))), atol=1e-12)
        g = np.linspace(0, 1, 201)
        A = p1 + g[:, None] * (q1 - p1)
        B = p2 + g[:, None] * (q2 - p2)
        assert d <= np.linalg.norm(A[:, None, :] - B[None, :, :], axis=2).min() + 1e-12


def _ring1(model):
    nb = [set() for _ in range(model.particle_count)]
    for e in model.edge_indices:
        nb[e[2]].add(int(e[3]))
        nb[e[3]].add(int(e[2]))
    return nb


def test_detection_matches_pairwise_filter_and_distance():
    """Vertex-triangle / edge-edge candidates of a folded cloth: incident pairs, pairs within one
    ring (threshold 2) and pairs beyond the margin are excluded; all others are found."""
    model, q0 = scenes.single_cloth(n=10, side=0.5, seed=1, pin_top_corners=False, ground=None, device="cpu")
    q = q0.copy().astype(np.float64)
    # fold the cloth over the line x = 0 so the halves lie 4 mm apart
    right = q[:, 0] > 0.0
    q[right, 0] = -q[right, 0]
    q[right, 2] += 0.004
    q = q.astype(np.float32)
    orc = oracle.VBDOracle(model, "f32")
    margin = 0.006
    orc.set_self_contact(radius=0.004, margin=margin, vertex_buffer=64, edge_buffer=128)
    vc, vl, ec, el, dropped = orc.self_contact_detect(q)
    assert dropped == 0
    nb = _ring1(model)
    tris, edges = model.tri_indices, model.edge_indices
    for v in range(model.particle_count):
        expect = []
        for t, (a, b, c) in enumerate(tris):
            if v in (a, b, c) or ({a, b, c} & nb[v]):
                continue
            cp, _ = oracle.triangle_closest_point(q[a], q[b], q[c], q[v])
            if np.linalg.norm(cp - q[v].astype(np.float64)) < margin - 1e-6:
                expect.append(t)
        got = set(vl[v, :vc[v]].tolist())
        assert set(expect) <= got
        assert all(t not in got or not ({*tris[t]} & (nb[v] | {v})) for t in range(len(tris)))
    for e, (_, _, a0, a1) in enumerate(edges):
        got = set(el[e, :ec[e]].tolist())
        near = nb[a0] | nb[a1]
        for f in got:
            b0, b1 = edges[f, 2], edges[f, 3]
            assert not ({a0, a1} & {b0, b1}) and not ({b0, b1} & near)
            assert e in set(el[f, :ec[f]].tolist())  # symmetric
    assert vc.sum() > 0 and ec.sum() > 0


def test_external_filter_maps_remove_exactly_their_pairs():
    """particle_external_vertex/edge_contact_filtering_map: the listed candidates disappear from the
    lists of the rows that name them, and nothing else changes (per side for edge-edge pairs)."""
    model, q0 = scenes.single_cloth(n=10, side=0.5, seed=1, pin_top_corners=False, ground=None, device="cpu")
    q = q0.copy().astype(np.float64)
    right = q[:, 0] > 0.0
    q[right, 0] = -q[right, 0]
    q[right, 2] += 0.004
    q = q.astype(np.float32)
    orc = oracle.VBDOracle(model, "f32")
    orc.set_self_contact(radius=0.004, margin=0.006, vertex_buffer=64, edge_buffer=128)
    vc, vl, ec, el, _ = orc.self_contact_detect(q)
    v = int(np.argmax(vc))
    e = int(np.argmax(ec))
    drop_t = set(vl[v, :2].tolist())
    drop_g = set(el[e, :3].tolist())
    orc.set_self_contact(radius=0.004, margin=0.006, vertex_buffer=64, edge_buffer=128,
                         vertex_filter_map={v: drop_t}, edge_filter_map={e: drop_g})
    vc2, vl2, ec2, el2, _ = orc.self_contact_detect(q)
    assert set(vl2[v, :vc2[v]].tolist()) == set(vl[v, :vc[v]].tolist()) - drop_t
    assert set(el2[e, :ec2[e]].tolist()) == set(el[e, :ec[e]].tolist()) - drop_g
    other = np.ones(model.particle_count, bool)
    other[v] = False
    np.testing.assert_array_equal(vc2[other], vc[other])
    for g in drop_g:  # the other side keeps the pair unless its own map names it
        assert e in set(el2[g, :ec2[g]].tolist())
