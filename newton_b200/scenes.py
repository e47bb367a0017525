"""Seeded synthetic cloth scenes with the shapes, sizes and materials of the VBD cloth workloads.

Every scene takes ``builder_cls`` (default ``ModelBuilder``): a subclass that computes the
connectivity and coloring another way builds the same scene.

* ``single_cloth``   one square cloth, horizontal (XY plane, Z up) with U(-1 mm, 1 mm) z-noise
                     on the initial positions (rest shape flat), optional pinned corners, ground
                     plane and sphere collider.  Materials default to the cloth workload:
                     tri_ke = tri_ka = 1e4, tri_kd = 1e-3, edge_ke = 1e-2, edge_kd = 0,
                     density 0.1 kg/m^2, gravity -9.81 m/s^2.
* ``hanging_cloth``  32 x 32 vertices, 1 m side, hanging in the XZ plane (top edge at z = 0.05,
                     bottom edge 5 cm above the ground at z = -1), two top corners pinned; the
                     1 mm noise is applied normal to the cloth (along y): noise along z would lie
                     in the plane of a cloth hanging in XZ.
* ``draped_cloth``   256 x 256 vertices, 2 m side, flat, falling onto a static sphere (r = 0.4 m)
                     and the ground; contact ke = 1e4 (particle and shape side), margin 5 mm.
* ``cloth_on_boxes`` 1024 x 1024 vertices, 4 m side, 0.8 m above 16 static boxes (seeded yaw and
                     position in [-1.5, 1.5]^2, half-extents U[0.1, 0.4], resting on the ground);
                     the self-contact workload (radius 2 mm, margin 3 mm in the solver).
* ``batched_worlds`` independent cloth worlds of uneven size (N ~ U{16..96}, side ~ U[0.5, 2] m,
                     tri_ke ~ logU[1e3, 1e5] with ka = ke, edge_ke ~ logU[1e-3, 1e-1], 0-4 random
                     boundary pins, a ground plane per world), merged into one model whose color
                     groups pair small with large groups across worlds.
"""

from __future__ import annotations

import numpy as np

from .builder import ModelBuilder
from .model import ParticleFlags

CLOTH_MATERIAL = dict(tri_ke=1.0e4, tri_ka=1.0e4, tri_kd=1.0e-3, edge_ke=1.0e-2, edge_kd=0.0)


def _cloth(builder: ModelBuilder, n: int, side: float, height: float, density: float, particle_radius: float,
           material: dict, center=(0.0, 0.0), vertical: bool = False) -> int:
    verts, tris = ModelBuilder.grid_mesh(n - 1, n - 1, side / (n - 1), side / (n - 1))
    start = builder.particle_count
    if vertical:
        # rotation by +90 degrees about x: grid (x, y, 0) -> (x, 0, y); the top edge (largest grid y)
        # ends at z = height
        s2 = float(np.sqrt(0.5))
        pos, rot = (center[0] - 0.5 * side, center[1], height - side), (s2, 0.0, 0.0, s2)
    else:
        pos, rot = (center[0] - 0.5 * side, center[1] - 0.5 * side, height), (0.0, 0.0, 0.0, 1.0)
    builder.add_cloth_mesh(pos=pos, rot=rot, scale=1.0, vel=(0.0, 0.0, 0.0), vertices=verts, indices=tris,
                           density=density, particle_radius=particle_radius, **material)
    return start


def _pin(builder: ModelBuilder, indices) -> None:
    idx = np.asarray(indices, dtype=np.int64)
    builder.set_particle_mass(idx, 0.0)
    flags = builder.particle_flags[idx] & ~ParticleFlags.ACTIVE
    builder.set_particle_flags(idx, flags)


def single_cloth(n: int = 32, side: float = 1.0, seed: int = 0, pin_top_corners: bool = True, ground: float | None = -1.0,
                 sphere: tuple | None = None, height: float = 0.0, particle_radius: float = 5.0e-3,
                 density: float = 0.1, material: dict | None = None, contact_ke: float = 1.0e4,
                 include_bending: bool = True, z_noise: float = 1.0e-3, vertical: bool = False, device="cuda:0",
                 builder_cls=ModelBuilder):
    """Returns (model, initial particle_q float32 [V,3] with U(-z_noise, z_noise) noise normal to the
    cloth: along z for a horizontal cloth, along y for a ``vertical`` one (XZ plane, top edge at
    z = ``height``))."""
    material = dict(CLOTH_MATERIAL if material is None else material)
    b = builder_cls()
    start = _cloth(b, n, side, height, density, particle_radius, material, vertical=vertical)
    if pin_top_corners:
        _pin(b, [start + (n - 1) * n, start + n * n - 1])
    cfg = ModelBuilder.ShapeConfig(ke=contact_ke)
    if ground is not None:
        b.add_ground_plane(height=ground, cfg=cfg)
    if sphere is not None:
        center, radius = sphere
        b.add_shape_sphere(-1, xform=(tuple(center), (0.0, 0.0, 0.0, 1.0)), radius=radius, cfg=cfg)
    b.color(include_bending=include_bending)
    m = b.finalize(device=device)
    m.soft_contact_ke = contact_ke
    rng = np.random.default_rng(seed)
    q0 = m.particle_q.copy()
    if z_noise > 0:
        q0[:, 1 if vertical else 2] += rng.uniform(-z_noise, z_noise, size=m.particle_count).astype(np.float32)
    return m, q0


def hanging_cloth(seed: int = 0, device="cuda:0", builder_cls=ModelBuilder):
    """32 x 32 vertices (1,922 triangles), 1 m side, hanging in the XZ plane from its two pinned top
    corners (top edge at z = 0.05), ground at z = -1."""
    return single_cloth(n=32, side=1.0, seed=seed, pin_top_corners=True, ground=-1.0, height=0.05, vertical=True,
                        device=device, builder_cls=builder_cls)


def draped_cloth(n: int = 256, seed: int = 0, device="cuda:0", offset: tuple = (0.0, 0.0), height: float = 1.1,
                 builder_cls=ModelBuilder):
    """256 x 256 vertices (130,050 triangles), 2 m side, flat and at rest 0.2 m above a static
    sphere of radius 0.4 m (centre offset by ``offset`` in x, y), and the ground plane."""
    return single_cloth(n=n, side=2.0, seed=seed, pin_top_corners=False, ground=0.0,
                        sphere=((offset[0], offset[1], 0.5), 0.4), height=height, z_noise=0.0, device=device,
                        builder_cls=builder_cls)


def cloth_on_boxes(n: int = 1024, side: float = 4.0, boxes: int = 16, seed: int = 0, height: float = 0.8,
                   device="cuda:0", builder_cls=ModelBuilder):
    """Large cloth falling onto seeded static boxes on the ground (self-contact workload)."""
    rng = np.random.default_rng(seed)
    b = builder_cls()
    _cloth(b, n, side, height, 0.1, 1.0e-3, dict(CLOTH_MATERIAL))
    cfg = ModelBuilder.ShapeConfig(ke=1.0e4)
    b.add_ground_plane(height=0.0, cfg=cfg)
    for _ in range(boxes):
        # at the 4 m side: half-extents U[0.1, 0.4] m, centres in [-1.5, 1.5]^2 (scaled with the side)
        hx, hy, hz = (float(v) for v in rng.uniform(0.025 * side, 0.1 * side, size=3))
        x, y = (float(v) for v in rng.uniform(-0.375 * side, 0.375 * side, size=2))
        yaw = float(rng.uniform(0.0, 2.0 * np.pi))
        rot = (0.0, 0.0, float(np.sin(0.5 * yaw)), float(np.cos(0.5 * yaw)))
        b.add_shape_box(-1, xform=((x, y, hz), rot), hx=hx, hy=hy, hz=hz, cfg=cfg)
    b.color(include_bending=True)
    m = b.finalize(device=device)
    m.soft_contact_ke = 1.0e4
    return m, m.particle_q.copy()


def batched_worlds(num_worlds: int = 512, seed: int = 0, n_range=(16, 96), device="cuda:0", include_bending=True,
                   builder_cls=ModelBuilder):
    """Independent cloth worlds of uneven size merged into one model (colors combined per world)."""
    rng = np.random.default_rng(seed)
    top = builder_cls()
    for w in range(num_worlds):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        side = float(rng.uniform(0.5, 2.0))
        ke = float(10.0 ** rng.uniform(3.0, 5.0))
        eke = float(10.0 ** rng.uniform(-3.0, -1.0))
        npin = int(rng.integers(0, 5))
        b = builder_cls()
        mat = dict(tri_ke=ke, tri_ka=ke, tri_kd=1.0e-3, edge_ke=eke, edge_kd=0.0)
        _cloth(b, n, side, 0.5, 0.1, 5.0e-3, mat)
        if npin:
            ring = np.concatenate([np.arange(n), np.arange(n) + (n - 1) * n, np.arange(1, n - 1) * n,
                                   np.arange(1, n - 1) * n + n - 1])
            _pin(b, rng.choice(ring, size=npin, replace=False))
        b.add_ground_plane(height=0.0, cfg=ModelBuilder.ShapeConfig(ke=1.0e4))
        b.color(include_bending=include_bending)
        top.add_builder(b, world=w)
    m = top.finalize(device=device)
    m.soft_contact_ke = 1.0e4
    return m, m.particle_q.copy()
