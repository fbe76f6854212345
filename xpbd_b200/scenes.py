"""Seeded synthetic scene builders.

Each builder adds bodies and constraints to an already-constructed solver through
the public scene-building API (``add_particle`` / ``add_distance`` /
``add_floor_contact`` / ``enable_self_collision`` for the 3-DOF ``Solver``;
``add_box`` / ``add_particle`` / ``add_joint`` for ``Solver6DOF``).  Because only
that API is used, the same builder produces the identical scene on the reference
solver, on the CPU oracle and on the B200 engine.

Workloads (all ``numpy.random.default_rng(seed)``):

* cloth      -- N x N particle grid, two pinned corners, structural + shear + bend
                DISTANCE rows and one FLOOR row per particle (32 x 32: 1984 + 1922
                + 1920 + 1024 rows).
* sphere pile -- lattice of jittered spheres with FLOOR rows and sphere-sphere
                self collision (16 x 8 x 16 = 2048 spheres).
* box pile   -- lattice of randomly sized, randomly oriented boxes
                (12 x 10 x 12 = 1440 boxes, half extents U[0.1, 0.3] m, density
                1000 kg/m^3, orientation uniform on S^3).
"""

from __future__ import annotations

import numpy as np


def build_cloth(s, res=32, spacing=0.02, mass=0.01, y=1.0, compliance=1e-8,
                floor_y=0.0, mu=0.3, velocity=(0.0, 0.0, 0.0), floor=True,
                origin=(0.0, 0.0)):
    """Horizontal cloth in the x-z plane at height ``y``; particles (0, 0) and
    (res-1, 0) are static.  Rows are added type by type: structural (right,
    down per node), shear (both diagonals per cell), bend (2 apart, right and
    down per node), then FLOOR rows."""
    idx = np.empty((res, res), np.int64)
    handles = {}
    for iy in range(res):
        for ix in range(res):
            pinned = iy == 0 and ix in (0, res - 1)
            b = s.add_particle((origin[0] + ix * spacing, y, origin[1] + iy * spacing),
                               mass=0.0 if pinned else mass, velocity=velocity,
                               collide=False)
            idx[iy, ix] = b.index
            handles[b.index] = b
    H = lambda iy, ix: handles[int(idx[iy, ix])]  # noqa: E731
    for iy in range(res):
        for ix in range(res):
            if ix + 1 < res:
                s.add_distance(H(iy, ix), H(iy, ix + 1), compliance=compliance)
            if iy + 1 < res:
                s.add_distance(H(iy, ix), H(iy + 1, ix), compliance=compliance)
    for iy in range(res - 1):
        for ix in range(res - 1):
            s.add_distance(H(iy, ix), H(iy + 1, ix + 1), compliance=compliance)
            s.add_distance(H(iy, ix + 1), H(iy + 1, ix), compliance=compliance)
    for iy in range(res):
        for ix in range(res):
            if ix + 2 < res:
                s.add_distance(H(iy, ix), H(iy, ix + 2), compliance=compliance)
            if iy + 2 < res:
                s.add_distance(H(iy, ix), H(iy + 2, ix), compliance=compliance)
    if floor:
        for iy in range(res):
            for ix in range(res):
                s.add_floor_contact(H(iy, ix), floor_y=floor_y, friction=mu)
    return idx


def build_sphere_pile(s, nx=16, ny=8, nz=16, pitch=0.11, y0=0.2, jitter=0.01,
                      r=0.05, mass=1.0, mu=0.5, margin=0.0, seed=0):
    """Jittered sphere lattice; every sphere gets a FLOOR row at ``y = r`` and
    sphere-sphere self collision is enabled with friction ``mu``."""
    rng = np.random.default_rng(seed)
    for ly in range(ny):
        for ix in range(nx):
            for iz in range(nz):
                j = rng.uniform(-jitter, jitter, 3)
                b = s.add_particle((ix * pitch + j[0], y0 + ly * pitch + j[1],
                                    iz * pitch + j[2]), mass=mass, radius=r,
                                   friction=mu)
                s.add_floor_contact(b, floor_y=r, friction=mu)
    s.enable_self_collision(True, margin=margin, default_friction=mu)


def box_pile_arrays(nx=12, ny=10, nz=12, pitch=0.8, y0=0.5, he_lo=0.1, he_hi=0.3,
                    density=1000.0, seed=0):
    """Positions, half extents, masses and orientations of the box pile."""
    rng = np.random.default_rng(seed)
    pos, he, mass, quat = [], [], [], []
    for ly in range(ny):
        for ix in range(nx):
            for iz in range(nz):
                e = rng.uniform(he_lo, he_hi, 3)
                q = rng.normal(size=4)
                q = q / np.linalg.norm(q)
                pos.append((ix * pitch, y0 + ly * pitch, iz * pitch))
                he.append(tuple(e))
                mass.append(density * 8.0 * e[0] * e[1] * e[2])
                quat.append(tuple(q))
    return pos, he, mass, quat


def build_box_pile(s, **kw):
    pos, he, mass, quat = box_pile_arrays(**kw)
    for p, e, m, q in zip(pos, he, mass, quat):
        s.add_box(p, e, float(m), quaternion=q)
