"""Seeded synthetic inputs of the five benchmark configurations.

No dataset or mesh ships with the reference for these workloads, so every
input is generated here from a fixed seed (numpy default_rng):

  C1 cube64      cube 0.1 m, 12 tris, dense 64^3 with 4 voxels of padding;
                 100k uniform points in the padded box (seed 0), Trilinear.
  C2 cylinder    hollow cylinder R 50 / r 40 / H 20 mm, 512 x 16 segments
                 (34,816 tris); dense 128^3 (snapped to 128x128x64) and
                 sparse band 3 voxels, 8^3 bricks; 1M Tricubic points on the
                 surface offset along the normal by N(0, (2h)^2) (seed 1).
  C3 ring-cube   cube 100 mm at 128^3; torus R 50 / r 10 mm, 192 x 20
                 (7,680 tris) as quadrature body; 4096 poses (seed 2).
  C4 gears       256 star-profile gear prisms, sparse grids (seed 3).
  C5 icosphere   perturbed icosphere (1.31M tris), sparse 512^3 (seed 4).
"""
from __future__ import annotations

import math

import numpy as np

from . import meshes as M

CUBE_SIDE = 0.1


def c1_cube64(n_points=100_000, seed=0):
    v, t = M.cube(CUBE_SIDE)
    h = CUBE_SIDE / 56.0
    params = dict(voxel_size=h, padding=4.0 * h / (CUBE_SIDE * math.sqrt(3.0)),
                  target_resolution=64, max_resolution=64)
    return dict(name="cube64", verts=v, tris=t, build=params, n_points=n_points, seed=seed)


def c1_points(grid_bmin, grid_bmax, n=100_000, seed=0):
    rng = np.random.default_rng(seed)
    return rng.uniform(grid_bmin, grid_bmax, size=(n, 3)).astype(np.float32)


def c2_cylinder():
    v, t = M.hollow_cylinder(0.05, 0.04, 0.02, n_az=512, n_vert=16, n_rad=1)
    dense = dict(target_resolution=128, max_resolution=128, padding=0.1)
    sparse = dict(dense, block_dim=8, band_voxels=3, halo_voxels=2)
    return dict(name="hollow_cylinder", verts=v, tris=t, dense=dense, sparse=sparse)


def c2_points(verts, tris, voxel, n=1_000_000, seed=1):
    rng = np.random.default_rng(seed)
    return M.surface_points(verts, tris, n, 2.0 * voxel, rng).astype(np.float32)


def c3_ring_cube(n_poses=4096, seed=2):
    cv, ct = M.cube(CUBE_SIDE)
    tv, tt = M.torus(0.05, 0.01, 192, 20)
    qx, qw = M.centroid_quadrature(tv, tt)
    rng = np.random.default_rng(seed)
    z = rng.uniform(0.060, 0.070, n_poses)
    phi = rng.uniform(0.0, 2.0 * np.pi, n_poses)
    ang = np.deg2rad(5.0) * rng.uniform(0.0, 1.0, n_poses)
    axis = np.stack([np.cos(phi), np.sin(phi), np.zeros(n_poses)], 1)
    R = _axis_angle(axis, ang)

    def ball(radius):
        d = rng.normal(size=(n_poses, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        return d * (radius * rng.uniform(0.0, 1.0, n_poses) ** (1.0 / 3.0))[:, None]

    v = ball(0.1)
    w = ball(1.0)
    r = np.stack([np.zeros(n_poses), np.zeros(n_poses), z], 1)
    return dict(name="ring_on_cube", cube=(cv, ct), torus=(tv, tt), quad_x=qx, quad_w=qw,
                build=dict(target_resolution=128, max_resolution=128, padding=0.1),
                r=r, R=R, v=v, w=w,
                params=dict(stiffness=1e11, order=2.0, damping=1e4, friction=0.3,
                            regularizer=1e-4, activation_distance=1e-5))


def be_ring_drops(n_scenes=2048, seed=5):
    """Batched drops of the ring of c3_ring_cube (torus R 50 mm, r 10 mm,
    7,680 centroid quadrature points, steel) on a 0.3 x 0.3 x 0.05 m slab
    whose top face is the plane z = 0 of its SDF frame (dense, target
    resolution 128), with the same contact law as c3_ring_cube.  Each scene
    starts with the ring's lowest point 0.5-3 mm above the plane, tilted by
    at most 5 degrees, falling at 0.1-0.3 m/s with |v_xy| <= 0.1 m/s and
    |w| <= 1 rad/s."""
    cv, ct = M.cube(1.0)
    sv = cv * np.array([0.3, 0.3, 0.05]) + np.array([0.0, 0.0, -0.025])
    tv, tt = M.torus(0.05, 0.01, 192, 20)
    qx, qw = M.centroid_quadrature(tv, tt)
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0.0, 2.0 * np.pi, n_scenes)
    ang = np.deg2rad(5.0) * rng.uniform(0.0, 1.0, n_scenes)
    axis = np.stack([np.cos(phi), np.sin(phi), np.zeros(n_scenes)], 1)
    R = _axis_angle(axis, ang)
    low = np.einsum("nij,qj->nqi", R, qx)[:, :, 2].min(axis=1)
    r = np.stack([rng.uniform(-0.05, 0.05, n_scenes), rng.uniform(-0.05, 0.05, n_scenes),
                  -low + rng.uniform(0.0005, 0.003, n_scenes)], 1)
    v = np.stack([rng.uniform(-0.07, 0.07, n_scenes), rng.uniform(-0.07, 0.07, n_scenes),
                  -rng.uniform(0.1, 0.3, n_scenes)], 1)
    d = rng.normal(size=(n_scenes, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = d * rng.uniform(0.0, 1.0, n_scenes)[:, None]
    Rr, rr, rho = 0.05, 0.01, 7800.0
    mass = rho * 2.0 * np.pi ** 2 * Rr * rr * rr
    inertia = np.diag([mass * (Rr * Rr / 2 + 5 * rr * rr / 8)] * 2 + [mass * (Rr * Rr + 3 * rr * rr / 4)])
    return dict(name="ring_drops_on_slab", slab=(sv, ct), torus=(tv, tt), quad_x=qx, quad_w=qw,
                build=dict(target_resolution=128, max_resolution=128, padding=0.1),
                r=r, R=R, v=v, w=w, mass=mass, inertia=inertia,
                params=dict(stiffness=1e11, order=2, damping=1e4, friction=0.3, regularizer=1e-4,
                            activation_distance=1e-5))


def _axis_angle(axis, ang):
    k = axis / np.maximum(np.linalg.norm(axis, axis=1, keepdims=True), 1e-300)
    K = np.zeros((len(k), 3, 3))
    K[:, 0, 1], K[:, 0, 2] = -k[:, 2], k[:, 1]
    K[:, 1, 0], K[:, 1, 2] = k[:, 2], -k[:, 0]
    K[:, 2, 0], K[:, 2, 1] = -k[:, 1], k[:, 0]
    s, c = np.sin(ang)[:, None, None], np.cos(ang)[:, None, None]
    return np.eye(3)[None] + s * K + (1 - c) * (K @ K)


def c4_gears(n_gears=256, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_gears):
        teeth = int(rng.integers(20, 61))
        r_out = float(rng.uniform(0.020, 0.080))
        thick = float(rng.uniform(0.005, 0.020))
        target = int(round(math.exp(rng.uniform(math.log(2000), math.log(60000)))))
        res = int(rng.choice([64, 96, 128, 192, 256]))
        v, t = M.gear_prism(teeth, r_out, thick, target)
        out.append(dict(verts=v, tris=t, teeth=teeth, r_outer=r_out, thickness=thick,
                        resolution=res,
                        sparse=dict(target_resolution=res, max_resolution=res, padding=0.1,
                                    block_dim=8, band_voxels=3, halo_voxels=2)))
    return out


def c5_icosphere(subdivisions=8, seed=4):
    v, t = M.perturbed_icosphere(subdivisions, 0.1, 0.002, 8, 1, 6, seed)
    return dict(name="perturbed_icosphere", verts=v, tris=t,
                sparse=dict(target_resolution=512, max_resolution=512, padding=0.1, block_dim=8,
                            band_voxels=3, halo_voxels=2))


def c5_points(verts, tris, voxel, n=16_000_000, seed=4, chunk=2_000_000):
    """C5 queries: surface points (triangle by area, uniform barycentric)
    offset along the face normal by U(-4h, 4h), drawn in chunks of ``chunk``
    from one generator; float32 (n, 3)."""
    rng = np.random.default_rng(seed)
    nrm, area = M.face_normals(verts, tris)
    cdf = np.cumsum(area)
    cdf /= cdf[-1]
    out = np.empty((n, 3), np.float32)
    for a in range(0, n, chunk):
        m = min(n, a + chunk) - a
        idx = np.minimum(np.searchsorted(cdf, rng.random(m), side="right"), len(tris) - 1)
        s = np.sqrt(rng.random(m))
        r2 = rng.random(m)
        t = tris[idx]
        x = ((1.0 - s)[:, None] * verts[t[:, 0]] + (s * (1.0 - r2))[:, None] * verts[t[:, 1]] +
             (s * r2)[:, None] * verts[t[:, 2]])
        off = rng.uniform(-4.0 * voxel, 4.0 * voxel, m)
        out[a:a + m] = x + off[:, None] * nrm[idx]
    return out


def near_surface_points(verts, tris, voxel, n, seed, band_voxels=4.0):
    """Surface points offset along the normal by U(-band*h, band*h)."""
    rng = np.random.default_rng(seed)
    return M.surface_points(verts, tris, n, band_voxels * voxel, rng,
                            uniform_offset=True).astype(np.float32)
