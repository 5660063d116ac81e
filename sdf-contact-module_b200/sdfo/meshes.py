"""Procedural triangle meshes and quadrature used by the benchmarks and tests.

All meshes are closed, consistently wound (counter-clockwise seen from
outside, so the face normal (b-a)x(c-a) points out of the solid), and returned
as ``(vertices float64 (V,3), triangles int32 (T,3))``.

The shapes restate the workloads the SdfOracle hot path is measured on:
an axis-aligned cube, a hollow cylinder (the generator in the reference's
scripts/gen_meshes.py:79-144 builds the same topology: two cylindrical walls
plus annular caps), a torus ring, star-profile gear prisms and a perturbed
icosphere.  Sizes are in metres.
"""
from __future__ import annotations

import math

import numpy as np


def signed_volume(verts: np.ndarray, tris: np.ndarray) -> float:
    """Divergence-theorem volume; positive for outward winding."""
    a, b, c = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def cube(side: float = 0.1, center=(0.0, 0.0, 0.0)):
    """Axis-aligned cube with 8 vertices and 12 triangles (2 per face)."""
    h = 0.5 * side
    c = np.asarray(center, dtype=np.float64)
    v = np.array([[x, y, z] for z in (-h, h) for y in (-h, h) for x in (-h, h)],
                 dtype=np.float64) + c
    # vertex id = x + 2y + 4z (bits)
    t = np.array([
        [0, 2, 1], [1, 2, 3],  # z-
        [4, 5, 6], [5, 7, 6],  # z+
        [0, 1, 4], [1, 5, 4],  # y-
        [2, 6, 3], [3, 6, 7],  # y+
        [0, 4, 2], [2, 4, 6],  # x-
        [1, 3, 5], [3, 7, 5],  # x+
    ], dtype=np.int32)
    return v, t


def hollow_cylinder(r_outer=0.05, r_inner=0.04, height=0.02, n_az=512, n_vert=16,
                    n_rad=1, z0=0.0):
    """Hollow cylinder: outer and inner walls of n_az x n_vert quads and two
    annular caps of n_az x n_rad quads.  The default (512 x 16, one radial
    ring) has 2*16384 + 2*1024 = 34,816 triangles."""
    verts = []
    tris = []

    def wall(r, outward):
        base = sum(len(x) for x in verts)
        th = 2.0 * np.pi * np.arange(n_az) / n_az
        z = z0 + height * np.arange(n_vert + 1) / n_vert
        zz, tt = np.meshgrid(z, th, indexing="ij")
        ring = np.stack([r * np.cos(tt), r * np.sin(tt), zz], axis=-1).reshape(-1, 3)
        verts.append(ring)
        k, j = np.meshgrid(np.arange(n_vert), np.arange(n_az), indexing="ij")
        j1 = (j + 1) % n_az
        i0 = base + k * n_az + j
        i1 = base + k * n_az + j1
        i2 = base + (k + 1) * n_az + j
        i3 = base + (k + 1) * n_az + j1
        if outward:
            q = np.stack([np.stack([i0, i1, i2], -1), np.stack([i1, i3, i2], -1)], -2)
        else:
            q = np.stack([np.stack([i0, i2, i1], -1), np.stack([i1, i2, i3], -1)], -2)
        tris.append(q.reshape(-1, 3))

    def cap(z, up):
        base = sum(len(x) for x in verts)
        th = 2.0 * np.pi * np.arange(n_az) / n_az
        r = r_inner + (r_outer - r_inner) * np.arange(n_rad + 1) / n_rad
        tt, rr = np.meshgrid(th, r, indexing="ij")
        pts = np.stack([rr * np.cos(tt), rr * np.sin(tt), np.full_like(rr, z)], -1)
        verts.append(pts.reshape(-1, 3))
        j, i = np.meshgrid(np.arange(n_az), np.arange(n_rad), indexing="ij")
        j1 = (j + 1) % n_az
        i0 = base + j * (n_rad + 1) + i
        i1 = i0 + 1
        i2 = base + j1 * (n_rad + 1) + i
        i3 = i2 + 1
        if up:
            q = np.stack([np.stack([i0, i1, i2], -1), np.stack([i1, i3, i2], -1)], -2)
        else:
            q = np.stack([np.stack([i0, i2, i1], -1), np.stack([i1, i2, i3], -1)], -2)
        tris.append(q.reshape(-1, 3))

    wall(r_inner, outward=False)
    wall(r_outer, outward=True)
    cap(z0, up=False)
    cap(z0 + height, up=True)
    v = np.concatenate(verts).astype(np.float64)
    t = np.concatenate(tris).astype(np.int32)
    return v, t


def torus(R=0.05, r=0.01, n_major=192, n_minor=20, center=(0.0, 0.0, 0.0)):
    """Torus about the z axis; n_major * n_minor * 2 triangles (7,680 by default)."""
    u = 2.0 * np.pi * np.arange(n_major) / n_major
    w = 2.0 * np.pi * np.arange(n_minor) / n_minor
    uu, ww = np.meshgrid(u, w, indexing="ij")
    x = (R + r * np.cos(ww)) * np.cos(uu)
    y = (R + r * np.cos(ww)) * np.sin(uu)
    z = r * np.sin(ww)
    v = np.stack([x, y, z], -1).reshape(-1, 3) + np.asarray(center, np.float64)
    i, j = np.meshgrid(np.arange(n_major), np.arange(n_minor), indexing="ij")
    i1 = (i + 1) % n_major
    j1 = (j + 1) % n_minor
    a = i * n_minor + j
    b = i1 * n_minor + j
    c = i1 * n_minor + j1
    d = i * n_minor + j1
    q = np.stack([np.stack([a, b, c], -1), np.stack([a, c, d], -1)], -2)
    return v, q.reshape(-1, 3).astype(np.int32)


def gear_prism(teeth: int, r_outer: float, thickness: float, target_tris: int,
               root_ratio: float = 0.8):
    """Star-profile extrusion: 2*teeth profile corners alternating between the
    outer and root radius, each profile edge subdivided, side walls split into
    layers, caps fan-triangulated from the axis.  Triangle count is close to
    ``target_tris`` (2*P*L side + 2*P caps for P profile points, L layers)."""
    corners = 2 * teeth
    # choose per-edge subdivision s and layer count L so 2P(L+1) ~ target
    s = max(1, int(round(math.sqrt(target_tris / (4.0 * corners)))))
    P = corners * s
    L = max(1, int(round(target_tris / (2.0 * P) - 1.0)))
    ang = 2.0 * np.pi * np.arange(corners) / corners
    rad = np.where(np.arange(corners) % 2 == 0, r_outer, root_ratio * r_outer)
    cx, cy = rad * np.cos(ang), rad * np.sin(ang)
    nx, ny = np.roll(cx, -1), np.roll(cy, -1)
    f = np.arange(s) / s
    px = (cx[:, None] * (1 - f) + nx[:, None] * f).reshape(-1)
    py = (cy[:, None] * (1 - f) + ny[:, None] * f).reshape(-1)
    z = -0.5 * thickness + thickness * np.arange(L + 1) / L
    zz, pp = np.meshgrid(z, np.arange(P), indexing="ij")
    side = np.stack([px[pp], py[pp], zz], -1).reshape(-1, 3)
    k, j = np.meshgrid(np.arange(L), np.arange(P), indexing="ij")
    j1 = (j + 1) % P
    i0 = k * P + j
    i1 = k * P + j1
    i2 = (k + 1) * P + j
    i3 = (k + 1) * P + j1
    walls = np.stack([np.stack([i0, i1, i2], -1), np.stack([i1, i3, i2], -1)], -2).reshape(-1, 3)
    nside = len(side)
    centers = np.array([[0.0, 0.0, -0.5 * thickness], [0.0, 0.0, 0.5 * thickness]])
    v = np.concatenate([side, centers])
    cb, ct = nside, nside + 1
    jj = np.arange(P)
    bot = np.stack([np.full(P, cb), (jj + 1) % P, jj], -1)
    top = np.stack([np.full(P, ct), L * P + jj, L * P + (jj + 1) % P], -1)
    t = np.concatenate([walls, bot, top]).astype(np.int32)
    return v.astype(np.float64), t


def icosphere(subdivisions: int, radius: float = 1.0):
    """Icosahedron with each triangle split into 4, ``subdivisions`` times,
    vertices projected to the sphere: 20 * 4**s triangles."""
    p = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0],
                  [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
                  [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], dtype=np.float64)
    t = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdivisions):
        e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
        es = np.sort(e, axis=1)
        key = es[:, 0] * (len(v) + 1) + es[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (len(v) + 1)
        b = uniq % (len(v) + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        mids = len(v) + inv.reshape(3, -1).T  # (T,3): m01, m12, m20
        v = np.concatenate([v, mid])
        m01, m12, m20 = mids[:, 0], mids[:, 1], mids[:, 2]
        t = np.concatenate([
            np.stack([t[:, 0], m01, m20], -1),
            np.stack([t[:, 1], m12, m01], -1),
            np.stack([t[:, 2], m20, m12], -1),
            np.stack([m01, m12, m20], -1),
        ])
    return v * radius, t.astype(np.int32)


def _real_sph_harm(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Real spherical harmonic of degree l, order m (theta polar, phi azimuth),
    from the associated Legendre function (scipy.special.lpmv)."""
    from scipy.special import lpmv

    am = abs(m)
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    P = lpmv(am, l, np.cos(theta))
    if m > 0:
        return math.sqrt(2.0) * norm * P * np.cos(am * phi)
    if m < 0:
        return math.sqrt(2.0) * norm * P * np.sin(am * phi)
    return norm * P


def perturbed_icosphere(subdivisions=8, radius=0.1, amplitude=0.002, n_terms=8,
                        l_min=1, l_max=6, seed=4):
    """Icosphere with a radial perturbation amplitude * S(dir) / max|S| where S
    is a sum of ``n_terms`` real spherical harmonics with random degree in
    [l_min, l_max], random order and N(0,1) coefficients (seeded)."""
    v, t = icosphere(subdivisions, 1.0)
    rng = np.random.default_rng(seed)
    theta = np.arccos(np.clip(v[:, 2], -1.0, 1.0))
    phi = np.arctan2(v[:, 1], v[:, 0])
    s = np.zeros(len(v))
    for _ in range(n_terms):
        l = int(rng.integers(l_min, l_max + 1))
        m = int(rng.integers(-l, l + 1))
        s += rng.standard_normal() * _real_sph_harm(l, m, theta, phi)
    s /= max(np.abs(s).max(), 1e-30)
    r = radius + amplitude * s
    return v * r[:, None], t


def centroid_quadrature(verts: np.ndarray, tris: np.ndarray, normalize: bool = True):
    """Triangle-centroid quadrature: points = centroids, weights = areas
    (normalised to sum 1 as SDFContactEngine.register_pair does in the
    reference prototype/src/dynamics/contacts_sdf.py:52-62; the centroid rule
    itself is prototype/src/geometry/quadrature.py:32-48)."""
    p = verts[tris]
    x = p.mean(axis=1)
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    area = 0.5 * np.linalg.norm(n, axis=1)
    w = area / area.sum() if normalize and area.sum() > 1e-30 else area
    return x, w


def face_normals(verts: np.ndarray, tris: np.ndarray):
    p = verts[tris]
    n = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    area = 0.5 * np.linalg.norm(n, axis=1)
    return n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-300), area


def surface_points(verts, tris, n, sigma, rng, uniform_offset=False):
    """Points on the surface (triangle chosen by area, uniform barycentric)
    offset along the face normal by N(0, sigma^2), or U(-sigma, sigma) when
    ``uniform_offset`` is set."""
    nrm, area = face_normals(verts, tris)
    prob = area / area.sum()
    idx = rng.choice(len(tris), size=n, p=prob)
    r1 = rng.random(n)
    r2 = rng.random(n)
    s = np.sqrt(r1)
    b0, b1, b2 = 1.0 - s, s * (1.0 - r2), s * r2
    p = verts[tris[idx]]
    x = b0[:, None] * p[:, 0] + b1[:, None] * p[:, 1] + b2[:, None] * p[:, 2]
    off = rng.uniform(-sigma, sigma, n) if uniform_offset else rng.normal(0.0, sigma, n)
    return x + off[:, None] * nrm[idx]


def write_obj(path: str, verts: np.ndarray, tris: np.ndarray) -> None:
    with open(path, "w") as f:
        for p in verts:
            f.write(f"v {p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
        for t in tris:
            f.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


def corner_normals(verts: np.ndarray, tris: np.ndarray, kind: str = "face",
                   crease_degrees: float = 30.0) -> np.ndarray:
    """Per-triangle corner normals (nt, 3, 3) for contact-aware builds
    (CornerNormalTriangleMesh, SdfSurfaceMesh.h:16-21):
      "face"   every corner carries its triangle's unit normal (sharp edges);
      "smooth" area-weighted vertex normals;
      "crease" vertex normals averaged only over incident faces within
               ``crease_degrees`` of the corner's own face (smooth surfaces
               keep their shading, sharp edges stay sharp)."""
    v = np.asarray(verts, np.float64)
    t = np.asarray(tris, np.int64)
    fn, area = face_normals(v, t)
    if kind == "face":
        return np.repeat(fn[:, None, :], 3, axis=1).copy()
    weighted = fn * area[:, None]
    if kind == "smooth":
        acc = np.zeros_like(v)
        for c in range(3):
            np.add.at(acc, t[:, c], weighted)
        vn = acc / np.maximum(np.linalg.norm(acc, axis=1, keepdims=True), 1e-300)
        return vn[t]
    if kind != "crease":
        raise ValueError(f"unknown corner-normal kind {kind!r}")
    cos_c = np.cos(np.deg2rad(crease_degrees))
    incident = [[] for _ in range(len(v))]
    for f in range(len(t)):
        for c in range(3):
            incident[int(t[f, c])].append(f)
    out = np.zeros((len(t), 3, 3))
    for f in range(len(t)):
        for c in range(3):
            acc = np.zeros(3)
            for g in incident[int(t[f, c])]:
                if fn[g] @ fn[f] >= cos_c:
                    acc += weighted[g]
            out[f, c] = acc / max(np.linalg.norm(acc), 1e-300)
    return out


def write_ca_surface(path: str, verts: np.ndarray, tris: np.ndarray, cnormals: np.ndarray,
                     name: str = "body") -> None:
    """A NEXDYN_CONTACT_AWARE_SURFACE 1 file (the format
    loadContactAwareSurfaceFile reads, SdfSurfaceMesh.cpp:157-344), one
    surface, identity transform, 1-based ids."""
    with open(path, "w") as f:
        f.write("NEXDYN_CONTACT_AWARE_SURFACE 1\n")
        f.write(f"surface {name}\n")
        f.write(f"vertices {len(verts)}\n")
        for i, p in enumerate(verts):
            f.write(f"v {i + 1} {p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
        f.write(f"triangles {len(tris)}\n")
        for i, (tri, cn) in enumerate(zip(tris, cnormals)):
            nums = " ".join(f"{x:.17g}" for x in np.asarray(cn).reshape(-1))
            f.write(f"tri {i + 1} {tri[0] + 1} {tri[1] + 1} {tri[2] + 1} {nums}\n")
        f.write("end\n")
