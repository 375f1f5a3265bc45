"""Seeded synthetic inputs: noised icospheres, ellipsoid hulls and pair poses.

The reference ships only six STL files and no generator for its benchmark shapes, so the workloads
(two-particle contact, the mixed-size pair sweep, the adjoint pairs, the pour) are built here from a
seed.  An icosphere at subdivision s has 20*4**s triangles; "noised" scales every vertex radius by
1 + U(-noise, noise), which makes the surface concave in places.  Triangles are wound counter-clockwise
seen from outside, like the wall STLs of geometry/create_wall.py.
"""
from __future__ import annotations

import numpy as np

_PHI = (1.0 + 5.0 ** 0.5) / 2.0


def icosphere(subdiv: int):
    """Unit icosphere: (vertices (V,3), faces (F,3) int) with F = 20*4**subdiv."""
    v = [(-1, _PHI, 0), (1, _PHI, 0), (-1, -_PHI, 0), (1, -_PHI, 0),
         (0, -1, _PHI), (0, 1, _PHI), (0, -1, -_PHI), (0, 1, -_PHI),
         (_PHI, 0, -1), (_PHI, 0, 1), (-_PHI, 0, -1), (-_PHI, 0, 1)]
    verts = [np.asarray(p, float) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.asarray(verts, float), np.asarray(faces, np.int64)


_ICO_CACHE: dict = {}


def _ico(subdiv):
    if subdiv not in _ICO_CACHE:
        _ICO_CACHE[subdiv] = icosphere(subdiv)
    return _ICO_CACHE[subdiv]


def noised_icosphere(subdiv: int, radius: float, noise: float, rng: np.random.Generator) -> np.ndarray:
    """Triangle soup (F,3,3) float64 of an icosphere whose vertex radii are scaled by 1+U(-noise,noise)."""
    verts, faces = _ico(subdiv)
    scale = 1.0 + rng.uniform(-noise, noise, size=len(verts))
    vv = verts * (radius * scale)[:, None]
    return vv[faces]


def noised_icospheres(subdiv: int, count: int, radius: float, noise: float, rng: np.random.Generator) -> np.ndarray:
    """`count` independent noised icospheres of one subdivision, (count,F,3,3)."""
    verts, faces = _ico(subdiv)
    scale = 1.0 + rng.uniform(-noise, noise, size=(count, len(verts)))
    vv = verts[None, :, :] * (radius * scale)[:, :, None]
    return vv[:, faces]


def convex_hull_tris(points: np.ndarray) -> np.ndarray:
    """Triangle soup of the convex hull of `points`, wound outward (scipy's Qhull does the hull)."""
    from scipy.spatial import ConvexHull

    hull = ConvexHull(points)
    tris = points[hull.simplices]
    c = points.mean(axis=0)
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    flip = np.einsum("ij,ij->i", n, tris[:, 0] - c) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return np.ascontiguousarray(tris)


def ellipsoid_hull(npts: int, axes, circumradius: float, rng: np.random.Generator) -> np.ndarray:
    """Convex hull of `npts` random points on an ellipsoid with the given axis ratios."""
    d = rng.normal(size=(npts, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    p = d * np.asarray(axes, float)[None, :]
    p *= circumradius / np.max(np.linalg.norm(p, axis=1))
    return convex_hull_tris(p)


def random_unit_quat(rng: np.random.Generator, n: int | None = None) -> np.ndarray:
    """Uniform random unit quaternion(s), (w, x, y, z)."""
    q = rng.normal(size=(4,) if n is None else (n, 4))
    return q / np.linalg.norm(q, axis=-1, keepdims=True)


def random_dirs(rng: np.random.Generator, n: int) -> np.ndarray:
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def pair_poses(rng: np.random.Generator, n: int, radius: float, depth_lo: float, depth_hi: float) -> np.ndarray:
    """Poses (n, 14) = posA(3) quatA(4) posB(3) quatB(4) for overlapping pairs.

    A sits at the origin with the identity rotation; B gets a random rotation and is moved along a
    random direction so that the nominal overlap depth is U(depth_lo, depth_hi) * radius."""
    poses = np.zeros((n, 14))
    poses[:, 3] = 1.0
    depth = rng.uniform(depth_lo, depth_hi, size=n) * radius
    poses[:, 7:10] = random_dirs(rng, n) * (2.0 * radius - depth)[:, None]
    poses[:, 10:14] = random_unit_quat(rng, n)
    return poses
