"""Seeded synthetic scenes of the zdem_cpu config grammar (src/main.cpp:1531-1689), written to disk.

pour_scene: 100,000 particles from five templates (three convex hulls of 64 points on a 1 : 0.8 : 0.6
ellipsoid, noised icospheres of subdivision 2 and 3; circumradius 1 mm) on a jittered lattice inside a
closed 12-triangle box, gravity -z, with small random velocities so that collisions start within a few
hundred steps.  100,000 particles of circumradius 1 mm cannot sit inside a 60 x 60 x 120 mm box without
overlapping (the densest packing of their circumspheres holds about 76,000), so the box keeps the
60 x 60 mm floor and is as tall as the lattice needs.

two_particle_scene: two 320-triangle noised icospheres colliding head-on.

calibration_scene: a lattice of 320-triangle noised icospheres resting on a 2-triangle plane, the
feng_min law (a calibration target for k and the restitution).
"""
from __future__ import annotations

import os
import struct

import numpy as np

from . import synth

MATERIAL = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}


def write_binary_stl(path: str, tris) -> None:
    """Binary STL (float32 corners), the format load_stl reads (src/main.cpp:308-371)."""
    tris = np.asarray(tris, np.float64).reshape(-1, 3, 3)
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where(ln > 0, n / np.where(ln > 0, ln, 1.0), n)
    rec = np.zeros(len(tris), dtype=[("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")])
    rec["n"] = n
    rec["v"] = tris.reshape(-1, 9)
    with open(path, "wb") as f:
        f.write(b"zdemx synthetic mesh".ljust(80, b"\0"))
        f.write(struct.pack("<I", len(tris)))
        f.write(rec.tobytes())


def box_tris(sx: float, sy: float, sz: float) -> np.ndarray:
    """Closed axis-aligned box centred at the origin, 12 triangles wound outward."""
    hx, hy, hz = sx / 2, sy / 2, sz / 2
    v = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [hx, hy, hz], [-hx, hy, hz]])
    f = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (2, 3, 7), (2, 7, 6), (0, 4, 7), (0, 7, 3),
         (1, 2, 6), (1, 6, 5)]
    return v[np.array(f)]


def _fmt(v) -> str:
    return " ".join(repr(float(x)) for x in np.atleast_1d(v))


def pour_templates(rng: np.random.Generator, circumradius: float = 1e-3) -> list[np.ndarray]:
    """The five particle templates: three ellipsoid hulls, icospheres of subdivision 2 and 3."""
    noise = 0.15
    out = [synth.ellipsoid_hull(64, (1.0, 0.8, 0.6), circumradius, rng) for _ in range(3)]
    out.append(synth.noised_icosphere(2, circumradius / (1 + noise), noise, rng))
    out.append(synth.noised_icosphere(3, circumradius / (1 + noise), noise, rng))
    return out


def pour_scene(dirpath: str, n: int = 100_000, seed: int = 0, steps: int = 10_000, dt: float = 2e-6,
               spacing: float = 2.02e-3, floor: float = 60e-3, vel_sigma: float = 0.05,
               output_interval: int = 1 << 30) -> str:
    """Writes the templates, the box and the config under dirpath; returns the config path."""
    rng = np.random.default_rng(seed)
    os.makedirs(dirpath, exist_ok=True)
    names = []
    for k, t in enumerate(pour_templates(rng)):
        p = os.path.join(dirpath, f"template{k}.stl")
        write_binary_stl(p, t)
        names.append(p)
    per_row = int(floor // spacing)
    per_layer = per_row * per_row
    layers = (n + per_layer - 1) // per_layer
    height = layers * spacing + 2 * spacing
    box = os.path.join(dirpath, "box.stl")
    write_binary_stl(box, box_tris(floor, floor, height))
    k = np.arange(n)
    ix, iy, iz = k % per_row, (k // per_row) % per_row, k // per_layer
    x0 = -0.5 * (per_row - 1) * spacing
    pos = np.stack([x0 + ix * spacing, x0 + iy * spacing, spacing * 0.55 + iz * spacing], 1)
    pos += rng.uniform(-5e-6, 5e-6, size=pos.shape)
    vel = rng.normal(0.0, vel_sigma, size=(n, 3))
    quat = synth.random_unit_quat(rng, n)
    tmpl = rng.integers(0, len(names), size=n)
    lines = [f"steps = {steps}", f"dt = {dt!r}", "gravity = 0 0 -9.81", "split_contacts = 1",
             f"output_interval = {output_interval}", f"output_dir = {os.path.join(dirpath, 'out')}",
             "vtk_prefix = pour", "wall", f"stl = {box}", f"pos = 0 0 {height / 2!r}", "quat = 1 0 0 0", "scale = 1",
             "mu = 0.5", "restitution = 0.5", "end_wall"]
    mat = [f"{key} = {val}" for key, val in MATERIAL.items()]
    for i in range(n):
        lines += ["particle", f"stl = {names[tmpl[i]]}", f"pos = {_fmt(pos[i])}", f"vel = {_fmt(vel[i])}",
                  f"quat = {_fmt(quat[i])}", "omega = 0 0 0", "scale = 1"] + mat + ["end_particle"]
    cfg = os.path.join(dirpath, "pour.txt")
    with open(cfg, "w") as f:
        f.write("\n".join(lines) + "\n")
    return cfg


def two_particle_scene(dirpath: str, seed: int = 1, steps: int = 2000, dt: float = 1e-6,
                       output_interval: int = 1 << 30) -> str:
    """Two 320-triangle noised icospheres (radius 1 mm), 1.9 mm apart, approaching at 0.05 m/s each."""
    rng = np.random.default_rng(seed)
    os.makedirs(dirpath, exist_ok=True)
    paths = []
    for k in range(2):
        p = os.path.join(dirpath, f"m{k}.stl")
        write_binary_stl(p, synth.noised_icosphere(2, 1e-3, 0.15, rng))
        paths.append(p)
    lines = [f"steps = {steps}", f"dt = {dt!r}", "gravity = 0 0 0", "split_contacts = 1",
             f"output_interval = {output_interval}", f"output_dir = {os.path.join(dirpath, 'out')}", "vtk_prefix = p"]
    mat = [f"{key} = {val}" for key, val in MATERIAL.items()]
    for p, x, v in ((paths[0], "0 0 0", "0.05 0 0"), (paths[1], "0.0019 0 0", "-0.05 0 0")):
        lines += ["particle", f"stl = {p}", f"pos = {x}", f"vel = {v}", "quat = 1 0 0 0", "omega = 0 0 0",
                  "scale = 1"] + mat + ["end_particle"]
    cfg = os.path.join(dirpath, "two.txt")
    with open(cfg, "w") as f:
        f.write("\n".join(lines) + "\n")
    return cfg


def plane_tris(half: float) -> np.ndarray:
    """Two triangles spanning [-half, half]^2 at z = 0, normal +z; their shared edge is the diagonal y = x."""
    h = half
    return np.array([[[-h, -h, 0.0], [h, -h, 0.0], [h, h, 0.0]], [[-h, -h, 0.0], [h, h, 0.0], [-h, h, 0.0]]])


def calibration_scene(dirpath: str, n_side: int = 10, seed: int = 5, steps: int = 2000, dt: float = 2e-6,
                      k: float = 1e7, restitution: float = 0.5, spacing: float = 1.85e-3, vel_sigma: float = 0.02,
                      output_interval: int = 1 << 30) -> str:
    """n_side^3 noised icospheres (320 triangles, circumradius 1 mm) in a lattice resting on a 2-triangle
    plane, the feng_min law with stiffness k; the lattice sits inside one of the plane's triangles (well
    away from the shared diagonal).  Returns the config path."""
    rng = np.random.default_rng(seed)
    os.makedirs(dirpath, exist_ok=True)
    mesh = os.path.join(dirpath, "ico320.stl")
    write_binary_stl(mesh, synth.noised_icosphere(2, 1e-3 / 1.15, 0.15, rng))
    plane = os.path.join(dirpath, "plane.stl")
    write_binary_stl(plane, plane_tris(0.1))
    n = n_side ** 3
    k_ = np.arange(n)
    ix, iy, iz = k_ % n_side, (k_ // n_side) % n_side, k_ // (n_side * n_side)
    pos = np.stack([10e-3 + ix * spacing, -10e-3 - iy * spacing, 0.95e-3 + iz * spacing], 1)
    pos += rng.uniform(-2e-6, 2e-6, size=pos.shape)
    vel = rng.normal(0.0, vel_sigma, size=(n, 3))
    quat = synth.random_unit_quat(rng, n)
    lines = [f"steps = {steps}", f"dt = {dt!r}", "gravity = 0 0 -9.81", "split_contacts = 1",
             "force_law = feng_min", f"feng_k = {k!r}", f"output_interval = {output_interval}",
             f"output_dir = {os.path.join(dirpath, 'out')}", "vtk_prefix = cal", "wall", f"stl = {plane}",
             "pos = 0 0 0", "quat = 1 0 0 0", "scale = 1", "mu = 0.5", "restitution = 0.5", "end_wall"]
    mat = [f"density = {MATERIAL['density']}", f"young = {MATERIAL['young']}", f"poisson = {MATERIAL['poisson']}",
           f"mu = {MATERIAL['mu']}", f"restitution = {restitution!r}"]
    for i in range(n):
        lines += ["particle", f"stl = {mesh}", f"pos = {_fmt(pos[i])}", f"vel = {_fmt(vel[i])}",
                  f"quat = {_fmt(quat[i])}", "omega = 0 0 0", "scale = 1"] + mat + ["end_particle"]
    cfg = os.path.join(dirpath, "calibration.txt")
    with open(cfg, "w") as f:
        f.write("\n".join(lines) + "\n")
    return cfg


def independent_pair_library(n_pairs: int, seed: int, radius: float = 1e-3, noise: float = 0.15,
                             threads: int | None = None, out_tris=None):
    """The pair sweep with every pair's two meshes its own: 2 n_pairs seeded noised icospheres, each
    subdivision drawn from U{1..4}, built with build_mesh (zdx_mesh_build) on `threads` host threads.

    Meshes are numbered level by level (pair sides of subdivision 1 first), so a pair's two meshes are
    two distinct ids.  `out_tris`, if given, is a float64 array of shape (T, 9) (T = the total triangle
    count, from ``independent_pair_sizes``) that receives the built triangles, e.g. a pinned host
    buffer.  Returns (MeshLibrary, pair_mesh (n_pairs, 2) int32)."""
    import ctypes as C
    from concurrent.futures import ThreadPoolExecutor

    from . import _lib
    from .contact import MeshLibrary

    side_level, off, pm = independent_pair_sizes(n_pairs, seed)
    n_mesh = 2 * n_pairs
    tris = out_tris if out_tris is not None else np.empty((int(off[-1]), 9))
    if tris.shape != (int(off[-1]), 9) or tris.dtype != np.float64 or not tris.flags.c_contiguous:
        raise ValueError("out_tris must be a C-contiguous float64 (T, 9) array")
    props = np.empty((n_mesh, 17))
    L = _lib.lib()
    dp = C.POINTER(C.c_double)
    chunks = []
    for lvl in (1, 2, 3, 4):
        ids = np.nonzero(side_level == lvl)[0]
        for a in range(0, len(ids), 256):
            chunks.append((lvl, int(ids[a]), min(len(ids), a + 256) - a))

    def work(ci):
        lvl, m0, cnt = chunks[ci]
        raw = np.ascontiguousarray(synth.noised_icospheres(lvl, cnt, radius, noise, np.random.default_rng([seed, ci])))
        nt = 20 * 4 ** lvl
        for k in range(cnt):
            m = m0 + k
            _lib.check(L.zdx_mesh_build(raw[k].ctypes.data_as(dp), nt, 1, tris[off[m]:off[m + 1]].ctypes.data_as(dp),
                                        props[m].ctypes.data_as(dp)))

    with ThreadPoolExecutor(threads or os.cpu_count() or 1) as ex:
        list(ex.map(work, range(len(chunks))))
    return MeshLibrary(tris, off, props[:, 5].copy(), props[:, 6].copy(), props), pm


def independent_pair_sizes(n_pairs: int, seed: int):
    """Subdivision level of every mesh (level-major numbering), the triangle offsets and the pairs' mesh
    ids of ``independent_pair_library``."""
    rng = np.random.default_rng([seed, 0x1D])
    lv = rng.integers(1, 5, size=(n_pairs, 2))
    order = np.argsort(lv.ravel(), kind="stable")
    side_level = lv.ravel()[order]
    mesh_of_side = np.empty(2 * n_pairs, np.int64)
    mesh_of_side[order] = np.arange(2 * n_pairs)
    ntri = (20 * 4 ** side_level).astype(np.int64)
    off = np.zeros(2 * n_pairs + 1, np.int64)
    off[1:] = np.cumsum(ntri)
    return side_level, off, mesh_of_side.reshape(n_pairs, 2).astype(np.int32)
