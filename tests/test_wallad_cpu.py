"""The particle-wall contact and its hand-written reverse mode (zedm-x_b200/csrc/zdx_wallad.cuh), built for
the host: the section, clip, area and centroid against the oracle's compute_wall_contact (itself pinned
to the reference, tests/test_oracle_pin.py) bit for bit, and the adjoint of the force, torque and history
against central differences of the same forward, for particles over a two-triangle plane wall (sections
inside one triangle and sections that the diagonal clips) and a box corner (several triangles in a row
sharing the tangential history)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = str(tmp_path / "wallad_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "zedm-x_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "cpp", "wallad_check.cpp")], check=True, timeout=300)
    return exe


def _fmt(a):
    return " ".join(repr(float(x)) for x in np.ravel(a))


def _quat(rng):
    q = rng.normal(size=4)
    return q / np.linalg.norm(q) * rng.uniform(0.9, 1.1)  # not quite unit: the normalisation is differentiated


def _run(exe, mesh, wall, items, steps):
    lines = [str(len(mesh)), _fmt(mesh), str(len(wall)), _fmt(wall), str(len(items)), _fmt(steps)]
    lines += [_fmt(it) for it in items]
    p = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    out = p.stdout.split("\n")
    normals = np.array([float(x) for x in out[0].split()[1:]]).reshape(-1, 3)
    recs = []
    for k in range(len(items)):
        g, f, a, d = (out[1 + 4 * k + j].split() for j in range(4))
        recs.append({"G": g[1:], "F": np.array([float(x) for x in f[1:10]]), "Fi": [int(x) for x in f[10:13]],
                     "A": np.array([float(x) for x in a[1:18]]), "Ast": int(a[18]),
                     "D": np.array([float(x) for x in d[1:18]]), "Dst": int(d[18])})
    return normals, recs


def _mesh(rng):
    from zdemx import synth

    t = synth.noised_icosphere(2, 1e-3, 0.15, rng)
    c = t.reshape(-1, 3).mean(0)
    return (t - c).reshape(-1, 9)


MAT = [5.0e-6, 2.0e5, 1.2e-3, 1.0e-3, 1e7, 0.25, 0.5, 0.5, 0, 0, 0, 0, 0, 0, 0, 0, 0]  # mass, 1/m, r, R_eq, E, nu, mu, e


def _items(rng, centers):
    items = []
    for c in centers:
        x = np.asarray(c, float)
        q = _quat(rng)
        v = rng.normal(size=3) * 0.05
        w = rng.normal(size=3) * 20.0
        ds = rng.normal(size=3) * 1e-7
        e = rng.uniform(0.2, 0.8)
        g = rng.normal(size=9)
        g[0:3] *= 1e3
        g[3:6] *= 1e6
        g[6:9] *= 1e9
        items.append(np.r_[x, q, v, w, MAT, 1.8e-5, 0.4, ds, e, 2e-6, g])
    return items


STEPS = [1e-10, 1e-8, 1e-7, 1e-5, 1e-12, 1e-7]  # x, q, v, w, ds, e


def _check(exe, mesh, wall, items, oracle):
    normals, recs = _run(exe, mesh, wall, items, STEPS)
    n_contact = n_checked = 0
    for it, r in zip(items, recs):
        # geometry of each wall triangle against the oracle, bit for bit
        g = r["G"]
        for j in range(0, len(g), 6):
            t, ok = int(g[j]), int(g[j + 1])
            area, cp = float(g[j + 2]), np.array([float(x) for x in g[j + 3: j + 6]])
            ook, oarea, ocp, _ = oracle.wall_contact(mesh, it[0:7], wall[t], normals[t], it[15], it[30])
            assert ok == int(ook), (t, ok, ook)
            if ok:
                n_contact += 1
                assert area == oarea and np.array_equal(cp, ocp), (t, area, oarea, cp, ocp)
        assert r["Fi"][2] == 0 and r["Ast"] == 0
        if not r["Fi"][0] or r["Dst"]:
            continue
        # adjoint against central differences, per input group, relative to the group's scale
        n_checked += 1
        A, D = r["A"], r["D"]
        for name, sl in (("x", slice(0, 3)), ("q", slice(3, 7)), ("v", slice(7, 10)), ("w", slice(10, 13)),
                         ("ds", slice(13, 16)), ("e", slice(16, 17))):
            scale = max(np.max(np.abs(D[sl])), np.max(np.abs(A[sl])), 1e-300)
            err = np.max(np.abs(A[sl] - D[sl])) / scale
            assert err < 2e-5, (name, A[sl], D[sl], err)
    return n_contact, n_checked


def test_plane_wall_sections_and_adjoint(tmp_path, oracle):
    exe = _build(tmp_path)
    rng = np.random.default_rng(21)
    mesh = _mesh(rng)
    s = 5e-3
    wall = np.array([[-s, -s, 0, s, -s, 0, s, s, 0], [-s, -s, 0, s, s, 0, -s, s, 0]], float)
    centers = [[rng.uniform(-3e-3, 3e-3), rng.uniform(-3e-3, 3e-3), rng.uniform(0.75e-3, 0.95e-3)] for _ in range(12)]
    # near the diagonal x = y, where the section is clipped by both triangles
    centers += [[d, d + rng.uniform(-2e-4, 2e-4), rng.uniform(0.7e-3, 0.9e-3)] for d in rng.uniform(-2e-3, 2e-3, 12)]
    n_contact, n_checked = _check(exe, mesh, wall, _items(rng, centers), oracle)
    assert n_contact >= 20 and n_checked >= 15


def test_box_corner_shares_the_history(tmp_path, oracle):
    exe = _build(tmp_path)
    rng = np.random.default_rng(22)
    mesh = _mesh(rng)
    s = 4e-3
    # floor z = 0 and wall x = 0, two triangles each, the wall's triangles in a row
    wall = np.array([[0, 0, 0, s, 0, 0, s, s, 0], [0, 0, 0, s, s, 0, 0, s, 0],
                     [0, 0, 0, 0, s, 0, 0, s, s], [0, 0, 0, 0, s, s, 0, 0, s]], float)
    centers = [[rng.uniform(0.7e-3, 0.95e-3), rng.uniform(1e-3, 3e-3), rng.uniform(0.7e-3, 0.95e-3)] for _ in range(16)]
    n_contact, n_checked = _check(exe, mesh, wall, _items(rng, centers), oracle)
    assert n_contact >= 16 and n_checked >= 10
