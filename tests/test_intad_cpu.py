"""integrate_particle and its hand-written reverse mode (zedm-x_b200/csrc/zdx_intad.cuh), built for the
host: the forward against a numpy restatement of the step's integration (src/main.cpp:1494-1510), and the
gradient of a random linear functional of the new state with respect to position, quaternion (not of
unit length), velocity, angular momentum, force and torque against central differences."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = str(tmp_path / "intad_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "zedm-x_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "cpp", "intad_check.cpp")], check=True, timeout=300)
    return exe


def _rotmat(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _qmul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw])


def _np_step(x, q, v, L, F, T, mat, g, dt):
    vel = v + (F * mat[1] + g) * dt
    pos = x + vel * dt
    R = _rotmat(q / np.linalg.norm(q))
    Iinv = R @ mat[8:17].reshape(3, 3) @ R.T
    Ln = L + T * dt
    om = Iinv @ Ln
    q1 = q + 0.5 * _qmul(np.r_[0.0, om], q) * dt
    return np.r_[pos, q1 / np.linalg.norm(q1), vel, om, Ln]


def test_integration_adjoint_against_central_differences(tmp_path):
    exe = _build(tmp_path)
    rng = np.random.default_rng(7)
    items = []
    for i in range(24):
        x = rng.normal(size=3) * 1e-3
        q = rng.normal(size=4)
        q *= rng.uniform(0.5, 2.0) / np.linalg.norm(q)  # stored quaternions drift from unit length
        v = rng.normal(size=3) * 0.1
        L = rng.normal(size=3) * 1e-9
        F = rng.normal(size=3) * 1e-2
        T = rng.normal(size=3) * 1e-5
        A = rng.normal(size=(3, 3))
        Ib = np.linalg.inv(A @ A.T + 3 * np.eye(3)) * 1e7  # symmetric positive definite inverse inertia
        mat = np.r_[1e-5, 1e5, 1e-3, 1e-3, 1e7, 0.25, 0.5, 0.5, Ib.ravel()]
        g = np.array([0.0, 0.0, -9.81])
        dt = [2e-6, 1e-4, 1e-2][i % 3]  # large steps too, so that the rotation terms matter
        gout = rng.normal(size=16) * np.r_[[1e3] * 3, [1.0] * 4, [1.0] * 3, [1e-3] * 3, [1e6] * 3]
        items.append((np.r_[x, q, v, L, F, T], mat, g, dt, gout))
    text = f"{len(items)}\n" + "\n".join(
        " ".join(repr(float(t)) for t in np.r_[a, mat, g, dt, gout]) for a, mat, g, dt, gout in items) + "\n"
    p = subprocess.run([exe], input=text, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = p.stdout.strip().split("\n")
    assert len(lines) == 3 * len(items)
    names = [("x", 0, 3), ("q", 3, 7), ("v", 7, 10), ("L", 10, 13), ("F", 13, 16), ("T", 16, 19)]
    for i, (a, mat, g, dt, gout) in enumerate(items):
        Fo = np.array([float(t) for t in lines[3 * i].split()[1:]])
        want = _np_step(a[0:3], a[3:7], a[7:10], a[10:13], a[13:16], a[16:19], mat, g, dt)
        assert np.allclose(Fo, want, rtol=1e-13, atol=1e-13 * np.abs(want).max()), (i, Fo - want)
        A = np.array([float(t) for t in lines[3 * i + 1].split()[1:]])
        D = np.array([float(t) for t in lines[3 * i + 2].split()[1:]])
        for name, lo, hi in names:
            scale = max(np.abs(A[lo:hi]).max(), np.abs(D[lo:hi]).max())
            assert scale > 0, (i, name)
            err = np.abs(A[lo:hi] - D[lo:hi]).max() / scale
            assert err < 1e-5, (i, name, A[lo:hi], D[lo:hi], err)
