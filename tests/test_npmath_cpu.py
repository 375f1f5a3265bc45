"""zedm-x_b200/csrc/zdx_npmath.cuh, host build, against numpy itself on this platform: np.dot of two
3-vectors, np.linalg.norm of a 3- and a 4-vector, the row norms of np.linalg.norm(x, axis=1) and np.cross,
bit for bit on 20,000 random vector pairs over many magnitudes."""
import os
import shutil
import subprocess
import struct

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", float(x)))[0]


def test_numpy_arithmetic_matches_numpy(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = str(tmp_path / "npmath_check")
    src = os.path.join(ROOT, "tests", "cpp", "npmath_check.cpp")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "zedm-x_b200", "csrc"),
                    "-o", exe, src], check=True, timeout=300)
    rng = np.random.default_rng(12)
    n = 20000
    A = rng.normal(size=(n, 3)) * 10.0 ** rng.integers(-9, 4, size=(n, 1))
    B = rng.normal(size=(n, 3)) * 10.0 ** rng.integers(-9, 4, size=(n, 1))
    text = "\n".join(" ".join("%016x" % _bits(x) for x in np.r_[A[i], B[i]]) for i in range(n)) + "\n"
    p = subprocess.run([exe], input=text, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    out = p.stdout.split()
    assert len(out) == 7 * n
    row = np.linalg.norm(A, axis=1)
    for i in range(n):
        want = [np.dot(A[i], B[i]), np.linalg.norm(A[i]), np.linalg.norm(np.r_[A[i], B[i, 0]]), row[i],
                *np.cross(A[i], B[i])]
        got = out[7 * i: 7 * i + 7]
        assert got == ["%016x" % _bits(w) for w in want], i


def test_numpy_triangle_stage_matches_oracle_numpy_mode(tmp_path, oracle):
    """The header's triangle stage (transform, tri_normals, plane_from_tri, AABBs, tri_tri in numpy's
    arithmetic) against the oracle's numpy mode, itself bit-exact with polyline.py: the same segments in
    the same order, to the bit, on the polyline fixtures' pairs and on seeded pairs."""
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    from zdemx import synth

    exe = str(tmp_path / "np_segments_check")
    src = os.path.join(ROOT, "tests", "cpp", "np_segments_check.cpp")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "zedm-x_b200", "csrc"),
                    "-o", exe, src], check=True, timeout=300)
    cases = []
    for fx in ("polyline_ref.npz", "polyline_split_ref.npz", "polyline_hard_ref.npz"):
        z = np.load(os.path.join(ROOT, "tests", "golden", fx))
        for ci in range(int(z["ncase"])):
            cases.append((np.asarray(z[f"c{ci}_A"], float), np.asarray(z[f"c{ci}_B"], float), z[f"c{ci}_pose"]))
    rng = np.random.default_rng(13)
    for _ in range(12):
        A = synth.noised_icosphere(int(rng.integers(1, 3)), 1e-3, 0.15, rng)
        B = synth.noised_icosphere(int(rng.integers(1, 3)), 1e-3, 0.15, rng)
        pose = synth.pair_poses(rng, 1, 1e-3, 0.0, 0.2)[0]
        pose[3:7] = synth.random_unit_quat(rng) * rng.uniform(0.5, 2.0)  # not unit: the normalisation counts
        cases.append((A, B, pose))
    lines = []
    for A, B, pose in cases:
        vals = np.r_[A.reshape(-1), B.reshape(-1), pose]
        lines.append("%d %d " % (len(A.reshape(-1, 9)), len(B.reshape(-1, 9))) + " ".join("%016x" % _bits(x) for x in vals))
    p = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    out = p.stdout.splitlines()
    assert len(out) == len(cases)
    total = 0
    for k, ((A, B, pose), line) in enumerate(zip(cases, out)):
        r = oracle.pair(A.reshape(-1, 3, 3), 0.0, 0.0, B.reshape(-1, 3, 3), pose[:7], pose[7:], split=False, mode=2,
                        tol=1e-5)
        f = line.split()
        assert int(f[0]) == r["nseg"], (k, f[0], r["nseg"])
        assert f[1:] == ["%016x" % _bits(x) for x in r["seg"].reshape(-1)], k
        total += r["nseg"]
    assert total > 300


# numpy's evaluation of polyline.py's rebuild expressions (seg_seg_dist2 :227-265, point_segment_dist2_and_t
# :420-431, accumulate_Sn_Gn_from_polyline :193-209, contact_point_xc0 :211-218), with numpy's own calls
def _np_seg_seg_dist2(p1, q1, p2, q2):
    d1, d2, r = q1 - p1, q2 - p2, p1 - p2
    a, e, f = float(np.dot(d1, d1)), float(np.dot(d2, d2)), float(np.dot(d2, r))
    if a <= 1e-12 and e <= 1e-12:
        return float(np.dot(p1 - p2, p1 - p2))
    if a <= 1e-12:
        c = p2 + np.clip(f / e, 0.0, 1.0) * d2
        return float(np.dot(p1 - c, p1 - c))
    if e <= 1e-12:
        c = p1 + np.clip(-np.dot(d1, r) / a, 0.0, 1.0) * d1
        return float(np.dot(c - p2, c - p2))
    b, c = float(np.dot(d1, d2)), float(np.dot(d1, r))
    denom = a * e - b * b
    s = np.clip((b * f - c * e) / denom, 0.0, 1.0) if abs(denom) > 0.0 else 0.0
    t = (b * s + f) / e
    if t < 0.0:
        t, s = 0.0, np.clip(-c / a, 0.0, 1.0)
    elif t > 1.0:
        t, s = 1.0, np.clip((b - c) / a, 0.0, 1.0)
    diff = (p1 + s * d1) - (p2 + t * d2)
    return float(np.dot(diff, diff))


def _np_point_seg(p, a, b):
    ab = b - a
    denom = float(np.dot(ab, ab))
    if denom <= 1e-12:
        return float(np.dot(p - a, p - a)), 0.0
    t = min(1.0, max(0.0, float(np.dot(p - a, ab) / denom)))
    proj = a + t * ab
    return float(np.dot(p - proj, p - proj)), t


def _np_loop(P):
    Sn, Gn = np.zeros(3), np.zeros(3)
    for i in range(len(P)):
        p0, p1 = P[i], P[(i + 1) % len(P)]
        Sn += 0.5 * np.cross(p0, p1)
        dx = p1 - p0
        s = np.dot(p0, p1) + (1.0 / 3.0) * np.dot(dx, dx)
        Gn += -(1.0 / 3.0) * s * dx
    a = float(np.linalg.norm(Sn))
    if a < 1e-14:
        return list(Sn) + list(Gn) + [0.0] * 7
    nA = -Sn / a
    return list(Sn) + list(Gn) + [a] + list(nA) + list(np.cross(nA, Gn) / a)


def test_numpy_rebuild_arithmetic_matches_numpy(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = str(tmp_path / "np_rebuild_check")
    src = os.path.join(ROOT, "tests", "cpp", "np_rebuild_check.cpp")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "zedm-x_b200", "csrc"),
                    "-o", exe, src], check=True, timeout=300)
    rng = np.random.default_rng(14)
    hx = lambda v: " ".join("%016x" % _bits(x) for x in np.ravel(v))
    cmds, want = [], []
    for k in range(6000):
        sc = 10.0 ** rng.integers(-6, 1)
        p1, q1, p2, q2 = (rng.normal(size=3) * sc for _ in range(4))
        if k % 7 == 0:
            q1 = p1 + rng.normal(size=3) * 1e-8  # short segments: the EPS branches
        if k % 11 == 0:
            q2 = p2.copy()
        if k % 13 == 0:
            q2 = p2 + (q1 - p1) * 2.0  # parallel
        cmds.append("D " + hx(np.r_[p1, q1, p2, q2]))
        want.append(["ok", "%016x" % _bits(_np_seg_seg_dist2(p1, q1, p2, q2))])
        cmds.append("P " + hx(np.r_[q1, p2, q2]))
        d, t = _np_point_seg(q1, p2, q2)
        want.append(["ok", "%016x" % _bits(d), "%016x" % _bits(t)])
    for k in range(2000):
        m = int(rng.integers(3, 40))
        ang = np.sort(rng.uniform(0, 2 * np.pi, m))
        P = np.stack([np.cos(ang), np.sin(ang), rng.normal(size=m) * 0.1], 1) * 10.0 ** rng.integers(-5, 0)
        P = P @ np.linalg.qr(rng.normal(size=(3, 3)))[0] + rng.normal(size=3) * 1e-3
        if k % 17 == 0:
            P[:] = P[0]  # a degenerate loop: |Sn| below 1e-14, xc0 None
        cmds.append("L %d " % m + hx(P))
        want.append(["ok"] + ["%016x" % _bits(x) for x in _np_loop(P)])
    p = subprocess.run([exe], input="\n".join(cmds) + "\n", capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    out = p.stdout.splitlines()
    assert len(out) == len(want)
    for k, (line, w) in enumerate(zip(out, want)):
        assert line.split() == w, (k, cmds[k][:60])
