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
