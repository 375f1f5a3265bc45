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
