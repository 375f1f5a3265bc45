"""The particle-particle force law and its hand-written reverse mode (zedm-x_b200/csrc/zdx_ppad.cuh),
built for the host: the gradient of the pair's force, torques and history with respect to both
particles' states, the history in, k, e and every contact's point, normal and area, against central
differences, for both laws (zdem and feng_min), pairs of one to four contacts sharing the history, in
the sliding (Coulomb-capped) and sticking regimes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = str(tmp_path / "ppad_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "zedm-x_b200", "csrc"),
                    "-o", exe, os.path.join(ROOT, "tests", "cpp", "ppad_check.cpp")], check=True, timeout=300)
    return exe


MAT = [5.0e-6, 2.0e5, 1.2e-3, 1.0e-3, 1e7, 0.25, 0.5, 0.5] + [0.0] * 9


def _item(rng, law, nc, sliding):
    xa = rng.normal(size=3) * 1e-3
    xb = xa + np.array([1.9e-3, 0, 0]) + rng.normal(size=3) * 1e-5
    v = rng.normal(size=(4, 3)) * [[0.05], [0.05], [30.0], [30.0]]
    ds = rng.normal(size=3) * (1e-5 if sliding else 1e-9)
    vals = [law, 1.3e7, rng.uniform(0.2, 0.8), 2e-6, *xa, *xb, *v.ravel(), *ds, *MAT, *MAT, nc]
    for _ in range(nc):
        xc = (xa + xb) / 2 + rng.normal(size=3) * 1e-4
        n = np.array([1.0, 0, 0]) + rng.normal(size=3) * 0.1
        n /= np.linalg.norm(n)
        vals += [*xc, *n, rng.uniform(1e-8, 1e-7)]
    g = rng.normal(size=12) * np.repeat([1.0, 1e3, 1e3, 1e6], 3)
    return vals + list(g)


def test_pair_force_adjoint_against_central_differences(tmp_path):
    exe = _build(tmp_path)
    rng = np.random.default_rng(41)
    items = [_item(rng, law, nc, sl) for law in (0, 1) for nc in (1, 2, 4) for sl in (False, True) for _ in range(2)]
    text = f"{len(items)}\n" + "\n".join(" ".join(repr(float(x)) for x in it) for it in items) + "\n"
    p = subprocess.run([exe], input=text, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = p.stdout.strip().split("\n")
    assert len(lines) == 3 * len(items)
    groups = [("xa", 0, 3), ("xb", 3, 6), ("va", 6, 9), ("vb", 9, 12), ("wa", 12, 15), ("wb", 15, 18),
              ("ds", 18, 21), ("k", 21, 22), ("e", 22, 23)]
    for i, it in enumerate(items):
        A = np.array([float(x) for x in lines[3 * i + 1].split()[1:]])
        D = np.array([float(x) for x in lines[3 * i + 2].split()[1:]])
        nc = int(it[4 + 21 + 34])
        gl = groups + [(f"c{q}{nm}", 23 + 7 * q + a, 23 + 7 * q + b) for q in range(nc)
                       for nm, a, b in (("x", 0, 3), ("n", 3, 6), ("A", 6, 7))]
        for name, a, b in gl:
            scale = max(np.max(np.abs(D[a:b])), np.max(np.abs(A[a:b])))
            if scale == 0.0:
                continue  # k under the zdem law
            err = np.max(np.abs(A[a:b] - D[a:b])) / scale
            assert err < 1e-5, (i, name, A[a:b], D[a:b], err)
