"""The rebuild kernel's polyline-mode candidate order (zedm-x_b200/csrc/zdx_pyset.cuh), host build,
against this interpreter itself: the slot order of a CPython set of ints built by adding distinct keys
(polyline.py:288-299, 324)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    out = str(tmp_path_factory.mktemp("pyset") / "pyset_check")
    src = os.path.join(ROOT, "tests", "cpp", "pyset_check.cpp")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "zedm-x_b200", "csrc"), "-o", out, src],
                   check=True, timeout=300)
    return out


def _run(exe, lines):
    p = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    return p.stdout.splitlines()


def test_set_order_matches_cpython(exe):
    rng = np.random.default_rng(17)
    cases = []
    for t in range(2000):
        n = int(rng.integers(0, 500))
        hi = int(rng.choice([8, 40, 300, 5000, 1 << 22]))
        cases.append(list(dict.fromkeys(int(x) for x in rng.integers(0, hi, size=n))))
    cases += [list(range(2000)), list(range(4000, 0, -3)), [k * 1024 for k in range(300)]]
    out = _run(exe, ["S %d %s" % (len(c), " ".join(map(str, c))) for c in cases])
    for c, line in zip(cases, out):
        s = set()
        for k in c:
            s.add(k)
        assert line.split() == ["ok"] + [str(k) for k in s], c[:10]

