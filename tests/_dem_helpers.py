"""Helpers for the DEM tests: write STL and config files, run the reference program, parse its outputs."""
from __future__ import annotations

import os
import re
import struct
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write_binary_stl(path, tris):
    tris = np.asarray(tris, float).reshape(-1, 3, 3)
    with open(path, "wb") as f:
        f.write(b"zdemx test mesh".ljust(80, b"\0"))
        f.write(struct.pack("<I", len(tris)))
        for t in tris:
            n = np.cross(t[1] - t[0], t[2] - t[0])
            ln = np.linalg.norm(n)
            n = n / ln if ln > 0 else n
            f.write(struct.pack("<3f", *n))
            f.write(struct.pack("<9f", *t.reshape(-1)))
            f.write(struct.pack("<H", 0))


def plane_tris(size):
    h = size / 2.0
    v = np.array([[-h, -h, 0.0], [h, -h, 0.0], [h, h, 0.0], [-h, h, 0.0]])
    return np.array([[v[0], v[1], v[2]], [v[0], v[2], v[3]]])


def box_tris(sx, sy, sz):
    hx, hy, hz = sx / 2, sy / 2, sz / 2
    v = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [hx, hy, -hz], [-hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [hx, hy, hz], [-hx, hy, hz]])
    f = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (2, 3, 7), (2, 7, 6), (0, 4, 7), (0, 7, 3),
         (1, 2, 6), (1, 6, 5)]
    return v[np.array(f)]


def fmt(v):
    return " ".join(repr(float(x)) for x in np.atleast_1d(v))


def write_config(path, glob: dict, particles: list, walls: list = ()):
    lines = [f"{k} = {v}" for k, v in glob.items()]
    for w in walls:
        lines.append("wall")
        lines += [f"{k} = {v}" for k, v in w.items()]
        lines.append("end_wall")
    for p in particles:
        lines.append("particle")
        lines += [f"{k} = {v}" for k, v in p.items()]
        lines.append("end_particle")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def run_reference(config_path, hiprec=True, timeout=600):
    """Run the reference program (oracle/_ref) on a config; returns its stdout."""
    from oracle import LIB_REF, LIB_REF_HIPREC

    lib = LIB_REF_HIPREC if hiprec else LIB_REF
    code = ("import sys; sys.path.insert(0, %r); from oracle import Reference; "
            "import ctypes; r = Reference(%r); rc = r.main(['--config', %r]); "
            "ctypes.CDLL(None).fflush(None); sys.exit(rc)") % (os.path.join(ROOT, "oracle"), lib, config_path)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=timeout)
    assert p.returncode == 0, p.stderr
    return p.stdout


LOG_RE = re.compile(r"step=(\d+) contacts=(\d+) step_ms=\d+ tri_ms=\d+ rebuild_ms=\d+ output_ms=\d+ tri_checks=(\d+) "
                    r"segments=(\d+) comps=(\d+) loops=(\d+)")


def parse_log(text):
    """{step: (contacts, tri_checks, segments, comps, loops)} from the step log lines."""
    out = {}
    for m in LOG_RE.finditer(text):
        out[int(m.group(1))] = tuple(int(m.group(k)) for k in range(2, 7))
    return out


def parse_state_txt(path):
    """(np, 16) pos quat vel omega (L unknown -> 0) from a state txt file (either precision)."""
    rows = []
    cur = {}
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line == "particle":
                cur = {}
            elif line == "end_particle":
                rows.append(np.r_[cur["pos"], cur["quat"], cur["vel"], cur["omega"], 0.0, 0.0, 0.0])
            elif "=" in line:
                k, v = line.split("=", 1)
                k = k.strip()
                if k in ("pos", "quat", "vel", "omega"):
                    cur[k] = np.array([float(x) for x in v.split()])
    return np.asarray(rows)


def out_file(dirname, prefix, step, ext):
    return os.path.join(dirname, f"{prefix}_{step:06d}{ext}")
