"""The reference program's two smaller modes on the GPU: the legacy row config (no particle blocks; `n`
particles of `stl` placed `spacing` apart along x, the first two moving with `v0`, `v1`;
src/main.cpp:1916-1934) and the `contact_debug` prints (src/main.cpp:2288-2299, 2436-2444), compared with
the reference program's own output."""
import os
import re
import subprocess

import numpy as np
import pytest

from _dem_helpers import (ROOT, out_file, parse_log, parse_state_txt, plane_tris, run_reference, write_binary_stl,
                          write_config)

pytestmark = pytest.mark.gpu

MAT = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}
ZDEM_GPU = os.path.join(ROOT, "zedm-x_b200", "bin", "zdem_gpu")
ZDEM_CPU = os.path.join(ROOT, "oracle", "_ref", "zdem_cpu")


def test_legacy_row_mode(tmp_path):
    """Three particles from one STL in a row: same step-log counters, states within 1e-9 relative."""
    from zdemx import synth
    from zdemx.dem import Scene

    rng = np.random.default_rng(11)
    stl = str(tmp_path / "m.stl")
    write_binary_stl(stl, synth.noised_icosphere(1, 1e-3, 0.1, rng))
    ref_dir = str(tmp_path / "ref")
    cfg = str(tmp_path / "row.txt")
    steps, every = 60, 5
    write_config(cfg, {"stl": stl, "n": 3, "spacing": 1.85e-3, "v0": "0.05 0 0", "v1": "-0.05 0 0", "steps": steps,
                       "dt": 2e-8, "gravity": "0 0 0", "output_interval": every, "output_dir": ref_dir,
                       "vtk_prefix": "p"}, [])
    log = parse_log(run_reference(cfg))
    sc = Scene(cfg)
    assert sc.info()["particles"] == 3
    done = 0
    contact_steps = 0
    for s in range(0, steps, every):
        sc.step(s + 1 - done)
        done = s + 1
        info = sc.info()
        got = (info["contacts"], info["tri_checks"], info["segments"], info["comps"], info["loops"])
        assert got == log[s], f"step {s}: gpu {got} reference {log[s]}"
        contact_steps += info["contacts"] > 0
        ref = parse_state_txt(out_file(ref_dir, "p", s, ".txt"))
        st = sc.state()[0]
        np.testing.assert_array_equal(st[:, 0:3] == 0, ref[:, 0:3] == 0)
        for cols in (slice(0, 3), slice(3, 7), slice(7, 10), slice(10, 13)):
            scale = max(np.max(np.abs(ref[:, cols])), 1e-300)
            assert np.max(np.abs(st[:, cols] - ref[:, cols])) / scale <= 1e-9
    assert contact_steps >= 3


NUM = r"[-+0-9.eE]+|[-+]?(?:inf|nan)"
FIELD_RE = re.compile(r"(\w+)=((?:%s)(?:,(?:%s))*)" % (NUM, NUM))


def _debug_lines(text):
    return [ln for ln in text.splitlines() if ln.startswith("  contact_debug:") or ln.startswith("  wall_contact:")]


def _fields(line):
    head = line.split(":", 1)[0].strip()
    return head, [(k, [float(x) for x in v.split(",")]) for k, v in FIELD_RE.findall(line)]


def _run(exe, cfg, *extra):
    p = subprocess.run([exe, "--config", cfg, *extra], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr
    return p.stdout


def test_contact_debug_prints_match_reference_program(tmp_path):
    """Two particles on a plane wall, colliding: the contact_debug and wall_contact lines of every step,
    in the same order, with the same indices and the same printed values (6 significant digits; a value
    whose last printed digit rounds differently is allowed a relative 2e-5 of its vector)."""
    from zdemx import synth

    rng = np.random.default_rng(12)
    write_binary_stl(str(tmp_path / "p.stl"), synth.noised_icosphere(1, 1e-3, 0.1, rng))
    write_binary_stl(str(tmp_path / "plane.stl"), plane_tris(0.02))
    walls = [dict(stl=str(tmp_path / "plane.stl"), pos="0 0 0", quat="1 0 0 0", scale=1, mu=0.4, restitution=0.3)]
    parts = [dict(stl=str(tmp_path / "p.stl"), pos="0 0.0 0.00095", vel="0.05 0 -0.01", quat="1 0 0 0",
                  omega="0 2 0", scale=1, **MAT),
             dict(stl=str(tmp_path / "p.stl"), pos="1.75e-3 0.0 0.00096", vel="-0.05 0 -0.01",
                  quat="0.9238795325112867 0 0.3826834323650898 0", omega="0 0 0", scale=1, **MAT)]
    outs = {}
    for who, exe, extra in (("ref", ZDEM_CPU, ()), ("gpu", ZDEM_GPU, ()), ("graph", ZDEM_GPU, ("--graph",))):
        cfg = str(tmp_path / f"{who}.txt")
        write_config(cfg, {"steps": 60, "dt": 1e-6, "gravity": "0 0 -9.81", "output_interval": 20,
                           "contact_debug": 1, "output_dir": str(tmp_path / who), "vtk_prefix": "p"}, parts, walls)
        outs[who] = _run(exe, cfg, *extra)
    ref, gpu = _debug_lines(outs["ref"]), _debug_lines(outs["gpu"])
    assert len(ref) > 20
    assert any(ln.startswith("  contact_debug:") for ln in ref)
    assert any(ln.startswith("  wall_contact:") for ln in ref)
    assert len(gpu) == len(ref)
    for a, b in zip(ref, gpu):
        ha, fa = _fields(a)
        hb, fb = _fields(b)
        assert ha == hb and [k for k, _ in fa] == [k for k, _ in fb], (a, b)
        for (k, va), (_, vb) in zip(fa, fb):
            if k in ("i", "j", "particle", "wall", "tri"):
                assert va == vb, (a, b)
            else:
                va, vb = np.array(va), np.array(vb)
                tol = 2e-5 * max(np.max(np.abs(va)), 1e-300)
                assert np.max(np.abs(va - vb)) <= tol, (k, a, b)
    # the graph runner keeps the plain step when contact_debug is set: identical output
    assert _debug_lines(outs["graph"]) == gpu
    # and the step log is unchanged by the prints
    assert parse_log(outs["gpu"]) == parse_log(outs["ref"])
