"""The DEM step on the GPU against the reference program itself (oracle/_ref, run in a subprocess).

The step-log counters (contacts, tri_checks, segments, components, loops) must be identical at every
output step; positions, quaternions, velocities and angular velocities must agree to a relative 1e-9
(force laws call pow/cbrt/log, whose last bit differs between CUDA and glibc)."""
import os

import numpy as np
import pytest

from _dem_helpers import (box_tris, out_file, parse_log, parse_state_txt, plane_tris, run_reference, write_binary_stl,
                          write_config)

pytestmark = pytest.mark.gpu

MAT = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}


def _compare_run(tmp_path, glob, particles, walls=(), rtol=1e-9, min_contact_steps=1):
    from zdemx.dem import Scene

    ref_dir = str(tmp_path / "ref")
    cfg = str(tmp_path / "sim.txt")
    g = dict(glob)
    g.update({"output_dir": ref_dir, "vtk_prefix": "p"})
    write_config(cfg, g, particles, walls)
    log = parse_log(run_reference(cfg))
    steps, every = int(glob["steps"]), int(glob["output_interval"])
    sc = Scene(cfg)
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
        for cols, name in ((slice(0, 3), "pos"), (slice(3, 7), "quat"), (slice(7, 10), "vel"), (slice(10, 13), "omega")):
            a, b = st[:, cols], ref[:, cols]
            scale = max(np.max(np.abs(b)), 1e-300)
            err = np.max(np.abs(a - b)) / scale
            assert err <= rtol, f"step {s} {name}: rel err {err}"
    assert contact_steps >= min_contact_steps
    return sc


def test_two_noised_icospheres_config1_like(tmp_path):
    """The two-particle workload's shape: two 320-triangle noised icospheres, 1 mm, 1.9 mm apart, +-0.05 m/s."""
    from zdemx import synth

    rng = np.random.default_rng(1)
    for k in range(2):
        write_binary_stl(str(tmp_path / f"m{k}.stl"), synth.noised_icosphere(2, 1e-3, 0.15, rng))
    parts = [dict(stl=str(tmp_path / "m0.stl"), pos="0 0 0", vel="0.05 0 0", quat="1 0 0 0", omega="0 0 0", scale=1, **MAT),
             dict(stl=str(tmp_path / "m1.stl"), pos="1.9e-3 0 0", vel="-0.05 0 0", quat="1 0 0 0", omega="0 0 0", scale=1,
                  **MAT)]
    _compare_run(tmp_path, {"steps": 120, "dt": 1e-6, "split_contacts": 1, "gravity": "0 0 0", "output_interval": 5},
                 parts, min_contact_steps=5)


def test_walls_plane_and_box(tmp_path):
    """Particles pressed onto a plane wall and into a box wall (compute_wall_contact, wall history)."""
    from zdemx import synth

    rng = np.random.default_rng(3)
    write_binary_stl(str(tmp_path / "p.stl"), synth.noised_icosphere(2, 1e-3, 0.15, rng))
    write_binary_stl(str(tmp_path / "plane.stl"), plane_tris(0.02))
    write_binary_stl(str(tmp_path / "box.stl"), box_tris(0.01, 0.01, 0.002))
    walls = [dict(stl=str(tmp_path / "plane.stl"), pos="0 0 0", quat="1 0 0 0", scale=1, mu=0.4, restitution=0.3),
             dict(stl=str(tmp_path / "box.stl"), pos="0.02 0 0", quat="1 0 0 0", scale=1, mu=0.5, restitution=0.5)]
    parts = [dict(stl=str(tmp_path / "p.stl"), pos="0.001 0.0 0.0009", vel="0.01 0 -0.05", quat="1 0 0 0",
                  omega="0 3 0", scale=1, **MAT),
             dict(stl=str(tmp_path / "p.stl"), pos="0.02 0.0 0.0018", vel="0 0 -0.02",
                  quat="0.9238795325112867 0 0.3826834323650898 0", omega="0 0 0", scale=1, **MAT)]
    _compare_run(tmp_path, {"steps": 200, "dt": 2e-6, "split_contacts": 1, "gravity": "0 0 -9.81",
                            "output_interval": 20}, parts, walls, min_contact_steps=5)


def test_cli_outputs_match_reference_program(tmp_path):
    """zdem_gpu --config writes the same files and log line shape as zdem_cpu."""
    import subprocess

    from zdemx import synth

    rng = np.random.default_rng(4)
    write_binary_stl(str(tmp_path / "m.stl"), synth.noised_icosphere(1, 1e-3, 0.15, rng))
    parts = [dict(stl=str(tmp_path / "m.stl"), pos="0 0 0", vel="0.05 0 0", quat="1 0 0 0", omega="0 0 0", scale=1, **MAT),
             dict(stl=str(tmp_path / "m.stl"), pos="1.9e-3 0 0", vel="-0.05 0 0", quat="1 0 0 0", omega="0 0 0",
                  scale=1, **MAT)]
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for who in ("ref", "gpu"):
        cfg = str(tmp_path / f"{who}.txt")
        write_config(cfg, {"steps": 20, "dt": 1e-6, "gravity": "0 0 0", "output_interval": 10,
                           "output_dir": str(tmp_path / who), "vtk_prefix": "particles"}, parts)
        if who == "ref":
            p = subprocess.run([os.path.join(root, "oracle", "_ref", "zdem_cpu"), "--config", cfg], capture_output=True,
                               text=True, timeout=300)
        else:
            p = subprocess.run([os.path.join(root, "zedm-x_b200", "bin", "zdem_gpu"), "--config", cfg],
                               capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        assert p.stdout.strip().endswith("done")
    for step in (0, 10):
        a = open(out_file(str(tmp_path / "ref"), "particles", step, ".vtk")).read().split("\n")
        b = open(out_file(str(tmp_path / "gpu"), "particles", step, ".vtk")).read().split("\n")
        assert len(a) == len(b)
        for x, y in zip(a, b):
            if x == y:
                continue
            xs, ys = x.split(), y.split()
            assert len(xs) == len(ys)
            np.testing.assert_allclose([float(v) for v in ys], [float(v) for v in xs], rtol=2e-6, atol=1e-12)
        ta = parse_state_txt(out_file(str(tmp_path / "ref"), "particles", step, ".txt"))
        tb = parse_state_txt(out_file(str(tmp_path / "gpu"), "particles", step, ".txt"))
        np.testing.assert_allclose(tb, ta, rtol=0, atol=2e-9)
    # bad arguments and configs fail like the reference
    assert subprocess.run([os.path.join(root, "zedm-x_b200", "bin", "zdem_gpu"), "--bogus"], capture_output=True).returncode == 1
    bad = tmp_path / "bad.txt"
    bad.write_text("steps = 3\n")
    assert subprocess.run([os.path.join(root, "zedm-x_b200", "bin", "zdem_gpu"), "--config", str(bad)],
                          capture_output=True).returncode == 1


def test_lattice_of_216_particles_on_a_plane(tmp_path):
    """More particles than one block of the broad-phase kernels: every candidate pair of the reference's
    O(N^2) loop is found (the step log's tri_checks counts their triangle tests)."""
    from zdemx.workloads import calibration_scene

    cfg = calibration_scene(str(tmp_path / "lat"), n_side=6, seed=9, steps=6, spacing=1.85e-3)
    text = "\n".join(ln for ln in open(cfg).read().splitlines()
                     if not ln.startswith(("force_law", "feng_k", "output_interval", "output_dir")))
    glob = {"output_interval": 2, "output_dir": str(tmp_path / "ref")}
    text = "\n".join(f"{k} = {v}" for k, v in glob.items()) + "\n" + text
    path = str(tmp_path / "lattice.txt")
    open(path, "w").write(text + "\n")
    from zdemx.dem import Scene

    log = parse_log(run_reference(path))
    sc = Scene(path)
    done = 0
    for s in range(0, 6, 2):
        sc.step(s + 1 - done)
        done = s + 1
        info = sc.info()
        got = (info["contacts"], info["tri_checks"], info["segments"], info["comps"], info["loops"])
        assert got == log[s], f"step {s}: gpu {got} reference {log[s]}"
        assert info["pairs"] > 256
    ref = parse_state_txt(out_file(str(tmp_path / "ref"), "cal", 4, ".txt"))
    st = sc.state()[0]
    scale = np.max(np.abs(ref[:, 0:3]))
    assert np.max(np.abs(st[:, 0:3] - ref[:, 0:3])) / scale <= 1e-9
