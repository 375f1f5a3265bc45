"""The DEM step captured in a CUDA graph (zdx_scene_step_graph) against the plain step (zdx_scene_step,
itself checked against the reference program in test_dem_gpu.py): state, forces and the step log's
counters identical bit for bit, including after capacity overflows that make it grow and capture
again, and when plain and graph steps alternate (the tangential history moves between them)."""
import os
import subprocess

import numpy as np
import pytest

from _dem_helpers import box_tris, fmt, out_file, parse_state_txt, plane_tris, write_binary_stl, write_config

pytestmark = pytest.mark.gpu

MAT = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}
COUNTERS = ("contacts", "tri_checks", "segments", "comps", "loops", "pairs", "wall_contacts")


def _cluster_config(tmp_path, n=8, walls=True, seed=2):
    from zdemx import synth

    rng = np.random.default_rng(seed)
    write_binary_stl(str(tmp_path / "a.stl"), synth.noised_icosphere(1, 1e-3, 0.15, rng))
    write_binary_stl(str(tmp_path / "b.stl"), synth.noised_icosphere(2, 1e-3, 0.1, rng))
    write_binary_stl(str(tmp_path / "plane.stl"), plane_tris(0.05))
    write_binary_stl(str(tmp_path / "box.stl"), box_tris(0.012, 0.012, 0.012))
    parts = []
    for i in range(n):
        pos = np.array([(i % 2) * 1.85e-3, ((i // 2) % 2) * 1.85e-3, 1.05e-3 + (i // 4) * 1.85e-3])
        pos += rng.uniform(-5e-5, 5e-5, 3)
        parts.append(dict(stl=str(tmp_path / ("a.stl" if i % 3 else "b.stl")), pos=fmt(pos),
                          vel=fmt(rng.normal(size=3) * 0.02), quat=fmt(synth.random_unit_quat(rng)),
                          omega=fmt(rng.normal(size=3) * 5.0), scale=1, **MAT))
    wl = []
    if walls:
        wl = [dict(stl=str(tmp_path / "plane.stl"), pos="0 0 0", quat="1 0 0 0", scale=1, mu=0.4, restitution=0.3),
              dict(stl=str(tmp_path / "box.stl"), pos="0.001 0.001 0.004", quat="1 0 0 0", scale=1, mu=0.5,
                   restitution=0.5)]
    cfg = str(tmp_path / "sim.txt")
    write_config(cfg, {"steps": 100, "dt": 2e-6, "split_contacts": 1, "gravity": "0 0 -9.81", "output_interval": 10,
                       "output_dir": str(tmp_path / "out"), "vtk_prefix": "p"}, parts, wl)
    return cfg


def _same(a, b, what):
    sa, fa, ta, ca = a.state()
    sb, fb, tb, cb = b.state()
    for x, y, name in ((sa, sb, "state"), (fa, fb, "force"), (ta, tb, "torque"), (ca, cb, "contact_count")):
        assert np.array_equal(x, y), f"{what}: {name} differs (max {np.max(np.abs(x - y))})"
    ia, ib = a.info(), b.info()
    for k in COUNTERS + ("steps", "history", "wall_history"):
        assert ia[k] == ib[k], f"{what}: {k} plain {ia[k]} graph {ib[k]}"


@pytest.mark.parametrize("reserve", [None, (1, 1, 16, 8)])
def test_graph_step_matches_plain_step(tmp_path, reserve):
    from zdemx.dem import Scene

    cfg = _cluster_config(tmp_path)
    plain, graph = Scene(cfg), Scene(cfg)
    if reserve:
        graph.graph_reserve(*reserve)  # tiny capacities: every kind of overflow, growth, capture again
    seen_contacts = 0
    for chunk in (1, 4, 10, 25, 20):
        plain.step(chunk)
        graph.step_graph(chunk)
        _same(plain, graph, f"after {plain.info()['steps']} steps")
        seen_contacts += plain.info()["contacts"]
    assert seen_contacts > 0


def test_plain_and_graph_steps_alternate(tmp_path):
    from zdemx.dem import Scene

    cfg = _cluster_config(tmp_path, seed=2)
    ref, mix = Scene(cfg), Scene(cfg)
    carried = 0
    for k, n in enumerate((3, 7, 13, 5, 20, 15, 9)):
        ref.step(n)
        (mix.step if k % 2 else mix.step_graph)(n)
        _same(ref, mix, f"alternating, after {ref.info()['steps']} steps")
        carried += ref.info()["history"] + ref.info()["wall_history"]
    assert carried > 0, "no tangential history crossed a switch"


def test_zdem_gpu_graph_flag_writes_the_same_files(tmp_path):
    cfg = _cluster_config(tmp_path, n=4, seed=7)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "zedm-x_b200", "bin", "zdem_gpu")
    outs = {}
    for mode in ("plain", "graph"):
        text = open(cfg).read().replace(str(tmp_path / "out"), str(tmp_path / mode))
        c = str(tmp_path / f"{mode}.txt")
        open(c, "w").write(text)
        args = [exe, "--config", c] + (["--graph"] if mode == "graph" else [])
        p = subprocess.run(args, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        outs[mode] = [ln.split(" step_ms")[0] + " " + ln.split("output_ms=")[1].split(" ", 1)[1]
                      for ln in p.stdout.splitlines() if ln.startswith("step=")]
    assert outs["plain"] == outs["graph"]
    for step in range(0, 100, 10):
        a = parse_state_txt(out_file(str(tmp_path / "plain"), "p", step, ".txt"))
        b = parse_state_txt(out_file(str(tmp_path / "graph"), "p", step, ".txt"))
        assert np.array_equal(a, b)


def test_graph_step_matches_plain_step_with_many_particles(tmp_path):
    """216 particles: more than one block of every per-particle kernel, on both step forms."""
    from zdemx.dem import Scene
    from zdemx.workloads import calibration_scene

    cfg = calibration_scene(str(tmp_path / "lat"), n_side=6, seed=9, steps=40, spacing=1.85e-3)
    plain, graph = Scene(cfg), Scene(cfg)
    for chunk in (1, 9, 30):
        plain.step(chunk)
        graph.step_graph(chunk)
        _same(plain, graph, f"after {plain.info()['steps']} steps")
    assert plain.info()["pairs"] > 256
