"""Asynchronous outputs (zdx_scene_write_output_async): the files written from a device snapshot on a
writer thread, while later steps run, are byte-identical to the synchronous writer's for the same step."""
import filecmp
import os

import numpy as np
import pytest

from _dem_helpers import out_file, plane_tris, write_binary_stl, write_config

pytestmark = pytest.mark.gpu

MAT = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}


def _scene_cfg(tmp_path, outdir, name, n=27):
    from zdemx import synth

    rng = np.random.default_rng(21)
    write_binary_stl(str(tmp_path / "p.stl"), synth.noised_icosphere(1, 1e-3, 0.1, rng))
    write_binary_stl(str(tmp_path / "plane.stl"), plane_tris(0.05))
    walls = [dict(stl=str(tmp_path / "plane.stl"), pos="0 0 0", quat="1 0 0 0", scale=1, mu=0.4, restitution=0.3)]
    parts = []
    for k in range(n):
        x, y, z = k % 3, (k // 3) % 3, k // 9
        pos = np.array([x * 1.9e-3, y * 1.9e-3, 0.00097 + z * 1.9e-3]) + rng.uniform(-2e-5, 2e-5, 3)
        parts.append(dict(stl=str(tmp_path / "p.stl"), pos=" ".join(map(repr, pos)),
                          vel=" ".join(map(repr, rng.normal(size=3) * 0.01)), quat="1 0 0 0", omega="0 0 0", scale=1,
                          **MAT))
    cfg = str(tmp_path / f"{name}.txt")
    write_config(cfg, {"steps": 40, "dt": 1e-6, "gravity": "0 0 -9.81", "output_interval": 10, "output_dir": outdir,
                       "vtk_prefix": "p"}, parts, walls)
    return cfg


def test_async_outputs_equal_sync_outputs(tmp_path):
    """Two scenes from one config step identically; one writes synchronously after each batch of steps,
    the other queues its outputs and keeps stepping before they are written."""
    from zdemx.dem import Scene

    a_dir, b_dir = str(tmp_path / "sync"), str(tmp_path / "async")
    sa = Scene(_scene_cfg(tmp_path, a_dir, "a"))
    sb = Scene(_scene_cfg(tmp_path, b_dir, "b"))
    steps = []
    sb.write_output(0, wait=False)  # before any step: zero forces and counts
    sa.write_output(0)
    steps.append(0)
    for k in range(6):
        sa.step(3)
        sb.step(3)
        step = 3 * (k + 1)
        steps.append(step)
        sa.write_output(step)
        sb.write_output(step, wait=False)
    sb.output_wait()
    for step in steps:
        for ext in (".vtk", ".txt"):
            a, b = out_file(a_dir, "p", step, ext), out_file(b_dir, "p", step, ext)
            assert os.path.getsize(a) > 0
            assert filecmp.cmp(a, b, shallow=False), (step, ext)
    assert sa.info()["contacts"] > 0


def test_async_outputs_while_stepping_in_graph_mode(tmp_path):
    """run_config's plain and graph runners queue their outputs; both give the same files."""
    from zdemx.dem import run_config

    for who in ("plain", "graph"):
        cfg = _scene_cfg(tmp_path, str(tmp_path / who / "out"), who)
        assert run_config(cfg, graph=(who == "graph")) == 0
    for step in (0, 10, 20, 30):
        for ext in (".vtk", ".txt"):
            a = out_file(str(tmp_path / "plain" / "out"), "p", step, ext)
            b = out_file(str(tmp_path / "graph" / "out"), "p", step, ext)
            assert filecmp.cmp(a, b, shallow=False), (step, ext)
