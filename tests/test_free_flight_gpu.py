"""Candidate-free steps through the single-block kernel (k_free_flight) give the full step's results bit
for bit: the same states, forces, torques, contact counts, step counters and histories, in the plain and
the graph runner, across the switches between free flight and contact."""
import numpy as np
import pytest

from _dem_helpers import plane_tris, write_binary_stl, write_config

pytestmark = pytest.mark.gpu

MAT = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}


def _compare(cfg, steps, every, graph):
    from zdemx.dem import Scene

    a, b = Scene(cfg), Scene(cfg)
    b.set_free_flight(False)
    free = contact = 0
    for _ in range(steps // every):
        for sc in (a, b):
            (sc.step_graph if graph else sc.step)(every)
        ia, ib = a.info(), b.info()
        assert ia == ib
        sa, sb = a.state(), b.state()
        for x, y in zip(sa, sb):
            np.testing.assert_array_equal(x, y)
        free += ia["pairs"] == 0
        contact += ia["contacts"] > 0
    return free, contact


@pytest.mark.parametrize("graph", [False, True])
def test_two_particles_collide_and_separate(tmp_path, graph):
    """The config-1 pair: in contact for the first few dozen steps, then apart for the rest."""
    from zdemx.workloads import two_particle_scene

    cfg = two_particle_scene(str(tmp_path), seed=1, steps=400)
    free, contact = _compare(cfg, 400, 8, graph)
    assert free >= 30 and contact >= 2


@pytest.mark.parametrize("graph", [False, True])
def test_many_particles_falling_onto_a_plane(tmp_path, graph):
    """96 particles in free fall above a plane wall reach it at different steps; some collide on the way."""
    from zdemx import synth

    rng = np.random.default_rng(31)
    write_binary_stl(str(tmp_path / "p.stl"), synth.noised_icosphere(1, 1e-3, 0.1, rng))
    write_binary_stl(str(tmp_path / "plane.stl"), plane_tris(0.2))
    walls = [dict(stl=str(tmp_path / "plane.stl"), pos="0 0 0", quat="1 0 0 0", scale=1, mu=0.4, restitution=0.3)]
    parts = []
    for k in range(96):
        x, y = (k % 12) * 4e-3, (k // 12) * 4e-3
        z = 1.3e-3 + 2e-4 * (k % 7)
        vel = [0.0, 0.0, -0.5 - 0.05 * (k % 5)]
        if k % 12 == 1:
            vel[0] = -2.0  # towards its neighbour
        parts.append(dict(stl=str(tmp_path / "p.stl"), pos=f"{x!r} {y!r} {z!r}", vel=" ".join(map(repr, vel)),
                          quat="1 0 0 0", omega="0 0 0", scale=1, **MAT))
    cfg = str(tmp_path / "fall.txt")
    write_config(cfg, {"steps": 2000, "dt": 1e-6, "gravity": "0 0 -9.81", "output_interval": 1000,
                       "output_dir": str(tmp_path / "o"), "vtk_prefix": "p"}, parts, walls)
    free, contact = _compare(cfg, 2000, 50, graph)
    assert free >= 3 and contact >= 3
