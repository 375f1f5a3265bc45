"""Pins the oracle's DEM step (zo_dem_step in oracle/zdx_oracle.c: broad phase, pair contacts, the
particle and wall force laws with tangential history, the scatter, integration and history prune,
src/main.cpp:2034-2468) to the reference program itself (oracle/_ref, its state writer printing 17
significant digits), on the CPU: the step log's counters at every output step, and positions,
quaternions, velocities and angular velocities bit for bit.  Same scenes as the GPU DEM tests."""
import numpy as np

from _dem_helpers import (box_tris, fmt, out_file, parse_log, parse_state_txt, plane_tris, run_reference,
                          write_binary_stl, write_config)

MAT = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}


def _vec(s):
    return [float(x) for x in str(s).split()]


def _compare(tmp_path, oracle, ref, glob, particles, walls=(), min_contact_steps=1):
    from oracle import DemScene

    ref_dir = str(tmp_path / "ref")
    cfg = str(tmp_path / "sim.txt")
    g = dict(glob)
    g.update({"output_dir": ref_dir, "vtk_prefix": "p"})
    write_config(cfg, g, particles, walls)
    log = parse_log(run_reference(cfg))
    mat = lambda d: {k: float(d[k]) for k in ("density", "young", "poisson", "mu", "restitution") if k in d}
    parts = [dict(tris=ref.load_stl(p["stl"]), scale=float(p.get("scale", 1)), pos=_vec(p["pos"]), quat=_vec(p["quat"]),
                  vel=_vec(p["vel"]), omega=_vec(p["omega"]), **mat(p)) for p in particles]
    wl = [dict(tris=ref.load_stl(w["stl"]), scale=float(w.get("scale", 1)), pos=_vec(w["pos"]), quat=_vec(w["quat"]),
               mu=float(w["mu"]), restitution=float(w["restitution"])) for w in walls]
    sc = DemScene(oracle, parts, wl, gravity=_vec(glob.get("gravity", "0 0 0")), dt=float(glob["dt"]),
                  split=bool(int(glob.get("split_contacts", 1))))
    steps, every = int(glob["steps"]), int(glob["output_interval"])
    contact_steps = 0
    for s in range(steps):
        c = sc.step()
        if s % every:
            continue
        got = (c["contacts"], c["tri_checks"], c["segments"], c["comps"], c["loops"])
        assert got == log[s], f"step {s}: oracle {got} reference {log[s]}"
        contact_steps += c["contacts"] > 0
        want = parse_state_txt(out_file(ref_dir, "p", s, ".txt"))
        assert np.array_equal(sc.state[:, :13], want[:, :13]), (s, np.max(np.abs(sc.state[:, :13] - want[:, :13])))
    assert contact_steps >= min_contact_steps


def test_two_noised_icospheres(tmp_path, oracle, ref):
    from zdemx import synth

    rng = np.random.default_rng(1)
    for k in range(2):
        write_binary_stl(str(tmp_path / f"m{k}.stl"), synth.noised_icosphere(2, 1e-3, 0.15, rng))
    parts = [dict(stl=str(tmp_path / "m0.stl"), pos="0 0 0", vel="0.05 0 0", quat="1 0 0 0", omega="0 0 0", scale=1,
                  **MAT),
             dict(stl=str(tmp_path / "m1.stl"), pos="1.9e-3 0 0", vel="-0.05 0 0", quat="1 0 0 0", omega="0 0 0",
                  scale=1, **MAT)]
    _compare(tmp_path, oracle, ref, {"steps": 120, "dt": 1e-6, "split_contacts": 1, "gravity": "0 0 0",
                                     "output_interval": 5}, parts, min_contact_steps=5)


def test_cluster_with_spin_and_split_off(tmp_path, oracle, ref):
    from zdemx import synth

    rng = np.random.default_rng(2)
    write_binary_stl(str(tmp_path / "a.stl"), synth.noised_icosphere(1, 1e-3, 0.15, rng))
    write_binary_stl(str(tmp_path / "b.stl"), synth.noised_icosphere(2, 1e-3, 0.1, rng))
    parts = []
    for i in range(8):
        pos = np.array([(i % 2) * 1.85e-3, ((i // 2) % 2) * 1.85e-3, (i // 4) * 1.85e-3]) + rng.uniform(-5e-5, 5e-5, 3)
        q = synth.random_unit_quat(rng)
        parts.append(dict(stl=str(tmp_path / ("a.stl" if i % 3 else "b.stl")), pos=fmt(pos),
                          vel=fmt(rng.normal(size=3) * 0.02), quat=fmt(q), omega=fmt(rng.normal(size=3) * 5.0),
                          scale=1, **MAT))
    _compare(tmp_path, oracle, ref, {"steps": 40, "dt": 1e-6, "split_contacts": 0, "gravity": "0 0 -9.81",
                                     "output_interval": 2}, parts, min_contact_steps=5)


def test_walls_plane_and_box(tmp_path, oracle, ref):
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
    _compare(tmp_path, oracle, ref, {"steps": 200, "dt": 2e-6, "split_contacts": 1, "gravity": "0 0 -9.81",
                                     "output_interval": 20}, parts, walls, min_contact_steps=5)
