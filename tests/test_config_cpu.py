"""The config grammar and the scene set-up on the host, without a GPU (zdx_config_check), against the
reference program itself (oracle/_ref, run in a subprocess with steps = 0 so that it only reads and sets
up): the same configs accepted, and for a rejected one the same message on stderr and exit status 1
(src/main.cpp:1531-1689, 1872-1881, 1936-1987)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from _dem_helpers import ROOT, plane_tris, write_binary_stl, write_config

MAT = {"density": 2500, "young": 1e7, "poisson": 0.25, "mu": 0.5, "restitution": 0.5}


def _reference(cfg_path):
    from oracle import LIB_REF

    if not os.path.exists(LIB_REF):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    code = ("import sys; sys.path.insert(0, %r); from oracle import Reference; import ctypes; "
            "r = Reference(%r); rc = r.main(['--config', %r]); ctypes.CDLL(None).fflush(None); sys.exit(rc)") % (
        os.path.join(ROOT, "oracle"), LIB_REF, cfg_path)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    return p.returncode, p.stderr.strip()


def _cases(tmp):
    from zdemx import synth

    rng = np.random.default_rng(3)
    stl = os.path.join(tmp, "p.stl")
    write_binary_stl(stl, synth.noised_icosphere(1, 1e-3, 0.1, rng))
    ascii_stl = os.path.join(tmp, "a.stl")
    with open(ascii_stl, "w") as f:
        f.write("solid a\n")
        for t in synth.noised_icosphere(1, 1e-3, 0.1, rng):
            f.write(" facet normal 0 0 0\n  outer loop\n")
            for v in t:
                f.write("   vertex %r %r %r\n" % tuple(float(x) for x in v))
            f.write("  endloop\n endfacet\n")
        f.write("endsolid a\n")
    empty_stl = os.path.join(tmp, "empty.stl")
    write_binary_stl(empty_stl, np.zeros((0, 3, 3)))
    plane = os.path.join(tmp, "plane.stl")
    write_binary_stl(plane, plane_tris(0.02))
    out = os.path.join(tmp, "out")
    g = {"steps": 0, "dt": 1e-6, "output_dir": out}
    part = lambda path, **kw: dict(dict(stl=path, pos="0 0 0", vel="0 0 0", quat="1 0 0 0", omega="0 0 0", scale=1, **MAT), **kw)
    cases = {
        "two_blocks": (g, [part(stl), part(ascii_stl, pos="2e-3 0 0")], []),
        "scaled_and_defaults": (g, [part(stl, scale=2), {"stl": stl, "pos": "0 0 1e-2"}], []),
        "legacy_row": (dict(g, stl=stl, n=3, spacing=2e-3, v0="1 0 0", v1="-1 0 0"), [], []),
        "legacy_zero_rows": (dict(g, stl=stl, n=0), [], []),
        "no_particles_no_stl": (g, [], []),
        "missing_stl": (g, [{"pos": "0 0 0"}], []),
        "unreadable_stl": (g, [part(os.path.join(tmp, "nope.stl"))], []),
        "empty_stl": (g, [part(empty_stl)], []),
        "global_stl_for_blocks": (dict(g, stl=stl), [{"pos": "0 0 0"}, {"pos": "0 3e-3 0"}], []),
        "walls": (g, [part(stl)], [dict(stl=plane, pos="0 0 0", quat="1 0 0 0", scale=1, mu=0.4, restitution=0.3),
                                   dict(pos="0 0 0")]),
        "unknown_keys_and_clamp": (dict(g, colour="red", output_interval=0), [part(stl, flavour="x")], []),
        # this library's own keys (the graph step's clearance cache), which the reference ignores
        "cache_keys": (dict(g, contact_cache=0, contact_cache_tau=0.02), [part(stl)], []),
    }
    return cases


def test_config_acceptance_and_messages_match_reference(tmp_path):
    from zdemx import _lib

    accepted = rejected = 0
    for name, (glob, parts, walls) in _cases(str(tmp_path)).items():
        cfg = str(tmp_path / f"{name}.txt")
        write_config(cfg, glob, parts, walls)
        rc, msg, counts = _lib.config_check(cfg)
        ref_rc, ref_err = _reference(cfg)
        assert (rc == 0) == (ref_rc == 0), (name, rc, msg, ref_rc, ref_err)
        if rc:
            assert msg == ref_err, (name, msg, ref_err)
            rejected += 1
        else:
            accepted += 1
    assert accepted >= 6 and rejected >= 4, (accepted, rejected)
    # a file that does not exist
    missing = str(tmp_path / "none.txt")
    rc, msg, _ = _lib.config_check(missing)
    ref_rc, ref_err = _reference(missing)
    assert rc != 0 and ref_rc == 1 and msg == ref_err


def test_config_counts(tmp_path):
    from zdemx import _lib

    cases = _cases(str(tmp_path))
    want = {"two_blocks": (2, 0, 2), "scaled_and_defaults": (2, 0, 2), "legacy_row": (3, 0, 1),
            "legacy_zero_rows": (0, 0, 0), "global_stl_for_blocks": (2, 0, 1), "walls": (1, 1, 2)}
    for name, w in want.items():
        glob, parts, walls = cases[name]
        cfg = str(tmp_path / f"{name}.txt")
        write_config(cfg, glob, parts, walls)
        rc, msg, counts = _lib.config_check(cfg)
        assert rc == 0, (name, msg)
        assert counts[:3] == w, (name, counts)


def test_reference_sample_configs(tmp_path):
    """The reference's own sample configs (its config/ folder), with their STL paths made absolute, the
    output folder moved here and steps = 0: accepted by both, with the same particle, wall and mesh
    counts as the files describe.  Runs where the reference tree is present (oracle/_ref/REF_ROOT)."""
    import re

    from zdemx import _lib

    root_file = os.path.join(ROOT, "oracle", "_ref", "REF_ROOT")
    ref_root = open(root_file).read().strip() if os.path.exists(root_file) else ""
    cfg_dir = os.path.join(ref_root, "config")
    if not (ref_root and os.path.isdir(cfg_dir)):
        pytest.skip("the reference's config folder is not here")
    names = sorted(f for f in os.listdir(cfg_dir) if f.endswith(".txt"))
    assert names
    for name in names:
        text = open(os.path.join(cfg_dir, name)).read()
        text = re.sub(r"(?m)^(\s*stl\s*=?\s*)(\S+)", lambda m: m.group(1) + os.path.join(ref_root, m.group(2)), text)
        text = re.sub(r"(?m)^(\s*output_dir\s*=?\s*)(\S+)", lambda m: m.group(1) + str(tmp_path / "out"), text)
        text = re.sub(r"(?m)^(\s*steps\s*=?\s*)(\S+)", lambda m: m.group(1) + "0", text)
        cfg = str(tmp_path / name)
        open(cfg, "w").write(text)
        rc, msg, counts = _lib.config_check(cfg)
        ref_rc, ref_err = _reference(cfg)
        assert rc == 0 and ref_rc == 0, (name, msg, ref_err)
        nblocks = len(re.findall(r"(?m)^\s*particle\s*$", text))
        nwalls = len(re.findall(r"(?m)^\s*wall\s*$", text))
        assert counts[0] == nblocks and counts[1] == nwalls, (name, counts)
