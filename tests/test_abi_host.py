"""libzdemx.so loads, exports every entry point of include/zdemx.h, and its host-side set-up (STL
loading, build_mesh) is bit-exact with the reference.  No GPU needed."""
import ctypes as C
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN


def test_library_exports_every_declared_symbol():
    from zdemx import _lib

    L = _lib.lib()
    names = _lib.exported_symbols()
    assert len(names) >= 9
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/zdemx.h but not exported"
    assert L.zdx_version().decode().startswith("zdemx")
    assert L.zdx_status_string(3).decode() == "capacity exceeded"


def test_create_without_device_reports_status():
    import torch

    from zdemx import _lib

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    assert _lib.lib().zdx_create(C.byref(h), 0) == _lib.ZDX_ERR_NO_DEVICE


def test_mesh_build_matches_reference_golden():
    from zdemx import _lib

    z = np.load(os.path.join(GOLDEN, "mesh_ref.npz"))
    for i in range(int(z["nmesh"])):
        out, p = _lib.mesh_build(z[f"m{i}_in"], True)
        assert np.array_equal(out, z[f"m{i}_out"]) and np.array_equal(p["raw"], z[f"m{i}_props"])
        out, p = _lib.mesh_build(z[f"m{i}_in"], False)
        assert np.array_equal(out, z[f"m{i}_out_nc"]) and np.array_equal(p["raw"], z[f"m{i}_props_nc"])


def test_mesh_build_matches_reference_live(ref):
    from zdemx import _lib, synth

    rng = np.random.default_rng(8)
    for s in range(5):
        t = synth.noised_icosphere(s, 1e-3, 0.15, rng) + rng.normal(size=3) * 1e-3
        for center in (True, False):
            a, pa = ref.build_mesh(t, center)
            b, pb = _lib.mesh_build(t, center)
            assert np.array_equal(a, b) and np.array_equal(pa, pb["raw"]), (s, center)
    # near-duplicate corners (closer than 1e-5) collapse exactly as unique_vertices does
    t = synth.noised_icosphere(2, 1e-3, 0.0, rng)
    t[5, 1] += 3e-6
    t[9, 2] -= 9e-6
    a, pa = ref.build_mesh(t, True)
    b, pb = _lib.mesh_build(t, True)
    assert np.array_equal(pa, pb["raw"])


def _write_binary_stl(path, tris):
    with open(path, "wb") as f:
        f.write(b"zdemx test".ljust(80, b"\0"))
        f.write(struct.pack("<I", len(tris)))
        for t in tris:
            f.write(struct.pack("<3f", 0, 0, 1))
            f.write(struct.pack("<9f", *np.asarray(t, np.float32).reshape(-1)))
            f.write(struct.pack("<H", 0))


def _write_ascii_stl(path, tris):
    with open(path, "w") as f:
        f.write("solid test\n")
        for t in tris:
            f.write("  facet normal 0 0 1\n    outer loop\n")
            for v in t:
                f.write(f"      vertex {v[0]:.6e} {v[1]:.6e} {v[2]:.6e}\n")
            f.write("    endloop\n  endfacet\n")
        f.write("endsolid test\n")


def test_stl_loader_matches_reference(tmp_path, ref):
    from zdemx import _lib, synth

    rng = np.random.default_rng(2)
    t = synth.noised_icosphere(2, 1.0, 0.15, rng)
    for writer, name in ((_write_binary_stl, "b.stl"), (_write_ascii_stl, "a.stl")):
        p = str(tmp_path / name)
        writer(p, t)
        a = ref.load_stl(p)
        b = _lib.stl_load(p)
        assert a.shape == b.shape and np.array_equal(a, b)
    # the reference's own fixture STLs, where the tree the oracle was built from is present
    root_file = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "REF_ROOT")
    ref_geo = os.path.join(open(root_file).read().strip(), "geometry") if os.path.exists(root_file) else ""
    if ref_geo and os.path.isdir(ref_geo):
        for f in sorted(os.listdir(ref_geo)):
            if f.endswith(".stl"):
                a = ref.load_stl(os.path.join(ref_geo, f))
                b = _lib.stl_load(os.path.join(ref_geo, f))
                assert np.array_equal(a, b), f
                # and build_mesh on them, at the reference configs' scale and unscaled
                for scale in (1.0, 1e-3):
                    for center in (True, False):
                        ma, pa = ref.build_mesh(a * scale, center)
                        mb, pb = _lib.mesh_build(b * scale, center)
                        assert np.array_equal(ma, mb) and np.array_equal(pa, pb["raw"]), (f, scale, center)


def test_stl_loader_errors(tmp_path):
    from zdemx import _lib, polyline

    p = tmp_path / "short.stl"
    p.write_bytes(b"abc")
    with pytest.raises(_lib.ZdxError):
        _lib.stl_load(str(p))
    with pytest.raises(ValueError):
        polyline.load_stl(str(p))
    q = tmp_path / "text.stl"
    q.write_text("solid nothing here\n" * 10)
    with pytest.raises(ValueError):
        polyline.load_stl(str(q))


def test_header_is_self_contained_c_and_cpp(tmp_path):
    """include/zdemx.h compiles on its own as C99 and as C++11 (pedantic, warnings as errors): a caller
    in either language includes it first and needs nothing else."""
    import shutil
    import subprocess

    src = tmp_path / "use.c"
    src.write_text('#include "zdemx.h"\n'
                   "int main(void) {\n"
                   "    zdx_pair_opts o = {ZDX_MODE_POLYLINE, 1, 1e-6, 1.0, ZDX_MEM_HOST, ZDX_SCHED_BATCHED, 1, 0};\n"
                   "    (void)o;\n"
                   "    return zdx_version() ? 0 : 1;\n"
                   "}\n")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    for cc, args in (("gcc", ["-std=c99"]), ("g++", ["-std=c++11", "-x", "c++"])):
        if shutil.which(cc) is None:
            continue
        p = subprocess.run([cc] + args + ["-Wall", "-Wextra", "-pedantic", "-Werror", "-I", inc, "-fsyntax-only",
                                          str(src)], capture_output=True, text=True, timeout=120)
        assert p.returncode == 0, (cc, p.stderr)
