"""The polyline mirror's command line against polyline.py's own (polyline.py:707-834), on the seeded STL
pairs of tests/golden/cli_ref.npz (its argv, stdout and the three VTK files it wrote):

* CPU: the transformed-mesh VTK files byte for byte (host code only), and main's printing and file
  logic, with the pair call replaced by the counts polyline.py printed, byte for byte on the cases
  without contacts (no segments; segments whose loops all snap away).  With the pair call computed in
  numpy's own arithmetic (the oracle's mode 2), stdout and all three files byte for byte on every case.
* GPU: the whole command line, its pair call in numpy's arithmetic (the default): stdout and all three
  files byte for byte.  In the C++ program's arithmetic (MODE_POLYLINE) lines and files are identical
  except for FP64 numbers, which agree within 1e-9 relative."""
import contextlib
import io
import os
import re

import numpy as np
import pytest

from _dem_helpers import write_binary_stl
from conftest import GOLDEN

NUM = re.compile(r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?")


def _cases():
    z = np.load(os.path.join(GOLDEN, "cli_ref.npz"))
    out = []
    for ci in range(int(z["ncase"])):
        out.append({k: z[f"c{ci}_{k}"] for k in ("name", "A", "B", "argv", "stdout", "vtkA", "vtkB", "loops")})
        for k in ("name", "argv", "stdout", "vtkA", "vtkB", "loops"):
            out[-1][k] = str(out[-1][k])
    return out


def _run_main(case, tmp):
    from zdemx import polyline

    write_binary_stl(os.path.join(tmp, "A.stl"), case["A"])
    write_binary_stl(os.path.join(tmp, "B.stl"), case["B"])
    cwd = os.getcwd()
    os.chdir(tmp)
    buf = io.StringIO()
    try:
        with contextlib.redirect_stdout(buf):
            polyline.main(case["argv"].split())
    finally:
        os.chdir(cwd)

    def read(f):
        p = os.path.join(tmp, f)
        return open(p, encoding="utf-8").read() if os.path.exists(p) else ""

    return buf.getvalue(), read("A_transformed.vtk"), read("B_transformed.vtk"), read("routeB_intersection.vtk")


def _same_up_to_rounding(got, want, what):
    """Identical text once every number is masked; the numbers within 1e-9 relative."""
    assert NUM.sub("#", got) == NUM.sub("#", want), what
    a = np.array([float(x) for x in NUM.findall(got)])
    b = np.array([float(x) for x in NUM.findall(want)])
    assert len(a) == len(b), what
    bad = np.abs(a - b) > 1e-9 * np.maximum(np.abs(a), np.abs(b)) + 1e-15
    assert not bad.any(), (what, a[bad][:5], b[bad][:5])


def test_transformed_meshes_match_reference(tmp_path):
    from zdemx import polyline

    for case in _cases():
        write_binary_stl(str(tmp_path / "A.stl"), case["A"])
        write_binary_stl(str(tmp_path / "B.stl"), case["B"])
        args = polyline.parse_args(case["argv"].split())
        for f, pose, comment, want in ((args.stlA, (args.tA, args.qA), "Mesh A (transformed)", case["vtkA"]),
                                       (args.stlB, (args.tB, args.qB), "Mesh B (transformed)", case["vtkB"])):
            tris0 = polyline.load_stl(str(tmp_path / f))
            tris = polyline.transform_points(tris0.reshape(-1, 3), *pose).reshape(-1, 3, 3)
            out = str(tmp_path / "m.vtk")
            polyline.write_vtk_polydata_tris(out, tris, comment=comment)
            assert open(out, encoding="utf-8").read() == want, (case["name"], f)


def test_main_without_contacts_matches_reference(tmp_path, monkeypatch):
    """main's own logic around the pair call: the messages, the component lines and the (empty) loops
    file, with the pair call giving the counts polyline.py printed."""
    from zdemx import polyline

    checked = 0
    for case in _cases():
        if "[Contact" in case["stdout"]:
            continue
        m = re.search(r"Raw intersection segments: (\d+)", case["stdout"])
        nseg = int(m.group(1)) if m else 0
        comps = [tuple(int(x) for x in c) for c in
                 re.findall(r"rawSeg=(\d+) snappedV=(\d+) edges=(\d+) loops=(\d+)", case["stdout"])]

        def fake(*a, comp_cap=0, _n=nseg, _c=comps):
            return {"idA": 0, "idB": 1, "contacts": []}, [], [], [], _n, len(_c), _c

        monkeypatch.setattr(polyline, "_pair_call", fake)
        d = tmp_path / case["name"]
        d.mkdir()
        stdout, va, vb, loops = _run_main(case, str(d))
        assert stdout == case["stdout"], case["name"]
        assert (va, vb, loops) == (case["vtkA"], case["vtkB"], case["loops"]), case["name"]
        checked += 1
    assert checked == 2


def test_main_with_numpy_arithmetic_is_byte_identical(tmp_path, monkeypatch, oracle):
    """With the pair call computed in numpy's own arithmetic (the oracle's mode 2), main's stdout and all
    three VTK files are byte-identical with polyline.py's, so its command line is reproduced exactly.
    (The GPU's polyline mode follows the C++ arithmetic and agrees to 1e-9: test_main_matches_reference.)"""
    from _helpers import expected_contacts
    from zdemx import polyline

    def pair_call(trisA, trisB, tA, qA, tB, qB, k, tol, split, idA, idB, ctx, comp_cap=0):
        A, B = np.asarray(trisA, float).reshape(-1, 3, 3), np.asarray(trisB, float).reshape(-1, 3, 3)
        r = oracle.pair(A, 0.0, 0.0, B, np.r_[tA, qA], np.r_[tB, qB], split=split, mode=2, tol=tol)
        e = expected_contacts(r, polyline=True)
        geom = np.asarray([np.r_[g, 0.5 * k * g[12], g[9:12] * (0.5 * k * g[12]), -(g[9:12] * (0.5 * k * g[12]))]
                           for g in e["geom"]]).reshape(-1, 20)
        info = np.array([[0, c, e["nvert"][c], e["comp"][c]] for c in range(len(geom))], np.int32).reshape(-1, 4)
        man = polyline._manifold(idA, idB, geom, info, k)
        comps = [(int(r["comp_off"][c + 1] - r["comp_off"][c]), int(r["v_off"][c + 1] - r["v_off"][c]),
                  int(r["e2_off"][c + 1] - r["e2_off"][c]), int(np.sum(e["comp"] == c))) for c in range(r["ncomp"])]
        loops = [[p.copy() for p in pts] for pts in e["points"]]
        xc0s = [None if g[12] == 0.0 else g[6:9].copy() for g in geom]
        return man, loops, xc0s, list(range(len(geom))), int(r["nseg"]), r["ncomp"], comps

    monkeypatch.setattr(polyline, "_pair_call", pair_call)
    for case in _cases():
        d = tmp_path / case["name"]
        d.mkdir()
        stdout, va, vb, loops = _run_main(case, str(d))
        assert stdout == case["stdout"], case["name"]
        assert (va, vb, loops) == (case["vtkA"], case["vtkB"], case["loops"]), case["name"]


@pytest.mark.gpu
def test_main_matches_reference(tmp_path):
    for case in _cases():
        d = tmp_path / case["name"]
        d.mkdir()
        stdout, va, vb, loops = _run_main(case, str(d))
        assert (va, vb) == (case["vtkA"], case["vtkB"]), case["name"]
        assert stdout == case["stdout"], case["name"]
        assert loops == case["loops"], case["name"]


@pytest.mark.gpu
def test_main_in_cpp_arithmetic_agrees_to_1e9(tmp_path, monkeypatch):
    import functools

    from zdemx import _lib, polyline

    monkeypatch.setattr(polyline, "_pair_call", functools.partial(polyline._pair_call, mode=_lib.MODE_POLYLINE))
    for case in _cases():
        d = tmp_path / case["name"]
        d.mkdir()
        stdout, va, vb, loops = _run_main(case, str(d))
        assert (va, vb) == (case["vtkA"], case["vtkB"]), case["name"]
        _same_up_to_rounding(stdout, case["stdout"], (case["name"], "stdout"))
        _same_up_to_rounding(loops, case["loops"], (case["name"], "loops vtk"))


@pytest.mark.parametrize("argv", [[], ["a.stl"], ["a.stl", "b.stl", "--tol"], ["a.stl", "b.stl", "--tA", "1", "2"],
                                  ["a.stl", "b.stl", "--bogus"], ["--help"]])
def test_argument_errors_match_reference_script(tmp_path, argv):
    """`python -m zdemx.polyline` against the reference's own `python polyline.py` on bad or missing
    arguments: the same stdout, stderr and exit status (argparse's usage and messages).  Runs where the
    reference tree is present (oracle/_ref/REF_ROOT)."""
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    root_file = os.path.join(root, "oracle", "_ref", "REF_ROOT")
    ref_root = open(root_file).read().strip() if os.path.exists(root_file) else ""
    ref_py = os.path.join(ref_root, "polyline.py")
    if not (ref_root and os.path.exists(ref_py)):
        pytest.skip("the reference tree is not here")
    env = dict(os.environ, PYTHONPATH=os.path.join(root, "zedm-x_b200"))
    got = subprocess.run([sys.executable, "-m", "zdemx.polyline"] + argv, capture_output=True, text=True,
                         timeout=120, cwd=str(tmp_path), env=env)
    want = subprocess.run([sys.executable, ref_py] + argv, capture_output=True, text=True, timeout=120,
                          cwd=str(tmp_path))
    assert got.returncode == want.returncode, (got.stderr, want.stderr)
    assert got.stderr == want.stderr
    assert got.stdout == want.stdout
