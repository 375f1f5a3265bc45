"""The polyline mirror's host code against polyline.py's own: its two VTK writers against the text
polyline.py's writers gave for the same inputs (polyline.py:544-649; fixture tests/golden/vtk_ref.npz),
byte for byte, including the 1e-9 point merge, skipped one-point loops, None contact points and contact
lists shorter than the loop list; and build_contacts_from_loops on polyline.py's traced loops."""
import os

import numpy as np

from conftest import GOLDEN


def _load():
    return np.load(os.path.join(GOLDEN, "vtk_ref.npz"))


def test_loop_writer_matches_reference_text(tmp_path):
    from zdemx import polyline

    z = _load()
    out = str(tmp_path / "loops.vtk")
    seen_none = seen_short = seen_mismatch = 0
    for ci in range(int(z["nloopcase"])):
        lens = z[f"l{ci}_loop_len"]
        pts = z[f"l{ci}_loop_pts"]
        loops = np.split(pts, np.cumsum(lens)[:-1]) if len(lens) else []
        cps = [None if none else p for none, p in zip(z[f"l{ci}_cp_none"], z[f"l{ci}_cp"])]
        cids = [int(c) for c in z[f"l{ci}_cids"]]
        polyline.write_vtk_polydata_polylines(out, loops, cps, cids)
        with open(out, encoding="utf-8") as f:
            assert f.read() == str(z[f"l{ci}_text"]), ci
        seen_none += any(c is None for c in cps)
        seen_short += any(len(x) < 2 for x in loops)
        seen_mismatch += len(cps) != len([x for x in loops if len(x) >= 2])
    assert seen_none and seen_short and seen_mismatch


def test_triangle_writer_matches_reference_text(tmp_path):
    from zdemx import polyline

    z = _load()
    out = str(tmp_path / "mesh.vtk")
    for ti in range(int(z["ntricase"])):
        polyline.write_vtk_polydata_tris(out, z[f"t{ti}_tris"], comment=f"mesh {ti}")
        with open(out, encoding="utf-8") as f:
            assert f.read() == str(z[f"t{ti}_text"]), ti


def test_build_contacts_from_loops_matches_reference_bit_for_bit():
    """The mirror's host build_contacts_from_loops (polyline.py:655-701, for loops a caller already holds)
    on the loops polyline.py traced in the three polyline fixtures: the same numpy expressions, so Sn,
    Gn, xc0, nA, |Sn|, Fn and F_A are identical to the bit."""
    from zdemx import polyline

    n = 0
    for fixture in ("polyline_ref.npz", "polyline_split_ref.npz", "polyline_hard_ref.npz"):
        z = np.load(os.path.join(GOLDEN, fixture))
        for ci in range(int(z["ncase"])):
            lens = list(z[f"c{ci}_loop_len"])
            loops = np.split(z[f"c{ci}_loop_pts"], np.cumsum(lens)[:-1]) if lens else []
            man = polyline.build_contacts_from_loops(0, 1, loops, list(range(len(loops))), k_stiff=1e7)
            geo = np.asarray([c["Sn"] + c["Gn"] + (c["xc0"] or [0, 0, 0]) + c["nA"] + [c["area"], c["Fn"]] +
                              c["F_A"] for c in man["contacts"]], float).reshape(-1, 17)
            assert np.array_equal(geo, z[f"c{ci}_geom"]), (fixture, ci)
            n += len(geo)
    assert n >= 40
