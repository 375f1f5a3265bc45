"""The polyline mirror's two VTK writers against the text polyline.py's own writers gave for the same
inputs (polyline.py:544-649; fixture tests/golden/vtk_ref.npz): byte for byte, including the 1e-9 point
merge, skipped one-point loops, None contact points and contact lists shorter than the loop list."""
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
