"""Pair contacts of flat faces and sharp edges on the GPU against the oracle, bit for bit, in both modes:
offset, coplanar, rotated and tilted cubes, spheres in a face and on an edge, hulls, a mesh with a
T-junction, grazing spheres (the shapes of tests/golden/polyline_hard_ref.npz, whose polyline-mode
results come from polyline.py itself).  The oracle is pinned to the reference on the same shapes on the
CPU (tests/test_oracle_pin.py)."""
import os

import numpy as np
import pytest

from _helpers import compare_gpu_to_expected, expected_contacts, gpu_pair_slice
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_flat_shapes_match_oracle_both_modes(ctx, oracle):
    from zdemx import _lib
    from zdemx.contact import MeshLibrary

    z = np.load(os.path.join(GOLDEN, "polyline_hard_ref.npz"))
    checked = 0
    for ci in range(int(z["ncase"])):
        A, B, pose = z[f"c{ci}_A"], z[f"c{ci}_B"], z[f"c{ci}_pose"]
        tol, split = float(z[f"c{ci}_tol"]), bool(z[f"c{ci}_split"])
        lib = MeshLibrary.build([A, B], center=False)  # the fixture's frames
        for mode in (0, 1):
            t = tol if mode == 1 else 0.0
            res = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, [[0, 1]],
                                         pose[None, :], mode=mode, split=split, tol=t, k=1e7, want_points=True)
            r = oracle.pair(lib.mesh(0), lib.mean_edge[0], lib.bbox_diag[0], lib.mesh(1), pose[:7], pose[7:],
                            split=split, mode=mode, tol=t)
            e = expected_contacts(r, polyline=mode == 1)
            bad = compare_gpu_to_expected(gpu_pair_slice(res, 0), e, r)
            assert bad == [], (str(z[f"c{ci}_name"]), split, mode, bad)
            checked += 1
            if mode == 1:
                # and polyline.py's own loops
                assert list(e["nvert"]) == list(z[f"c{ci}_loop_len"]), str(z[f"c{ci}_name"])
    assert checked == 2 * int(z["ncase"])
