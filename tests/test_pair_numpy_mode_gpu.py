"""ZDX_MODE_POLYLINE_NUMPY on the GPU: the pair kernels in numpy's own arithmetic (zdx_npmath.cuh)
against the oracle's numpy mode, bit for bit, on the three polyline fixtures, split and not.  The
oracle's numpy mode is itself bit-exact with polyline.py on them (tests/test_oracle_pin.py), so this is
the GPU against polyline.py's own numbers."""
import os

import numpy as np
import pytest

from _helpers import compare_gpu_to_expected, expected_contacts, gpu_pair_slice
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fixture", ["polyline_ref.npz", "polyline_split_ref.npz", "polyline_hard_ref.npz"])
def test_numpy_mode_matches_oracle_and_polyline_py(ctx, oracle, fixture):
    from zdemx import _lib
    from zdemx.contact import MeshLibrary

    z = np.load(os.path.join(GOLDEN, fixture))
    for ci in range(int(z["ncase"])):
        A, B, pose, tol = z[f"c{ci}_A"], z[f"c{ci}_B"], z[f"c{ci}_pose"], float(z[f"c{ci}_tol"])
        split = bool(z[f"c{ci}_split"]) if f"c{ci}_split" in z.files else fixture == "polyline_split_ref.npz"
        lib = MeshLibrary.build([np.asarray(A, float), np.asarray(B, float)], center=False)
        res = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, [[0, 1]],
                                     pose[None, :], mode=_lib.MODE_POLYLINE_NUMPY, split=split, tol=tol, k=1e7,
                                     want_points=True)
        r = oracle.pair(lib.mesh(0), 0.0, 0.0, lib.mesh(1), pose[:7], pose[7:], split=split, mode=2, tol=tol)
        e = expected_contacts(r, polyline=True)
        assert compare_gpu_to_expected(gpu_pair_slice(res, 0), e, r) == [], (fixture, ci)
        # and polyline.py's own numbers
        lens = list(z[f"c{ci}_loop_len"])
        pts = np.split(z[f"c{ci}_loop_pts"], np.cumsum(lens)[:-1]) if lens else []
        g = gpu_pair_slice(res, 0)
        for c, p in enumerate(pts):
            assert np.array_equal(g["points"][c], p), (fixture, ci, c)
            gg = g["geom"][c]
            assert np.array_equal(np.r_[gg[:17]], z[f"c{ci}_geom"][c]), (fixture, ci, c)
