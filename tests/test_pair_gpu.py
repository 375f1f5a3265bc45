"""Parity of the CUDA pair-contact path (through the C ABI) with the oracle and with the reference.

Integer results (segment counts, components, raw loops, contact count, loop vertex counts, component
of each contact, contact ids) must be identical; with --fmad=false on both sides the FP64 geometry
(Sn, Gn, xc0, nA, |Sn|) and the snapped loop vertices are bit-exact too, which is stronger than the
1e-9 relative bound the path promises."""
import os

import numpy as np
import pytest

from _helpers import compare_gpu_to_expected, expected_contacts, gpu_pair_slice
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _library(raw_meshes):
    from zdemx.contact import MeshLibrary

    return MeshLibrary.build(raw_meshes)


def _run(ctx, lib, pm, pp, **kw):
    from zdemx import contact

    return contact.pair_contacts_batch(ctx, lib, pm, pp, want_points=True, **kw)


def test_gpu_matches_reference_golden(ctx):
    z = np.load(os.path.join(GOLDEN, "pairs_ref.npz"))
    from test_oracle_pin import _golden_case

    for ci in range(int(z["ncase"])):
        lib = _library([z[f"c{ci}_A"], z[f"c{ci}_B"]])
        split = bool(z[f"c{ci}_split"])
        res = _run(ctx, lib, [[0, 1]], z[f"c{ci}_pose"][None, :], split=split, k=1e7)
        g = _golden_case(z, ci)
        bad = compare_gpu_to_expected(gpu_pair_slice(res, 0), expected_contacts(g), g)
        assert bad == [], f"case {ci}: {bad}"


@pytest.mark.parametrize("split", [True, False])
def test_gpu_matches_oracle_mixed_batch(ctx, oracle, split):
    from zdemx import synth

    rng = np.random.default_rng(42 + split)
    meshes = [synth.noised_icosphere(s, 1e-3, 0.15, rng) for s in (1, 1, 2, 2, 2, 3, 3)]
    lib = _library(meshes)
    npairs = 96
    pm = rng.integers(0, lib.n_mesh, size=(npairs, 2)).astype(np.int32)
    pp = synth.pair_poses(rng, npairs, 1e-3, 0.0, 0.12)
    pp[5, 7:10] = [0.01, 0.0, 0.0]  # a pair far apart
    res = _run(ctx, lib, pm, pp, split=split, k=1e7)
    nct = 0
    for p in range(npairs):
        a, b = pm[p]
        r = oracle.pair(lib.mesh(a), lib.mean_edge[a], lib.bbox_diag[a], lib.mesh(b), pp[p, :7], pp[p, 7:],
                        split=split)
        e = expected_contacts(r)
        nct += len(e["geom"])
        bad = compare_gpu_to_expected(gpu_pair_slice(res, p), e, r)
        assert bad == [], f"pair {p}: {bad}"
        assert res["stats"][p, 0] == r["nseg"]
    assert nct > npairs  # most pairs touch, several with more than one loop
    assert res["totals"][0] == nct


def test_gpu_force_law_feng_min(ctx):
    from zdemx import synth

    rng = np.random.default_rng(3)
    lib = _library([synth.noised_icosphere(2, 1e-3, 0.15, rng) for _ in range(2)])
    pp = synth.pair_poses(rng, 8, 1e-3, 0.03, 0.1)
    res = _run(ctx, lib, np.array([[0, 1]] * 8, np.int32), pp, k=1e7)
    g = res["geom"]
    assert len(g) > 0
    # Fn = k/2 |Sn| (polyline.py:677); zdem mode: F_A = -Fn nA, F_B = -F_A, nA toward B
    assert np.array_equal(g[:, 13], 0.5 * 1e7 * g[:, 12])
    assert np.array_equal(g[:, 14:17], g[:, 9:12] * (-g[:, 13:14]))
    assert np.array_equal(g[:, 17:20], -g[:, 14:17])
    for c in range(len(g)):
        p = res["info"][c, 0]
        assert np.dot(g[c, 9:12], pp[p, 7:10] - pp[p, 0:3]) >= 0.0


def test_batched_equals_plain(ctx):
    from zdemx import _lib, synth

    rng = np.random.default_rng(9)
    lib = _library([synth.noised_icosphere(s, 1e-3, 0.15, rng) for s in (1, 2, 3)])
    pm = rng.integers(0, 3, size=(24, 2)).astype(np.int32)
    pp = synth.pair_poses(rng, 24, 1e-3, 0.0, 0.1)
    a = _run(ctx, lib, pm, pp, sched=_lib.SCHED_BATCHED)
    b = _run(ctx, lib, pm, pp, sched=_lib.SCHED_PLAIN)
    c = _run(ctx, lib, pm, pp, sched=_lib.SCHED_PER_STAGE)
    for k in ("ncontact", "contact_off", "stats", "geom", "info", "points", "point_off"):
        assert np.array_equal(a[k], b[k]), k
        assert np.array_equal(a[k], c[k]), k
    # the per-stage form has no culls: it counts the same triangle tests as the reference
    assert a["totals"][2] == c["totals"][2]


def test_edge_cases(ctx, oracle):
    from zdemx import _lib, synth

    rng = np.random.default_rng(4)
    A = synth.noised_icosphere(2, 1e-3, 0.15, rng)
    B = synth.noised_icosphere(1, 1e-3, 0.0, rng)
    # a degenerate (zero-area) triangle and a sliver in B
    B[3, 2] = B[3, 0]
    B[7, 1] = B[7, 0] + 1e-16
    lib = _library([A, B, A[:0]])
    # empty batch
    r0 = _run(ctx, lib, np.zeros((0, 2), np.int32), np.zeros((0, 14)))
    assert r0["totals"][0] == 0 and len(r0["contact_off"]) == 1
    pp = synth.pair_poses(rng, 6, 1e-3, 0.02, 0.1)
    pp[1, 7:10] = 0.0                      # concentric: B well inside A's hull region
    pp[2, 10:14] = pp[2, 3:7]              # same orientation
    pp[3, 7:10] = [2.3e-3, 0, 0]           # just apart
    pm = np.array([[0, 1], [0, 1], [1, 0], [0, 1], [0, 0], [0, 2]], np.int32)   # last: empty mesh B
    res = _run(ctx, lib, pm, pp)
    for p in range(len(pm)):
        a, b = pm[p]
        r = oracle.pair(lib.mesh(a), lib.mean_edge[a], lib.bbox_diag[a], lib.mesh(b), pp[p, :7], pp[p, 7:], split=True)
        assert compare_gpu_to_expected(gpu_pair_slice(res, p), expected_contacts(r), r) == [], p
    assert res["stats"][5, 0] == 0
    # bad mesh index is rejected before any work
    with pytest.raises(_lib.ZdxError):
        _run(ctx, lib, np.array([[0, 7]], np.int32), pp[:1])


def test_capacity_is_reported_not_truncated(ctx):
    from zdemx import _lib, synth

    rng = np.random.default_rng(6)
    lib = _library([synth.noised_icosphere(3, 1e-3, 0.15, rng) for _ in range(2)])
    pp = synth.pair_poses(rng, 1, 1e-3, 0.08, 0.08)
    with pytest.raises(_lib.ZdxError) as ei:
        _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, [[0, 1]], pp,
                               max_seg_per_pair=4)
    assert ei.value.status == _lib.ZDX_ERR_CAPACITY


def test_polyline_mode_matches_oracle_and_python_reference(ctx, oracle):
    """The mirror's pair call in the C++ program's arithmetic (MODE_POLYLINE): bit for bit the oracle's
    polyline mode, within 1e-9 of polyline.py; in its default, numpy's arithmetic: polyline.py's numbers
    bit for bit."""
    from zdemx import _lib, polyline

    z = np.load(os.path.join(GOLDEN, "polyline_ref.npz"))
    for ci in range(int(z["ncase"])):
        A, B, pose, tol = z[f"c{ci}_A"], z[f"c{ci}_B"], z[f"c{ci}_pose"], float(z[f"c{ci}_tol"])
        man, loops, xc0s, cids = polyline.pair_contacts(A, B, pose[0:3], pose[3:7], pose[7:10], pose[10:14], k=1e7,
                                                        tol=tol, split_contacts=False, ctx=ctx,
                                                        mode=_lib.MODE_POLYLINE)
        o = oracle.pair(A, 0.0, 0.0, B, pose[:7], pose[7:], split=False, mode=1, tol=tol)
        e = expected_contacts(o, polyline=True)
        # GPU vs oracle in polyline mode: bit-exact
        assert len(man["contacts"]) == len(e["geom"])
        for c, cc in enumerate(man["contacts"]):
            got = np.r_[cc["Sn"], cc["Gn"], cc["xc0"] or [0, 0, 0], cc["nA"], cc["area"]]
            assert np.array_equal(got, e["geom"][c]), (ci, c)
            assert np.array_equal(np.asarray(loops[c]), e["points"][c])
        # vs polyline.py itself (numpy arithmetic, so within tolerance): same loops, same numbers
        assert len(loops) == int(z[f"c{ci}_nloop"])
        assert [len(x) for x in loops] == list(z[f"c{ci}_loop_len"])
        ref = z[f"c{ci}_geom"]
        for c, cc in enumerate(man["contacts"]):
            got = np.r_[cc["Sn"], cc["Gn"], cc["xc0"] or [0, 0, 0], cc["nA"], cc["area"], cc["Fn"], cc["F_A"]]
            assert np.allclose(got, ref[c], rtol=1e-9, atol=1e-9 * np.max(np.abs(ref[c]))), (ci, c)
        _same_as_polyline_py(polyline, z, ci, A, B, pose, tol, False, ctx)


def _same_as_polyline_py(polyline, z, ci, A, B, pose, tol, split, ctx):
    """The default mode against polyline.py's own loops and numbers, bit for bit."""
    man, loops, _, _ = polyline.pair_contacts(A, B, pose[0:3], pose[3:7], pose[7:10], pose[10:14], k=1e7, tol=tol,
                                              split_contacts=split, ctx=ctx)
    lens = list(z[f"c{ci}_loop_len"])
    assert [len(x) for x in loops] == lens, ci
    pts = np.split(z[f"c{ci}_loop_pts"], np.cumsum(lens)[:-1]) if lens else []
    for c, p in enumerate(pts):
        assert np.array_equal(np.asarray(loops[c]), p), (ci, c)
    ref = z[f"c{ci}_geom"]
    for c, cc in enumerate(man["contacts"]):
        got = np.r_[cc["Sn"], cc["Gn"], cc["xc0"] or [0, 0, 0], cc["nA"], cc["area"], cc["Fn"], cc["F_A"]]
        assert np.array_equal(got, ref[c]), (ci, c)


def test_polyline_tol_none_is_the_mean_edge_rule(ctx):
    """pair_contacts(tol=None) snaps with the zdem_cpu step's tolerance, 0.1 x A's mean edge
    (src/main.cpp:2118-2121): the same contacts as the explicit value."""
    from zdemx import _lib, polyline, synth

    rng = np.random.default_rng(31)
    A = synth.noised_icosphere(2, 1e-3, 0.15, rng)
    B = synth.noised_icosphere(2, 1e-3, 0.15, rng)
    pose = synth.pair_poses(rng, 1, 1e-3, 0.05, 0.06)[0]
    me = _lib.mesh_build(A, False)[1]["mean_edge"]
    assert me > 0
    a = polyline.pair_contacts(A, B, pose[0:3], pose[3:7], pose[7:10], pose[10:14], k=1e7, tol=None, ctx=ctx)
    b = polyline.pair_contacts(A, B, pose[0:3], pose[3:7], pose[7:10], pose[10:14], k=1e7, tol=0.1 * me, ctx=ctx)
    assert len(a[0]["contacts"]) == len(b[0]["contacts"]) > 0
    for x, y in zip(a[0]["contacts"], b[0]["contacts"]):
        assert np.array_equal(x["Sn"], y["Sn"]) and x["area"] == y["area"]


def test_polyline_split_matches_oracle_and_python_reference(ctx, oracle):
    """--split-contacts in polyline mode: components searched in the iteration order of polyline.py's
    candidate sets, so loops start and run as polyline.py's do.  GPU == oracle bit for bit; against
    polyline.py itself (tests/golden/polyline_split_ref.npz) the same components, loops and loop points,
    numbers within 1e-9; in the default numpy arithmetic, polyline.py's numbers bit for bit."""
    from zdemx import _lib, polyline

    z = np.load(os.path.join(GOLDEN, "polyline_split_ref.npz"))
    for ci in range(int(z["ncase"])):
        A, B, pose, tol = z[f"c{ci}_A"], z[f"c{ci}_B"], z[f"c{ci}_pose"], float(z[f"c{ci}_tol"])
        man, loops, xc0s, cids = polyline.pair_contacts(A, B, pose[0:3], pose[3:7], pose[7:10], pose[10:14], k=1e7,
                                                        tol=tol, split_contacts=True, ctx=ctx,
                                                        mode=_lib.MODE_POLYLINE)
        o = oracle.pair(A, 0.0, 0.0, B, pose[:7], pose[7:], split=True, mode=1, tol=tol)
        e = expected_contacts(o, polyline=True)
        assert len(man["contacts"]) == len(e["geom"]), ci
        for c, cc in enumerate(man["contacts"]):
            got = np.r_[cc["Sn"], cc["Gn"], cc["xc0"] or [0, 0, 0], cc["nA"], cc["area"]]
            assert np.array_equal(got, e["geom"][c]), (ci, c)
            assert np.array_equal(np.asarray(loops[c]), e["points"][c]), (ci, c)
        lens = list(z[f"c{ci}_loop_len"])
        assert [len(x) for x in loops] == lens, ci
        pts = np.split(z[f"c{ci}_loop_pts"], np.cumsum(lens)[:-1])
        for c, p in enumerate(pts):
            assert np.allclose(np.asarray(loops[c]), p, rtol=1e-9, atol=1e-15), (ci, c)
        ref = z[f"c{ci}_geom"]
        for c, cc in enumerate(man["contacts"]):
            got = np.r_[cc["Sn"], cc["Gn"], cc["xc0"] or [0, 0, 0], cc["nA"], cc["area"], cc["Fn"], cc["F_A"]]
            assert np.allclose(got, ref[c], rtol=1e-9, atol=1e-9 * np.max(np.abs(ref[c]))), (ci, c)
        _same_as_polyline_py(polyline, z, ci, A, B, pose, tol, True, ctx)


@pytest.mark.parametrize("split,mode", [(True, 0), (False, 0), (False, 1), (True, 1)])
def test_large_pairs(ctx, oracle, split, mode):
    """Pairs of 1,280- and 5,120-triangle meshes (160 to 560 segments and up to 17 contacts a pair: long
    component searches, large snap classes, many T-junction candidates) against the oracle, bit for bit;
    polyline mode (mode 1) too."""
    from zdemx import contact, synth

    rng = np.random.default_rng(77 + 2 * split + mode)
    meshes = [synth.noised_icosphere(s, 1e-3, 0.15, rng) for s in (3, 4, 4)]
    lib = _library(meshes)
    npairs = 12
    pm = np.array([[1 + (p % 2), 1 + ((p // 2) % 2)] if p % 3 else [0, 2] for p in range(npairs)], np.int32)
    pp = synth.pair_poses(rng, npairs, 1e-3, 0.02, 0.12)
    if mode == 1:
        tol = 2e-5
        res = contact.pair_contacts_batch(ctx, lib, pm, pp, want_points=True, split=split, k=1e7, mode=1, tol=tol)
    else:
        tol = 0.0
        res = _run(ctx, lib, pm, pp, split=split, k=1e7)
    big = 0
    for p in range(npairs):
        a, b = pm[p]
        r = oracle.pair(lib.mesh(a), lib.mean_edge[a], lib.bbox_diag[a], lib.mesh(b), pp[p, :7], pp[p, 7:],
                        split=split, mode=mode, tol=tol)
        e = expected_contacts(r, polyline=mode == 1)
        bad = compare_gpu_to_expected(gpu_pair_slice(res, p), e, r)
        assert bad == [], f"pair {p}: {bad}"
        assert res["stats"][p, 0] == r["nseg"]
        big += r["nseg"] > 200
    assert big >= 4


@pytest.mark.parametrize("split,mode,sched", [(True, 0, 0), (True, 1, 0), (False, 1, 1)])
def test_component_counts_match_oracle(ctx, oracle, split, mode, sched):
    """The optional per-component counts (segments, snapped vertices, edges after the T-junction split)
    against the oracle's components, batched and plain; components past the cap stay 0."""
    from zdemx import _lib, synth

    rng = np.random.default_rng(5 + 2 * split + mode)
    meshes = [synth.noised_icosphere(s, 1e-3, 0.15, rng) for s in (1, 2, 2, 3)]
    lib = _library(meshes)
    npairs = 40
    pm = rng.integers(0, lib.n_mesh, size=(npairs, 2)).astype(np.int32)
    pp = synth.pair_poses(rng, npairs, 1e-3, 0.0, 0.15)
    tol = 2e-5 if mode == 1 else 0.0
    cap = 3
    res = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pm, pp, mode=mode,
                                 split=split, tol=tol, k=1e7, sched=sched, comp_cap=cap)
    cs = res["comp_stats"]
    assert cs.shape == (npairs, cap, 3)
    multi = 0
    for p in range(npairs):
        a, b = pm[p]
        r = oracle.pair(lib.mesh(a), lib.mean_edge[a], lib.bbox_diag[a], lib.mesh(b), pp[p, :7], pp[p, 7:],
                        split=split, mode=mode, tol=tol)
        want = np.zeros((cap, 3), np.int32)
        for c in range(min(r["ncomp"], cap)):
            want[c] = [r["comp_off"][c + 1] - r["comp_off"][c], r["v_off"][c + 1] - r["v_off"][c],
                       r["e2_off"][c + 1] - r["e2_off"][c]]
        assert np.array_equal(cs[p], want), (p, cs[p], want)
        multi += r["ncomp"] > 1
    assert multi >= (3 if split else 0)
