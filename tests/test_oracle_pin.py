"""Pins the oracle (oracle/zdx_oracle.c) to the reference: golden fixtures made by running the reference
(tests/golden/make_golden.py), and -- where oracle/_ref is built -- the reference library itself."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import compare_pair

FIELDS = ["seg", "comp_off", "comp_idx", "v_off", "V", "e_off", "E", "e2_off", "E2", "loop_comp", "loop_off",
          "loop_vid", "loop_status", "loop_geom"]


def _golden_case(z, ci):
    r = {k: z[f"c{ci}_{k}"] for k in FIELDS}
    s = z[f"c{ci}_scalars"]
    r.update(nseg=int(s[0]), ncomp=int(s[1]), nloop=int(s[2]), tri_checks=int(s[3]))
    r["seg"] = r["seg"].reshape(-1, 6)
    r["V"] = r["V"].reshape(-1, 3)
    r["E"] = r["E"].reshape(-1, 2)
    r["E2"] = r["E2"].reshape(-1, 2)
    r["loop_geom"] = r["loop_geom"].reshape(-1, 13)
    return r


def test_oracle_matches_reference_golden_pairs(oracle):
    z = np.load(os.path.join(GOLDEN, "pairs_ref.npz"))
    n_with_loops = 0
    for ci in range(int(z["ncase"])):
        A, B, pose, split = z[f"c{ci}_A"], z[f"c{ci}_B"], z[f"c{ci}_pose"], bool(z[f"c{ci}_split"])
        Ab, pA = oracle.build_mesh(A)
        Bb, _ = oracle.build_mesh(B)
        o = oracle.pair(Ab, pA[5], pA[6], Bb, pose[:7], pose[7:], split=split)
        g = _golden_case(z, ci)
        assert o["tri_checks"] == g["tri_checks"]
        assert compare_pair(g, o, exact=True) == [], f"case {ci}"
        n_with_loops += g["nloop"] > 0
    assert n_with_loops >= 8


def test_oracle_mesh_build_golden(oracle):
    z = np.load(os.path.join(GOLDEN, "mesh_ref.npz"))
    for i in range(int(z["nmesh"])):
        out, props = oracle.build_mesh(z[f"m{i}_in"], True)
        assert np.array_equal(out, z[f"m{i}_out"]) and np.array_equal(props, z[f"m{i}_props"])
        out, props = oracle.build_mesh(z[f"m{i}_in"], False)
        assert np.array_equal(out, z[f"m{i}_out_nc"]) and np.array_equal(props, z[f"m{i}_props_nc"])


def test_sort_replica_golden(oracle):
    z = np.load(os.path.join(GOLDEN, "sort_ref.npz"))
    for i in range(int(z["ncase"])):
        n = len(z[f"s{i}_perm"])
        got = oracle.sort(int(z[f"s{i}_kind"]), n, z[f"s{i}_ikey"], z[f"s{i}_dkey"])
        assert np.array_equal(got, z[f"s{i}_perm"]), i


def _antiqsort_keys(oracle, n):
    """McIlroy's adversary against the sort replica: keys fixed lazily so every pivot is bad, which drives
    introsort into its heapsort fallback.  Plays the adversary in Python over the replica's compares."""
    # Cheap stand-in: an organ-pipe with many ties also exercises deep partitions.
    k = np.concatenate([np.arange(n // 2), np.arange(n - n // 2)[::-1]]) % 7
    return k.astype(np.int32)


def test_sort_replica_live(oracle, ref):
    rng = np.random.default_rng(5)
    for trial in range(400):
        kind = trial % 3
        n = int(rng.integers(0, 600))
        ik = rng.integers(0, int(rng.integers(1, 8)), size=max(n, 1)).astype(np.int32)
        dk = rng.integers(0, int(rng.integers(1, 8)), size=max(n, 1)).astype(float)
        assert np.array_equal(ref.std_sort(kind, n, ik, dk), oracle.sort(kind, n, ik, dk))
    for n in (17, 100, 1000, 5000):
        ik = _antiqsort_keys(oracle, n)
        for kind in (0, 1):
            assert np.array_equal(ref.std_sort(kind, n, ik), oracle.sort(kind, n, ik))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_matches_reference_live(oracle, ref, seed):
    from zdemx import synth

    rng = np.random.default_rng(1000 + seed)
    for trial in range(25):
        sA, sB = int(rng.integers(1, 4)), int(rng.integers(1, 4))
        A = synth.noised_icosphere(sA, 1e-3, 0.15, rng)
        B = synth.noised_icosphere(sB, 1e-3, 0.15, rng)
        Ab, pA = ref.build_mesh(A)
        Bb, pB = ref.build_mesh(B)
        pose = synth.pair_poses(rng, 1, 1e-3, 0.0, 0.12)[0]
        split = bool(trial % 3)
        r = ref.pair(Ab, pA[5], pA[6], Bb, pose[:7], pose[7:], split=split)
        o = oracle.pair(Ab, pA[5], pA[6], Bb, pose[:7], pose[7:], split=split)
        assert compare_pair(r, o, exact=True) == [], (seed, trial)


def test_oracle_wall_and_integrate_live(oracle, ref):
    from zdemx import synth

    rng = np.random.default_rng(3)
    hits = 0
    for trial in range(30):
        P = synth.noised_icosphere(2, 1e-3, 0.15, rng)
        Pb, pp = ref.build_mesh(P)
        pose = np.r_[rng.uniform(-5e-4, 5e-4, 2), rng.uniform(-8e-4, 8e-4), synth.random_unit_quat(rng)]
        wt = np.array([-0.01, -0.01, 0.0, 0.01, -0.01, 0.0, 0.01, 0.01, 0.0])
        wn = np.array([0.0, 0.0, 1.0])
        a = ref.wall_contact(Pb, pose, wt, wn, pp[4], pp[5] * 0.1)
        b = oracle.wall_contact(Pb, pose, wt, wn, pp[4], pp[5] * 0.1)
        assert a[0] == b[0]
        if a[0]:
            hits += 1
            assert a[1] == b[1] and np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
        st = np.r_[pose, rng.normal(size=9), 1.0 / 3.0, rng.normal(size=9)]
        f, t, g = rng.normal(size=3), rng.normal(size=3), np.array([0.0, 0.0, -9.81])
        assert np.array_equal(ref.integrate(st, f, t, g, 1e-5)[:16], oracle.integrate(st, f, t, g, 1e-5)[:16])
    assert hits > 5


@pytest.mark.parametrize("fixture,split", [("polyline_ref.npz", False), ("polyline_split_ref.npz", True),
                                           ("polyline_hard_ref.npz", None)])
def test_oracle_polyline_mode_matches_polyline_py(oracle, fixture, split):
    """The oracle's polyline mode against polyline.py's own pipeline (polyline.py:743-822, with
    --split-contacts for the second fixture and per case for the third, whose cases are flat faces and
    sharp edges): the same segment count, components (sizes in order), loops (vertex counts, component
    of each) and loop points; the FP64 numbers within 1e-9 relative, since polyline.py computes them
    with numpy."""
    from _helpers import expected_contacts

    z = np.load(os.path.join(GOLDEN, fixture))
    for ci in range(int(z["ncase"])):
        A, B, pose, tol = z[f"c{ci}_A"], z[f"c{ci}_B"], z[f"c{ci}_pose"], float(z[f"c{ci}_tol"])
        if fixture == "polyline_hard_ref.npz":
            split = bool(z[f"c{ci}_split"])
        r = oracle.pair(A, 0.0, 0.0, B, pose[:7], pose[7:], split=split, mode=1, tol=tol)
        e = expected_contacts(r, polyline=True)
        assert r["nseg"] == int(z[f"c{ci}_nseg"]), ci
        lens = list(z[f"c{ci}_loop_len"])
        assert list(e["nvert"]) == lens, ci
        if split:
            assert r["ncomp"] == int(z[f"c{ci}_ncomp"]), ci
            assert list(np.diff(r["comp_off"])) == list(z[f"c{ci}_comp_sz"]), ci
            assert list(e["comp"]) == list(z[f"c{ci}_loop_comp"]), ci
        pts = np.split(z[f"c{ci}_loop_pts"], np.cumsum(lens)[:-1]) if lens else []
        for c, p in enumerate(pts):
            assert np.allclose(e["points"][c], p, rtol=1e-9, atol=1e-15), (ci, c)
        ref = z[f"c{ci}_geom"]
        for c in range(len(e["geom"])):
            g = e["geom"][c]
            Fn = 0.5 * 1e7 * g[12]
            got = np.r_[g, Fn, Fn * g[9:12]]
            assert np.allclose(got, ref[c], rtol=1e-9, atol=1e-9 * np.max(np.abs(ref[c]))), (ci, c)


def test_pyset_order_matches_cpython(oracle):
    """The oracle's restatement of CPython's set table (the order polyline.py visits a segment's
    candidates in) against real sets of this interpreter: distinct ints added in a random order, small
    and large, dense and sparse (collisions, linear probes, perturbed probes, resizes)."""
    rng = np.random.default_rng(8)
    for t in range(3000):
        n = int(rng.integers(0, 400))
        hi = int(rng.choice([16, 64, 500, 4000, 1 << 20]))
        keys = list(dict.fromkeys(int(x) for x in rng.integers(0, hi, size=n)))
        s = set()
        for k in keys:
            s.add(k)
        assert list(oracle.pyset_order(keys)) == list(s), (t, keys[:10])


def test_oracle_matches_reference_flat_shapes(oracle, ref):
    """zdem mode on flat faces and sharp edges against the reference C++ itself, bit for bit: offset,
    coplanar, rotated and tilted cubes, spheres in a face and on an edge, hulls, a mesh with a
    T-junction, grazing spheres; with and without the split."""
    from _dem_helpers import box_tris
    from zdemx import synth

    rng = np.random.default_rng(321)
    a = 1e-3
    cube = box_tris(a, a, a)
    h = a / 2
    v0, v1, v2, v3 = np.array([[-h, -h, h], [h, -h, h], [h, h, h], [-h, h, h]])
    m = (v0 + v2) / 2
    tbox = np.asarray([t for t in cube if not np.allclose(t[:, 2], h)] +
                      [np.array([v0, v1, m]), np.array([m, v1, v2]), np.array([v0, v2, v3])])
    ident = [1.0, 0.0, 0.0, 0.0]
    qz45 = [np.cos(np.pi / 8), 0.0, 0.0, np.sin(np.pi / 8)]
    qtilt = synth.random_unit_quat(rng)
    sphere = synth.noised_icosphere(2, 0.6e-3, 0.0, rng)
    rough = synth.noised_icosphere(2, 0.6e-3, 0.15, rng)
    hullA = synth.ellipsoid_hull(64, (1.0, 0.8, 0.6), 1e-3, rng)
    hullB = synth.ellipsoid_hull(64, (1.0, 0.8, 0.6), 1e-3, rng)
    cases = [(cube, cube, [0.6 * a, 0.3 * a, 0.2 * a], ident), (cube, cube, [0.5 * a, 0, 0], ident),
             (cube, cube, [0.8 * a, 0.1 * a, 0.05 * a], qz45), (cube, cube, [0.9 * a, 0.2 * a, -0.1 * a], qtilt),
             (cube, sphere, [0.0, 0.0, 0.9e-3], ident), (cube, rough, [0.85e-3, 0.0, 0.85e-3], qtilt),
             (hullA, hullB, [1.7e-3, 0.2e-3, 0.0], qtilt), (tbox, sphere, [0.05e-3, 0.05e-3, 0.95e-3], ident),
             (rough, sphere, [0.0, 0.0, 1.1995e-3], qtilt)]
    contacts = 0
    for k, (A, B, tB, qB) in enumerate(cases):
        Ab, pA = ref.build_mesh(np.asarray(A, float))
        Bb, pB = ref.build_mesh(np.asarray(B, float))
        poseA, poseB = np.r_[0.0, 0.0, 0.0, ident], np.r_[tB, qB].astype(float)
        for split in (False, True):
            r = ref.pair(Ab, pA[5], pA[6], Bb, poseA, poseB, split=split)
            o = oracle.pair(Ab, pA[5], pA[6], Bb, poseA, poseB, split=split)
            assert compare_pair(r, o, exact=True) == [], (k, split)
            contacts += r["nloop"]
    assert contacts >= 10


def test_oracle_wall_contact_flat_shapes(oracle, ref):
    """compute_wall_contact (src/main.cpp:1205-1258: plane section, Sutherland-Hodgman clip, area and
    centroid) on degenerate sections, against the reference C++ bit for bit: a cube face-down on the
    wall plane (coplanar with it, and just above and below), on an edge, on a corner, tilted, a cube
    straddling the wall triangle's edge, and icospheres touching at a vertex."""
    from _dem_helpers import box_tris
    from zdemx import synth

    rng = np.random.default_rng(9)
    a = 1e-3
    cube, cp = ref.build_mesh(box_tris(a, a, a))
    ball, bp = ref.build_mesh(synth.noised_icosphere(1, 1e-3, 0.0, rng))
    wall = np.array([-0.01, -0.01, 0.0, 0.01, -0.01, 0.0, 0.01, 0.01, 0.0])
    small = np.array([-4e-4, -4e-4, 0.0, 4e-4, -4e-4, 0.0, -4e-4, 4e-4, 0.0])  # edge under the cube
    wn = np.array([0.0, 0.0, 1.0])
    q_edge = [np.cos(np.pi / 8), np.sin(np.pi / 8), 0.0, 0.0]  # 45 deg about x: an edge down
    v = np.array([1.0, 1.0, 0.0]) / np.sqrt(2.0)
    ang = np.arccos(1.0 / np.sqrt(3.0))  # a body diagonal down: a corner
    q_corner = [np.cos(ang / 2), *(np.sin(ang / 2) * v)]
    ident = [1.0, 0.0, 0.0, 0.0]
    h = a / 2
    poses = []
    for dz in (0.0, 1e-9, -1e-9, -1e-5, -1e-4):
        poses.append((cube, cp, [0.0, 0.0, h + dz], ident, wall))
        poses.append((cube, cp, [1e-4, -2e-4, h + dz], ident, small))
    for dz in (0.0, -1e-6, -5e-5):
        poses.append((cube, cp, [0.0, 0.0, h * np.sqrt(2.0) + dz], q_edge, wall))
        poses.append((cube, cp, [0.0, 0.0, h * np.sqrt(3.0) + dz], q_corner, wall))
    for _ in range(8):
        poses.append((cube, cp, [0.0, 0.0, h * rng.uniform(0.9, 1.6)], list(synth.random_unit_quat(rng)), wall))
    poses.append((ball, bp, [0.0, 0.0, 1e-3 - 1e-7], ident, wall))
    poses.append((ball, bp, [0.0, 0.0, 1e-3], ident, wall))
    hits = 0
    for k, (tris, props, t, q, wt) in enumerate(poses):
        pose = np.r_[t, q].astype(float)
        ra = ref.wall_contact(tris, pose, wt, wn, props[4], props[5] * 0.1)
        rb = oracle.wall_contact(tris, pose, wt, wn, props[4], props[5] * 0.1)
        assert ra[0] == rb[0], k
        if ra[0]:
            hits += 1
            assert ra[1] == rb[1] and np.array_equal(ra[2], rb[2]) and np.array_equal(ra[3], rb[3]), k
    assert hits >= 12


def test_oracle_matches_reference_on_its_own_meshes(oracle, ref):
    """The oracle against the reference C++, bit for bit, on the reference's own sample meshes (its
    geometry/ folder: a convex particle, a low-poly banana and pug, a table; non-convex, with long thin
    triangles), each pair at seeded overlapping poses, with and without the split.  Runs where the
    reference tree is present (its path is recorded by oracle/Makefile in oracle/_ref/REF_ROOT)."""
    from zdemx import synth

    root_file = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                             "REF_ROOT")
    geo = os.path.join(open(root_file).read().strip(), "geometry") if os.path.exists(root_file) else ""
    if not (geo and os.path.isdir(geo)):
        pytest.skip("the reference's geometry folder is not here")
    names = ["convex-particle.stl", "low-poly-banbana.stl", "pug-lowpoly.stl", "table.stl"]
    meshes = []
    for f in names:
        p = os.path.join(geo, f)
        if not os.path.exists(p):
            pytest.skip(f"{f} missing")
        t = np.asarray(ref.load_stl(p), float).reshape(-1, 3, 3)
        t = t / np.max(np.linalg.norm(t.reshape(-1, 3) - t.reshape(-1, 3).mean(0), axis=1)) * 1e-3  # 1 mm scale
        meshes.append(ref.build_mesh(t))
    rng = np.random.default_rng(4)
    loops = 0
    for a in range(len(meshes)):
        for b in range(len(meshes)):
            (Ab, pA), (Bb, pB) = meshes[a], meshes[b]
            for trial in range(4):
                pose = synth.pair_poses(rng, 1, 0.5 * (pA[4] + pB[4]), 0.3, 1.2)[0]
                pose[3:7] = synth.random_unit_quat(rng)
                split = bool(trial % 2)
                r = ref.pair(Ab, pA[5], pA[6], Bb, pose[:7], pose[7:], split=split)
                o = oracle.pair(Ab, pA[5], pA[6], Bb, pose[:7], pose[7:], split=split)
                assert compare_pair(r, o, exact=True) == [], (names[a], names[b], trial)
                loops += r["nloop"]
    assert loops >= 40


@pytest.mark.parametrize("fixture", ["polyline_ref.npz", "polyline_split_ref.npz", "polyline_hard_ref.npz"])
def test_oracle_numpy_mode_is_bit_exact_with_polyline_py(oracle, fixture):
    """The oracle's numpy-arithmetic polyline mode (mode 2: np.dot and np.linalg.norm as this platform's
    FMA chains, tri_normals' normals for the triangle test) against polyline.py's own pipeline: every
    loop's points and Sn, Gn, xc0, nA, |Sn|, Fn, F_A identical to the bit, split or not."""
    from _helpers import expected_contacts

    z = np.load(os.path.join(GOLDEN, fixture))
    loops = 0
    for ci in range(int(z["ncase"])):
        A, B, pose, tol = z[f"c{ci}_A"], z[f"c{ci}_B"], z[f"c{ci}_pose"], float(z[f"c{ci}_tol"])
        split = bool(z[f"c{ci}_split"]) if f"c{ci}_split" in z.files else fixture == "polyline_split_ref.npz"
        r = oracle.pair(A, 0.0, 0.0, B, pose[:7], pose[7:], split=split, mode=2, tol=tol)
        e = expected_contacts(r, polyline=True)
        lens = list(z[f"c{ci}_loop_len"])
        assert r["nseg"] == int(z[f"c{ci}_nseg"]) and list(e["nvert"]) == lens, ci
        pts = np.split(z[f"c{ci}_loop_pts"], np.cumsum(lens)[:-1]) if lens else []
        for c, p in enumerate(pts):
            g = e["geom"][c]
            Fn = 0.5 * 1e7 * g[12]
            assert np.array_equal(e["points"][c], p), (ci, c)
            assert np.array_equal(np.r_[g, Fn, Fn * g[9:12]], z[f"c{ci}_geom"][c]), (ci, c)
            loops += 1
    assert loops >= 3


def test_oracle_numpy_mode_on_the_reference_meshes(oracle, ref):
    """The numpy-arithmetic mode against polyline.py itself, imported live from the reference tree where it
    is present, on the reference's own non-convex sample meshes at seeded overlapping poses, split and
    not: every loop's points and numbers identical to the bit."""
    import importlib.util
    import sys

    from _helpers import expected_contacts
    from zdemx import synth

    root_file = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                             "REF_ROOT")
    root = open(root_file).read().strip() if os.path.exists(root_file) else ""
    if not (root and os.path.exists(os.path.join(root, "polyline.py"))):
        pytest.skip("the reference tree is not here")
    spec = importlib.util.spec_from_file_location("_ref_polyline", os.path.join(root, "polyline.py"))
    P = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(P)
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import polyline_pipeline

    meshes = []
    for f in ("convex-particle.stl", "low-poly-banbana.stl", "pug-lowpoly.stl"):
        t = np.asarray(ref.load_stl(os.path.join(root, "geometry", f)), float).reshape(-1, 3, 3)
        c = t.reshape(-1, 3).mean(0)
        meshes.append((t - c) / np.max(np.linalg.norm(t.reshape(-1, 3) - c, axis=1)) * 1e-3)
    rng = np.random.default_rng(6)
    loops = 0
    for a in range(3):
        for b in range(3):
            pose = synth.pair_poses(rng, 1, 1e-3, 0.3, 1.0)[0]
            pose[3:7] = synth.random_unit_quat(rng)
            for split in (False, True):
                want = polyline_pipeline(P, meshes[a], meshes[b], pose, 1e-5, split)
                r = oracle.pair(meshes[a], 0.0, 0.0, meshes[b], pose[:7], pose[7:], split=split, mode=2, tol=1e-5)
                e = expected_contacts(r, polyline=True)
                lens = list(want["loop_len"])
                assert r["nseg"] == int(want["nseg"]) and list(e["nvert"]) == lens, (a, b, split)
                pts = np.split(want["loop_pts"], np.cumsum(lens)[:-1]) if lens else []
                for c, p in enumerate(pts):
                    g = e["geom"][c]
                    Fn = 0.5 * 1e7 * g[12]
                    assert np.array_equal(e["points"][c], p), (a, b, split, c)
                    assert np.array_equal(np.r_[g, Fn, Fn * g[9:12]], want["geom"][c]), (a, b, split, c)
                    loops += 1
    assert loops >= 10
