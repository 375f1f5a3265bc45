"""Generate the golden fixtures of tests/golden from the reference itself.

Run here, where the reference is present:  python tests/golden/make_golden.py
It needs oracle/_ref (built by `make -C oracle ref` from the reference's src/main.cpp) and imports the
reference's polyline.py from /root/reference (read-only).  The fixtures it writes are small .npz files;
the tests that use them never touch the reference.

* pairs_ref.npz      seeded noised-icosphere pairs through the reference C++ per-pair code
                     (src/main.cpp:2062-2219): segments, components, snapped vertices/edges, loops,
                     Sn/Gn/xc0/nA/area and the loop filters.
* mesh_ref.npz       build_mesh (src/main.cpp:445-497) on a few meshes.
* sort_ref.npz       std::sort permutations under the reference's three comparators.
* polyline_ref.npz   polyline.py's own pipeline (polyline.py:743-822) on a few pairs.
* vtk_ref.npz        the text polyline.py's two VTK writers (polyline.py:544-649) give for seeded loops,
                     contact points and triangle soups: near-duplicate points inside and outside the
                     1e-9 merge, loops too short to draw, None contact points, and contact lists
                     shorter than the loop list.

* cli_ref.npz        polyline.py's command line (polyline.py:707-834) on seeded binary STL pairs:
                     its argv, stdout and the three VTK files it writes (no split, split into two
                     components, no intersection, segments whose loops all snap away).

* polyline_split_ref.npz  the same pipeline with --split-contacts (label_segments_by_contact_greedy,
                     polyline.py:267-341) on pairs whose contact splits into several components.
* polyline_hard_ref.npz   the same pipeline, with and without the split, on flat faces and sharp edges:
                     offset, coplanar, rotated and tilted cubes, a sphere in a face and on an edge,
                     hulls, a T-junction in a mesh, grazing spheres.

`python tests/golden/make_golden.py vtk` regenerates only the named fixtures.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "zedm-x_b200"), os.path.join(ROOT, "oracle")]

from oracle import Reference  # noqa: E402
from zdemx import synth  # noqa: E402

REF_PY = os.environ.get("ZDX_REFERENCE_ROOT", "/root/reference")


def pack(prefix, r, d):
    for k in ["seg", "comp_off", "comp_idx", "v_off", "V", "e_off", "E", "e2_off", "E2", "loop_comp", "loop_off",
              "loop_vid", "loop_status", "loop_geom"]:
        d[f"{prefix}{k}"] = r[k]
    d[f"{prefix}scalars"] = np.array([r["nseg"], r["ncomp"], r["nloop"], r["tri_checks"]], np.int64)


def make_pairs(R):
    rng = np.random.default_rng(20261203)
    d = {}
    cases = [(1, 1), (1, 2), (2, 1), (2, 2), (2, 2), (2, 2), (1, 3), (2, 3), (3, 2), (2, 2), (2, 2), (1, 1), (3, 3)]
    for ci, (sA, sB) in enumerate(cases):
        A = synth.noised_icosphere(sA, 1e-3, 0.15, rng)
        B = synth.noised_icosphere(sB, 1e-3, 0.15, rng)
        pose = synth.pair_poses(rng, 1, 1e-3, 0.0, 0.1)[0]
        if ci == 11:  # far apart: no contact
            pose[7:10] = [5e-3, 0.0, 0.0]
        split = ci % 4 != 3
        Ab, pA = R.build_mesh(A)
        Bb, _ = R.build_mesh(B)
        r = R.pair(Ab, pA[5], pA[6], Bb, pose[:7], pose[7:], split=split)
        d[f"c{ci}_A"] = A
        d[f"c{ci}_B"] = B
        d[f"c{ci}_pose"] = pose
        d[f"c{ci}_split"] = np.array(split)
        pack(f"c{ci}_", r, d)
    d["ncase"] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, "pairs_ref.npz"), **d)


def make_mesh(R):
    rng = np.random.default_rng(7)
    d = {}
    for i, s in enumerate([0, 1, 2]):
        t = synth.noised_icosphere(s, 1e-3, 0.15, rng) + np.array([1e-3, -2e-3, 5e-4])
        out, props = R.build_mesh(t, True)
        d[f"m{i}_in"] = t
        d[f"m{i}_out"] = out
        d[f"m{i}_props"] = props
        out2, props2 = R.build_mesh(t, False)
        d[f"m{i}_out_nc"] = out2
        d[f"m{i}_props_nc"] = props2
    d["nmesh"] = np.array(3)
    np.savez_compressed(os.path.join(HERE, "mesh_ref.npz"), **d)


def make_sort(R):
    rng = np.random.default_rng(11)
    d = {}
    n_cases = 60
    for i in range(n_cases):
        kind = i % 3
        n = int(rng.integers(0, 120))
        ik = rng.integers(0, int(rng.integers(1, 6)), size=max(n, 1)).astype(np.int32)
        dk = rng.integers(0, int(rng.integers(1, 6)), size=max(n, 1)).astype(float)
        d[f"s{i}_kind"] = np.array(kind)
        d[f"s{i}_ikey"] = ik
        d[f"s{i}_dkey"] = dk
        d[f"s{i}_perm"] = R.std_sort(kind, n, ik, dk)
    d["ncase"] = np.array(n_cases)
    np.savez_compressed(os.path.join(HERE, "sort_ref.npz"), **d)


def make_polyline():
    sys.path.insert(0, REF_PY)
    import polyline as P  # the reference module, imported read-only

    rng = np.random.default_rng(99)
    d = {}
    n_cases = 4
    for ci in range(n_cases):
        A = synth.noised_icosphere(1 + ci % 2, 1e-3, 0.15, rng)
        B = synth.noised_icosphere(1, 1e-3, 0.15, rng)
        pose = synth.pair_poses(rng, 1, 1e-3, 0.02, 0.1)[0]
        tol = 1e-5
        trisA = P.transform_points(A.reshape(-1, 3), pose[0:3], pose[3:7]).reshape(-1, 3, 3)
        trisB = P.transform_points(B.reshape(-1, 3), pose[7:10], pose[10:14]).reshape(-1, 3, 3)
        nA_all = P.tri_normals(trisA)
        nB_all = P.tri_normals(trisB)
        planesA = [P.plane_from_tri(trisA[i]) for i in range(len(trisA))]
        planesB = [P.plane_from_tri(trisB[i]) for i in range(len(trisB))]
        aminA, amaxA = trisA.min(axis=1), trisA.max(axis=1)
        aminB, amaxB = trisB.min(axis=1), trisB.max(axis=1)
        segs = []
        for i in range(len(trisA)):
            nAi, dAi = planesA[i]
            if nAi is None:
                continue
            for j in range(len(trisB)):
                if (amaxA[i, 0] < aminB[j, 0] or aminA[i, 0] > amaxB[j, 0] or amaxA[i, 1] < aminB[j, 1] or
                        aminA[i, 1] > amaxB[j, 1] or amaxA[i, 2] < aminB[j, 2] or aminA[i, 2] > amaxB[j, 2]):
                    continue
                nBj, dBj = planesB[j]
                if nBj is None:
                    continue
                s = P.tri_tri_intersection_segment(trisA[i], nA_all[i], dAi, trisB[j], nB_all[j], dBj)
                if s is not None:
                    segs.append(s)
        loops, cids = [], []
        comps = [list(range(len(segs)))]
        for comp in comps:
            V, E = P.snap_endpoints([segs[i] for i in comp], tol=tol)
            V2, E2 = P.split_t_junctions(V, E, tol=tol)
            for lv in P.extract_loops(V2, E2):
                if len(lv) < 3:
                    continue
                pts = [V2[i] for i in lv]
                if np.linalg.norm(np.max(pts, axis=0) - np.min(pts, axis=0)) < tol * 2:
                    continue
                loops.append(np.asarray(pts))
                cids.append(len(cids))
        man = P.build_contacts_from_loops(0, 1, loops, cids, k_stiff=1e7)
        d[f"c{ci}_A"] = A
        d[f"c{ci}_B"] = B
        d[f"c{ci}_pose"] = pose
        d[f"c{ci}_tol"] = np.array(tol)
        d[f"c{ci}_nseg"] = np.array(len(segs))
        d[f"c{ci}_nloop"] = np.array(len(loops))
        d[f"c{ci}_loop_len"] = np.array([len(x) for x in loops], np.int64)
        d[f"c{ci}_loop_pts"] = np.concatenate(loops) if loops else np.zeros((0, 3))
        geo = [c["Sn"] + c["Gn"] + (c["xc0"] or [0, 0, 0]) + c["nA"] + [c["area"], c["Fn"]] + c["F_A"]
               for c in man["contacts"]]
        d[f"c{ci}_geom"] = np.asarray(geo, float).reshape(-1, 17)
    d["ncase"] = np.array(n_cases)
    np.savez_compressed(os.path.join(HERE, "polyline_ref.npz"), **d)


def _vtk_cases(rng):
    """Seeded inputs of the VTK writers: (loops, contact points or None, contact ids) per case."""
    cases = []
    for ci in range(6):
        nloop = int(rng.integers(0, 5))
        loops = []
        for _ in range(nloop):
            m = int(rng.integers(1, 7))  # a loop of one point is skipped by the writer
            base = rng.normal(size=(m, 3)) * 10.0 ** rng.integers(-4, 1)
            if m > 2 and rng.random() < 0.5:
                base[m - 1] = base[0] + rng.choice([3e-10, 3e-9]) * rng.normal(size=3)  # merge or not
            loops.append(base)
        if loops and rng.random() < 0.7:  # a loop sharing points with the previous one
            prev = loops[-1]
            loops.append(prev[::-1] + 1e-10 * rng.normal(size=prev.shape))
        nl = len(loops)
        ncp = nl if ci % 3 != 2 else max(0, nl - 1)
        cps = []
        for k in range(ncp):
            if rng.random() < 0.25:
                cps.append(None)
            elif rng.random() < 0.3 and loops:
                cps.append(loops[k % nl][0] + 2e-10)  # lands on a loop point
            else:
                cps.append(rng.normal(size=3))
        cids = [int(x) for x in rng.integers(-1, 50, size=nl + int(ci == 4))]
        cases.append((loops, cps, cids))
    return cases


def make_vtk():
    sys.path.insert(0, REF_PY)
    import tempfile

    import polyline as P  # the reference module, imported read-only

    rng = np.random.default_rng(7)
    d = {}
    cases = _vtk_cases(rng)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "x.vtk")
        for ci, (loops, cps, cids) in enumerate(cases):
            P.write_vtk_polydata_polylines(path, loops, cps, cids)
            d[f"l{ci}_loop_len"] = np.array([len(x) for x in loops], np.int64)
            d[f"l{ci}_loop_pts"] = np.concatenate(loops) if loops else np.zeros((0, 3))
            d[f"l{ci}_cp_none"] = np.array([c is None for c in cps], bool)
            d[f"l{ci}_cp"] = np.array([np.zeros(3) if c is None else c for c in cps], float).reshape(-1, 3)
            d[f"l{ci}_cids"] = np.array(cids, np.int64)
            d[f"l{ci}_text"] = np.array(open(path, encoding="utf-8").read())
        for ti in range(3):
            n = int(rng.integers(1, 40))
            verts = rng.normal(size=(max(3, n // 2), 3))
            tris = verts[rng.integers(0, len(verts), size=(n, 3))]
            tris[::3] += 4e-10 * rng.normal(size=tris[::3].shape)  # inside the merge
            tris[1::5] += 5e-9  # outside it
            P.write_vtk_polydata_tris(path, tris, comment=f"mesh {ti}")
            d[f"t{ti}_tris"] = tris
            d[f"t{ti}_text"] = np.array(open(path, encoding="utf-8").read())
    d["nloopcase"] = np.array(len(cases))
    d["ntricase"] = np.array(3)
    np.savez_compressed(os.path.join(HERE, "vtk_ref.npz"), **d)


def polyline_pipeline(P, A, B, pose, tol, split):
    """polyline.py main's pipeline (polyline.py:743-822) on mesh-local triangles A, B at pose (14 values),
    recorded as the fixture fields of one case."""
    trisA = P.transform_points(A.reshape(-1, 3), pose[0:3], pose[3:7]).reshape(-1, 3, 3)
    trisB = P.transform_points(B.reshape(-1, 3), pose[7:10], pose[10:14]).reshape(-1, 3, 3)
    nA_all, nB_all = P.tri_normals(trisA), P.tri_normals(trisB)
    planesA = [P.plane_from_tri(trisA[i]) for i in range(len(trisA))]
    planesB = [P.plane_from_tri(trisB[i]) for i in range(len(trisB))]
    aminA, amaxA = trisA.min(axis=1), trisA.max(axis=1)
    aminB, amaxB = trisB.min(axis=1), trisB.max(axis=1)
    segs = []
    for i in range(len(trisA)):
        nAi, dAi = planesA[i]
        if nAi is None:
            continue
        for j in range(len(trisB)):
            if (amaxA[i, 0] < aminB[j, 0] or aminA[i, 0] > amaxB[j, 0] or amaxA[i, 1] < aminB[j, 1] or
                    aminA[i, 1] > amaxB[j, 1] or amaxA[i, 2] < aminB[j, 2] or aminA[i, 2] > amaxB[j, 2]):
                continue
            nBj, dBj = planesB[j]
            if nBj is None:
                continue
            sg = P.tri_tri_intersection_segment(trisA[i], nA_all[i], dAi, trisB[j], nB_all[j], dBj)
            if sg is not None:
                segs.append(sg)
    if split:
        _, ncomp, comps = P.label_segments_by_contact_greedy(segs, tol=tol) if segs else (None, 0, [])
    else:
        ncomp, comps = (1, [list(range(len(segs)))]) if segs else (0, [])
    loops, comp_of, comp_sz = [], [], []
    for c, comp in enumerate(comps):
        comp_sz.append(len(comp))
        V, E = P.snap_endpoints([segs[i] for i in comp], tol=tol)
        V2, E2 = P.split_t_junctions(V, E, tol=tol)
        for lv in P.extract_loops(V2, E2):
            if len(lv) < 3:
                continue
            pts = [V2[i] for i in lv]
            if np.linalg.norm(np.max(pts, axis=0) - np.min(pts, axis=0)) < tol * 2:
                continue
            loops.append(np.asarray(pts))
            comp_of.append(c)
    man = P.build_contacts_from_loops(0, 1, loops, list(range(len(loops))), k_stiff=1e7)
    geo = [c["Sn"] + c["Gn"] + (c["xc0"] or [0, 0, 0]) + c["nA"] + [c["area"], c["Fn"]] + c["F_A"]
           for c in man["contacts"]]
    return {"A": A, "B": B, "pose": pose, "tol": np.array(tol), "split": np.array(int(split)),
            "nseg": np.array(len(segs)), "ncomp": np.array(ncomp), "comp_sz": np.array(comp_sz, np.int64),
            "loop_comp": np.array(comp_of, np.int64), "loop_len": np.array([len(x) for x in loops], np.int64),
            "loop_pts": np.concatenate(loops) if loops else np.zeros((0, 3)),
            "geom": np.asarray(geo, float).reshape(-1, 17)}


def make_polyline_split():
    sys.path.insert(0, REF_PY)
    import polyline as P  # the reference module, imported read-only

    rng = np.random.default_rng(123)
    d = {}
    n_cases = 6
    for ci in range(n_cases):
        A = synth.noised_icosphere(2, 1e-3, 0.15, rng)
        # B: two or three blobs around A, so that the contact splits
        nb = 2 + ci % 2
        blobs = []
        for b in range(nb):
            u = synth.random_dirs(rng, 1)[0]
            blobs.append(synth.noised_icosphere(1 + (b + ci) % 2, 0.6e-3, 0.1, rng) + u * rng.uniform(1.35e-3, 1.5e-3))
        B = np.concatenate(blobs)
        q = synth.random_unit_quat(rng)
        pose = np.r_[rng.normal(size=3) * 1e-5, q, np.zeros(3), [1.0, 0.0, 0.0, 0.0]]
        for k, v in polyline_pipeline(P, A, B, pose, 1e-5, True).items():
            if k != "split":
                d[f"c{ci}_{k}"] = v
    d["ncase"] = np.array(n_cases)
    np.savez_compressed(os.path.join(HERE, "polyline_split_ref.npz"), **d)


def _t_junction_box(a):
    """A cube of side a whose top face has a T-junction: one of its two triangles is split at the
    midpoint of the shared diagonal, the other is not."""
    from _dem_helpers import box_tris

    tris = [t for t in box_tris(a, a, a) if not np.allclose(t[:, 2], a / 2)]
    h = a / 2
    v0, v1, v2, v3 = np.array([[-h, -h, h], [h, -h, h], [h, h, h], [-h, h, h]])
    m = (v0 + v2) / 2
    tris += [np.array([v0, v1, m]), np.array([m, v1, v2]), np.array([v0, v2, v3])]
    return np.asarray(tris)


def _hard_cases(rng):
    """(name, A, B, pose, tol, split): contacts of flat faces and sharp edges, where segments meet at
    triangle corners, run along edges or lie in coplanar faces."""
    from _dem_helpers import box_tris

    a = 1e-3
    cube = box_tris(a, a, a)
    ident = [1.0, 0.0, 0.0, 0.0]
    qz45 = [np.cos(np.pi / 8), 0.0, 0.0, np.sin(np.pi / 8)]
    qtilt = synth.random_unit_quat(rng)
    sphere = synth.noised_icosphere(2, 0.6e-3, 0.0, rng)
    rough = synth.noised_icosphere(2, 0.6e-3, 0.15, rng)
    hullA = synth.ellipsoid_hull(64, (1.0, 0.8, 0.6), 1e-3, rng)
    hullB = synth.ellipsoid_hull(64, (1.0, 0.8, 0.6), 1e-3, rng)
    tbox = _t_junction_box(a)
    P = lambda tA, qA, tB, qB: np.r_[tA, qA, tB, qB].astype(float)
    cases = [
        ("cubes_offset", cube, cube, P([0, 0, 0], ident, [0.6 * a, 0.3 * a, 0.2 * a], ident)),
        ("cubes_coplanar", cube, cube, P([0, 0, 0], ident, [0.5 * a, 0, 0], ident)),
        ("cubes_rotated", cube, cube, P([0, 0, 0], ident, [0.8 * a, 0.1 * a, 0.05 * a], qz45)),
        ("cubes_tilted", cube, cube, P([0, 0, 0], ident, [0.9 * a, 0.2 * a, -0.1 * a], qtilt)),
        ("sphere_in_cube_face", cube, sphere, P([0, 0, 0], ident, [0.0, 0.0, 0.9e-3], ident)),
        ("sphere_on_cube_edge", cube, rough, P([0, 0, 0], ident, [0.85e-3, 0.0, 0.85e-3], qtilt)),
        ("hulls", hullA, hullB, P([0, 0, 0], ident, [1.7e-3, 0.2e-3, 0.0], qtilt)),
        ("t_junction_box", tbox, sphere, P([0, 0, 0], ident, [0.05e-3, 0.05e-3, 0.95e-3], ident)),
        ("grazing_spheres", rough, sphere, P([0, 0, 0], ident, [0.0, 0.0, 1.1995e-3], qtilt)),
    ]
    out = []
    for name, A, B, pose in cases:
        for tol, split in ((1e-6, False), (1e-5, True)):
            out.append((name, A, B, pose, tol, split))
    return out


def make_polyline_hard():
    sys.path.insert(0, REF_PY)
    sys.path.insert(0, os.path.dirname(HERE))
    import polyline as P  # the reference module, imported read-only

    rng = np.random.default_rng(321)
    d = {}
    cases = _hard_cases(rng)
    for ci, (name, A, B, pose, tol, split) in enumerate(cases):
        d[f"c{ci}_name"] = np.array(name)
        for k, v in polyline_pipeline(P, np.asarray(A, float), np.asarray(B, float), pose, tol, split).items():
            d[f"c{ci}_{k}"] = v
    d["ncase"] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, "polyline_hard_ref.npz"), **d)


CLI_CASES = [
    # (name, mesh A spec, mesh B spec, extra argv); a spec is a list of (subdivision, centre) blobs
    ("plain", [(2, (0, 0, 0))], [(2, (0, 0, 0))], ["--tB", "1.9e-3", "1e-4", "0", "--qB", "0.9", "0.1", "0.3", "0.2",
                                                  "--k", "1e7"]),
    ("split", [(2, (0, 0, 0))], [(1, (0, 1.7e-3, 0)), (1, (0, -1.7e-3, 0))],
     ["--tA", "1e-4", "0", "0", "--qA", "1", "0.05", "0", "0", "--split-contacts", "--tol", "1e-5"]),
    ("apart", [(1, (0, 0, 0))], [(1, (0, 0, 0))], ["--tB", "5e-3", "0", "0"]),
    ("snapped_away", [(1, (0, 0, 0))], [(1, (0, 0, 0))], ["--tB", "1.8e-3", "0", "0", "--tol", "1e-2"]),
]


def cli_mesh(spec, rng):
    """Triangles of a union of noised icospheres of radius 1 mm, rounded to float32 as in a binary STL."""
    parts = [synth.noised_icosphere(sub, 1e-3, 0.1, rng) + np.asarray(c, float) for sub, c in spec]
    return np.concatenate(parts).astype(np.float32).astype(np.float64)


def make_cli():
    sys.path.insert(0, REF_PY)
    sys.path.insert(0, os.path.dirname(HERE))
    import contextlib
    import io
    import tempfile

    import polyline as P  # the reference module, imported read-only
    from _dem_helpers import write_binary_stl

    rng = np.random.default_rng(11)
    d = {}
    cwd = os.getcwd()
    for ci, (name, sa, sb, extra) in enumerate(CLI_CASES):
        A, B = cli_mesh(sa, rng), cli_mesh(sb, rng)
        with tempfile.TemporaryDirectory() as tmp:
            os.chdir(tmp)
            try:
                write_binary_stl("A.stl", A)
                write_binary_stl("B.stl", B)
                argv = ["A.stl", "B.stl"] + extra
                old = sys.argv
                sys.argv = ["polyline.py"] + argv
                buf = io.StringIO()
                try:
                    with contextlib.redirect_stdout(buf):
                        P.main()
                finally:
                    sys.argv = old
                files = {}
                for f in ("A_transformed.vtk", "B_transformed.vtk", "routeB_intersection.vtk"):
                    files[f] = open(f, encoding="utf-8").read() if os.path.exists(f) else ""
            finally:
                os.chdir(cwd)
        d[f"c{ci}_name"] = np.array(name)
        d[f"c{ci}_A"] = A
        d[f"c{ci}_B"] = B
        d[f"c{ci}_argv"] = np.array(" ".join(argv))
        d[f"c{ci}_stdout"] = np.array(buf.getvalue())
        d[f"c{ci}_vtkA"] = np.array(files["A_transformed.vtk"])
        d[f"c{ci}_vtkB"] = np.array(files["B_transformed.vtk"])
        d[f"c{ci}_loops"] = np.array(files["routeB_intersection.vtk"])
    d["ncase"] = np.array(len(CLI_CASES))
    np.savez_compressed(os.path.join(HERE, "cli_ref.npz"), **d)


if __name__ == "__main__":
    only = set(sys.argv[1:])
    want = lambda name: not only or name in only
    if want("pairs") or want("mesh") or want("sort"):
        R = Reference()
        if want("pairs"):
            make_pairs(R)
        if want("mesh"):
            make_mesh(R)
        if want("sort"):
            make_sort(R)
    if want("polyline"):
        make_polyline()
    if want("polyline_split"):
        make_polyline_split()
    if want("polyline_hard"):
        make_polyline_hard()
    if want("vtk"):
        make_vtk()
    if want("cli"):
        make_cli()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
