"""Drop-in mirror of the reference's pair-contact module polyline.py, computed on the GPU.

Same names, arguments and error behaviour as polyline.py: ``load_stl`` raises ``ValueError`` on a bad
file, ``pair_contacts`` returns the ContactManifold dict of ``build_contacts_from_loops``
(polyline.py:655-701), the VTK writers produce the same files, and ``main`` is the same command line
(polyline.py:707-834).  The geometry (triangle tests, components, snap, T-junction split, loop trace,
Sn/Gn/xc0 and the minimal law Fn = k/2 |Sn|) runs in libzdemx.so; there is no CPU path.

Semantics follow polyline.py, not zdem_cpu: the tolerance is the --tol argument (default 1e-6), loops
are dropped when shorter than 3 vertices or when their bounding-box diagonal is below 2 tol, sorts are
stable, nA = -Sn/|Sn| is not flipped, and a loop with |Sn| < 1e-14 is still a contact with xc0 None.
With --split-contacts, polyline.py visits each segment's candidates in the iteration order of a Python
set of ints; the kernel rebuilds CPython 3.12's set table to visit them in the same order, so loops
start, run and are numbered as polyline.py's.

The pair call computes in numpy's own arithmetic by default (``_lib.MODE_POLYLINE_NUMPY``: numpy's
dot and norm chains, zdx_npmath.cuh), so the numbers, stdout and VTK files are polyline.py's bit for
bit; ``mode=_lib.MODE_POLYLINE`` follows the reference C++ program's arithmetic instead (the same loops,
numbers within 1e-9 of polyline.py's).
"""
from __future__ import annotations

import argparse
import os
import struct

import numpy as np

from . import _lib

__all__ = ["load_stl", "quat_normalize", "quat_rotate", "transform_points", "tri_normals", "pair_contacts",
           "build_contacts_from_loops", "write_vtk_polydata_tris", "write_vtk_polydata_polylines", "main"]

_CTX = None


def _ctx():
    global _CTX
    if _CTX is None:
        _CTX = _lib.Context(int(os.environ.get("ZDEMX_DEVICE", "0")))
    return _CTX


# ---------------------------------------------------------------- host helpers (polyline.py:36-106)
def quat_normalize(q):
    q = np.asarray(q, dtype=float)
    n = np.linalg.norm(q)
    if n < 1e-30:
        return np.array([1.0, 0.0, 0.0, 0.0])
    return q / n


def quat_rotate(q, v):
    q = quat_normalize(q)
    w, x, y, z = q
    v = np.asarray(v, dtype=float)
    qv = np.array([x, y, z], dtype=float)
    t = 2.0 * np.cross(qv, v)
    return v + w * t + np.cross(qv, t)


def transform_points(pts, t, q):
    pts = np.asarray(pts, dtype=float)
    return quat_rotate(q, pts) + np.asarray(t, dtype=float)


def load_stl(path):
    """Binary when the size is exactly 84 + 50 n, ASCII otherwise; ValueError when neither parses."""
    with open(path, "rb") as f:
        f.read(80)
        nb = f.read(4)
        if len(nb) < 4:
            raise ValueError("Invalid STL.")
        n_tri = struct.unpack("<I", nb)[0]
        if 84 + n_tri * 50 == os.path.getsize(path):
            return _lib.stl_load(path)
    tris = []
    with open(path, "r", encoding="utf-8", errors="ignore") as f:
        vs = []
        for line in f:
            s = line.strip().lower()
            if s.startswith("vertex"):
                parts = s.split()
                if len(parts) >= 4:
                    vs.append([float(parts[1]), float(parts[2]), float(parts[3])])
            if s.startswith("endloop") and len(vs) >= 3:
                tris.append(vs[-3:])
    if not tris:
        raise ValueError("Failed to parse STL (neither binary nor ascii).")
    return np.array(tris, dtype=float)


def tri_normals(tris):
    e1 = tris[:, 1] - tris[:, 0]
    e2 = tris[:, 2] - tris[:, 0]
    n = np.cross(e1, e2)
    ln = np.linalg.norm(n, axis=1)
    good = ln > 1e-30
    n[good] /= ln[good][:, None]
    return n


# ---------------------------------------------------------------- the pair call
def pair_contacts(trisA, trisB, tA=(0.0, 0.0, 0.0), qA=(1.0, 0.0, 0.0, 0.0), tB=(0.0, 0.0, 0.0),
                  qB=(1.0, 0.0, 0.0, 0.0), k=1.0, tol=1e-6, split_contacts=False, idA=0, idB=1, ctx=None,
                  mode=_lib.MODE_POLYLINE_NUMPY):
    """Contacts between mesh A at pose (tA, qA) and mesh B at (tB, qB), as polyline.py main computes
    them (polyline.py:743-829).  Returns (manifold, loops_pts, xc0s, contact_ids): manifold is the dict
    of build_contacts_from_loops (polyline.py:681-701), the rest what main passes to its writers.
    tol=None takes the snap tolerance as the zdem_cpu step does, from A's mean edge length
    (src/main.cpp:2118-2121: 0.1 mean edge, else 1 % of the bounding-box diagonal, else 1e-6).
    mode: _lib.MODE_POLYLINE_NUMPY (numpy's arithmetic, polyline.py's numbers bit for bit) or
    _lib.MODE_POLYLINE (the C++ program's arithmetic)."""
    if tol is None:
        tol = _mean_edge_tol(trisA)
    return _pair_call(trisA, trisB, tA, qA, tB, qB, k, tol, split_contacts, idA, idB, ctx, mode=mode)[:4]


def _mean_edge_tol(tris) -> float:
    """The snap tolerance rule of src/main.cpp:2118-2121 on build_mesh's mean edge and bbox diagonal."""
    _, props = _lib.mesh_build(np.asarray(tris, dtype=float), False)
    me, bd = props["mean_edge"], props["bbox_diag"]
    tol = me * 0.1 if me > 0.0 else bd * 1e-2
    return tol if tol > 0.0 else 1e-6


# components recorded by the command line: at most one per segment, and a pair holds at most the
# library's default segment capacity
_COMP_CAP = 16384


def _pair_call(trisA, trisB, tA, qA, tB, qB, k, tol, split_contacts, idA, idB, ctx, comp_cap=0,
               mode=_lib.MODE_POLYLINE_NUMPY):
    """pair_contacts, plus the pair's segment and component counts and (comp_cap > 0) the per-component
    counts (segments, snapped vertices, edges, loops) main prints."""
    A = np.ascontiguousarray(trisA, dtype=float).reshape(-1, 3, 3)
    B = np.ascontiguousarray(trisB, dtype=float).reshape(-1, 3, 3)
    tris = np.concatenate([A.reshape(-1), B.reshape(-1)])
    off = np.array([0, len(A), len(A) + len(B)], np.int64)
    pose = np.concatenate([np.asarray(tA, float), np.asarray(qA, float), np.asarray(tB, float), np.asarray(qB, float)])
    r = _lib.pair_contacts_raw(ctx or _ctx(), tris, off, np.zeros(2), np.zeros(2), np.array([[0, 1]], np.int32),
                               pose[None, :], mode=mode, split=split_contacts, tol=tol, k=k,
                               want_points=True, comp_cap=comp_cap)
    loops, xc0s, cids = [], [], []
    for c in range(len(r["geom"])):
        pts = r["points"][r["point_off"][c]: r["point_off"][c + 1]]
        loops.append([p.copy() for p in pts])
        g = r["geom"][c]
        xc0s.append(None if g[12] == 0.0 else g[6:9].copy())
        cids.append(int(r["info"][c, 1]))
    manifold = _manifold(idA, idB, r["geom"], r["info"], k)
    nseg, ncomp = int(r["stats"][0, 0]), int(r["stats"][0, 1])
    comps = None
    if comp_cap > 0:
        # (segments, snapped vertices, edges, loops) per component; its loops are its contacts
        nloop = np.bincount(r["info"][:, 3], minlength=ncomp)[:ncomp]
        comps = [tuple(int(x) for x in r["comp_stats"][0, c]) + (int(nloop[c]),) for c in range(ncomp)]
    return manifold, loops, xc0s, cids, nseg, ncomp, comps


def _manifold(idA, idB, geom, info, k):
    contacts = []
    for c in range(len(geom)):
        g = geom[c]
        degenerate = g[12] == 0.0
        contacts.append({
            "idA": idA, "idB": idB, "cid": int(info[c, 1]), "nVert": int(info[c, 2]),
            "Sn": g[0:3].tolist(), "Gn": g[3:6].tolist(), "area": float(g[12]),
            "nA": g[9:12].tolist(), "nB": (-g[9:12]).tolist(),
            "xc0": None if degenerate else g[6:9].tolist(),
            "k": float(k), "Fn": float(g[13]), "F_A": g[14:17].tolist(), "F_B": g[17:20].tolist(),
        })
    return {"idA": idA, "idB": idB, "contacts": contacts}


def build_contacts_from_loops(idA, idB, loops_pts, contact_ids, k_stiff=1.0):
    """polyline.py:655-701 for loops that are already known; the Route-B sums run on the GPU path only
    through pair_contacts, so this host form is kept for callers that hand in their own loops."""
    contacts = []
    k_stiff = float(k_stiff)
    for k, loop in enumerate(loops_pts):
        P = np.asarray(loop, float)
        m = len(P)
        Sn = np.zeros(3)
        Gn = np.zeros(3)
        for i in range(m):
            p0, p1 = P[i], P[(i + 1) % m]
            Sn += 0.5 * np.cross(p0, p1)
            dx = p1 - p0
            s = np.dot(p0, p1) + (1.0 / 3.0) * np.dot(dx, dx)
            Gn += -(1.0 / 3.0) * s * dx
        a = float(np.linalg.norm(Sn))
        if a < 1e-14:
            xc0, nA, area = None, np.zeros(3), 0.0
        else:
            nA = -Sn / a
            xc0, area = np.cross(nA, Gn) / a, a
        Fn = 0.5 * k_stiff * float(area)
        FA = (Fn * np.asarray(nA, float)).tolist()
        contacts.append({"idA": idA, "idB": idB, "cid": int(contact_ids[k]), "nVert": int(m), "Sn": Sn.tolist(),
                         "Gn": Gn.tolist(), "area": float(area), "nA": nA.tolist(), "nB": (-nA).tolist(),
                         "xc0": None if xc0 is None else xc0.tolist(), "k": k_stiff, "Fn": float(Fn), "F_A": FA,
                         "F_B": (-np.asarray(FA, float)).tolist()})
    return {"idA": idA, "idB": idB, "contacts": contacts}


# ---------------------------------------------------------------- VTK writers (polyline.py:544-649)
class _PointSet:
    """Point list with the writer's 1e-9 merge (a linear scan, like polyline.py, so ids match)."""

    def __init__(self):
        self.pts = []

    def add(self, p):
        p = np.asarray(p, float)
        if self.pts:
            arr = np.asarray(self.pts)
            d = np.linalg.norm(arr - p[None, :], axis=1)
            hit = np.nonzero(d < 1e-9)[0]
            if len(hit):
                return int(hit[0])
        self.pts.append(p.copy())
        return len(self.pts) - 1


def write_vtk_polydata_tris(path, tris, comment="mesh"):
    ps = _PointSet()
    faces = [[ps.add(t[0]), ps.add(t[1]), ps.add(t[2])] for t in tris]
    with open(path, "w", encoding="utf-8") as f:
        f.write("# vtk DataFile Version 3.0\n")
        f.write(f"{comment}\n")
        f.write("ASCII\n")
        f.write("DATASET POLYDATA\n")
        f.write(f"POINTS {len(ps.pts)} float\n")
        for p in ps.pts:
            f.write(f"{p[0]} {p[1]} {p[2]}\n")
        f.write(f"POLYGONS {len(faces)} {len(faces) * 4}\n")
        for a, b, c in faces:
            f.write(f"3 {a} {b} {c}\n")


def write_vtk_polydata_polylines(path, loops_pts, contact_points, loop_contact_ids):
    """Each loop one LINE cell (closed by repeating its first point), each xc0 one VERTEX cell, and
    CELL_DATA contact_id over all cells."""
    ps = _PointSet()
    line_cells = []
    for loop in loops_pts:
        ids = [ps.add(p) for p in loop]
        if len(ids) < 2:
            continue
        ids.append(ids[0])
        line_cells.append(ids)
    vtx_ids = [ps.add(cp) for cp in contact_points if cp is not None]
    n_lines, n_verts = len(line_cells), len(vtx_ids)
    cell_ids = [int(c) for c in loop_contact_ids[:n_lines]]
    if len(contact_points) == n_lines:
        cell_ids += [int(c) for c in loop_contact_ids[:n_lines]]
    else:
        cell_ids += [-1] * n_verts
    with open(path, "w", encoding="utf-8") as f:
        f.write("# vtk DataFile Version 3.0\n")
        f.write("reconstructed_contact_loops\n")
        f.write("ASCII\n")
        f.write("DATASET POLYDATA\n")
        f.write(f"POINTS {len(ps.pts)} float\n")
        for p in ps.pts:
            f.write(f"{p[0]} {p[1]} {p[2]}\n")
        total_ints = sum(1 + len(ids) for ids in line_cells)
        f.write(f"LINES {n_lines} {total_ints}\n")
        for ids in line_cells:
            f.write(str(len(ids)) + " " + " ".join(str(i) for i in ids) + "\n")
        if n_verts > 0:
            f.write(f"VERTICES {n_verts} {n_verts * 2}\n")
            for vid in vtx_ids:
                f.write(f"1 {vid}\n")
        f.write(f"\nCELL_DATA {n_lines + n_verts}\n")
        f.write("SCALARS contact_id int 1\n")
        f.write("LOOKUP_TABLE default\n")
        for cid in cell_ids:
            f.write(f"{cid}\n")


# ---------------------------------------------------------------- command line (polyline.py:707-834)
def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("stlA")
    ap.add_argument("stlB")
    ap.add_argument("--tA", nargs=3, type=float, default=[0.0, 0.0, 0.0])
    ap.add_argument("--qA", nargs=4, type=float, default=[1.0, 0.0, 0.0, 0.0])
    ap.add_argument("--tB", nargs=3, type=float, default=[0.0, 0.0, 0.0])
    ap.add_argument("--qB", nargs=4, type=float, default=[1.0, 0.0, 0.0, 0.0])
    ap.add_argument("--split-contacts", action="store_true",
                    help="coarsely split into components before loop reconstruction")
    ap.add_argument("--tol", type=float, default=1e-6, help="snap / adjacency tolerance (try 1e-5 if needed)")
    ap.add_argument("--k", type=float, default=1.0,
                    help="contact stiffness parameter k for minimal energy model (paper-consistent): Fn = 0.5*k*|Sn|")
    ap.add_argument("--vtk", default="routeB_intersection.vtk")
    ap.add_argument("--outA", default="A_transformed.vtk")
    ap.add_argument("--outB", default="B_transformed.vtk")
    return ap.parse_args(argv)


def main(argv=None):
    args = parse_args(argv)
    trisA0 = load_stl(args.stlA)
    trisB0 = load_stl(args.stlB)
    trisA = transform_points(trisA0.reshape(-1, 3), args.tA, args.qA).reshape(-1, 3, 3)
    trisB = transform_points(trisB0.reshape(-1, 3), args.tB, args.qB).reshape(-1, 3, 3)
    write_vtk_polydata_tris(args.outA, trisA, comment="Mesh A (transformed)")
    write_vtk_polydata_tris(args.outB, trisB, comment="Mesh B (transformed)")
    print(f"Transformed meshes written: {args.outA}, {args.outB}")
    manifold, loops, xc0s, cids, nseg, ncomp, comps = _pair_call(
        trisA0, trisB0, args.tA, args.qA, args.tB, args.qB, args.k, args.tol, args.split_contacts, 0, 1, None,
        comp_cap=_COMP_CAP)
    if nseg == 0:
        print("No intersection segments found.")
        return
    print(f"Raw intersection segments: {nseg}")
    tol = float(args.tol)
    if args.split_contacts:
        print(f"Coarse components: {ncomp} (tol={tol})")
    else:
        print("Coarse components: 1 (no split)")
    c = 0
    for comp_idx, (raw_seg, snapped_v, edges, nloop) in enumerate(comps):
        print(f"\n[Component {comp_idx}] rawSeg={raw_seg} snappedV={snapped_v} edges={edges} loops={nloop}")
        for _ in range(nloop):
            cc, x = manifold["contacts"][c], xc0s[c]
            print(f"  [Contact {cc['cid']}] nVert={len(loops[c])} |Sn|={cc['area']}")
            print(f"    nA={cc['nA']}")
            print(f"    xc(0)={None if x is None else x.tolist()}")
            c += 1
    write_vtk_polydata_polylines(args.vtk, loops, xc0s, cids)
    print(f"\nReconstructed-loop VTK written: {args.vtk}")
    print('ParaView: color by CELL "contact_id". Each loop is one polyline cell.')
    print("\n=== DEM ContactManifold ===")
    print(f"idA={manifold['idA']} idB={manifold['idB']} nContact={len(manifold['contacts'])}")
    for c in manifold["contacts"]:
        print(f"  [cid={c['cid']}] nVert={c['nVert']} area={c['area']} Fn={c['Fn']}")
        print(f"    nA={c['nA']} xc0={c['xc0']} F_A={c['F_A']}")


if __name__ == "__main__":
    main()
