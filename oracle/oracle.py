"""ctypes bindings of the two checkers.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``    -> oracle/liboracle.so, the C restatement of the contact path (zdx_oracle.c).
* ``Reference`` -> oracle/_ref/libzdem_ref.so, the reference's own src/main.cpp compiled unchanged.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU baseline leg import this module, and only to
check or time against the CUDA path.  The product (zedm-x_b200/) never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libzdem_ref.so")
LIB_REF_HIPREC = os.path.join(HERE, "_ref", "libzdem_ref_hiprec.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

_COMMON = [
    ("tri_checks", C.c_int64), ("nseg", C.c_int), ("seg", _dp), ("ncomp", C.c_int), ("comp_off", _ip),
    ("comp_idx", _ip), ("v_off", _ip), ("V", _dp), ("e_off", _ip), ("E", _ip), ("e2_off", _ip), ("E2", _ip),
    ("nloop", C.c_int), ("loop_comp", _ip), ("loop_off", _ip), ("loop_vid", _ip), ("loop_status", _ip),
    ("loop_geom", _dp),
]


class _RefOut(C.Structure):
    _fields_ = _COMMON


class _OracleOut(C.Structure):
    _fields_ = _COMMON + [("ncontact", C.c_int), ("contact_loop", _ip), ("tol", C.c_double)]


LOOP_SHORT, LOOP_TINY, LOOP_SMALL, LOOP_ACCEPT, LOOP_BBOX, LOOP_DEGEN = range(6)

_i64p = C.POINTER(C.c_int64)


class _ZoScene(C.Structure):
    _fields_ = [("nmesh", C.c_int), ("mesh_tris", _dp), ("mesh_off", _i64p), ("mesh_props", _dp), ("np", C.c_int),
                ("p_mesh", _ip), ("p_state", _dp), ("p_mat", _dp), ("nwall", C.c_int), ("w_mesh", _ip),
                ("w_pose", _dp), ("w_mat", _dp), ("gravity", C.c_double * 3), ("dt", C.c_double),
                ("split_contacts", C.c_int), ("nhist", C.c_int), ("hist_key", _i64p), ("hist_ds", _dp),
                ("nwhist", C.c_int), ("whist_key", _i64p), ("whist_ds", _dp), ("force", _dp), ("torque", _dp),
                ("contact_count", _ip), ("contacts", C.c_int), ("loops", C.c_int), ("comps", C.c_int),
                ("segments", C.c_int), ("tri_checks", C.c_int64)]


# ---- zdem_cpu's particle set-up (src/main.cpp:1936-1987), in Python floats (IEEE doubles) with the
# reference's operation order, so that the scene handed to zo_dem_step is the reference's to the bit
def _quat_normalize(q):
    n = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    if n < 1e-14:
        return (1.0, 0.0, 0.0, 0.0)
    return (q[0] / n, q[1] / n, q[2] / n, q[3] / n)


def _quat_to_mat3(q):  # src/main.cpp:150-163
    w, x, y, z = _quat_normalize(q)
    return [[1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w)],
            [2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w)],
            [2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)]]


def _mat3_mul(a, b):  # src/main.cpp:173-184
    r = [[0.0] * 3 for _ in range(3)]
    for i in range(3):
        for j in range(3):
            acc = 0.0
            for k in range(3):
                acc += a[i][k] * b[k][j]
            r[i][j] = acc
    return r


def _mat3_inverse(a):  # src/main.cpp:196-217
    det = (a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0])
           + a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]))
    if abs(det) < 1e-18:
        return [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]
    inv = 1.0 / det
    return [[(a[1][1] * a[2][2] - a[1][2] * a[2][1]) * inv, -(a[0][1] * a[2][2] - a[0][2] * a[2][1]) * inv,
             (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * inv],
            [-(a[1][0] * a[2][2] - a[1][2] * a[2][0]) * inv, (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * inv,
             -(a[0][0] * a[1][2] - a[0][2] * a[1][0]) * inv],
            [(a[1][0] * a[2][1] - a[1][1] * a[2][0]) * inv, -(a[0][0] * a[2][1] - a[0][1] * a[2][0]) * inv,
             (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * inv]]


class DemScene:
    """A zdem_cpu scene for zo_dem_step (the oracle's DEM step, src/main.cpp:2034-2468).  particles: dicts
    with tris (raw, as loaded), scale, pos, quat, vel, omega, density, young, poisson, mu, restitution;
    walls: dicts with tris, scale, pos, quat, mu, restitution.  Meshes are built with the oracle's
    build_mesh; masses, inertias and L0 as src/main.cpp:1936-1987."""

    def __init__(self, oracle, particles, walls=(), gravity=(0.0, 0.0, 0.0), dt=1e-6, split=True, center=True):
        self.o = oracle
        tris, offs, props = [], [0], []

        def add_mesh(t, scale):
            t = np.asarray(t, float).reshape(-1, 3, 3) * float(scale)
            out, pr = oracle.build_mesh(t, center)
            tris.append(out.reshape(-1, 9))
            offs.append(offs[-1] + len(out))
            props.append(pr)
            return len(props) - 1

        p_mesh, state, mat = [], [], []
        for p in particles:
            m = add_mesh(p["tris"], p.get("scale", 1.0))
            pr = props[m]
            vol, radius = float(pr[0]), float(pr[4])
            dens = float(p.get("density", 1.0))
            dens = dens if dens > 0.0 else 1.0
            if vol > 0.0:
                mass = dens * vol
                Ib = [[float(pr[7 + 3 * i + j]) * dens for j in range(3)] for i in range(3)]
            else:
                mass = dens
                I = 0.4 * mass * radius * radius
                Ib = [[I, 0.0, 0.0], [0.0, I, 0.0], [0.0, 0.0, I]]
            Ibi = _mat3_inverse(Ib)
            eq = math.cbrt(3.0 * vol / (4.0 * 3.141592653589793)) if vol > 0.0 else radius
            q = [float(x) for x in p.get("quat", (1.0, 0.0, 0.0, 0.0))]
            om = [float(x) for x in p.get("omega", (0.0, 0.0, 0.0))]
            R = _quat_to_mat3(q)
            Rt = [[R[j][i] for j in range(3)] for i in range(3)]
            Iw = _mat3_mul(_mat3_mul(R, Ib), Rt)
            L = [Iw[i][0] * om[0] + Iw[i][1] * om[1] + Iw[i][2] * om[2] for i in range(3)]
            p_mesh.append(m)
            state.append(list(map(float, p.get("pos", (0, 0, 0)))) + q + list(map(float, p.get("vel", (0, 0, 0))))
                         + om + L)
            mat.append([mass, 1.0 / mass, radius, eq, float(p.get("young", 1e7)), float(p.get("poisson", 0.25)),
                        float(p.get("mu", 0.5)), float(p.get("restitution", 0.5))] + [Ibi[i][j] for i in range(3)
                                                                                    for j in range(3)])
        w_mesh, w_pose, w_mat = [], [], []
        for w in walls:
            w_mesh.append(add_mesh(w["tris"], w.get("scale", 1.0)))
            w_pose.append(list(map(float, w.get("pos", (0, 0, 0)))) + list(map(float, w.get("quat", (1, 0, 0, 0)))))
            w_mat.append([float(w.get("mu", 0.5)), float(w.get("restitution", 0.5))])
        n = len(particles)
        self.mesh_tris = np.ascontiguousarray(np.concatenate(tris) if tris else np.zeros((0, 9)))
        self.mesh_off = np.asarray(offs, np.int64)
        self.mesh_props = np.ascontiguousarray(np.asarray(props, float).reshape(-1, 17))
        self.p_mesh = np.asarray(p_mesh, np.int32)
        self.state = np.ascontiguousarray(np.asarray(state, float).reshape(-1, 16))
        self.mat = np.ascontiguousarray(np.asarray(mat, float).reshape(-1, 17))
        self.w_mesh = np.asarray(w_mesh or [0], np.int32)
        self.w_pose = np.ascontiguousarray(np.asarray(w_pose or [[0] * 7], float))
        self.w_mat = np.ascontiguousarray(np.asarray(w_mat or [[0, 0]], float))
        self.force = np.zeros((max(n, 1), 3))
        self.torque = np.zeros((max(n, 1), 3))
        self.count = np.zeros(max(n, 1), np.int32)
        sc = _ZoScene()
        sc.nmesh = len(props)
        sc.mesh_tris = self.mesh_tris.ctypes.data_as(_dp)
        sc.mesh_off = self.mesh_off.ctypes.data_as(_i64p)
        sc.mesh_props = self.mesh_props.ctypes.data_as(_dp)
        sc.np = n
        sc.p_mesh = self.p_mesh.ctypes.data_as(_ip)
        sc.p_state = self.state.ctypes.data_as(_dp)
        sc.p_mat = self.mat.ctypes.data_as(_dp)
        sc.nwall = len(walls)
        sc.w_mesh = self.w_mesh.ctypes.data_as(_ip)
        sc.w_pose = self.w_pose.ctypes.data_as(_dp)
        sc.w_mat = self.w_mat.ctypes.data_as(_dp)
        for k in range(3):
            sc.gravity[k] = float(gravity[k])
        sc.dt = float(dt)
        sc.split_contacts = int(bool(split))
        sc.force = self.force.ctypes.data_as(_dp)
        sc.torque = self.torque.ctypes.data_as(_dp)
        sc.contact_count = self.count.ctypes.data_as(_ip)
        self.sc = sc

    def step(self, n=1):
        for _ in range(n):
            self.o.lib.zo_dem_step(C.byref(self.sc))
        s = self.sc
        return {"contacts": s.contacts, "tri_checks": int(s.tri_checks), "segments": s.segments, "comps": s.comps,
                "loops": s.loops}

    def __del__(self):
        try:
            self.o.lib.zo_scene_free_history(C.byref(self.sc))
        except Exception:
            pass


def _arr(ptr, n, dtype):
    if n <= 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def _unpack(o) -> dict:
    ncomp, nloop = o.ncomp, o.nloop
    r = {"tri_checks": int(o.tri_checks), "nseg": o.nseg, "seg": _arr(o.seg, 6 * o.nseg, float).reshape(-1, 6)}
    r["ncomp"] = ncomp
    r["comp_off"] = _arr(o.comp_off, ncomp + 1, np.int64) if ncomp else np.zeros(1, np.int64)
    r["comp_idx"] = _arr(o.comp_idx, int(r["comp_off"][-1]), np.int64)
    r["v_off"] = _arr(o.v_off, ncomp + 1, np.int64) if ncomp else np.zeros(1, np.int64)
    r["V"] = _arr(o.V, 3 * int(r["v_off"][-1]), float).reshape(-1, 3)
    r["e_off"] = _arr(o.e_off, ncomp + 1, np.int64) if ncomp else np.zeros(1, np.int64)
    r["E"] = _arr(o.E, 2 * int(r["e_off"][-1]), np.int64).reshape(-1, 2)
    r["e2_off"] = _arr(o.e2_off, ncomp + 1, np.int64) if ncomp else np.zeros(1, np.int64)
    r["E2"] = _arr(o.E2, 2 * int(r["e2_off"][-1]), np.int64).reshape(-1, 2)
    r["nloop"] = nloop
    r["loop_comp"] = _arr(o.loop_comp, nloop, np.int64)
    r["loop_off"] = _arr(o.loop_off, nloop + 1, np.int64)
    r["loop_vid"] = _arr(o.loop_vid, int(r["loop_off"][-1]) if nloop else 0, np.int64)
    r["loop_status"] = _arr(o.loop_status, nloop, np.int64)
    r["loop_geom"] = _arr(o.loop_geom, 13 * nloop, float).reshape(-1, 13)
    return r


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


class Oracle:
    """The C restatement (oracle/zdx_oracle.c)."""

    def __init__(self, path: str = LIB_ORACLE):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle)")
        self.lib = L = C.CDLL(path)
        L.zo_pair.argtypes = [_dp, C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp, _dp, C.c_int, C.c_int,
                              C.c_double, C.POINTER(_OracleOut)]
        L.zo_pair_free.argtypes = [C.POINTER(_OracleOut)]
        L.zo_build_mesh.argtypes = [_dp, C.c_int, C.c_int, _dp, _dp]
        L.zo_sort.argtypes = [C.c_int, _ip, C.c_int, _ip, _dp, C.c_int]
        L.zo_pyset_order.argtypes = [_ip, C.c_int, _ip]
        L.zo_dem_step.argtypes = [C.POINTER(_ZoScene)]
        L.zo_scene_free_history.argtypes = [C.POINTER(_ZoScene)]
        L.zo_wall_contact.argtypes = [_dp, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp, _dp]
        L.zo_integrate.argtypes = [_dp, _dp, _dp, _dp, C.c_double]

    def build_mesh(self, tris, center=True):
        t, tp = _d(tris)
        out = np.zeros_like(t)
        props = np.zeros(17)
        self.lib.zo_build_mesh(tp, len(t), int(center), out.ctypes.data_as(_dp), props.ctypes.data_as(_dp))
        return out, props

    def pair(self, trisA, mean_edgeA, bbox_diagA, trisB, poseA, poseB, split=True, mode=0, tol=0.0) -> dict:
        a, ap = _d(trisA)
        b, bp = _d(trisB)
        pa, pap = _d(poseA)
        pb, pbp = _d(poseB)
        o = _OracleOut()
        self.lib.zo_pair(ap, len(a), mean_edgeA, bbox_diagA, bp, len(b), pap, pbp, int(split), int(mode), float(tol),
                         C.byref(o))
        r = _unpack(o)
        r["ncontact"] = o.ncontact
        r["contact_loop"] = _arr(o.contact_loop, o.ncontact, np.int64)
        r["tol"] = o.tol
        self.lib.zo_pair_free(C.byref(o))
        return r

    def pyset_order(self, keys):
        k = np.ascontiguousarray(keys, dtype=np.int32)
        out = np.zeros(max(len(k), 1), np.int32)
        self.lib.zo_pyset_order(k.ctypes.data_as(_ip), len(k), out.ctypes.data_as(_ip))
        return out[: len(k)]

    def sort(self, kind, n, ikey=None, dkey=None, stable=False):
        idx = np.arange(n, dtype=np.int32)
        ik = np.ascontiguousarray(ikey if ikey is not None else np.zeros(max(n, 1)), dtype=np.int32)
        dk = np.ascontiguousarray(dkey if dkey is not None else np.zeros(max(n, 1)), dtype=np.float64)
        self.lib.zo_sort(kind, idx.ctypes.data_as(_ip), n, ik.ctypes.data_as(_ip), dk.ctypes.data_as(_dp), int(stable))
        return idx

    def wall_contact(self, tris, pose, wall_tri, wall_normal, radius, tol):
        t, tp = _d(tris)
        p, pp = _d(pose)
        w, wp = _d(wall_tri)
        n, np_ = _d(wall_normal)
        area = np.zeros(1)
        pt = np.zeros(3)
        nn = np.zeros(3)
        ok = self.lib.zo_wall_contact(tp, len(t), pp, wp, np_, radius, tol, area.ctypes.data_as(_dp),
                                      pt.ctypes.data_as(_dp), nn.ctypes.data_as(_dp))
        return bool(ok), float(area[0]), pt, nn

    def integrate(self, state, force, torque, gravity, dt):
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        f, fp = _d(force)
        t, tp = _d(torque)
        g, gp = _d(gravity)
        self.lib.zo_integrate(s.ctypes.data_as(_dp), fp, tp, gp, dt)
        return s


class Reference:
    """The reference's src/main.cpp compiled unchanged (oracle/_ref)."""

    def __init__(self, path: str = LIB_REF):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle ref, needs the reference sources)")
        self.path = path
        self.lib = L = C.CDLL(path)
        L.zdx_ref_pair.argtypes = [_dp, C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp, _dp, C.c_int,
                                   C.POINTER(_RefOut)]
        L.zdx_ref_pair_free.argtypes = [C.POINTER(_RefOut)]
        L.zdx_ref_build_mesh.argtypes = [_dp, C.c_int, C.c_int, _dp, _dp]
        L.zdx_ref_std_sort.argtypes = [C.c_int, _ip, C.c_int, _ip, _dp]
        L.zdx_ref_wall_contact.argtypes = [_dp, C.c_int, _dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp, _dp]
        L.zdx_ref_integrate.argtypes = [_dp, _dp, _dp, _dp, C.c_double]
        L.zdx_ref_load_stl.argtypes = [C.c_char_p, _dp, C.c_int]
        L.zdx_ref_main.argtypes = [C.c_int, C.POINTER(C.c_char_p)]

    def build_mesh(self, tris, center=True):
        t, tp = _d(tris)
        out = np.zeros_like(t)
        props = np.zeros(17)
        self.lib.zdx_ref_build_mesh(tp, len(t), int(center), out.ctypes.data_as(_dp), props.ctypes.data_as(_dp))
        return out, props

    def pair(self, trisA, mean_edgeA, bbox_diagA, trisB, poseA, poseB, split=True) -> dict:
        a, ap = _d(trisA)
        b, bp = _d(trisB)
        pa, pap = _d(poseA)
        pb, pbp = _d(poseB)
        o = _RefOut()
        self.lib.zdx_ref_pair(ap, len(a), mean_edgeA, bbox_diagA, bp, len(b), pap, pbp, int(split), C.byref(o))
        r = _unpack(o)
        self.lib.zdx_ref_pair_free(C.byref(o))
        return r

    def std_sort(self, kind, n, ikey=None, dkey=None):
        idx = np.arange(n, dtype=np.int32)
        ik = np.ascontiguousarray(ikey if ikey is not None else np.zeros(max(n, 1)), dtype=np.int32)
        dk = np.ascontiguousarray(dkey if dkey is not None else np.zeros(max(n, 1)), dtype=np.float64)
        self.lib.zdx_ref_std_sort(kind, idx.ctypes.data_as(_ip), n, ik.ctypes.data_as(_ip), dk.ctypes.data_as(_dp))
        return idx

    def wall_contact(self, tris, pose, wall_tri, wall_normal, radius, tol):
        t, tp = _d(tris)
        p, pp = _d(pose)
        w, wp = _d(wall_tri)
        n, np_ = _d(wall_normal)
        area = np.zeros(1)
        pt = np.zeros(3)
        nn = np.zeros(3)
        ok = self.lib.zdx_ref_wall_contact(tp, len(t), pp, wp, np_, radius, tol, area.ctypes.data_as(_dp),
                                           pt.ctypes.data_as(_dp), nn.ctypes.data_as(_dp))
        return bool(ok), float(area[0]), pt, nn

    def integrate(self, state, force, torque, gravity, dt):
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        f, fp = _d(force)
        t, tp = _d(torque)
        g, gp = _d(gravity)
        self.lib.zdx_ref_integrate(s.ctypes.data_as(_dp), fp, tp, gp, dt)
        return s

    def load_stl(self, path, cap=1 << 20):
        buf = np.zeros(9 * cap)
        n = self.lib.zdx_ref_load_stl(path.encode(), buf.ctypes.data_as(_dp), cap)
        return buf[: 9 * min(n, cap)].reshape(-1, 3, 3)

    def main(self, args):
        argv = (C.c_char_p * (len(args) + 1))(*[a.encode() for a in ["zdem_cpu"] + list(args)])
        return self.lib.zdx_ref_main(len(args) + 1, argv)


def compare_pair(a: dict, b: dict, exact=True, geom_rtol=0.0) -> list[str]:
    """Field-by-field comparison of two pair results; returns a list of mismatch descriptions."""
    bad = []
    for k in ["nseg", "ncomp", "nloop"]:
        if a[k] != b[k]:
            bad.append(f"{k}: {a[k]} != {b[k]}")
    if bad:
        return bad
    for k in ["comp_off", "comp_idx", "v_off", "e_off", "E", "e2_off", "E2", "loop_comp", "loop_off", "loop_vid",
              "loop_status"]:
        if not np.array_equal(a[k], b[k]):
            bad.append(f"{k} differs")
    for k in ["seg", "V", "loop_geom"]:
        x, y = a[k], b[k]
        if x.shape != y.shape:
            bad.append(f"{k} shape {x.shape} != {y.shape}")
        elif exact and not np.array_equal(x, y):
            bad.append(f"{k} not bit-exact (max abs diff {np.max(np.abs(x - y)) if x.size else 0})")
        elif not exact and x.size and not np.allclose(x, y, rtol=geom_rtol, atol=0):
            bad.append(f"{k} beyond rtol {geom_rtol}")
    return bad
