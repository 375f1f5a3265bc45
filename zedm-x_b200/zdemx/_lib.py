"""ctypes binding of libzdemx.so (include/zdemx.h).

The library is built in-tree (``make -C zedm-x_b200``) and loaded from ``zedm-x_b200/lib``.  There is no
fallback: if the shared library is missing, or no CUDA device is usable, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("ZDEMX_LIB", os.path.join(PKG_ROOT, "lib", "libzdemx.so"))

ZDX_OK = 0
ZDX_ERR_INVALID = 1
ZDX_ERR_CUDA = 2
ZDX_ERR_CAPACITY = 3
ZDX_ERR_IO = 4
ZDX_ERR_NO_DEVICE = 5
ZDX_ERR_CONFIG = 6
ZDX_ERR_STATE = 7

MODE_ZDEM = 0
MODE_POLYLINE = 1
MODE_POLYLINE_NUMPY = 2  # polyline mode in numpy's own arithmetic
MEM_HOST = 0
MEM_DEVICE = 1
SCHED_BATCHED = 0
SCHED_PLAIN = 1
SCHED_PER_STAGE = 2  # one launch per stage over the batch, no work queue, no cost order, no culls

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


class PairOpts(C.Structure):
    _fields_ = [("mode", C.c_int), ("split_contacts", C.c_int), ("tol", C.c_double), ("k", C.c_double),
                ("mem", C.c_int), ("sched", C.c_int), ("want_loop_points", C.c_int), ("max_seg_per_pair", C.c_int)]


class MeshSet(C.Structure):
    _fields_ = [("n_mesh", C.c_int32), ("tris", C.c_void_p), ("tri_off", C.c_void_p), ("mean_edge", C.c_void_p),
                ("bbox_diag", C.c_void_p)]


class PairBatch(C.Structure):
    _fields_ = [("n_pairs", C.c_int64), ("mesh", C.c_void_p), ("pose", C.c_void_p)]


class PairResult(C.Structure):
    _fields_ = [("pair_ncontact", C.c_void_p), ("pair_contact_off", C.c_void_p), ("pair_stats", C.c_void_p),
                ("contact_cap", C.c_int64), ("contact_geom", C.c_void_p), ("contact_info", C.c_void_p),
                ("loop_point_cap", C.c_int64), ("loop_points", C.c_void_p), ("contact_point_off", C.c_void_p),
                ("totals", C.c_int64 * 4), ("comp_stats_cap", C.c_int64), ("comp_stats", C.c_void_p)]


class Tuning(C.Structure):
    _fields_ = [("tri_ctas_per_sm", C.c_int32), ("rebuild_warps", C.c_int32), ("flat_max", C.c_int64),
                ("split_tests", C.c_int64), ("rebuild_arena", C.c_int32), ("arena_warps", C.c_int32),
                ("arena_min_seg", C.c_int32), ("arena_pad", C.c_int32)]


class WallItems(C.Structure):
    _fields_ = [("n_items", C.c_int64), ("x", C.c_void_p), ("q", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("mat", C.c_void_p), ("mesh", C.c_void_p), ("wall", C.c_void_p), ("ds_in", C.c_void_p),
                ("e", C.c_double), ("dt", C.c_double), ("max_mesh_tris", C.c_int32), ("mesh_tris", C.c_void_p),
                ("mesh_off", C.c_void_p), ("mesh_tol", C.c_void_p), ("wall_tris", C.c_void_p),
                ("wall_normals", C.c_void_p), ("wall_off", C.c_void_p), ("wall_mu", C.c_void_p)]


class PPPairs(C.Structure):
    _fields_ = [("n_pairs", C.c_int64), ("contact_off", C.c_void_p), ("xa", C.c_void_p), ("xb", C.c_void_p),
                ("va", C.c_void_p), ("vb", C.c_void_p), ("wa", C.c_void_p), ("wb", C.c_void_p), ("mat_a", C.c_void_p),
                ("mat_b", C.c_void_p), ("ds_in", C.c_void_p), ("xc0", C.c_void_p), ("normal", C.c_void_p),
                ("area", C.c_void_p), ("law", C.c_int32), ("k", C.c_double), ("e", C.c_double), ("dt", C.c_double)]


class IntegrateArgs(C.Structure):
    _fields_ = [("n", C.c_int64), ("state", C.c_void_p), ("mat", C.c_void_p), ("force", C.c_void_p),
                ("torque", C.c_void_p), ("gravity", C.c_double * 3), ("dt", C.c_double)]


class ZdxError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"zdemx status {status}: {msg}")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """Load libzdemx.so once (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `make -C zedm-x_b200` (or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    L.zdx_version.restype = C.c_char_p
    L.zdx_status_string.restype = C.c_char_p
    L.zdx_status_string.argtypes = [C.c_int]
    L.zdx_last_error.restype = C.c_char_p
    L.zdx_last_error.argtypes = [C.c_void_p]
    L.zdx_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
    L.zdx_destroy.argtypes = [C.c_void_p]
    L.zdx_stl_load.restype = C.c_int64
    L.zdx_stl_load.argtypes = [C.c_char_p, _dp, C.c_int64]
    L.zdx_mesh_build.argtypes = [_dp, C.c_int64, C.c_int, _dp, _dp]
    L.zdx_pair_contacts.argtypes = [C.c_void_p, C.POINTER(PairOpts), C.POINTER(MeshSet), C.POINTER(PairBatch),
                                    C.POINTER(PairResult)]
    L.zdx_pair_timings.argtypes = [C.c_void_p, _dp, _i64p]
    L.zdx_get_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    L.zdx_scene_load.argtypes = [C.c_void_p, C.c_char_p]
    L.zdx_config_check.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, _i64p]
    L.zdx_scene_step.argtypes = [C.c_void_p, C.c_int]
    L.zdx_scene_info.argtypes = [C.c_void_p, _i64p]
    L.zdx_scene_array.argtypes = [C.c_void_p, C.c_int, C.c_void_p, _i64p]
    L.zdx_scene_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _i32p]
    L.zdx_scene_set_state.argtypes = [C.c_void_p, _dp]
    L.zdx_scene_write_output.argtypes = [C.c_void_p, C.c_int64]
    L.zdx_scene_write_output_async.argtypes = [C.c_void_p, C.c_int64]
    L.zdx_scene_output_wait.argtypes = [C.c_void_p]
    L.zdx_scene_set_free_flight.argtypes = [C.c_void_p, C.c_int]
    L.zdx_run_config.argtypes = [C.c_char_p, C.c_int]
    L.zdx_run_config_graph.argtypes = [C.c_char_p, C.c_int]
    L.zdx_scene_step_graph.argtypes = [C.c_void_p, C.c_int]
    L.zdx_scene_graph_reserve.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int]
    L.zdx_scene_graph_cache.argtypes = [C.c_void_p, _i64p, _i64p]
    L.zdx_pair_contacts_adjoint.argtypes = [C.c_void_p, C.POINTER(PairOpts), C.POINTER(MeshSet), C.POINTER(PairBatch),
                                            C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.zdx_pair_contacts_noalloc.argtypes = [C.c_void_p, C.POINTER(PairOpts), C.POINTER(MeshSet), C.POINTER(PairBatch),
                                            C.POINTER(PairResult)]
    L.zdx_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    L.zdx_wall_forces.argtypes = [C.c_void_p, C.POINTER(WallItems)] + [C.c_void_p] * 4
    L.zdx_pp_forces.argtypes = [C.c_void_p, C.POINTER(PPPairs)] + [C.c_void_p] * 4
    L.zdx_pp_forces_adjoint.argtypes = [C.c_void_p, C.POINTER(PPPairs)] + [C.c_void_p] * 8
    L.zdx_wall_forces_adjoint.argtypes = [C.c_void_p, C.POINTER(WallItems)] + [C.c_void_p] * 9
    L.zdx_get_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
    L.zdx_integrate.argtypes = [C.c_void_p, C.POINTER(IntegrateArgs), C.c_void_p]
    L.zdx_integrate_adjoint.argtypes = [C.c_void_p, C.POINTER(IntegrateArgs)] + [C.c_void_p] * 4
    L.zdx_broad_phase.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, _i64p]
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names declared in include/zdemx.h (parsed from the header)."""
    import re

    hdr = os.path.join(os.path.dirname(PKG_ROOT), "include", "zdemx.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(zdx_[a-z0-9_]+)\s*\(", text)))


def check(status: int, ctx=None):
    if status != ZDX_OK:
        msg = lib().zdx_status_string(status).decode()
        if ctx is not None:
            detail = lib().zdx_last_error(ctx).decode()
            if detail:
                msg = f"{msg}: {detail}"
        raise ZdxError(status, msg)


def config_check(path: str):
    """zdx_config_check: (status, the message zdem_cpu would print, (particles, walls, meshes, steps)
    or None).  Host only, no GPU."""
    msg = C.create_string_buffer(4096)
    counts = np.zeros(4, np.int64)
    rc = lib().zdx_config_check(path.encode(), msg, 4096, counts.ctypes.data_as(_i64p))
    return rc, msg.value.decode(), (tuple(int(x) for x in counts) if rc == 0 else None)


def stl_load(path: str) -> np.ndarray:
    """load_stl (src/main.cpp:308-371; polyline.py:59-96).  Returns (n, 3, 3) float64."""
    L = lib()
    n = L.zdx_stl_load(path.encode(), None, 0)
    if n < 0:
        raise ZdxError(-n, f"cannot read STL {path}")
    out = np.zeros((max(n, 1), 3, 3))
    L.zdx_stl_load(path.encode(), out.ctypes.data_as(_dp), n)
    return out[:n]


def mesh_build(tris, center: bool = True):
    """build_mesh (src/main.cpp:445-497).  Returns (tris_out (n,3,3), props dict)."""
    t = np.ascontiguousarray(tris, dtype=np.float64).reshape(-1, 3, 3)
    out = np.zeros_like(t)
    props = np.zeros(17)
    check(lib().zdx_mesh_build(t.ctypes.data_as(_dp), len(t), int(center), out.ctypes.data_as(_dp),
                               props.ctypes.data_as(_dp)))
    return out, {"volume": props[0], "center": props[1:4].copy(), "radius": props[4], "mean_edge": props[5],
                 "bbox_diag": props[6], "inertia_unit": props[7:16].reshape(3, 3).copy(), "nvert": int(props[16]),
                 "raw": props}


class Context:
    """One GPU, one stream (zdx_create)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        self.device = int(device)
        self._ext = None
        check(lib().zdx_create(C.byref(self._h), int(device)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().zdx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream_ptr(self) -> int:
        """The context's cudaStream_t as an integer (torch.cuda.ExternalStream(ptr) orders / times on it)."""
        v = C.c_void_p()
        check(lib().zdx_get_stream(self.handle, C.byref(v)), self.handle)
        return int(v.value or 0)

    def after_torch(self):
        """Make the context stream wait, on the device, for the work queued so far on torch's current stream:
        a call that follows reads what torch wrote, with no host-side synchronisation.  (Each call returns
        once the context stream is done, so torch may use its outputs straight away.)"""
        import torch

        if self._ext is None:
            self._ext = torch.cuda.ExternalStream(self.stream_ptr(), device=torch.device("cuda", self.device))
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(torch.device("cuda", self.device)))
        self._ext.wait_event(ev)

    def tuning(self) -> dict:
        """The pair kernels' launch parameters in force (zdx_get_tuning)."""
        t = Tuning()
        check(lib().zdx_get_tuning(self.handle, C.byref(t)), self.handle)
        return {k: int(getattr(t, k)) for k, _ in Tuning._fields_ if k != "arena_pad"}

    def set_tuning(self, **kw) -> dict:
        """Change some launch parameters (zdx_set_tuning); the others keep their values."""
        cur = self.tuning()
        unknown = set(kw) - set(cur)
        if unknown:
            raise ValueError(f"unknown tuning keys {sorted(unknown)}")
        cur.update({k: int(v) for k, v in kw.items()})
        check(lib().zdx_set_tuning(self.handle, C.byref(Tuning(**cur))), self.handle)
        return cur

    def timings(self):
        t = np.zeros(5)
        n = C.c_int64(0)
        lib().zdx_pair_timings(self._h, t.ctypes.data_as(_dp), C.byref(n))
        return {"prep": t[0], "segments": t[1], "rebuild": t[2], "gather": t[3], "total": t[4],
                "launches": int(n.value)}


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor (device mode)."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())


def pair_contacts_raw(ctx: Context, mesh_tris, tri_off, mean_edge, bbox_diag, pair_mesh, pair_pose, *,
                      mode=MODE_ZDEM, split=True, tol=0.0, k=1.0, want_points=False, sched=SCHED_BATCHED,
                      contact_cap=None, point_cap=None, max_seg_per_pair=0, comp_cap=0):
    """Host-memory batched pair call.  Returns a dict of numpy arrays (CSR over pairs).  With comp_cap > 0
    it also holds "comp_stats" (pairs x comp_cap x 3: each component's segments, snapped vertices and edges
    after the T-junction split)."""
    tris = np.ascontiguousarray(mesh_tris, dtype=np.float64)
    off = np.ascontiguousarray(tri_off, dtype=np.int64)
    me = np.ascontiguousarray(mean_edge, dtype=np.float64)
    bd = np.ascontiguousarray(bbox_diag, dtype=np.float64)
    pm = np.ascontiguousarray(pair_mesh, dtype=np.int32).reshape(-1, 2)
    pp = np.ascontiguousarray(pair_pose, dtype=np.float64).reshape(-1, 14)
    npairs = len(pm)
    if contact_cap is None:
        contact_cap = max(64, 16 * npairs)
    if point_cap is None:
        point_cap = max(1024, 512 * npairs) if want_points else 0
    for attempt in range(2):
        ncontact = np.zeros(max(npairs, 1), np.int32)
        coff = np.zeros(npairs + 1, np.int64)
        stats = np.zeros((max(npairs, 1), 4), np.int32)
        geom = np.zeros((max(contact_cap, 1), 20))
        info = np.zeros((max(contact_cap, 1), 4), np.int32)
        pts = np.zeros((max(point_cap, 1), 3))
        cpo = np.zeros(max(contact_cap, 1) + 1, np.int64)
        comp = np.zeros((max(npairs, 1), max(comp_cap, 1), 3), np.int32)
        opts = PairOpts(mode, int(split), float(tol), float(k), MEM_HOST, sched, int(want_points), int(max_seg_per_pair))
        ms = MeshSet(len(off) - 1, tris.ctypes.data, off.ctypes.data, me.ctypes.data, bd.ctypes.data)
        pb = PairBatch(npairs, pm.ctypes.data, pp.ctypes.data)
        res = PairResult(ncontact.ctypes.data, coff.ctypes.data, stats.ctypes.data, contact_cap, geom.ctypes.data,
                         info.ctypes.data, point_cap, pts.ctypes.data, cpo.ctypes.data, (C.c_int64 * 4)(),
                         int(comp_cap), comp.ctypes.data if comp_cap > 0 else None)
        st = lib().zdx_pair_contacts(ctx.handle, C.byref(opts), C.byref(ms), C.byref(pb), C.byref(res))
        totals = list(res.totals)
        if st == ZDX_ERR_CAPACITY and attempt == 0 and (totals[0] > contact_cap or totals[3] > point_cap):
            contact_cap = int(totals[0]) + 16
            point_cap = int(totals[3]) + 16 if want_points else 0
            continue
        check(st, ctx.handle)
        break
    nct = int(totals[0])
    return {"ncontact": ncontact[:npairs], "contact_off": coff, "stats": stats[:npairs], "geom": geom[:nct],
            "info": info[:nct], "points": pts[: int(totals[3])] if want_points else None,
            "point_off": cpo[: nct + 1] if want_points else None, "totals": totals,
            "comp_stats": comp[:npairs] if comp_cap > 0 else None}


def pair_contacts_device(ctx: Context, meshes: dict, pairs: dict, out: dict, *, mode=MODE_ZDEM, split=True, tol=0.0,
                         k=1.0, sched=SCHED_BATCHED, mem=MEM_DEVICE):
    """Batched pair call on caller-owned buffers given as dicts of tensors: CUDA tensors with
    mem=MEM_DEVICE, (pinned) host tensors with mem=MEM_HOST.  Returns the totals."""
    opts = PairOpts(mode, int(split), float(tol), float(k), mem, sched, 0, 0)
    ms = MeshSet(int(meshes["tri_off"].numel() - 1), _ptr(meshes["tris"]), _ptr(meshes["tri_off"]),
                 _ptr(meshes["mean_edge"]), _ptr(meshes["bbox_diag"]))
    pb = PairBatch(int(pairs["mesh"].shape[0]), _ptr(pairs["mesh"]), _ptr(pairs["pose"]))
    res = PairResult(_ptr(out["ncontact"]), _ptr(out["contact_off"]), _ptr(out["stats"]), int(out["geom"].shape[0]),
                     _ptr(out["geom"]), _ptr(out["info"]), 0, 0, 0)
    check(lib().zdx_pair_contacts(ctx.handle, C.byref(opts), C.byref(ms), C.byref(pb), C.byref(res)), ctx.handle)
    return list(res.totals)


def pair_contacts_noalloc(ctx: Context, meshes: dict, pairs: dict, out: dict, *, mode=MODE_ZDEM, split=True, tol=0.0,
                          k=1.0):
    """zdx_pair_contacts_noalloc on caller-owned CUDA tensors (the library allocates no device memory;
    limits and sharing rules in include/zdemx.h).  Returns the totals."""
    opts = PairOpts(mode, int(split), float(tol), float(k), MEM_DEVICE, SCHED_BATCHED, 0, 0)
    ms = MeshSet(int(meshes["tri_off"].numel() - 1), _ptr(meshes["tris"]), _ptr(meshes["tri_off"]),
                 _ptr(meshes["mean_edge"]), _ptr(meshes["bbox_diag"]))
    pb = PairBatch(int(pairs["mesh"].shape[0]), _ptr(pairs["mesh"]), _ptr(pairs["pose"]))
    res = PairResult(_ptr(out["ncontact"]), _ptr(out["contact_off"]), _ptr(out["stats"]), int(out["geom"].shape[0]),
                     _ptr(out["geom"]), _ptr(out["info"]), 0, 0, 0)
    check(lib().zdx_pair_contacts_noalloc(ctx.handle, C.byref(opts), C.byref(ms), C.byref(pb), C.byref(res)),
          ctx.handle)
    return list(res.totals)


def pair_contacts_adjoint(ctx: Context, meshes: dict, pairs: dict, grad_contact, grad_tris, grad_pose, *,
                          mode=MODE_ZDEM, split=True, tol=0.0, k=1.0, mem=MEM_DEVICE, sched=SCHED_BATCHED):
    """zdx_pair_contacts_adjoint on caller buffers (torch tensors or numpy arrays, all on one side)."""
    opts = PairOpts(mode, int(split), float(tol), float(k), mem, sched, 0, 0)
    ms = MeshSet(int(meshes["tri_off"].shape[0] - 1), _ptr(meshes["tris"]), _ptr(meshes["tri_off"]),
                 _ptr(meshes["mean_edge"]), _ptr(meshes["bbox_diag"]))
    pb = PairBatch(int(pairs["mesh"].shape[0]), _ptr(pairs["mesh"]), _ptr(pairs["pose"]))
    n = int(grad_contact.shape[0])
    check(lib().zdx_pair_contacts_adjoint(ctx.handle, C.byref(opts), C.byref(ms), C.byref(pb), _ptr(grad_contact), n,
                                          _ptr(grad_tris), _ptr(grad_pose)), ctx.handle)


def _wall_items(items: dict, e: float, dt: float, max_mesh_tris: int) -> WallItems:
    n = int(items["x"].shape[0])
    return WallItems(n, _ptr(items["x"]), _ptr(items["q"]), _ptr(items["v"]), _ptr(items["w"]), _ptr(items["mat"]),
                     _ptr(items["mesh"]), _ptr(items["wall"]), _ptr(items["ds_in"]), float(e), float(dt),
                     int(max_mesh_tris), _ptr(items["mesh_tris"]), _ptr(items["mesh_off"]), _ptr(items["mesh_tol"]),
                     _ptr(items["wall_tris"]), _ptr(items["wall_normals"]), _ptr(items["wall_off"]),
                     _ptr(items["wall_mu"]))


def wall_forces(ctx: Context, items: dict, e: float, dt: float, max_mesh_tris: int, out: dict) -> None:
    """zdx_wall_forces on CUDA tensors: items as the fields of zdx_wall_items, out["f"], out["t"], out["ds"]
    (n x 3 float64) and out["flags"] (n int32) written."""
    wi = _wall_items(items, e, dt, max_mesh_tris)
    check(lib().zdx_wall_forces(ctx.handle, C.byref(wi), _ptr(out["f"]), _ptr(out["t"]), _ptr(out["ds"]),
                                _ptr(out["flags"])), ctx.handle)


def wall_forces_adjoint(ctx: Context, items: dict, e: float, dt: float, max_mesh_tris: int, grad_out: dict,
                        grad_in: dict) -> None:
    """zdx_wall_forces_adjoint: grad_out["f"], ["t"], ["ds"] in; grad_in["x"], ["q"], ["v"], ["w"], ["ds_in"],
    ["e"] (per item) written."""
    wi = _wall_items(items, e, dt, max_mesh_tris)
    check(lib().zdx_wall_forces_adjoint(ctx.handle, C.byref(wi), _ptr(grad_out["f"]), _ptr(grad_out["t"]),
                                        _ptr(grad_out["ds"]), _ptr(grad_in["x"]), _ptr(grad_in["q"]),
                                        _ptr(grad_in["v"]), _ptr(grad_in["w"]), _ptr(grad_in["ds_in"]),
                                        _ptr(grad_in["e"])), ctx.handle)


def _pp_pairs(pairs: dict, law: int, k: float, e: float, dt: float) -> PPPairs:
    return PPPairs(int(pairs["xa"].shape[0]), _ptr(pairs["contact_off"]), _ptr(pairs["xa"]), _ptr(pairs["xb"]),
                   _ptr(pairs["va"]), _ptr(pairs["vb"]), _ptr(pairs["wa"]), _ptr(pairs["wb"]), _ptr(pairs["mat_a"]),
                   _ptr(pairs["mat_b"]), _ptr(pairs["ds_in"]), _ptr(pairs["xc0"]), _ptr(pairs["normal"]),
                   _ptr(pairs["area"]), int(law), float(k), float(e), float(dt))


def _integrate_args(state, mat, force, torque, gravity, dt):
    return IntegrateArgs(int(state.shape[0]), _ptr(state), _ptr(mat), _ptr(force), _ptr(torque),
                         (C.c_double * 3)(*[float(g) for g in gravity]), float(dt))


def integrate(ctx: Context, state, mat, force, torque, gravity, dt, out) -> None:
    """zdx_integrate on contiguous CUDA float64 tensors: out (n, 16) receives the new state rows."""
    a = _integrate_args(state, mat, force, torque, gravity, dt)
    check(lib().zdx_integrate(ctx.handle, C.byref(a), _ptr(out)), ctx.handle)


def integrate_adjoint(ctx: Context, state, mat, force, torque, gravity, dt, g_out, g_state, g_force, g_torque) -> None:
    """zdx_integrate_adjoint: g_out (n, 16) in; g_state (n, 16), g_force and g_torque (n, 3) written."""
    a = _integrate_args(state, mat, force, torque, gravity, dt)
    check(lib().zdx_integrate_adjoint(ctx.handle, C.byref(a), _ptr(g_out), _ptr(g_state), _ptr(g_force),
                                      _ptr(g_torque)), ctx.handle)


def broad_phase(ctx: Context, state, mat, pairs=None):
    """zdx_broad_phase on CUDA tensors: state (np, 16) and mat (np, 17) float64.  Returns (candidates,
    buffer): an (n, 2) int32 tensor of the candidate pairs (i < j, in i then j order), a view of the
    buffer, which is `pairs` (an (m, 2) int32 tensor) or, when that is missing or too small, a new one
    to pass next time."""
    import torch

    np_ = int(state.shape[0])
    dev = state.device
    if pairs is None:
        pairs = torch.empty(max(8 * np_, 64), 2, dtype=torch.int32, device=dev)
    n = C.c_int64(0)
    st, mt = state.contiguous(), mat.contiguous()
    rc = lib().zdx_broad_phase(ctx.handle, _ptr(st), _ptr(mt), np_, _ptr(pairs), int(pairs.shape[0]), C.byref(n))
    if rc == ZDX_ERR_CAPACITY:
        pairs = torch.empty(int(n.value) + 64, 2, dtype=torch.int32, device=dev)
        rc = lib().zdx_broad_phase(ctx.handle, _ptr(st), _ptr(mt), np_, _ptr(pairs), int(pairs.shape[0]), C.byref(n))
    check(rc, ctx.handle)
    return pairs[: int(n.value)], pairs


def pp_forces(ctx: Context, pairs: dict, law: int, k: float, e: float, dt: float, out: dict) -> None:
    """zdx_pp_forces on CUDA tensors: out["fb"], ["ta"], ["tb"], ["ds"] (n x 3) written."""
    pp = _pp_pairs(pairs, law, k, e, dt)
    check(lib().zdx_pp_forces(ctx.handle, C.byref(pp), _ptr(out["fb"]), _ptr(out["ta"]), _ptr(out["tb"]),
                              _ptr(out["ds"])), ctx.handle)


def pp_forces_adjoint(ctx: Context, pairs: dict, law: int, k: float, e: float, dt: float, grad_out: dict,
                      grad_in: dict) -> None:
    """zdx_pp_forces_adjoint: grad_out["fb"], ["ta"], ["tb"], ["ds"] in; grad_in["pair"] (n x 21), ["k"], ["e"]
    (n) and ["contact"] (contacts x 7) written."""
    pp = _pp_pairs(pairs, law, k, e, dt)
    check(lib().zdx_pp_forces_adjoint(ctx.handle, C.byref(pp), _ptr(grad_out["fb"]), _ptr(grad_out["ta"]),
                                      _ptr(grad_out["tb"]), _ptr(grad_out["ds"]), _ptr(grad_in["pair"]),
                                      _ptr(grad_in["k"]), _ptr(grad_in["e"]), _ptr(grad_in["contact"])), ctx.handle)
