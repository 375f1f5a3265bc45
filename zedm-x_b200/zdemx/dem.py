"""The DEM scene of zdem_cpu on the GPU: load a config (same grammar), step, read the state back.

    sc = Scene("config.txt")      # parse_config_file + particle/wall set-up (src/main.cpp:1531-2022)
    sc.step(100)                   # 100 iterations of the step loop body (src/main.cpp:2034-2468)
    sc.step_graph(100)             # the same steps, replayed from one captured CUDA graph
    st = sc.state()                # (np, 16): pos quat(w,x,y,z) vel omega L
    sc.info()                      # the step log's counters for the last step
    sc.write_output(step)          # the particle VTK and state txt files (src/main.cpp:1710-1870)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

INFO_KEYS = ("particles", "walls", "steps", "contacts", "tri_checks", "segments", "comps", "loops", "pairs",
             "wall_contacts", "history", "wall_history")


class Scene:
    def __init__(self, config_path: str, ctx: _lib.Context | None = None, device: int = 0):
        self.ctx = ctx or _lib.Context(device)
        _lib.check(_lib.lib().zdx_scene_load(self.ctx.handle, config_path.encode()), self.ctx.handle)
        self.n = self.info()["particles"]

    def step(self, n: int = 1):
        _lib.check(_lib.lib().zdx_scene_step(self.ctx.handle, int(n)), self.ctx.handle)

    def step_graph(self, n: int = 1):
        """n steps through the captured CUDA graph (device-resident counts, same results as step)."""
        _lib.check(_lib.lib().zdx_scene_step_graph(self.ctx.handle, int(n)), self.ctx.handle)

    def graph_reserve(self, pairs: int = 0, contacts: int = 0, segments: int = 0, seg_per_pair: int = 0):
        """Initial capacities of the graph step (0 = default); it grows them on overflow."""
        _lib.check(_lib.lib().zdx_scene_graph_reserve(self.ctx.handle, int(pairs), int(contacts), int(segments),
                                                      int(seg_per_pair)), self.ctx.handle)

    ARRAYS = {"mat": (0, np.float64, 17), "pmesh": (1, np.int32, 1), "mesh_tris": (2, np.float64, 9),
              "mesh_off": (3, np.int64, 1), "mesh_props": (4, np.float64, 17), "wall_tris": (5, np.float64, 9),
              "wall_normals": (6, np.float64, 3), "wall_off": (7, np.int64, 1), "wall_mat": (8, np.float64, 2),
              "wall_pose": (9, np.float64, 7), "wall_mesh": (10, np.int32, 1), "params": (11, np.float64, 1)}

    def graph_cache(self) -> dict:
        """The graph step's clearance cache: entries after the last graph step, pairs that step skipped."""
        e, k = C.c_int64(0), C.c_int64(0)
        _lib.check(_lib.lib().zdx_scene_graph_cache(self.ctx.handle, C.byref(e), C.byref(k)), self.ctx.handle)
        return {"entries": int(e.value), "skipped": int(k.value)}

    def array(self, name: str) -> np.ndarray:
        """A set-up array of the scene (zdx_scene_array): mat, pmesh, mesh_tris, mesh_off, mesh_props,
        wall_tris, wall_normals, wall_off, wall_mat, wall_pose, wall_mesh, params (dt, gravity, split,
        force_law, feng_k)."""
        which, dt, width = self.ARRAYS[name]
        n = C.c_int64(0)
        _lib.check(_lib.lib().zdx_scene_array(self.ctx.handle, which, None, C.byref(n)), self.ctx.handle)
        out = np.zeros(max(n.value, 1), dt)
        _lib.check(_lib.lib().zdx_scene_array(self.ctx.handle, which, out.ctypes.data, C.byref(n)), self.ctx.handle)
        out = out[: n.value]
        return out.reshape(-1, width) if width > 1 else out

    def info(self) -> dict:
        v = np.zeros(12, np.int64)
        _lib.check(_lib.lib().zdx_scene_info(self.ctx.handle, v.ctypes.data_as(_lib._i64p)), self.ctx.handle)
        return dict(zip(INFO_KEYS, (int(x) for x in v)))

    def state(self, out=None):
        """(state n x 16, force n x 3, torque n x 3, contact_count n).  out: the four arrays of an
        earlier call to fill again instead of new ones (a loop that reads the state every step then
        allocates nothing)."""
        if out is None:
            st = np.zeros((self.n, 16))
            f = np.zeros((self.n, 3))
            t = np.zeros((self.n, 3))
            c = np.zeros(self.n, np.int32)
        else:
            st, f, t, c = out
            for a, shape, dt in ((st, (self.n, 16), np.float64), (f, (self.n, 3), np.float64),
                                 (t, (self.n, 3), np.float64), (c, (self.n,), np.int32)):
                if a.shape != shape or a.dtype != dt or not a.flags["C_CONTIGUOUS"] or not a.flags["WRITEABLE"]:
                    raise ValueError(f"state(out=...): expected a writable C-contiguous {dt.__name__} array of shape {shape}")
        _lib.check(_lib.lib().zdx_scene_get_state(self.ctx.handle, st.ctypes.data_as(_lib._dp), f.ctypes.data_as(_lib._dp),
                                                  t.ctypes.data_as(_lib._dp), c.ctypes.data_as(_lib._i32p)),
                   self.ctx.handle)
        return st, f, t, c

    def set_state(self, st):
        st = np.ascontiguousarray(st, dtype=np.float64)
        _lib.check(_lib.lib().zdx_scene_set_state(self.ctx.handle, st.ctypes.data_as(_lib._dp)), self.ctx.handle)

    def write_output(self, step: int, wait: bool = True):
        """The particle VTK and state txt files of `step`.  wait=False snapshots the particles on the device
        and writes the files on a background thread while stepping goes on; output_wait() joins them."""
        if wait:
            _lib.check(_lib.lib().zdx_scene_write_output(self.ctx.handle, int(step)), self.ctx.handle)
        else:
            _lib.check(_lib.lib().zdx_scene_write_output_async(self.ctx.handle, int(step)), self.ctx.handle)

    def set_free_flight(self, enable: bool):
        """Candidate-free steps of a small scene through the single-block kernel (default on)."""
        _lib.check(_lib.lib().zdx_scene_set_free_flight(self.ctx.handle, int(bool(enable))), self.ctx.handle)

    def output_wait(self):
        _lib.check(_lib.lib().zdx_scene_output_wait(self.ctx.handle), self.ctx.handle)


def run_config(config_path: str, device: int = 0, graph: bool = False) -> int:
    """zdem_cpu's whole run (outputs and log line included); returns the exit code."""
    if graph:
        return _lib.lib().zdx_run_config_graph(config_path.encode(), int(device))
    return _lib.lib().zdx_run_config(config_path.encode(), int(device))
