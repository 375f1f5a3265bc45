"""Batched pair contacts: a library of meshes and many (mesh A, pose A, mesh B, pose B) pairs per call.

This is the per-pair body of the zdem_cpu step (src/main.cpp:2062-2219) applied to a whole batch, with
the minimal force law of polyline.py:677 (Fn = k/2 |Sn|).  In zdem mode the tolerance comes from mesh
A's mean edge (src/main.cpp:2118), loops are filtered on |Sn| (src/main.cpp:2188-2208) and nA is flipped
toward B (src/main.cpp:2209-2219).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class MeshLibrary:
    """Meshes as build_mesh leaves them (centred triangles, mean edge, bbox diagonal)."""

    tris: np.ndarray       # (T, 9) float64, all meshes back to back
    tri_off: np.ndarray    # (M+1,) int64
    mean_edge: np.ndarray  # (M,)
    bbox_diag: np.ndarray  # (M,)
    props: np.ndarray      # (M, 17) build_mesh properties

    @property
    def n_mesh(self) -> int:
        return len(self.tri_off) - 1

    def mesh(self, m: int) -> np.ndarray:
        return self.tris[self.tri_off[m]: self.tri_off[m + 1]].reshape(-1, 3, 3)

    @staticmethod
    def build(meshes, center: bool = True) -> "MeshLibrary":
        """Run build_mesh (host C++) on each raw triangle soup."""
        outs, props = [], []
        for t in meshes:
            o, p = _lib.mesh_build(t, center)
            outs.append(o.reshape(-1, 9))
            props.append(p["raw"])
        counts = np.array([len(o) for o in outs], np.int64)
        off = np.zeros(len(outs) + 1, np.int64)
        off[1:] = np.cumsum(counts)
        tris = np.concatenate(outs) if outs else np.zeros((0, 9))
        props = np.asarray(props).reshape(-1, 17)
        return MeshLibrary(np.ascontiguousarray(tris), off, props[:, 5].copy(), props[:, 6].copy(), props)


def pair_contacts_batch(ctx: _lib.Context, lib: MeshLibrary, pair_mesh, pair_pose, *, k=1e7, split=True,
                        mode=_lib.MODE_ZDEM, tol=0.0, sched=_lib.SCHED_BATCHED, want_points=False):
    """Host-memory call.  Returns the CSR dict of ``_lib.pair_contacts_raw``."""
    return _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pair_mesh, pair_pose,
                                  mode=mode, split=split, tol=tol, k=k, want_points=want_points, sched=sched)
