"""torch.autograd wrapper of the batched pair contacts, backed by the hand-written CUDA adjoint.

``PairContactGeometry`` differentiates the two vector integrals of every contact loop, Sn and Gn, with
respect to the mesh-local triangle corners and the poses (zdx_pair_contacts_adjoint).  Everything the
reference derives from them is closed-form and is written here in torch, so autograd carries it:

    |Sn|, nA = -Sn/|Sn| (flipped toward B in zdem mode), xc0 = nA x Gn / |Sn|   (src/main.cpp:1042-1052)
    Fn = k/2 |Sn|, F_A, F_B                                                   (polyline.py:655-701)

so gradients reach k (and anything else the caller builds on top) without further kernels.  Poses are
(pos(3), quat(w,x,y,z)) per body; the quaternion gradient is the derivative along the unit sphere
(the forward normalises the quaternion, as the reference does).  Loop topology is piecewise constant:
gradients are those of the topology the forward pass found.
"""
from __future__ import annotations

import torch

from . import _lib


def quat_mul(a, b):
    aw, ax, ay, az = a.unbind(-1)
    bw, bx, by, bz = b.unbind(-1)
    return torch.stack([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                        aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw], -1)


def quat_exp(theta):
    """Unit quaternion of a rotation vector (w, x, y, z)."""
    ang = theta.norm(dim=-1, keepdim=True)
    half = 0.5 * ang
    small = ang < 1e-8
    s = torch.where(small, 0.5 - ang * ang / 48.0, torch.sin(half) / torch.where(small, torch.ones_like(ang), ang))
    return torch.cat([torch.cos(half), theta * s], -1)


def _rot_grad_to_quat(g_theta, q):
    """dL/dq for q -> q/|q| from the world-frame rotation-vector gradient: 2 (0, g) x qn / |q|."""
    n = q.norm(dim=-1, keepdim=True)
    qn = q / n
    zero = torch.zeros_like(g_theta[..., :1])
    return 2.0 * quat_mul(torch.cat([zero, g_theta], -1), qn) / n


class PairContactGeometry(torch.autograd.Function):
    """(tris, pose) -> per-contact Sn, Gn (+ non-differentiable bookkeeping)."""

    @staticmethod
    def forward(ctx, tris, pose, tri_off, mean_edge, bbox_diag, pair_mesh, mode, split, tol):
        dev = tris.device
        P = pair_mesh.shape[0]
        cap = max(64, 16 * P)
        for _ in range(2):
            out = {"ncontact": torch.zeros(max(P, 1), dtype=torch.int32, device=dev),
                   "contact_off": torch.zeros(P + 1, dtype=torch.int64, device=dev),
                   "stats": torch.zeros(max(P, 1), 4, dtype=torch.int32, device=dev),
                   "geom": torch.zeros(cap, 20, dtype=torch.float64, device=dev),
                   "info": torch.zeros(cap, 4, dtype=torch.int32, device=dev)}
            meshes = {"tris": tris.detach(), "tri_off": tri_off, "mean_edge": mean_edge, "bbox_diag": bbox_diag}
            pairs = {"mesh": pair_mesh, "pose": pose.detach()}
            ctx_handle(dev).after_torch()
            try:
                totals = _lib.pair_contacts_device(ctx_handle(dev), meshes, pairs, out, mode=mode, split=split, tol=tol)
                break
            except _lib.ZdxError as e:
                if e.status != _lib.ZDX_ERR_CAPACITY:
                    raise
                cap *= 4
        n = int(totals[0])
        geom = out["geom"][:n]
        info = out["info"][:n]
        Sn = geom[:, 0:3].clone()
        Gn = geom[:, 3:6].clone()
        if mode == _lib.MODE_ZDEM:
            sign = torch.where((geom[:, 9:12] * -Sn).sum(1) < 0, -1.0, 1.0).to(geom.dtype)
        else:
            sign = torch.ones(n, dtype=geom.dtype, device=dev)
        ctx.save_for_backward(tris, pose, tri_off, mean_edge, bbox_diag, pair_mesh)
        ctx.opts = (mode, split, tol)
        ctx.mark_non_differentiable(info, sign, out["contact_off"])
        return Sn, Gn, info, sign, out["contact_off"]

    @staticmethod
    def backward(ctx, gSn, gGn, g_info, g_sign, g_off):
        tris, pose, tri_off, mean_edge, bbox_diag, pair_mesh = ctx.saved_tensors
        mode, split, tol = ctx.opts
        n = gSn.shape[0]
        gc = torch.cat([gSn, gGn], 1).contiguous().to(torch.float64)
        gt = torch.zeros_like(tris)
        P = pair_mesh.shape[0]
        gp12 = torch.zeros(max(P, 1), 12, dtype=torch.float64, device=tris.device)
        meshes = {"tris": tris.detach(), "tri_off": tri_off, "mean_edge": mean_edge, "bbox_diag": bbox_diag}
        pairs = {"mesh": pair_mesh, "pose": pose.detach()}
        ctx_handle(tris.device).after_torch()
        if n > 0:
            _lib.pair_contacts_adjoint(ctx_handle(tris.device), meshes, pairs, gc, gt, gp12, mode=mode, split=split,
                                       tol=tol)
        gp12 = gp12[:P]
        gpose = torch.zeros_like(pose)
        gpose[:, 0:3] = gp12[:, 0:3]
        gpose[:, 7:10] = gp12[:, 6:9]
        gpose[:, 3:7] = _rot_grad_to_quat(gp12[:, 3:6], pose[:, 3:7].detach())
        gpose[:, 10:14] = _rot_grad_to_quat(gp12[:, 9:12], pose[:, 10:14].detach())
        return gt, gpose, None, None, None, None, None, None, None


_CTX: dict = {}


def ctx_handle(dev) -> _lib.Context:
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    if idx not in _CTX:
        _CTX[idx] = _lib.Context(idx)
    return _CTX[idx]


def pair_contacts(tris, pose, tri_off, mean_edge, bbox_diag, pair_mesh, k=1.0, mode=_lib.MODE_ZDEM, split=True,
                  tol=0.0):
    """Differentiable batched pair contacts on CUDA tensors.

    tris (T, 9) float64, pose (P, 14) float64 [posA quatA posB quatB], tri_off (M+1,) int64, mean_edge and
    bbox_diag (M,), pair_mesh (P, 2) int32; k a float or a tensor.  Returns a dict of per-contact tensors
    Sn, Gn, area, nA, xc0, Fn, F_A, F_B (differentiable) and pair, contact_id, contact_off."""
    Sn, Gn, info, sign, coff = PairContactGeometry.apply(tris, pose, tri_off, mean_edge, bbox_diag, pair_mesh, mode,
                                                         split, tol)
    area = Sn.norm(dim=1)
    safe = torch.where(area > 0, area, torch.ones_like(area))
    nA0 = -Sn / safe[:, None]
    xc0 = torch.cross(nA0, Gn, dim=1) / safe[:, None]
    nA = nA0 * sign[:, None]
    Fn = 0.5 * k * area
    F_A = -Fn[:, None] * nA if mode == _lib.MODE_ZDEM else Fn[:, None] * nA
    return {"Sn": Sn, "Gn": Gn, "area": area, "nA": nA, "xc0": xc0, "Fn": Fn, "F_A": F_A, "F_B": -F_A,
            "pair": info[:, 0].long(), "contact_id": info[:, 1], "contact_off": coff}
