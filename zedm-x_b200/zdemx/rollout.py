"""Differentiable DEM rollouts: the step of zdx_scene_step written with torch autograd around the CUDA
contact geometry and its hand-written adjoint (zdemx.autograd), with checkpointed segments.

The step follows the device step operation for operation (zdx_scene.cu, after src/main.cpp:2034-2468):
broad phase (i < j, |xj - xi|^2 <= (ri + rj)^2), pair contacts (Sn, Gn -> |Sn|, nA, xc0 from the CUDA
kernels), the particle-particle law with its tangential history shared by the loops of a pair in loop
order, the wall contact (plane section of the particle mesh, unique_points, Sutherland-Hodgman, shoelace
area and mean centroid, src/main.cpp:1093-1258, 2308-2447) with its history shared by the wall's
triangles in order, and integrate_particle (src/main.cpp:1494-1510).  Sums run in a different order than
the device step's, so trajectories agree to rounding, not bit for bit.

What is differentiable: everything continuous in the particle state and in the parameters k (feng_min
stiffness) and e (restitution, one value for all particles).  Topology (which pairs, loops, wall
contacts, Coulomb regime) is taken from the forward pass.  The wall contacts (section, clip, area,
centroid, force law and history, every triangle of a wall in order) run in CUDA with a hand-written
reverse mode (zdx_wall_forces / zdx_wall_forces_adjoint, one thread per particle near a wall); sections
clipped by a wall triangle's edges are differentiated too.  ``DiffScene._walls_torch`` keeps the same
computation in torch autograd (sections inside their triangle only), the check the kernels are tested
against.

    ds = DiffScene(scene)                   # a loaded zdemx.dem.Scene
    x, aux = ds.rollout(state0, k, e, steps=2000, checkpoint_every=100)
    loss = ((x[:, 0:3] - target) ** 2).sum(); loss.backward()
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from .autograd import pair_contacts

PI = 3.141592653589793


def _cross(a, b):
    return torch.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                        a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _qmul(a, b):
    aw, ax, ay, az = a.unbind(-1)
    bw, bx, by, bz = b.unbind(-1)
    return torch.stack([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                        aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw], -1)


def _qnormalize(q):
    return q / torch.sqrt(q[..., 0] * q[..., 0] + q[..., 1] * q[..., 1] + q[..., 2] * q[..., 2] +
                          q[..., 3] * q[..., 3])[..., None]


def _rotate(qn, v):
    """quat_rotate with a normalised quaternion: q (0, v) q* (src/main.cpp:93-98)."""
    p = torch.cat([torch.zeros_like(v[..., :1]), v], -1)
    c = qn * torch.tensor([1.0, -1.0, -1.0, -1.0], dtype=qn.dtype, device=qn.device)
    return _qmul(_qmul(qn, p), c)[..., 1:]


def _rotmat(qn):
    w, x, y, z = qn.unbind(-1)
    return torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1).reshape(*qn.shape[:-1], 3, 3)


class _Rows(torch.autograd.Function):
    """src[idx] along dim 0, with the cotangent scattered back by index_add_ (FP64 atomics: the sums'
    order, and so their last bits, may vary between runs) rather than by the sorted scatter of an indexing
    backward."""

    @staticmethod
    def forward(ctx, src, idx):
        ctx.save_for_backward(idx)
        ctx.n = src.shape[0]
        return src.index_select(0, idx)

    @staticmethod
    def backward(ctx, g):
        (idx,) = ctx.saved_tensors
        out = torch.zeros((ctx.n,) + tuple(g.shape[1:]), dtype=g.dtype, device=g.device)
        out.index_add_(0, idx, g)
        return out, None


def _rows(src, idx):
    return _Rows.apply(src, idx) if src.requires_grad else src.index_select(0, idx)


def _lookup(keys, query):
    """Index of each query key in the sorted key array, -1 where absent."""
    if keys.numel() == 0 or query.numel() == 0:
        return torch.full_like(query, -1)
    pos = torch.searchsorted(keys, query).clamp(max=keys.numel() - 1)
    return torch.where(keys[pos] == query, pos, torch.full_like(pos, -1))


class _WallForces(torch.autograd.Function):
    """Per (particle, wall) item: summed force, torque, history after the wall (CUDA, zdx_wall_forces) and
    their reverse (zdx_wall_forces_adjoint)."""

    @staticmethod
    def forward(ctx, x, q, v, w, ds_in, e, mat, mesh, wall, consts):
        n = x.shape[0]
        dev = x.device
        items = dict(consts["items"])
        items.update({"x": x.detach().contiguous(), "q": q.detach().contiguous(), "v": v.detach().contiguous(),
                      "w": w.detach().contiguous(), "ds_in": ds_in.detach().contiguous(), "mat": mat, "mesh": mesh,
                      "wall": wall})
        out = {"f": torch.empty(n, 3, dtype=torch.float64, device=dev),
               "t": torch.empty(n, 3, dtype=torch.float64, device=dev),
               "ds": torch.empty(n, 3, dtype=torch.float64, device=dev),
               "flags": torch.empty(n, dtype=torch.int32, device=dev)}
        ev = float(e)
        consts["ctx"].after_torch()
        _lib.wall_forces(consts["ctx"], items, ev, consts["dt"], consts["max_tris"], out)
        # per-call tensors through save_for_backward (a checkpointed rollout frees and recomputes them);
        # the scene's constant arrays stay in consts
        ctx.save_for_backward(items["x"], items["q"], items["v"], items["w"], items["ds_in"], items["mat"],
                              items["mesh"], items["wall"])
        ctx.consts = consts
        ctx.ev = ev
        ctx.mark_non_differentiable(out["flags"])
        return out["f"], out["t"], out["ds"], out["flags"]

    @staticmethod
    def backward(ctx, gf, gt, gds, gflags):
        consts = ctx.consts
        items = dict(consts["items"])
        for name, t in zip(("x", "q", "v", "w", "ds_in", "mat", "mesh", "wall"), ctx.saved_tensors):
            items[name] = t
        n = items["x"].shape[0]
        dev = items["x"].device
        z = lambda k: torch.zeros(n, k, dtype=torch.float64, device=dev)
        grad_in = {"x": z(3), "q": z(4), "v": z(3), "w": z(3), "ds_in": z(3),
                   "e": torch.zeros(n, dtype=torch.float64, device=dev)}
        g = {"f": (gf if gf is not None else z(3)).contiguous(), "t": (gt if gt is not None else z(3)).contiguous(),
             "ds": (gds if gds is not None else z(3)).contiguous()}
        consts["ctx"].after_torch()
        _lib.wall_forces_adjoint(consts["ctx"], items, ctx.ev, consts["dt"], consts["max_tris"], g, grad_in)
        return (grad_in["x"], grad_in["q"], grad_in["v"], grad_in["w"], grad_in["ds_in"], grad_in["e"].sum(), None, None,
                None, None)


class _Integrate(torch.autograd.Function):
    """integrate_particle for every particle through zdx_integrate; backward through zdx_integrate_adjoint
    (the cotangents of the old state, of the forces and of the torques)."""

    @staticmethod
    def forward(ctx, state, F, T, consts):
        st, f, t = state.detach().contiguous(), F.detach().contiguous(), T.detach().contiguous()
        out = torch.empty_like(st)
        consts["ctx"].after_torch()
        _lib.integrate(consts["ctx"], st, consts["mat"], f, t, consts["g"], consts["dt"], out)
        ctx.save_for_backward(st, f, t)
        ctx.consts = consts
        return out

    @staticmethod
    def backward(ctx, g_out):
        st, f, t = ctx.saved_tensors
        c = ctx.consts
        g_st, g_f, g_t = torch.empty_like(st), torch.empty_like(f), torch.empty_like(t)
        c["ctx"].after_torch()
        _lib.integrate_adjoint(c["ctx"], st, c["mat"], f, t, c["g"], c["dt"], g_out.contiguous(), g_st, g_f, g_t)
        return g_st, g_f, g_t, None


_PP_SAVED = ("contact_off", "mat_a", "mat_b", "xa", "xb", "va", "vb", "wa", "wb", "ds_in", "xc0", "normal", "area")


class _PPForces(torch.autograd.Function):
    """Per candidate pair: the summed force on B, the torques on A and B and the history after its contacts
    (CUDA, zdx_pp_forces), and their reverse (zdx_pp_forces_adjoint)."""

    @staticmethod
    def forward(ctx, xa, xb, va, vb, wa, wb, ds_in, xc0, normal, area, k, e, contact_off, mat_a, mat_b, consts):
        n = xa.shape[0]
        dev = xa.device
        pairs = {"contact_off": contact_off, "mat_a": mat_a, "mat_b": mat_b}
        for name, t in (("xa", xa), ("xb", xb), ("va", va), ("vb", vb), ("wa", wa), ("wb", wb), ("ds_in", ds_in),
                        ("xc0", xc0), ("normal", normal), ("area", area)):
            pairs[name] = t.detach().contiguous()
        out = {nm: torch.empty(n, 3, dtype=torch.float64, device=dev) for nm in ("fb", "ta", "tb", "ds")}
        kv, ev = float(k), float(e)
        consts["ctx"].after_torch()
        _lib.pp_forces(consts["ctx"], pairs, consts["law"], kv, ev, consts["dt"], out)
        ctx.save_for_backward(*(pairs[nm] for nm in _PP_SAVED))
        ctx.consts, ctx.kv, ctx.ev = consts, kv, ev
        ctx.k_is_tensor = torch.is_tensor(k)
        return out["fb"], out["ta"], out["tb"], out["ds"]

    @staticmethod
    def backward(ctx, gfb, gta, gtb, gds):
        consts = ctx.consts
        pairs = dict(zip(_PP_SAVED, ctx.saved_tensors))
        n = pairs["xa"].shape[0]
        nc = pairs["area"].shape[0]
        dev = pairs["xa"].device
        z3 = lambda g: (g if g is not None else torch.zeros(n, 3, dtype=torch.float64, device=dev)).contiguous()
        gout = {"fb": z3(gfb), "ta": z3(gta), "tb": z3(gtb), "ds": z3(gds)}
        gin = {"pair": torch.zeros(n, 21, dtype=torch.float64, device=dev),
               "k": torch.zeros(n, dtype=torch.float64, device=dev), "e": torch.zeros(n, dtype=torch.float64, device=dev),
               "contact": torch.zeros(max(nc, 1), 7, dtype=torch.float64, device=dev)}
        consts["ctx"].after_torch()
        _lib.pp_forces_adjoint(consts["ctx"], pairs, consts["law"], ctx.kv, ctx.ev, consts["dt"], gout, gin)
        g = gin["pair"]
        gc = gin["contact"][:nc]
        gk = gin["k"].sum() if ctx.k_is_tensor else None
        return (g[:, 0:3], g[:, 3:6], g[:, 6:9], g[:, 9:12], g[:, 12:15], g[:, 15:18], g[:, 18:21], gc[:, 0:3],
                gc[:, 3:6], gc[:, 6], gk, gin["e"].sum(), None, None, None, None)


class DiffScene:
    """Constants of a loaded zdemx.dem.Scene on the GPU, and its differentiable step."""

    def __init__(self, scene, device="cuda"):
        dev = torch.device(device)
        T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
        self.dev = dev
        self.mat = T(scene.array("mat"))
        self.pmesh = T(scene.array("pmesh"), torch.int32)
        self.tris = T(scene.array("mesh_tris"))
        self.tri_off = T(scene.array("mesh_off"), torch.int64)
        props = scene.array("mesh_props")
        self.props = T(props)
        self.mean_edge = T(props[:, 5])
        self.bbox_diag = T(props[:, 6])
        self.wtris = T(scene.array("wall_tris")).reshape(-1, 3, 3)
        self.wnorm = T(scene.array("wall_normals"))
        self.woff = scene.array("wall_off").astype(np.int64)
        self.wmat = T(scene.array("wall_mat"))
        self.wpose = T(scene.array("wall_pose"))
        wmesh = scene.array("wall_mesh")
        self.wrad = T(props[wmesh, 4]) if len(wmesh) else T(np.zeros(0))
        prm = scene.array("params")
        self.dt = float(prm[0])
        self.g = T(prm[1:4])
        self.g_host = [float(a) for a in prm[1:4]]
        self.split = bool(prm[4] != 0)
        self.law = int(prm[5])
        self.feng_k = float(prm[6])
        self.np = self.mat.shape[0]
        self.nw = len(self.woff) - 1
        # particle meshes as (mesh -> padded triangle corners) for the wall section
        off = scene.array("mesh_off")
        self.mesh_ntri = torch.as_tensor(np.diff(off), device=dev)
        self.max_ntri = int(np.max(np.diff(off))) if len(off) > 1 else 0
        nm = len(off) - 1
        pad = np.zeros((nm, max(self.max_ntri, 1), 9))
        for m in range(nm):
            pad[m, : off[m + 1] - off[m]] = scene.array("mesh_tris")[off[m]: off[m + 1]]
        self.mesh_pad = T(pad).reshape(nm, -1, 3, 3)
        tolm = np.where(props[:, 5] > 0, props[:, 5] * 0.1, props[:, 6] * 1e-2)
        self.mesh_tol = T(np.where(tolm > 0, tolm, 1e-6))
        # the wall kernels' constant arrays
        self.mesh_off_t = T(off, torch.int64)
        self.wall_off_t = T(self.woff, torch.int64)
        self.wall_mu = self.wmat[:, 0].contiguous() if self.nw else T(np.zeros(1))
        self.wtris_flat = self.wtris.reshape(-1, 9).contiguous()
        self.wnorm_c = self.wnorm.contiguous()
        self._wctx = None
        self._bp_buf = None

    # ------------------------------------------------------------------------------------------------
    def initial_history(self):
        z64 = torch.zeros(0, dtype=torch.int64, device=self.dev)
        z3 = torch.zeros(0, 3, dtype=torch.float64, device=self.dev)
        return z64, z3, z64.clone(), z3.clone()

    def step(self, state, hkey, hds, wkey, wds, k, e):
        """One step; returns (state, hkey, hds, wkey, wds, stats)."""
        dev, N = self.dev, self.np
        mat = self.mat
        F = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        Tq = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        stats = {}
        # ---- broad phase (no gradient: decides topology only), binned on the GPU
        with torch.no_grad():
            if self._wctx is None:
                from .autograd import ctx_handle

                self._wctx = ctx_handle(dev)
            self._wctx.after_torch()
            cand, self._bp_buf = _lib.broad_phase(self._wctx, state.detach(), mat, self._bp_buf)
            pi, pj = cand[:, 0].long(), cand[:, 1].long()
        P = pi.numel()
        stats["pairs"] = P
        new_hkey = torch.zeros(0, dtype=torch.int64, device=dev)
        new_hds = torch.zeros(0, 3, dtype=torch.float64, device=dev)
        if P > 0:
            sa, sb = _rows(state, pi), _rows(state, pj)  # each pair's two particles, once
            pose = torch.cat([sa[:, 0:7], sb[:, 0:7]], 1)
            pm = torch.stack([self.pmesh[pi], self.pmesh[pj]], 1).contiguous()
            out = pair_contacts(self.tris, pose, self.tri_off, self.mean_edge, self.bbox_diag, pm, k=1.0,
                                mode=_lib.MODE_ZDEM, split=self.split)
            nc = out["area"].shape[0]
            stats["contacts"] = nc
            if nc > 0:
                cpair = out["pair"]
                coff = out["contact_off"]
                key = (pi.to(torch.int64) << 32) | pj.to(torch.int64)
                hpos = _lookup(hkey, key)
                zero3 = torch.zeros(P, 3, dtype=torch.float64, device=dev)
                ds_in = torch.where((hpos >= 0)[:, None], _rows(hds, hpos.clamp(min=0)) if hds.shape[0] else zero3, zero3)
                if self._wctx is None:
                    from .autograd import ctx_handle

                    self._wctx = ctx_handle(dev)
                consts = {"ctx": self._wctx, "law": self.law, "dt": self.dt}
                fb, ta, tb, ds_pair = _PPForces.apply(sa[:, 0:3], sb[:, 0:3], sa[:, 7:10], sb[:, 7:10], sa[:, 10:13],
                                                      sb[:, 10:13], ds_in, out["xc0"],
                                                      out["nA"], out["area"], k, e, coff.contiguous(),
                                                      mat[pi].contiguous(), mat[pj].contiguous(), consts)
                F = F.index_add(0, pi, -fb).index_add(0, pj, fb)
                Tq = Tq.index_add(0, pi, ta).index_add(0, pj, tb)
                act = torch.nonzero(torch.bincount(cpair, minlength=P) > 0).squeeze(1)
                new_hkey = key.index_select(0, act)
                new_hds = _rows(ds_pair, act)
        # ---- walls
        new_wkey = torch.zeros(0, dtype=torch.int64, device=dev)
        new_wds = torch.zeros(0, 3, dtype=torch.float64, device=dev)
        nwc = 0
        if self.nw > 0:
            Fw, Tw, new_wkey, new_wds, nwc = self._walls(state, wkey, wds, e)
            F = F + Fw
            Tq = Tq + Tw
        stats["wall_contacts"] = nwc
        # ---- integrate_particle (src/main.cpp:1494-1510), in CUDA with its reverse mode
        new_state = _Integrate.apply(state, F, Tq, {"ctx": self._wctx, "mat": mat, "g": self.g_host, "dt": self.dt})
        return new_state, new_hkey, new_hds, new_wkey, new_wds, stats

    def integrate_torch(self, state, F, Tq):
        """integrate_particle in torch autograd (the kernels' check)."""
        N, dev, mat = self.np, self.dev, self.mat
        x, q, v, L = state[:, 0:3], state[:, 3:7], state[:, 7:10], state[:, 13:16]
        acc = F * mat[:, 1:2] + self.g
        vel = v + acc * self.dt
        pos = x + vel * self.dt
        qn = _qnormalize(q)
        R = _rotmat(qn)
        Ib = mat[:, 8:17].reshape(N, 3, 3)
        Iinv = (R @ Ib) @ R.transpose(1, 2)
        Ln = L + Tq * self.dt
        om = (Iinv @ Ln[:, :, None])[:, :, 0]
        qd = _qmul(torch.cat([torch.zeros(N, 1, dtype=q.dtype, device=dev), om], 1), q)
        qq = _qnormalize(q + 0.5 * qd * self.dt)
        return torch.cat([pos, qq, vel, om, Ln], 1)

    def broad_phase_torch(self, x):
        """The candidate pairs by the O(np^2) all-pairs sphere test in torch (the binned kernel's check)."""
        with torch.no_grad():
            r = self.mat[:, 2]
            d = x[None, :, :] - x[:, None, :]
            dist2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
            rs = r[:, None] + r[None, :]
            ok = torch.triu(~(dist2 > rs * rs), diagonal=1)
            return torch.nonzero(ok, as_tuple=True)

    # ------------------------------------------------------------------------------------------------
    def _walls(self, state, wkey, wds, e):
        """Wall contacts of every particle near a wall, through the CUDA kernels (see _WallForces)."""
        dev, N, mat = self.dev, self.np, self.mat
        r = mat[:, 2]
        Fw = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        Tw = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        with torch.no_grad():
            d = state.detach()[:, None, 0:3] - self.wpose[None, :, 0:3]
            dist2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
            rs = r[:, None] + self.wrad[None, :]
            ci, cw = torch.nonzero(~(dist2 > rs * rs), as_tuple=True)
        C = ci.numel()
        if C == 0:
            z = torch.zeros(0, dtype=torch.int64, device=dev)
            return Fw, Tw, z, torch.zeros(0, 3, dtype=torch.float64, device=dev), 0
        key = (ci.to(torch.int64) << 16) | cw.to(torch.int64)
        hpos = _lookup(wkey, key)
        zero3 = torch.zeros(C, 3, dtype=torch.float64, device=dev)
        ds_c = torch.where((hpos >= 0)[:, None], _rows(wds, hpos.clamp(min=0)) if wds.shape[0] else zero3, zero3)
        if self._wctx is None:
            from .autograd import ctx_handle

            self._wctx = ctx_handle(dev)
        consts = {"ctx": self._wctx, "dt": self.dt, "max_tris": self.max_ntri,
                  "items": {"mesh_tris": self.tris, "mesh_off": self.mesh_off_t, "mesh_tol": self.mesh_tol,
                            "wall_tris": self.wtris_flat, "wall_normals": self.wnorm_c, "wall_off": self.wall_off_t,
                            "wall_mu": self.wall_mu}}
        sc = _rows(state, ci)
        f, t, ds_out, flags = _WallForces.apply(sc[:, 0:3], sc[:, 3:7], sc[:, 7:10], sc[:, 10:13], ds_c, e,
                                                mat[ci].contiguous(),
                                                self.pmesh[ci].contiguous(), cw.to(torch.int32).contiguous(), consts)
        with torch.no_grad():
            fl = flags.to(torch.int64)
            if bool(((fl >> 16) & 1).any()):
                raise RuntimeError("a wall section exceeded 256 crossings")
            touched = (fl & 1) != 0
            nwc = int(((fl >> 1) & 0x7FFF).sum())
        Fw = Fw.index_add(0, ci, f)
        Tw = Tw.index_add(0, ci, t)
        tidx = torch.nonzero(touched).squeeze(1)
        return Fw, Tw, key.index_select(0, tidx), _rows(ds_out, tidx), nwc

    def _walls_torch(self, state, wkey, wds, e):
        """The wall contacts in torch autograd (sections inside their wall triangle only); the kernels'
        check."""
        dev, N, mat = self.dev, self.np, self.mat
        x, q, v, w = state[:, 0:3], state[:, 3:7], state[:, 7:10], state[:, 10:13]
        r = mat[:, 2]
        Fw = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        Tw = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        with torch.no_grad():
            d = state.detach()[:, None, 0:3] - self.wpose[None, :, 0:3]
            dist2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
            rs = r[:, None] + self.wrad[None, :]
            ci, cw = torch.nonzero(~(dist2 > rs * rs), as_tuple=True)
        C = ci.numel()
        if C == 0:
            z = torch.zeros(0, dtype=torch.int64, device=dev)
            return Fw, Tw, z, torch.zeros(0, 3, dtype=torch.float64, device=dev), 0
        key = (ci.to(torch.int64) << 16) | cw.to(torch.int64)
        hpos = _lookup(wkey, key)
        zero3 = torch.zeros(C, 3, dtype=torch.float64, device=dev)
        ds_c = torch.where((hpos >= 0)[:, None], _rows(wds, hpos.clamp(min=0)) if wds.shape[0] else zero3, zero3)
        touched = torch.zeros(C, dtype=torch.bool, device=dev)
        qn = _qnormalize(q[ci])
        xp = x[ci]
        rp = r[ci]
        nwc = 0
        max_wtri = int(np.max(np.diff(self.woff)))
        woff = torch.as_tensor(self.woff, device=dev)
        for slot in range(max_wtri):
            with torch.no_grad():
                t = woff[cw] + slot
                valid = t < woff[cw + 1]
                tt = torch.where(valid, t, torch.zeros_like(t))
                wt = self.wtris[tt]
                wmn, wmx = wt.min(1).values, wt.max(1).values
                pmn, pmx = xp.detach() - rp[:, None], xp.detach() + rp[:, None]
                hit = valid & ~((pmx < wmn) | (pmn > wmx)).any(1)
            sel = torch.nonzero(hit, as_tuple=True)[0]
            if sel.numel() == 0:
                continue
            ok, area, cpt = self._wall_contact(ci[sel], qn[sel], xp[sel], tt[sel])
            sel2 = sel[ok]
            if sel2.numel() == 0:
                continue
            area, cpt = area[ok], cpt[ok]
            nwc += int(sel2.numel())
            i_ = ci[sel2]
            n = self.wnorm[tt[sel2]]
            to_p = x[i_] - cpt
            cn = torch.where((_dot(n, to_p) < 0.0)[:, None], -n, n)
            rP = cpt - x[i_]
            vrel = v[i_] + _cross(w[i_], rP)
            vn = _dot(vrel, cn)
            mp = mat[i_]
            Rp, Ep, nup = mp[:, 3].clamp(min=1e-12), mp[:, 4].clamp(min=1e-12), mp[:, 5]
            kn = (Ep / Rp) * area
            kt = (Ep / (2.0 * (1.0 + nup) * Rp)) * area
            m_eff = mp[:, 0]
            ee = torch.clamp(e * torch.ones_like(area), 1e-6, 0.9999)
            loge = torch.log(ee)
            cnd = torch.abs(2.0 * loge * torch.sqrt(kn * m_eff) / torch.sqrt(loge * loge + PI * PI))
            ctd = torch.abs(2.0 * loge * torch.sqrt(kt * m_eff) / torch.sqrt(loge * loge + PI * PI))
            fn = kn * torch.pow(torch.pow(area, 1.5), 1.0 / 3.0) + -cnd * vn
            fn = torch.clamp(fn, min=0.0)
            vt = vrel - cn * vn[:, None]
            ds = ds_c[sel2] + vt * self.dt
            ds = ds - cn * _dot(ds, cn)[:, None]
            ft = ds * (-kt)[:, None] + vt * (-ctd)[:, None]
            mu = torch.minimum(mp[:, 6], self.wmat[cw[sel2], 0])
            ftn = torch.sqrt(_dot(ft, ft))
            ftmax = mu * fn
            cap = (ftn > ftmax) & (ftn > 1e-14)
            ft = torch.where(cap[:, None], ft * (ftmax / torch.where(cap, ftn, torch.ones_like(ftn)))[:, None], ft)
            ds = torch.where((cap & (kt > 1e-12))[:, None], ft * (-1.0 / torch.where(kt > 1e-12, kt, torch.ones_like(kt)))[:, None], ds)
            ds_c = ds_c.index_copy(0, sel2, ds)
            touched = touched.index_fill(0, sel2, True)
            f = cn * fn[:, None] + ft
            Fw = Fw.index_add(0, i_, f)
            Tw = Tw.index_add(0, i_, _cross(rP, f))
        return Fw, Tw, key[touched], ds_c[touched], nwc

    def _wall_contact(self, pidx, qn, xp, tidx):
        """compute_wall_contact (src/main.cpp:1205-1258) for particle/wall-triangle items; returns
        (ok, area, contact point)."""
        dev = self.dev
        mesh = self.pmesh[pidx].long()
        tris = self.mesh_pad[mesh]                                  # (C, Tm, 3, 3) local
        ntri = self.mesh_ntri[mesh]
        Cn, Tm = tris.shape[0], tris.shape[1]
        tol = self.mesh_tol[mesh]
        wt = self.wtris[tidx]
        n = self.wnorm[tidx]
        dpl = -_dot(n, wt[:, 0])
        with torch.no_grad():
            W = _rotate(qn.detach()[:, None, None, :].expand(Cn, Tm, 3, 4), tris) + xp.detach()[:, None, None, :]
            p0, p1 = W, torch.roll(W, -1, dims=2)
            d0 = _dot(n[:, None, None, :], p0) + dpl[:, None, None]
            d1 = _dot(n[:, None, None, :], p1) + dpl[:, None, None]
            cross = (d0 * d1 < 0.0) & (torch.arange(Tm, device=dev)[None, :, None] < ntri[:, None, None])
            cidx, ct, ce = torch.nonzero(cross, as_tuple=True)          # (triangle, edge) order per item
        # crossing points, differentiable in the pose
        a0 = tris[cidx, ct, ce]
        a1 = tris[cidx, ct, (ce + 1) % 3]
        w0 = _rotate(qn[cidx], a0) + xp[cidx]
        w1 = _rotate(qn[cidx], a1) + xp[cidx]
        e0 = _dot(n[cidx], w0) + dpl[cidx]
        e1 = _dot(n[cidx], w1) + dpl[cidx]
        tpar = torch.clamp(e0 / (e0 - e1), 0.0, 1.0)
        ip = w0 + (w1 - w0) * tpar[:, None]
        cnt = torch.bincount(cidx, minlength=Cn)
        K = int(cnt.max().item()) if cidx.numel() else 0
        ok = torch.zeros(Cn, dtype=torch.bool, device=dev)
        area = torch.zeros(Cn, dtype=torch.float64, device=dev)
        cpt = torch.zeros(Cn, 3, dtype=torch.float64, device=dev)
        if K < 3:
            return ok, area, cpt
        start = torch.cumsum(cnt, 0) - cnt
        slot = torch.arange(cidx.numel(), device=dev) - start[cidx]
        pts = torch.zeros(Cn, K, 3, dtype=torch.float64, device=dev).index_put((cidx, slot), ip)
        present = torch.zeros(Cn, K, dtype=torch.bool, device=dev).index_put((cidx, slot), torch.ones_like(slot, dtype=torch.bool))
        # unique_points (src/main.cpp:561-577): keep a point unless an earlier kept one is within tol
        with torch.no_grad():
            pd = pts.detach()
            keep = torch.zeros(Cn, K, dtype=torch.bool, device=dev)
            tol2 = (tol * tol)[:, None]
            for kk in range(K):
                dd = pd - pd[:, kk: kk + 1, :]
                d2 = dd[..., 0] * dd[..., 0] + dd[..., 1] * dd[..., 1] + dd[..., 2] * dd[..., 2]
                near = ((d2 <= tol2) & keep).any(1)
                keep[:, kk] = present[:, kk] & ~near
            nu = keep.sum(1)
            order = torch.argsort((~keep).to(torch.int8), dim=1, stable=True)   # kept points first, in order
        kp = torch.gather(pts, 1, order[:, :, None].expand(Cn, K, 3))
        # 2-D frame of the wall plane (build_basis) and the section polygon in it
        with torch.no_grad():
            ex = torch.tensor([1.0, 0.0, 0.0], dtype=torch.float64, device=dev).expand(Cn, 3)
            ey = torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64, device=dev).expand(Cn, 3)
            u = torch.where((torch.abs(n[:, 0]) < 0.9)[:, None], _cross(n, ex), _cross(n, ey))
            un = torch.sqrt(_dot(u, u))
            bu = torch.where((un < 1e-14)[:, None], torch.zeros_like(u), u / un[:, None])
            bv = _cross(n, bu)
        o = wt[:, 0]
        dd = kp - o[:, None, :]
        px, py = _dot(dd, bu[:, None, :]), _dot(dd, bv[:, None, :])
        with torch.no_grad():
            cl = wt - o[:, None, :]
            cx, cy = _dot(cl, bu[:, None, :]), _dot(cl, bv[:, None, :])
            valid = torch.arange(K, device=dev)[None, :] < nu[:, None]
            # Sutherland-Hodgman (src/main.cpp:1093-1122): a section inside all three edges comes back
            # unchanged; one wholly outside any edge comes back empty (its clipped part stays outside that
            # edge); a section that an edge cuts is not handled here
            all_out = torch.zeros(Cn, dtype=torch.bool, device=dev)
            cut = torch.zeros(Cn, dtype=torch.bool, device=dev)
            for c in range(3):
                c1x, c1y = cx[:, (c + 2) % 3, None], cy[:, (c + 2) % 3, None]
                c2x, c2y = cx[:, c, None], cy[:, c, None]
                ins = ((c2x - c1x) * (py - c1y) - (c2y - c1y) * (px - c1x)) >= 0.0
                n_in = (valid & ins).sum(1)
                all_out |= n_in == 0
                cut |= (n_in > 0) & (n_in < nu)
            if bool((cut & ~all_out & (nu >= 3)).any()):
                raise NotImplementedError("differentiable wall contact: a section is clipped by a wall triangle edge")
        idx = torch.arange(K, device=dev)[None, :].expand(Cn, K)
        nxt = torch.where(idx + 1 < nu[:, None], idx + 1, torch.zeros_like(idx))
        qx, qy = torch.gather(px, 1, nxt), torch.gather(py, 1, nxt)
        cr = torch.where(valid, px * qy - py * qx, torch.zeros_like(px))
        ar = torch.abs(cr.sum(1)) * 0.5
        nuf = nu.clamp(min=1).to(torch.float64)
        mx = torch.where(valid, px, torch.zeros_like(px)).sum(1) / nuf
        my = torch.where(valid, py, torch.zeros_like(py)).sum(1) / nuf
        ok = (nu >= 3) & ~all_out & ~(ar.detach() < (tol * tol * 0.01))
        cpt = o + bu * mx[:, None] + bv * my[:, None]
        return ok, ar, cpt

    # ------------------------------------------------------------------------------------------------
    def rollout(self, state0, k, e, steps, checkpoint_every=None):
        """steps steps from state0; returns (final state, stats of the last step).  With
        checkpoint_every, each segment of that many steps keeps only its input for the backward pass and
        recomputes its inside (torch.utils.checkpoint)."""
        hk, hd, wk, wd = self.initial_history()
        hd = hd + 0.0 * k  # the history tensors take part in the graph from the start
        wd = wd + 0.0 * k
        st = state0
        stats = {}

        def seg(st, hd, wd, k, e, hk, wk, n):
            last = {}
            for _ in range(n):
                st, hk, hd, wk, wd, last = self.step(st, hk, hd, wk, wd, k, e)
            return st, hd, wd, hk, wk, last

        done = 0
        while done < steps:
            n = min(checkpoint_every or steps, steps - done)
            if checkpoint_every:
                st, hd, wd, hk, wk, stats = torch.utils.checkpoint.checkpoint(seg, st, hd, wd, k, e, hk, wk, n,
                                                                              use_reentrant=False)
            else:
                st, hd, wd, hk, wk, stats = seg(st, hd, wd, k, e, hk, wk, n)
            done += n
        return st, stats
