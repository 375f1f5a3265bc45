"""Hand-written adjoint of the contact geometry (zdx_pair_contacts_adjoint, zdemx.autograd).

* Central finite differences of L = sum_c wS_c.Sn_c + wG_c.Gn_c through the forward call, with respect
  to the translations, world-frame rotation vectors and quaternion components of both bodies and to
  sampled mesh-local triangle corners: relative error <= 1e-6 of the gradient group's scale.  A
  coordinate whose +h or -h evaluation changes the topology (segment, component, loop or contact counts,
  loop vertex counts) is skipped, since the function is only piecewise smooth there.
* Host-memory and device-memory adjoint calls, and the batched and plain forms, agree to rounding (the
  scatter is atomic).
* The physical identity d(overlap volume)/d(translation of B) = -Sn for convex bodies: the overlap volume
  of two convex hulls comes from scipy's half-space intersection, independent of the library.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R = 1e-3


def _library(rng, kind="ico"):
    from zdemx import synth
    from zdemx.contact import MeshLibrary

    if kind == "ico":
        soups = [synth.noised_icosphere(2, R, 0.15, rng) for _ in range(2)]
    else:
        soups = [synth.ellipsoid_hull(80, (1.0, 0.8, 0.6), R, rng) for _ in range(2)]
    return MeshLibrary.build(soups)


def _poses(rng, n):
    from zdemx import synth

    p = synth.pair_poses(rng, n, R, 0.01, 0.08)
    p[:, 3:7] = synth.random_unit_quat(rng, n)
    return p


def _qexp(theta):
    a = np.linalg.norm(theta)
    if a < 1e-300:
        return np.array([1.0, 0, 0, 0])
    return np.r_[np.cos(a / 2), np.sin(a / 2) * theta / a]


def _qmul(a, b):
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw])


class _Objective:
    """L and the topology signature of one forward call on host buffers."""

    def __init__(self, ctx, lib, pm, mode, split, tol, rng):
        from zdemx import _lib

        self.ctx, self.lib, self.pm, self.mode, self.split, self.tol = ctx, lib, pm, mode, split, tol
        self._lib = _lib
        self.base_tris = lib.tris.copy()
        self.wS = self.wG = None
        self.rng = rng

    def run(self, tris, pose):
        r = self._lib.pair_contacts_raw(self.ctx, tris, self.lib.tri_off, self.lib.mean_edge, self.lib.bbox_diag,
                                        self.pm, pose, mode=self.mode, split=self.split, tol=self.tol)
        return r

    def weights(self, n):
        self.wS = self.rng.normal(size=(n, 3)) / R ** 2
        self.wG = self.rng.normal(size=(n, 3)) / R ** 3

    def value(self, r):
        g = r["geom"]
        return float(np.sum(self.wS * g[:, 0:3]) + np.sum(self.wG * g[:, 3:6]))

    @staticmethod
    def topo(r):
        return (r["stats"].tobytes(), r["info"].tobytes(), r["contact_off"].tobytes())


def _fd_check(ctx, lib, pose, pm, mode, split, tol, rng, n_corners=16, h_rel=1e-6):
    from zdemx import _lib

    obj = _Objective(ctx, lib, pm, mode, split, tol, rng)
    base = obj.run(lib.tris, pose)
    n = int(base["totals"][0])
    assert n > 0, "no contacts to differentiate"
    obj.weights(n)
    sig = obj.topo(base)
    gc = np.ascontiguousarray(np.concatenate([obj.wS, obj.wG], 1))
    gt = np.zeros_like(lib.tris)
    gp = np.zeros((len(pm), 12))
    meshes = {"tris": lib.tris, "tri_off": lib.tri_off, "mean_edge": lib.mean_edge, "bbox_diag": lib.bbox_diag}
    pairs = {"mesh": np.ascontiguousarray(pm, np.int32), "pose": np.ascontiguousarray(pose)}
    _lib.pair_contacts_adjoint(ctx, meshes, pairs, gc, gt, gp, mode=mode, split=split, tol=tol, mem=_lib.MEM_HOST)
    h = h_rel * R
    checked, skipped = {"pos": [], "rot": [], "corner": []}, 0

    def central(fp, fm):
        nonlocal skipped
        rp, rm = fp(), fm()
        if obj.topo(rp) != sig or obj.topo(rm) != sig:
            skipped += 1
            return None
        return (obj.value(rp) - obj.value(rm)) / (2 * h)

    for p in range(len(pm)):
        for b in range(2):
            for k in range(3):
                def shifted(s, p=p, b=b, k=k):
                    q = pose.copy()
                    q[p, 7 * b + k] += s
                    return obj.run(lib.tris, q)

                fd = central(lambda: shifted(h), lambda: shifted(-h))
                if fd is not None:
                    checked["pos"].append((gp[p, 6 * b + k], fd))

                def rotated(s, p=p, b=b, k=k):
                    q = pose.copy()
                    e = np.zeros(3)
                    e[k] = s / R
                    q[p, 7 * b + 3: 7 * b + 7] = _qmul(_qexp(e), pose[p, 7 * b + 3: 7 * b + 7])
                    return obj.run(lib.tris, q)

                fd = central(lambda: rotated(h), lambda: rotated(-h))
                if fd is not None:
                    checked["rot"].append((gp[p, 6 * b + 3 + k], fd * R))
    nz = np.flatnonzero(np.abs(gt).reshape(-1) > 0)
    z = np.flatnonzero(np.abs(gt).reshape(-1) == 0)
    pick = list(rng.choice(nz, size=min(n_corners, len(nz)), replace=False)) + list(rng.choice(z, size=4, replace=False))
    for idx in pick:
        def moved(s, idx=idx):
            t = lib.tris.copy().reshape(-1)
            t[idx] += s
            return obj.run(t.reshape(lib.tris.shape), pose)

        fd = central(lambda: moved(h), lambda: moved(-h))
        if fd is not None:
            checked["corner"].append((gt.reshape(-1)[idx], fd))
    for name, rows in checked.items():
        assert len(rows) >= 3, f"too few {name} coordinates checked ({len(rows)}, skipped {skipped})"
        a = np.array(rows)
        scale = np.max(np.abs(a[:, 1]))
        err = np.max(np.abs(a[:, 0] - a[:, 1])) / scale
        assert err <= 1e-6, f"{name}: adjoint vs central difference rel err {err:.3e}\n{a}"
    return gt, gp, skipped


def test_adjoint_matches_central_differences_zdem(ctx):
    rng = np.random.default_rng(11)
    lib = _library(rng)
    pose = _poses(rng, 3)
    pm = np.array([[0, 1], [1, 0], [0, 0]], np.int32)
    _fd_check(ctx, lib, pose, pm, mode=0, split=True, tol=0.0, rng=rng)


def test_adjoint_matches_central_differences_polyline(ctx):
    rng = np.random.default_rng(12)
    lib = _library(rng)
    pose = _poses(rng, 2)
    pm = np.array([[0, 1], [1, 1]], np.int32)
    _fd_check(ctx, lib, pose, pm, mode=1, split=False, tol=1e-6 * R * 10, rng=rng, n_corners=12)


def test_adjoint_host_and_device_agree(ctx):
    import torch

    from zdemx import _lib

    rng = np.random.default_rng(13)
    lib = _library(rng)
    pose = _poses(rng, 8)
    pm = np.ascontiguousarray(rng.integers(0, 2, size=(8, 2)), np.int32)
    base = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pm, pose)
    n = int(base["totals"][0])
    gc = rng.normal(size=(n, 6))
    meshes = {"tris": lib.tris, "tri_off": lib.tri_off, "mean_edge": lib.mean_edge, "bbox_diag": lib.bbox_diag}
    pairs = {"mesh": pm, "pose": pose}
    gt_h, gp_h = np.zeros_like(lib.tris), np.zeros((8, 12))
    _lib.pair_contacts_adjoint(ctx, meshes, pairs, gc, gt_h, gp_h, mem=_lib.MEM_HOST)
    dev = torch.device("cuda:0")
    dm = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in meshes.items()}
    dp = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in pairs.items()}
    gt_d = torch.zeros(lib.tris.shape, dtype=torch.float64, device=dev)
    gp_d = torch.zeros(8, 12, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    _lib.pair_contacts_adjoint(ctx, dm, dp, torch.from_numpy(gc).to(dev), gt_d, gp_d, mem=_lib.MEM_DEVICE)
    # the scatter is atomic, so summation order may differ between calls: agree to rounding
    np.testing.assert_allclose(gt_d.cpu().numpy(), gt_h, rtol=1e-12, atol=1e-12 * np.max(np.abs(gt_h)))
    np.testing.assert_allclose(gp_d.cpu().numpy(), gp_h, rtol=1e-12, atol=1e-12 * np.max(np.abs(gp_h)))
    # a wrong contact count is an error, not a silent mismatch
    with pytest.raises(_lib.ZdxError):
        _lib.pair_contacts_adjoint(ctx, meshes, pairs, gc[:-1].copy(), gt_h, gp_h, mem=_lib.MEM_HOST)
    # the plain form (one launch per pair per stage) gives the same gradients
    gt_p, gp_p = np.zeros_like(lib.tris), np.zeros((8, 12))
    _lib.pair_contacts_adjoint(ctx, meshes, pairs, gc, gt_p, gp_p, mem=_lib.MEM_HOST, sched=_lib.SCHED_PLAIN)
    np.testing.assert_allclose(gt_p, gt_h, rtol=1e-12, atol=1e-12 * np.max(np.abs(gt_h)))
    np.testing.assert_allclose(gp_p, gp_h, rtol=1e-12, atol=1e-12 * np.max(np.abs(gp_h)))


def test_autograd_pose_quaternion_and_k(ctx):
    """torch.autograd through zdemx.autograd.pair_contacts: quaternion components (the forward
    normalises them) against central differences, and dFn/dk = |Sn|/2."""
    import torch

    from zdemx import _lib
    from zdemx.autograd import pair_contacts

    rng = np.random.default_rng(14)
    lib = _library(rng)
    pose = _poses(rng, 2)
    pm = np.array([[0, 1], [1, 0]], np.int32)
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    tris = T(lib.tris).requires_grad_(True)
    pose_t = T(pose).requires_grad_(True)
    k = torch.tensor(1e7, dtype=torch.float64, device=dev, requires_grad=True)
    out = pair_contacts(tris, pose_t, T(lib.tri_off), T(lib.mean_edge), T(lib.bbox_diag), T(pm), k=k)
    n = out["Sn"].shape[0]
    assert n > 0
    wS = torch.from_numpy(rng.normal(size=(n, 3)) / R ** 2).to(dev)
    wG = torch.from_numpy(rng.normal(size=(n, 3)) / R ** 3).to(dev)
    L = (wS * out["Sn"]).sum() + (wG * out["Gn"]).sum() + out["Fn"].sum() / 1e7 / R ** 2
    L.backward()
    np.testing.assert_allclose(k.grad.item(), (out["area"].sum() / 2 / 1e7 / R ** 2).item(), rtol=1e-12)
    gq = pose_t.grad.cpu().numpy()

    def value(p):
        r = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pm, p, k=1e7)
        g = r["geom"]
        if len(g) != n:
            return None
        return float(np.sum(wS.cpu().numpy() * g[:, 0:3]) + np.sum(wG.cpu().numpy() * g[:, 3:6]) +
                     np.sum(g[:, 13]) / 1e7 / R ** 2)

    h = 1e-7
    rows = []
    for p in range(2):
        for c in list(range(3, 7)) + list(range(10, 14)):
            a, b = pose.copy(), pose.copy()
            a[p, c] += h
            b[p, c] -= h
            va, vb = value(a), value(b)
            if va is None or vb is None:
                continue
            rows.append((gq[p, c], (va - vb) / (2 * h)))
    a = np.array(rows)
    assert len(a) >= 8
    err = np.max(np.abs(a[:, 0] - a[:, 1])) / np.max(np.abs(a[:, 1]))
    assert err <= 1e-6, f"quaternion grad rel err {err:.3e}\n{a}"


def _overlap_volume(tris_a, pose_a, tris_b, pose_b):
    from scipy.optimize import linprog
    from scipy.spatial import ConvexHull, HalfspaceIntersection

    def halfspaces(tris, pose):
        q = pose[3:7] / np.linalg.norm(pose[3:7])
        w, x, y, z = q
        Rm = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                       [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                       [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        W = (tris.reshape(-1, 3) @ Rm.T + pose[:3]).reshape(-1, 3, 3)
        nrm = np.cross(W[:, 1] - W[:, 0], W[:, 2] - W[:, 0])
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        return np.c_[nrm, -np.einsum("ij,ij->i", nrm, W[:, 0])]

    H = np.r_[halfspaces(tris_a, pose_a), halfspaces(tris_b, pose_b)]
    nn = np.linalg.norm(H[:, :3], axis=1)
    lp = linprog(np.r_[0, 0, 0, -1.0], A_ub=np.c_[H[:, :3], nn], b_ub=-H[:, 3], bounds=[(None, None)] * 3 + [(0, None)])
    return ConvexHull(HalfspaceIntersection(H, lp.x[:3]).intersections).volume


@pytest.mark.parametrize("mode,tol,rtol", [(1, 1e-9 * R, 1e-6), (0, 0.0, 0.08)])
def test_volume_identity(ctx, mode, tol, rtol):
    """dV_overlap/dt_B = -Sn for convex bodies.  With a snap tolerance far below the mesh size the loop
    is the exact intersection polygon and the identity holds to rounding.  In zdem mode the loop's
    traversal direction is arbitrary and the reference orients the contact by flipping nA toward B, so
    the identity reads dV/dt_B = -|Sn| nA; zdem's snap tolerance (a tenth of the mean edge) moves loop
    vertices, so there it holds to a few percent."""
    from zdemx import _lib

    rng = np.random.default_rng(15)
    lib = _library(rng, kind="hull")
    A, B = lib.mesh(0), lib.mesh(1)
    poses = []
    for _ in range(3):
        p = np.zeros(14)
        p[3] = 1.0
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        p[7:10] = d * R * 1.0
        p[10:14] = rng.normal(size=4)
        p[10:14] /= np.linalg.norm(p[10:14])
        poses.append(p)
    poses = np.array(poses)
    pm = np.array([[0, 1]] * len(poses), np.int32)
    r = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pm, poses, mode=mode,
                               split=mode == 0, tol=tol)
    h = 1e-7 * R
    for p in range(len(poses)):
        a, b = r["contact_off"][p], r["contact_off"][p + 1]
        if b == a:
            continue
        geom = r["geom"][a:b]
        Sn = geom[:, 0:3].sum(0) if mode == 1 else (geom[:, 12:13] * geom[:, 9:12]).sum(0)
        g = np.zeros(3)
        for k in range(3):
            pp, pm_ = poses[p].copy(), poses[p].copy()
            pp[7 + k] += h
            pm_[7 + k] -= h
            g[k] = (_overlap_volume(A, pp[:7], B, pp[7:]) - _overlap_volume(A, pm_[:7], B, pm_[7:])) / (2 * h)
        err = np.linalg.norm(g + Sn) / np.linalg.norm(Sn)
        assert err <= rtol, f"pair {p}: dV/dt_B {g} vs -Sn {-Sn} (rel {err:.3e})"
