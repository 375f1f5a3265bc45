"""Differentiable rollouts (zdemx.rollout): the torch step against the CUDA scene step, reverse-mode
gradients of a final-position loss against central differences, checkpointed against unsegmented."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene(tmp_path, n_side=3, seed=5):
    from zdemx.dem import Scene
    from zdemx.workloads import calibration_scene

    cfg = calibration_scene(str(tmp_path / "cal"), n_side=n_side, seed=seed, steps=100, spacing=1.8e-3)
    return Scene(cfg)


def test_torch_step_follows_the_cuda_step(tmp_path):
    """Same counters every step; state within summation-order rounding (forces summed in another order)."""
    import torch

    from zdemx.rollout import DiffScene

    sc = _scene(tmp_path)
    ds = DiffScene(sc)
    st = torch.from_numpy(sc.state()[0]).cuda()
    hk, hd, wk, wd = ds.initial_history()
    k = torch.tensor(ds.feng_k, dtype=torch.float64, device="cuda")
    e = torch.tensor(float(ds.mat[0, 7]), dtype=torch.float64, device="cuda")
    seen = 0
    with torch.no_grad():
        for s in range(40):
            sc.step(1)
            st, hk, hd, wk, wd, stats = ds.step(st, hk, hd, wk, wd, k, e)
            info = sc.info()
            assert info["pairs"] == stats["pairs"], f"step {s}: pairs"
            assert info["contacts"] == stats.get("contacts", 0) + stats["wall_contacts"], f"step {s}: contacts"
            assert info["wall_contacts"] == stats["wall_contacts"], f"step {s}: wall contacts"
            assert info["history"] == hk.numel() and info["wall_history"] == wk.numel()
            seen += info["contacts"]
    ref = sc.state()[0]
    got = st.cpu().numpy()
    for cols, tol in ((slice(0, 3), 1e-12), (slice(7, 10), 1e-7), (slice(3, 7), 1e-12)):
        scale = max(np.max(np.abs(ref[:, cols])), 1e-300)
        err = np.max(np.abs(got[:, cols] - ref[:, cols])) / scale
        assert err <= tol, f"cols {cols}: rel err {err}"
    assert seen > 0


def _loss_fn(ds, state0, v_init, target, steps):
    import torch

    def loss(k, e, v0, checkpoint_every=None):
        st = torch.cat([state0[:, 0:7], v0, state0[:, 10:16]], 1)
        xT, _ = ds.rollout(st, k, e, steps, checkpoint_every=checkpoint_every)
        return ((xT[:, 0:3] - target) ** 2).sum()

    return loss


def test_rollout_gradients_match_central_differences(tmp_path):
    import torch

    from zdemx.rollout import DiffScene

    sc = _scene(tmp_path)
    ds = DiffScene(sc)
    state0 = torch.from_numpy(sc.state()[0]).cuda()
    steps = 30
    with torch.no_grad():
        tgt, _ = ds.rollout(state0, torch.tensor(1.3e7, dtype=torch.float64, device="cuda"),
                            torch.tensor(0.35, dtype=torch.float64, device="cuda"), steps)
    target = tgt[:, 0:3].clone()
    loss = _loss_fn(ds, state0, None, target, steps)
    k = torch.tensor(1e7, dtype=torch.float64, device="cuda", requires_grad=True)
    e = torch.tensor(0.5, dtype=torch.float64, device="cuda", requires_grad=True)
    v0 = state0[:, 7:10].clone().requires_grad_(True)
    L = loss(k, e, v0)
    L.backward()
    assert k.grad is not None and e.grad is not None, "no particle-particle contact in the rollout"
    gk, ge, gv = k.grad.item(), e.grad.item(), v0.grad.cpu().numpy()
    with torch.no_grad():
        def fd(fn, h):
            return (fn(h) - fn(-h)) / (2 * h)

        fk = fd(lambda h: loss(k + h, e, v0).item(), 1e7 * 1e-6)
        fe = fd(lambda h: loss(k, e + h, v0).item(), 1e-6)
        idx = [(0, 0), (13, 2), (26, 1)]
        fv = []
        for i, c in idx:
            def f(h, i=i, c=c):
                vv = v0.clone()
                vv[i, c] += h
                return loss(k, e, vv).item()
            fv.append(fd(f, 1e-7))
    assert abs(gk - fk) <= 1e-4 * abs(fk) + 1e-30, (gk, fk)
    assert abs(ge - fe) <= 1e-4 * abs(fe) + 1e-30, (ge, fe)
    for (i, c), f in zip(idx, fv):
        assert abs(gv[i, c] - f) <= 1e-4 * max(abs(f), np.max(np.abs(gv)) * 1e-3), (i, c, gv[i, c], f)


def test_checkpointed_rollout_gives_the_same_gradients(tmp_path):
    import torch

    from zdemx.rollout import DiffScene

    sc = _scene(tmp_path, seed=6)
    ds = DiffScene(sc)
    state0 = torch.from_numpy(sc.state()[0]).cuda()
    target = state0[:, 0:3] + 1e-5
    loss = _loss_fn(ds, state0, None, target, 24)
    out = []
    for ck in (None, 8):
        k = torch.tensor(1e7, dtype=torch.float64, device="cuda", requires_grad=True)
        e = torch.tensor(0.5, dtype=torch.float64, device="cuda", requires_grad=True)
        v0 = state0[:, 7:10].clone().requires_grad_(True)
        L = loss(k, e, v0, checkpoint_every=ck)
        L.backward()
        out.append((L.item(), k.grad.item(), e.grad.item(), v0.grad.cpu().numpy()))
    (l0, k0, e0, v0a), (l1, k1, e1, v1a) = out
    assert l0 == l1
    np.testing.assert_allclose([k1, e1], [k0, e0], rtol=1e-10)
    np.testing.assert_allclose(v1a, v0a, rtol=1e-10, atol=1e-10 * np.max(np.abs(v0a)))


def test_cuda_wall_contacts_match_the_torch_ones(tmp_path):
    """The wall contacts through the CUDA kernels and their hand-written reverse mode against the same
    computation in torch autograd (sections inside their triangle, where both apply): forces, torques,
    histories and contact counts to rounding, and the gradients of a random linear functional of them
    with respect to the state and e."""
    import torch

    from zdemx.rollout import DiffScene

    sc = _scene(tmp_path, seed=7)
    ds = DiffScene(sc)
    st = torch.from_numpy(sc.state()[0]).cuda()
    hk, hd, wk, wd = ds.initial_history()
    k = torch.tensor(ds.feng_k, dtype=torch.float64, device="cuda")
    e0 = torch.tensor(0.5, dtype=torch.float64, device="cuda")
    with torch.no_grad():
        for _ in range(25):
            st, hk, hd, wk, wd, stats = ds.step(st, hk, hd, wk, wd, k, e0)
    assert wk.numel() > 0, "no wall contact yet"
    rng = np.random.default_rng(3)
    res = []
    for fn in (ds._walls, ds._walls_torch):
        s = st.clone().requires_grad_(True)
        e = e0.clone().requires_grad_(True)
        wdd = wd.clone().requires_grad_(True)
        Fw, Tw, key, dso, nwc = fn(s, wk, wdd, e)
        a = torch.from_numpy(rng.normal(size=Fw.shape)).cuda()
        b = torch.from_numpy(rng.normal(size=Tw.shape)).cuda() * 1e3
        c = torch.from_numpy(rng.normal(size=dso.shape)).cuda() * 1e6
        rng = np.random.default_rng(3)  # the same functional for both
        L = (a * Fw).sum() + (b * Tw).sum() + (c * dso).sum()
        L.backward()
        res.append((Fw.detach(), Tw.detach(), key, dso.detach(), nwc, s.grad, e.grad, wdd.grad))
    (F1, T1, k1, d1, n1, gs1, ge1, gw1), (F2, T2, k2, d2, n2, gs2, ge2, gw2) = res
    assert n1 == n2 > 0 and torch.equal(k1, k2)
    for x, y in ((F1, F2), (T1, T2), (d1, d2), (gs1, gs2), (gw1, gw2)):
        scale = float(y.abs().max())
        assert scale > 0 and float((x - y).abs().max()) <= 1e-9 * scale
    assert abs(float(ge1) - float(ge2)) <= 1e-9 * abs(float(ge2))


@pytest.mark.parametrize("n, spread, seed", [(1, 1.0, 0), (2, 5e-4, 1), (700, 0.02, 2), (3000, 0.05, 3)])
def test_binned_broad_phase_matches_all_pairs(n, spread, seed):
    """zdx_broad_phase (cells, sort, sphere test) gives the all-pairs test's candidates in its (i, j) order,
    also when the caller's buffer is too small (the binding grows it) and with unequal radii."""
    import torch

    from zdemx import _lib
    from zdemx.autograd import ctx_handle

    rng = np.random.default_rng(seed)
    state = np.zeros((n, 16))
    state[:, 0:3] = rng.uniform(0.0, spread, size=(n, 3))
    state[:, 3] = 1.0
    mat = np.zeros((n, 17))
    mat[:, 2] = rng.uniform(5e-4, 1.5e-3, size=n)
    st = torch.from_numpy(state).cuda()
    mt = torch.from_numpy(mat).cuda()
    x = st[:, 0:3]
    d = x[None, :, :] - x[:, None, :]
    dist2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
    rs = mt[:, 2][:, None] + mt[:, 2][None, :]
    pi, pj = torch.nonzero(torch.triu(~(dist2 > rs * rs), diagonal=1), as_tuple=True)
    ctx = ctx_handle(torch.device("cuda", 0))
    small = torch.zeros(1, 2, dtype=torch.int32, device="cuda")
    for buf in (None, small):
        cand, _ = _lib.broad_phase(ctx, st, mt, buf)
        assert cand.shape[0] == pi.numel()
        assert torch.equal(cand[:, 0].long(), pi) and torch.equal(cand[:, 1].long(), pj)
    if n > 1:
        assert pi.numel() > 0


def test_cuda_integration_matches_the_torch_one(tmp_path):
    """zdx_integrate and its hand-written reverse mode against integrate_particle in torch autograd: the new
    state to rounding, and the gradients of a random linear functional of it with respect to the old state
    (quaternions off unit length), the forces and the torques."""
    import torch

    from zdemx.autograd import ctx_handle
    from zdemx.rollout import DiffScene, _Integrate

    sc = _scene(tmp_path, seed=9)
    ds = DiffScene(sc)
    rng = np.random.default_rng(4)
    n = ds.np
    st0 = torch.from_numpy(sc.state()[0]).cuda()
    st0[:, 3:7] *= torch.from_numpy(rng.uniform(0.8, 1.2, size=(n, 1))).cuda()
    st0[:, 13:16] = torch.from_numpy(rng.normal(size=(n, 3)) * 1e-9).cuda()
    F0 = torch.from_numpy(rng.normal(size=(n, 3)) * 1e-2).cuda()
    T0 = torch.from_numpy(rng.normal(size=(n, 3)) * 1e-5).cuda()
    w = torch.from_numpy(rng.normal(size=(n, 16))).cuda()
    consts = {"ctx": ctx_handle(st0.device), "mat": ds.mat, "g": ds.g_host, "dt": ds.dt}
    res = []
    for fn in (lambda s, f, t: _Integrate.apply(s, f, t, consts), ds.integrate_torch):
        s, f, t = (a.clone().requires_grad_(True) for a in (st0, F0, T0))
        out = fn(s, f, t)
        (w * out).sum().backward()
        res.append((out.detach(), s.grad, f.grad, t.grad))
    for a, b in zip(res[0], res[1]):
        scale = float(b.abs().max())
        assert scale > 0 and float((a - b).abs().max()) <= 1e-12 * scale
