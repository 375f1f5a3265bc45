"""Launch parameters of the pair kernels (zdx_tuning): the tuning file zdx_create reads, range checks, and
results that do not depend on the parameters (every value of every knob, against the defaults, bit for
bit), plus the autotuner on a small calibration sample."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tuning_file_and_range_checks(tmp_path):
    path = tmp_path / "t.json"
    path.write_text(json.dumps({"flat_max": 2048, "rebuild_warps": 2, "tri_ctas_per_sm": 1, "other": 5}))
    code = ("import sys; sys.path.insert(0, %r); from zdemx import _lib; c = _lib.Context(0); "
            "import json; print(json.dumps(c.tuning()))") % os.path.join(ROOT, "zedm-x_b200")
    env = dict(os.environ, ZDX_TUNING=str(path))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    got = json.loads(p.stdout.strip().splitlines()[-1])
    assert got == {"tri_ctas_per_sm": 1, "rebuild_warps": 2, "flat_max": 2048, "split_tests": 0,
                   "rebuild_arena": 0, "arena_warps": 8, "arena_min_seg": 192}
    # a value out of range leaves the defaults
    path.write_text(json.dumps({"flat_max": 2048, "rebuild_warps": 99}))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert json.loads(p.stdout.strip().splitlines()[-1])["rebuild_warps"] == 4

    from zdemx import _lib

    ctx = _lib.Context(0)
    try:
        with pytest.raises(_lib.ZdxError):
            ctx.set_tuning(tri_ctas_per_sm=3)
        with pytest.raises(_lib.ZdxError):
            ctx.set_tuning(rebuild_warps=0)
        with pytest.raises(_lib.ZdxError):
            ctx.set_tuning(rebuild_arena=4)
        with pytest.raises(_lib.ZdxError):
            ctx.set_tuning(arena_warps=0)
        assert ctx.set_tuning(flat_max=0)["flat_max"] == 0
    finally:
        ctx.close()


def test_results_do_not_depend_on_launch_parameters():
    import torch

    from zdemx import _lib, autotune

    lib, pm, pp = autotune.sweep_sample(192, seed=11, per_level=3)
    meshes, pairs, out = autotune.device_batch(lib, pm, pp, torch.device("cuda", 0))
    ctx = _lib.Context(0)
    try:
        for split in (True, False):
            ctx.set_tuning(**autotune.DEFAULTS)
            tot = _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7, split=split)
            ref = {k: v.clone() for k, v in out.items()}
            n = int(tot[0])
            assert n > 0
            # every knob value, and the arena form's test of its fallback path (rebuild_arena 3)
            cases = [(knob, v) for knob, values in autotune.GRID.items() for v in values] + [("rebuild_arena", 3)]
            for knob, v in cases:
                ctx.set_tuning(**dict(autotune.DEFAULTS, **{knob: v}))
                t2 = _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7, split=split)
                assert t2[:3] == tot[:3], (knob, v)
                for key in ("ncontact", "contact_off", "stats"):
                    assert torch.equal(out[key], ref[key]), (knob, v, key)
                assert torch.equal(out["geom"][:n], ref["geom"][:n]), (knob, v)
                assert torch.equal(out["info"][:n], ref["info"][:n]), (knob, v)
    finally:
        ctx.close()


def test_autotuner_picks_from_its_grid_and_writes_the_file(tmp_path):
    import torch

    from zdemx import _lib, autotune

    lib, pm, pp = autotune.sweep_sample(512, seed=12, per_level=4)
    meshes, pairs, out = autotune.device_batch(lib, pm, pp, torch.device("cuda", 0))
    ctx = _lib.Context(0)
    try:
        res = autotune.tune(ctx, meshes, pairs, out, reps=2, passes=1)
        best = res["best"]
        for knob, values in autotune.GRID.items():
            assert best[knob] in values
        assert res["best_ms"] <= res["default_ms"]
        assert ctx.tuning() == best
        path = tmp_path / "tuned.json"
        autotune.save(str(path), best)
        assert json.loads(path.read_text()) == best
    finally:
        ctx.close()


def test_split_pairs_give_the_same_adjoint():
    """The adjoint re-runs the forward call with its tape; with large pairs split across CTAs the tape's
    segment provenance is joined with the segments, so the gradients are those of the unsplit call (to
    the last bits that the adjoint's FP64 atomics may reorder)."""
    import torch

    from zdemx import _lib, autotune

    lib, pm, pp = autotune.sweep_sample(48, seed=13, per_level=2)
    dev = torch.device("cuda", 0)
    meshes, pairs, out = autotune.device_batch(lib, pm, pp, dev)
    ctx = _lib.Context(0)
    try:
        grads = []
        for split_tests in (0, 16384):
            ctx.set_tuning(split_tests=split_tests)
            tot = _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7)
            n = int(tot[0])
            assert n > 10
            w = torch.from_numpy(np.random.default_rng(3).normal(size=(n, 6))).to(dev)
            gt = torch.zeros_like(meshes["tris"])
            gp = torch.zeros(len(pm), 12, dtype=torch.float64, device=dev)
            _lib.pair_contacts_adjoint(ctx, meshes, pairs, w, gt, gp)
            grads.append((gt.cpu().numpy(), gp.cpu().numpy()))
        for a, b in zip(grads[0], grads[1]):
            scale = np.max(np.abs(a))
            assert scale > 0 and np.max(np.abs(a - b)) <= 1e-12 * scale
    finally:
        ctx.close()
