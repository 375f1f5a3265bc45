"""Autotuner of the pair kernels' launch parameters (zdx_tuning), written for this library.

The knobs change how the batched pair call is launched, never what it computes:

* ``tri_ctas_per_sm``  triangle-stage CTAs resident per SM (each holds one pair's survivors);
* ``flat_max``         survivor pairs nA' x nB' up to which the triangle stage tests every box pair
                       directly, above which it uses the Morton-ordered group boxes;
* ``rebuild_warps``    warps per rebuild block (one warp per pair);
* ``split_tests``      in a batch with fewer pairs than triangle-stage CTAs, the triangle tests per work
                       item into which large pairs are split (0: no split);
* ``rebuild_arena``    the rebuild's form: one warp per pair over global-memory slots (0), the large
                       pairs in arenas alongside form 0 on the small ones (1), or arenas for every
                       pair (2);
* ``arena_warps``      warps per SM given arenas;
* ``arena_min_seg``    the segment count from which form 1 gives a pair an arena.

On a seeded calibration sample of a workload the tuner times the call (the library's own CUDA events)
for each candidate value of one knob with the others held, keeps the fastest, and goes over the knobs
twice (coordinate descent).  Every candidate's results are compared with the default launch's, bit for
bit; a candidate that changed them would be a bug and stops the tuning.  The winner is written as the
JSON file that ``zdx_create`` reads when the environment variable ZDX_TUNING names it.

    python -m zdemx.autotune --pairs 16384 --out tuning.json     # the pair sweep's mix
"""
from __future__ import annotations

import json
import statistics

import numpy as np

from . import _lib

GRID = {
    "flat_max": (0, 2048, 8192, 32768, 131072),
    "tri_ctas_per_sm": (1, 2),
    "rebuild_warps": (1, 2, 4),
    "split_tests": (0, 16384, 131072),
    "rebuild_arena": (0, 1, 2),
    "arena_warps": (4, 8, 12, 16),
    "arena_min_seg": (96, 192, 384),
}
DEFAULTS = {"tri_ctas_per_sm": 2, "rebuild_warps": 4, "flat_max": 8192, "split_tests": 0, "rebuild_arena": 0,
            "arena_warps": 8, "arena_min_seg": 192}


def _snapshot(out, n_contacts):
    return {k: out[k].clone() for k in ("ncontact", "contact_off", "stats")} | {"geom": out["geom"][:n_contacts].clone()}


def _same(a, b) -> bool:
    import torch

    return all(torch.equal(a[k], b[k]) for k in a)


def tune(ctx: _lib.Context, meshes: dict, pairs: dict, out: dict, *, reps: int = 3, passes: int = 2, k: float = 1e7,
         split: bool = True, grid: dict | None = None, flush=None) -> dict:
    """Tune the launch parameters of `ctx` on one batch (device tensors, as ``_lib.pair_contacts_device``
    takes them).  Leaves the best parameters set on `ctx` and returns them with every trial's time."""
    import torch

    grid = dict(GRID if grid is None else grid)
    trials = []

    def timed(params):
        ctx.set_tuning(**params)
        tot = _lib.pair_contacts_device(ctx, meshes, pairs, out, k=k, split=split)
        ms = []
        for _ in range(reps):
            if flush is not None:
                flush.zero_()
            torch.cuda.synchronize()
            _lib.pair_contacts_device(ctx, meshes, pairs, out, k=k, split=split)
            ms.append(ctx.timings()["total"])
        return statistics.median(ms), tot

    best = dict(DEFAULTS)
    best_ms, tot0 = timed(best)
    ref = _snapshot(out, int(tot0[0]))
    trials.append({"params": dict(best), "ms": best_ms})
    default_ms = best_ms
    for _ in range(passes):
        changed = False
        for knob, values in grid.items():
            for v in values:
                if v == best[knob]:
                    continue
                cand = dict(best)
                cand[knob] = v
                ms, tot = timed(cand)
                if not _same(ref, _snapshot(out, int(tot[0]))):
                    ctx.set_tuning(**DEFAULTS)
                    raise RuntimeError(f"launch parameters {cand} changed the results")
                trials.append({"params": dict(cand), "ms": ms})
                if ms < best_ms * 0.99:
                    best, best_ms, changed = cand, ms, True
        if not changed:
            break
    ctx.set_tuning(**best)
    return {"best": best, "best_ms": best_ms, "default_ms": default_ms, "pairs": int(pairs["mesh"].shape[0]),
            "trials": trials}


def save(path: str, params: dict) -> None:
    """Write the tuning file zdx_create reads (ZDX_TUNING=path)."""
    with open(path, "w") as f:
        json.dump({k: int(params[k]) for k in DEFAULTS}, f, indent=1)


def sweep_sample(n_pairs: int, seed: int, per_level: int = 64):
    """A calibration sample of the pair sweep's mix: pairs of noised icospheres of subdivision U{1..4}
    (radius 1 mm, +-15 % noise) at overlap depth U(0, 0.1) r, meshes from a library of `per_level` per
    subdivision.  Returns (MeshLibrary, pair_mesh, pair_pose)."""
    from . import synth
    from .contact import MeshLibrary

    rng = np.random.default_rng(seed)
    raw = []
    for s in (1, 2, 3, 4):
        raw.extend(list(synth.noised_icospheres(s, per_level, 1e-3, 0.15, rng)))
    lib = MeshLibrary.build(raw)
    lv = rng.integers(0, 4, size=(n_pairs, 2))
    pm = (lv * per_level + rng.integers(0, per_level, size=(n_pairs, 2))).astype(np.int32)
    pp = synth.pair_poses(rng, n_pairs, 1e-3, 0.0, 0.1)
    return lib, pm, pp


def device_batch(lib, pm, pp, device):
    """The device tensors of one batch and its output buffers (16 contacts a pair)."""
    import torch

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    meshes = {"tris": t(lib.tris), "tri_off": t(lib.tri_off), "mean_edge": t(lib.mean_edge), "bbox_diag": t(lib.bbox_diag)}
    pairs = {"mesh": t(pm), "pose": t(pp)}
    n = len(pm)
    out = {"ncontact": torch.zeros(n, dtype=torch.int32, device=device),
           "contact_off": torch.zeros(n + 1, dtype=torch.int64, device=device),
           "stats": torch.zeros(n, 4, dtype=torch.int32, device=device),
           "geom": torch.zeros(16 * n, 20, dtype=torch.float64, device=device),
           "info": torch.zeros(16 * n, 4, dtype=torch.int32, device=device)}
    return meshes, pairs, out


def main(argv=None) -> int:
    import argparse

    import torch

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--pairs", type=int, default=16384)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default="zdemx_tuning.json")
    args = ap.parse_args(argv)
    dev = torch.device("cuda", args.device)
    ctx = _lib.Context(args.device)
    lib, pm, pp = sweep_sample(args.pairs, args.seed)
    meshes, pairs, out = device_batch(lib, pm, pp, dev)
    res = tune(ctx, meshes, pairs, out)
    save(args.out, res["best"])
    print(json.dumps({k: v for k, v in res.items() if k != "trials"}))
    ctx.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
