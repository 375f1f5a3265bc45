#!/usr/bin/env python3
"""Benchmark: the batched contact-geometry sweep (pair-contacts/s) on B200.

Workload (one step): 65,536 independent pairs of seeded noised icospheres, each mesh's subdivision drawn
uniformly from {1,2,3,4} (80-5120 triangles, radius 1 mm, +-15 % radial noise), B rotated by a random unit
quaternion and moved along a random direction so the nominal overlap depth is U(0, 0.1) r.  Outputs per
pair: loop count and, per contact, Sn, n, xc(0), Fn = k/2 |Sn| with k = 1e7 (FP64).  The meshes of a pair
are drawn from a seeded library of `--lib-per-level` meshes per subdivision (1024 meshes, 125 MB FP64),
built with build_mesh on the host.  Synthetic data: the reference publishes no dataset.

  --impl zdemx      (default) the CUDA path through libzdemx.so.  `value` times the call with inputs and
                    outputs resident on the GPU (CUDA events on the library's stream, L2 flushed between
                    steps); `e2e` times the same call with pinned host buffers (copies inside).
  --impl reference  the reference's own C++ per-pair code (oracle/_ref, src/main.cpp compiled unchanged)
                    on all host threads, over a bounded sample of the same workload per step.

Multi-GPU: pairs are independent, so each rank runs its own 65,536-pair batch (weak scaling, no
collective on the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "zedm-x_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "pair-contacts/s"
UNIT = "pairs/s"
L2_BYTES = 126 * 2**20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["zdemx", "reference"], default="zdemx")
    ap.add_argument("--pairs", type=int, default=65536)
    ap.add_argument("--lib-per-level", type=int, default=256)
    ap.add_argument("--plain-pairs", type=int, default=2048, help="pairs timed in the plain per-pair form")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--workload", choices=["sweep", "pour", "two", "adjoint", "rollout"], default="sweep",
                    help="sweep: the batched pair sweep (default); pour: 100k-particle DEM step in one CUDA graph; "
                         "two: the two-particle DEM run; adjoint: contact geometry + its adjoint; "
                         "rollout: gradients of a 2000-step, 1000-particle rollout, checkpointed vs stored")
    ap.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                    help="sweep on N GPUs: weak = every rank its own batch; strong = one batch cut into "
                         "cost-balanced shards, outputs gathered")
    ap.add_argument("--particles", type=int, default=100_000, help="pour: particle count")
    ap.add_argument("--preroll", type=int, default=1500, help="pour: untimed steps before warm-up (collisions start)")
    ap.add_argument("--rollout-steps", type=int, default=2000, help="rollout: steps of the rollout")
    ap.add_argument("--rollout-side", type=int, default=10, help="rollout: particles per lattice side")
    ap.add_argument("--extras", type=int, default=1,
                    help="sweep at N=1: 0 prints the headline line alone (no parity, comparisons, independent "
                         "meshes or DEM legs), e.g. under a profiler")
    ap.add_argument("--tune-pairs", type=int, default=16384,
                    help="sweep: pairs of the autotuner's calibration sample (0: keep the default launch parameters)")
    return ap.parse_args()


def workload(args, rank, builder="zdemx"):
    """The sweep's mesh library and pairs.  builder="reference" builds the meshes with the reference's own
    build_mesh (oracle/_ref), so that the reference arm loads nothing of this library."""
    from zdemx import synth
    from zdemx.contact import MeshLibrary

    rng = np.random.default_rng(args.seed)
    raw = []
    for s in (1, 2, 3, 4):
        raw.extend(list(synth.noised_icospheres(s, args.lib_per_level, 1e-3, 0.15, rng)))
    if builder == "reference":
        from oracle import Reference

        ref = Reference()
        built = [ref.build_mesh(t, True) for t in raw]
        outs = [o.reshape(-1, 9) for o, _ in built]
        props = np.asarray([p for _, p in built]).reshape(-1, 17)
        off = np.zeros(len(outs) + 1, np.int64)
        off[1:] = np.cumsum([len(o) for o in outs])
        lib = MeshLibrary(np.ascontiguousarray(np.concatenate(outs)), off, props[:, 5].copy(), props[:, 6].copy(), props)
    else:
        lib = MeshLibrary.build(raw)
    from zdemx.replicas import rank_seed

    prng = np.random.default_rng(rank_seed(args.seed, rank))
    lv = prng.integers(0, 4, size=(args.pairs, 2))
    idx = prng.integers(0, args.lib_per_level, size=(args.pairs, 2))
    pm = (lv * args.lib_per_level + idx).astype(np.int32)
    pp = synth.pair_poses(prng, args.pairs, 1e-3, 0.0, 0.1)
    return lib, pm, pp


def algorithmic_bytes(lib, pm):
    """Bytes one step must move at minimum: each pair's two FP64 triangle soups (72 B per triangle),
    its two poses (2 x 56 B) and ~100 B of outputs."""
    n = np.diff(lib.tri_off)
    return float(np.sum(72.0 * (n[pm[:, 0]] + n[pm[:, 1]])) + (112 + 100) * len(pm))


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, max clock, throttle reasons)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Per-pair counters of the two pair kernels from one ncu capture of the 4,096-pair sweep sample
# (profiles/pair_kernels_pairsweep4096.md gives the command and the raw figures).  They hold only for the
# kernel sources they were captured on: KERNEL_SOURCES hashed to `sources_sha256`.  When the sources
# differ, the figures are reported as stale (null) rather than applied to other code.
PROFILED = {
    "sources_sha256": "135042396fbbeaa48ad9bd45fb3c1ff9b10caa902436010dbe6b68c960a739cc",
    "k_segments": {"warp_inst_per_pair": 124798.8, "dram_bytes_per_pair": 280501.6},
    "k_rebuild": {"warp_inst_per_pair": 147357.0, "dram_bytes_per_pair": 17377.0},
}
KERNEL_SOURCES = ("zdx_pair.cu", "zdx_pair.cuh", "zdx_math.cuh", "zdx_npmath.cuh", "zdx_pyset.cuh",
                  "zdx_sortrep.cuh", "zdx_radix.cuh")


def kernel_sources_sha256():
    import hashlib

    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        with open(os.path.join(ROOT, "zedm-x_b200", "csrc", name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def profiled_current():
    """The profiled per-pair figures if they were captured on the kernel sources in this tree."""
    return PROFILED if PROFILED["sources_sha256"] == kernel_sources_sha256() else None


def issue_roofline(reb_s, seg_s, pairs, clocks):
    """Issue-rate roofline of the two pair kernels: profiled warp instructions per pair x pairs over the
    live kernel time, against 4 warp instructions per cycle per SM at the median SM clock of the run."""
    import torch

    prof = profiled_current()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
    peak = 4.0 * sms * mhz * 1e6
    out = {"unit": "warp-inst/s", "peak": peak, "peak_kind": f"4 per cycle per SM x {sms} SMs x {mhz:.0f} MHz"}
    if prof is None:
        out["stale"] = "kernel sources differ from the profiled ones: no instruction count for this code"
        return out
    out["profiled_sources_sha256"] = prof["sources_sha256"]
    for name, t in (("k_rebuild", reb_s), ("k_segments", seg_s)):
        inst = float(prof[name]["warp_inst_per_pair"]) * pairs
        out[name] = {"bound": "issue", "achieved": inst / t, "frac": inst / t / peak, "warp_inst_per_launch": inst}
    return out


def _ref_batch_lib():
    import ctypes as C

    from oracle import LIB_REF

    L = C.CDLL(LIB_REF)
    L.zdx_ref_pair_batch.restype = C.c_int64
    L.zdx_ref_pair_batch.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                        C.c_void_p]
    L.zdx_ref_pair_batch_rec.restype = C.c_int64
    L.zdx_ref_pair_batch_rec.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_int,
                                                            C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    return L


PARITY_GEOM_CAP = 64


def cpu_reference_rate(lib, pm, pp, nthreads, seconds, rng_seed=5, fixed=None, record=False):
    """Time the reference's own per-pair code (oracle/_ref) on a bounded random sample of the workload.
    With record, the sample's per-pair results (segments, components, raw loops, contacts and the
    accepted loops' Sn Gn xc0 nA area) come back too, for the parity check against the GPU."""
    L = _ref_batch_lib()
    rng = np.random.default_rng(rng_seed)
    order = rng.permutation(len(pm))
    rec = {}

    def run(sel):
        spm = np.ascontiguousarray(pm[sel])
        spp = np.ascontiguousarray(pp[sel])
        args = (lib.tris.ctypes.data, lib.tri_off.ctypes.data, lib.mean_edge.ctypes.data, lib.bbox_diag.ctypes.data,
                lib.n_mesh, len(sel), spm.ctypes.data, spp.ctypes.data, 1, nthreads)
        if record:
            rec["stats"] = np.zeros((len(sel), 4), np.int32)
            rec["geom"] = np.zeros((len(sel), PARITY_GEOM_CAP, 13))
            t0 = time.perf_counter()
            L.zdx_ref_pair_batch_rec(*args, rec["stats"].ctypes.data, PARITY_GEOM_CAP, rec["geom"].ctypes.data)
        else:
            t0 = time.perf_counter()
            L.zdx_ref_pair_batch(*args, None)
        return time.perf_counter() - t0

    if fixed is not None:
        dt = run(fixed)
        return len(fixed) / dt, len(fixed), dt, fixed, rec
    n = 32 * nthreads
    dt = run(order[:n])
    n = int(min(len(pm), max(n, n * seconds / max(dt, 1e-3))))
    sel = order[:n]
    dt = run(sel)
    return n / dt, n, dt, sel, rec


def parity_check(sel, rec, stats, coff, geom):
    """The GPU's results for the sampled pairs against the reference's: per pair the segment, component,
    raw-loop and contact counts, and every contact's Sn Gn xc0 nA area, bit for bit."""
    bad_pairs = 0
    fields = {"segments": 0, "components": 0, "raw_loops": 0, "contacts": 0, "contact_geometry": 0}
    checked_contacts = 0
    for k, p in enumerate(sel):
        r = rec["stats"][k]
        g = stats[p]
        nc = int(coff[p + 1] - coff[p])
        bad = False
        for f, a, b in (("segments", g[0], r[0]), ("components", g[1], r[1]), ("raw_loops", g[2], r[2]),
                        ("contacts", nc, r[3])):
            if int(a) != int(b):
                fields[f] += 1
                bad = True
        if not bad:
            m = min(nc, PARITY_GEOM_CAP)
            checked_contacts += m
            if m and not np.array_equal(geom[coff[p]:coff[p] + m, :13], rec["geom"][k, :m]):
                fields["contact_geometry"] += 1
                bad = True
        bad_pairs += bad
    return {"pairs": int(len(sel)), "contacts": int(checked_contacts), "mismatches": int(bad_pairs),
            "mismatches_by_field": fields, "against": "oracle/_ref (the reference's src/main.cpp, unchanged)",
            "compare": "bit for bit: segments, components, raw loops, contacts per pair; Sn Gn xc0 nA area per contact"}


def emit(d):
    print(json.dumps(d), flush=True)


_T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


def _sweep_buffers(dev, npairs, cap):
    import torch

    return {"ncontact": torch.zeros(npairs, dtype=torch.int32, device=dev),
            "contact_off": torch.zeros(npairs + 1, dtype=torch.int64, device=dev),
            "stats": torch.zeros(npairs, 4, dtype=torch.int32, device=dev),
            "geom": torch.zeros(cap, 20, dtype=torch.float64, device=dev),
            "info": torch.zeros(cap, 4, dtype=torch.int32, device=dev)}


def _device_steps(ctx, call, flush, steps):
    """Run `call` steps times (L2 flushed before each); the library's own CUDA-event times per call."""
    import torch

    ms, seg, reb = [], [], []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        tot = call()
        t = ctx.timings()
        ms.append(t["total"])
        seg.append(t["segments"])
        reb.append(t["rebuild"])
    return tot, ms, seg, reb


def run_reference_sweep(args, base_cfg):
    """The reference's own C++ per-pair code on all host threads, over a bounded sample per step."""
    from oracle import LIB_REF

    if not os.path.exists(LIB_REF):
        emit({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"})
        return
    lib, pm, pp = workload(args, 0, builder="reference")
    nthreads = os.cpu_count() or 1
    # size one step's sample to ~2 s of work on all threads
    rate, n, dt, sel, _ = cpu_reference_rate(lib, pm, pp, nthreads, 2.0)
    times = []
    for i in range(args.warmup + args.steps):
        r, _, d, _, _ = cpu_reference_rate(lib, pm, pp, nthreads, 0.0, fixed=sel)
        if i >= args.warmup:
            times.append(d)
    T = sum(times)
    value = len(sel) * len(times) / T
    sample = f"{len(sel)} random pairs of the {args.pairs}-pair workload per step"
    emit({"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * T / len(times),
          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
          "data": "synthetic (seeded noised icospheres)", "config": base_cfg,
          "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "reference", "sample": sample},
          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})


def main():
    args = parse()
    if args.workload == "pour":
        return run_pour(args)
    if args.workload == "two":
        return run_two(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "rollout":
        return run_rollout(args)
    if args.scaling == "strong" and args.impl != "reference":
        return run_strong(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3:
        args.warmup = 3

    workload_desc = (f"pair sweep: {args.pairs} pairs of noised icospheres (subdivision U{{1..4}}, 80-5120 tris, "
                     f"r 1 mm, +-15% noise), overlap depth U(0,0.1) r, k=1e7, split_contacts=1, FP64")
    base_cfg = {"workload": workload_desc, "pairs_per_gpu": args.pairs, "mesh_library": 4 * args.lib_per_level,
                "parallelism": f"replicas x{world} (independent pair batches)", "seed": args.seed}

    if args.impl == "reference":
        if rank == 0:
            run_reference_sweep(args, base_cfg)
        return

    import torch

    from zdemx import _lib

    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib, pm, pp = workload(args, rank)
    ctx = _lib.Context(local)

    # device-resident inputs and outputs
    d_tris = torch.from_numpy(lib.tris).to(dev)
    d_off = torch.from_numpy(lib.tri_off).to(dev)
    d_me = torch.from_numpy(lib.mean_edge).to(dev)
    d_bd = torch.from_numpy(lib.bbox_diag).to(dev)
    d_pm = torch.from_numpy(pm).to(dev)
    d_pp = torch.from_numpy(pp).to(dev)
    cap = 16 * args.pairs
    out = _sweep_buffers(dev, args.pairs, cap)
    meshes = {"tris": d_tris, "tri_off": d_off, "mean_edge": d_me, "bbox_diag": d_bd}
    pairs = {"mesh": d_pm, "pose": d_pp}
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def step():
        return _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7, split=True)

    # launch parameters from the autotuner, on a calibration sample of the same mix (another seed)
    tuning = {"best": ctx.tuning(), "calibration_pairs": 0}
    if args.tune_pairs > 0:
        from zdemx import autotune

        clib, cpm, cpp = autotune.sweep_sample(args.tune_pairs, args.seed + 1)
        cm, cp, co = autotune.device_batch(clib, cpm, cpp, dev)
        tres = autotune.tune(ctx, cm, cp, co, flush=flush)
        tuning = {"best": tres["best"], "calibration_pairs": tres["pairs"], "calibration_ms": tres["best_ms"],
                  "calibration_default_ms": tres["default_ms"], "trials": len(tres["trials"]),
                  "tuner": "zdemx.autotune (coordinate descent over " + ", ".join(autotune.GRID) + ")"}
        del cm, cp, co
        torch.cuda.empty_cache()

    for _ in range(args.warmup):
        totals = step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.timings()["launches"]
    wall0 = time.perf_counter()
    with ClockSampler(local) as clk:
        totals, step_ms, seg_ms, reb_ms = _device_steps(ctx, step, flush, args.steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    launches = ctx.timings()["launches"] - launches0
    T = sum(step_ms) / 1e3
    if world > 1:
        from zdemx.replicas import max_over_ranks

        T = max_over_ranks(T, dev)
        dist.barrier()
    value = world * args.pairs * args.steps / T
    # the last timed step's outputs, for the parity check and the comparisons below
    res = {k: v.cpu().numpy() for k, v in out.items() if k != "info"}

    # e2e: the same call with pinned host buffers, copies inside the timed region
    h = {k: torch.from_numpy(v).pin_memory() for k, v in
         {"tris": lib.tris, "off": lib.tri_off, "me": lib.mean_edge, "bd": lib.bbox_diag, "pm": pm, "pp": pp}.items()}
    hout = {k: v.cpu().pin_memory() for k, v in out.items()}
    hmeshes = {"tris": h["tris"], "tri_off": h["off"], "mean_edge": h["me"], "bbox_diag": h["bd"]}
    hpairs = {"mesh": h["pm"], "pose": h["pp"]}

    def e2e_step():
        return _lib.pair_contacts_device(ctx, hmeshes, hpairs, hout, k=1e7, split=True, mem=_lib.MEM_HOST)

    for _ in range(2):
        e2e_step()
    e2e_t = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tot_e = e2e_step()
        e2e_t.append(time.perf_counter() - t0)
    TE = sum(e2e_t)
    if world > 1:
        from zdemx.replicas import max_over_ranks

        TE = max_over_ranks(TE, dev)
    e2e_value = world * args.pairs * args.steps / TE
    h2d = sum(int(v.numel() * v.element_size()) for v in h.values())
    nct = int(tot_e[0])
    d2h = args.pairs * (4 + 8 + 16) + 8 + nct * (160 + 16)
    del h, hout, hmeshes, hpairs

    if world > 1:
        # the scaling run reports the headline numbers only; the comparisons below run at N=1
        dist.barrier()
        if rank == 0:
            emit(_sweep_line(args, world, value, T, totals, launches, clk, wall, e2e_value, h2d, d2h, lib, pm,
                             seg_ms, reb_ms, step_ms, base_cfg, extras={"tuning": tuning}))
        dist.barrier()
        dist.destroy_process_group()
        return

    log(f"sweep: {value:.4g} pairs/s device, {e2e_value:.4g} e2e")
    extras = {"tuning": tuning}
    if not args.extras:
        emit(_sweep_line(args, world, value, T, totals, launches, clk, wall, e2e_value, h2d, d2h, lib, pm, seg_ms,
                         reb_ms, step_ms, base_cfg, extras))
        return
    # parity of this step's output with the reference's own code on the CPU baseline's sample
    rate, n_cpu, dt_cpu, sel, rec = cpu_reference_rate(lib, pm, pp, 1, args.cpu_seconds, record=True)
    extras["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
                              "sample": f"{n_cpu} random pairs of the workload through oracle/_ref, {dt_cpu:.1f} s"}
    extras["parity"] = parity_check(sel, rec, res["stats"], res["contact_off"], res["geom"])
    log(f"parity: {extras['parity']['pairs']} pairs, {extras['parity']['mismatches']} mismatches")
    extras.update(sweep_comparisons(args, ctx, dev, meshes, pairs, out, res, flush, step_ms))
    extras["strong_shards"] = shard_balance(args, ctx, dev, meshes, pairs, flush, statistics.mean(step_ms))
    log("strong shards: " + ", ".join(f"{k} {v['balance_mean_over_max']:.3f}" for k, v in extras["strong_shards"].items()
                                      if isinstance(v, dict)))
    del d_tris
    log("comparisons done")
    extras["independent_meshes"] = sweep_independent(args, ctx, dev, flush)
    log("independent meshes done")
    torch.cuda.empty_cache()
    # 100 timed steps (about 0.3 s): long enough for the clock sampler to see the region
    extras["dem"] = {"pour": measure_pour(args, ctx, steps=max(args.steps, 100), cpu=False)}
    log("pour done")
    extras["dem"]["two_particles"] = measure_two(args, ctx, reps=3, extras=False)
    log("two particles done")
    emit(_sweep_line(args, world, value, T, totals, launches, clk, wall, e2e_value, h2d, d2h, lib, pm, seg_ms,
                     reb_ms, step_ms, base_cfg, extras))


def _sweep_line(args, world, value, T, totals, launches, clk, wall, e2e_value, h2d, d2h, lib, pm, seg_ms, reb_ms,
                step_ms, base_cfg, extras):
    # roofline of the dominant kernel (the rebuild): it reads each segment of the arena once (6 doubles)
    # and writes each contact once (20 doubles + 4 ints); the triangle stage's line follows it
    peak, peak_kind = measured_peaks()
    reb_s = statistics.mean(reb_ms) / 1e3
    reb_bytes = 48.0 * int(totals[1]) + 176.0 * int(totals[0])
    abytes = algorithmic_bytes(lib, pm)
    seg_s = statistics.mean(seg_ms) / 1e3
    achieved = abytes / seg_s / 1e9
    prof = profiled_current()
    traffic = prof["k_segments"]["dram_bytes_per_pair"] * args.pairs if prof else None
    reb_traffic = prof["k_rebuild"]["dram_bytes_per_pair"] * args.pairs if prof else None
    cfg = dict(base_cfg)
    cfg.update({"l2": "flushed (256 MB write) before every timed step", "inputs": "device-resident for value",
                "contacts_per_step": int(totals[0]), "segments_per_step": int(totals[1]),
                "tri_aabb_checks_per_step": int(totals[2])})
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic (seeded noised icospheres, {4 * args.lib_per_level}-mesh library)", "config": cfg,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": reb_bytes / reb_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": reb_bytes / reb_s / 1e9 / peak, "traffic": reb_traffic, "kernel": "k_rebuild",
                         "peak_kind": f"{peak_kind} hbm_gbs", "algorithmic_bytes_per_launch": reb_bytes,
                         "kernel_ms": 1e3 * reb_s,
                         "note": "latency bound (serial per-pair topology in the reference's order); see profiles/"},
            "roofline_k_segments": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                    "frac": achieved / peak, "traffic": traffic, "kernel": "k_segments",
                                    "algorithmic_bytes_per_launch": abytes, "kernel_ms": 1e3 * seg_s,
                                    "note": "FP64 compare/ALU issue and scratch latency bound; see profiles/"},
            "roofline_issue": issue_roofline(reb_s, seg_s, args.pairs, clk.summary()),
            "stages_ms": {"triangle_tests": statistics.mean(seg_ms), "rebuild": statistics.mean(reb_ms),
                          "whole_call": statistics.mean(step_ms)},
            "clocks": clk.summary(), "wall_s_timed": wall}
    line.update(extras)
    return line


def sweep_comparisons(args, ctx, dev, meshes, pairs, out, res, flush, step_ms):
    """The batched call against its plain forms and the no-allocation entry, each on the same pairs and
    checked to give the same results."""
    import torch

    from zdemx import _lib

    out_ = {}
    batched_ms = statistics.mean(step_ms)
    # plain per-stage form on the whole batch: one launch per stage, no work queue, no cost order, no culls
    ps = _sweep_buffers(dev, args.pairs, out["geom"].shape[0])
    _lib.pair_contacts_device(ctx, meshes, pairs, ps, k=1e7, split=True, sched=_lib.SCHED_PER_STAGE)
    _, ps_ms, ps_seg, ps_reb = _device_steps(
        ctx, lambda: _lib.pair_contacts_device(ctx, meshes, pairs, ps, k=1e7, split=True, sched=_lib.SCHED_PER_STAGE),
        flush, 2)
    same = all(np.array_equal(ps[k].cpu().numpy(), res[k]) for k in ("ncontact", "contact_off", "stats")) and \
        np.array_equal(ps["geom"].cpu().numpy()[: int(res["contact_off"][-1])], res["geom"][: int(res["contact_off"][-1])])
    out_["plain_per_stage"] = {
        "value": args.pairs / (statistics.mean(ps_ms) / 1e3), "unit": UNIT, "pairs": args.pairs,
        "ms_per_step": statistics.mean(ps_ms), "stages_ms": {"triangle_tests": statistics.mean(ps_seg),
                                                             "rebuild": statistics.mean(ps_reb)},
        "speedup_batched_vs_plain_per_stage": statistics.mean(ps_ms) / batched_ms, "results_identical": bool(same),
        "form": "one launch per stage over the batch; pairs in a fixed grid-stride order (no work queue, no cost "
                "order); every nA x nB triangle pair AABB-tested (no certificate, cube, slab or hierarchical culls)"}
    del ps
    # plain per-pair form on a subset (one launch per stage per pair)
    plain_n = min(args.plain_pairs, args.pairs)
    sub = {"mesh": pairs["mesh"][:plain_n].contiguous(), "pose": pairs["pose"][:plain_n].contiguous()}
    sub_out = _sweep_buffers(dev, plain_n, 16 * plain_n)
    _lib.pair_contacts_device(ctx, meshes, sub, sub_out, k=1e7, split=True, sched=_lib.SCHED_PLAIN)
    torch.cuda.synchronize()
    _lib.pair_contacts_device(ctx, meshes, sub, sub_out, k=1e7, split=True, sched=_lib.SCHED_PLAIN)
    plain_ms = ctx.timings()["total"]
    _lib.pair_contacts_device(ctx, meshes, sub, sub_out, k=1e7, split=True)
    batched_sub_ms = ctx.timings()["total"]
    plain_value = plain_n / (plain_ms / 1e3)
    out_["plain"] = {"value": plain_value, "unit": UNIT, "pairs": plain_n,
                     "batched_same_pairs": plain_n / (batched_sub_ms / 1e3),
                     "speedup_batched_vs_plain": (plain_n / (batched_sub_ms / 1e3)) / plain_value,
                     "form": "one launch per stage per pair"}
    # the no-allocation entry against the allocating call: 384 pairs of the sweep's mix (about 40,000
    # segments of its 65,536), over at most 65,536 triangles (16, 8, 16 and 8 meshes of subdivision 1 to 4)
    nn = min(384, args.pairs)
    per_level = (16, 8, 16, 8)
    tri_off = meshes["tri_off"].cpu().numpy()
    ids = [lv * args.lib_per_level + i for lv in range(4) for i in range(min(per_level[lv], args.lib_per_level))]
    sub_tris = torch.cat([meshes["tris"][int(tri_off[m]):int(tri_off[m + 1])] for m in ids])
    sub_off = np.zeros(len(ids) + 1, np.int64)
    sub_off[1:] = np.cumsum([tri_off[m + 1] - tri_off[m] for m in ids])
    first = np.cumsum([0] + [min(c, args.lib_per_level) for c in per_level])
    srng = np.random.default_rng([args.seed, 0x4E])
    slv = srng.integers(0, 4, size=(nn, 2))
    spm = (first[slv] + srng.integers(0, 1 << 30, size=(nn, 2)) % np.minimum(per_level, args.lib_per_level)[slv])
    idx_t = torch.as_tensor(np.asarray(ids), device=dev)
    nmesh = {"tris": sub_tris.contiguous(), "tri_off": torch.from_numpy(sub_off).to(dev),
             "mean_edge": meshes["mean_edge"][idx_t].contiguous(), "bbox_diag": meshes["bbox_diag"][idx_t].contiguous()}
    sub = {"mesh": torch.from_numpy(spm.astype(np.int32)).to(dev), "pose": pairs["pose"][:nn].contiguous()}
    a_out = _sweep_buffers(dev, nn, 16384)
    b_out = _sweep_buffers(dev, nn, 16384)
    _lib.pair_contacts_device(ctx, nmesh, sub, a_out, k=1e7, split=True)
    _, a_ms, _, _ = _device_steps(ctx, lambda: _lib.pair_contacts_device(ctx, nmesh, sub, a_out, k=1e7, split=True),
                                  flush, 3)
    _lib.pair_contacts_noalloc(ctx, nmesh, sub, b_out, k=1e7, split=True)
    _, b_ms, _, _ = _device_steps(ctx, lambda: _lib.pair_contacts_noalloc(ctx, nmesh, sub, b_out, k=1e7, split=True),
                                  flush, 3)
    n_c = int(a_out["contact_off"][-1])
    same = all(torch.equal(a_out[k], b_out[k]) for k in ("ncontact", "contact_off", "stats")) and \
        torch.equal(a_out["geom"][:n_c], b_out["geom"][:n_c])
    out_["noalloc"] = {"value": nn / (statistics.mean(b_ms) / 1e3), "unit": UNIT, "pairs": nn,
                       "allocating_call_same_pairs": nn / (statistics.mean(a_ms) / 1e3),
                       "results_identical": bool(same),
                       "meshes": len(ids), "triangles": int(sub_off[-1]),
                       "note": "zdx_pair_contacts_noalloc: scratch in the library's fixed 16 MiB device array"}
    return out_


def shard_balance(args, ctx, dev, meshes, pairs, flush, batch_ms):
    """Strong-scaling shards of the sweep batch, run one after another on this GPU: per world size and
    shard mode, every shard's device time as its own batch (no rank waits on another, so one GPU times
    them all).  The slowest shard bounds a strong-scaling step; mean / max is that step's balance."""
    import torch

    from zdemx import _lib
    from zdemx.replicas import strong_shards

    tri_off = meshes["tri_off"].cpu().numpy()
    pm = pairs["mesh"].cpu().numpy()
    res = {}
    for world in (2, 4, 8):
        for mode in ("ranges", "dealt"):
            shard_ms = []
            for idx in strong_shards(tri_off, pm, world, mode=mode):
                it = torch.from_numpy(idx).to(dev)
                sub = {"mesh": pairs["mesh"][it].contiguous(), "pose": pairs["pose"][it].contiguous()}
                so = _sweep_buffers(dev, len(idx), 16 * max(len(idx), 1))
                call = lambda: _lib.pair_contacts_device(ctx, meshes, sub, so, k=1e7, split=True)
                call()
                _, ms, _, _ = _device_steps(ctx, call, flush, 2)
                shard_ms.append(statistics.mean(ms))
                del so
            mx, mean = max(shard_ms), statistics.mean(shard_ms)
            res[f"{mode}_x{world}"] = {"shard_ms": [round(x, 3) for x in shard_ms], "max_ms": mx,
                                       "balance_mean_over_max": mean / mx, "speedup_bound": batch_ms / mx}
    res["note"] = ("shards timed one after another on one GPU; speedup_bound = the whole batch's time over the "
                   "slowest shard's (the all-gather not included)")
    return res


def sweep_independent(args, ctx, dev, flush):
    """The sweep with every pair's two meshes its own (2 x pairs meshes), device-timed and end to end."""
    import torch

    from zdemx import _lib
    from zdemx.workloads import independent_pair_library, independent_pair_sizes
    from zdemx import synth

    t0 = time.perf_counter()
    _, off, _ = independent_pair_sizes(args.pairs, args.seed)
    h_tris = torch.empty((int(off[-1]), 9), dtype=torch.float64, pin_memory=True)
    lib, pm = independent_pair_library(args.pairs, args.seed, out_tris=h_tris.numpy())
    pp = synth.pair_poses(np.random.default_rng([args.seed, 0x1E]), args.pairs, 1e-3, 0.0, 0.1)
    build_s = time.perf_counter() - t0
    h = {"tris": h_tris, "tri_off": torch.from_numpy(lib.tri_off).pin_memory(),
         "mean_edge": torch.from_numpy(lib.mean_edge).pin_memory(),
         "bbox_diag": torch.from_numpy(lib.bbox_diag).pin_memory()}
    hp = {"mesh": torch.from_numpy(pm).pin_memory(), "pose": torch.from_numpy(pp).pin_memory()}
    d = {k: v.to(dev) for k, v in h.items()}
    dp = {k: v.to(dev) for k, v in hp.items()}
    cap = 16 * args.pairs
    out = _sweep_buffers(dev, args.pairs, cap)
    call = lambda: _lib.pair_contacts_device(ctx, d, dp, out, k=1e7, split=True)
    call()
    tot, ms, seg, reb = _device_steps(ctx, call, flush, args.steps)
    del d, dp
    torch.cuda.empty_cache()
    hout = {k: v.cpu().pin_memory() for k, v in out.items()}
    del out
    torch.cuda.empty_cache()
    call_h = lambda: _lib.pair_contacts_device(ctx, h, hp, hout, k=1e7, split=True, mem=_lib.MEM_HOST)
    call_h()
    e2e = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        te = call_h()
        e2e.append(time.perf_counter() - t1)
    h2d = sum(int(v.numel() * v.element_size()) for v in list(h.values()) + list(hp.values()))
    d2h = args.pairs * (4 + 8 + 16) + 8 + int(te[0]) * (160 + 16)
    return {"value": args.pairs * args.steps / (sum(ms) / 1e3), "unit": UNIT, "meshes": int(lib.n_mesh),
            "triangle_bytes": int(lib.tris.nbytes), "contacts_per_step": int(tot[0]),
            "stages_ms": {"triangle_tests": statistics.mean(seg), "rebuild": statistics.mean(reb),
                          "whole_call": statistics.mean(ms)},
            "e2e": {"value": args.pairs * args.steps / sum(e2e), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "host_build_s": build_s,
            "workload": "the same sweep with both meshes of every pair independent seeded noised icospheres "
                        "(subdivision U{1..4}), built by zdx_mesh_build on all host threads"}


def run_strong(args):
    """One sweep batch spread over the ranks: each rank takes a cost-balanced shard of the cost-ordered
    pairs, and one all-gather brings every rank's contacts (geometry and per-pair counts) to all ranks.
    Timed per step from before the pair call to after the gather, max over ranks."""
    import datetime

    import torch
    import torch.distributed as dist

    from zdemx import _lib
    from zdemx.replicas import gather_counts, gather_rows, max_over_ranks, strong_shards

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    args.warmup = max(args.warmup, 3)
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib, pm, pp = workload(args, 0)  # the same batch on every rank
    mine = strong_shards(lib.tri_off, pm, world)[rank]
    spm, spp = np.ascontiguousarray(pm[mine]), np.ascontiguousarray(pp[mine])
    ctx = _lib.Context(local)
    n = len(mine)
    cap = 16 * max(n, 1)
    meshes = {"tris": torch.from_numpy(lib.tris).to(dev), "tri_off": torch.from_numpy(lib.tri_off).to(dev),
              "mean_edge": torch.from_numpy(lib.mean_edge).to(dev), "bbox_diag": torch.from_numpy(lib.bbox_diag).to(dev)}
    pairs = {"mesh": torch.from_numpy(spm).to(dev), "pose": torch.from_numpy(spp).to(dev)}
    out = {"ncontact": torch.zeros(n, dtype=torch.int32, device=dev),
           "contact_off": torch.zeros(n + 1, dtype=torch.int64, device=dev),
           "stats": torch.zeros(n, 4, dtype=torch.int32, device=dev),
           "geom": torch.zeros(cap, 20, dtype=torch.float64, device=dev),
           "info": torch.zeros(cap, 4, dtype=torch.int32, device=dev)}
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    stream = _lib_stream(ctx)

    def step():
        tot = _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7, split=True)
        with torch.cuda.stream(stream):
            g = gather_rows(out["geom"][: int(tot[0])])
            c = gather_rows(out["ncontact"])
        return tot, g, c

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = []
    launches0 = ctx.timings()["launches"]
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            tot, g, c = step()
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
    launches = ctx.timings()["launches"] - launches0
    T = max_over_ranks(sum(ms) / 1e3, dev)
    contacts = sum(int(x.shape[0]) for x in g)
    pairs_seen = sum(int(x.shape[0]) for x in c)
    shard_sizes = gather_counts(n, dev)
    if world > 1:
        dist.barrier()
    if rank == 0:
        emit({"metric": METRIC, "value": args.pairs * args.steps / T, "unit": UNIT, "n_gpus": world,
              "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps,
              "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
              "data": "synthetic (seeded noised icospheres, 1024-mesh library)",
              "config": {"workload": f"pair sweep: {args.pairs} pairs (one batch over {world} ranks), "
                                     "the cost-ordered pairs dealt to the ranks, one all-gather of the contacts",
                         "pairs_total": args.pairs, "shard_sizes": shard_sizes, "seed": args.seed,
                         "parallelism": f"pair shards x{world}", "l2": "flushed (256 MB write) before every timed step"},
              "gathered": {"contacts": contacts, "pairs": pairs_seen},
              "gpu_launches": int(launches), "clocks": clk.summary()})
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------- DEM legs
def _ref_exe():
    return os.path.join(ROOT, "oracle", "_ref", "zdem_cpu")


def _ref_step_ms(cfg_path, steps, timeout=3600):
    """zdem_cpu (the reference program, oracle/_ref) on a copy of the config with `steps` steps and an
    output every step: per step its own std::chrono step time minus its output time (step_ms - output_ms of
    its log line).  Each output path is made a directory, so the reference's writers fail to open it and
    return at once (src/main.cpp:1716-1719, 1846-1849): a 100k-particle VTK is gigabytes of text."""
    import re
    import tempfile

    text = open(cfg_path).read()
    out = tempfile.mkdtemp(prefix="zdx_ref_")
    prefix = re.search(r"(?m)^vtk_prefix = (.*)$", text).group(1).strip()
    text = re.sub(r"(?m)^steps = .*$", f"steps = {steps}", text)
    text = re.sub(r"(?m)^output_interval = .*$", "output_interval = 1", text)
    text = re.sub(r"(?m)^output_dir = .*$", f"output_dir = {out}", text)
    for k in range(steps):
        for ext in (".vtk", ".txt"):
            os.makedirs(os.path.join(out, f"{prefix}_{k:06d}{ext}"))
    c = os.path.join(out, "ref.cfg")
    open(c, "w").write(text)
    p = subprocess.run([_ref_exe(), "--config", c], capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(p.stderr[-500:])
    ms = [float(a) - float(b) for a, b in re.findall(r"step_ms=([0-9.]+).*?output_ms=([0-9.]+)", p.stdout)]
    return ms, p.stdout


def _ref_run_wall(cfg_path, steps, dt=None, every=None, hiprec=False, timeout=3600, exe=None):
    """The reference program (or `exe`, a command line taking --config) on a copy of the config: wall
    seconds of the whole run and its output dir."""
    import re
    import tempfile

    text = open(cfg_path).read()
    out = tempfile.mkdtemp(prefix="zdx_ref_")
    text = re.sub(r"(?m)^steps = .*$", f"steps = {steps}", text)
    if dt is not None:
        text = re.sub(r"(?m)^dt = .*$", f"dt = {dt!r}", text)
    text = re.sub(r"(?m)^output_interval = .*$", f"output_interval = {every or (1 << 30)}", text)
    text = re.sub(r"(?m)^output_dir = .*$", f"output_dir = {out}", text)
    c = os.path.join(out, "ref.cfg")
    open(c, "w").write(text)
    if hiprec:
        from oracle import LIB_REF_HIPREC

        code = ("import sys; sys.path.insert(0, %r); from oracle import Reference; import ctypes; "
                "r = Reference(%r); rc = r.main(['--config', %r]); ctypes.CDLL(None).fflush(None); sys.exit(rc)") % (
            os.path.join(ROOT, "oracle"), LIB_REF_HIPREC, c)
        cmd = [sys.executable, "-c", code]
    else:
        cmd = (list(exe) if exe else [_ref_exe()]) + ["--config", c]
    t0 = time.perf_counter()
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(p.stderr[-500:])
    return wall, out


def _state_txt(path):
    rows, cur = [], {}
    for line in open(path):
        line = line.strip()
        if line == "particle":
            cur = {}
        elif line == "end_particle":
            rows.append(np.r_[cur["pos"], cur["quat"], cur["vel"], cur["omega"]])
        elif "=" in line:
            k, v = [x.strip() for x in line.split("=", 1)]
            if k in ("pos", "quat", "vel", "omega"):
                cur[k] = np.array([float(x) for x in v.split()])
    return np.asarray(rows)


def _mean_particle_tris(cfg_path):
    """Mean triangle count over the particles of a config (binary STL headers)."""
    import re
    from collections import Counter

    paths = Counter(re.findall(r"(?ms)^particle\nstl = (.*?)$", open(cfg_path).read()))
    total = 0
    for p, c in paths.items():
        with open(p, "rb") as f:
            f.seek(80)
            total += c * int(np.frombuffer(f.read(4), "<u4")[0])
    return total / max(sum(paths.values()), 1)


def _lib_stream(ctx):
    import torch

    return torch.cuda.ExternalStream(ctx.stream_ptr())


def _timed_steps(sc, stream, flush, n, graph):
    """Device time of n single steps (CUDA events on the library stream, L2 flushed before each)."""
    import torch

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    for k in range(n):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[k][0].record(stream)
        (sc.step_graph if graph else sc.step)(1)
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def measure_pour(args, ctx, steps, cpu=True):
    """The 100,000-particle pour (five templates, closed box, gravity), the whole step as one CUDA graph:
    `steps` timed steps after the pre-roll.  Returns the measurement (steps/s, e2e, roofline, clocks)."""
    import tempfile

    import torch

    from zdemx.dem import Scene
    from zdemx.workloads import pour_scene

    d = tempfile.mkdtemp(prefix="zdx_pour_")
    cfg_path = pour_scene(d, n=args.particles, seed=args.seed)
    desc = (f"pour: {args.particles} particles (3 ellipsoid hulls of 64 points + icospheres s=2,3; circumradius 1 mm), "
            "jittered lattice in a closed 12-triangle box (60 x 60 mm floor), g=-9.81 z, dt=2e-6, "
            "velocities N(0, 0.05 m/s), zdem force law, split_contacts=1, FP64, graph step's clearance cache on")
    dev = torch.device("cuda", 0)
    t0 = time.perf_counter()
    sc = Scene(cfg_path, ctx)
    load_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    sc.step_graph(args.preroll)
    preroll_s = time.perf_counter() - t0
    sc.step_graph(max(args.warmup, 3))
    stream = _lib_stream(ctx)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    launches0 = ctx.timings()["launches"]
    infos, caches = [], []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(0) as clk:
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                ev[k][0].record(stream)
            sc.step_graph(1)
            with torch.cuda.stream(stream):
                ev[k][1].record(stream)
            infos.append(sc.info())
            caches.append(sc.graph_cache())
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    launches = ctx.timings()["launches"] - launches0
    T = sum(step_ms) / 1e3
    value = steps / T
    # the same steps without the graph (one launch per kernel, the host reads the counts)
    plain_ms = _timed_steps(sc, stream, flush, 3, graph=False)
    # e2e: the graph step plus the whole state brought back to the host every step
    e2e = []
    host = sc.state()  # the caller's buffers, filled again every step
    for k in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        sc.step_graph(1)
        sc.state(out=host)
        e2e.append(time.perf_counter() - t1)
    np_ = sc.n
    d2h = np_ * (16 * 8 + 3 * 8 * 2 + 4)
    peak, peak_kind = measured_peaks()
    # algorithmic bytes of a step: particle state read + written, material read, every candidate pair's
    # two FP64 triangle soups (72 B per triangle) read once, except for the pairs skipped on the clearance
    # cache, which read and write their 128-B entry instead
    pairs = int(np.mean([i["pairs"] for i in infos]))
    skipped = int(np.mean([c["skipped"] for c in caches]))
    mean_tris = _mean_particle_tris(cfg_path)
    abytes = np_ * (2 * 128 + 136) + (pairs - skipped) * 72.0 * 2 * mean_tris + skipped * 256.0
    achieved = abytes / (T / steps) / 1e9
    cpu_line = {"value": None, "unit": "steps/s", "cores": 1, "kind": "reference",
                "sample": "not run here (one zdem_cpu step of this scene takes about a minute): --workload pour"}
    if cpu:
        try:
            if args.cpu_seconds <= 0:
                raise RuntimeError("skipped (--cpu-seconds 0)")
            ms_ref, _ = _ref_step_ms(cfg_path, 1)
            cpu_line = {"value": 1e3 / ms_ref[0], "unit": "steps/s", "cores": 1, "kind": "reference",
                        "sample": f"step 0 of zdem_cpu on the same config ({ms_ref[0] / 1e3:.1f} s, its step_ms - output_ms)"}
        except Exception as e:
            cpu_line["sample"] = f"unavailable: {e}"
    last = infos[-1]
    return {"metric": "DEM steps/s", "value": value, "unit": "steps/s", "steps": steps, "ms_per_step": 1e3 * T / steps,
            "config": {"workload": desc, "particles": np_, "preroll_steps": args.preroll, "mean_tris": mean_tris,
                       "l2": "flushed (256 MB write) before every timed step", "graph": "whole step, one CUDA graph",
                       "pairs_per_step": pairs, "contacts_last_step": last["contacts"],
                       "clearance_cache": {"pairs_skipped_per_step": skipped, "entries_last_step": caches[-1]["entries"]},
                       "wall_contacts_last_step": last["wall_contacts"], "segments_last_step": last["segments"],
                       "load_s": load_s, "preroll_s": preroll_s},
            "e2e": {"value": steps / sum(e2e), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "whole step (graph)", "peak_kind": f"{peak_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": abytes},
            "plain_step_ms": plain_ms, "cpu_baseline": cpu_line, "clocks": clk.summary()}


def run_pour(args):
    """A 100,000-particle pour (five templates, closed box, gravity), the whole step as one CUDA graph."""
    import tempfile

    import torch

    from zdemx import _lib
    from zdemx.workloads import pour_scene

    if int(os.environ.get("RANK", "0")) != 0:
        return
    if args.impl == "reference":
        if not os.path.exists(_ref_exe()):
            emit({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"})
            return
        d = tempfile.mkdtemp(prefix="zdx_pour_")
        cfg_path = pour_scene(d, n=args.particles, seed=args.seed)
        ms, _ = _ref_step_ms(cfg_path, max(1, min(args.steps, 2)))
        T = sum(ms) / 1e3
        value = len(ms) / T
        emit({"impl": "reference", "metric": "DEM steps/s", "value": value, "unit": "steps/s", "n_gpus": 1,
              "steps": len(ms), "warmup": 0, "ms_per_step": 1e3 * T / len(ms), "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded pour scene)",
              "config": {"workload": f"pour: {args.particles} particles (see --impl zdemx)"},
              "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "reference",
                               "sample": f"the first {len(ms)} steps of zdem_cpu on the same config (its step_ms)"},
              "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctx = _lib.Context(0)
    m = measure_pour(args, ctx, args.steps, cpu=True)
    line = {"metric": m.pop("metric"), "value": m.pop("value"), "unit": m.pop("unit"), "n_gpus": 1,
            "steps": m.pop("steps"), "warmup": max(args.warmup, 3), "ms_per_step": m.pop("ms_per_step"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded pour scene)"}
    line.update(m)
    emit(line)


def measure_two(args, ctx, reps, extras=True):
    """Two 320-triangle noised icospheres colliding (2000 steps, dt 1e-6): steps/s of whole runs through
    the graph step, the trajectory against the reference program and the run end to end.  With extras,
    also the plain step, every step through the full step, the whole program with outputs and the same
    pair held in contact (dt 1e-15)."""
    import tempfile

    import torch

    from zdemx.dem import Scene
    from zdemx.workloads import two_particle_scene

    d = tempfile.mkdtemp(prefix="zdx_two_")
    steps_run = 2000
    cfg_path = two_particle_scene(d, seed=args.seed, steps=steps_run)
    desc = ("two particles: 320-triangle noised icospheres (r 1 mm, +-15%), 1.9 mm apart, +-0.05 m/s, dt=1e-6, "
            "2000 steps, split_contacts=1, zdem force law, FP64")
    dev = torch.device("cuda", 0)
    stream = _lib_stream(ctx)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def whole_runs(graph, free_flight=True):
        """Device time of `reps` whole 2000-step runs from the initial state (L2 flushed before each).  One
        untimed run first (it captures the graph); the pair ends every run apart, with no history, so each
        run restarts from the initial state alone and must end in the same state."""
        s = Scene(cfg_path, ctx)
        s.set_free_flight(free_flight)
        st0 = s.state()[0].copy()
        adv = s.step_graph if graph else s.step
        adv(steps_run)
        assert s.info()["history"] == 0 and s.info()["wall_history"] == 0
        fin = s.state()[0].copy()
        ms, same = [], True
        launches0 = ctx.timings()["launches"]
        for _ in range(reps):
            s.set_state(st0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.zero_()
                e0.record(stream)
            adv(steps_run)
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            same = same and bool(np.array_equal(s.state()[0], fin))
        return ms, same, (ctx.timings()["launches"] - launches0) // reps, s, st0, fin

    with ClockSampler(0) as clk:
        g_ms, g_same, launches, sc, st0, fin = whole_runs(graph=True)
    final = fin[:, :13]
    # end to end through the public API: state in from host memory, the run, state back out (a context
    # holds one scene: load it again, with free flight, and run it once untimed)
    sc = Scene(cfg_path, ctx)
    sc.step_graph(steps_run)
    e2e = []
    for _ in range(reps):
        t1 = time.perf_counter()
        sc.set_state(st0)
        sc.step_graph(steps_run)
        sc.state()
        e2e.append(time.perf_counter() - t1)
    try:
        _, out = _ref_run_wall(cfg_path, steps_run, every=steps_run - 1, hiprec=True)
        ref = _state_txt(os.path.join(out, f"p_{steps_run - 1:06d}.txt"))
        traj = {}
        for name, cols in (("pos", slice(0, 3)), ("quat", slice(3, 7)), ("vel", slice(7, 10)), ("omega", slice(10, 13))):
            scale = max(np.max(np.abs(ref[:, cols])), 1e-300)
            traj[name] = float(np.max(np.abs(final[:, cols] - ref[:, cols])) / scale)
    except Exception as e:
        traj = {"unavailable": str(e)[:200]}
    cpu = {"value": None, "unit": "steps/s", "cores": 1, "kind": "reference", "sample": "unavailable"}
    try:
        wall, _ = _ref_run_wall(cfg_path, steps_run)
        cpu = {"value": steps_run / wall, "unit": "steps/s", "cores": 1, "kind": "reference",
               "sample": f"the whole {steps_run}-step zdem_cpu run (wall clock, 1 thread)"}
    except Exception as e:
        cpu["sample"] = f"unavailable: {e}"
    T = sum(g_ms) / 1e3
    n_all = steps_run * reps
    res = {"metric": "DEM steps/s", "value": n_all / T, "unit": "steps/s", "steps": n_all, "warmup": steps_run,
           "ms_per_step": 1e3 * T / n_all,
           "config": {"workload": desc, "timed": f"{reps} whole {steps_run}-step runs from the initial state",
                      "l2": "flushed (256 MB write) before every timed run",
                      "graph": "candidate-free steps in one single-block kernel, the others one CUDA graph each"},
           "e2e": {"value": n_all / sum(e2e), "unit": "steps/s",
                   "h2d_bytes_per_step": 2 * 16 * 8 / steps_run, "d2h_bytes_per_step": 2 * (16 * 8 + 6 * 8 + 4) / steps_run},
           "gpu_launches": int(launches) * reps, "repeat_runs_identical": g_same,
           "trajectory_rel_err_vs_reference": traj, "cpu_baseline": cpu, "clocks": clk.summary()}
    if not extras:
        return res
    p_ms, p_same, _, sp, _, pfin = whole_runs(graph=False)
    nf_ms, _, nf_launches, _, _, nffin = whole_runs(graph=True, free_flight=False)
    res["repeat_runs_identical"] = g_same and p_same
    res["plain"] = {"value": n_all / (sum(p_ms) / 1e3), "unit": "steps/s", "bit_identical_to_graph": bool(np.array_equal(pfin, fin))}
    res["every_step_full"] = {"value": n_all / (sum(nf_ms) / 1e3), "unit": "steps/s", "gpu_launches": int(nf_launches) * reps,
                              "bit_identical_to_free_flight": bool(np.array_equal(nffin, fin))}
    # sustained contact: the same pair with dt = 1e-15 (it stays in contact every step)
    sus_path = os.path.join(d, "sustained.txt")
    open(sus_path, "w").write(open(cfg_path).read().replace("dt = 1e-06", "dt = 1e-15"))
    ss = Scene(sus_path, ctx)
    ss.step_graph(10)
    s_ms = _timed_steps(ss, stream, flush, 500, graph=True)
    sus_contacts = ss.info()["contacts"]
    # the whole program at the reference's default output_interval = 1: a particle VTK and a state txt
    # every step.  zdem_gpu queues each output behind a device snapshot and writes it on writer threads.
    prog = {"steps": steps_run, "output_interval": 1, "unit": "steps/s"}
    try:
        gexe = [os.path.join(ROOT, "zedm-x_b200", "bin", "zdem_gpu"), "--graph"]
        gw, gout = _ref_run_wall(cfg_path, steps_run, every=1, exe=gexe)
        rw, rout = _ref_run_wall(cfg_path, steps_run, every=1)
        same_files = all(open(os.path.join(gout, f"p_{k:06d}.vtk")).read() ==
                         open(os.path.join(rout, f"p_{k:06d}.vtk")).read() for k in (0, steps_run // 2, steps_run - 1))
        prog.update({"value": steps_run / gw, "reference_value": steps_run / rw, "wall_s": gw, "reference_wall_s": rw,
                     "vtk_identical_at_first_middle_last": same_files,
                     "note": "wall clock of each program, process start and CUDA context creation included"})
        import shutil

        shutil.rmtree(gout, ignore_errors=True)
        shutil.rmtree(rout, ignore_errors=True)
    except Exception as e:
        prog["unavailable"] = str(e)[:200]
    sus_ref = None
    try:
        wall_s, _ = _ref_run_wall(sus_path, 500)
        sus_ref = 500 / wall_s
    except Exception:
        pass
    res["program_with_outputs"] = prog
    res["sustained_contact"] = {"value": 500 / (sum(s_ms) / 1e3), "unit": "pair-contacts/s", "dt": 1e-15,
                                "contacts_per_step": sus_contacts, "reference_value": sus_ref}
    return res


def run_two(args):
    """Two 320-triangle noised icospheres colliding (2000 steps, dt 1e-6), and the same pair held in
    contact (dt 1e-15): steps/s of the whole DEM step, graph and plain, and the trajectory against the
    reference program."""
    import tempfile

    import torch

    from zdemx import _lib
    from zdemx.workloads import two_particle_scene

    if int(os.environ.get("RANK", "0")) != 0:
        return
    steps_run = 2000
    if args.impl == "reference":
        if not os.path.exists(_ref_exe()):
            emit({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"})
            return
        d = tempfile.mkdtemp(prefix="zdx_two_")
        cfg_path = two_particle_scene(d, seed=args.seed, steps=steps_run)
        wall, _ = _ref_run_wall(cfg_path, steps_run)
        value = steps_run / wall
        emit({"impl": "reference", "metric": "DEM steps/s", "value": value, "unit": "steps/s", "n_gpus": 1,
              "steps": steps_run, "warmup": 0, "ms_per_step": 1e3 / value, "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
              "config": {"workload": "two particles, 2000 steps (see --impl zdemx)"},
              "cpu_baseline": {"value": value, "unit": "steps/s", "cores": 1, "kind": "reference",
                               "sample": f"the whole {steps_run}-step zdem_cpu run (wall clock)"},
              "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        return
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctx = _lib.Context(0)
    m = measure_two(args, ctx, reps=max(int(args.steps), 1), extras=True)
    line = {"metric": m.pop("metric"), "value": m.pop("value"), "unit": m.pop("unit"), "n_gpus": 1,
            "steps": m.pop("steps"), "warmup": m.pop("warmup"), "ms_per_step": m.pop("ms_per_step"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)"}
    line.update(m)
    emit(line)


def run_adjoint(args):
    """16,384 pairs of 320-triangle noised icospheres at depth U(0.01, 0.08) r: the forward call plus the
    hand-written adjoint (dL/d corners and poses from dL/dSn, dL/dGn), and a batched central-difference
    check of the pose gradients (h = 1e-7 r) with pairs whose stencil changes the loop topology flagged."""
    import torch

    from zdemx import _lib, synth
    from zdemx.contact import MeshLibrary

    if int(os.environ.get("RANK", "0")) != 0:
        return
    if args.impl == "reference":
        emit({"impl": "reference", "unavailable": "the reference has no derivatives (no adjoint to time)"})
        return
    npairs = 16384
    rng = np.random.default_rng(args.seed)
    lib = MeshLibrary.build(list(synth.noised_icospheres(2, 256, 1e-3, 0.15, rng)))
    pm = rng.integers(0, 256, size=(npairs, 2)).astype(np.int32)
    pp = synth.pair_poses(rng, npairs, 1e-3, 0.01, 0.08)
    pp[:, 3:7] = synth.random_unit_quat(rng, npairs)
    desc = ("adjoint: 16384 pairs of 320-triangle noised icospheres (256-mesh library, r 1 mm, +-15%), depth "
            "U(0.01,0.08) r; forward + reverse of Sn, Gn w.r.t. corners and poses; FP64")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctx = _lib.Context(0)
    stream = _lib_stream(ctx)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    meshes = {"tris": T(lib.tris), "tri_off": T(lib.tri_off), "mean_edge": T(lib.mean_edge), "bbox_diag": T(lib.bbox_diag)}
    pairs = {"mesh": T(pm), "pose": T(pp)}
    cap = 8 * npairs
    out = {"ncontact": torch.zeros(npairs, dtype=torch.int32, device=dev),
           "contact_off": torch.zeros(npairs + 1, dtype=torch.int64, device=dev),
           "stats": torch.zeros(npairs, 4, dtype=torch.int32, device=dev),
           "geom": torch.zeros(cap, 20, dtype=torch.float64, device=dev),
           "info": torch.zeros(cap, 4, dtype=torch.int32, device=dev)}
    tot = _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7)
    nc = int(tot[0])
    wrng = np.random.default_rng(7)
    w = np.concatenate([wrng.normal(size=(nc, 3)) / 1e-6, wrng.normal(size=(nc, 3)) / 1e-9], 1)
    gc = T(w)
    gt = torch.zeros_like(meshes["tris"])
    gp = torch.zeros(npairs, 12, dtype=torch.float64, device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    for _ in range(max(args.warmup, 3)):
        _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7)
        _lib.pair_contacts_adjoint(ctx, meshes, pairs, gc, gt, gp)
    fwd, adj = [], []
    launches0 = ctx.timings()["launches"]
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            torch.cuda.synchronize()
            _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7)
            fwd.append(ctx.timings()["total"])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                flush.zero_()
                e0.record(stream)
            _lib.pair_contacts_adjoint(ctx, meshes, pairs, gc, gt, gp)
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize()
            adj.append(e0.elapsed_time(e1))
    launches = ctx.timings()["launches"] - launches0
    step_s = (sum(fwd) + sum(adj)) / 1e3 / args.steps
    # the plain forms -- one launch per stage over the subset (no queue, cost order or culls), and one
    # launch per pair per stage -- against the batched one on the same subset of pairs
    ns = min(args.plain_pairs, npairs)
    sub_p = {"mesh": pairs["mesh"][:ns].contiguous(), "pose": pairs["pose"][:ns].contiguous()}
    sub_o = {kk: (v[:ns].contiguous() if kk in ("ncontact", "stats") else v) for kk, v in out.items()}
    sub_o["contact_off"] = out["contact_off"][: ns + 1].contiguous()
    forms = {}
    for name, sched in (("batched", _lib.SCHED_BATCHED), ("per_stage", _lib.SCHED_PER_STAGE), ("plain", _lib.SCHED_PLAIN)):
        tt = []
        for rep in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tsub = _lib.pair_contacts_device(ctx, meshes, sub_p, sub_o, k=1e7, sched=sched)
            gsub = torch.zeros(int(tsub[0]), 6, dtype=torch.float64, device=dev)
            gsub[:] = gc[: int(tsub[0])] if int(tsub[0]) <= gc.shape[0] else 0.0
            gps = torch.zeros(ns, 12, dtype=torch.float64, device=dev)
            _lib.pair_contacts_adjoint(ctx, meshes, sub_p, gsub, gt, gps, sched=sched)
            torch.cuda.synchronize()
            tt.append(time.perf_counter() - t0)
        forms[name] = (min(tt[1:]), gps.clone())
    plain_form = {"pairs": ns, "batched_pairs_per_s": ns / forms["batched"][0], "plain_pairs_per_s": ns / forms["plain"][0],
                  "speedup_batched_vs_plain": forms["plain"][0] / forms["batched"][0],
                  "per_stage_pairs_per_s": ns / forms["per_stage"][0],
                  "speedup_batched_vs_plain_per_stage": forms["per_stage"][0] / forms["batched"][0],
                  "grad_pose_max_abs_diff": float((forms["plain"][1] - forms["batched"][1]).abs().max()),
                  "grad_pose_max_abs_diff_per_stage": float((forms["per_stage"][1] - forms["batched"][1]).abs().max()),
                  "note": "forward with tape + reverse, wall clock around each call (host syncs included)"}
    # batched central differences of the per-pair objective w.r.t. the 12 pose coordinates
    gpose = gp.cpu().numpy()
    base = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pm, pp)
    coff = base["contact_off"]
    incontact = np.diff(coff) > 0

    def per_pair(r):
        """Per pair sum of w . (Sn, Gn), contacts matched to the base call's by position within the pair
        (pairs whose contact count changed are flagged by topo())."""
        cr = r["contact_off"]
        cnt = np.diff(cr)
        pid = np.repeat(np.arange(npairs), cnt)
        same = cnt == np.diff(coff)
        loc = np.arange(len(pid)) - cr[pid]
        bidx = np.where(same[pid], coff[pid] + loc, 0)
        g = r["geom"]
        v = np.einsum("ij,ij->i", w[bidx, 0:3], g[:, 0:3]) + np.einsum("ij,ij->i", w[bidx, 3:6], g[:, 3:6])
        v = np.where(same[pid], v, 0.0)
        return np.bincount(pid, weights=v, minlength=npairs)

    def topo(r):
        return np.concatenate([r["stats"], np.diff(r["contact_off"])[:, None]], 1)

    def qmul(a, b):
        aw, ax, ay, az = a
        bw, bx, by, bz = b.T
        return np.stack([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                         aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw], 1)

    t_base = topo(base)
    flagged = np.zeros(npairs, bool)
    fds = []
    for h in (1e-7 * 1e-3, 0.25e-7 * 1e-3):
        fd = np.zeros((npairs, 12))
        fds.append(fd)
        for b in range(2):
            for k in range(3):
                for kind in ("pos", "rot"):
                    vals = []
                    for sgn in (1, -1):
                        q = pp.copy()
                        if kind == "pos":
                            q[:, 7 * b + k] += sgn * h
                        else:
                            th = sgn * h / 1e-3
                            qe = np.zeros(4)
                            qe[0] = np.cos(abs(th) / 2)
                            qe[1 + k] = np.sin(th / 2)
                            q[:, 7 * b + 3: 7 * b + 7] = qmul(qe, q[:, 7 * b + 3: 7 * b + 7])
                        r = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pm, q)
                        flagged |= ~np.all(topo(r) == t_base, axis=1)
                        vals.append(per_pair(r))
                    col = 6 * b + (k if kind == "pos" else 3 + k)
                    fd[:, col] = (vals[0] - vals[1]) / (2 * h) * (1.0 if kind == "pos" else 1e-3)
    fd = fds[0]
    # a stencil that straddles a kink of the piecewise-smooth map (a clamp, a dedup or snap decision that
    # flips without changing any count) shows as disagreement between the two step sizes
    nonsmooth = np.zeros(npairs, bool)
    rel = np.zeros(npairs)
    for cols in ([0, 1, 2, 6, 7, 8], [3, 4, 5, 9, 10, 11]):  # translations, rotation vectors: each to its own scale
        sc2 = np.maximum(np.max(np.abs(fds[1][:, cols]), 1), 1e-300)
        nonsmooth |= np.max(np.abs(fds[0][:, cols] - fds[1][:, cols]), 1) / sc2 > 1e-4
        scale = np.maximum(np.max(np.abs(fd[:, cols]), 1), 1e-300)
        rel = np.maximum(rel, np.max(np.abs(gpose[:, cols] - fd[:, cols]), 1) / scale)
    ok = (~flagged) & (~nonsmooth) & incontact
    rel_ok = rel[ok]
    emit({"metric": "gradient pairs/s", "value": npairs / step_s, "unit": "pairs/s", "n_gpus": 1, "steps": args.steps,
          "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * step_s, "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded noised icospheres)",
          "config": {"workload": desc, "contacts": nc, "l2": "flushed (256 MB write) before the forward and the adjoint"},
          "stages_ms": {"forward": statistics.mean(fwd), "adjoint_call (forward with tape + reverse)": statistics.mean(adj)},
          "plain": plain_form,
          "gpu_launches": int(launches),
          "fd_check": {"pairs_in_contact": int(incontact.sum()), "pairs_checked": int(ok.sum()),
                       "pairs_flagged_topology_change": int(np.sum(flagged & incontact)),
                       "pairs_flagged_nonsmooth_stencil": int(np.sum(nonsmooth & ~flagged & incontact)),
                       "max_rel_err": float(rel_ok.max()) if len(rel_ok) else None,
                       "median_rel_err": float(np.median(rel_ok)) if len(rel_ok) else None,
                       "frac_within_1e-6": float(np.mean(rel_ok <= 1e-6)) if len(rel_ok) else None,
                       "h": "1e-7 r (and 2.5e-8 r for the smoothness flag)"},
          "clocks": clk.summary()})


def run_rollout(args):
    """Calibration rollout: n^3 320-triangle icospheres on a 2-triangle plane, the feng_min law, 2000
    steps of dt 2e-6; loss = sum of squared final-position errors against a target made with k = 1.3e7,
    e = 0.35; gradients w.r.t. k, e and the initial velocities v0, with the rollout checkpointed every
    100 steps and with every step's intermediates stored."""
    import tempfile

    import torch

    from zdemx import _lib
    from zdemx.dem import Scene
    from zdemx.rollout import DiffScene
    from zdemx.workloads import calibration_scene

    if int(os.environ.get("RANK", "0")) != 0:
        return
    d = tempfile.mkdtemp(prefix="zdx_cal_")
    steps = args.rollout_steps
    cfg_path = calibration_scene(d, n_side=args.rollout_side, seed=args.seed, steps=steps)
    n = args.rollout_side ** 3
    desc = (f"calibration rollout: {n} noised icospheres (320 triangles, circumradius 1 mm) on a 2-triangle plane, "
            f"feng_min law, {steps} steps of dt 2e-6; loss = sum |x_T - x_T(k=1.3e7, e=0.35)|^2; "
            "gradients w.r.t. k, e, v0 (reverse mode through the CUDA contact adjoint), FP64")
    if args.impl == "reference":
        emit({"impl": "reference", "unavailable": "the reference has no derivatives (no gradient rollout to time)"})
        return
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctx = _lib.Context(0)
    sc = Scene(cfg_path, ctx)
    ds = DiffScene(sc)
    state0 = torch.from_numpy(sc.state()[0]).to(dev)
    f64 = lambda v: torch.tensor(v, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.no_grad():
        tgt, _ = ds.rollout(state0, f64(1.3e7), f64(0.35), steps)
    torch.cuda.synchronize()
    fwd_torch_s = time.perf_counter() - t0
    target = tgt[:, 0:3].clone()
    del tgt

    def grad_run(ck):
        k = f64(1e7).requires_grad_(True)
        e = f64(0.5).requires_grad_(True)
        v0 = state0[:, 7:10].clone().requires_grad_(True)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        base = torch.cuda.memory_allocated()
        t1 = time.perf_counter()
        st = torch.cat([state0[:, 0:7], v0, state0[:, 10:16]], 1)
        xT, last = ds.rollout(st, k, e, steps, checkpoint_every=ck)
        loss = ((xT[:, 0:3] - target) ** 2).sum()
        loss.backward()
        torch.cuda.synchronize()
        dt_s = time.perf_counter() - t1
        peak = torch.cuda.max_memory_allocated() - base
        free, total = torch.cuda.mem_get_info()
        print(f"rollout ck={ck}: {dt_s:.1f} s, torch peak {peak / 1e9:.2f} GB, reserved "
              f"{torch.cuda.memory_reserved() / 1e9:.2f} GB, device free {free / 1e9:.1f} of {total / 1e9:.1f} GB",
              file=sys.stderr, flush=True)
        return {"seconds": dt_s, "peak_torch_bytes": int(peak), "loss": loss.item(), "dL_dk": k.grad.item(),
                "dL_de": e.grad.item(), "dL_dv0_norm": float(v0.grad.norm().item()), "last_step": last}

    ck = grad_run(100)
    try:
        full = grad_run(None)
        same = abs(full["dL_dk"] - ck["dL_dk"]) <= 1e-9 * abs(ck["dL_dk"])
        full["matches_checkpointed"] = bool(same)
    except torch.cuda.OutOfMemoryError as exc:
        full = {"unavailable": f"out of memory: {str(exc)[:120]}"}
    torch.cuda.empty_cache()
    free, total = torch.cuda.mem_get_info()
    print(f"before the graph forward: device free {free / 1e9:.1f} of {total / 1e9:.1f} GB", file=sys.stderr, flush=True)
    # the same forward on the CUDA graph step (no gradients)
    try:
        sg = Scene(cfg_path, ctx)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        sg.step_graph(steps)
        torch.cuda.synchronize()
        graph_s = time.perf_counter() - t1
        moved = float(np.max(np.abs(sg.state()[0][:, 0:3] - state0[:, 0:3].cpu().numpy())))
    except _lib.ZdxError as exc:
        graph_s, moved = None, f"unavailable: {exc}"
    cpu = {"value": None, "unit": "steps/s", "cores": 1, "kind": "reference", "sample": "skipped (--cpu-seconds 0)"}
    if args.cpu_seconds > 0 and os.path.exists(_ref_exe()):
        try:
            ms, _ = _ref_step_ms(cfg_path, 3)
            cpu = {"value": 1e3 / np.mean(ms), "unit": "steps/s", "cores": 1, "kind": "reference",
                   "sample": "3 forward steps of zdem_cpu on the same scene (its zdem law; it has no feng_min and no "
                             "gradients)"}
        except Exception as exc:
            cpu["sample"] = f"unavailable: {exc}"
    value = steps / ck["seconds"]
    emit({"metric": "gradient rollout steps/s", "value": value, "unit": "steps/s", "n_gpus": 1, "steps": steps,
          "warmup": 0, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
          "dtype": "f64", "data": "synthetic (seeded calibration scene)",
          "config": {"workload": desc, "particles": n, "checkpoint_every": 100},
          "checkpointed": ck, "stored": full,
          "forward_only": {"torch_step_s": fwd_torch_s, "cuda_graph_step_s": graph_s,
                           "max_displacement_m": moved},
          "cpu_baseline": cpu})


if __name__ == "__main__":
    main()

