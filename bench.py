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
    return ap.parse_args()


def workload(args, rank):
    from zdemx import synth
    from zdemx.contact import MeshLibrary

    rng = np.random.default_rng(args.seed)
    raw = []
    for s in (1, 2, 3, 4):
        raw.extend(list(synth.noised_icospheres(s, args.lib_per_level, 1e-3, 0.15, rng)))
    lib = MeshLibrary.build(raw)
    prng = np.random.default_rng(args.seed + 1 + rank)
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


def profiled_traffic():
    """DRAM bytes per pair of the triangle-test kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


def cpu_reference_rate(lib, pm, pp, nthreads, seconds, rng_seed=5, fixed=None):
    """Time the reference's own per-pair code (oracle/_ref) on a bounded random sample of the workload."""
    import ctypes as C

    from oracle import LIB_REF

    L = C.CDLL(LIB_REF)
    L.zdx_ref_pair_batch.restype = C.c_int64
    L.zdx_ref_pair_batch.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                        C.c_void_p]
    rng = np.random.default_rng(rng_seed)
    order = rng.permutation(len(pm))

    def run(sel):
        spm = np.ascontiguousarray(pm[sel])
        spp = np.ascontiguousarray(pp[sel])
        t0 = time.perf_counter()
        L.zdx_ref_pair_batch(lib.tris.ctypes.data, lib.tri_off.ctypes.data, lib.mean_edge.ctypes.data,
                             lib.bbox_diag.ctypes.data, lib.n_mesh, len(sel), spm.ctypes.data, spp.ctypes.data, 1,
                             nthreads, None)
        return time.perf_counter() - t0

    if fixed is not None:
        dt = run(fixed)
        return len(fixed) / dt, len(fixed), dt, fixed
    n = 32 * nthreads
    dt = run(order[:n])
    n = int(min(len(pm), max(n, n * seconds / max(dt, 1e-3))))
    sel = order[:n]
    dt = run(sel)
    return n / dt, n, dt, sel


def emit(d):
    print(json.dumps(d), flush=True)


def main():
    args = parse()
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
        if rank != 0:
            return
        from oracle import LIB_REF

        if not os.path.exists(LIB_REF):
            emit({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"})
            return
        lib, pm, pp = workload(args, 0)
        nthreads = os.cpu_count() or 1
        # size one step's sample to ~2 s of work on all threads
        rate, n, dt, sel = cpu_reference_rate(lib, pm, pp, nthreads, 2.0)
        times = []
        for i in range(args.warmup + args.steps):
            r, _, d, _ = cpu_reference_rate(lib, pm, pp, nthreads, 0.0, fixed=sel)
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
    out = {"ncontact": torch.zeros(args.pairs, dtype=torch.int32, device=dev),
           "contact_off": torch.zeros(args.pairs + 1, dtype=torch.int64, device=dev),
           "stats": torch.zeros(args.pairs, 4, dtype=torch.int32, device=dev),
           "geom": torch.zeros(cap, 20, dtype=torch.float64, device=dev),
           "info": torch.zeros(cap, 4, dtype=torch.int32, device=dev)}
    meshes = {"tris": d_tris, "tri_off": d_off, "mean_edge": d_me, "bbox_diag": d_bd}
    pairs = {"mesh": d_pm, "pose": d_pp}
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def step():
        return _lib.pair_contacts_device(ctx, meshes, pairs, out, k=1e7, split=True)

    for _ in range(args.warmup):
        totals = step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.timings()["launches"]
    step_ms, seg_ms, reb_ms = [], [], []
    wall0 = time.perf_counter()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            totals = step()
            t = ctx.timings()
            step_ms.append(t["total"])
            seg_ms.append(t["segments"])
            reb_ms.append(t["rebuild"])
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    launches = ctx.timings()["launches"] - launches0
    T = sum(step_ms) / 1e3
    if world > 1:
        tt = torch.tensor([T], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        T = float(tt.item())
        dist.barrier()
    value = world * args.pairs * args.steps / T

    # e2e: the same call with pinned host buffers, copies inside the timed region
    h = {k: torch.from_numpy(v).pin_memory() for k, v in
         {"tris": lib.tris, "off": lib.tri_off, "me": lib.mean_edge, "bd": lib.bbox_diag, "pm": pm, "pp": pp}.items()}
    hout = {"ncontact": torch.zeros(args.pairs, dtype=torch.int32).pin_memory(),
            "contact_off": torch.zeros(args.pairs + 1, dtype=torch.int64).pin_memory(),
            "stats": torch.zeros(args.pairs, 4, dtype=torch.int32).pin_memory(),
            "geom": torch.zeros(cap, 20, dtype=torch.float64).pin_memory(),
            "info": torch.zeros(cap, 4, dtype=torch.int32).pin_memory()}
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
        tt = torch.tensor([TE], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        TE = float(tt.item())
    e2e_value = world * args.pairs * args.steps / TE
    h2d = sum(int(v.numel() * v.element_size()) for v in h.values())
    nct = int(tot_e[0])
    d2h = args.pairs * (4 + 8 + 16) + 8 + nct * (160 + 16)

    # plain form on a subset (one launch per stage per pair)
    plain_n = min(args.plain_pairs, args.pairs)
    sub = {"mesh": d_pm[:plain_n].contiguous(), "pose": d_pp[:plain_n].contiguous()}
    _lib.pair_contacts_device(ctx, meshes, sub, out, k=1e7, split=True, sched=_lib.SCHED_PLAIN)
    torch.cuda.synchronize()
    _lib.pair_contacts_device(ctx, meshes, sub, out, k=1e7, split=True, sched=_lib.SCHED_PLAIN)
    plain_ms = ctx.timings()["total"]
    _lib.pair_contacts_device(ctx, meshes, sub, out, k=1e7, split=True)
    batched_sub_ms = ctx.timings()["total"]
    plain_value = plain_n / (plain_ms / 1e3)

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # roofline of the triangle-test kernel (dominant): algorithmic bytes / its measured duration
    peak, peak_kind = measured_peaks()
    abytes = algorithmic_bytes(lib, pm)
    seg_s = statistics.mean(seg_ms) / 1e3
    achieved = abytes / seg_s / 1e9
    tr = profiled_traffic()
    traffic = None
    if tr and "dram_bytes_per_pair" in tr:
        traffic = float(tr["dram_bytes_per_pair"]) * args.pairs

    rate, n_cpu, dt_cpu, _ = cpu_reference_rate(lib, pm, pp, 1, args.cpu_seconds)
    cfg = dict(base_cfg)
    cfg.update({"l2": "flushed (256 MB write) before every timed step", "inputs": "device-resident for value",
                "contacts_per_step": int(totals[0]), "segments_per_step": int(totals[1]),
                "tri_aabb_checks_per_step": int(totals[2])})
    emit({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
          "warmup": args.warmup, "ms_per_step": 1e3 * T / args.steps, "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded noised icospheres, 1024-mesh library)",
          "config": cfg,
          "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
          "gpu_launches": int(launches),
          "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "traffic": traffic, "kernel": "k_segments", "peak_kind": f"{peak_kind} hbm_gbs",
                       "algorithmic_bytes_per_launch": abytes, "kernel_ms": 1e3 * seg_s,
                       "note": "FP64 compare/ALU (SM-issue) bound, not HBM bound; issue utilisation in profiles/"},
          "stages_ms": {"triangle_tests": statistics.mean(seg_ms), "rebuild": statistics.mean(reb_ms),
                        "whole_call": statistics.mean(step_ms)},
          "plain": {"value": plain_value, "unit": UNIT, "pairs": plain_n, "batched_same_pairs": plain_n / (batched_sub_ms / 1e3),
                    "speedup_batched_vs_plain": (plain_n / (batched_sub_ms / 1e3)) / plain_value},
          "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
                           "sample": f"{n_cpu} random pairs of the workload through oracle/_ref, {dt_cpu:.1f} s"},
          "clocks": clk.summary(), "wall_s_timed": wall})
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
