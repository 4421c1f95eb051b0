#!/usr/bin/env python3
"""PairHMM forward-pass benchmark (one JSON line on rank 0).

Workload (default): 4096 uneven active regions -- reads per region lognormal
(median 60, sigma 0.75, 20-500), read length U(50, 250), 2-32 haplotypes of
U(200, 700) bp per region, 1% SNVs and 0-2 indels per haplotype, 1% read
substitutions, q ~ U(10, 40), i = d = 45, c = 10 -- seeded synthetic data.
A step scores every read against every haplotype of its region: ~5.4 M pairs,
~3.7e11 DP cells.

* value    pairs/s with the batch resident in HBM (staged once), device time of
           the step's kernels from CUDA events on the engine's stream; the
           inputs (~274 MB) exceed the 126 MB L2, so nothing is flushed.
* e2e      pairs/s through bv_phmm_compute_regions with host buffers (page-
           locked): validation and planning, host->device copies, kernels and
           the device->host copy of the log10 results inside the timed region.
* roofline the FP32 forward kernels against the measured FP32 FMA peak (12
           algorithmic flops per DP cell, the reference's computeMXY count).
* cpu_baseline  Biovoltron's own AVX PairHMM kernel (oracle/_ref, compiled
           from the reference sources) on all host cores, on a seeded sample of
           the same regions.

--impl reference times that CPU kernel alone, on the same workload.
Multi-GPU (torchrun): every rank scores its own batch (different seed) on its
own GPU, no data-path collective (weak scaling); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from biovoltron_b200 import workloads as W  # noqa: E402

METRIC = "PairHMM GCUPS & pairs/s on 1 B200: learned-band+batched vs plain DP, <=1e-3 log10L err"
FLOPS_PER_CELL = 12  # computeMXY: 8 mul + 4 add (avx-pairhmm-template.h:183-198)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(name: str, seed: int, regions: int = 0) -> W.RegionBatch:
    if name == "config1":
        return W.config1(seed=seed, n_regions=regions or 4096)
    if name == "config0":
        return W.config0(seed)
    if name == "config2":
        return W.config2(seed=seed)
    if name == "config4":
        return W.config4(seed=seed)
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = [r.split(", ") for r in out.strip().splitlines() if r.strip()]
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_rate(batch: W.RegionBatch, target_s: float, seed: int = 0):
    """Times Biovoltron's AVX kernel (or, if it was not built, the C oracle) on
    all host threads over a seeded sample of regions sized for ~target_s."""
    from oracle.oracle import Oracle, Reference, TestcaseArray
    kind = "reference" if Reference.available() else "port"
    impl = Reference() if kind == "reference" else Oracle()
    run = (lambda t: impl.log10(t)) if kind == "reference" else (lambda t: impl.log10_reference_rule(t))
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    order = rng.permutation(batch.n_regions)
    nr = np.diff(batch.region_reads)
    nh = np.diff(batch.region_haps)

    def sample(frac_cells):
        total = batch.n_cells()
        want = frac_cells * total
        picked, acc = [], 0.0
        rl = batch.read_lengths()
        hl = batch.hap_lengths()
        for g in order:
            r0, r1 = batch.region_reads[g], batch.region_reads[g + 1]
            h0, h1 = batch.region_haps[g], batch.region_haps[g + 1]
            acc += float(rl[r0:r1].sum()) * float(hl[h0:h1].sum())
            picked.append(int(g))
            if acc >= want:
                break
        return W.subsample_regions(batch, picked)

    cal = sample(0.002)
    tc = TestcaseArray.for_batch(cal)
    t0 = time.perf_counter()
    run(tc)
    dt = max(time.perf_counter() - t0, 1e-6)
    rate = cal.n_cells() / dt
    frac = min(1.0, target_s * rate / batch.n_cells())
    smp = sample(frac)
    tc = TestcaseArray.for_batch(smp)
    t0 = time.perf_counter()
    run(tc)
    dt = time.perf_counter() - t0
    cells = smp.n_cells()
    return {
        "kind": kind, "cores": threads, "pairs": smp.n_pairs, "cells": cells, "seconds": dt,
        "pairs_per_s": smp.n_pairs / dt, "gcups": cells / dt / 1e9,
        "sample": f"{smp.n_regions} of {batch.n_regions} regions (seeded), {smp.n_pairs} pairs, {cells:.3e} cells",
    }


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def allreduce(pg, x: float, op: str) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op={"max": pg.ReduceOp.MAX, "sum": pg.ReduceOp.SUM}[op])
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_reference(args):
    world, rank, local, pg = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0, None
    if rank != 0:
        return
    batch = make_workload(args.workload, args.seed, args.regions)
    per_step = []
    info = None
    for k in range(args.warmup + args.steps):
        info = cpu_reference_rate(batch, target_s=args.ref_seconds, seed=k)
        if k >= args.warmup:
            per_step.append(info)
    pps = float(np.mean([p["pairs_per_s"] for p in per_step]))
    gc = float(np.mean([p["gcups"] for p in per_step]))
    line = {
        "impl": "reference", "metric": METRIC, "value": pps, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean([p["seconds"] for p in per_step]) * 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded)", "gcups": gc,
        "config": {"workload": batch.name, "pairs": batch.n_pairs, "cells": batch.n_cells(),
                   "sample_per_step": info["sample"], "l2": "inputs > L2"},
        "cpu_baseline": {"value": pps, "unit": "pairs/s", "cores": info["cores"], "kind": info["kind"],
                         "sample": info["sample"], "gcups": gc},
        "e2e": {"value": pps, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="config1")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--regions", type=int, default=0, help="config1 only: fewer regions (profiling cases)")
    ap.add_argument("--ref-seconds", type=float, default=10.0, help="CPU seconds per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--haps-per-warp", type=int, default=0, help="0: engine default, 1 or 2")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    world, rank, local, pg = dist_setup(args)
    from biovoltron_b200.native import load
    from biovoltron_b200.pairhmm import PairHMMEngine
    import ctypes as C

    batch = make_workload(args.workload, args.seed + 1000 * rank, args.regions)
    log(f"[rank {rank}] workload: {batch.name}: {batch.n_pairs} pairs, {batch.n_cells():.3e} cells")
    eng = PairHMMEngine(device=local, haps_per_warp=args.haps_per_warp)
    lib = load()
    peak = C.c_double(0)
    st = lib.bv_phmm_measure_fp32_peak(local, C.byref(peak))
    fp32_peak = peak.value if st == 0 else None

    # ---- device-resident throughput -------------------------------------
    n = eng.stage(batch)
    for _ in range(args.warmup):
        eng.run()
    barrier(pg)
    clocks = ClockSampler(local)
    clocks.start()
    dev_ms, fp32_ms, fp64_ms = [], [], []
    stats = None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        stats = eng.run()
        fp32_ms.append(stats["ms_fp32"])
        fp64_ms.append(stats["ms_fp64"])
        dev_ms.append(stats["ms_fp32"] + stats["ms_fp64"])
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    barrier(pg)
    t_dev = allreduce(pg, float(np.sum(dev_ms)), "max")
    total_pairs = allreduce(pg, float(n * args.steps), "sum")
    value = total_pairs / (t_dev / 1e3)
    cells = stats["cells"]
    gcups = allreduce(pg, float(cells * args.steps), "sum") / (t_dev / 1e3) / 1e9
    results = eng.fetch(n)

    # ---- end to end through the public API --------------------------------
    arrays = [batch.read_bases, batch.read_q, batch.read_i, batch.read_d, batch.read_c, batch.hap_bases]
    for a in arrays:
        eng.host_register(a)
    out = np.empty(max(n, 1), np.float64)
    eng.host_register(out)
    for _ in range(max(1, args.warmup)):
        eng.compute_regions(batch, out=out)
    barrier(pg)
    e2e_t = []
    for _ in range(args.steps):
        t1 = time.perf_counter()
        eng.compute_regions(batch, out=out)
        e2e_t.append(time.perf_counter() - t1)
    barrier(pg)
    for a in arrays + [out]:
        eng.host_unregister(a)
    e2e_time = allreduce(pg, float(np.sum(e2e_t)), "max")
    e2e = total_pairs / e2e_time
    same = bool(np.array_equal(out[:n], results))

    # ---- CPU baseline (rank 0, one GPU only) ------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(batch, target_s=args.ref_seconds)

    if rank == 0:
        fp32_mean = float(np.mean(fp32_ms))
        achieved = FLOPS_PER_CELL * cells / (fp32_mean / 1e3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
            "gcups": gcups,
            "config": {"workload": batch.name, "form": "plain full DP, batched (persistent length-binned launches)",
                       "pairs_per_gpu": n, "cells_per_gpu": cells, "rescued_per_step": stats["rescued"],
                       "l2": "inputs 274 MB > 126 MB L2, no flush", "parallelism": f"dp{world} (independent regions)"},
            "e2e": {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(batch.nbytes()),
                    "d2h_bytes_per_step": int(8 * n), "results_identical_to_device_run": same},
            "roofline": {"bound": "fp32", "kernel": "k_forward<float> (all rows-per-lane variants)",
                         "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": (achieved / fp32_peak) if fp32_peak else None, "traffic": None,
                         "peak_source": "measured: FP32 FMA probe kernel in this run (bv_phmm_measure_fp32_peak)",
                         "flops_per_cell": FLOPS_PER_CELL},
            "kernel_ms": {"fp32": fp32_mean, "fp64_rescue": float(np.mean(fp64_ms))},
            "gpu_launches": int(stats["kernel_launches"]) * args.steps,
            "clocks": clk,
            "wall_s_timed": wall,
        }
        if cpu:
            line["cpu_baseline"] = {"value": cpu["pairs_per_s"], "unit": "pairs/s", "cores": cpu["cores"],
                                    "kind": cpu["kind"], "sample": cpu["sample"], "gcups": cpu["gcups"]}
        print(json.dumps(line), flush=True)
    eng.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
