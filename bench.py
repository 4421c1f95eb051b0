#!/usr/bin/env python3
"""PairHMM forward-pass benchmark (one JSON line on rank 0).

Default workload (config 4, the headline): 200,000 active regions of 300 bp
over a 60 Mb uniform-ACGT synthetic reference, 30x coverage of 150 bp reads
(1% substitutions, 0.1% indels), 2-16 haplotypes per region spanning the
region +-75 bp with SNV/indel alleles at 1/1000 bp; q ~ U(10, 40), i = d =
45, c = 10.  Every read is scored against every haplotype of its region:
~1.08e8 pairs, ~7.3e12 DP cells.  Seeded synthetic data (no dataset).

The full chosen form runs: the band MLP is first trained on the GPU (labels
from the full DP's posterior spreads, 1M pairs drawn from config 1's
distribution, its own seed); then every step scores the whole batch with the
learned band (featuriser, BF16 MLP, banded forward pass with the ring test
-- the band widened by 4 or 8 diagonals per side is the result, a ring share
above the threshold widens the band, after 32 diagonals the full DP takes the
pair; banded pairs more than --cap-margin log10 units below their read's best
are then scored again by the full DP -- and a sampled audit against the full
DP) and FP32 with FP64 rescue.  The plain
full-DP kernels score the same batch in the same run for the comparison.

* value        pairs/s of the full chosen form with the batch resident in HBM
               (device time from CUDA events on the engine's stream; inputs of
               ~9.9 GB exceed the 126 MB L2, so nothing is flushed).
* plain        the same for the plain full DP (FP32 + FP64 rescue).
* e2e          pairs/s through bv_phmm_compute_regions in band mode with
               page-locked host buffers: validation, planning, host->device
               copies, all kernels and the device->host copy of the results
               (the call splits the batch into region chunks over two
               contexts so copies overlap kernels).  The workloads' gap
               penalties are constant (as SamRecord's are), so they go as the
               batch's three uniform gap bytes: 2 bytes cross per read base.
* genotype     the device genotyper on the staged batch's matrix (normalise,
               filter, marginalise, diploid genotype likelihoods), outside
               the timed region.
* accuracy     max / p99 |dlog10L| of both forms against the FP64 oracle on a
               seeded sample of pairs, and of the band against the full DP on
               every pair.
* roofline     the dominant kernels (the banded forward passes) against the
               measured FP32 FMA peak, 12 algorithmic flops per band cell;
               roofline_plain the full-DP kernels, 12 flops per cell
               (the reference's computeMXY count).
* cpu_baseline Biovoltron's own AVX PairHMM kernel (oracle/_ref, compiled from
               the reference sources) on all host cores, on a seeded sample of
               the same regions.

--impl reference times that CPU kernel alone, on the same workload.
--workload config0|config1|config2|config3 --form plain|band run the other configs
(config3 = the learned band on config 1's workload, with the plain full DP of
the same batch beside it and every pair's band-vs-full difference).
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

from biovoltron_b200 import replicas  # noqa: E402
from biovoltron_b200 import workloads as W  # noqa: E402

METRIC = "PairHMM GCUPS & pairs/s on 1 B200: learned-band+batched vs plain DP, <=1e-3 log10L err"
FLOPS_PER_CELL = 12  # computeMXY: 8 mul + 4 add (avx-pairhmm-template.h:183-198)
# DRAM bytes (read + write) per pair from one ncu capture of a config-4-shaped
# batch of 2,000 regions: the full-size step is too large to capture, and both
# kernels' traffic grows with the pairs.
DRAM_BYTES_PER_PAIR_PLAIN = 101.6  # k_forward<float, 5, 0, 1>: 111.2 MB per launch, 1.094e6 pairs
DRAM_BYTES_PER_BAND_PAIR = 179.4   # k_band_ring_f32<8..32>: 194.8 MB per step, 1.086e6 banded pairs
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum on 2,000 config-4 regions, "
                  "scaled by the step's pairs")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(name: str, seed: int, regions: int = 0) -> W.RegionBatch:
    if name in ("config1", "config3"):  # config 3 is the learned band on config 1's workload
        return W.config1(seed=seed, n_regions=regions or 4096)
    if name == "config0":
        return W.config0(seed)
    if name == "config2":
        return W.config2(seed=seed)
    if name == "config4":
        return W.config4(seed=seed, n_regions=regions or 200_000)
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
        rows = [r for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]

        def num(x):
            try:
                return float(x)
            except ValueError:
                return 0.0
        # under load: samples drawing at least half of the highest power seen
        pmax = max([num(r[3]) for r in rows], default=0.0)
        loaded = [r for r in rows if num(r[3]) >= 0.5 * pmax] or rows
        sm = [float(r[1]) for r in loaded]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(sm),
                "power_w_max": pmax}


def pinned_h2d_gbps(device: int, nbytes: int = 1 << 30) -> float:
    """One page-locked host->device copy of ``nbytes``, timed with CUDA events
    (best of three): the link rate the end-to-end copies can reach."""
    import torch
    src = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    dst = torch.empty(nbytes, dtype=torch.uint8, device=f"cuda:{device}")
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        e1.synchronize()
        best = max(best, nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del src, dst
    return best


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


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:  # rank 0 alone times the host kernel
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


def train_band(eng, args, local_seed: int) -> dict:
    """Trains the band MLP on the GPU (or loads --weights) and installs it."""
    if args.weights:
        eng.band_load(args.weights)
        return {"weights": args.weights}
    # 1M pairs drawn from config 1's distribution (regions added until the pair count is reached)
    per_region = 5_388_348 / 4096
    n_reg = max(8, int(round(args.train_pairs / per_region)))
    tb = W.config1(seed=7000 + local_seed, n_regions=n_reg)
    rep = eng.band_train(tb, epochs=args.train_epochs, alpha=args.train_alpha, tau=args.train_tau,
                         seed=1234 + local_seed)
    rep["train_workload"] = tb.name
    return rep


def time_form(eng, batch, args, rep, band: bool):
    """Stages the batch once; returns per-step stats, device ms and results."""
    n = eng.stage(batch)
    for _ in range(args.warmup):
        eng.run()
    rep.barrier()
    steps = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        steps.append(eng.run())
    wall = time.perf_counter() - t0
    rep.barrier()
    res = eng.fetch(n)
    return n, steps, wall, res


def genotype_staged_timing(eng, batch) -> dict:
    """The device genotyper on the staged batch (the step after the PairHMM in
    HaplotypeCaller): two alleles per region, the first haplotype carrying the
    reference allele and the others the alternate, 90 % of reads overlapping
    the site (seeded)."""
    rng = np.random.default_rng(77)
    A = np.full(batch.n_regions, 2, np.int32)
    nh = np.diff(batch.region_haps)
    hap_allele = np.ones(batch.n_haps, np.int32)
    hap_allele[batch.region_haps[:-1][nh > 0]] = 0
    overlap = (rng.random(batch.n_reads) < 0.9).astype(np.uint8)
    eng.genotype_staged(batch, A, hap_allele, overlap)  # warm-up (table upload)
    t0 = time.perf_counter()
    out = eng.genotype_staged(batch, A, hap_allele, overlap)
    call = time.perf_counter() - t0
    return {"regions": int(batch.n_regions), "alleles_per_region": 2, "kernel_ms": out["kernel_ms"],
            "call_ms_with_d2h": call * 1e3, "kept_reads": int(out["kept_count"].sum()),
            "regions_per_s": batch.n_regions / (out["kernel_ms"] / 1e3) if out["kernel_ms"] > 0 else None}


def accuracy(batch, got_band, got_plain, n_sample: int, seed: int):
    """max / p99 |dlog10| against the FP64 oracle on a seeded sample of pairs."""
    from oracle.oracle import Oracle, TestcaseArray
    rng = np.random.default_rng(seed)
    sel = np.sort(rng.choice(batch.n_pairs, size=min(n_sample, batch.n_pairs), replace=False))
    truth = Oracle().log10_rescaled(TestcaseArray.for_batch(batch, sel=sel))
    out = {"oracle_sample_pairs": int(sel.size)}
    for name, got in (("band", got_band), ("plain", got_plain)):
        if got is None:
            continue
        g = got[sel]
        fin = np.isfinite(truth)
        err = np.abs(g[fin] - truth[fin])
        out[name] = {"max_abs_dlog10_vs_fp64_oracle": float(err.max(initial=0)),
                     "p99_abs_dlog10_vs_fp64_oracle": float(np.quantile(err, 0.99)) if err.size else 0.0,
                     "nonfinite_mismatch": int(np.sum(np.isfinite(g[~fin])) + np.sum(~np.isfinite(g[fin])))}
    if got_band is not None and got_plain is not None:
        both = np.isfinite(got_band) & np.isfinite(got_plain)
        d = np.abs(got_band[both] - got_plain[both])
        out["band_vs_full_dp_all_pairs"] = {"max": float(d.max(initial=0)),
                                            "p99": float(np.quantile(d, 0.99)) if d.size else 0.0,
                                            "over_1e-3": int(np.sum(d > 1e-3)), "pairs": int(both.sum())}
        nb, nf = normalized(batch, got_band), normalized(batch, got_plain)
        both = np.isfinite(nb) & np.isfinite(nf)
        d = np.abs(nb[both] - nf[both])
        out["band_vs_full_dp_normalized"] = {
            "what": "the call's result: each read's row capped at its best - 4.5 (PairHMM::normalize_likelihoods)",
            "max": float(d.max(initial=0)), "over_1e-3": int(np.sum(d > 1e-3)), "pairs": int(both.sum())}
    return out


def normalized(batch, lk):
    """Each read's likelihoods raised to at least the read's best - 4.5, as
    PairHMM::normalize_likelihoods (pairhmm.hpp:83-93) does to the call's result.
    Results are region by region, read-major: a read's haplotypes are contiguous."""
    nr = np.diff(batch.region_reads)
    nh = np.diff(batch.region_haps)
    per_read = np.repeat(nh, nr)
    keep = per_read > 0
    starts = np.concatenate([[0], np.cumsum(per_read)[:-1]])[keep]
    best = np.maximum.reduceat(lk, starts) if starts.size else np.zeros(0)
    cap = np.repeat(best - 4.5, per_read[keep])
    return np.maximum(lk, cap)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="config4")
    ap.add_argument("--form", choices=["band", "plain"], default=None,
                    help="band: learned band + batched (default for config4/config1); plain: full DP only")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--regions", type=int, default=0, help="config1/config4: fewer regions (profiling cases)")
    ap.add_argument("--ref-seconds", type=float, default=10.0, help="CPU seconds per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="band form only (profiling)")
    ap.add_argument("--haps-per-warp", type=int, default=0, help="0: engine default, 1 or 2")
    ap.add_argument("--train-pairs", type=int, default=1_000_000)
    ap.add_argument("--train-epochs", type=int, default=8)
    ap.add_argument("--train-alpha", type=float, default=16.0, help="MLP loss weight of a too-narrow band")
    ap.add_argument("--train-tau", type=float, default=1e-4, help="posterior threshold of the training labels")
    ap.add_argument("--weights", default="", help="load band MLP weights instead of training")
    ap.add_argument("--save-weights", default="", help="write the trained band MLP weights here")
    ap.add_argument("--audit-period", type=int, default=1024)
    ap.add_argument("--oracle-sample", type=int, default=20000)
    ap.add_argument("--edge-threshold", type=float, default=1e-3)
    ap.add_argument("--fixed-half", type=int, default=-1,
                    help=">= 0: band of seed diagonal +- this many diagonals (and the 11-mer extent), no MLP")
    ap.add_argument("--margin", type=int, default=2, help="diagonals added on both sides of the predicted band")
    ap.add_argument("--cap-margin", type=float, default=12.0,
                    help="banded pairs more than this many log10 units below their read's best are scored "
                         "again by the full DP (0: off)")
    ap.add_argument("--pipeline-chunks", type=int, default=0,
                    help="region chunks of the end-to-end call (0: the library default, one per 4M pairs; 1: one pass)")
    ap.add_argument("--per-base-gaps", action="store_true",
                    help="e2e: pass the per-base i, d, c arrays even when they are uniform")
    ap.add_argument("--tune-regions", type=int, default=500,
                    help="regions of the workload the launch-shape autotuner times (0: default shapes)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    form = args.form or ("band" if args.workload in ("config4", "config3", "config1") else "plain")

    rep = replicas.setup("nccl")
    world, rank, local = rep.world, rep.rank, rep.local
    from biovoltron_b200.native import load
    from biovoltron_b200.pairhmm import PairHMMEngine
    import ctypes as C

    t_gen = time.perf_counter()
    batch = make_workload(args.workload, rep.shard_seed(args.seed), args.regions)
    t_gen = time.perf_counter() - t_gen
    log(f"[rank {rank}] workload: {batch.name}: {batch.n_pairs} pairs, {batch.n_cells():.3e} cells "
        f"(generated in {t_gen:.1f} s)")
    lib = load()
    peak = C.c_double(0)
    st = lib.bv_phmm_measure_fp32_peak(local, C.byref(peak))
    fp32_peak = peak.value if st == 0 else None
    st = lib.bv_phmm_measure_fp64_peak(local, C.byref(peak))
    fp64_peak = peak.value if st == 0 else None

    plain = band = None
    train_rep = None
    tuning = None
    long_tuning = None
    if args.tune_regions > 0 and args.haps_per_warp == 0:
        # launch shapes per rows-per-lane bin, and the long-read kernel's warps per pair when the
        # workload has reads of 256 bases or more, timed on a seeded sample of the workload's regions
        picks = np.random.default_rng(5).choice(batch.n_regions, size=min(args.tune_regions, batch.n_regions),
                                                replace=False)
        sample = W.subsample_regions(batch, sorted(picks.tolist()))
        with PairHMMEngine(device=local) as et:
            tuning = et.autotune(sample, repeats=3)
            if sample.read_lengths().max() >= 256:
                long_tuning = et.autotune_long(sample, repeats=3)

    def configure(e):
        if tuning:
            e.set_tuning(tuning)
        if long_tuning:
            e.set_long_warps(long_tuning["warps_per_pair"])

    h2d_link = pinned_h2d_gbps(local)
    clocks = ClockSampler(local)  # sampled over every timed section below
    clocks.start()
    # ---- plain full DP, device-resident --------------------------------------
    if form == "plain" or not args.no_plain:
        with PairHMMEngine(device=local, haps_per_warp=args.haps_per_warp) as ep:
            configure(ep)
            n, steps, wall, res = time_form(ep, batch, args, rep, band=False)
        plain = {"n": n, "steps": steps, "wall": wall, "res": res}
    # ---- learned band, device-resident --------------------------------------
    eb = None
    geno = None
    if form == "band":
        eb = PairHMMEngine(device=local, haps_per_warp=args.haps_per_warp, pipeline_chunks=args.pipeline_chunks)
        configure(eb)
        train_rep = train_band(eb, args, rank)
        if args.save_weights and rank == 0:
            eb.band_save(args.save_weights)
        if args.fixed_half >= 0:  # seed-centred band of +-fixed_half diagonals instead of the MLP's
            eb.set_band_options(use_mlp=False, fixed_half=args.fixed_half, margin=args.margin,
                                edge_threshold=args.edge_threshold, audit_period=args.audit_period,
                                cap_margin=args.cap_margin)
        else:
            eb.set_band_options(use_mlp=True, margin=args.margin, edge_threshold=args.edge_threshold,
                                audit_period=args.audit_period, cap_margin=args.cap_margin)
        n, steps, wall, res = time_form(eb, batch, args, rep, band=True)
        band = {"n": n, "steps": steps, "wall": wall, "res": res}
        geno = genotype_staged_timing(eb, batch)
    main_run = band if band else plain
    n = main_run["n"]

    def device_ms(run):
        return [s_["ms_fp32"] + s_["ms_fp64"] for s_ in run["steps"]]

    # ---- end to end through the public API (host buffers) ---------------------
    if eb is not None:
        e2e_eng = eb
    else:
        e2e_eng = PairHMMEngine(device=local, haps_per_warp=args.haps_per_warp, pipeline_chunks=args.pipeline_chunks)
        configure(e2e_eng)
    # the caller's view of a SamRecord batch: when every read base has the same
    # gap-open and gap-continuation qualities they go as three bytes
    gaps = None if args.per_base_gaps else batch.uniform_gaps()
    arrays = [batch.read_bases, batch.read_q, batch.hap_bases, batch.read_offsets, batch.hap_offsets]
    if gaps is None:
        arrays += [batch.read_i, batch.read_d, batch.read_c]
    for a in arrays:
        e2e_eng.host_register(a)
    out = np.empty(max(n, 1), np.float64)
    e2e_eng.host_register(out)
    for _ in range(max(1, min(args.warmup, 2))):
        e2e_eng.compute_regions(batch, out=out, uniform_gaps=gaps)
    rep.barrier()
    e2e_t = []
    e2e_st = None
    for _ in range(args.steps):
        t1 = time.perf_counter()
        _, e2e_st = e2e_eng.compute_regions(batch, out=out, with_stats=True, uniform_gaps=gaps)
        e2e_t.append(time.perf_counter() - t1)
    h2d_bytes = int(sum(a.nbytes for a in arrays) + batch.region_reads.nbytes + batch.region_haps.nbytes)
    clk = clocks.stop()
    rep.barrier()
    for a in arrays + [out]:
        e2e_eng.host_unregister(a)
    same = bool(np.array_equal(out[:n], main_run["res"], equal_nan=True))
    e2e_eng.close()

    # ---- aggregate over ranks --------------------------------------------------
    agg = replicas.aggregate(rep, float(n * args.steps), [m / 1e3 for m in device_ms(main_run)])
    t_dev = agg["seconds"] * 1e3
    total_pairs = agg["pairs"]
    total_cells = rep.allreduce(float(batch.n_cells() * args.steps), "sum")
    value = agg["pairs_per_s"]
    e2e = replicas.aggregate(rep, float(n * args.steps), e2e_t)["pairs_per_s"]
    plain_pps = None
    if plain is not None:
        plain_pps = replicas.aggregate(rep, float(n * args.steps), [m / 1e3 for m in device_ms(plain)])["pairs_per_s"]

    acc = None
    cpu = None
    if rank == 0 and args.oracle_sample > 0:
        acc = accuracy(batch, band["res"] if band else None, plain["res"] if plain else None, args.oracle_sample,
                       seed=99)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(batch, target_s=args.ref_seconds)

    if rank == 0:
        def mean(run, key):
            return float(np.mean([s_[key] for s_ in run["steps"]]))

        last = main_run["steps"][-1]
        ms_step = t_dev / args.steps
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
            "gcups_effective": total_cells / (t_dev / 1e3) / 1e9,
            "config": {"workload": batch.name,
                       "form": ("learned band + batched (persistent length-binned launches, graph replay) + "
                                "FP32 with FP64 rescue") if band else "plain full DP, batched, FP32 with FP64 rescue",
                       "pairs_per_gpu": n, "cells_per_gpu": batch.n_cells(),
                       "l2": f"inputs {batch.nbytes() / 1e9:.2f} GB > 126 MB L2, no flush",
                       "parallelism": f"dp{world} (independent regions, one replica per GPU)",
                       "generate_s": round(t_gen, 1),
                       "launch_shapes": tuning or "engine defaults (2 haplotypes per warp, 4 warps per block)",
                       "long_read_kernel": long_tuning or "engine default (4 warps per pair, reads of 512 bases on)"},
        }
        if plain is not None:
            pl = plain["steps"][-1]
            ms_plain = float(np.mean(device_ms(plain)))
            # cells the FP32 kernels computed: a pair whose strip proves the FP32 result below the
            # rescue threshold goes to the FP64 pass without its remaining strips
            fp32_cells = batch.n_cells() - int(pl.get("fp32_skipped_cells", 0))
            ach = FLOPS_PER_CELL * fp32_cells / (mean(plain, "ms_full") / 1e3) / 1e12
            line["plain"] = {"value": plain_pps, "unit": "pairs/s", "ms_per_step": ms_plain,
                             "gcups": batch.n_cells() / (ms_plain / 1e3) / 1e9,
                             "rescued_per_step": pl["rescued"], "kernel_ms": {
                                 "fp32": mean(plain, "ms_full"), "fp64_rescue": mean(plain, "ms_fp64")}}
            line["roofline_plain"] = {"bound": "fp32", "kernel": "k_forward<float> (full DP, all variants)",
                                      "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s",
                                      "frac": (ach / fp32_peak) if fp32_peak else None,
                                      "flops_per_cell": FLOPS_PER_CELL, "cells": fp32_cells,
                                      "cells_left_to_fp64": batch.n_cells() - fp32_cells,
                                      "traffic": DRAM_BYTES_PER_PAIR_PLAIN * n if args.workload == "config4" else None,
                                      "traffic_source": TRAFFIC_SOURCE if args.workload == "config4" else None}
            if band is not None:
                line["speedup_vs_plain"] = value / plain_pps
        if band is not None:
            ms_band = mean(band, "ms_band")
            band_cells = int(last["band_cells"])
            result_cells = int(last["band_result_cells"])
            ach = FLOPS_PER_CELL * band_cells / (ms_band / 1e3) / 1e12 if ms_band > 0 else 0.0
            ach_result = FLOPS_PER_CELL * result_cells / (ms_band / 1e3) / 1e12 if ms_band > 0 else 0.0
            line["band"] = {
                "kernel_ms": {"seed_features_mlp_route": mean(band, "ms_seed"), "banded_dp": ms_band,
                              "fallback_full_dp": mean(band, "ms_full"), "fp64_rescue": mean(band, "ms_fp64")},
                "band_pairs": int(last["band_pairs"]), "routed_full": int(last["band_routed_full"]),
                "edge_fallback": int(last["band_fallback"]), "promoted": int(last["band_promoted"]),
                "fallback_rate": (int(last["band_routed_full"]) + int(last["band_fallback"])) / max(n, 1),
                # banded pairs far below their read's best, scored again by the full DP
                "rescored": int(last["band_rescored"]),
                "band_cells": band_cells, "band_result_cells": result_cells,
                # computed cells per second of the banded kernels (band + ring + inner band)
                "gcups_computed_banded_dp": band_cells / (ms_band / 1e3) / 1e9 if ms_band > 0 else None,
                "rescued": int(last["rescued"]),
                "audit_pairs": int(last["audit_pairs"]), "audit_max_err": float(last["audit_max_err"]),
                "audit_p99_err": float(last["audit_p99_err"]), "train": train_rep}
            line["roofline"] = {"bound": "fp32", "kernel": "k_band_ring_f32<W> (banded forward, band and ring, W = 8/16/24/32)",
                                "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s",
                                "frac": (ach / fp32_peak) if fp32_peak else None,
                                "cells_counted": "both sweeps: the result band (band + ring) and the inner band "
                                                 "the ring test recomputes",
                                "achieved_result_band": ach_result,
                                "frac_result_band": (ach_result / fp32_peak) if fp32_peak else None,
                                "flops_per_cell": FLOPS_PER_CELL,
                                "traffic": DRAM_BYTES_PER_BAND_PAIR * int(last["band_pairs"])
                                if args.workload == "config4" else None,
                                "traffic_source": TRAFFIC_SOURCE if args.workload == "config4" else None}
        else:
            line["roofline"] = line.get("roofline_plain")
        line["peak_source"] = ("measured: FP32 and FP64 FMA probe kernels in this run (bv_phmm_measure_fp32_peak, "
                               "bv_phmm_measure_fp64_peak); MEASURED_PEAKS.json holds HBM and bf16 tensor peaks only")
        fp64_ms = mean(main_run, "ms_fp64")
        fp64_cells = int(last["rescued_cells"])
        if fp64_cells > 0 and fp64_ms > 0:
            a64 = FLOPS_PER_CELL * fp64_cells / (fp64_ms / 1e3) / 1e12
            line["roofline_fp64"] = {"bound": "fp64",
                                     "kernel": "k_forward_long<4> (reads >= 512 bases, a block of four warps per "
                                               "pair) and k_forward<double, 4, multi-strip> (FP64 pass)",
                                     "achieved": a64, "peak": fp64_peak, "unit": "TFLOP/s",
                                     "frac": (a64 / fp64_peak) if fp64_peak else None,
                                     "cells": fp64_cells, "ms": fp64_ms, "flops_per_cell": FLOPS_PER_CELL}
            if band is None and fp64_ms > mean(main_run, "ms_full"):
                # the FP64 pass dominates the step (every pair rescued): the roofline is the FP64 kernels'
                line["roofline"] = line["roofline_fp64"]
        line["accuracy"] = acc
        if geno is not None:
            line["genotype"] = geno
        line["e2e"] = {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": h2d_bytes,
                       "pinned_h2d_gbps_one_copy": h2d_link,
                       "inputs": ("bases, base qualities and offsets; uniform gap penalties "
                                  f"(ins, del, gcp) = {gaps}") if gaps else "per-base q, i, d, c arrays",
                       "d2h_bytes_per_step": int(8 * n), "results_identical_to_device_run": same}
        if e2e_st is not None:
            # last step: copies (first H2D to packed qualities, events; they overlap the host's
            # planning), kernels (events), result D2H and the whole call (host clock)
            line["e2e"]["last_step_ms"] = {"h2d_and_pack": e2e_st["ms_h2d"],
                                           "kernels": e2e_st["ms_fp32"] + e2e_st["ms_fp64"],
                                           "d2h": e2e_st["ms_d2h"], "call": e2e_st["ms_total"]}
        line["gpu_launches"] = int(last["kernel_launches"]) * args.steps
        line["clocks"] = clk
        line["wall_s_timed"] = main_run["wall"]
        if cpu:
            line["cpu_baseline"] = {"value": cpu["pairs_per_s"], "unit": "pairs/s", "cores": cpu["cores"],
                                    "kind": cpu["kind"], "sample": cpu["sample"], "gcups": cpu["gcups"]}
        print(json.dumps(line), flush=True)
    rep.close()


if __name__ == "__main__":
    main()
