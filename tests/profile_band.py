"""Runs the band path on a seeded batch (timing and profiling case).

    python tests/profile_band.py --workload config1 --regions 512 \
        --weights band.bvw --threshold 1e-3 --runs 3

With --weights the learned band is used (--train-regions > 0 trains and
saves them first, on a batch of its own seed); without, the fixed band of
half-width --half.  Prints per-run statistics and the full-DP time of the
same batch as JSON lines; used under ncu to list the band pipeline's kernels.
"""
import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from biovoltron_b200 import workloads as W  # noqa: E402
from biovoltron_b200.pairhmm import PairHMMEngine  # noqa: E402


def _batch(workload: str, regions: int, seed: int):
    if workload == "config4":
        return W.config4(seed=seed, n_regions=regions)
    if workload == "config2":  # long pairs: `regions` pairs
        return W.config2(seed=seed, n_pairs=regions)
    return W.config1(seed=seed, n_regions=regions)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="config1", choices=["config1", "config2", "config4"])
    ap.add_argument("--regions", type=int, default=512)
    ap.add_argument("--half", type=int, default=6)
    ap.add_argument("--margin", type=int, default=2)
    ap.add_argument("--threshold", type=float, default=1e-3)
    ap.add_argument("--cap-margin", type=float, default=12.0,
                    help="rescore banded pairs this many log10 units below their read's best (0: off)")
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--weights", default="")
    ap.add_argument("--train-regions", type=int, default=0)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--full", action="store_true", help="also time the full DP on the same batch")
    ap.add_argument("--plain-only", action="store_true", help="only the full DP (FP32 with FP64 rescue)")
    a = ap.parse_args()
    if a.weights and a.train_regions > 0:
        with PairHMMEngine() as e:
            rep = e.band_train(_batch(a.workload, a.train_regions, 1000), epochs=a.epochs)
            e.band_save(a.weights)
        print(json.dumps({"train": rep}))
    b = _batch(a.workload, a.regions, 1)
    print(json.dumps({"pairs": b.n_pairs, "cells": b.n_cells()}))
    if a.plain_only:
        with PairHMMEngine() as e:
            e.stage(b)
            for _ in range(a.runs):
                print(json.dumps({"full": e.run()}))
        return
    with PairHMMEngine() as e:
        use_mlp = bool(a.weights) and os.path.exists(a.weights)
        if use_mlp:
            e.band_load(a.weights)
        e.set_band_options(use_mlp=use_mlp, fixed_half=a.half, margin=a.margin, edge_threshold=a.threshold,
                           cap_margin=a.cap_margin)
        e.stage(b)
        for _ in range(a.runs):
            print(json.dumps({"band": e.run()}))
    if a.full:
        with PairHMMEngine() as e:
            e.stage(b)
            for _ in range(a.runs):
                print(json.dumps({"full": e.run()}))


if __name__ == "__main__":
    main()
