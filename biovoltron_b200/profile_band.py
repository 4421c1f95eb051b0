"""Runs the band path once on a seeded config-1-shaped batch (profiling case).

    python -m biovoltron_b200.profile_band --regions 512 --half 6 --threshold 1e-2

Prints the run's statistics as one JSON line; used under ncu to list the
band pipeline's kernels.
"""
import argparse
import json

from . import workloads as W
from .pairhmm import PairHMMEngine


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--regions", type=int, default=512)
    ap.add_argument("--half", type=int, default=6)
    ap.add_argument("--threshold", type=float, default=1e-2)
    ap.add_argument("--runs", type=int, default=2)
    a = ap.parse_args()
    b = W.config1(seed=1, n_regions=a.regions)
    with PairHMMEngine() as e:
        e.set_band_options(fixed_half=a.half, margin=2, edge_threshold=a.threshold)
        e.stage(b)
        st = None
        for _ in range(a.runs):
            st = e.run()
    print(json.dumps(st))


if __name__ == "__main__":
    main()
