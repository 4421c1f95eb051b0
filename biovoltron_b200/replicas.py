"""Replica plumbing for runs over several GPUs of one node.

PairHMM pairs are independent, and ``normalize_likelihoods`` /
``filter_poorly_modeled_reads`` act per read inside one region
(include/biovoltron/algo/align/inexact_match/pairhmm.hpp:83-114), so a batch of
active regions splits across GPUs by region with no exchange of data: each
process drives one GPU and scores its own regions.  The only collectives are
scalar reductions of the per-rank counts and times (sum of pairs, max of
times) and barriers around the timed region, taken by every rank in the same
order.

One batch held by every rank is split with ``split_batch``: the same greedy
LPT partition the library's multi-device call uses (bv_phmm_plan_partition,
one region per block), so every rank computes the same plan without talking
to the others; ``gather_results`` puts the ranks' results back in region
order (one all-gather, after the scoring).
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np


@dataclass
class Replicas:
    world: int = 1
    rank: int = 0
    local: int = 0
    backend: Optional[str] = None  # None: single process, no process group

    @property
    def device(self) -> str:
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"

    def shard_seed(self, seed: int) -> int:
        """Seed of this rank's regions: every rank draws its own independent batch."""
        return seed + 1000 * self.rank

    def allreduce(self, x: float, op: str) -> float:
        if self.backend is None:
            return float(x)
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op={"max": dist.ReduceOp.MAX, "sum": dist.ReduceOp.SUM}[op])
        return float(t.item())

    def barrier(self) -> None:
        if self.backend is not None:
            import torch.distributed as dist
            dist.barrier()

    def close(self) -> None:
        if self.backend is not None:
            import torch.distributed as dist
            dist.destroy_process_group()
            self.backend = None


def setup(backend: str = "nccl", timeout_s: float = 300.0) -> Replicas:
    """Joins the process group that torchrun's environment describes (one rank
    per GPU); a single process (WORLD_SIZE unset or 1) gets no group."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Replicas(1, 0, local, None)
    import torch
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, **kw)
    return Replicas(world, rank, local, backend)


def aggregate(rep: Replicas, pairs: float, seconds: Sequence[float]) -> dict:
    """Whole-job throughput: the pairs all ranks scored over the slowest rank's
    time (each rank's time is the sum of its timed steps)."""
    total = rep.allreduce(pairs, "sum")
    t = rep.allreduce(float(sum(seconds)), "max")
    return {"pairs": total, "seconds": t, "pairs_per_s": total / t if t > 0 else 0.0}


def split_batch(rep: Replicas, batch) -> Tuple[object, np.ndarray]:
    """This rank's share of ``batch`` (regions dealt by greedy LPT on their DP
    cells, in region order) and the batch-wide result slots of the share's
    results, in the share's result order."""
    from .pairhmm import plan_partition, regions_of_part
    from .workloads import subsample_regions
    bs, bp, _ = plan_partition(batch, rep.world)
    regions = regions_of_part(bs, bp, rep.rank)
    offs = batch.result_offsets()
    slots = np.concatenate([np.arange(offs[g], offs[g + 1]) for g in regions] or [np.zeros(0, np.int64)])
    return subsample_regions(batch, regions.tolist()), slots.astype(np.int64)


def gather_results(rep: Replicas, local: np.ndarray, slots: np.ndarray, n_total: int) -> np.ndarray:
    """Every rank's results at their batch-wide slots: the whole batch's
    result array, on every rank."""
    out = np.full(n_total, np.nan, np.float64)
    if rep.backend is None:
        out[slots] = local
        return out
    import torch.distributed as dist
    parts = [None] * rep.world
    dist.all_gather_object(parts, (np.asarray(slots, np.int64), np.asarray(local, np.float64)))
    for sl, val in parts:
        out[sl] = val
    return out
