"""Multi-rank host logic on CPU: two gloo ranks, each with its own seeded
batch of regions, scored by the oracle; throughput aggregated as the bench
does (pairs summed over ranks, the slowest rank's time).  And one batch split
over two gloo ranks by the library's LPT partition, each rank scoring its
share with the oracle standing in for its GPU: the gathered result equals
the one-rank result, in region order."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys, time
sys.path.insert(0, os.environ["BV_ROOT"])
import numpy as np
from biovoltron_b200 import replicas, workloads as W
from oracle.oracle import Oracle, TestcaseArray

rep = replicas.setup("gloo", timeout_s=60)
batch = W.config1(seed=rep.shard_seed(11), n_regions=3)
res = Oracle().log10_reference_rule(TestcaseArray.for_batch(batch))
rep.barrier()
fake_seconds = [0.25 * (rep.rank + 1), 0.5]  # per-step times this rank reports
agg = replicas.aggregate(rep, float(batch.n_pairs), fake_seconds)
out = {"rank": rep.rank, "world": rep.world, "seed": rep.shard_seed(11), "pairs": batch.n_pairs,
       "checksum": float(np.nansum(res)), "agg": agg}
rep.close()
with open(os.path.join(os.environ["BV_OUT"], f"rank{out['rank']}.json"), "w") as f:
    json.dump(out, f)
"""


SPLIT_WORKER = r"""
import json, os, sys
sys.path.insert(0, os.environ["BV_ROOT"])
import numpy as np
from biovoltron_b200 import replicas, workloads as W
from oracle.oracle import Oracle, TestcaseArray

rep = replicas.setup("gloo", timeout_s=60)
batch = W.config1(seed=17, n_regions=9)  # the same batch on every rank
share, slots = replicas.split_batch(rep, batch)
local = Oracle().log10_reference_rule(TestcaseArray.for_batch(share))[0]
full = replicas.gather_results(rep, local, slots, batch.n_pairs)
np.save(os.path.join(os.environ["BV_OUT"], f"split{rep.rank}.npy"), full)
with open(os.path.join(os.environ["BV_OUT"], f"split{rep.rank}.json"), "w") as f:
    json.dump({"regions": int(share.n_regions), "pairs": int(share.n_pairs), "cells": int(share.n_cells())}, f)
rep.close()
"""


def _run_ranks(code, tmp_path, n=2):
    port = _free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, BV_ROOT=ROOT, BV_OUT=str(tmp_path), WORLD_SIZE=str(n), RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    for p in procs:
        try:
            out, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("gloo ranks did not finish")
        assert p.returncode == 0, out


def test_one_batch_split_over_two_gloo_ranks_equals_one_rank(tmp_path):
    pytest.importorskip("torch.distributed")
    from biovoltron_b200 import workloads as W
    from oracle.oracle import Oracle, TestcaseArray
    _run_ranks(SPLIT_WORKER, tmp_path)
    batch = W.config1(seed=17, n_regions=9)
    want = Oracle().log10_reference_rule(TestcaseArray.for_batch(batch))[0]
    parts = [json.load(open(tmp_path / f"split{r}.json")) for r in range(2)]
    assert sum(p["regions"] for p in parts) == batch.n_regions
    assert sum(p["pairs"] for p in parts) == batch.n_pairs and min(p["pairs"] for p in parts) > 0
    for r in range(2):
        got = np.load(tmp_path / f"split{r}.npy")
        assert np.array_equal(got, want)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_regions_and_aggregate(tmp_path):
    pytest.importorskip("torch.distributed")
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, BV_ROOT=ROOT, BV_OUT=str(tmp_path), WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    for p in procs:
        try:
            out, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("gloo ranks did not finish")
        assert p.returncode == 0, out
    ranks = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert [x["world"] for x in ranks] == [2, 2]
    # each rank scored its own, different regions
    assert ranks[0]["seed"] != ranks[1]["seed"]
    assert ranks[0]["checksum"] != ranks[1]["checksum"]
    total = ranks[0]["pairs"] + ranks[1]["pairs"]
    for x in ranks:
        assert x["agg"]["pairs"] == total
        assert x["agg"]["seconds"] == pytest.approx(1.0)  # max over ranks of (0.25 (r + 1) + 0.5)
        assert x["agg"]["pairs_per_s"] == pytest.approx(total / 1.0)


def test_single_process_has_no_group(monkeypatch):
    from biovoltron_b200 import replicas
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    rep = replicas.setup("nccl")
    assert rep.backend is None and rep.world == 1
    assert rep.shard_seed(5) == 5
    agg = replicas.aggregate(rep, 10.0, [1.0, 1.0])
    assert agg == {"pairs": 10.0, "seconds": 2.0, "pairs_per_s": 5.0}
    rep.barrier()
    rep.close()
    assert np.isfinite(agg["pairs_per_s"])
