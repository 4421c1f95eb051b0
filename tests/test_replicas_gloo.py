"""Multi-rank host logic on CPU: two gloo ranks, each with its own seeded
batch of regions, scored by the oracle; throughput aggregated as the bench
does (pairs summed over ranks, the slowest rank's time)."""
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
