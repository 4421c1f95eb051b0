import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from biovoltron_b200 import workloads as W  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
FIXTURES = ("config0", "edge_cases", "ref_test", "long_pairs", "config4_small")
BATCH_FIELDS = ("read_bases", "read_q", "read_i", "read_d", "read_c", "read_offsets", "hap_bases", "hap_offsets",
                "region_reads", "region_haps")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built native library")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    b = W.RegionBatch(**{k: z[k] for k in BATCH_FIELDS}, name=name)
    exp = {k: z[k] for k in z.files if k not in BATCH_FIELDS}
    return b, exp


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference kernel not built (oracle/_ref)")
    return Reference()


@pytest.fixture(scope="session")
def engine():
    from biovoltron_b200.pairhmm import PairHMMEngine
    e = PairHMMEngine(device=0)
    yield e
    e.close()
