"""The C++20 adapter header compiles against the C ABI and, on a GPU, gives
the same [read][hap] matrix and read filtering as the Python mirror."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
SRC = os.path.join(ROOT, "tests", "cpp", "adapter_check.cpp")
LIBDIR = os.path.join(ROOT, "biovoltron_b200", "_native")
EXE = os.path.join(ROOT, "tests", "cpp", "_build", "adapter_check")


def _run(args, txt):
    """Runs the adapter check program; its stderr is shown when it fails."""
    p = subprocess.run([EXE] + args, input=txt, capture_output=True, text=True)
    assert p.returncode == 0, f"adapter_check {args} exited {p.returncode}: {p.stderr[-2000:]}"
    return p.stdout.splitlines()


def _build():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), SRC, "-o", EXE,
           "-L" + LIBDIR, "-lbv_pairhmm", "-Wl,-rpath," + LIBDIR]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


@pytest.mark.skipif(not os.path.exists(os.path.join(LIBDIR, "libbv_pairhmm.so")), reason="native library not built")
def test_adapter_compiles_and_links():
    _build()
    assert os.path.exists(EXE)


@pytest.mark.gpu
def test_adapter_matches_python_mirror(engine):
    from biovoltron_b200 import workloads as W
    from biovoltron_b200.pairhmm import GpuPairHMM, Haplotype, SamRecord
    _build()
    rng = np.random.default_rng(12)
    base = bytes(W._random_seq(rng, 500))
    haps = [base, base[:250] + b"G" + base[251:], bytes(W._random_seq(rng, 480))]
    reads = [(base[100:250], bytes(rng.integers(43, 74, size=150).astype(np.uint8))),
             (base[200:260], b"5" * 60), (bytes(W._random_seq(rng, 90)), b"+" * 90),
             (base[0:200], b";" * 200)]
    txt = "".join(f"H {h.decode()}\n" for h in haps) + "".join(f"R {s.decode()} {q.decode()}\n" for s, q in reads)
    out = _run([], txt)
    kept = [int(x) for x in out[0].split()[1:]]
    mat = [[float(x) for x in l.split()] for l in out[1:]]
    py_reads = [SamRecord(s, q) for s, q in reads]
    ids = {id(r): k for k, r in enumerate(py_reads)}
    ll = GpuPairHMM(engine=engine).compute_likelihoods([Haplotype(h) for h in haps], py_reads)
    assert kept == [ids[id(r)] for r in py_reads]
    assert np.allclose(np.array(mat), np.array(ll), rtol=0, atol=1e-8)


@pytest.mark.gpu
def test_scalar_adapter_matches_python_mirror():
    from biovoltron_b200 import workloads as W
    from biovoltron_b200.pairhmm import GpuScalarPairHMM, Haplotype, SamRecord
    _build()
    rng = np.random.default_rng(13)
    base = bytes(W._random_seq(rng, 400))
    haps = [base, base[:200] + b"A" + base[201:]]
    reads = [(base[50:200], bytes(rng.integers(43, 74, size=150).astype(np.uint8))),
             (bytes(W._random_seq(rng, 70)), b"+" * 70), (base[100:180], b"5" * 80)]
    txt = "".join(f"H {h.decode()}\n" for h in haps) + "".join(f"R {s.decode()} {q.decode()}\n" for s, q in reads)
    out = _run(["scalar"], txt)
    kept = [int(x) for x in out[0].split()[1:]]
    mat = [[float(x) for x in l.split()] for l in out[1:]]
    py_reads = [SamRecord(s, q) for s, q in reads]
    ids = {id(r): k for k, r in enumerate(py_reads)}
    ll = GpuScalarPairHMM().compute_likelihoods([Haplotype(h) for h in haps], py_reads)
    assert kept == [ids[id(r)] for r in py_reads]
    assert np.allclose(np.array(mat), np.array(ll), rtol=0, atol=1e-8)


@pytest.mark.gpu
def test_region_batcher_adapter_matches_one_call():
    from biovoltron_b200 import workloads as W
    _build()
    rng = np.random.default_rng(14)
    base = bytes(W._random_seq(rng, 400))
    haps = [base, base[:220] + b"C" + base[221:], bytes(W._random_seq(rng, 350))]
    reads = [(base[30:180], bytes(rng.integers(43, 74, size=150).astype(np.uint8))),
             (bytes(W._random_seq(rng, 70)), b"+" * 70), (base[150:250], b"5" * 100)]
    txt = "".join(f"H {h.decode()}\n" for h in haps) + "".join(f"R {s.decode()} {q.decode()}\n" for s, q in reads)
    one = _run([], txt)
    two = _run(["batch"], txt)
    n = len(one)
    assert len(two) == 2 * n
    assert two[:n] == one and two[n:] == one
