"""The CPU oracle is pinned to Biovoltron's own PairHMM kernel.

* Against the committed golden vectors (produced by the reference kernel,
  tests/golden/make_golden.py): the oracle's FP32 and FP64 probabilities are
  bit-identical and its log10 under the rescue rule is identical.
* Against the reference kernel itself, live, where oracle/_ref is built.
* The scalar PairHMM model's restatement against Biovoltron's scalar
  PairHMM (golden vectors and, where built, live).
* The rescaled FP64 variant agrees with the plain FP64 wherever that is finite.
* Hand-computable cases.
"""
import math

import numpy as np
import pytest

from biovoltron_b200 import workloads as W
from conftest import FIXTURES, load_golden
from oracle.oracle import TestcaseArray


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.array_equal(a, b) or np.array_equal(np.nan_to_num(a, nan=1e300), np.nan_to_num(b, nan=1e300))


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_bit_exact_vs_golden(name, oracle):
    b, exp = load_golden(name)
    tcs = TestcaseArray.for_batch(b)
    pf = oracle.prob_f32(tcs)
    pd = oracle.prob_f64(tcs)
    assert np.array_equal(pf.view(np.uint32), exp["ref_prob_f32"].view(np.uint32))
    assert np.array_equal(pd.view(np.uint64), exp["ref_prob_f64"].view(np.uint64))
    lg, used = oracle.log10_reference_rule(tcs)
    assert _same(lg, exp["ref_log10"])
    assert np.array_equal(used, exp["ref_used_f64"])


@pytest.mark.parametrize("name", FIXTURES)
def test_rescaled_oracle_vs_golden(name, oracle):
    b, exp = load_golden(name)
    tcs = TestcaseArray.for_batch(b)
    rs = oracle.log10_rescaled(tcs)
    assert _same(rs, exp["oracle_rescaled"])
    ref = exp["ref_log10"]
    fin = np.isfinite(ref)
    # FP32-path values differ from the FP64 truth by single-precision rounding only
    assert np.max(np.abs(rs[fin] - ref[fin])) < 5e-5


def test_tables_identical_to_reference(oracle, reference):
    a, b = oracle.tables(), reference.tables()
    for k in a:
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k


def test_product_tables_identical_to_reference(reference):
    """The tables the CUDA path uploads are built by the product's own host
    code (phmm_tables.cpp); compare them with the reference's statics."""
    import ctypes as C
    import os
    so = os.path.join(os.path.dirname(__file__), "..", "biovoltron_b200", "_native", "libbv_pairhmm.so")
    if not os.path.exists(so):
        pytest.skip("native library not built")
    from biovoltron_b200.native import load
    lib = load()
    fn = lib.bv_phmm_debug_tables
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    n = 127 * 128 // 2 + 127 + 1
    pf = np.zeros(128, np.float32); pd = np.zeros(128, np.float64)
    mf = np.zeros(n, np.float32); md = np.zeros(n, np.float64)
    assert fn(pf.ctypes.data, pd.ctypes.data, mf.ctypes.data, md.ctypes.data, n) == 0
    r = reference.tables()
    assert np.array_equal(pf.view(np.uint32), r["ph2pr_f32"].view(np.uint32))
    assert np.array_equal(pd.view(np.uint64), r["ph2pr_f64"].view(np.uint64))
    assert np.array_equal(mf.view(np.uint32), r["mm_f32"][:n].view(np.uint32))
    assert np.array_equal(md.view(np.uint64), r["mm_f64"][:n].view(np.uint64))


def test_oracle_bit_exact_vs_live_reference(oracle, reference):
    b = W.config1(seed=123, n_regions=12)
    tcs = TestcaseArray.for_batch(b)
    assert np.array_equal(oracle.prob_f32(tcs).view(np.uint32), reference.prob_f32(tcs).view(np.uint32))
    lo, uo = oracle.log10_reference_rule(tcs)
    lr, ur = reference.log10(tcs)
    assert _same(lo, lr)
    assert np.array_equal(uo, ur)


def test_one_by_one_known_answers(oracle):
    # M(1,1) = e * pGAPM * Y(0,0), Y(0,0) = INITIAL/1; X(1,1) = 0
    # => L = e * (1 - 10^-c/10); e = 1 - 10^-q/10 (match) or 10^-q/10 / 3.
    q, c = 30, 10
    b = W.from_pairs([(b"A", bytes([q]), bytes([45]), bytes([45]), bytes([c]), b"A"),
                      (b"A", bytes([q]), bytes([45]), bytes([45]), bytes([c]), b"G"),
                      (b"N", bytes([q]), bytes([45]), bytes([45]), bytes([c]), b"G"),
                      (b"T", bytes([q]), bytes([45]), bytes([45]), bytes([c]), b"N")])
    tcs = TestcaseArray.for_batch(b)
    got = oracle.log10_rescaled(tcs)
    eps = 10 ** (-q / 10)
    gp = 1 - 10 ** (-c / 10)
    exp = [math.log10((1 - eps) * gp), math.log10(eps / 3 * gp), math.log10((1 - eps) * gp),
           math.log10((1 - eps) * gp)]
    assert np.allclose(got, exp, rtol=0, atol=1e-12)


def test_identical_read_scores_near_uniform_start(oracle):
    # A read equal to a window of the haplotype at Q40: the likelihood is
    # dominated by the single exact placement, ~ prod(1-eps) * pMM^(n-1) *
    # pGAPM / H.
    rng = np.random.default_rng(3)
    hap = bytes(W._random_seq(rng, 300))
    read = hap[100:200]
    n = len(read)
    b = W.from_pairs([(read, bytes([40]) * n, bytes([45]) * n, bytes([45]) * n, bytes([10]) * n, hap)])
    got = oracle.log10_rescaled(TestcaseArray.for_batch(b))[0]
    eps = 1e-4
    tab = oracle.tables()
    pmm = float(tab["mm_f64"][45 * 46 // 2 + 45])
    approx = n * math.log10(1 - eps) + (n - 1) * math.log10(pmm) + math.log10(0.9 / 300)
    assert abs(got - approx) < 1e-3


def _scalar_pairs(b):
    r, h = b.pair_index()
    ro, ho = b.read_offsets, b.hap_offsets
    for k in range(len(r)):
        yield (bytes(b.read_bases[ro[r[k]]:ro[r[k] + 1]]), bytes(b.read_q[ro[r[k]]:ro[r[k] + 1]]),
               bytes(b.hap_bases[ho[h[k]]:ho[h[k] + 1]]))


def test_scalar_oracle_bit_exact_vs_golden(oracle):
    """The scalar model's restatement equals Biovoltron's scalar PairHMM
    (pairhmm.hpp:56-80, compiled from the reference) bit for bit, with the
    default and with a custom transition matrix."""
    b, exp = load_golden("scalar")
    trans = [float(x) for x in exp["custom_trans"]]
    got_d = [oracle.scalar_log10(rd, q, hp) for rd, q, hp in _scalar_pairs(b)]
    got_c = [oracle.scalar_log10(rd, q, hp, trans) for rd, q, hp in _scalar_pairs(b)]
    assert _same(got_d, exp["ref_scalar_default"])
    assert _same(got_c, exp["ref_scalar_custom"])


def test_scalar_oracle_bit_exact_vs_live_reference(oracle):
    from oracle.oracle import ReferenceScalar
    if not ReferenceScalar.available():
        pytest.skip("reference scalar model not built (oracle/_ref)")
    ref = ReferenceScalar()
    rng = np.random.default_rng(3)
    for k in range(200):
        rl, hl = int(rng.integers(1, 120)), int(rng.integers(1, 200))
        rd = bytes(rng.choice(list(b"ACGTN"), rl, p=[.24, .24, .24, .24, .04]).astype(np.uint8))
        hp = bytes(rng.choice(list(b"ACGTN"), hl, p=[.24, .24, .24, .24, .04]).astype(np.uint8))
        q = bytes(rng.integers(0, 128, rl).astype(np.uint8))
        tr = None if k % 2 else [0.99, 0.005, 0.005, 0.8, 0.2, 0.7, 0.3]
        assert _same(oracle.scalar_log10(rd, q, hp, tr), ref.log10(rd, q, hp, tr))
