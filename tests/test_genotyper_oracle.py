"""The genotyper steps after the PairHMM (normalise, filter, overlap
selection, marginalisation, diploid genotype likelihoods): the CPU
restatement is pinned to Biovoltron's own genotyper code compiled here
(oracle/_ref/libref_genotyper.so) bit for bit, and the product's Jacobian log
table equals the reference's."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import genotyper as OG

REF = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libref_genotyper.so")


def _ref():
    if not os.path.exists(REF):
        pytest.skip("reference genotyper not built (oracle/_ref)")
    L = C.CDLL(REF)
    L.ref_jacobian_table.restype = C.c_int
    L.ref_jacobian_table.argtypes = [C.c_void_p, C.c_int]
    L.ref_approximate_log10_sum_log10.restype = C.c_double
    L.ref_approximate_log10_sum_log10.argtypes = [C.c_double, C.c_double]
    L.ref_genotype.restype = C.c_int
    L.ref_genotype.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]
    return L


def _ref_table(L):
    n = L.ref_jacobian_table(None, 0)
    t = np.zeros(n)
    L.ref_jacobian_table(t.ctypes.data, n)
    return t


def test_oracle_table_equals_reference():
    L = _ref()
    assert np.array_equal(np.array(OG.jacobian_table()), _ref_table(L))


def test_product_table_equals_reference():
    from biovoltron_b200.native import load
    lib = load()
    L = _ref()
    ref = _ref_table(L)
    n = lib.bv_phmm_debug_jacobian_table(None, 0)
    t = np.zeros(n)
    lib.bv_phmm_debug_jacobian_table(t.ctypes.data, n)
    assert n == len(ref) and np.array_equal(t, ref)


def test_approximate_sum_equals_reference():
    L = _ref()
    rng = np.random.default_rng(4)
    for a, b in list(rng.normal(-10, 5, (300, 2))) + [(-1.0, -1.0), (-3.0, -11.5), (-np.inf, -2.0),
                                                      (-1.7976931348623157e308, -1.0)]:
        assert OG.approximate_log10_sum_log10(float(a), float(b)) == L.ref_approximate_log10_sum_log10(a, b)


def random_window(rng, nr, nh):
    ll = rng.normal(-8, 4, (nr, nh))
    ll[rng.random((nr, nh)) < 0.05] = -np.inf
    read_len = rng.integers(20, 250, nr).astype(np.int32)
    overlap = (rng.random(nr) < 0.8).astype(np.uint8)
    A = int(rng.integers(1, 5))
    hap_allele = rng.integers(0, A, nh).astype(np.uint32)
    return ll, read_len, overlap, A, hap_allele


@pytest.mark.parametrize("seed", range(6))
def test_oracle_genotype_equals_reference(seed):
    L = _ref()
    rng = np.random.default_rng(seed)
    for _ in range(20):
        nr, nh = int(rng.integers(1, 40)), int(rng.integers(1, 10))
        ll, read_len, overlap, A, hap_allele = random_window(rng, nr, nh)
        kept_r = np.zeros(nr, np.int32)
        al_r = np.zeros(nr * A)
        ge_r = np.zeros(A * (A + 1) // 2)
        llc = np.ascontiguousarray(ll)
        k = L.ref_genotype(nr, nh, llc.ctypes.data, read_len.ctypes.data, overlap.ctypes.data, A,
                           hap_allele.ctypes.data, kept_r.ctypes.data, al_r.ctypes.data, ge_r.ctypes.data)
        kept, al, ge = OG.genotype_window(ll.tolist(), read_len.tolist(), overlap.tolist(), A, hap_allele.tolist())
        assert kept == kept_r[:k].tolist()
        assert np.array_equal(np.array(al).reshape(-1), al_r[:k * A])
        assert np.array_equal(np.array(ge), ge_r)
