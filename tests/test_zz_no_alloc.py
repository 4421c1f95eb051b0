"""The allocation-free entry point bv_phmm_forward_f64_noalloc.

It serves callers that cannot allocate device memory when they score pairs
(their framework's allocator owns the GPU's memory, or a policy forbids new
allocations), so it writes into caller-provided device memory and uses only a
fixed scratch array compiled into the library.  This test calls it through the
C ABI with device buffers that the test itself owns, twice in a row, and
checks both outputs against the allocating entry point (bv_phmm_compute_regions
with FP64 precision, the same arithmetic) within the FP64 tolerance the other
tests use; it also checks that a call after the first reserves no device memory, that
an over-long haplotype bound is rejected, and that pairs the kernel's own
bounds checks refuse (a haplotype longer than the maximum, a haplotype index
out of range) get NaN while the others are still scored.
It lives in its own file so pytest collects it after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from biovoltron_b200 import native as N
from biovoltron_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-9


class DevicePairs(C.Structure):
    _fields_ = [("num_pairs", C.c_int64), ("pairs", C.c_void_p), ("num_reads", C.c_int64),
                ("read_offsets", C.c_void_p), ("read_bases", C.c_void_p), ("read_quals", C.c_void_p),
                ("num_haps", C.c_int64), ("hap_offsets", C.c_void_p), ("hap_bases", C.c_void_p),
                ("max_hap_len", C.c_int32)]


def _batch():
    rng = np.random.default_rng(5)
    base = W.config0(3)
    extra = []
    for n, hl in ((300, 900), (600, 2000), (40, 120)):  # multi-strip reads, long haplotype, short pair
        hap = bytes(W._random_seq(rng, hl))
        read = bytes(W._substitute(rng, np.frombuffer(hap[50:50 + n], np.uint8), 0.03))
        q = bytes(rng.integers(10, 41, size=n).astype(np.uint8))
        extra.append((read, q, bytes([45]) * n, bytes([45]) * n, bytes([10]) * n, hap))
    ex = W.from_pairs(extra)
    parts = []
    for b in (base, ex):
        for g in range(b.n_regions):
            r0, r1 = int(b.region_reads[g]), int(b.region_reads[g + 1])
            h0, h1 = int(b.region_haps[g]), int(b.region_haps[g + 1])
            reads = [tuple(np.frombuffer(x, np.uint8) for x in b.read(k)) for k in range(r0, r1)]
            haps = [np.frombuffer(b.hap(k), np.uint8) for k in range(h0, h1)]
            parts.append((reads, haps))
    return W._build(parts, "no-alloc check")


def test_noalloc_matches_allocating_entry_point():
    import torch
    from biovoltron_b200.pairhmm import PairHMMEngine

    lib = N.load()
    fn = lib.bv_phmm_forward_f64_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.POINTER(DevicePairs), C.c_void_p, C.c_int64, C.c_void_p]

    b = _batch()
    with PairHMMEngine(device=0, precision="f64") as eng:
        expect = eng.compute_regions(b)

    dev = torch.device("cuda", 0)
    r, h = b.pair_index()
    pairs = np.zeros(len(r), dtype=[("read", np.int32), ("hap", np.int32), ("out", np.int64)])
    pairs["read"], pairs["hap"], pairs["out"] = r, h, np.arange(len(r))
    quals = np.stack([b.read_q, b.read_i, b.read_d, b.read_c], axis=1).reshape(-1)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in dict(
        pairs=pairs.view(np.uint8), read_offsets=b.read_offsets.astype(np.int64), read_bases=b.read_bases,
        read_quals=quals, hap_offsets=b.hap_offsets.astype(np.int64), hap_bases=b.hap_bases).items()}
    out = torch.full((len(r),), float("nan"), dtype=torch.float64, device=dev)
    dp = DevicePairs(num_pairs=len(r), pairs=t["pairs"].data_ptr(), num_reads=b.n_reads,
                     read_offsets=t["read_offsets"].data_ptr(), read_bases=t["read_bases"].data_ptr(),
                     read_quals=t["read_quals"].data_ptr(), num_haps=b.n_haps,
                     hap_offsets=t["hap_offsets"].data_ptr(), hap_bases=t["hap_bases"].data_ptr(),
                     max_hap_len=int(b.hap_lengths().max()))
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize(dev)
    results = []
    free = []
    for _ in range(2):  # two calls in a row share the scratch array
        out.fill_(float("nan"))
        torch.cuda.synchronize(dev)
        free.append(torch.cuda.mem_get_info(dev)[0])
        assert fn(0, C.byref(dp), out.data_ptr(), len(r), stream) == N.BV_OK
        free.append(torch.cuda.mem_get_info(dev)[0])
        results.append(out.cpu().numpy().copy())
    # after the first call on the device (module load, set-up) a call reserves no device memory
    assert free[3] == free[2], free
    for got in results:
        fin = np.isfinite(expect)
        assert np.array_equal(np.isneginf(got), np.isneginf(expect))
        assert np.all(np.isfinite(got[fin]))
        assert np.max(np.abs(got[fin] - expect[fin])) <= TOL_F64

    dp.max_hap_len = N_MAX + 1
    assert fn(0, C.byref(dp), out.data_ptr(), len(r), stream) == N.BV_ERR_INVALID_ARG


N_MAX = 2048  # BV_PHMM_NOALLOC_MAX_HAP_LEN


def test_noalloc_device_checks_flag_bad_pairs():
    """A pair whose haplotype is longer than the maximum (the caller's stated
    bound notwithstanding) and a pair whose haplotype index is out of range
    are skipped by the kernel's bounds checks: their slots read NaN, the call
    returns BV_ERR_INVALID_ARG, and the valid pairs match the allocating
    entry point."""
    import torch
    from biovoltron_b200.pairhmm import PairHMMEngine

    lib = N.load()
    fn = lib.bv_phmm_forward_f64_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.POINTER(DevicePairs), C.c_void_p, C.c_int64, C.c_void_p]
    rng = np.random.default_rng(9)
    pairs_in = []
    for n, hl in ((120, 400), (90, N_MAX + 1), (60, 300)):
        hap = bytes(W._random_seq(rng, hl))
        read = bytes(W._substitute(rng, np.frombuffer(hap[20:20 + n], np.uint8), 0.02))
        q = bytes(rng.integers(10, 41, size=n).astype(np.uint8))
        pairs_in.append((read, q, bytes([45]) * n, bytes([45]) * n, bytes([10]) * n, hap))
    b = W.from_pairs(pairs_in)
    good = W.from_pairs([pairs_in[0], pairs_in[2]])
    with PairHMMEngine(device=0, precision="f64") as eng:
        expect = eng.compute_regions(good)
    dev = torch.device("cuda", 0)
    # slots: 0 valid, 1 haplotype of N_MAX + 1 bases, 2 valid, 3 haplotype index out of range
    pairs = np.zeros(4, dtype=[("read", np.int32), ("hap", np.int32), ("out", np.int64)])
    pairs["read"] = [0, 1, 2, 0]
    pairs["hap"] = [0, 1, 2, b.n_haps]
    pairs["out"] = [0, 1, 2, 3]
    quals = np.stack([b.read_q, b.read_i, b.read_d, b.read_c], axis=1).reshape(-1)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in dict(
        pairs=pairs.view(np.uint8), read_offsets=b.read_offsets.astype(np.int64), read_bases=b.read_bases,
        read_quals=quals, hap_offsets=b.hap_offsets.astype(np.int64), hap_bases=b.hap_bases).items()}
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    dp = DevicePairs(num_pairs=4, pairs=t["pairs"].data_ptr(), num_reads=b.n_reads,
                     read_offsets=t["read_offsets"].data_ptr(), read_bases=t["read_bases"].data_ptr(),
                     read_quals=t["read_quals"].data_ptr(), num_haps=b.n_haps,
                     hap_offsets=t["hap_offsets"].data_ptr(), hap_bases=t["hap_bases"].data_ptr(),
                     max_hap_len=N_MAX)
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize(dev)
    assert fn(0, C.byref(dp), out.data_ptr(), 4, stream) == N.BV_ERR_INVALID_ARG
    got = out.cpu().numpy()
    assert np.isnan(got[1]) and np.isnan(got[3])
    assert np.max(np.abs(got[[0, 2]] - expect)) <= TOL_F64
