"""ctypes bindings to the CPU checkers (test infrastructure only).

* ``Oracle``    -- oracle/_build/liboracle.so, the C restatement of Biovoltron's
                   PairHMM (pairhmm_oracle.c).
* ``Reference`` -- oracle/_ref/libref_pairhmm.so, Biovoltron's own kernel
                   (lib/intel_native/pairhmm) compiled from its sources by
                   oracle/Makefile; absent where the reference tree is absent
                   and nothing was prebuilt.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs use this
module; the product library never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_pairhmm.so")


class Testcase(C.Structure):
    """Layout of ``testcase`` (lib/intel_native/pairhmm/pairhmm_common.h:20-24)."""

    _fields_ = [
        ("rslen", C.c_int), ("haplen", C.c_int),
        ("q", C.c_void_p), ("i", C.c_void_p), ("d", C.c_void_p), ("c", C.c_void_p),
        ("hap", C.c_void_p), ("rs", C.c_void_p),
    ]


TESTCASE_DTYPE = np.dtype([("rslen", np.int32), ("haplen", np.int32), ("q", np.uint64), ("i", np.uint64),
                           ("d", np.uint64), ("c", np.uint64), ("hap", np.uint64), ("rs", np.uint64)])
assert TESTCASE_DTYPE.itemsize == C.sizeof(Testcase)


class TestcaseArray:
    """Testcases pointing into a RegionBatch's arrays (which must stay alive).

    Built with numpy in the C struct's layout, so millions of pairs cost
    milliseconds."""

    __test__ = False

    def __init__(self, batch, reads: np.ndarray, haps: np.ndarray):
        self.batch = batch
        reads = np.asarray(reads, np.int64)
        haps = np.asarray(haps, np.int64)
        n = len(reads)
        self.n = n
        ro, ho = batch.read_offsets.astype(np.int64), batch.hap_offsets.astype(np.int64)
        a = np.zeros(max(n, 1), TESTCASE_DTYPE)
        if n:
            start = ro[reads]
            a["rslen"][:n] = (ro[reads + 1] - start).astype(np.int32)
            a["haplen"][:n] = (ho[haps + 1] - ho[haps]).astype(np.int32)
            for f, arr in (("q", batch.read_q), ("i", batch.read_i), ("d", batch.read_d), ("c", batch.read_c),
                           ("rs", batch.read_bases)):
                a[f][:n] = np.uint64(arr.ctypes.data) + start.astype(np.uint64)
            a["hap"][:n] = np.uint64(batch.hap_bases.ctypes.data) + ho[haps].astype(np.uint64)
        self.np = a
        self.arr = a.ctypes.data_as(C.POINTER(Testcase))

    def __getitem__(self, k):
        return self.arr[k]

    @classmethod
    def for_batch(cls, batch, limit: Optional[int] = None, sel: Optional[np.ndarray] = None):
        r, h = batch.pair_index()
        if sel is not None:
            r, h = r[sel], h[sel]
        if limit is not None:
            r, h = r[:limit], h[:limit]
        return cls(batch, r, h)


def _bind(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle`)")
        self.lib = C.CDLL(path)
        L = self.lib
        P = C.POINTER(Testcase)
        self._f32 = _bind(L, "orc_prob_f32", C.c_float, [P])
        self._f64 = _bind(L, "orc_prob_f64", C.c_double, [P])
        self._rule = _bind(L, "orc_log10_reference_rule", C.c_double, [P, C.POINTER(C.c_int)])
        self._resc = _bind(L, "orc_log10_rescaled", C.c_double, [P])
        self._scalar = _bind(L, "orc_scalar_log10", C.c_double,
                             [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_void_p])
        self._b_rule = _bind(L, "orc_batch_reference_rule", None, [C.c_long, P, C.c_void_p, C.c_void_p, C.c_int])
        self._b_resc = _bind(L, "orc_batch_rescaled", None, [C.c_long, P, C.c_void_p, C.c_int])
        self._b_f32 = _bind(L, "orc_batch_prob_f32", None, [C.c_long, P, C.c_void_p, C.c_int])
        self._b_f64 = _bind(L, "orc_batch_prob_f64", None, [C.c_long, P, C.c_void_p, C.c_int])
        for nm, t in (("orc_table_ph2pr_f32", C.c_float), ("orc_table_ph2pr_f64", C.c_double),
                      ("orc_table_mm_f32", C.c_float), ("orc_table_mm_f64", C.c_double)):
            _bind(L, nm, C.POINTER(t), [])
        _bind(L, "orc_table_mm_size", C.c_int, [])
        self._band = _bind(L, "orc_band_log10", C.c_double, [P, C.c_int, C.c_int])
        self._post = _bind(L, "orc_posterior_diag", C.c_int, [P, C.c_void_p])
        self._leak = _bind(L, "orc_band_leak_bound", C.c_double, [])
        self.set_rho = _bind(L, "orc_band_set_rho", None, [C.c_double])
        self.set_r0 = _bind(L, "orc_band_set_r0", None, [C.c_int])
        self._pedge = _bind(L, "orc_band_posterior_edge", C.c_double, [P, C.c_int, C.c_int])
        self._bdet = _bind(L, "orc_band_detail", C.c_double,
                           [P, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)])

    # banded DP and posterior spread (learned-band path) ---------------------
    def band_log10(self, tcs: TestcaseArray, d_lo, W) -> np.ndarray:
        d_lo = np.broadcast_to(np.asarray(d_lo, np.int64), (tcs.n,))
        W = np.broadcast_to(np.asarray(W, np.int64), (tcs.n,))
        return np.array([self._band(C.pointer(tcs.arr[k]), int(d_lo[k]), int(W[k])) for k in range(tcs.n)])

    def band_detail(self, tcs: TestcaseArray, d_lo, W):
        """Banded log10 plus the kernel's edge statistics (row_ratio, end_frac)."""
        d_lo = np.broadcast_to(np.asarray(d_lo, np.int64), (tcs.n,))
        W = np.broadcast_to(np.asarray(W, np.int64), (tcs.n,))
        out = np.zeros((tcs.n, 4))
        a, b = C.c_double(), C.c_double()
        for k in range(tcs.n):
            out[k, 0] = self._bdet(C.pointer(tcs.arr[k]), int(d_lo[k]), int(W[k]), C.byref(a), C.byref(b))
            out[k, 1], out[k, 2] = a.value, b.value
            out[k, 3] = self._leak()
        return out

    def band_posterior_edge(self, tcs: TestcaseArray, d_lo, W) -> np.ndarray:
        """Upper bound on the posterior mass of the band's two edge diagonals."""
        d_lo = np.broadcast_to(np.asarray(d_lo, np.int64), (tcs.n,))
        W = np.broadcast_to(np.asarray(W, np.int64), (tcs.n,))
        return np.array([self._pedge(C.pointer(tcs.arr[k]), int(d_lo[k]), int(W[k])) for k in range(tcs.n)])

    def posterior_diag(self, tcs: TestcaseArray, k: int):
        """Per-diagonal max-over-rows posterior for pair k: (dmin, pstar array)."""
        t = tcs.arr[k]
        out = np.zeros(t.rslen + t.haplen - 1, np.float64)
        st = self._post(C.pointer(t), out.ctypes.data)
        return (1 - t.rslen, out) if st == 0 else (1 - t.rslen, None)

    # batch forms ------------------------------------------------------------
    def log10_reference_rule(self, tcs: TestcaseArray, threads: int = 0) -> Tuple[np.ndarray, np.ndarray]:
        out = np.zeros(tcs.n, np.float64)
        used = np.zeros(tcs.n, np.int32)
        self._b_rule(tcs.n, tcs.arr, out.ctypes.data, used.ctypes.data, threads)
        return out, used.astype(bool)

    def log10_rescaled(self, tcs: TestcaseArray, threads: int = 0) -> np.ndarray:
        out = np.zeros(tcs.n, np.float64)
        self._b_resc(tcs.n, tcs.arr, out.ctypes.data, threads)
        return out

    def prob_f32(self, tcs: TestcaseArray, threads: int = 0) -> np.ndarray:
        out = np.zeros(tcs.n, np.float32)
        self._b_f32(tcs.n, tcs.arr, out.ctypes.data, threads)
        return out

    def prob_f64(self, tcs: TestcaseArray, threads: int = 0) -> np.ndarray:
        out = np.zeros(tcs.n, np.float64)
        self._b_f64(tcs.n, tcs.arr, out.ctypes.data, threads)
        return out

    def scalar_log10(self, read: bytes, qual: bytes, hap: bytes, trans: Optional[Sequence[float]] = None) -> float:
        t = None
        if trans is not None:
            buf = (C.c_double * 7)(*trans)
            t = C.cast(buf, C.c_void_p)
        return self._scalar(read, qual, len(read), hap, len(hap), t)

    def tables(self):
        L = self.lib
        n = L.orc_table_mm_size()
        return {
            "ph2pr_f32": np.ctypeslib.as_array(L.orc_table_ph2pr_f32(), (128,)).copy(),
            "ph2pr_f64": np.ctypeslib.as_array(L.orc_table_ph2pr_f64(), (128,)).copy(),
            "mm_f32": np.ctypeslib.as_array(L.orc_table_mm_f32(), (n,)).copy(),
            "mm_f64": np.ctypeslib.as_array(L.orc_table_mm_f64(), (n,)).copy(),
        }


REF_SCALAR_SO = os.path.join(HERE, "_ref", "libref_scalar.so")


class ReferenceScalar:
    """Biovoltron's scalar PairHMM (pairhmm.hpp), one pair at a time through
    its per-pair step (oracle/ref_scalar_shim.cpp)."""

    def __init__(self, path: str = REF_SCALAR_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference scalar model not built: {path}")
        self.lib = C.CDLL(path)
        self._f = _bind(self.lib, "ref_scalar_log10", C.c_double,
                        [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_void_p])

    @staticmethod
    def available(path: str = REF_SCALAR_SO) -> bool:
        return os.path.exists(path)

    def log10(self, read: bytes, qual: bytes, hap: bytes, trans: Optional[Sequence[float]] = None) -> float:
        t = None if trans is None else (C.c_double * 7)(*trans)
        return self._f(read, qual, len(read), hap, len(hap), C.cast(t, C.c_void_p) if t is not None else None)


class Reference:
    """Biovoltron's own PairHMM kernel, called as AvxPairHMM calls it."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference kernel not built: {path}")
        self.lib = C.CDLL(path)
        L = self.lib
        P = C.POINTER(Testcase)
        self._f32 = _bind(L, "ref_prob_f32", C.c_float, [P])
        self._f64 = _bind(L, "ref_prob_f64", C.c_double, [P])
        self._batch = _bind(L, "ref_batch_log10", None, [C.c_long, P, C.c_void_p, C.c_void_p, C.c_int])
        self.threads = _bind(L, "ref_threads", C.c_int, [])
        for nm, t in (("ref_table_ph2pr_f32", C.c_float), ("ref_table_ph2pr_f64", C.c_double),
                      ("ref_table_mm_f32", C.c_float), ("ref_table_mm_f64", C.c_double)):
            _bind(L, nm, C.POINTER(t), [])
        _bind(L, "ref_table_mm_size", C.c_int, [])

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def log10(self, tcs: TestcaseArray, threads: int = 0) -> Tuple[np.ndarray, np.ndarray]:
        out = np.zeros(tcs.n, np.float64)
        used = np.zeros(tcs.n, np.int32)
        self._batch(tcs.n, tcs.arr, out.ctypes.data, used.ctypes.data, threads)
        return out, used.astype(bool)

    def prob_f32(self, tcs: TestcaseArray) -> np.ndarray:
        return np.array([self._f32(C.pointer(tcs.arr[k])) for k in range(tcs.n)], np.float32)

    def prob_f64(self, tcs: TestcaseArray) -> np.ndarray:
        return np.array([self._f64(C.pointer(tcs.arr[k])) for k in range(tcs.n)], np.float64)

    def tables(self):
        L = self.lib
        n = L.ref_table_mm_size()
        return {
            "ph2pr_f32": np.ctypeslib.as_array(L.ref_table_ph2pr_f32(), (128,)).copy(),
            "ph2pr_f64": np.ctypeslib.as_array(L.ref_table_ph2pr_f64(), (128,)).copy(),
            "mm_f32": np.ctypeslib.as_array(L.ref_table_mm_f32(), (n,)).copy(),
            "mm_f64": np.ctypeslib.as_array(L.ref_table_mm_f64(), (n,)).copy(),
        }


SEED_STRIDE = 5


def _sample_positions(read_len: int, k: int):
    """Read positions whose k-mers the featuriser looks up: 0, s, 2 s, ...
    and the last one, read_len - k, with s = max(SEED_STRIDE, ceil(last / 31))
    so that at most 32 positions are sampled."""
    last = read_len - k
    stride = max(SEED_STRIDE, (last + 30) // 31)
    pos = list(range(0, last + 1, stride))
    if pos[-1] != last:
        pos.append(last)
    return pos


def _seed_hits(read: bytes, hap: bytes, k: int):
    idx = {}
    for j in range(len(hap) - k + 1):
        s = hap[j:j + k]
        if all(c in b"ACGT" for c in s):
            idx.setdefault(s, []).append(j)
    return [(i, j - i) for i in _sample_positions(len(read), k) for j in idx.get(read[i:i + k], ())]


def seed_diagonal(read: bytes, hap: bytes, k: int = 11):
    """The featuriser's seed diagonal: the most frequent j - i over the shared
    k-mers (haplotype position j, sampled read position i, A/C/G/T only),
    smallest on ties; None without a shared k-mer."""
    if len(read) < k or len(hap) < k:
        return None
    counts = {}
    for _, d in _seed_hits(read, hap, k):
        counts[d] = counts.get(d, 0) + 1
    if not counts:
        return None
    best = max(counts.values())
    return min(d for d, c in counts.items() if c == best)


END_ROWS = 24


def seed_extent(read: bytes, hap: bytes, k: int = 11):
    """The featuriser's band extent, or None without a shared k-mer: the
    lowest and highest diagonal j - i of a shared (sampled) k-mer, widened by
    the read ends' triangles -- t_pre = first sampled read position with a
    hit, t_suf = read bases after the last sampled hit; the first hit's diagonal + t_pre and the last
    hit's diagonal - t_suf (smallest diagonal where a position has several
    hits) are included, and so is d - tail (d + head) for every voted
    diagonal d whose last hit leaves tail <= END_ROWS read bases after it
    (whose first hit starts head <= END_ROWS bases into the read)."""
    if len(read) < k or len(hap) < k:
        return None
    hits = _seed_hits(read, hap, k)
    if not hits:
        return None
    ds = [d for _, d in hits]
    i0 = min(i for i, _ in hits)
    i1 = max(i for i, _ in hits)
    d0 = min(d for i, d in hits if i == i0)
    d1 = min(d for i, d in hits if i == i1)
    t_pre, t_suf = i0, len(read) - k - i1
    lo, hi = min(min(ds), d1 - t_suf), max(max(ds), d0 + t_pre)
    first, last = {}, {}
    for i, d in hits:
        first[d] = min(first.get(d, i), i)
        last[d] = max(last.get(d, i), i)
    for d in first:
        tail, head = len(read) - k - last[d], first[d]
        if tail <= END_ROWS:
            lo = min(lo, d - tail)
        if head <= END_ROWS:
            hi = max(hi, d + head)
    return lo, hi


def _bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (round to nearest even), returned as FP32."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def _onehot(c: int) -> int:
    # the banded kernels' match nibble: N matches everything, other unknown bytes read as A
    return {ord("C"): 2, ord("T"): 4, ord("G"): 8, ord("N"): 15}.get(c, 1)


HIST_BINS = 64


def seed_features(read: bytes, hap: bytes, k: int = 11) -> np.ndarray:
    """The 80 MLP inputs of a pair (BF16 values as FP32), zeros without a
    shared k-mer: 64 bins of the sampled-hit histogram over diagonals
    d* - 32 .. d* + 31, each divided by the number of sampled read positions,
    and 16 scalars -- hits, hits outside the window, read length / 256,
    haplotype length / 1024, (d* + R) / (R + H), 1, the mode's hits, the
    window's non-empty bins / 64, t_pre / 32, t_suf / 32, the first and last
    hit's diagonal relative to d* / 32, the mismatches of the first and last
    16 read bases along those diagonals / 16, and the lowest and highest hit
    diagonal relative to d* / 32 clipped to [-2, 2].  FP32 arithmetic in the
    kernel's order, then BF16 rounding."""
    f = np.zeros(80, np.float32)
    R, H = len(read), len(hap)
    if R < k or H < k:
        return f
    hits = _seed_hits(read, hap, k)
    if not hits:
        return f
    n_samp = len(_sample_positions(R, k))
    inv = np.float32(1.0) / np.float32(n_samp)
    counts = {}
    for _, d in hits:
        counts[d + R] = counts.get(d + R, 0) + 1
    best = max(counts.values())
    best_slot = min(s for s, c in counts.items() if c == best)
    ds = best_slot - R
    i0 = min(i for i, _ in hits)
    i1 = max(i for i, _ in hits)
    d_first = min(d for i, d in hits if i == i0)
    d_last = min(d for i, d in hits if i == i1)
    t_pre, t_suf = i0, R - k - i1
    n_end = min(16, R)
    mis_pre = sum(1 for ip in range(n_end)
                  if not (0 <= ip + d_first < H) or not (_onehot(read[ip]) & _onehot(hap[ip + d_first])))
    mis_suf = sum(1 for l in range(n_end)
                  if not (0 <= R - 1 - l + d_last < H) or not (_onehot(read[R - 1 - l]) & _onehot(hap[R - 1 - l + d_last])))
    win = nonzero = peak = 0
    for t in range(HIST_BINS):
        s = best_slot - HIST_BINS // 2 + t
        cb = counts.get(s, 0) if 0 <= s < R + H else 0
        f[t] = np.float32(cb) * inv
        win += cb
        nonzero += cb > 0
        peak = max(peak, cb)
    total = len(hits)
    smin, smax = min(counts), max(counts)
    F = np.float32
    v = [F(total) * inv, F(total - win) * inv, F(R) / F(256), F(H) / F(1024), F(ds + R) / F(R + H), F(1),
         F(peak) * inv, F(nonzero) / F(HIST_BINS), F(t_pre) / F(32), F(t_suf) / F(32), F(d_first - ds) / F(32),
         F(d_last - ds) / F(32), F(mis_pre) / F(16), F(mis_suf) / F(16),
         max(F(smin - R - ds) / F(32), F(-2)), min(F(smax - R - ds) / F(32), F(2))]
    f[HIST_BINS:] = np.array(v, np.float32)
    return _bf16(f)
