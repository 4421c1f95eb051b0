"""Host-side interface mirroring Biovoltron's PairHMM call, over the C ABI.

``GpuPairHMM.compute_likelihoods(haplotypes, reads)`` has the signature,
result layout and side effects of ``AvxPairHMM::compute_likelihoods``
(include/biovoltron/algo/align/inexact_match/pairhmm_avx.hpp:160-171): it
returns a ``[read][hap]`` list of log10 likelihoods, caps each row at
``best - 4.5`` (``PairHMM::normalize_likelihoods``, pairhmm.hpp:83-93) and
keeps only the reads whose best likelihood is *below*
``min(2, ceil(0.02 * len)) * -4`` (``filter_poorly_modeled_reads``,
pairhmm.hpp:95-114 -- the reference's comparison, kept as is), removing the
other reads from ``reads`` in place.

``PairHMMEngine`` exposes the batched entry points (regions, testcases, the
shacc batch hook and the device-resident stage/run/fetch cycle).
"""
from __future__ import annotations

import ctypes as C
import os
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import native as N
from .workloads import RegionBatch

__all__ = ["PairHMMEngine", "GpuPairHMM", "Haplotype", "SamRecord", "normalize_likelihoods",
           "filter_poorly_modeled_reads"]

# pairhmm.hpp:27-31
MAXIMUM_BEST_ALT_LIKELIHOOD_DIFFERENCE = -4.5
EXPECTED_ERROR_RATE_PER_BASE = 0.02
LOG10_QUALITY_PER_BASE = -4.0
MAXIMUM_EXPECTED_ERROR_PER_READ = 2.0
# sam.hpp:19-31: gap-open 40 and gap-continuation 10 as '!'-offset characters,
# consumed raw by the kernel.
GAP_OPEN_PENALTY_BYTE = 40 + ord("!")
GAP_CONTINUATION_PENALTY_BYTE = 10 + ord("!")


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


class _BatchView:
    """Keeps the numpy arrays of a RegionBatch alive behind a C struct.

    With ``uniform_gaps`` = (insertion, deletion, continuation) Phred values
    the per-base i, d and c arrays are not passed (NULL): every read base
    takes those values and only bases and base qualities are copied."""

    def __init__(self, b: RegionBatch, uniform_gaps: Optional[Tuple[int, int, int]] = None):
        self.b = b
        # no copies of arrays that already have the C layout (a copy would cost
        # host time on every call and lose a page-locked registration)
        i64 = lambda x: np.ascontiguousarray(x, dtype=np.int64)
        self.arrs = [i64(b.region_reads), i64(b.region_haps), i64(b.read_offsets)] + [
            np.ascontiguousarray(x) for x in (b.read_bases, b.read_q, b.read_i, b.read_d, b.read_c)] + [
            i64(b.hap_offsets), np.ascontiguousarray(b.hap_bases)]
        rr, rh, ro, rb, rq, ri, rd, rc, ho, hb = self.arrs
        gi = gd = gc = 0
        if uniform_gaps is not None:
            gi, gd, gc = (int(x) for x in uniform_gaps)
            ri = rd = rc = np.zeros(0, np.uint8)  # NULL pointers
        self.c = N.RegionBatchC(
            num_regions=b.n_regions, region_reads=_ptr(rr), region_haps=_ptr(rh),
            num_reads=b.n_reads, read_offsets=_ptr(ro), read_bases=_ptr(rb), read_q=_ptr(rq), read_i=_ptr(ri),
            read_d=_ptr(rd), read_c=_ptr(rc), num_haps=b.n_haps, hap_offsets=_ptr(ho), hap_bases=_ptr(hb),
            gap_ins=gi, gap_del=gd, gap_gcp=gc)


class PairHMMEngine:
    """One ``bv_phmm_ctx`` (a CUDA stream and its device buffers on one GPU)."""

    def __init__(self, device: int = 0, precision: str = "auto", mode: str = "full", haps_per_unit: int = 8,
                 haps_per_warp: int = 0, pipeline_chunks: int = 0, pipeline_min_pairs: int = 0):
        self.lib = N.load()
        o = N.Options()
        self.lib.bv_phmm_default_options(C.byref(o))
        o.device = device
        o.precision = {"auto": N.BV_PRECISION_AUTO, "f64": N.BV_PRECISION_F64}[precision]
        o.mode = {"full": N.BV_MODE_FULL, "band": N.BV_MODE_BAND}[mode]
        o.haps_per_unit = haps_per_unit
        o.haps_per_warp = haps_per_warp
        o.pipeline_chunks = pipeline_chunks
        o.pipeline_min_pairs = pipeline_min_pairs
        h = C.c_void_p()
        st = self.lib.bv_phmm_create(C.byref(o), C.byref(h))
        if st != N.BV_OK:
            raise N.NativeError(st, self.lib.bv_phmm_status_string(st).decode())
        self.h = h
        self._staged: Optional[_BatchView] = None
        self._staged_n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.bv_phmm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int):
        if st != N.BV_OK:
            msg = self.lib.bv_phmm_last_error(self.h)
            raise N.NativeError(st, (msg or b"").decode())

    # --- batched entry points ---------------------------------------------
    def compute_regions(self, batch: RegionBatch, out: Optional[np.ndarray] = None, with_stats: bool = False,
                        uniform_gaps: Optional[Tuple[int, int, int]] = None):
        """Scores every region of the batch (bv_phmm_compute_regions).  With
        ``uniform_gaps`` = (ins, del, gcp) the batch's per-base gap arrays are
        replaced by those constants (see _BatchView)."""
        v = _BatchView(batch, uniform_gaps)
        n = int(self.lib.bv_phmm_region_results(C.byref(v.c)))
        if out is None:
            out = np.empty(max(n, 1), np.float64)
        st = N.Stats()
        self._check(self.lib.bv_phmm_compute_regions(self.h, C.byref(v.c), _ptr(out), C.byref(st)))
        self._staged_n = n
        res = out[:n]
        return (res, st.as_dict()) if with_stats else res

    def stage(self, batch: RegionBatch, uniform_gaps: Optional[Tuple[int, int, int]] = None) -> int:
        v = _BatchView(batch, uniform_gaps)
        self._check(self.lib.bv_phmm_stage_regions(self.h, C.byref(v.c)))
        self._staged = v
        self._staged_n = int(self.lib.bv_phmm_region_results(C.byref(v.c)))
        return self._staged_n

    def run(self) -> dict:
        st = N.Stats()
        self._check(self.lib.bv_phmm_run_staged(self.h, C.byref(st)))
        return st.as_dict()

    def fetch(self, n: Optional[int] = None, out: Optional[np.ndarray] = None) -> np.ndarray:
        n = self._staged_n if n is None else n
        if out is None:
            out = np.empty(max(n, 1), np.float64)
        self._check(self.lib.bv_phmm_fetch_results(self.h, _ptr(out), n))
        return out[:n]

    def genotype_staged(self, batch: RegionBatch, allele_count, hap_allele, read_overlaps) -> dict:
        """Device genotyping of the staged, run batch (bv_phmm_genotype_staged):
        per region the kept reads, allele likelihoods [kept][A] and diploid
        genotype likelihoods, as numpy arrays."""
        v = _BatchView(batch)
        ac = np.ascontiguousarray(allele_count, np.int32)
        ha = np.ascontiguousarray(hap_allele, np.int32)
        ov = np.ascontiguousarray(read_overlaps, np.uint8)
        g = N.GenotypeBatch(allele_count=_ptr(ac), hap_allele=_ptr(ha), read_overlaps=_ptr(ov))
        nr = np.diff(batch.region_reads)
        n_al = int(np.sum(nr * ac)) if len(ac) else 0
        n_ge = int(np.sum(ac * (ac + 1) // 2)) if len(ac) else 0
        kept = np.zeros(max(batch.n_regions, 1), np.int32)
        kept_reads = np.full(max(batch.n_reads, 1), -1, np.int32)
        al = np.zeros(max(n_al, 1), np.float64)
        ge = np.zeros(max(n_ge, 1), np.float64)
        ms = C.c_double(0)
        self._check(self.lib.bv_phmm_genotype_staged(self.h, C.byref(v.c), C.byref(g), _ptr(kept), _ptr(kept_reads),
                                                     _ptr(al), _ptr(ge), C.byref(ms)))
        return {"kept_count": kept[:batch.n_regions], "kept_reads": kept_reads[:batch.n_reads],
                "allele_lik": al[:n_al], "genotype_lik": ge[:n_ge], "kernel_ms": ms.value}

    def set_transitions(self, trans: Optional[Sequence[float]]):
        """Constant transitions for every row (the scalar PairHMM model, seven
        values in PairHMM::TrasMatrx order), or None for the quality-derived ones
        (bv_phmm_set_transitions)."""
        arr = None if trans is None else (C.c_double * 7)(*[float(x) for x in trans])
        self._check(self.lib.bv_phmm_set_transitions(self.h, arr))

    def transitions(self) -> Optional[List[float]]:
        arr = (C.c_double * 7)()
        return list(arr) if self.lib.bv_phmm_get_transitions(self.h, arr) else None

    def set_band_options(self, enabled: bool = True, use_mlp: bool = False, fixed_half: int = 8, margin: int = 2,
                         audit_period: int = 0, edge_threshold: float = 1e-3, cap_margin: float = 12.0):
        """Routes pairs through the banded kernel (see bv_band_options).

        cap_margin: banded pairs whose result lies more than this many log10
        units below their read's best result are scored again by the full DP
        (0 switches the rescore off)."""
        o = N.BandOptions()
        self.lib.bv_phmm_default_band_options(C.byref(o))
        o.enabled, o.use_mlp, o.fixed_half, o.margin = int(enabled), int(use_mlp), fixed_half, margin
        o.audit_period, o.edge_threshold, o.cap_margin = audit_period, edge_threshold, cap_margin
        self._check(self.lib.bv_phmm_set_band_options(self.h, C.byref(o)))

    # --- learned band: training and weights ---------------------------------
    def band_train(self, batch: RegionBatch, epochs: int = 20, batch_size: int = 1024, lr: float = 2e-3,
                   alpha: float = 16.0, tau: float = 1e-4, clip: float = 20.0, margin: int = 2,
                   seed: int = 1234) -> dict:
        """Labels `batch` on the GPU and trains the band MLP (bv_phmm_band_train)."""
        o = N.BandTrainOptions()
        self.lib.bv_phmm_default_band_train_options(C.byref(o))
        o.epochs, o.batch, o.lr, o.alpha, o.tau, o.clip, o.margin, o.seed = (
            epochs, batch_size, lr, alpha, tau, clip, margin, seed)
        v = _BatchView(batch)
        rep = N.BandTrainReport()
        self._check(self.lib.bv_phmm_band_train(self.h, C.byref(v.c), C.byref(o), C.byref(rep)))
        self._staged = None
        return rep.as_dict()

    def band_labels(self, batch: RegionBatch, tau: float = 1e-4, features: bool = False, extent: bool = False):
        """Seed diagonal, label spread lo/hi (absolute diagonals) and, on
        request, the MLP inputs and the shared-11-mer diagonal extent of every
        result slot."""
        v = _BatchView(batch)
        n = int(self.lib.bv_phmm_region_results(C.byref(v.c)))
        ds, lo, hi, km, kx = (np.empty(max(n, 1), np.int32) for _ in range(5))
        feat = np.empty((max(n, 1), 80), np.float32) if features else None
        self._check(self.lib.bv_phmm_band_labels(self.h, C.byref(v.c), tau, _ptr(ds), _ptr(lo), _ptr(hi),
                                                 _ptr(feat) if features else None, _ptr(km), _ptr(kx)))
        self._staged = None
        out = (ds[:n], lo[:n], hi[:n])
        if features:
            out = out + (feat[:n],)
        if extent:
            out = out + (km[:n], kx[:n])
        return out

    def band_routes(self):
        """Route of every result slot of the last band-mode run:
        (d_lo, width, route), route 0 banded, 1 routed to the full DP,
        2 edge-check fallback, 3 FP64 recompute."""
        n = self._staged_n
        d_lo, width, route = (np.empty(max(n, 1), np.int32) for _ in range(3))
        self._check(self.lib.bv_phmm_band_routes(self.h, n, _ptr(d_lo), _ptr(width), _ptr(route)))
        return d_lo[:n], width[:n], route[:n]

    def band_weights(self) -> np.ndarray:
        w = np.empty(int(self.lib.bv_phmm_band_param_count()), np.float32)
        self._check(self.lib.bv_phmm_band_get_weights(self.h, _ptr(w), w.size))
        return w

    def set_band_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        self._check(self.lib.bv_phmm_band_set_weights(self.h, _ptr(w), w.size))

    def band_save(self, path: str):
        self._check(self.lib.bv_phmm_band_save(self.h, os.fsencode(path)))

    def band_load(self, path: str):
        self._check(self.lib.bv_phmm_band_load(self.h, os.fsencode(path)))

    def band_mlp_infer(self, x: np.ndarray) -> np.ndarray:
        """The band MLP inference kernel on features x [n, 80] with the installed
        weights (bv_phmm_band_mlp_infer): outputs [n, 2]."""
        x = np.ascontiguousarray(x, np.float32)
        n = x.shape[0]
        out = np.empty((max(n, 1), 2), np.float32)
        self._check(self.lib.bv_phmm_band_mlp_infer(self.h, _ptr(x), n, _ptr(out)))
        return out[:n]

    def band_mlp_eval(self, w: np.ndarray, x: np.ndarray, targets: np.ndarray, alpha: float, grad: bool = True):
        """Training objective on the GPU: (outputs [n, 2], loss, gradient or None)."""
        w = np.ascontiguousarray(w, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        n = x.shape[0]
        out = np.empty((n, 2), np.float32)
        loss = np.zeros(1, np.float32)
        g = np.empty_like(w) if grad else None
        self._check(self.lib.bv_phmm_band_mlp_eval(self.h, _ptr(w), _ptr(x), _ptr(t), n, alpha, _ptr(out),
                                                   _ptr(loss), _ptr(g) if grad else None))
        return out, float(loss[0]), g

    # --- launch-shape autotuning -------------------------------------------
    def autotune(self, sample: RegionBatch, repeats: int = 3) -> List[dict]:
        """Times every launch shape per rows-per-lane bin on `sample` and keeps
        the fastest (bv_phmm_autotune); returns the chosen shape per bin."""
        v = _BatchView(sample)
        out = (N.TuneEntry * 8)()
        n = C.c_int32(0)
        self._check(self.lib.bv_phmm_autotune(self.h, C.byref(v.c), repeats, out, C.byref(n)))
        self._staged = None
        return [out[k].as_dict() for k in range(n.value)]

    def tuning(self) -> List[dict]:
        out = (N.TuneEntry * 8)()
        n = C.c_int32(0)
        self._check(self.lib.bv_phmm_get_tuning(self.h, out, C.byref(n)))
        return [out[k].as_dict() for k in range(n.value)]

    def set_tuning(self, entries: Sequence[dict]):
        arr = (N.TuneEntry * max(len(entries), 1))()
        for k, e in enumerate(entries):
            arr[k] = N.TuneEntry(e["rows_per_lane"], e["haps_per_warp"], e["warps_per_block"], 0, 0.0)
        self._check(self.lib.bv_phmm_set_tuning(self.h, arr, len(entries)))
        self._staged = None

    def set_long_warps(self, warps: int):
        """Warps per pair of the FP64 long-read kernel (2, 4 or 8; reads of at
        least 128 x warps bases take it)."""
        self._check(self.lib.bv_phmm_set_long_warps(self.h, int(warps)))
        self._staged = None

    def long_warps(self) -> int:
        return int(self.lib.bv_phmm_get_long_warps(self.h))

    def autotune_long(self, sample: RegionBatch, repeats: int = 3) -> dict:
        """Times the FP64 pass of `sample` with 2, 4 and 8 warps per long-read
        pair and installs the fastest (bv_phmm_autotune_long)."""
        v = _BatchView(sample)
        warps = C.c_int32(0)
        ms = np.zeros(3, np.float64)
        self._check(self.lib.bv_phmm_autotune_long(self.h, C.byref(v.c), repeats, C.byref(warps), _ptr(ms)))
        self._staged = None
        return {"warps_per_pair": int(warps.value), "fp64_ms": {2: float(ms[0]), 4: float(ms[1]), 8: float(ms[2])}}

    def host_register(self, arr: np.ndarray):
        self._check(self.lib.bv_phmm_host_register(self.h, _ptr(arr), arr.nbytes))

    def host_unregister(self, arr: np.ndarray):
        self._check(self.lib.bv_phmm_host_unregister(self.h, _ptr(arr)))

    def compute_testcases(self, tcs: Sequence[tuple]) -> np.ndarray:
        """tcs: (read, q, i, d, c, hap) byte strings; returns log10 per testcase."""
        keep = []
        arr = (N.TestcaseC * max(len(tcs), 1))()
        cache = {}
        def buf(b: bytes):
            key = id(b)
            if key not in cache:
                a = np.frombuffer(bytes(b), dtype=np.uint8).copy()
                cache[key] = a
                keep.append(a)
            return _ptr(cache[key])
        for k, (rs, q, i, d, c, hap) in enumerate(tcs):
            t = arr[k]
            t.rslen, t.haplen = len(rs), len(hap)
            t.rs, t.q, t.i, t.d, t.c, t.hap = buf(rs), buf(q), buf(i), buf(d), buf(c), buf(hap)
        out = np.empty(max(len(tcs), 1), np.float64)
        self._check(self.lib.bv_phmm_compute_testcases(self.h, arr, len(tcs), _ptr(out), None))
        return out[: len(tcs)]

    def shacc_calculate(self, reads: Sequence[tuple], haps: Sequence[bytes]) -> np.ndarray:
        """reads: (bases, q, i, d, c) byte strings; returns float32 [reads, haps] log10."""
        keep = []
        def b(x):
            a = np.frombuffer(bytes(x), dtype=np.uint8).copy()
            keep.append(a)
            return _ptr(a)
        ra = (N.ShaccRead * max(len(reads), 1))()
        for k, (s, q, i, d, c) in enumerate(reads):
            ra[k] = N.ShaccRead(len(s), b(s), b(q), b(i), b(d), b(c))
        ha = (N.ShaccHap * max(len(haps), 1))()
        for k, s in enumerate(haps):
            ha[k] = N.ShaccHap(len(s), b(s))
        res = np.zeros(max(len(reads) * len(haps), 1), np.float32)
        cells = sum(len(r[0]) for r in reads) * sum(len(h) for h in haps)
        bt = N.ShaccBatch(len(reads), len(haps), cells, ra, ha, res.ctypes.data_as(C.POINTER(C.c_float)))
        self._check(self.lib.bv_phmm_shacc_calculate(self.h, C.byref(bt)))
        return res[: len(reads) * len(haps)].reshape(len(reads), len(haps))


def plan_partition(batch: RegionBatch, n_parts: int, n_blocks: Optional[int] = None):
    """The split of ``batch`` over ``n_parts`` devices (bv_phmm_plan_partition):
    contiguous region blocks of about equal DP cells dealt by greedy LPT.
    Returns (block_start [n_blocks + 1], block_part [n_blocks], part_cells
    [n_parts]); ``n_blocks`` defaults to one block per region."""
    lib = N.load()
    v = _BatchView(batch)
    nb = max(1, batch.n_regions if n_blocks is None else int(n_blocks))
    bs = np.zeros(nb + 1, np.int64)
    bp = np.zeros(nb, np.int32)
    pc = np.zeros(n_parts, np.int64)
    got = int(lib.bv_phmm_plan_partition(C.byref(v.c), n_parts, nb, _ptr(bs), _ptr(bp), _ptr(pc)))
    if got < 0:
        raise ValueError("invalid batch or part count")
    return bs[:got + 1], bp[:got], pc


def regions_of_part(block_start: np.ndarray, block_part: np.ndarray, part: int) -> np.ndarray:
    """The regions one part scores, in region order."""
    return np.concatenate([np.arange(block_start[b], block_start[b + 1]) for b in range(len(block_part))
                           if block_part[b] == part] or [np.zeros(0, np.int64)]).astype(np.int64)


def compute_regions_multi(engines: Sequence["PairHMMEngine"], batch: RegionBatch,
                          out: Optional[np.ndarray] = None, with_stats: bool = False,
                          uniform_gaps: Optional[Tuple[int, int, int]] = None):
    """Scores one batch over several engines (one per GPU) with the LPT split
    of bv_phmm_compute_regions_multi; results in region order."""
    lib = N.load()
    v = _BatchView(batch, uniform_gaps)
    n = int(lib.bv_phmm_region_results(C.byref(v.c)))
    if out is None:
        out = np.empty(max(n, 1), np.float64)
    hs = (C.c_void_p * len(engines))(*[e.h for e in engines])
    st = N.Stats()
    status = lib.bv_phmm_compute_regions_multi(hs, len(engines), C.byref(v.c), _ptr(out), C.byref(st))
    if status != N.BV_OK:
        msgs = "; ".join((lib.bv_phmm_last_error(e.h) or b"").decode() for e in engines)
        raise N.NativeError(status, msgs)
    return (out[:n], st.as_dict()) if with_stats else out[:n]


# --- reference-shaped objects ------------------------------------------------
class Haplotype:
    """The field of ``biovoltron::Haplotype`` the PairHMM reads (haplotype.hpp:12)."""

    def __init__(self, seq):
        self.seq = seq.encode() if isinstance(seq, str) else bytes(seq)


class SamRecord:
    """The fields and penalty views of ``SamRecord`` the PairHMM reads (sam.hpp:186-475).

    The reference's ``insertion_gop()``/``deletion_gop()``/``overall_gcp()``
    return views of 256-byte static strings and overrun them for longer reads;
    here they have the read's length, filled with the same bytes.
    """

    def __init__(self, seq, qual):
        self.seq = seq.encode() if isinstance(seq, str) else bytes(seq)
        self.qual = qual.encode() if isinstance(qual, str) else bytes(qual)

    def size(self) -> int:
        return len(self.seq)

    def insertion_gop(self) -> bytes:
        return bytes([GAP_OPEN_PENALTY_BYTE]) * len(self.seq)

    def deletion_gop(self) -> bytes:
        return bytes([GAP_OPEN_PENALTY_BYTE]) * len(self.seq)

    def overall_gcp(self) -> bytes:
        return bytes([GAP_CONTINUATION_PENALTY_BYTE]) * len(self.seq)


def normalize_likelihoods(ll: List[List[float]]) -> None:
    """PairHMM::normalize_likelihoods (pairhmm.hpp:83-93), in place."""
    for row in ll:
        if not row:
            continue
        cap = max(row) + MAXIMUM_BEST_ALT_LIKELIHOOD_DIFFERENCE
        for k, v in enumerate(row):
            if v < cap:
                row[k] = cap


def filter_poorly_modeled_reads(reads: list, ll: List[List[float]]) -> None:
    """PairHMM::filter_poorly_modeled_reads (pairhmm.hpp:95-114), in place.

    Keeps the rows whose best likelihood is below the threshold, exactly as
    the reference compares.
    """
    kept_r, kept_l = [], []
    for r, row in zip(reads, ll):
        best = max(row)
        thr = min(MAXIMUM_EXPECTED_ERROR_PER_READ, math.ceil(r.size() * EXPECTED_ERROR_RATE_PER_BASE)) * LOG10_QUALITY_PER_BASE
        if best < thr:
            kept_r.append(r)
            kept_l.append(row)
    reads[:] = kept_r
    ll[:] = kept_l


ORIGINAL_DEFAULT = (0.9998, 0.0001, 0.0001, 0.9, 0.1, 0.9, 0.1)  # pairhmm.hpp:32-33


def _windows_batch(windows: Sequence[tuple], scalar: bool):
    """One region per (haplotypes, reads) window, as bv_phmm_compute_regions
    takes them, and the uniform gap penalties to pass instead of the per-base
    arrays when every read's three penalty views hold one byte throughout
    (SamRecord fills them from constant strings); the scalar model reads no
    gap bytes at all."""
    rb, rq, ri, rd, rc, hb = [], [], [], [], [], []
    nreads, nhaps = [], []
    for haps, reads in windows:
        for r in reads:
            q = np.frombuffer(r.qual, np.uint8)
            rb.append(np.frombuffer(r.seq, np.uint8))
            rq.append(q)
            ri.append(q if scalar else np.frombuffer(r.insertion_gop(), np.uint8))
            rd.append(q if scalar else np.frombuffer(r.deletion_gop(), np.uint8))
            rc.append(q if scalar else np.frombuffer(r.overall_gcp(), np.uint8))
        hb.extend(np.frombuffer(h.seq, np.uint8) for h in haps)
        nreads.append(len(reads))
        nhaps.append(len(haps))

    def cat(parts):
        if not parts:
            return np.zeros(0, np.uint8), np.zeros(1, np.int64)
        lens = np.array([len(p) for p in parts], np.int64)
        return np.concatenate(parts).astype(np.uint8), np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)

    read_bases, read_off = cat(rb)
    batch = RegionBatch(read_bases=read_bases, read_q=cat(rq)[0], read_i=cat(ri)[0], read_d=cat(rd)[0],
                        read_c=cat(rc)[0], read_offsets=read_off, hap_bases=cat(hb)[0], hap_offsets=cat(hb)[1],
                        region_reads=np.concatenate([[0], np.cumsum(nreads)]).astype(np.int64),
                        region_haps=np.concatenate([[0], np.cumsum(nhaps)]).astype(np.int64),
                        name="windows")
    uniform = (0, 0, 0) if scalar else batch.uniform_gaps()
    return batch, uniform


class GpuScalarPairHMM:
    """Drop-in for the scalar ``biovoltron::PairHMM`` (pairhmm.hpp:14-141) on
    one GPU: constant transitions, the base qualities' emission prior, then
    normalize_likelihoods and filter_poorly_modeled_reads as PairHMM does."""

    def __init__(self, device: int = 0, engine: Optional[PairHMMEngine] = None):
        self.engine = engine or PairHMMEngine(device=device)

    def compute_likelihoods(self, haplotypes: Sequence[Haplotype], reads: list,
                            trans: Sequence[float] = ORIGINAL_DEFAULT) -> List[List[float]]:
        nr, nh = len(reads), len(haplotypes)
        if nr == 0:
            return []
        self.engine.set_transitions(trans)
        try:
            batch, gaps = _windows_batch([(list(haplotypes), reads)], scalar=True)
            flat = self.engine.compute_regions(batch, uniform_gaps=gaps) if nh else np.zeros(0)
        finally:
            self.engine.set_transitions(None)
        ll = [list(map(float, flat[k * nh:(k + 1) * nh])) for k in range(nr)]
        if nh == 0:
            return ll
        normalize_likelihoods(ll)
        filter_poorly_modeled_reads(reads, ll)
        return ll


class GpuPairHMM:
    """Drop-in for ``AvxPairHMM`` (pairhmm_avx.hpp:24-172) on one GPU."""

    def __init__(self, device: int = 0, use_double: bool = False, engine: Optional[PairHMMEngine] = None):
        self.engine = engine or PairHMMEngine(device=device, precision="f64" if use_double else "auto")

    def compute_likelihoods(self, haplotypes: Sequence[Haplotype], reads: list) -> List[List[float]]:
        nr, nh = len(reads), len(haplotypes)
        if nr == 0:
            return []
        # the window is one region: each haplotype crosses to the device once
        batch, gaps = _windows_batch([(list(haplotypes), reads)], scalar=False)
        flat = self.engine.compute_regions(batch, uniform_gaps=gaps) if nh else np.zeros(0)
        ll = [list(map(float, flat[k * nh:(k + 1) * nh])) for k in range(nr)]
        if nh == 0:
            return ll
        normalize_likelihoods(ll)
        filter_poorly_modeled_reads(reads, ll)
        return ll


class RegionBatcher:
    """Queues many active regions and scores them in one GPU call.

    ``HaplotypeCaller::run`` calls the PairHMM once per window, one window
    after another (haplotypecaller.hpp:126-151; the call at :90).  Here a
    caller adds each window's haplotypes and reads, runs the queue once
    (``bv_phmm_compute_regions`` over all of them: one batch, one set of
    launches) and reads each window's matrix back, normalised and filtered
    exactly as ``compute_likelihoods`` would have done for that window alone
    (the filter removes reads from the window's own list).  ``model="scalar"``
    scores with the scalar PairHMM's constant transitions instead.
    """

    def __init__(self, engine: Optional[PairHMMEngine] = None, device: int = 0, model: str = "avx",
                 trans: Sequence[float] = ORIGINAL_DEFAULT):
        if model not in ("avx", "scalar"):
            raise ValueError("model is 'avx' or 'scalar'")
        self.engine = engine or PairHMMEngine(device=device)
        self.model, self.trans = model, tuple(trans)
        self._queue: List[tuple] = []
        self._results: List[Optional[List[List[float]]]] = []

    def add(self, haplotypes: Sequence[Haplotype], reads: list) -> int:
        """Queues one window; returns its handle for ``result``."""
        self._queue.append((list(haplotypes), reads))
        self._results.append(None)
        return len(self._results) - 1

    def run(self) -> None:
        """Scores every queued window in one call and stores the results."""
        if not self._queue:
            return
        scalar = self.model == "scalar"
        batch, gaps = _windows_batch(self._queue, scalar)
        if scalar:
            self.engine.set_transitions(self.trans)
        try:
            flat = self.engine.compute_regions(batch, uniform_gaps=gaps)
        finally:
            if scalar:
                self.engine.set_transitions(None)
        pos = 0
        for k, (haps, reads) in enumerate(self._queue):
            nr, nh = len(reads), len(haps)
            ll = [list(map(float, flat[pos + i * nh: pos + (i + 1) * nh])) for i in range(nr)]
            pos += nr * nh
            if nh and nr:
                normalize_likelihoods(ll)
                filter_poorly_modeled_reads(reads, ll)
            self._results[k] = ll
        self._queue = []

    def result(self, handle: int) -> List[List[float]]:
        r = self._results[handle]
        if r is None:
            raise RuntimeError("window not scored yet: call run()")
        return r
