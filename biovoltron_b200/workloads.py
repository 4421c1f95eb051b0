"""Seeded synthetic PairHMM workloads.

A workload is a ``RegionBatch``: active regions, each holding a set of reads
and a set of haplotypes; every read of a region is scored against every
haplotype of that region, which is exactly the ``[read][hap]`` matrix that
``AvxPairHMM::compute_likelihoods(haps, reads)`` returns for one region
(include/biovoltron/algo/align/inexact_match/pairhmm_avx.hpp:160-171).

Byte conventions follow the reference's kernel input (``testcase``,
lib/intel_native/pairhmm/pairhmm_common.h:20-24): bases are ASCII
``A C G T N``; the four quality arrays are raw Phred bytes, used ``& 127``
without any ASCII offset (avx-pairhmm-template.h:110-126).

Generators (all seeded, numpy only):

* ``config0`` -- one region, 8 haplotypes of 300 bp derived from a random base
  haplotype by 1% SNVs and 0-2 indels of 1-10 bp, 64 reads of 150 bp with 1%
  substitutions; q ~ U(10, 40), i = d = 45, c = 10.
* ``config1`` -- 4096 uneven regions: reads per region lognormal (median 60,
  sigma 0.75, clipped to 20-500), read length U(50, 250), haplotypes per region
  U(2, 32) of region length U(200, 700); same mutation and quality model.
* ``config2`` -- 2000 long pairs: reads U(1000, 10000) bp, haplotypes
  max(read + 500, U(1500, 12000)) bp, 8% substitutions and 4% indels of 1-3 bp,
  q ~ U(5, 30).
* ``config4`` -- a uniform-ACGT reference cut into 300 bp regions at 30x
  coverage of 150 bp reads (1% substitutions, 0.1% indels); haplotypes span the
  region +-75 bp and carry random SNV/indel alleles at 1/1000 bp, 2-16 per region.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence, Tuple

import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)

__all__ = [
    "RegionBatch",
    "config0",
    "config1",
    "config2",
    "config4",
    "from_pairs",
    "subsample_regions",
]


@dataclasses.dataclass
class RegionBatch:
    """Flat, contiguous arrays describing many active regions.

    ``read_offsets``/``hap_offsets`` are prefix sums of lengths (length n+1);
    ``region_reads``/``region_haps`` are prefix sums of per-region counts.
    The result of scoring the batch is the concatenation, region by region, of
    read-major ``[reads_in_region x haps_in_region]`` blocks.
    """

    read_bases: np.ndarray
    read_q: np.ndarray
    read_i: np.ndarray
    read_d: np.ndarray
    read_c: np.ndarray
    read_offsets: np.ndarray
    hap_bases: np.ndarray
    hap_offsets: np.ndarray
    region_reads: np.ndarray
    region_haps: np.ndarray
    name: str = ""

    # ---- sizes -------------------------------------------------------------
    @property
    def n_regions(self) -> int:
        return len(self.region_reads) - 1

    @property
    def n_reads(self) -> int:
        return len(self.read_offsets) - 1

    @property
    def n_haps(self) -> int:
        return len(self.hap_offsets) - 1

    def read_lengths(self) -> np.ndarray:
        return np.diff(self.read_offsets)

    def hap_lengths(self) -> np.ndarray:
        return np.diff(self.hap_offsets)

    def result_offsets(self) -> np.ndarray:
        nr = np.diff(self.region_reads)
        nh = np.diff(self.region_haps)
        return np.concatenate([[0], np.cumsum(nr * nh)]).astype(np.int64)

    @property
    def n_pairs(self) -> int:
        return int(self.result_offsets()[-1])

    def pair_index(self) -> Tuple[np.ndarray, np.ndarray]:
        """(read index, hap index) of every result slot, in result order."""
        nr = np.diff(self.region_reads)
        nh = np.diff(self.region_haps)
        cnt = nr * nh
        reg = np.repeat(np.arange(self.n_regions), cnt)
        start = np.concatenate([[0], np.cumsum(cnt)])[:-1]
        local = np.arange(cnt.sum()) - np.repeat(start, cnt)
        nh_r = nh[reg]
        r = self.region_reads[reg] + local // np.maximum(nh_r, 1)
        h = self.region_haps[reg] + local % np.maximum(nh_r, 1)
        return r.astype(np.int64), h.astype(np.int64)

    def n_cells(self) -> int:
        r, h = self.pair_index()
        rl = self.read_lengths().astype(np.int64)
        hl = self.hap_lengths().astype(np.int64)
        return int((rl[r] * hl[h]).sum())

    def nbytes(self) -> int:
        return sum(
            a.nbytes
            for a in (
                self.read_bases, self.read_q, self.read_i, self.read_d, self.read_c,
                self.read_offsets, self.hap_bases, self.hap_offsets,
                self.region_reads, self.region_haps,
            )
        )

    def uniform_gaps(self) -> Optional[Tuple[int, int, int]]:
        """(i, d, c) when every read base has the same insertion, deletion and
        continuation quality (then the batch can be passed without those
        arrays), else None."""
        if self.read_i.size == 0:
            return None
        vals = []
        for a in (self.read_i, self.read_d, self.read_c):
            v = int(a[0])
            if not np.all(a == v):
                return None
            vals.append(v)
        return tuple(vals)

    # ---- accessors ---------------------------------------------------------
    def read(self, k: int) -> Tuple[bytes, bytes, bytes, bytes, bytes]:
        a, b = int(self.read_offsets[k]), int(self.read_offsets[k + 1])
        return (
            self.read_bases[a:b].tobytes(), self.read_q[a:b].tobytes(), self.read_i[a:b].tobytes(),
            self.read_d[a:b].tobytes(), self.read_c[a:b].tobytes(),
        )

    def hap(self, k: int) -> bytes:
        a, b = int(self.hap_offsets[k]), int(self.hap_offsets[k + 1])
        return self.hap_bases[a:b].tobytes()


def _concat(parts: Sequence[np.ndarray]) -> Tuple[np.ndarray, np.ndarray]:
    lens = np.array([len(p) for p in parts], dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    flat = np.concatenate(parts).astype(np.uint8) if parts else np.zeros(0, np.uint8)
    return flat, off


def _random_seq(rng: np.random.Generator, n: int) -> np.ndarray:
    return ACGT[rng.integers(0, 4, size=n)]


def _substitute(rng: np.random.Generator, seq: np.ndarray, rate: float) -> np.ndarray:
    """Replace each base with probability ``rate`` by a different base."""
    out = seq.copy()
    m = rng.random(len(seq)) < rate
    if m.any():
        idx = np.searchsorted(ACGT, out[m])
        idx = np.where(idx >= 4, 0, idx)
        out[m] = ACGT[(idx + rng.integers(1, 4, size=int(m.sum()))) % 4]
    return out


def _apply_indels(rng: np.random.Generator, seq: np.ndarray, n_indels: int, lmin: int, lmax: int) -> np.ndarray:
    out = seq
    for _ in range(n_indels):
        if len(out) < 2 * lmax + 2:
            break
        ln = int(rng.integers(lmin, lmax + 1))
        pos = int(rng.integers(1, len(out) - ln - 1))
        if rng.random() < 0.5:
            out = np.concatenate([out[:pos], _random_seq(rng, ln), out[pos:]])
        else:
            out = np.concatenate([out[:pos], out[pos + ln:]])
    return out


def _mutate_read(rng, src: np.ndarray, start: int, length: int, sub: float, indel_rate: float,
                 indel_lmin: int, indel_lmax: int) -> np.ndarray:
    """Sample ``length`` bases from ``src`` at ``start`` with indels then substitutions."""
    if indel_rate <= 0:
        read = src[start:start + length]
    else:
        pieces: List[np.ndarray] = []
        got = 0
        pos = start
        n_ev = rng.poisson(indel_rate * length)
        ev_pos = np.sort(rng.integers(0, max(length, 1), size=n_ev)) if n_ev else np.zeros(0, int)
        last = 0
        for p in ev_pos:
            p = int(p)
            take = p - last
            if take > 0:
                pieces.append(src[pos:pos + take])
                pos += take
                got += take
                last = p
            ln = int(rng.integers(indel_lmin, indel_lmax + 1))
            if rng.random() < 0.5:
                pieces.append(_random_seq(rng, ln))
                got += ln
            else:
                pos += ln
        rest = length - got
        if rest > 0:
            pieces.append(src[pos:pos + rest])
        read = np.concatenate(pieces) if pieces else src[start:start]
        if len(read) < length:  # ran off the end of the source: pad from its start
            read = np.concatenate([read, src[: length - len(read)]])
        read = read[:length]
    return _substitute(rng, read, sub)


def _quals(rng, n: int, qlo: int, qhi: int, ins: int = 45, dele: int = 45, gcp: int = 10):
    q = rng.integers(qlo, qhi + 1, size=n).astype(np.uint8)
    return q, np.full(n, ins, np.uint8), np.full(n, dele, np.uint8), np.full(n, gcp, np.uint8)


def _build(regions, name: str) -> RegionBatch:
    """regions: list of (list of read tuples (bases,q,i,d,c), list of hap arrays)."""
    rb, rq, ri, rd, rc, hb = [], [], [], [], [], []
    nreads, nhaps = [], []
    for reads, haps in regions:
        for (b, q, i, d, c) in reads:
            rb.append(b); rq.append(q); ri.append(i); rd.append(d); rc.append(c)
        hb.extend(haps)
        nreads.append(len(reads))
        nhaps.append(len(haps))
    read_bases, read_off = _concat(rb)
    return RegionBatch(
        read_bases=read_bases,
        read_q=_concat(rq)[0], read_i=_concat(ri)[0], read_d=_concat(rd)[0], read_c=_concat(rc)[0],
        read_offsets=read_off,
        hap_bases=_concat(hb)[0], hap_offsets=_concat(hb)[1],
        region_reads=np.concatenate([[0], np.cumsum(nreads)]).astype(np.int64),
        region_haps=np.concatenate([[0], np.cumsum(nhaps)]).astype(np.int64),
        name=name,
    )


def _region(rng, hap_len: int, n_haps: int, n_reads: int, read_len_fn, qlo=10, qhi=40,
            sub=0.01, read_indel=0.0, read_indel_l=(1, 1)):
    base = _random_seq(rng, hap_len)
    haps = []
    for _ in range(n_haps):
        h = _substitute(rng, base, 0.01)
        h = _apply_indels(rng, h, int(rng.integers(0, 3)), 1, 10)
        haps.append(h)
    reads = []
    for _ in range(n_reads):
        src = haps[int(rng.integers(0, n_haps))]
        ln = int(min(read_len_fn(), len(src)))
        start = int(rng.integers(0, len(src) - ln + 1))
        b = _mutate_read(rng, src, start, ln, sub, read_indel, *read_indel_l)
        q, i, d, c = _quals(rng, len(b), qlo, qhi)
        reads.append((b, q, i, d, c))
    return reads, haps


def config0(seed: int = 0) -> RegionBatch:
    rng = np.random.default_rng(seed)
    reg = _region(rng, 300, 8, 64, lambda: 150)
    return _build([reg], "config0: 1 region, 64 reads x 8 haps, 150 bp x ~300 bp")


def config1(seed: int = 1, n_regions: int = 4096) -> RegionBatch:
    rng = np.random.default_rng(seed)
    regions = []
    for _ in range(n_regions):
        nr = int(np.clip(np.round(rng.lognormal(np.log(60.0), 0.75)), 20, 500))
        nh = int(rng.integers(2, 33))
        hl = int(rng.integers(200, 701))
        regions.append(_region(rng, hl, nh, nr, lambda: int(rng.integers(50, 251))))
    return _build(regions, f"config1: {n_regions} uneven regions, reads 50-250 bp, haps 200-700 bp")


def config2(seed: int = 2, n_pairs: int = 2000, max_read: int = 10000, max_hap: int = 12000) -> RegionBatch:
    rng = np.random.default_rng(seed)
    regions = []
    for _ in range(n_pairs):
        rl = int(rng.integers(min(1000, max_read), max_read + 1))
        hl = max(rl + 500, int(rng.integers(min(1500, max_hap), max_hap + 1)))
        hap = _random_seq(rng, hl)
        start = int(rng.integers(0, hl - rl + 1 - 50))
        b = _mutate_read(rng, hap, start, rl, 0.08, 0.04, 1, 3)
        q, i, d, c = _quals(rng, rl, 5, 30)
        regions.append(([(b, q, i, d, c)], [hap]))
    return _build(regions, f"config2: {n_pairs} long pairs, reads 1-10 kb, haps 1.5-12 kb")


def config4(seed: int = 4, n_regions: int = 200_000, region_len: int = 300, coverage: float = 30.0,
            read_len: int = 150, pad: int = 75, read_chunk: int = 1 << 20) -> RegionBatch:
    """Whole-genome-shaped batch.  Random draws are made in bulk and reads are
    built in chunks of ``read_chunk``, so 200k regions build in seconds with
    temporaries of a few hundred MB."""
    rng = np.random.default_rng(seed)
    genome_len = n_regions * region_len + 2 * pad + read_len
    genome = _random_seq(rng, genome_len)
    next_base = np.zeros(256, np.uint8)
    next_base[ACGT] = np.roll(ACGT, -1)  # SNV allele: the next base in ACGT order
    base_index = np.zeros(256, np.int64)
    base_index[ACGT] = np.arange(4)
    # haplotypes: span [start - pad, end + pad) of each region with allele edits
    span = region_len + 2 * pad
    nh = rng.integers(2, 17, size=n_regions)
    n_var = np.maximum(1, rng.poisson(span / 1000.0, size=n_regions) + 1)
    v_off = np.concatenate([[0], np.cumsum(n_var)])
    tot_v = int(v_off[-1])
    vpos = rng.integers(5, span - 15, size=tot_v)
    vkind = rng.integers(0, 3, size=tot_v)  # 0 SNV, 1 insertion, 2 deletion
    vlen = rng.integers(1, 6, size=tot_v)
    alt = _random_seq(rng, 8 * tot_v)
    h_off = np.concatenate([[0], np.cumsum(nh)])
    n_haps = int(h_off[-1])
    # carry[h, k]: haplotype h carries its region's variant k; each region's first haplotype is the reference
    kmax = int(n_var.max())
    carry = rng.random((n_haps, kmax)) < 0.5
    carry[h_off[:-1]] = False
    carry &= np.arange(kmax)[None, :] < n_var[np.repeat(np.arange(n_regions), nh)][:, None]
    # Haplotypes are built in region chunks on a (haplotype, position) grid: each cell emits the
    # bases inserted before the position (0-5) and then its base, substituted or deleted.
    hap_chunks, len_chunks = [], []
    reg_of_hap = np.repeat(np.arange(n_regions), nh)
    hap_windows = np.lib.stride_tricks.sliding_window_view(genome, span)
    for g0 in range(0, n_regions, 16384):
        g1 = min(n_regions, g0 + 16384)
        h0, h1 = int(h_off[g0]), int(h_off[g1])
        rg = reg_of_hap[h0:h1]
        base2d = hap_windows[rg * region_len]
        keep = np.ones(base2d.shape, bool)
        ins_len = np.zeros(base2d.shape, np.int8)
        ins_k = np.zeros(base2d.shape, np.int32)
        for kk in range(kmax):
            hh = np.nonzero(carry[h0:h1, kk])[0]
            if hh.size == 0:
                continue
            k = v_off[rg[hh]] + kk
            p, kind, ln = vpos[k], vkind[k], vlen[k]
            snv, dl, il = kind == 0, kind == 2, kind == 1
            base2d[hh[snv], p[snv]] = next_base[base2d[hh[snv], p[snv]]]
            for t in range(5):
                m = dl & (t < ln)
                keep[hh[m], p[m] + t] = False
            ins_len[hh[il], p[il]] = ln[il]
            ins_k[hh[il], p[il]] = k[il]
        cnt = (ins_len + keep).reshape(-1)
        hl = cnt.reshape(base2d.shape).sum(axis=1, dtype=np.int64)
        start = np.cumsum(cnt, dtype=np.int32) - cnt  # exclusive prefix over the grid
        out = np.empty(int(hl.sum()), np.uint8)
        kf, lf, sf = keep.reshape(-1), ins_len.reshape(-1), start
        out[sf[kf] + lf[kf]] = base2d.reshape(-1)[kf]
        ic = np.nonzero(lf)[0]
        for t in range(5):
            m = ic[lf[ic] > t]
            out[sf[m] + t] = alt[8 * ins_k.reshape(-1)[m] + t]
        hap_chunks.append(out)
        len_chunks.append(hl)
    hap_bases = np.concatenate(hap_chunks)
    hap_off = np.concatenate([[0], np.cumsum(np.concatenate(len_chunks))]).astype(np.int64)
    # reads: starts uniform; each read belongs to the region whose haplotype span contains it
    n_reads_total = int(round(n_regions * region_len * coverage / read_len))
    starts = np.sort(rng.integers(0, n_regions * region_len, size=n_reads_total))
    region_of = np.minimum(starts // region_len, n_regions - 1)
    offs = np.minimum(starts - region_of * region_len, span - read_len - 4)
    bases = np.empty((n_reads_total, read_len), np.uint8)
    k = np.arange(read_len)[None, :]
    windows = np.lib.stride_tricks.sliding_window_view(genome, read_len)
    for a in range(0, n_reads_total, read_chunk):
        b = min(n_reads_total, a + read_chunk)
        first = region_of[a:b] * region_len + offs[a:b]
        blk = windows[first]
        # 0.1% indels: at most one per read, applied by shifting the source index
        ind = np.nonzero(rng.random(b - a) < 0.001 * read_len)[0]
        if ind.size:
            p = rng.integers(10, read_len - 10, size=ind.size)[:, None]
            ln = rng.integers(1, 4, size=ind.size)[:, None]
            is_ins = (rng.random(ind.size) < 0.5)[:, None]
            shift = np.where(k >= p, np.where(is_ins, -ln, ln), 0)
            nb = genome[np.clip(first[ind][:, None] + k + shift, 0, genome_len - 1)]
            ins_mask = is_ins & (k >= p) & (k < p + ln)
            blk[ind] = np.where(ins_mask, ACGT[rng.integers(0, 4, size=nb.shape)], nb)
        # 1% substitutions (to one of the three other bases)
        n_sub = int(rng.binomial(blk.size, 0.01))
        flat_i = rng.integers(0, blk.size, size=n_sub)
        fb = blk.reshape(-1)
        fb[flat_i] = ACGT[(base_index[fb[flat_i]] + rng.integers(1, 4, size=n_sub)) % 4]
        bases[a:b] = blk
    flat = bases.reshape(-1)
    n = flat.size
    # base qualities U(10, 40): random bytes below 248 = 8 * 31, divided by 8
    q = np.frombuffer(rng.bytes(n), np.uint8).copy()
    bad = np.flatnonzero(q >= 248)
    while bad.size:
        q[bad] = np.frombuffer(rng.bytes(bad.size), np.uint8)
        bad = bad[q[bad] >= 248]
    q >>= 3
    q += 10
    counts = np.bincount(region_of, minlength=n_regions)
    return RegionBatch(
        read_bases=flat, read_q=q, read_i=np.full(n, 45, np.uint8), read_d=np.full(n, 45, np.uint8),
        read_c=np.full(n, 10, np.uint8),
        read_offsets=(np.arange(n_reads_total + 1, dtype=np.int64) * read_len),
        hap_bases=hap_bases, hap_offsets=hap_off,
        region_reads=np.concatenate([[0], np.cumsum(counts)]).astype(np.int64),
        region_haps=np.concatenate([[0], np.cumsum(nh)]).astype(np.int64),
        name=f"config4: {n_regions} regions of {region_len} bp, {coverage:g}x of {read_len} bp reads",
    )


def from_pairs(pairs: Sequence[Tuple[bytes, bytes, bytes, bytes, bytes, bytes]], name: str = "pairs") -> RegionBatch:
    """One region per (read, q, i, d, c, hap) tuple; handy for edge cases."""
    regions = []
    for read, q, i, d, c, hap in pairs:
        arr = lambda x: np.frombuffer(bytes(x), dtype=np.uint8).copy()
        regions.append(([(arr(read), arr(q), arr(i), arr(d), arr(c))], [arr(hap)]))
    return _build(regions, name)


def subsample_regions(batch: RegionBatch, regions: Sequence[int]) -> RegionBatch:
    """A new batch holding only the listed regions (in that order)."""
    parts = []
    for g in regions:
        r0, r1 = int(batch.region_reads[g]), int(batch.region_reads[g + 1])
        h0, h1 = int(batch.region_haps[g]), int(batch.region_haps[g + 1])
        reads = []
        for k in range(r0, r1):
            a, b = int(batch.read_offsets[k]), int(batch.read_offsets[k + 1])
            reads.append((batch.read_bases[a:b], batch.read_q[a:b], batch.read_i[a:b],
                          batch.read_d[a:b], batch.read_c[a:b]))
        haps = [batch.hap_bases[int(batch.hap_offsets[k]):int(batch.hap_offsets[k + 1])] for k in range(h0, h1)]
        parts.append((reads, haps))
    return _build(parts, batch.name + f" (subsample of {len(parts)} regions)")
