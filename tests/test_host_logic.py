"""Host-side logic: the normalise/filter step of the reference call, the
GpuPairHMM wrapper's layout and side effects (driven by the oracle through a
stand-in engine, no GPU), and the workload generators."""
import math

import numpy as np
import pytest

from biovoltron_b200 import workloads as W
from biovoltron_b200.pairhmm import (GpuPairHMM, Haplotype, SamRecord, filter_poorly_modeled_reads,
                                     normalize_likelihoods)
from oracle.oracle import TestcaseArray


def test_normalize_caps_at_best_minus_4_5():
    ll = [[-10.0, -20.0, -12.0], [-3.0, -3.0, -100.0]]
    normalize_likelihoods(ll)
    assert ll == [[-10.0, -14.5, -12.0], [-3.0, -3.0, -7.5]]


def test_filter_keeps_rows_below_threshold_like_the_reference():
    # threshold = min(2, ceil(0.02 * len)) * -4: -8 for reads of >= 51 bases,
    # -4 for reads of <= 50; the reference keeps rows whose best is BELOW it.
    reads = [SamRecord("A" * 100, "I" * 100), SamRecord("A" * 100, "I" * 100), SamRecord("A" * 40, "I" * 40),
             SamRecord("A" * 40, "I" * 40)]
    ll = [[-7.0, -9.0], [-8.5, -30.0], [-3.9, -5.0], [-4.1, -6.0]]
    filter_poorly_modeled_reads(reads, ll)
    assert ll == [[-8.5, -30.0], [-4.1, -6.0]]
    assert [r.size() for r in reads] == [100, 40]


class _OracleEngine:
    """Stand-in for PairHMMEngine that scores a region batch with the CPU
    oracle; uniform gap penalties fill the per-base arrays as the library
    does."""

    def __init__(self, oracle):
        self.oracle = oracle
        self.calls = []

    def compute_regions(self, batch, uniform_gaps=None):
        self.calls.append((batch.n_regions, batch.n_haps, uniform_gaps))
        if uniform_gaps is not None:
            n = batch.read_bases.size
            batch.read_i, batch.read_d, batch.read_c = (np.full(n, v, np.uint8) for v in uniform_gaps)
        out, _ = self.oracle.log10_reference_rule(TestcaseArray.for_batch(batch))
        return out


def test_gpu_pairhmm_wrapper_semantics(oracle):
    rng = np.random.default_rng(1)
    base = bytes(W._random_seq(rng, 400))
    haps = [Haplotype(base), Haplotype(base[:200] + b"A" + base[200:]), Haplotype(bytes(W._random_seq(rng, 400)))]
    reads = [SamRecord(base[50:150], b";" * 100), SamRecord(base[100:260], b"5" * 160),
             SamRecord(bytes(W._random_seq(rng, 120)), b"+" * 120)]
    orig = list(reads)
    w = GpuPairHMM(engine=_OracleEngine(oracle))
    ll = w.compute_likelihoods(haps, reads)
    # recompute by hand: testcases in [read][hap] order with SAM penalty bytes
    raw = []
    for r in orig:
        row = []
        for h in haps:
            tc = (r.seq, r.qual, bytes([73]) * r.size(), bytes([73]) * r.size(), bytes([43]) * r.size(), h.seq)
            b = W.from_pairs([tc])
            row.append(float(oracle.log10_reference_rule(TestcaseArray.for_batch(b))[0][0]))
        raw.append(row)
    normalize_likelihoods(raw)
    exp_reads = list(orig)
    filter_poorly_modeled_reads(exp_reads, raw)
    assert ll == raw
    assert [r.seq for r in reads] == [r.seq for r in exp_reads]
    # one window is one region, each haplotype sent once, SAM's constant penalties as three bytes
    assert w.engine.calls == [(1, 3, (73, 73, 43))]


def test_sam_penalty_views_have_read_length():
    r = SamRecord("ACGT" * 100, "I" * 400)
    assert r.insertion_gop() == bytes([73]) * 400
    assert r.deletion_gop() == bytes([73]) * 400
    assert r.overall_gcp() == bytes([43]) * 400


def test_config0_shape():
    b = W.config0(0)
    assert b.n_regions == 1 and b.n_reads == 64 and b.n_haps == 8
    assert set(b.read_lengths()) == {150}
    hl = b.hap_lengths()
    assert hl.min() >= 280 and hl.max() <= 320
    q = b.read_q
    assert q.min() >= 10 and q.max() <= 40
    assert set(np.unique(b.read_i)) == {45} and set(np.unique(b.read_c)) == {10}
    assert set(np.unique(b.read_bases)) <= set(b"ACGT")
    r, h = b.pair_index()
    assert len(r) == 512 and r[0] == 0 and h[:8].tolist() == list(range(8))


def test_config1_distribution_small():
    b = W.config1(seed=9, n_regions=64)
    nr = np.diff(b.region_reads)
    nh = np.diff(b.region_haps)
    assert nr.min() >= 20 and nr.max() <= 500
    assert nh.min() >= 2 and nh.max() <= 32
    rl = b.read_lengths()
    assert rl.min() >= 50 and rl.max() <= 250
    assert b.n_pairs == int((nr * nh).sum())


def test_config2_shape():
    b = W.config2(seed=2, n_pairs=4, max_read=3000, max_hap=4000)
    rl, hl = b.read_lengths(), b.hap_lengths()
    assert (hl >= rl + 500).all()
    assert b.read_q.min() >= 5 and b.read_q.max() <= 30


def test_generators_are_seeded():
    a, b = W.config1(seed=4, n_regions=3), W.config1(seed=4, n_regions=3)
    assert np.array_equal(a.read_bases, b.read_bases) and np.array_equal(a.hap_bases, b.hap_bases)


def _chunks(b, k):
    import ctypes as C
    from biovoltron_b200.native import load
    from biovoltron_b200.pairhmm import _BatchView
    lib = load()
    v = _BatchView(b)
    n = lib.bv_phmm_debug_chunks(C.byref(v.c), k, None, 0)
    out = np.zeros(max(4 * n, 1), np.int64)
    assert lib.bv_phmm_debug_chunks(C.byref(v.c), k, out.ctypes.data, n) == n
    return out[:4 * n].reshape(n, 4)


@pytest.mark.parametrize("k", [1, 2, 3, 7, 64])
def test_chunk_plan_covers_regions_in_order(k):
    """The chunked call's region cuts: consecutive, covering every region and
    result slot once, each chunk but the last holding at least total / k pairs."""
    b = W.config1(seed=3, n_regions=50)
    nr, nh = np.diff(b.region_reads), np.diff(b.region_haps)
    per = nr * nh
    c = _chunks(b, k)
    assert c[0, 0] == 0 and c[-1, 1] == b.n_regions
    assert np.all(c[1:, 0] == c[:-1, 1]) and np.all(c[:, 1] > c[:, 0])
    assert np.all(c[:, 2] == np.concatenate([[0], np.cumsum(c[:-1, 3])]))
    for g0, g1, o0, n in c:
        assert n == per[g0:g1].sum()
    target = -(-per.sum() // k)
    assert np.all(c[:-1, 3] >= target)
    assert len(c) <= k


def test_chunk_plan_with_empty_regions():
    b = W.config1(seed=4, n_regions=12)
    # drop the haplotypes of a few regions: zero-pair regions must still be covered
    keep = np.ones(b.n_regions, bool)
    keep[[0, 5, 11]] = False
    rh = b.region_haps.copy()
    nh = np.diff(rh)
    nh[~keep] = 0
    b2 = W.RegionBatch(read_bases=b.read_bases, read_q=b.read_q, read_i=b.read_i, read_d=b.read_d, read_c=b.read_c,
                       read_offsets=b.read_offsets, hap_bases=b.hap_bases, hap_offsets=b.hap_offsets,
                       region_reads=b.region_reads, region_haps=np.concatenate([[0], np.cumsum(nh)]).astype(np.int64),
                       name="holes")
    c = _chunks(b2, 4)
    assert c[0, 0] == 0 and c[-1, 1] == b2.n_regions and c[:, 3].sum() == b2.n_pairs


class _OracleRegionEngine:
    """Stands in for PairHMMEngine on the CPU: compute_regions scores a region
    batch with the oracle (AVX model, or the scalar model while constant
    transitions are set), so the host logic around the engine can be tested
    without a device."""

    def __init__(self):
        from oracle.oracle import Oracle
        self.oracle = Oracle()
        self.trans = None
        self.calls = 0

    def set_transitions(self, trans):
        self.trans = None if trans is None else list(trans)

    def compute_testcases(self, tcs):
        return np.array([self.oracle.scalar_log10(rs, q, hap, self.trans) if self.trans is not None else
                         self.oracle.log10_rescaled(_tcs_array((rs, q, i, d, c, hap)))[0]
                         for rs, q, i, d, c, hap in tcs])

    def compute_regions(self, batch, uniform_gaps=None):
        self.calls += 1
        if self.trans is None:
            if uniform_gaps is not None:  # the library fills every read base with the three values
                n = batch.read_bases.size
                batch.read_i, batch.read_d, batch.read_c = (np.full(n, v, np.uint8) for v in uniform_gaps)
            return self.oracle.log10_rescaled(TestcaseArray.for_batch(batch))
        r, h = batch.pair_index()
        ro, ho = batch.read_offsets, batch.hap_offsets
        return np.array([self.oracle.scalar_log10(bytes(batch.read_bases[ro[a]:ro[a + 1]]),
                                                  bytes(batch.read_q[ro[a]:ro[a + 1]]),
                                                  bytes(batch.hap_bases[ho[c]:ho[c + 1]]), self.trans)
                         for a, c in zip(r, h)])


@pytest.mark.parametrize("model", ["avx", "scalar"])
def test_region_batcher_assembles_slices_and_filters(model):
    """RegionBatcher packs the queued windows into one region batch (one
    engine call), slices the flat results back per window and normalises and
    filters each window as a per-window compute_likelihoods would."""
    from biovoltron_b200.pairhmm import ORIGINAL_DEFAULT, RegionBatcher
    from oracle.oracle import Oracle
    rng = np.random.default_rng(31)
    windows = []
    for w in range(5):
        base = bytes(W._random_seq(rng, int(rng.integers(150, 260))))
        haps = [Haplotype(base)] + [Haplotype(bytes(W._substitute(rng, np.frombuffer(base, np.uint8).copy(), 0.03)))
                                    for _ in range(int(rng.integers(0, 3)))]
        reads = []
        for _ in range(int(rng.integers(0, 6))):
            st = int(rng.integers(0, len(base) - 80))
            reads.append(SamRecord(base[st:st + 80], bytes(rng.integers(15, 41, 80).astype(np.uint8))))
        reads.append(SamRecord(bytes(W._random_seq(rng, 60)), bytes([30] * 60)))
        windows.append((haps, reads))
    eng = _OracleRegionEngine()
    bt = RegionBatcher(engine=eng, model=model)
    lists = [list(r) for _, r in windows]
    hs = [bt.add(haps, lists[k]) for k, (haps, _) in enumerate(windows)]
    bt.run()
    assert eng.calls == 1 and eng.trans is None
    o = Oracle()
    for k, (haps, reads) in enumerate(windows):
        if model == "scalar":
            ll = [[o.scalar_log10(r.seq, r.qual, h.seq, ORIGINAL_DEFAULT) for h in haps] for r in reads]
        else:
            tcs = [(r.seq, r.qual, r.insertion_gop(), r.deletion_gop(), r.overall_gcp(), h.seq)
                   for r in reads for h in haps]
            flat = [o.log10_rescaled(_tcs_array(t))[0] for t in tcs]
            ll = [flat[i * len(haps):(i + 1) * len(haps)] for i in range(len(reads))]
        rr = list(reads)
        normalize_likelihoods(ll)
        filter_poorly_modeled_reads(rr, ll)
        assert [id(r) for r in lists[k]] == [id(r) for r in rr]
        assert bt.result(hs[k]) == ll


def _tcs_array(t):
    rs, q, i, d, c, hap = t
    b = W.from_pairs([(rs, q, i, d, c, hap)])
    return TestcaseArray.for_batch(b)


def test_scalar_drop_in_host_logic():
    """GpuScalarPairHMM sets the constant transitions for its call only,
    scores [read][hap] in order, then normalises and filters."""
    from biovoltron_b200.pairhmm import ORIGINAL_DEFAULT, GpuScalarPairHMM
    from oracle.oracle import Oracle
    rng = np.random.default_rng(9)
    base = bytes(W._random_seq(rng, 200))
    haps = [Haplotype(base), Haplotype(base[:90] + b"G" + base[91:])]
    reads = [SamRecord(base[10:90], bytes(rng.integers(20, 41, 80).astype(np.uint8))),
             SamRecord(bytes(W._random_seq(rng, 70)), bytes([30] * 70))]
    eng = _OracleRegionEngine()
    rr = list(reads)
    trans = (0.999, 0.0005, 0.0005, 0.8, 0.2, 0.85, 0.15)
    ll = GpuScalarPairHMM(engine=eng).compute_likelihoods(haps, rr, trans)
    assert eng.trans is None
    o = Oracle()
    exp = [[o.scalar_log10(r.seq, r.qual, h.seq, trans) for h in haps] for r in reads]
    er = list(reads)
    normalize_likelihoods(exp)
    filter_poorly_modeled_reads(er, exp)
    assert ll == exp and [id(r) for r in rr] == [id(r) for r in er]
    assert tuple(ORIGINAL_DEFAULT) == (0.9998, 0.0001, 0.0001, 0.9, 0.1, 0.9, 0.1)


def _lpt_restatement(cells, n_parts):
    """Greedy LPT on per-block cells: largest first (lower index on ties), to
    the part with the fewest cells (lower index on ties)."""
    order = sorted(range(len(cells)), key=lambda k: (-cells[k], k))
    load = [0] * n_parts
    part = [0] * len(cells)
    for k in order:
        p = min(range(n_parts), key=lambda q: (load[q], q))
        part[k] = p
        load[p] += cells[k]
    return part, load


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partition_is_greedy_lpt_over_region_cells(parts):
    """bv_phmm_plan_partition with one block per region deals the regions by
    greedy LPT on their DP cells; every region is in exactly one part and the
    largest part exceeds the mean by less than the largest region."""
    from biovoltron_b200.pairhmm import plan_partition, regions_of_part
    b = W.config1(seed=21, n_regions=60)
    bs, bp, pc = plan_partition(b, parts)
    assert np.array_equal(bs, np.arange(b.n_regions + 1))
    rl, hl = b.read_lengths(), b.hap_lengths()
    cells = [int(rl[b.region_reads[g]:b.region_reads[g + 1]].sum()) * int(hl[b.region_haps[g]:b.region_haps[g + 1]].sum())
             for g in range(b.n_regions)]
    part, load = _lpt_restatement(cells, parts)
    assert bp.tolist() == part and pc.tolist() == load
    got = np.sort(np.concatenate([regions_of_part(bs, bp, p) for p in range(parts)]))
    assert np.array_equal(got, np.arange(b.n_regions))
    assert max(load) - sum(load) / parts < max(cells)


def test_partition_blocks_are_contiguous_and_balanced():
    """With fewer blocks than regions, blocks are contiguous runs of about
    equal cells, dealt by LPT; bad arguments are refused."""
    import ctypes as C
    from biovoltron_b200.native import load
    from biovoltron_b200.pairhmm import _BatchView, plan_partition
    b = W.config4(seed=3, n_regions=400)
    bs, bp, pc = plan_partition(b, 4, 64)
    assert bs[0] == 0 and bs[-1] == b.n_regions and np.all(np.diff(bs) > 0)
    assert len(bp) <= 64 and pc.sum() == b.n_cells()
    assert pc.max() / pc.mean() < 1.1
    v = _BatchView(b)
    assert load().bv_phmm_plan_partition(C.byref(v.c), 0, 4, None, None, None) == -1
