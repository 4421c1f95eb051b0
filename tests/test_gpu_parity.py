"""CUDA path vs the oracle and the reference's golden vectors, through the C ABI.

Tolerances: the FP32 path differs from the reference's FP32 kernel by
single-precision rounding (different operation order, fused multiply-adds);
log10 likelihoods are asserted within 1e-4 where the reference is finite and
within 1e-3 (the contract) against the FP64 oracle everywhere.
"""
import numpy as np
import pytest

from biovoltron_b200 import workloads as W
from conftest import FIXTURES, load_golden
from oracle.oracle import TestcaseArray

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-4
TOL_CONTRACT = 1e-3


def _check(got, ref_log10, truth, tol=TOL_FP32):
    got = np.asarray(got)
    fin = np.isfinite(truth)
    assert np.all(np.isfinite(got[fin])), "GPU result not finite where the FP64 oracle is"
    assert np.max(np.abs(got[fin] - truth[fin]), initial=0) <= TOL_CONTRACT
    rf = np.isfinite(ref_log10)
    assert np.max(np.abs(got[rf] - ref_log10[rf]), initial=0) <= tol
    # where the oracle says the likelihood is exactly zero, so does the GPU
    assert np.all(np.isneginf(got[~fin]))


@pytest.mark.parametrize("name", FIXTURES)
def test_golden_fixtures(engine, name):
    b, exp = load_golden(name)
    got, st = engine.compute_regions(b, with_stats=True)
    assert st["pairs"] == b.n_pairs
    _check(got, exp["ref_log10"], exp["oracle_rescaled"])


@pytest.mark.parametrize("name", ["config0", "edge_cases"])
def test_fp64_mode_matches_reference_fp64(name):
    from biovoltron_b200.pairhmm import PairHMMEngine
    b, exp = load_golden(name)
    with PairHMMEngine(precision="f64") as e:
        got = e.compute_regions(b)
    pd = exp["ref_prob_f64"].astype(np.float64)
    with np.errstate(divide="ignore"):
        ref = np.log10(pd) - 1020 * np.log10(2.0)
    fin = np.isfinite(ref)
    assert np.max(np.abs(got[fin] - ref[fin])) < 1e-9
    _check(got, exp["ref_log10"], exp["oracle_rescaled"], tol=TOL_FP32)


def test_rescue_flags_match_reference_rule(engine):
    b, exp = load_golden("edge_cases")
    _, st = engine.compute_regions(b, with_stats=True)
    # every pair the reference sends to FP64 is far below the threshold here,
    # so the GPU rescues the same pairs (and reports them)
    assert st["rescued"] == int(exp["ref_used_f64"].sum())


def test_config1_sample_vs_oracle(engine, oracle):
    b = W.config1(seed=77, n_regions=24)
    got = engine.compute_regions(b)
    truth = oracle.log10_rescaled(TestcaseArray.for_batch(b))
    ref, _ = oracle.log10_reference_rule(TestcaseArray.for_batch(b))
    _check(got, ref, truth)


def test_config2_long_reads_vs_rescaled_oracle(engine, oracle):
    b = W.config2(seed=21, n_pairs=8, max_read=3000, max_hap=4000)
    got, st = engine.compute_regions(b, with_stats=True)
    truth = oracle.log10_rescaled(TestcaseArray.for_batch(b))
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - truth)) <= TOL_CONTRACT
    assert st["rescued"] == b.n_pairs  # all far below 1e-28 (log10 ~ -hundreds)


def test_config2_full_length_long_reads(oracle):
    """Full-length config-2 pairs (reads up to 10 kb against haplotypes up to
    12 kb): every pair falls below 1e-28 in FP32 and is rescued; reads of 512
    bases or more run on the several-warps-per-pair FP64 kernel, whose groups
    of strips are renormalised between groups.  Against the rescaled FP64
    oracle, in the default precision and with every pair in FP64."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    b = W.config2(seed=23, n_pairs=6)
    assert b.read_lengths().max() > 6000
    truth = oracle.log10_rescaled(TestcaseArray.for_batch(b))
    for precision in ("auto", "f64"):
        with PairHMMEngine(device=0, precision=precision) as e:
            got, st = e.compute_regions(b, with_stats=True)
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - truth)) <= 1e-9, (precision, got - truth)
        assert st["rescued"] == b.n_pairs


def test_long_read_warps_per_pair_and_tuner(oracle):
    """The FP64 long-read kernel with 2, 4 and 8 warps per pair (reads of at
    least 256, 512 and 1024 bases take it, the rest the one-warp kernel)
    against the rescaled FP64 oracle; the long-read tuner times the three,
    installs one, and the call in the default precision still matches."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    b = W.config2(seed=29, n_pairs=8, max_read=3000, max_hap=4000)
    truth = oracle.log10_rescaled(TestcaseArray.for_batch(b))
    with PairHMMEngine(device=0, precision="f64") as e:
        assert e.long_warps() == 4
        for k in (2, 4, 8):
            e.set_long_warps(k)
            assert e.long_warps() == k
            got = e.compute_regions(b)
            assert np.max(np.abs(got - truth)) <= 1e-9, (k, got - truth)
        with pytest.raises(RuntimeError):
            e.set_long_warps(3)
    with PairHMMEngine(device=0) as e:
        rep = e.autotune_long(b, repeats=2)
        print("long-read tuner", rep)
        assert rep["warps_per_pair"] in (2, 4, 8) and e.long_warps() == rep["warps_per_pair"]
        assert all(v > 0 for v in rep["fp64_ms"].values())
        got = e.compute_regions(b)
        assert np.max(np.abs(got - truth)) <= 1e-9


def test_long_read_lengths_around_the_group_boundaries(oracle):
    """Reads whose strip counts fall on either side of a group of four strips
    (and of the long-read threshold of 512 bases), mixed with short reads in
    one batch, all in FP64: the long and the one-warp FP64 kernels share the
    FP64 list."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    rng = np.random.default_rng(31)
    regions = []
    for rl in (100, 383, 511, 512, 513, 639, 640, 767, 1023, 1024, 1025, 1600):
        hap = W._random_seq(rng, rl + 300)
        start = int(rng.integers(0, 250))
        read = W._mutate_read(rng, hap, start, rl, 0.02, 0.01, 1, 2)
        q, i, d, c = W._quals(rng, len(read), 10, 40)
        regions.append(([(read, q, i, d, c)], [hap, W._random_seq(rng, rl + 200)]))
    b = W._build(regions, "long-read lengths around the strip groups")
    truth = oracle.log10_rescaled(TestcaseArray.for_batch(b))
    with PairHMMEngine(device=0, precision="f64") as e:
        got = e.compute_regions(b)
        # staged runs (the second replays a graph) give the same results: the
        # pairs the long-read kernel hands back (the unrelated haplotypes fall
        # too far within a group of strips) are scored again each time
        n = e.stage(b)
        for _ in range(2):
            e.run()
            assert np.array_equal(e.fetch(n), got)
    fin = np.isfinite(truth)
    assert np.array_equal(np.isfinite(got), fin)
    assert np.max(np.abs(got[fin] - truth[fin])) <= 1e-9


def test_staged_graph_replay_is_deterministic(engine):
    b = W.config1(seed=3, n_regions=16)
    direct = engine.compute_regions(b)
    n = engine.stage(b)
    outs = []
    for _ in range(3):  # first run launches, later runs replay the captured graph
        st = engine.run()
        assert st["ms_fp32"] > 0 and st["ms_fp64"] > 0  # event nodes replay with the graph
        outs.append(engine.fetch(n).copy())
    for o in outs:
        assert np.array_equal(o, direct)


def test_testcase_and_shacc_entry_points_agree(engine):
    b, exp = load_golden("config0")
    r, h = b.pair_index()
    tcs = []
    for k in range(len(r)):
        rd = b.read(int(r[k]))
        tcs.append((rd[0], rd[1], rd[2], rd[3], rd[4], b.hap(int(h[k]))))
    got_tc = engine.compute_testcases(tcs)
    reads = [b.read(k) for k in range(b.n_reads)]
    haps = [b.hap(k) for k in range(b.n_haps)]
    got_sh = engine.shacc_calculate(reads, haps)
    got_rg = engine.compute_regions(b)
    assert np.array_equal(got_tc, got_rg)
    assert np.array_equal(got_sh.reshape(-1), got_rg.astype(np.float32))


def test_gpu_pairhmm_drop_in(engine):
    from biovoltron_b200.pairhmm import GpuPairHMM, Haplotype, SamRecord
    b, exp = load_golden("ref_test")
    haps = [Haplotype(b.hap(k)) for k in range(8)]
    reads = [SamRecord(b.read(k)[0], b.read(k)[1]) for k in range(3)]
    w = GpuPairHMM(engine=engine)
    ll = w.compute_likelihoods(haps, reads)
    raw = exp["ref_log10"].reshape(3, 8)
    for row in ll:
        assert len(row) == 8
    # rows kept are those whose best is below -8 (the reference's filter)
    kept = [k for k in range(3) if raw[k].max() < -8]
    assert len(ll) == len(kept)
    for row, k in zip(ll, kept):
        capped = np.maximum(raw[k], raw[k].max() - 4.5)
        assert np.max(np.abs(np.array(row) - capped)) < TOL_FP32


def test_empty_and_ragged_inputs(engine):
    # empty batch
    e = W.from_pairs([])
    assert engine.compute_regions(e).size == 0
    # regions with zero reads / zero haps, empty reads and haps
    parts = [(b"", b"", b"", b"", b"", b"ACGT"), (b"ACGT", b"IIII", b"----", b"----", b"++++", b""),
             (b"A", b"I", b"-", b"-", b"+", b"A")]
    b = W.from_pairs(parts)
    got = engine.compute_regions(b)
    assert np.isneginf(got[0]) and np.isneginf(got[1]) and np.isfinite(got[2])


def test_invalid_arguments_are_rejected(engine):
    from biovoltron_b200.native import NativeError
    b = W.config0(0)
    bad = W.RegionBatch(**{k: getattr(b, k) for k in ("read_bases", "read_q", "read_i", "read_d", "read_c",
                                                       "read_offsets", "hap_bases", "hap_offsets",
                                                       "region_reads")}, region_haps=np.array([0, 99], np.int64))
    with pytest.raises(NativeError) as ei:
        engine.compute_regions(bad)
    assert ei.value.status == 1
    long_hap = W.from_pairs([(b"ACGT", b"IIII", b"----", b"----", b"++++", b"A" * 40000)])
    with pytest.raises(NativeError):
        engine.compute_regions(long_hap)
    # the context still works afterwards
    assert np.isfinite(engine.compute_regions(W.config0(0))).all()


def test_alignment_ending_at_last_haplotype_base(engine, oracle):
    # The last column must be reached whatever haplotype length mod the
    # kernel's step chunking (8 single-strip, 32 multi-strip); reads here end
    # exactly at the haplotype's last base, so that column carries the mass.
    rng = np.random.default_rng(17)
    pairs = []
    for H in list(range(220, 236)) + list(range(985, 995)):
        hap = bytes(W._random_seq(rng, H))
        for n in (100, 300):
            read = hap[H - n:]
            pairs.append((read, bytes(rng.integers(20, 41, size=n).astype(np.uint8)), bytes([45]) * n,
                          bytes([45]) * n, bytes([10]) * n, hap))
    b = W.from_pairs(pairs)
    got = engine.compute_regions(b)
    truth = oracle.log10_rescaled(TestcaseArray.for_batch(b))
    ref, _ = oracle.log10_reference_rule(TestcaseArray.for_batch(b))
    _check(got, ref, truth)


@pytest.mark.parametrize("seed", [5, 6])
def test_paired_haplotypes_bit_identical_to_single(seed):
    """Two haplotypes per warp (packed FP32x2) run each pair's arithmetic in
    the single-haplotype order: identical results, including the FP64-rescued
    pairs and odd haplotype counts."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    b = W.config1(seed=seed, n_regions=24)
    with PairHMMEngine(haps_per_warp=1) as e1:
        one, st1 = e1.compute_regions(b, with_stats=True)
    with PairHMMEngine(haps_per_warp=2) as e2:
        two, st2 = e2.compute_regions(b, with_stats=True)
    assert st1["rescued"] == st2["rescued"]
    assert np.array_equal(one, two)


def test_autotune_picks_shapes_and_keeps_results():
    """The launch-shape autotuner times every shape per rows-per-lane bin; any
    shape gives the same results (each pair's arithmetic does not depend on
    the launch shape)."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    b = W.config1(seed=9, n_regions=24)
    with PairHMMEngine() as e:
        ref = e.compute_regions(b)
        chosen = e.autotune(b, repeats=2)
        assert chosen
        for c in chosen:
            assert 1 <= c["rows_per_lane"] <= 8 and c["haps_per_warp"] in (1, 2)
            assert 1 <= c["warps_per_block"] <= 4 and c["ms"] > 0
        assert {(c["rows_per_lane"], c["haps_per_warp"], c["warps_per_block"]) for c in chosen} <= \
            {(t["rows_per_lane"], t["haps_per_warp"], t["warps_per_block"]) for t in e.tuning()}
        assert np.array_equal(e.compute_regions(b), ref)
        e.set_tuning([{"rows_per_lane": rt, "haps_per_warp": 1, "warps_per_block": 1} for rt in range(1, 9)])
        assert np.array_equal(e.compute_regions(b), ref)
        with pytest.raises(RuntimeError):
            e.set_tuning([{"rows_per_lane": 9, "haps_per_warp": 1, "warps_per_block": 1}])
        with pytest.raises(RuntimeError):
            e.set_tuning([{"rows_per_lane": 3, "haps_per_warp": 3, "warps_per_block": 1}])


@pytest.mark.parametrize("chunks", [2, 3, 5])
def test_chunked_compute_matches_single_pass(chunks):
    """bv_phmm_compute_regions on a batch at or above the chunking threshold
    splits the regions into chunks that alternate between two contexts; every
    result equals the single-pass device-resident run, in full-DP and band
    mode, and the stats add up over the chunks."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    b = W.config1(seed=41, n_regions=40)
    with PairHMMEngine() as ref:
        n = ref.stage(b)
        ref.run()
        want = ref.fetch(n)
    with PairHMMEngine(pipeline_chunks=chunks, pipeline_min_pairs=1) as e:
        got, st = e.compute_regions(b, with_stats=True)
        assert np.array_equal(got, want)
        assert st["pairs"] == n and st["cells"] == b.n_cells()
        # again: the second context is reused
        assert np.array_equal(e.compute_regions(b), want)
        # band mode is mirrored into the second context
        e.set_band_options(fixed_half=8, margin=2)
        band, bst = e.compute_regions(b, with_stats=True)
    with PairHMMEngine() as one:
        one.set_band_options(fixed_half=8, margin=2)
        assert np.array_equal(band, one.compute_regions(b))
    assert bst["band_pairs"] > 0


def test_chunked_compute_rejects_an_invalid_chunk():
    """The chunked call validates each chunk's reads as it stages the chunk: a
    read whose offsets decrease in the last chunk fails the call with
    BV_ERR_INVALID_ARG, and the context stays usable."""
    import dataclasses
    from biovoltron_b200.pairhmm import PairHMMEngine
    b = W.config1(seed=43, n_regions=12)
    ro = b.read_offsets.copy()
    r = int(b.region_reads[-2]) + 1  # a read of the last region
    ro[r] = ro[r + 1] + 1
    bad = dataclasses.replace(b, read_offsets=ro)
    with PairHMMEngine(pipeline_chunks=3, pipeline_min_pairs=1) as e:
        with pytest.raises(RuntimeError, match="decrease"):
            e.compute_regions(bad)
        # the context stays usable
        with PairHMMEngine() as one:
            assert np.array_equal(e.compute_regions(b), one.compute_regions(b))


def test_chunked_compute_rejects_bad_options():
    from biovoltron_b200.pairhmm import PairHMMEngine
    with pytest.raises(RuntimeError):
        PairHMMEngine(pipeline_chunks=-1)
    with pytest.raises(RuntimeError):
        PairHMMEngine(pipeline_chunks=65)


def test_scalar_model_matches_reference_scalar_pairhmm():
    """Constant transitions (the scalar PairHMM model): the GPU result for the
    golden scalar cases is within FP32 tolerance of Biovoltron's scalar
    PairHMM (FP64), with the default and a custom transition matrix; turning
    the constants off gives the quality-derived results again."""
    from biovoltron_b200.pairhmm import ORIGINAL_DEFAULT, PairHMMEngine
    b, exp = load_golden("scalar")
    with PairHMMEngine() as e:
        plain = e.compute_regions(b)
        e.set_transitions(ORIGINAL_DEFAULT)
        assert e.transitions() == list(ORIGINAL_DEFAULT)
        got = e.compute_regions(b)
        want = exp["ref_scalar_default"]
        fin = np.isfinite(want)
        assert np.all(np.isneginf(got[~fin]))
        assert np.max(np.abs(got[fin] - want[fin])) <= TOL_FP32
        e.set_transitions([float(x) for x in exp["custom_trans"]])
        got = e.compute_regions(b)
        want = exp["ref_scalar_custom"]
        fin = np.isfinite(want)
        assert np.max(np.abs(got[fin] - want[fin])) <= TOL_FP32
        # the FP64 path with constants (precision f64 context)
        e.set_transitions(None)
        assert e.transitions() is None
        assert np.array_equal(e.compute_regions(b), plain)
        # the band path takes its transitions from the quality bytes
        e.set_band_options(fixed_half=8, margin=2)
        with pytest.raises(RuntimeError):
            e.set_transitions(ORIGINAL_DEFAULT)
    with PairHMMEngine(precision="f64") as e:
        e.set_transitions(ORIGINAL_DEFAULT)
        got = e.compute_regions(b)
        want = exp["ref_scalar_default"]
        fin = np.isfinite(want)
        assert np.max(np.abs(got[fin] - want[fin])) <= 1e-9
        with pytest.raises(RuntimeError):
            e.set_transitions([0.9998, 0.0001, 0.0001, 0.9, 0.1, 0.9, 1.5])


def test_scalar_drop_in_normalises_and_filters():
    """GpuScalarPairHMM mirrors PairHMM::compute_likelihoods: scalar-model
    likelihoods, normalised and filtered like the reference."""
    from biovoltron_b200.pairhmm import GpuScalarPairHMM, Haplotype, SamRecord
    from oracle.oracle import Oracle
    rng = np.random.default_rng(8)
    base = bytes(W._random_seq(rng, 300))
    haps = [Haplotype(base), Haplotype(base[:150] + b"T" + base[151:])]
    reads = [SamRecord(base[20:120], bytes(rng.integers(20, 41, 100).astype(np.uint8))),
             SamRecord(bytes(W._random_seq(rng, 80)), bytes([30] * 80))]
    raw = [[Oracle().scalar_log10(r.seq, r.qual, h.seq) for h in haps] for r in reads]
    keep = list(reads)
    ll = GpuScalarPairHMM().compute_likelihoods(haps, keep)
    exp = [list(row) for row in raw]
    from biovoltron_b200.pairhmm import filter_poorly_modeled_reads, normalize_likelihoods
    exp_reads = list(reads)
    normalize_likelihoods(exp)
    filter_poorly_modeled_reads(exp_reads, exp)
    assert [id(r) for r in keep] == [id(r) for r in exp_reads]
    assert np.allclose(np.array(ll), np.array(exp), rtol=0, atol=TOL_FP32)


@pytest.mark.parametrize("model", ["avx", "scalar"])
def test_region_batcher_equals_per_window_calls(model):
    """Windows queued in a RegionBatcher and scored in one call give the same
    normalised, filtered matrices (and the same kept reads) as one
    compute_likelihoods call per window."""
    from biovoltron_b200.pairhmm import GpuPairHMM, GpuScalarPairHMM, Haplotype, PairHMMEngine, RegionBatcher, SamRecord
    rng = np.random.default_rng(17)
    windows = []
    for w in range(6):
        base = bytes(W._random_seq(rng, int(rng.integers(200, 400))))
        haps = [Haplotype(base)] + [Haplotype(bytes(W._substitute(rng, np.frombuffer(base, np.uint8).copy(), 0.02)))
                                    for _ in range(int(rng.integers(0, 4)))]
        reads = []
        for _ in range(int(rng.integers(0, 12))):
            st = int(rng.integers(0, len(base) - 100))
            reads.append(SamRecord(base[st:st + 100], bytes(rng.integers(15, 41, 100).astype(np.uint8))))
        if w == 2:
            reads.append(SamRecord(bytes(W._random_seq(rng, 90)), bytes([30] * 90)))  # poorly modelled: kept
        windows.append((haps, reads))
    with PairHMMEngine() as e:
        one = GpuScalarPairHMM(engine=e) if model == "scalar" else GpuPairHMM(engine=e)
        want = []
        for haps, reads in windows:
            rr = list(reads)
            want.append((one.compute_likelihoods(haps, rr), [id(r) for r in rr]))
        bt = RegionBatcher(engine=e, model=model)
        lists = [list(reads) for _, reads in windows]
        hs = [bt.add(haps, lists[k]) for k, (haps, _) in enumerate(windows)]
        with pytest.raises(RuntimeError):
            bt.result(hs[0])
        bt.run()
        for k, h in enumerate(hs):
            ll, ids = want[k]
            assert [id(r) for r in lists[k]] == ids
            assert bt.result(h) == ll


@pytest.mark.parametrize("band", [False, True])
def test_device_genotyper_equals_reference_steps(band):
    """bv_phmm_genotype_staged on the staged batch's matrix equals, region by
    region, the reference's normalise / filter / overlap / marginalise /
    genotype-likelihood steps (restated in oracle/genotyper.py, pinned to
    the reference) applied to the same matrix, bit for bit."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    from oracle import genotyper as OG
    b = W.config1(seed=23, n_regions=30)
    rng = np.random.default_rng(5)
    nr, nh = np.diff(b.region_reads), np.diff(b.region_haps)
    A = rng.integers(1, 5, b.n_regions).astype(np.int32)
    hap_allele = np.concatenate([rng.integers(0, A[g], nh[g]) for g in range(b.n_regions)]).astype(np.int32)
    overlap = (rng.random(b.n_reads) < 0.85).astype(np.uint8)
    with PairHMMEngine() as e:
        if band:
            e.set_band_options(fixed_half=8, margin=2)
        n = e.stage(b)
        e.run()
        ll = e.fetch(n)
        out = e.genotype_staged(b, A, hap_allele, overlap)
    rl = np.diff(b.read_offsets)
    res = al_off = ge_off = 0
    for g in range(b.n_regions):
        r0, h0 = int(b.region_reads[g]), int(b.region_haps[g])
        m = ll[res:res + nr[g] * nh[g]].reshape(nr[g], nh[g])
        kept, al, ge = OG.genotype_window(m.tolist(), rl[r0:r0 + nr[g]].tolist(), overlap[r0:r0 + nr[g]].tolist(),
                                          int(A[g]), (hap_allele[h0:h0 + nh[g]]).tolist())
        k = int(out["kept_count"][g])
        assert k == len(kept)
        assert out["kept_reads"][r0:r0 + k].tolist() == [r0 + x for x in kept]
        assert np.array_equal(out["allele_lik"][al_off:al_off + k * A[g]], np.array(al).reshape(-1))
        assert np.array_equal(out["genotype_lik"][ge_off:ge_off + A[g] * (A[g] + 1) // 2], np.array(ge))
        res += nr[g] * nh[g]
        al_off += nr[g] * A[g]
        ge_off += A[g] * (A[g] + 1) // 2
    assert out["kernel_ms"] > 0


def test_uniform_gap_penalties_equal_per_base_arrays():
    """A batch passed without its i, d, c arrays (uniform gap penalties, the
    way SamRecord's constant views are sent) scores exactly as with the
    per-base arrays: full DP, band mode, and the chunked call over two
    contexts; giving only some of the three arrays is rejected."""
    import ctypes as C
    from biovoltron_b200.native import NativeError
    from biovoltron_b200.pairhmm import PairHMMEngine, _BatchView
    b = W.config4(seed=5, n_regions=40)
    g = b.uniform_gaps()
    assert g == (45, 45, 10)
    with PairHMMEngine() as e:
        want = e.compute_regions(b)
        assert np.array_equal(e.compute_regions(b, uniform_gaps=g), want)
        n = e.stage(b, uniform_gaps=g)
        e.run()
        assert np.array_equal(e.fetch(n), want)
        e.set_band_options(fixed_half=8, margin=2)
        band = e.compute_regions(b)
        assert np.array_equal(e.compute_regions(b, uniform_gaps=g), band)
        v = _BatchView(b)
        v.c.read_d = None
        out = np.empty(n, np.float64)
        assert e.lib.bv_phmm_compute_regions(e.h, C.byref(v.c), out.ctypes.data, None) == 1
    with PairHMMEngine(pipeline_chunks=3, pipeline_min_pairs=1) as e:
        assert np.array_equal(e.compute_regions(b, uniform_gaps=g), want)
        e.set_band_options(fixed_half=8, margin=2)
        assert np.array_equal(e.compute_regions(b, uniform_gaps=g), band)
    # a batch whose gap bytes differ per base is not uniform
    c1 = W.config0(0)
    c1.read_i = c1.read_i.copy()
    c1.read_i[3] = 40
    assert c1.uniform_gaps() is None


def test_multi_context_split_equals_one_context():
    """bv_phmm_compute_regions_multi over three contexts (on one GPU here; one
    per GPU in use) returns the single-context results in region order, in
    full-DP and band mode, and refuses a context given twice."""
    from biovoltron_b200.native import NativeError
    from biovoltron_b200.pairhmm import PairHMMEngine, compute_regions_multi
    b = W.config1(seed=51, n_regions=30)
    with PairHMMEngine() as one:
        want = one.compute_regions(b)
        one.set_band_options(fixed_half=8, margin=2)
        want_band = one.compute_regions(b)
    engines = [PairHMMEngine() for _ in range(3)]
    try:
        got, st = compute_regions_multi(engines, b, with_stats=True)
        assert np.array_equal(got, want)
        assert st["pairs"] == b.n_pairs and st["cells"] == b.n_cells()
        for e in engines:
            e.set_band_options(fixed_half=8, margin=2)
        assert np.array_equal(compute_regions_multi(engines, b, uniform_gaps=b.uniform_gaps()), want_band)
        with pytest.raises(NativeError):
            compute_regions_multi([engines[0], engines[0]], b)
    finally:
        for e in engines:
            e.close()
