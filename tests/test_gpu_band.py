"""The banded path on the GPU.

* With a fixed band around the 11-mer seed diagonal, every banded pair's
  result equals the oracle's banded DP on that band widened by the ring test's
  four (W = 8) or eight diagonals on each side (FP32 tolerance).
* Routed-out and fallback pairs equal the full DP.
* The audit compares banded against full results on a sample.
"""
import numpy as np
import pytest

from biovoltron_b200 import workloads as W
from oracle.oracle import TestcaseArray, seed_diagonal, seed_extent

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-4
TOL_CONTRACT = 1e-3


def _band_engine(**kw):
    from biovoltron_b200.pairhmm import PairHMMEngine
    e = PairHMMEngine(device=0)
    e.set_band_options(**kw)
    return e


def test_fixed_band_matches_oracle_band(oracle):
    b = W.config1(seed=31, n_regions=6)
    half, margin = 6, 1
    # the banded kernel's own values: no rescore of pairs far below their read's best
    with _band_engine(fixed_half=half, margin=margin, edge_threshold=1e30, cap_margin=0.0) as e:
        got, st = e.compute_regions(b, with_stats=True)
    assert st["band_pairs"] > 0.8 * b.n_pairs
    r, h = b.pair_index()
    tcs = TestcaseArray.for_batch(b)
    d_lo, wcls, sel = [], [], []
    for k in range(len(r)):
        rd, hp = b.read(int(r[k]))[0], b.hap(int(h[k]))
        ds = seed_diagonal(rd, hp)
        if ds is None or b.read_lengths()[r[k]] > 511:
            continue
        km, kx = seed_extent(rd, hp)
        blo, bhi = min(ds - half - margin, km), max(ds + half + margin, kx)
        width = bhi - blo + 1
        if width > 32:
            continue
        W_cls = 8 * ((width - 1) // 8 + 1)  # classes of 8, 16, 24 and 32 diagonals
        d_lo.append(blo - (W_cls - width) // 2)
        wcls.append(W_cls)
        sel.append(k)
    sel = np.array(sel)
    sub = TestcaseArray(b, r[sel], h[sel])
    # the result is the band widened by the ring (4 diagonals on each side, 8 from W = 16)
    ring = np.where(np.array(wcls) >= 16, 8, 4)
    exp = oracle.band_log10(sub, np.array(d_lo) - ring, np.array(wcls) + 2 * ring)
    fin = np.isfinite(exp) & (exp > -60)
    assert np.max(np.abs(got[sel][fin] - exp[fin])) <= TOL_FP32


def test_fixed_band_audit_reports_banded_error(oracle):
    # The fixed band is the ablation of the learned band: it may leave the
    # contract on pairs whose alignment spreads beyond it.  The audit must
    # see exactly the banded-vs-full differences of its sampled pairs.
    b = W.config1(seed=32, n_regions=8)
    period = 7
    with _band_engine(fixed_half=8, margin=2, edge_threshold=1e-3, audit_period=period) as e:
        got, st = e.compute_regions(b, with_stats=True)
    truth = oracle.log10_rescaled(TestcaseArray.for_batch(b))
    assert np.all(np.isfinite(got))
    err = np.abs(got - truth)
    sampled = err[::period]
    assert st["audit_pairs"] > 0
    assert st["audit_max_err"] <= sampled.max() + 1e-4
    assert st["band_pairs"] + st["band_routed_full"] == b.n_pairs


def test_band_mode_edge_cases_equal_full(engine):
    # no shared 11-mer, short reads and long reads all go to the full DP
    # (config0's ordinary pairs are held to the contract with the learned band)
    from conftest import load_golden
    for name in ("edge_cases", "long_pairs"):
        b, exp = load_golden(name)
        full = engine.compute_regions(b)
        with _band_engine(fixed_half=8, margin=2) as e:
            got, st = e.compute_regions(b, with_stats=True)
        truth = exp["oracle_rescaled"]
        fin = np.isfinite(truth)
        assert np.all(np.isneginf(got[~fin]))
        assert np.max(np.abs(got[fin] - truth[fin])) <= TOL_CONTRACT


def test_band_staged_replay_is_deterministic():
    b = W.config1(seed=33, n_regions=10)
    with _band_engine(fixed_half=8, margin=2, audit_period=5) as e:
        direct = e.compute_regions(b)
        n = e.stage(b)
        for _ in range(3):
            st = e.run()
            assert st["band_pairs"] > 0
            assert np.array_equal(e.fetch(n), direct)


def test_uniform_gap_rows_equal_the_general_rows():
    """A batch whose read bases all carry the same insertion, deletion and
    gap-continuation qualities lets the banded kernels take every row's
    transition constants from one set.  Changing one base's insertion quality
    (of the batch's last read) turns that off; every pair of the other reads
    must then come out bit for bit the same."""
    import dataclasses
    b = W.config1(seed=35, n_regions=8)
    assert b.uniform_gaps() is not None
    ri = b.read_i.copy()
    ri[-1] = 40
    b2 = dataclasses.replace(b, read_i=ri)
    assert b2.uniform_gaps() is None
    with _band_engine(fixed_half=8, margin=2) as e:
        uni, st1 = e.compute_regions(b, with_stats=True)
        gen, st2 = e.compute_regions(b2, with_stats=True)
    r, _ = b.pair_index()
    other = r != b.n_reads - 1
    assert st1["band_pairs"] > 0.8 * b.n_pairs and st2["band_pairs"] == st1["band_pairs"]
    assert np.array_equal(uni[other], gen[other])
    assert not np.array_equal(uni[~other], gen[~other])


def _repeat_pairs(seed):
    """Pairs whose sampled 11-mers vote for many diagonals: haplotypes made of
    a repeated unit (period 40 and 25), reads cut from them with a few
    substitutions; the unit featuriser hands these to the slow featuriser."""
    rng = np.random.default_rng(seed)
    out = []
    for period, copies, n in ((40, 10, 150), (25, 16, 120), (40, 6, 90)):
        unit = W._random_seq(rng, period)
        hap = np.tile(unit, copies)
        hap = W._substitute(rng, hap, 0.005)
        start = int(rng.integers(0, len(hap) - n))
        read = W._substitute(rng, hap[start:start + n], 0.01)
        q = rng.integers(10, 41, size=n).astype(np.uint8)
        out.append((bytes(read), bytes(q), bytes([45]) * n, bytes([45]) * n, bytes([10]) * n, bytes(hap)))
    return W.from_pairs(out, "repeats")


def test_features_match_oracle_restatement():
    """Every pair's 80 MLP inputs, seed diagonal and voted extent equal the
    oracle's restatement of the featuriser bit for bit: config-1- and
    config-4-shaped regions (thread per pair) and repeat-rich pairs (the warp
    featuriser's list)."""
    from biovoltron_b200.pairhmm import PairHMMEngine
    from oracle.oracle import seed_features
    batches = [W.config1(seed=43, n_regions=3), W.config4(seed=7, n_regions=3), _repeat_pairs(3)]
    for b in batches:
        with PairHMMEngine(device=0) as e:
            ds, _, _, feat, km, kx = e.band_labels(b, tau=1e-4, features=True, extent=True)
        r, h = b.pair_index()
        for k in range(b.n_pairs):
            rd, hp = b.read(int(r[k]))[0], b.hap(int(h[k]))
            exp_ds = seed_diagonal(rd, hp)
            assert ds[k] == (np.iinfo(np.int32).min if exp_ds is None else exp_ds), (b.name, k)
            if exp_ds is not None and len(rd) <= 511:
                assert (km[k], kx[k]) == seed_extent(rd, hp), (b.name, k)
            if len(rd) <= 511 and len(hp) <= 1024:
                f = seed_features(rd, hp)
                assert np.array_equal(feat[k], f), (b.name, k, np.nonzero(feat[k] != f)[0], feat[k][feat[k] != f],
                                                    f[feat[k] != f])
