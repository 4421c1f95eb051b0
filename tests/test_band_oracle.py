"""The banded-DP and posterior-spread definitions in the oracle (the learned
band path): a band wide enough to hold the whole matrix reproduces the full
DP, narrowing the band only loses probability, and the forward-backward
posterior concentrates on the diagonal the read was sampled from."""
import numpy as np

from biovoltron_b200 import workloads as W
from oracle.oracle import TestcaseArray


def _pairs(seed, n=6):
    rng = np.random.default_rng(seed)
    out, offs = [], []
    for _ in range(n):
        H = int(rng.integers(150, 400))
        hap = bytes(W._random_seq(rng, H))
        R = int(rng.integers(40, min(150, H - 10)))
        o = int(rng.integers(0, H - R))
        read = bytes(W._substitute(rng, np.frombuffer(hap[o:o + R], np.uint8), 0.02))
        q = bytes(rng.integers(10, 41, size=R).astype(np.uint8))
        out.append((read, q, bytes([45]) * R, bytes([45]) * R, bytes([10]) * R, hap))
        offs.append(o)
    return W.from_pairs(out), np.array(offs)


def test_full_width_band_equals_full_dp(oracle):
    b, _ = _pairs(1)
    tcs = TestcaseArray.for_batch(b)
    full = oracle.log10_rescaled(tcs)
    R, H = b.read_lengths(), b.hap_lengths()
    band = oracle.band_log10(tcs, -R, R + H + 1)
    assert np.max(np.abs(band - full)) < 1e-10


def test_band_is_a_lower_bound_and_tight_on_the_true_diagonal(oracle):
    b, offs = _pairs(2)
    tcs = TestcaseArray.for_batch(b)
    full = oracle.log10_rescaled(tcs)
    for w, tol in ((4, 5e-2), (16, 1e-6)):
        band = oracle.band_log10(tcs, offs - w, 2 * w + 1)
        assert np.all(band <= full + 1e-12)
        assert np.max(full - band) < tol
    off = oracle.band_log10(tcs, offs + 40, 9)  # a band that misses the alignment
    assert np.all(full - off > 5)


def test_posterior_peaks_on_the_sampled_diagonal(oracle):
    b, offs = _pairs(3)
    tcs = TestcaseArray.for_batch(b)
    for k in range(tcs.n):
        dmin, p = oracle.posterior_diag(tcs, k)
        assert p is not None
        assert int(np.argmax(p)) + dmin == offs[k]
        assert p.max() > 0.9
        far = np.abs(np.arange(len(p)) + dmin - offs[k]) > 20
        assert p[far].max() < 1e-6
