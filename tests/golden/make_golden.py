"""Generates the golden PairHMM fixtures in this directory.

Run from the repository root, naming the reference tree (the directory
that holds Biovoltron's include/, lib/ and tests/):

    make -C oracle REF=<reference tree> &&
    python tests/golden/make_golden.py --ref <reference tree>

Every expected value is produced by Biovoltron's own PairHMM kernel
(lib/intel_native/pairhmm, compiled by oracle/Makefile into
oracle/_ref/libref_pairhmm.so), called the way AvxPairHMM calls it
(pairhmm_avx.hpp:136-149): FP32, FP64 below 1e-28, log10 minus the scale.
Inputs are stored in the fixtures, so tests need neither the reference tree
nor this script.

Fixtures:
  config0.npz     the 64 x 8 region of config 0 (seed 0)
  edge_cases.npz  hand-built pairs: 1x1 match/mismatch, N reads/haps, unknown
                  bytes, extreme and >127 quals, pure indels, forced FP64 rescue
  ref_test.npz    the sequences of the reference's own AvxPairHMM test
                  (tests/algo/align/inexact_match/pairhmm_avx.cpp), read from
                  that file, scored with full-length SAM penalty arrays
  long_pairs.npz  a few config-2-shaped pairs (1-2 kb reads, 8% subs); the
                  reference's FP64 underflows on most, so the expected values
                  are the rescaled FP64 oracle, cross-checked against the
                  reference wherever the reference is finite
  config4_small.npz  two regions of the headline workload's shape (config 4:
                  150 bp reads at 30x, 2-16 haplotypes of ~450 bp, seed 44)
  scalar.npz      the scalar PairHMM model (pairhmm.hpp, compiled by
                  oracle/Makefile into oracle/_ref/libref_scalar.so): a small
                  region and edge pairs, expected log10 values with
                  ORIGINAL_DEFAULT and with one custom transition matrix
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from biovoltron_b200 import workloads as W  # noqa: E402
from oracle.oracle import Oracle, Reference, ReferenceScalar, TestcaseArray  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF_TEST_REL = os.path.join("tests", "algo", "align", "inexact_match", "pairhmm_avx.cpp")

BATCH_FIELDS = ("read_bases", "read_q", "read_i", "read_d", "read_c", "read_offsets", "hap_bases", "hap_offsets",
                "region_reads", "region_haps")


def save(name, batch, ref, oracle, extra=None):
    tcs = TestcaseArray.for_batch(batch)
    log10, used = ref.log10(tcs)
    pf = ref.prob_f32(tcs)
    pd = ref.prob_f64(tcs)
    resc = oracle.log10_rescaled(tcs)
    d = {k: getattr(batch, k) for k in BATCH_FIELDS}
    d.update(ref_log10=log10, ref_used_f64=used, ref_prob_f32=pf, ref_prob_f64=pd, oracle_rescaled=resc)
    if extra:
        d.update(extra)
    np.savez_compressed(os.path.join(HERE, name), **d)
    print(f"{name}: {batch.n_pairs} pairs, {int(used.sum())} FP64, "
          f"log10 range [{np.min(log10[np.isfinite(log10)]) if np.isfinite(log10).any() else 'n/a'}, {np.max(log10)}]")


def edge_batch() -> W.RegionBatch:
    rng = np.random.default_rng(7)
    P = []
    def q(n, v):
        return bytes([v]) * n
    # 1x1 match and mismatch at Q30
    P.append((b"A", q(1, 30), q(1, 45), q(1, 45), q(1, 10), b"A"))
    P.append((b"A", q(1, 30), q(1, 45), q(1, 45), q(1, 10), b"C"))
    # 2x2, 3x1, 1x3
    P.append((b"AC", q(2, 20), q(2, 40), q(2, 40), q(2, 10), b"AC"))
    P.append((b"ACG", q(3, 20), q(3, 40), q(3, 40), q(3, 10), b"G"))
    P.append((b"G", q(1, 20), q(1, 40), q(1, 40), q(1, 10), b"ACG"))
    # all-N read; N in haplotype; unknown and lowercase bytes (read as A)
    P.append((b"N" * 40, q(40, 30), q(40, 45), q(40, 45), q(40, 10), bytes(W._random_seq(rng, 90))))
    hap = bytearray(W._random_seq(rng, 120)); hap[30:40] = b"N" * 10
    P.append((bytes(hap[20:80]), q(60, 25), q(60, 45), q(60, 45), q(60, 10), bytes(hap)))
    P.append((b"acgtxACGT-" * 5, q(50, 30), q(50, 45), q(50, 45), q(50, 10), b"AAAAACGTAAACGT" * 8))
    # identical read/hap at Q40
    s = bytes(W._random_seq(rng, 150))
    P.append((s, q(150, 40), q(150, 45), q(150, 45), q(150, 10), s))
    # quals 0 and 127, and bytes >127 (masked to 0..127 by the kernel)
    qa = bytes(rng.integers(0, 128, size=100).astype(np.uint8))
    qb = bytes((rng.integers(0, 256, size=100)).astype(np.uint8))
    hh = bytes(W._random_seq(rng, 200))
    P.append((hh[50:150], qa, qa[::-1], qb, qa, hh))
    P.append((hh[40:140], q(100, 0), q(100, 0), q(100, 0), q(100, 0), hh))
    P.append((hh[40:140], q(100, 127), q(100, 127), q(100, 127), q(100, 127), hh))
    P.append((hh[40:140], qb, qb, qb, qb, hh))
    # pure insertion / pure deletion
    base = bytes(W._random_seq(rng, 300))
    ins = base[100:150] + b"TTTTT" + base[150:195]
    P.append((ins, q(100, 30), q(100, 45), q(100, 45), q(100, 10), base))
    dele = base[100:150] + base[160:210]
    P.append((dele, q(100, 30), q(100, 45), q(100, 45), q(100, 10), base))
    # forced FP64 rescue: a read against an unrelated haplotype (log10 << -64)
    r = bytes(W._random_seq(rng, 120)); h2 = bytes(W._random_seq(rng, 250))
    P.append((r, q(120, 35), q(120, 45), q(120, 45), q(120, 10), h2))
    # read longer than the haplotype; strip boundaries (32*k rows +-1)
    h3 = bytes(W._random_seq(rng, 100))
    P.append((h3 + h3[:60], q(160, 30), q(160, 45), q(160, 45), q(160, 10), h3))
    for n in (31, 32, 33, 63, 64, 65, 255, 256, 257, 300):
        hx = bytes(W._random_seq(rng, n + 80))
        rx = bytes(W._substitute(rng, np.frombuffer(hx[40:40 + n], np.uint8), 0.02))
        qx = bytes(rng.integers(10, 41, size=n).astype(np.uint8))
        P.append((rx, qx, q(n, 45), q(n, 45), q(n, 10), hx))
    # haplotype longer than 1000 (wavefront over many steps)
    hl = bytes(W._random_seq(rng, 1500))
    P.append((hl[700:850], bytes(rng.integers(10, 41, size=150).astype(np.uint8)), q(150, 45), q(150, 45), q(150, 10), hl))
    return W.from_pairs(P, "edge cases")


def ref_test_batch(ref_test: str) -> W.RegionBatch:
    src = open(ref_test).read()
    strings = re.findall(r'"([ACGTN]{500,})"', src)
    ref_seq = strings[0]
    haps = strings[1:9]
    # Mutations applied to the subject in that test: 5-base substitution at
    # 150..154, an inserted T at 300 and a deletion at 800.
    subject = list(ref_seq)
    for i in range(150, 155):
        subject[i] = "T"
    subject.insert(300, "T")
    del subject[800]
    subject = "".join(subject)
    reads = [subject[100:100 + 200], subject[200:200 + 400], subject[700:700 + 900]]
    regions = []
    for rd in reads:
        n = len(rd)
        b = np.frombuffer(rd.encode(), np.uint8).copy()
        qual = np.full(n, ord(";"), np.uint8)
        gop = np.full(n, 40 + 33, np.uint8)
        gcp = np.full(n, 10 + 33, np.uint8)
        regions.append(([(b, qual, gop, gop.copy(), gcp)], [np.frombuffer(h.encode(), np.uint8).copy() for h in haps]))
    return W._build(regions, "reference AvxPairHMM test sequences")


SCALAR_CUSTOM = (0.995, 0.003, 0.002, 0.85, 0.15, 0.7, 0.3)


def scalar_batch() -> W.RegionBatch:
    """A config-0-shaped region (16 reads x 4 haplotypes) and edge pairs,
    upper-case A/C/G/T/N only (the scalar model compares raw bytes)."""
    rng = np.random.default_rng(21)
    base = W._random_seq(rng, 300)
    haps = [W._apply_indels(rng, W._substitute(rng, base, 0.01), int(rng.integers(0, 3)), 1, 10) for _ in range(4)]
    reads = []
    for _ in range(16):
        src = haps[int(rng.integers(0, 4))]
        st = int(rng.integers(0, len(src) - 150 + 1))
        b = W._substitute(rng, src[st:st + 150].copy(), 0.01)
        q = rng.integers(10, 41, size=150).astype(np.uint8)
        reads.append((b, q, q, q, q))
    regions = [(reads, haps)]

    def arr(x):
        return np.frombuffer(x, np.uint8).copy()

    def pair(read, qual, hap):
        r, q = arr(read), np.full(len(read), qual, np.uint8) if isinstance(qual, int) else arr(qual)
        return ([(r, q, q, q, q)], [arr(hap)])

    regions += [pair(b"A", 30, b"A"), pair(b"A", 30, b"C"), pair(b"N" * 20, 30, b"ACGTACGTACGTACGTACGTACGT"),
                pair(b"ACGTACGTAC", 30, b"NNNNNNNNNNNN"), pair(b"ACGTACGTACGT", 0, b"ACGTACGTACGT"),
                pair(b"ACGTACGTACGT", 127, b"ACGTACGTACGT"),
                pair(b"ACGTAAAAACGTTT", 35, b"ACGTACGTTT"),        # insertion in the read
                pair(b"ACGTACGTTT", 35, b"ACGTAAAAACGTTT"),        # deletion from the read
                pair(b"GATTACA", bytes([5, 15, 25, 35, 45, 55, 65]), b"TTGATTACATT"),
                pair(b"ACGTTGCA" * 4, 25, b"A")]
    return W._build(regions, "scalar model cases")


def save_scalar(name, batch, ref_scalar):
    r, h = batch.pair_index()
    ro, ho = batch.read_offsets, batch.hap_offsets
    exp_d, exp_c = [], []
    for k in range(len(r)):
        rd = bytes(batch.read_bases[ro[r[k]]:ro[r[k] + 1]])
        q = bytes(batch.read_q[ro[r[k]]:ro[r[k] + 1]])
        hp = bytes(batch.hap_bases[ho[h[k]]:ho[h[k] + 1]])
        exp_d.append(ref_scalar.log10(rd, q, hp))
        exp_c.append(ref_scalar.log10(rd, q, hp, SCALAR_CUSTOM))
    d = {k: getattr(batch, k) for k in BATCH_FIELDS}
    d.update(ref_scalar_default=np.array(exp_d), ref_scalar_custom=np.array(exp_c),
             custom_trans=np.array(SCALAR_CUSTOM))
    np.savez_compressed(os.path.join(HERE, name), **d)
    print(f"{name}: {batch.n_pairs} pairs")


def main():
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference tree (holds include/, lib/ and tests/)")
    args = ap.parse_args()
    ref_test = os.path.join(args.ref, REF_TEST_REL)
    ref = Reference()
    oracle = Oracle()
    save("config0.npz", W.config0(0), ref, oracle)
    save("edge_cases.npz", edge_batch(), ref, oracle)
    if os.path.exists(ref_test):
        save("ref_test.npz", ref_test_batch(ref_test), ref, oracle)
    save("long_pairs.npz", W.config2(seed=11, n_pairs=6, max_read=2000, max_hap=2600), ref, oracle)
    save("config4_small.npz", W.config4(seed=44, n_regions=2), ref, oracle)
    save_scalar("scalar.npz", scalar_batch(), ReferenceScalar())


if __name__ == "__main__":
    main()
