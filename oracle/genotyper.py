"""CPU restatement of the genotyper steps that consume the PairHMM matrix
(test infrastructure).

What HaplotypeCaller does with one window's raw [read][hap] log10 matrix:
  * PairHMM::normalize_likelihoods: every value capped below at the read's
    best - 4.5 (include/biovoltron/algo/align/inexact_match/pairhmm.hpp:83-93);
  * PairHMM::filter_poorly_modeled_reads: keeps the reads whose best value is
    below min(2, ceil(0.02 len)) * -4 -- the reference's comparison (:95-114);
  * the genotyper keeps the remaining reads that overlap the site
    (genotyper.hpp:212-221; here an overlap mask over the window's reads);
  * Genotyper::marginal_likelihoods: per kept read and allele, the largest
    value over the haplotypes mapped to the allele, lowest() when none
    (genotyper.hpp:223-240);
  * diploid genotype likelihoods, genotypes (a1 <= a2) in order: the sum over
    kept reads of L[a] + log10(2) (a1 == a2) or
    MathUtils::approximate_log10_sum_log10(L[a1], L[a2]), minus
    kept * log10(2) (genotyper.hpp:254-315);
  * approximate_log10_sum_log10(a, b): with a <= b, b + table[round((b - a) /
    1e-4)] when b - a < 8, else b; table[i] = log10(1 + 10^(-1e-4 i))
    (math_utils.hpp:112-139).
Sums run read by read in order, as std::accumulate does.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

TABLE_STEP = 0.0001
MAX_TOLERANCE = 8.0
INV_STEP = 1.0 / TABLE_STEP
LOWEST = -1.7976931348623157e308
LOG10_2 = math.log10(2)

_table = None


def jacobian_table() -> List[float]:
    """log10(1 + 10^(-1e-4 i)), each step correctly rounded to double (the
    reference builds the table at compile time, where the compiler evaluates
    pow and log10 exactly before rounding)."""
    global _table
    if _table is None:
        import mpmath
        mpmath.mp.prec = 200
        n = int(MAX_TOLERANCE / TABLE_STEP) + 1
        t = []
        for i in range(n):
            x = -TABLE_STEP * i
            pw = float(mpmath.power(10, mpmath.mpf(x)))
            t.append(float(mpmath.log10(mpmath.mpf(1.0 + pw))))
        _table = t
    return _table


def approximate_log10_sum_log10(a: float, b: float) -> float:
    if a > b:
        a, b = b, a
    diff = b - a
    if diff < MAX_TOLERANCE:
        x = diff * INV_STEP
        idx = int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))  # round half away from zero
        return b + jacobian_table()[idx]
    return b


def genotype_window(ll: Sequence[Sequence[float]], read_len: Sequence[int], overlap: Sequence[int],
                    allele_count: int, hap_allele: Sequence[int]) -> Tuple[List[int], List[List[float]], List[float]]:
    """Returns (kept original read indices, allele likelihoods [kept][A],
    genotype likelihoods [A (A + 1) / 2])."""
    m = [list(map(float, row)) for row in ll]
    for row in m:  # normalize
        if row:
            cap = max(row) - 4.5
            for h, v in enumerate(row):
                if v < cap:
                    row[h] = cap
    survivors = []
    for r, row in enumerate(m):  # filter (the reference's comparison)
        best = max(row)
        thr = min(2.0, math.ceil(read_len[r] * 0.02)) * -4.0
        if best < thr:
            survivors.append(r)
    kept = [r for r in survivors if overlap[r]]
    al = []
    for r in kept:
        row = [LOWEST] * allele_count
        for h, v in enumerate(m[r]):
            a = hap_allele[h]
            if v > row[a]:
                row[a] = v
        al.append(row)
    geno = []
    for a1 in range(allele_count):
        for a2 in range(a1, allele_count):
            s = 0.0
            for row in al:
                s += (row[a1] + LOG10_2) if a1 == a2 else approximate_log10_sum_log10(row[a1], row[a2])
            geno.append(s - len(al) * LOG10_2)
    return kept, al, geno
