/*
 * pairhmm_oracle.c -- CPU oracle for the PairHMM forward pass.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is never linked into the product library, and only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * It restates, in plain scalar C, the arithmetic of Biovoltron's Intel-derived
 * PairHMM kernel and of its AvxPairHMM wrapper:
 *
 *   tables          lib/intel_native/pairhmm/Context.h:42-61 (Jacobian and
 *                   match-to-match tables), :67-90 (approximateLog10SumLog10),
 *                   :97-175 (ph2pr, INITIAL_CONSTANT, set_mm_prob)
 *   base codes      lib/intel_native/pairhmm/pairhmm_common.h:26-44
 *   match rule      lib/intel_native/pairhmm/avx-pairhmm-template.h:3-35
 *   per-row probs   avx-pairhmm-template.h:83-128, 150-158
 *   recurrence      avx-pairhmm-template.h:183-198 (computeMXY)
 *   initial row     avx-pairhmm-template.h:86-91, 151, 167 (Y = INITIAL/haplen)
 *   result          avx-pairhmm-template.h:308-343 (sum M, sum X, then add)
 *   rescue + log10  include/biovoltron/algo/align/inexact_match/pairhmm_avx.hpp:136-149
 *   scalar model    include/biovoltron/algo/align/inexact_match/pairhmm.hpp:39-80
 *
 * Every cell is evaluated with the same IEEE operations in the same order as
 * the reference's vector code (mul, add, no fused multiply-add; flush-to-zero
 * on, as AvxPairHMM::initNative sets it), so orc_prob_f32/orc_prob_f64 are
 * bit-identical to compute_full_prob_avxs/avxd when this file is compiled with
 * -ffp-contract=off.  That identity is checked by tests against the reference
 * kernel compiled from its own sources (oracle/_ref) and against committed
 * golden vectors generated from it.
 *
 * orc_log10_rescaled is an FP64 variant that renormalises every row by an
 * exact power of two and carries the exponent, so pairs whose likelihood lies
 * below the FP64 range (reads of several kilobases) still get a finite log10.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_QUAL 254
#define ORC_JAC_TOL 8.0
#define ORC_JAC_STEP 0.0001
#define ORC_JAC_INV_STEP (1.0 / ORC_JAC_STEP)
#define ORC_JAC_SIZE 80001 /* (int)(ORC_JAC_TOL / ORC_JAC_STEP) + 1, Context.h:10 */
#define ORC_MM_SIZE (((ORC_MAX_QUAL + 1) * (ORC_MAX_QUAL + 2)) >> 1)
#define ORC_MIN_ACCEPTED 1e-28f

/* Same field order as the reference's testcase (pairhmm_common.h:20-24). */
typedef struct {
    int rslen, haplen;
    const char *q, *i, *d, *c;
    const char *hap, *rs;
} orc_testcase;

static float jac_f[ORC_JAC_SIZE];
static double jac_d[ORC_JAC_SIZE];
static float mm_f[ORC_MM_SIZE];
static double mm_d[ORC_MM_SIZE];
static float ph2pr_f[128];
static double ph2pr_d[128];
static float init_f, log10_init_f;
static double init_d, log10_init_d;
static uint8_t base_code[256];
static int initialised = 0;

/* Context.h:67-70 */
static int fast_round_f(float d) { return (d > 0.0f) ? (int)(d + 0.5f) : (int)(d - 0.5f); }
static int fast_round_d(double d) { return (d > 0.0) ? (int)(d + 0.5) : (int)(d - 0.5); }

/* Context.h:72-90.  The -inf early return there compares a C++ bool with -1
 * and can never fire; the arguments used here are finite in any case. */
static float approx_log10_sum_f(float small, float big) {
    if (small > big) { float t = big; big = small; small = t; }
    float diff = big - small;
    if (diff >= (float)ORC_JAC_TOL) return big;
    int ind = fast_round_f((float)(diff * (float)ORC_JAC_INV_STEP));
    return big + jac_f[ind];
}
static double approx_log10_sum_d(double small, double big) {
    if (small > big) { double t = big; big = small; small = t; }
    double diff = big - small;
    if (diff >= (double)ORC_JAC_TOL) return big;
    int ind = fast_round_d((double)(diff * (double)ORC_JAC_INV_STEP));
    return big + jac_d[ind];
}

void orc_init(void) {
    if (initialised) return;
    /* Context.h:42-47 */
    for (int k = 0; k < ORC_JAC_SIZE; k++) {
        double v = log10(1.0 + pow(10.0, -((double)k) * ORC_JAC_STEP));
        jac_f[k] = (float)v;
        jac_d[k] = v;
    }
    /* Context.h:50-61: built per precision, the log-sum evaluated in that precision */
    double ln10 = log(10);
    double inv_ln10 = 1.0 / ln10;
    for (int i = 0, off = 0; i <= ORC_MAX_QUAL; off += ++i) {
        for (int j = 0; j <= i; j++) {
            double s_f = (double)approx_log10_sum_f((float)(-0.1 * i), (float)(-0.1 * j));
            double l_f = log1p(-fmin(1.0, pow(10, s_f))) * inv_ln10;
            mm_f[off + j] = (float)pow(10, l_f);
            double s_d = approx_log10_sum_d(-0.1 * i, -0.1 * j);
            double l_d = log1p(-fmin(1.0, pow(10, s_d))) * inv_ln10;
            mm_d[off + j] = pow(10, l_d);
        }
    }
    /* Context.h:104-110 and :144-150 */
    for (int x = 0; x < 128; x++) {
        ph2pr_d[x] = pow(10.0, -((double)x) / 10.0);
        ph2pr_f[x] = powf(10.f, -((float)x) / 10.f);
    }
    init_d = ldexp(1.0, 1020);
    log10_init_d = log10(init_d);
    init_f = ldexpf(1.f, 120);
    log10_init_f = log10f(init_f);
    /* pairhmm_common.h:26-44: A0 C1 T2 G3 N4; every other byte reads as 0 (A). */
    memset(base_code, 0, sizeof base_code);
    base_code['A'] = 0; base_code['C'] = 1; base_code['T'] = 2; base_code['G'] = 3; base_code['N'] = 4;
    initialised = 1;
}

/* Context.h:121-133 / :161-173 (quals are masked to 0..127 by the caller, so
 * the table branch is the only one reachable). */
static float set_mm_prob_f(int ins, int del) {
    int mn = del, mx = ins;
    if (ins <= del) { mn = ins; mx = del; }
    return ORC_MAX_QUAL < mx ? 1.0f - powf(10.0f, approx_log10_sum_f(-0.1f * mn, -0.1f * mx))
                             : mm_f[((mx * (mx + 1)) >> 1) + mn];
}
static double set_mm_prob_d(int ins, int del) {
    int mn = del, mx = ins;
    if (ins <= del) { mn = ins; mx = del; }
    return ORC_MAX_QUAL < mx ? 1.0 - pow(10.0, approx_log10_sum_d(-0.1 * mn, -0.1 * mx))
                             : mm_d[((mx * (mx + 1)) >> 1) + mn];
}

static inline int is_match(uint8_t rc, uint8_t hc) { return rc == hc || rc == 4 || hc == 4; }

static void set_ftz(void) { _mm_setcsr(_mm_getcsr() | 0x8000); }

/*
 * One forward pass, rolling over rows.  T is float or double; the body is
 * instantiated twice by the macro below so that each precision uses exactly
 * the reference's operation sequence.
 */
#define ORC_FORWARD(T, NAME, PH2PR, MMFN, INIT)                                          \
    T NAME(const orc_testcase *tc) {                                                     \
        orc_init();                                                                      \
        set_ftz();                                                                       \
        const int R = tc->rslen, H = tc->haplen;                                         \
        T *buf = (T *)calloc((size_t)6 * (H + 1), sizeof(T));                            \
        T *Mp = buf, *Xp = buf + (H + 1), *Yp = buf + 2 * (H + 1);                       \
        T *Mc = buf + 3 * (H + 1), *Xc = buf + 4 * (H + 1), *Yc = buf + 5 * (H + 1);     \
        uint8_t *hc = (uint8_t *)malloc((size_t)H + 1);                                  \
        for (int j = 0; j < H; j++) hc[j] = base_code[(uint8_t)tc->hap[j]];              \
        const T init_y = INIT / (T)H;                                                    \
        for (int j = 0; j <= H; j++) Yp[j] = init_y;                                     \
        T sumM = 0, sumX = 0;                                                            \
        for (int r = 1; r <= R; r++) {                                                   \
            const int qi = tc->i[r - 1] & 127, qd = tc->d[r - 1] & 127;                  \
            const int qc = tc->c[r - 1] & 127, qq = tc->q[r - 1] & 127;                  \
            const T pMM = MMFN(qi, qd);                                                  \
            const T pGAPM = (T)1.0 - PH2PR[qc];                                          \
            const T pMX = PH2PR[qi], pXX = PH2PR[qc];                                    \
            const T pMY = PH2PR[qd], pYY = PH2PR[qc];                                    \
            const T distm0 = PH2PR[qq];                                                  \
            const T one_m = (T)1.0 - distm0;                                             \
            const T mis = distm0 / (T)3.0;                                               \
            const uint8_t rc = base_code[(uint8_t)tc->rs[r - 1]];                        \
            Mc[0] = 0; Xc[0] = 0; Yc[0] = 0;                                             \
            for (int j = 1; j <= H; j++) {                                               \
                const T e = is_match(rc, hc[j - 1]) ? one_m : mis;                       \
                T a = Mp[j - 1] * pMM;                                                   \
                T b = Xp[j - 1] * pGAPM;                                                 \
                T c = Yp[j - 1] * pGAPM;                                                 \
                Mc[j] = ((a + b) + c) * e;                                               \
                T xa = Mp[j] * pMX;                                                      \
                T xb = Xp[j] * pXX;                                                      \
                Xc[j] = xa + xb;                                                         \
                T ya = Mc[j - 1] * pMY;                                                  \
                T yb = Yc[j - 1] * pYY;                                                  \
                Yc[j] = ya + yb;                                                         \
            }                                                                            \
            T *t;                                                                        \
            t = Mp; Mp = Mc; Mc = t;                                                     \
            t = Xp; Xp = Xc; Xc = t;                                                     \
            t = Yp; Yp = Yc; Yc = t;                                                     \
            if (r == 1) { /* row 0's M and X were zero from calloc; keep them so */      \
                memset(Mc, 0, sizeof(T) * (H + 1));                                      \
                memset(Xc, 0, sizeof(T) * (H + 1));                                      \
            }                                                                            \
        }                                                                                \
        if (R == 0) { free(buf); free(hc); return 0; }                                   \
        for (int j = 1; j <= H; j++) sumM = sumM + Mp[j];                                \
        for (int j = 1; j <= H; j++) sumX = sumX + Xp[j];                                \
        T res = sumM + sumX;                                                             \
        free(buf);                                                                       \
        free(hc);                                                                        \
        return res;                                                                      \
    }

ORC_FORWARD(float, orc_prob_f32, ph2pr_f, set_mm_prob_f, init_f)
ORC_FORWARD(double, orc_prob_f64, ph2pr_d, set_mm_prob_d, init_d)

/*
 * computeLikelihoodsNative's per-pair rule (pairhmm_avx.hpp:140-149): FP32
 * first; below MIN_ACCEPTED (1e-28) recompute in FP64.  The FP32 log is taken
 * in single precision, exactly as the reference does.
 */
double orc_log10_reference_rule(const orc_testcase *tc, int *used_f64) {
    orc_init();
    float rf = orc_prob_f32(tc);
    if (rf < ORC_MIN_ACCEPTED) {
        double rd = orc_prob_f64(tc);
        if (used_f64) *used_f64 = 1;
        return log10(rd) - log10_init_d;
    }
    if (used_f64) *used_f64 = 0;
    return (double)(log10f(rf) - log10_init_f);
}

/*
 * FP64 forward pass with an exact power-of-two renormalisation of every row.
 * Same recurrence and tables as orc_prob_f64; FTZ is left off so nothing is
 * flushed.  Returns log10 of the (unscaled) likelihood; -inf only if every
 * path has probability exactly zero.
 */
double orc_log10_rescaled(const orc_testcase *tc) {
    orc_init();
    const int R = tc->rslen, H = tc->haplen;
    if (R == 0 || H == 0) return -INFINITY;
    double *buf = (double *)calloc((size_t)6 * (H + 1), sizeof(double));
    double *Mp = buf, *Xp = buf + (H + 1), *Yp = buf + 2 * (H + 1);
    double *Mc = buf + 3 * (H + 1), *Xc = buf + 4 * (H + 1), *Yc = buf + 5 * (H + 1);
    uint8_t *hc = (uint8_t *)malloc((size_t)H + 1);
    for (int j = 0; j < H; j++) hc[j] = base_code[(uint8_t)tc->hap[j]];
    long long exp2_offset = 0; /* stored values = true values * 2^-exp2_offset */
    const double init_y = 1.0 / (double)H;
    for (int j = 0; j <= H; j++) Yp[j] = init_y;
    for (int r = 1; r <= R; r++) {
        const int qi = tc->i[r - 1] & 127, qd = tc->d[r - 1] & 127;
        const int qc = tc->c[r - 1] & 127, qq = tc->q[r - 1] & 127;
        const double pMM = set_mm_prob_d(qi, qd);
        const double pGAPM = 1.0 - ph2pr_d[qc];
        const double pMX = ph2pr_d[qi], pXX = ph2pr_d[qc];
        const double pMY = ph2pr_d[qd], pYY = ph2pr_d[qc];
        const double distm0 = ph2pr_d[qq];
        const double one_m = 1.0 - distm0, mis = distm0 / 3.0;
        const uint8_t rc = base_code[(uint8_t)tc->rs[r - 1]];
        Mc[0] = 0; Xc[0] = 0; Yc[0] = 0;
        double mx = 0;
        for (int j = 1; j <= H; j++) {
            const double e = is_match(rc, hc[j - 1]) ? one_m : mis;
            Mc[j] = ((Mp[j - 1] * pMM + Xp[j - 1] * pGAPM) + Yp[j - 1] * pGAPM) * e;
            Xc[j] = Mp[j] * pMX + Xp[j] * pXX;
            Yc[j] = Mc[j - 1] * pMY + Yc[j - 1] * pYY;
            double m = Mc[j] > Xc[j] ? Mc[j] : Xc[j];
            m = m > Yc[j] ? m : Yc[j];
            mx = mx > m ? mx : m;
        }
        if (mx > 0) {
            int e2;
            frexp(mx, &e2);
            double s = ldexp(1.0, -e2);
            for (int j = 0; j <= H; j++) { Mc[j] *= s; Xc[j] *= s; Yc[j] *= s; }
            exp2_offset += e2;
        }
        double *t;
        t = Mp; Mp = Mc; Mc = t;
        t = Xp; Xp = Xc; Xc = t;
        t = Yp; Yp = Yc; Yc = t;
        if (r == 1) {
            memset(Mc, 0, sizeof(double) * (H + 1));
            memset(Xc, 0, sizeof(double) * (H + 1));
        }
    }
    double sumM = 0, sumX = 0;
    for (int j = 1; j <= H; j++) sumM += Mp[j];
    for (int j = 1; j <= H; j++) sumX += Xp[j];
    free(buf);
    free(hc);
    double s = sumM + sumX;
    if (!(s > 0)) return -INFINITY;
    return log10(s) + (double)exp2_offset * log10(2.0);
}

/*
 * Scalar PairHMM with the constant transition matrix ORIGINAL_DEFAULT and the
 * quality-derived prior (pairhmm.hpp:32-33, 39-80).  Match is a raw byte
 * compare with 'N' as wildcard; the prior indexes the 10^(-Q/10) table by the
 * raw qual byte (quality_utils.hpp:25-28, 71-76), masked here to 0..127.
 */
double orc_scalar_log10(const char *read, const char *qual, int rl, const char *hap, int hl,
                        const double *trans /* 7 entries, NULL = ORIGINAL_DEFAULT */) {
    static const double def[7] = {0.9998, 0.0001, 0.0001, 0.9, 0.1, 0.9, 0.1};
    const double *t = trans ? trans : def;
    const double mm = t[0], mi = t[1], md = t[2], im = t[3], ii = t[4], dm = t[5], dd = t[6];
    double *buf = (double *)calloc((size_t)6 * (hl + 1), sizeof(double));
    double *Mp = buf, *Ip = buf + (hl + 1), *Dp = buf + 2 * (hl + 1);
    double *Mc = buf + 3 * (hl + 1), *Ic = buf + 4 * (hl + 1), *Dc = buf + 5 * (hl + 1);
    const double init = pow(2, 1020);
    const double initv = init / (double)hl;
    for (int j = 0; j <= hl; j++) Dp[j] = initv;
    for (int i = 1; i <= rl; i++) {
        const double err = pow(10, (qual[i - 1] & 127) / -10.0);
        const char x = read[i - 1];
        Mc[0] = 0; Ic[0] = 0; Dc[0] = 0;
        for (int j = 1; j <= hl; j++) {
            const char y = hap[j - 1];
            const double prior = (x == y || x == 'N' || y == 'N') ? 1 - err : err / 3.0;
            Mc[j] = prior * (Mp[j - 1] * mm + Ip[j - 1] * im + Dp[j - 1] * dm);
            Ic[j] = Mp[j] * mi + Ip[j] * ii;
            Dc[j] = Mc[j - 1] * md + Dc[j - 1] * dd;
        }
        double *tp;
        tp = Mp; Mp = Mc; Mc = tp;
        tp = Ip; Ip = Ic; Ic = tp;
        tp = Dp; Dp = Dc; Dc = tp;
        if (i == 1) {
            memset(Mc, 0, sizeof(double) * (hl + 1));
            memset(Ic, 0, sizeof(double) * (hl + 1));
        }
    }
    double s = 0;
    for (int j = 1; j <= hl; j++) s += Mp[j] + Ip[j];
    free(buf);
    return log10(s) - log10(init);
}

/* Batch forms: the OpenMP loop of computeLikelihoodsNative (pairhmm_avx.hpp:133-152). */
void orc_batch_reference_rule(long n, const orc_testcase *tcs, double *out, int *used_f64, int nthreads) {
    orc_init();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (long k = 0; k < n; k++) out[k] = orc_log10_reference_rule(&tcs[k], used_f64 ? &used_f64[k] : NULL);
}

void orc_batch_rescaled(long n, const orc_testcase *tcs, double *out, int nthreads) {
    orc_init();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (long k = 0; k < n; k++) out[k] = orc_log10_rescaled(&tcs[k]);
}

void orc_batch_prob_f32(long n, const orc_testcase *tcs, float *out, int nthreads) {
    orc_init();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (long k = 0; k < n; k++) out[k] = orc_prob_f32(&tcs[k]);
}

void orc_batch_prob_f64(long n, const orc_testcase *tcs, double *out, int nthreads) {
    orc_init();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (long k = 0; k < n; k++) out[k] = orc_prob_f64(&tcs[k]);
}

/* Table accessors, for the table-identity tests. */
const float *orc_table_ph2pr_f32(void) { orc_init(); return ph2pr_f; }
const double *orc_table_ph2pr_f64(void) { orc_init(); return ph2pr_d; }
const float *orc_table_mm_f32(void) { orc_init(); return mm_f; }
const double *orc_table_mm_f64(void) { orc_init(); return mm_d; }
int orc_table_mm_size(void) { return ORC_MM_SIZE; }

/* ------------------------------------------------------------------------ *
 * Learned-band support (the reference has no banded PairHMM; these define
 * the banded DP and the training labels the B200 path computes).
 *
 * Band: diagonals d = c - r in [d_lo, d_lo + W).  Row 0 carries
 * Y = 1/H on its band cells with 0 <= c <= H; in rows r >= 1 cells outside the
 * band or outside 1 <= c <= H are zero; in-band cells follow the reference
 * recurrence (avx-pairhmm-template.h:183-198) with out-of-band neighbours
 * zero.  Result: log10 of the sum over the last row's band cells with
 * 1 <= c <= H of M + X, rows renormalised by powers of two as in
 * orc_log10_rescaled.
 * ------------------------------------------------------------------------ */
double orc_band_log10(const orc_testcase *tc, int d_lo, int W) {
    orc_init();
    const int R = tc->rslen, H = tc->haplen;
    if (R == 0 || H == 0 || W <= 0) return -INFINITY;
    double *buf = (double *)calloc((size_t)6 * W, sizeof(double));
    double *Mp = buf, *Xp = buf + W, *Yp = buf + 2 * W, *Mc = buf + 3 * W, *Xc = buf + 4 * W, *Yc = buf + 5 * W;
    for (int k = 0; k < W; k++) {
        const int c = d_lo + k;
        Yp[k] = (c >= 0 && c <= H) ? 1.0 / (double)H : 0.0;
    }
    long long e2sum = 0;
    for (int r = 1; r <= R; r++) {
        const int qi = tc->i[r - 1] & 127, qd = tc->d[r - 1] & 127;
        const int qc = tc->c[r - 1] & 127, qq = tc->q[r - 1] & 127;
        const double pMM = set_mm_prob_d(qi, qd), gp = 1.0 - ph2pr_d[qc];
        const double pMX = ph2pr_d[qi], pMY = ph2pr_d[qd], g = ph2pr_d[qc];
        const double eps = ph2pr_d[qq], one_m = 1.0 - eps, mis = eps / 3.0;
        const uint8_t rc = base_code[(uint8_t)tc->rs[r - 1]];
        double mx = 0;
        for (int k = 0; k < W; k++) {
            const int c = r + d_lo + k;
            if (c < 1 || c > H) { Mc[k] = Xc[k] = Yc[k] = 0; continue; }
            const double e = is_match(rc, base_code[(uint8_t)tc->hap[c - 1]]) ? one_m : mis;
            Mc[k] = e * (pMM * Mp[k] + gp * Xp[k] + gp * Yp[k]);
            Xc[k] = (k + 1 < W) ? pMX * Mp[k + 1] + g * Xp[k + 1] : 0.0;
            Yc[k] = (k > 0) ? pMY * Mc[k - 1] + g * Yc[k - 1] : 0.0;
            double m = Mc[k] > Xc[k] ? Mc[k] : Xc[k];
            m = m > Yc[k] ? m : Yc[k];
            mx = mx > m ? mx : m;
        }
        if (mx > 0) {
            int e2; frexp(mx, &e2);
            const double s = ldexp(1.0, -e2);
            for (int k = 0; k < W; k++) { Mc[k] *= s; Xc[k] *= s; Yc[k] *= s; }
            e2sum += e2;
        }
        double *t;
        t = Mp; Mp = Mc; Mc = t; t = Xp; Xp = Xc; Xc = t; t = Yp; Yp = Yc; Yc = t;
    }
    double s = 0;
    for (int k = 0; k < W; k++) {
        const int c = R + d_lo + k;
        if (c >= 1 && c <= H) s += Mp[k] + Xp[k];
    }
    free(buf);
    if (!(s > 0)) return -INFINITY;
    return log10(s) + (double)e2sum * log10(2.0);
}

/*
 * Posterior spread over diagonals from the full forward-backward DP.
 * For each row r >= 1 the posterior of the cells, p_r(c) ~ sum over states
 * of F_s(r,c) B_s(r,c), is normalised to sum 1 over the row; pstar[d - dmin]
 * = max over rows of p_r at diagonal d = c - r, for d in [dmin, dmax] =
 * [1 - R, H - 1].  Returns 0, or -1 when the likelihood is zero.
 * Backward recurrences (successor weights of the forward):
 *   B_M(r,c) = mm(r+1) e(r+1,c+1) B_M(r+1,c+1) + mx(r+1) B_X(r+1,c) + my(r) B_Y(r,c+1) + [r==R]
 *   B_X(r,c) = gp(r+1) e(r+1,c+1) B_M(r+1,c+1) + g(r+1) B_X(r+1,c) + [r==R]
 *   B_Y(r,c) = gp(r+1) e(r+1,c+1) B_M(r+1,c+1) + g(r) B_Y(r,c+1)
 * Every row is renormalised by a power of two in both passes; the per-row
 * normalisation of p_r makes those scales cancel.
 */
int orc_posterior_diag(const orc_testcase *tc, double *pstar) {
    orc_init();
    const int R = tc->rslen, H = tc->haplen;
    if (R == 0 || H == 0) return -1;
    const size_t W = (size_t)H + 2;
    double *F = (double *)calloc((size_t)3 * (R + 1) * W, sizeof(double));
    double *B = (double *)calloc((size_t)3 * (R + 2) * W, sizeof(double));
    double *mm = malloc(sizeof(double) * (R + 2)), *gp = malloc(sizeof(double) * (R + 2));
    double *mx = malloc(sizeof(double) * (R + 2)), *my = malloc(sizeof(double) * (R + 2));
    double *gg = malloc(sizeof(double) * (R + 2)), *em = malloc(sizeof(double) * (R + 2));
    double *ex = malloc(sizeof(double) * (R + 2));
    uint8_t *rc = malloc((size_t)R + 2), *hc = malloc((size_t)H + 2);
    for (int c = 1; c <= H; c++) hc[c] = base_code[(uint8_t)tc->hap[c - 1]];
    for (int r = 1; r <= R; r++) {
        const int qi = tc->i[r - 1] & 127, qd = tc->d[r - 1] & 127, qc = tc->c[r - 1] & 127, qq = tc->q[r - 1] & 127;
        mm[r] = set_mm_prob_d(qi, qd); gp[r] = 1.0 - ph2pr_d[qc]; mx[r] = ph2pr_d[qi]; my[r] = ph2pr_d[qd];
        gg[r] = ph2pr_d[qc]; em[r] = 1.0 - ph2pr_d[qq]; ex[r] = ph2pr_d[qq] / 3.0;
        rc[r] = base_code[(uint8_t)tc->rs[r - 1]];
    }
#define FM(r, c) F[((size_t)3 * (r)) * W + (c)]
#define FX(r, c) F[((size_t)3 * (r) + 1) * W + (c)]
#define FY(r, c) F[((size_t)3 * (r) + 2) * W + (c)]
#define BM(r, c) B[((size_t)3 * (r)) * W + (c)]
#define BX(r, c) B[((size_t)3 * (r) + 1) * W + (c)]
#define BY(r, c) B[((size_t)3 * (r) + 2) * W + (c)]
#define EM(r, c) (is_match(rc[r], hc[c]) ? em[r] : ex[r])
    for (int c = 0; c <= H; c++) FY(0, c) = 1.0 / H;
    for (int r = 1; r <= R; r++) {
        double m = 0;
        for (int c = 1; c <= H; c++) {
            FM(r, c) = EM(r, c) * (mm[r] * FM(r - 1, c - 1) + gp[r] * (FX(r - 1, c - 1) + FY(r - 1, c - 1)));
            FX(r, c) = mx[r] * FM(r - 1, c) + gg[r] * FX(r - 1, c);
            FY(r, c) = my[r] * FM(r, c - 1) + gg[r] * FY(r, c - 1);
            double v = FM(r, c) > FX(r, c) ? FM(r, c) : FX(r, c);
            v = v > FY(r, c) ? v : FY(r, c);
            m = m > v ? m : v;
        }
        if (m > 0) { int e2; frexp(m, &e2); double s = ldexp(1.0, -e2);
            for (int c = 0; c <= H; c++) { FM(r, c) *= s; FX(r, c) *= s; FY(r, c) *= s; } }
    }
    for (int r = R; r >= 1; r--) {
        double m = 0;
        for (int c = H; c >= 1; c--) {
            double nm = 0, bx = 0, by = 0, bm = 0;
            if (r < R && c < H) nm = EM(r + 1, c + 1) * BM(r + 1, c + 1);
            if (r < R) { bm += mm[r + 1] * nm + mx[r + 1] * BX(r + 1, c); bx += gp[r + 1] * nm + gg[r + 1] * BX(r + 1, c); }
            else { bm += 1.0; bx += 1.0; }
            by = (r < R ? gp[r + 1] * nm : 0.0) + (c < H ? gg[r] * BY(r, c + 1) : 0.0);
            if (c < H) bm += my[r] * BY(r, c + 1);
            BM(r, c) = bm; BX(r, c) = bx; BY(r, c) = by;
            double v = bm > bx ? bm : bx; v = v > by ? v : by; m = m > v ? m : v;
        }
        if (m > 0 && r > 1) { int e2; frexp(m, &e2); double s = ldexp(1.0, -e2);
            for (int c = 1; c <= H; c++) { BM(r, c) *= s; BX(r, c) *= s; BY(r, c) *= s; } }
    }
    int ok = 0;
    const int dmin = 1 - R;
    for (int d = 0; d < R + H - 1; d++) pstar[d] = 0;
    for (int r = 1; r <= R; r++) {
        double tot = 0;
        for (int c = 1; c <= H; c++) tot += FM(r, c) * BM(r, c) + FX(r, c) * BX(r, c) + FY(r, c) * BY(r, c);
        if (!(tot > 0)) continue;
        ok = 1;
        for (int c = 1; c <= H; c++) {
            const double p = (FM(r, c) * BM(r, c) + FX(r, c) * BX(r, c) + FY(r, c) * BY(r, c)) / tot;
            const int d = c - r - dmin;
            if (p > pstar[d]) pstar[d] = p;
        }
    }
#undef FM
#undef FX
#undef FY
#undef BM
#undef BX
#undef BY
#undef EM
    free(F); free(B); free(mm); free(gp); free(mx); free(my); free(gg); free(em); free(ex); free(rc); free(hc);
    return ok ? 0 : -1;
}

/*
 * Banded DP as orc_band_log10, also returning the two edge statistics the
 * banded kernel uses for its fallback decision:
 *   row_ratio  max over rows r >= 8, r = 0 mod 4, of (A(r,0) + A(r,W-1)) / max_k A(r,k)
 *              with A = M + X + Y (true, unscaled values)
 *   end_frac   share of the last row's M + X on the band's two outer diagonals of each side
 */
/* leak_bound: sum over rows of the forward mass leaving the band (an
 * insertion step off the left edge, a deletion step off the right edge) times
 * the suffix's perfect-match probability prod_{r' > r} (1 - eps_r'), divided
 * by the band likelihood -- an upper bound, up to the sum over suffix paths,
 * on the relative mass the band loses. */
static double g_leak_bound;
static int g_r0 = 8; /* first row the edge ratio looks at */
void orc_band_set_r0(int r0) { g_r0 = r0; }
static double g_rho = 1.0; /* continuation discount per 11 bases (k-mer exclusion); 1 = none */
void orc_band_set_rho(double rho) { g_rho = rho; }
double orc_band_leak_bound(void) { return g_leak_bound; }

double orc_band_detail(const orc_testcase *tc, int d_lo, int W, double *row_ratio, double *end_frac) {
    orc_init();
    const int R = tc->rslen, H = tc->haplen;
    *row_ratio = 0; *end_frac = 0;
    if (R == 0 || H == 0 || W <= 0) return -INFINITY;
    double *buf = (double *)calloc((size_t)6 * W, sizeof(double));
    double *Mp = buf, *Xp = buf + W, *Yp = buf + 2 * W, *Mc = buf + 3 * W, *Xc = buf + 4 * W, *Yc = buf + 5 * W;
    for (int k = 0; k < W; k++) { const int c = d_lo + k; Yp[k] = (c >= 0 && c <= H) ? 1.0 / (double)H : 0.0; }
    long long e2sum = 0;
    double rr = 0;
    double leak_sum = 0, pre = 1;  /* sum leak(r) * 2^e2sum(r) / prod_{r' <= r}(1-eps), in row-scaled units */
    for (int r = 1; r <= R; r++) {
        const int qi = tc->i[r - 1] & 127, qd = tc->d[r - 1] & 127, qc = tc->c[r - 1] & 127, qq = tc->q[r - 1] & 127;
        const double pMM = set_mm_prob_d(qi, qd), gp = 1.0 - ph2pr_d[qc];
        const double pMX = ph2pr_d[qi], pMY = ph2pr_d[qd], g = ph2pr_d[qc];
        const double eps = ph2pr_d[qq], one_m = 1.0 - eps, mis = eps / 3.0;
        const uint8_t rc = base_code[(uint8_t)tc->rs[r - 1]];
        /* mass of row r-1 leaving through the left edge into row r's X */
        const double leak_l = pMX * Mp[0] + g * Xp[0];
        pre *= one_m;
        double mx = 0;
        for (int k = 0; k < W; k++) {
            const int c = r + d_lo + k;
            if (c < 1 || c > H) { Mc[k] = Xc[k] = Yc[k] = 0; continue; }
            const double e = is_match(rc, base_code[(uint8_t)tc->hap[c - 1]]) ? one_m : mis;
            Mc[k] = e * (pMM * Mp[k] + gp * Xp[k] + gp * Yp[k]);
            Xc[k] = (k + 1 < W) ? pMX * Mp[k + 1] + g * Xp[k + 1] : 0.0;
            Yc[k] = (k > 0) ? pMY * Mc[k - 1] + g * Yc[k - 1] : 0.0;
            double m = Mc[k] > Xc[k] ? Mc[k] : Xc[k]; m = m > Yc[k] ? m : Yc[k]; mx = mx > m ? mx : m;
        }
        /* mass of row r leaving through the right edge into Y */
        const double leak_r = pMY * Mc[W - 1] + g * Yc[W - 1];
        leak_sum += (leak_l + leak_r) * ldexp(1.0, (int)e2sum) / pre * pow(g_rho, (double)((R - r) / 11));
        if (r >= g_r0 && (r & 3) == 0) {
            double peak = 0;
            for (int k = 0; k < W; k++) { const double a = Mc[k] + Xc[k] + Yc[k]; peak = peak > a ? peak : a; }
            const double edge = Mc[0] + Xc[0] + Yc[0] + Mc[W - 1] + Xc[W - 1] + Yc[W - 1];
            if (edge > 0) { const double q = peak > 0 ? edge / peak : 1e300; rr = rr > q ? rr : q; }
        }
        if (mx > 0) { int e2; frexp(mx, &e2); const double s = ldexp(1.0, -e2);
            for (int k = 0; k < W; k++) { Mc[k] *= s; Xc[k] *= s; Yc[k] *= s; } e2sum += e2; }
        double *t; t = Mp; Mp = Mc; Mc = t; t = Xp; Xp = Xc; Xc = t; t = Yp; Yp = Yc; Yc = t;
    }
    double s = 0, outer = 0;
    for (int k = 0; k < W; k++) {
        const int c = R + d_lo + k;
        if (c >= 1 && c <= H) { s += Mp[k] + Xp[k]; if (k < 2 || k >= W - 2) outer += Mp[k] + Xp[k]; }
    }
    free(buf);
    *row_ratio = rr;
    *end_frac = s > 0 ? outer / s : 1.0;
    g_leak_bound = s > 0 ? leak_sum * pre / (s * ldexp(1.0, (int)e2sum)) : 1e300;
    if (!(s > 0)) return -INFINITY;
    return log10(s) + (double)e2sum * log10(2.0);
}

/*
 * Posterior mass on the band's two edge diagonals, from a banded
 * forward-backward pass (FP64, rows renormalised in both passes):
 *   edge = sum_r [ A_F(r,0) Bmax(r,0) + A_F(r,W-1) Bmax(r,W-1) ] / L_band
 * with A_F = M + X + Y forward and Bmax = max(B_M, B_X, B_Y) backward at the
 * cell (an upper bound on sum_s F_s B_s there).  Backward, band coordinates:
 *   B_M(r,k) = mm(r+1) e(r+1,k) B_M(r+1,k) + mx(r+1) B_X(r+1,k-1) + my(r) B_Y(r,k+1) + [r==R]
 *   B_X(r,k) = gp(r+1) e(r+1,k) B_M(r+1,k) + g(r+1) B_X(r+1,k-1) + [r==R]
 *   B_Y(r,k) = gp(r+1) e(r+1,k) B_M(r+1,k) + g(r) B_Y(r,k+1)
 * out-of-band or out-of-matrix successors contributing zero.
 */
double orc_band_posterior_edge(const orc_testcase *tc, int d_lo, int W) {
    orc_init();
    const int R = tc->rslen, H = tc->haplen;
    if (R == 0 || H == 0 || W <= 0) return 1.0;
    double *Af0 = calloc((size_t)R + 2, sizeof(double)), *Af1 = calloc((size_t)R + 2, sizeof(double));
    double *fs = calloc((size_t)R + 2, sizeof(double));  /* log2 scale of forward row r */
    double *mm = malloc(sizeof(double) * (R + 2)), *gp = malloc(sizeof(double) * (R + 2));
    double *mxp = malloc(sizeof(double) * (R + 2)), *myp = malloc(sizeof(double) * (R + 2));
    double *gg = malloc(sizeof(double) * (R + 2)), *em = malloc(sizeof(double) * (R + 2)), *ex = malloc(sizeof(double) * (R + 2));
    uint8_t *rc = malloc((size_t)R + 2);
    for (int r = 1; r <= R; r++) {
        const int qi = tc->i[r - 1] & 127, qd = tc->d[r - 1] & 127, qc = tc->c[r - 1] & 127, qq = tc->q[r - 1] & 127;
        mm[r] = set_mm_prob_d(qi, qd); gp[r] = 1.0 - ph2pr_d[qc]; mxp[r] = ph2pr_d[qi]; myp[r] = ph2pr_d[qd];
        gg[r] = ph2pr_d[qc]; em[r] = 1.0 - ph2pr_d[qq]; ex[r] = ph2pr_d[qq] / 3.0; rc[r] = base_code[(uint8_t)tc->rs[r - 1]];
    }
#define EMIS(r, k) ((r + d_lo + (k) >= 1 && r + d_lo + (k) <= H) ? (is_match(rc[r], base_code[(uint8_t)tc->hap[r + d_lo + (k) - 1]]) ? em[r] : ex[r]) : 0.0)
    double *buf = calloc((size_t)6 * W, sizeof(double));
    double *Mp = buf, *Xp = buf + W, *Yp = buf + 2 * W, *Mc = buf + 3 * W, *Xc = buf + 4 * W, *Yc = buf + 5 * W;
    for (int k = 0; k < W; k++) { const int c = d_lo + k; Yp[k] = (c >= 0 && c <= H) ? 1.0 / (double)H : 0.0; }
    double lsc = 0;
    for (int r = 1; r <= R; r++) {
        double m = 0;
        for (int k = 0; k < W; k++) {
            const int c = r + d_lo + k;
            if (c < 1 || c > H) { Mc[k] = Xc[k] = Yc[k] = 0; continue; }
            Mc[k] = EMIS(r, k) * (mm[r] * Mp[k] + gp[r] * (Xp[k] + Yp[k]));
            Xc[k] = (k + 1 < W) ? mxp[r] * Mp[k + 1] + gg[r] * Xp[k + 1] : 0.0;
            Yc[k] = (k > 0) ? myp[r] * Mc[k - 1] + gg[r] * Yc[k - 1] : 0.0;
            const double v = Mc[k] + Xc[k] + Yc[k]; m = m > v ? m : v;
        }
        Af0[r] = Mc[0] + Xc[0] + Yc[0]; Af1[r] = Mc[W - 1] + Xc[W - 1] + Yc[W - 1]; fs[r] = lsc;
        if (m > 0) { int e2; frexp(m, &e2); const double s = ldexp(1.0, -e2);
            for (int k = 0; k < W; k++) { Mc[k] *= s; Xc[k] *= s; Yc[k] *= s; } lsc += e2; }
        double *t; t = Mp; Mp = Mc; Mc = t; t = Xp; Xp = Xc; Xc = t; t = Yp; Yp = Yc; Yc = t;
    }
    double L = 0;
    for (int k = 0; k < W; k++) { const int c = R + d_lo + k; if (c >= 1 && c <= H) L += Mp[k] + Xp[k]; }
    const double lscL = lsc;  /* L_true = L * 2^lscL; A_F(r) true = Af(r) * 2^fs[r] */
    /* backward */
    double *BM = calloc(W, sizeof(double)), *BX = calloc(W, sizeof(double)), *BY = calloc(W, sizeof(double));
    double bls = 0, edge = 0;
    for (int r = R; r >= 1; r--) {
        double nBM[256], nBX[256], nBY[256];
        for (int k = W - 1; k >= 0; k--) {
            const int c = r + d_lo + k;
            if (c < 1 || c > H) { nBM[k] = nBX[k] = nBY[k] = 0; continue; }
            double tM = 0, tX = 0, tY = 0;
            if (r < R) {
                const double em1 = (c + 1 <= H) ? EMIS(r + 1, k) * BM[k] : 0.0;
                const double bxk = (k - 1 >= 0) ? BX[k - 1] : 0.0;
                tM = mm[r + 1] * em1 + mxp[r + 1] * bxk;
                tX = gp[r + 1] * em1 + gg[r + 1] * bxk;
                tY = gp[r + 1] * em1;
            } else { tM = 1.0 * ldexp(1.0, -(int)bls); tX = tM; tY = 0; }
            const double byk1 = (k + 1 < W && c + 1 <= H) ? nBY[k + 1] : 0.0;
            nBM[k] = tM + myp[r] * byk1;
            nBX[k] = tX;
            nBY[k] = tY + gg[r] * byk1;
        }
        double m = 0;
        for (int k = 0; k < W; k++) { BM[k] = nBM[k]; BX[k] = nBX[k]; BY[k] = nBY[k];
            const double v = BM[k] > BX[k] ? BM[k] : BX[k]; m = m > v ? m : v; }
        /* posterior bound at the edges: A_F(r) * Bmax(r) / L  (all in true units) */
        const double b0 = fmax(BM[0], fmax(BX[0], BY[0])), b1 = fmax(BM[W - 1], fmax(BX[W - 1], BY[W - 1]));
        edge += (Af0[r] * b0 + Af1[r] * b1) * ldexp(1.0, (int)(fs[r] + bls - lscL));
        if (m > 0) { int e2; frexp(m, &e2); const double s = ldexp(1.0, -e2);
            for (int k = 0; k < W; k++) { BM[k] *= s; BX[k] *= s; BY[k] *= s; } bls += e2; }
    }
#undef EMIS
    free(BM); free(BX); free(BY); free(buf); free(Af0); free(Af1); free(fs);
    free(mm); free(gp); free(mxp); free(myp); free(gg); free(em); free(ex); free(rc);
    return L > 0 ? edge / L : 1.0;
}
