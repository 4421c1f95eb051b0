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
#define ORC_JAC_SIZE ((int)(ORC_JAC_TOL / ORC_JAC_STEP) + 1)
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
