// phmm_tables.cpp -- the reference's probability tables, built on the host.
//
// lib/intel_native/pairhmm/Context.h defines, per precision:
//   ph2pr[x]            = 10^(-x/10)                         (:104-107, :144-147)
//   jacobian table      = log10(1 + 10^(-k * 1e-4)), k <= 8e4 (:42-47)
//   approx log10-sum    = big + table[round((big-small)*1e4)], or big when the
//                         gap is >= 8, evaluated in that precision (:72-90)
//   matchToMatchProb    = 10^(log1p(-min(1, 10^lsum(-i/10, -j/10))) / ln 10)
//                         for 0 <= j <= i <= 254, evaluated in double and
//                         stored in that precision (:50-61)
//   INITIAL_CONSTANT    = 2^120 (float) / 2^1020 (double)  (:108-109, :148-149)
// The kernels read these tables unchanged, so per-row probabilities equal the
// reference's bit for bit.
#include <cmath>
#include <quadmath.h>
#include <limits>
#include <algorithm>
#include <vector>

#include "phmm_common.h"
#include "phmm_kernels.h"
#include "phmm_genotype.h"

namespace bvphmm {
namespace {

constexpr double kJacStep = 0.0001;
constexpr int kJacSize = (int)(8.0 / kJacStep) + 1;
constexpr int kMaxQual = 254;

template <typename N>
int round_half_away(N d) {
  return (d > N(0)) ? (int)(d + N(0.5)) : (int)(d - N(0.5));
}

template <typename N>
struct LogSum {
  std::vector<N> jac;
  LogSum() : jac(kJacSize) {
    for (int k = 0; k < kJacSize; ++k) jac[k] = (N)std::log10(1.0 + std::pow(10.0, -((double)k) * kJacStep));
  }
  N operator()(N small, N big) const {
    if (small > big) std::swap(small, big);
    const N diff = big - small;
    if (diff >= (N)8.0) return big;
    const int ind = round_half_away<N>((N)(diff * (N)(1.0 / kJacStep)));
    return big + jac[ind];
  }
};

template <typename N>
void fill_mm(N* out) {
  LogSum<N> ls;
  const double inv_ln10 = 1.0 / std::log(10.0);
  // Only entries with max qual <= 127 are reachable (quals are masked & 127);
  // the triangular index of (max, min) is max*(max+1)/2 + min.
  for (int i = 0, off = 0; i <= kMaxQual; off += ++i) {
    for (int j = 0; j <= i; ++j) {
      const double s = (double)ls((N)(-0.1 * i), (N)(-0.1 * j));
      const double l = std::log1p(-std::min(1.0, std::pow(10.0, s))) * inv_ln10;
      if (off + j < kMMEntries) out[off + j] = (N)std::pow(10.0, l);
    }
  }
}

}  // namespace

void build_tables(Tables* t) {
  for (int x = 0; x < 128; ++x) {
    t->ph2pr_d[x] = std::pow(10.0, -((double)x) / 10.0);
    t->ph2pr_f[x] = powf(10.f, -((float)x) / 10.f);
    t->qp[x].p = t->ph2pr_f[x];
    t->qp[x].q = 1.f - t->ph2pr_f[x];
    t->qp[x].third = t->ph2pr_f[x] / 3.f;
    t->qp[x].inv = 1.f / t->ph2pr_f[x];
  }
  fill_mm<float>(t->mm_f);
  fill_mm<double>(t->mm_d);
  for (int x = 0; x < kMMEntries; ++x) t->mm_inv_f[x] = t->mm_f[x] >= kFoldMin ? 1.f / t->mm_f[x] : std::numeric_limits<float>::quiet_NaN();
  t->const_mode = 0;
  for (int k = 0; k < 8; ++k) {
    t->cf[k] = 0.f;
    t->cd[k] = 0.0;
  }
  t->init_f = std::ldexp(1.f, 120);
  t->log10_init_f = log10f(t->init_f);
  t->init_d = std::ldexp(1.0, 1020);
  t->log10_init_d = std::log10(t->init_d);
}

}  // namespace bvphmm

namespace bvphmm {

void set_constant_transitions(Tables* t, const double* trans) {
  if (!trans) {
    t->const_mode = 0;
    return;
  }
  t->const_mode = 1;
  for (int k = 0; k < 7; ++k) {
    t->cd[k] = trans[k];
    t->cf[k] = (float)trans[k];
  }
  t->cd[7] = 0.0;
  t->cf[7] = t->cf[0] >= kFoldMin ? 1.f / t->cf[0] : std::numeric_limits<float>::quiet_NaN();
}

}  // namespace bvphmm

namespace bvphmm {

void build_jacobian_table(double* out) {
  // MathUtils::JacobianLogTable (math_utils.hpp:122-139): entry i is
  // log10(1 + 10^(-1e-4 i)); each step is rounded once to double from
  // 113-bit arithmetic, which gives the correctly rounded values the
  // reference's compile-time table holds.
  constexpr double kStep = 0.0001;
  for (int i = 0; i < kJacobianEntries; ++i) {
    const double x = -kStep * i;
    const double pw = (double)powq((__float128)10, (__float128)x);
    const double s = 1.0 + pw;
    out[i] = (double)log10q((__float128)s);
  }
}

}  // namespace bvphmm
