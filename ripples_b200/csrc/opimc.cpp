// opimc.cpp -- OPIM-C sample-size and bound arithmetic (host).
//
// The OPIM-C driver (Tang, Tang, Xiao, Yuan, SIGMOD'18; the reference's
// include/ripples/opimc.h:150-243) grows two RRR pools R1, R2 from theta_0
// sets, doubling up to theta_max, and stops once the lower bound of the
// spread of the seeds picked on R1 (their coverage of R2) reaches
// (1 - 1/e - epsilon) times the upper bound of the optimum (the greedy
// coverage of R1).  These are the reference's formulas in the reference's
// float arithmetic (opimc.h:60-98: equations (16), (17), (5) and (8) of the
// paper), so theta_0, theta_max and the stopping test decide exactly as the
// reference decides for the same coverages.
#include <cmath>
#include <cstdint>
#include <cstddef>

#include "ripples_b200.h"

extern "C" double rip_log_binomial(uint64_t n, uint64_t k);

namespace rip_opimc {

constexpr float kOneMinusInvE = 0.6321203113733684;  // 1 - 1/e, as a float

// 2 (a sqrt(ln(6/delta)) + sqrt(a (ln C(n,k) + ln(6/delta))))^2, a = 1 - 1/e
inline float theta_helper(size_t n, float epsilon, size_t k, float delta) {
  (void)epsilon;
  float b = kOneMinusInvE * sqrt(log(6.0 / delta));
  float c = sqrt(kOneMinusInvE * (rip_log_binomial(n, k) + log(6.0 / delta)));
  float d = (b + c) * (b + c);
  return (2 * d);
}

}  // namespace rip_opimc

extern "C" uint64_t rip_opimc_theta_max(uint64_t n, float epsilon, uint64_t k, float delta) {
  return ceil((size_t)n * rip_opimc::theta_helper(n, epsilon, k, delta) /
              (epsilon * epsilon * (size_t)k));
}

extern "C" uint64_t rip_opimc_theta_zero(uint64_t n, float epsilon, uint64_t k, float delta) {
  return ceil(rip_opimc::theta_helper(n, epsilon, k, delta));
}

extern "C" float rip_opimc_lower_bound(uint64_t coverage, float delta2, uint64_t n,
                                       uint64_t theta) {
  float a = log(1 / delta2);
  float b = sqrt((size_t)coverage + 2 * a / 9);
  float c = sqrt(a / 2);
  float d = (b - c) * (b - c);
  float e = a / 18;
  return (float((size_t)n) / (size_t)theta) * (d - e);
}

extern "C" float rip_opimc_upper_bound(uint64_t coverage, float delta1, uint64_t n,
                                       uint64_t theta) {
  float b = (size_t)coverage / rip_opimc::kOneMinusInvE;
  float c = log(1 / delta1) / 2;
  float d = std::sqrt(b + c);
  // the reference's (D + sqrt(C))^2 is evaluated in double, then stored
  const double sc = std::sqrt((double)c);
  float e = (float)(((double)d + sc) * ((double)d + sc));
  return (float((size_t)n) / (size_t)theta) * e;
}
