// imm.cu -- theta math and the IMM driver behind include/ripples_b200.h.
#include "host.h"

// ---------------------------------------------------------------------------
// theta math: include/ripples/imm.h:77-128, utility.h:84-87
// ---------------------------------------------------------------------------
extern "C" double rip_log_binomial(uint64_t n, uint64_t k) {
  return lgamma(n + 1) - lgamma(n - k + 1) - lgamma(k + 1);
}

extern "C" int64_t rip_theta_prime(int64_t x, double epsilonPrime, double l,
                                   uint64_t k, uint64_t num_nodes) {
  k = std::min<uint64_t>(k, num_nodes / 2);
  return (ssize_t)((2 + 2. / 3. * epsilonPrime) *
                   (l * std::log(num_nodes) + rip_log_binomial(num_nodes, k) +
                    std::log(std::log2(num_nodes))) *
                   std::pow(2.0, x) / (epsilonPrime * epsilonPrime));
}

extern "C" int64_t rip_inv_theta_prime(int64_t rrsize, double epsilonPrime,
                                       double l, uint64_t k, uint64_t num_nodes) {
  k = std::min<uint64_t>(k, num_nodes / 2);
  return (ssize_t)std::log2(rrsize * epsilonPrime * epsilonPrime /
                            ((2 + 2. / 3. * epsilonPrime) *
                             (l * std::log(num_nodes) +
                              rip_log_binomial(num_nodes, k) +
                              std::log(std::log2(num_nodes)))));
}

extern "C" uint64_t rip_theta(double epsilon, double l, uint64_t k, double LB,
                              uint64_t num_nodes) {
  if (LB == 0) return 0;
  k = std::min<uint64_t>(k, num_nodes / 2);
  double term1 = 0.6321205588285577;  // 1 - 1/e
  double alpha = sqrt(l * std::log(num_nodes) + std::log(2));
  double beta = sqrt(term1 * (rip_log_binomial(num_nodes, k) +
                              l * std::log(num_nodes) + std::log(2)));
  double lamdaStar = 2 * num_nodes * (term1 * alpha + beta) *
                     (term1 * alpha + beta) * pow(epsilon, -2);
  return (size_t)(lamdaStar / LB);
}

// ---------------------------------------------------------------------------
// IMM driver: include/ripples/imm.h:145-260 (Sampling, omp) + :768-860 (IMM)
// ---------------------------------------------------------------------------
extern "C" int rip_imm_pool(rip_pool *p, uint32_t k, double epsilon, double l,
                            uint64_t seed, int tiebreak, int sampler,
                            uint32_t *seeds, uint32_t *num_seeds,
                            rip_imm_record *rec) {
  if (!p || !num_seeds || (k && !seeds) || !(epsilon > 0)) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  rip_imm_record R;
  std::memset(&R, 0, sizeof(R));
  const auto t_total = clk::now();
  const uint64_t n = p->g->n;
  l = l * (1 + 1 / std::log2(n));
  const double epsilonPrime = 1.4142135623730951 * epsilon;
  double LB = 0;
  std::vector<uint32_t> tmp_seeds(std::max<uint32_t>(k, 1));
  const auto t_est = clk::now();
  int64_t x = 1;
  if (p->num_sets != 0)
    x = rip_inv_theta_prime((int64_t)(p->num_sets / 2), epsilonPrime, l, k, n);
  for (; x < std::log2(n); ++x) {
    int64_t thetaPrime = rip_theta_prime(x, epsilonPrime, l, k, n);
    double f = 0;
    auto t0 = clk::now();
    uint64_t delta = 0;
    if ((uint64_t)std::max<int64_t>(thetaPrime, 0) > p->num_sets) {
      delta = (uint64_t)thetaPrime - p->num_sets;
      TRY(rip_sample(p, seed, delta, sampler));
      TRY(rip_sync(c));
    }
    double gen_ms = ms_since(t0);
    t0 = clk::now();
    uint32_t ns = 0;
    TRY(rip_select(p, p->num_sets, k, tiebreak, tmp_seeds.data(), nullptr, &ns, &f));
    double sel_ms = ms_since(t0);
    if (R.num_rounds < RIP_MAX_ROUNDS) {
      R.theta_prime_deltas[R.num_rounds] = delta;
      R.round_generate_ms[R.num_rounds] = gen_ms;
      R.round_select_ms[R.num_rounds] = sel_ms;
    }
    R.num_rounds++;
    if (f >= std::pow(2, -x)) {
      LB = (n * f) / (1 + epsilonPrime);
      break;
    }
  }
  const uint64_t theta = rip_theta(epsilon, l, k, LB, n);
  R.theta_estimation_ms = ms_since(t_est);
  R.theta = theta;
  auto t0 = clk::now();
  if (theta > p->num_sets) {
    TRY(rip_sample(p, seed, theta - p->num_sets, sampler));
    TRY(rip_sync(c));
  }
  R.generate_ms = ms_since(t0);
  t0 = clk::now();
  double f = 0;
  TRY(rip_select(p, std::min<uint64_t>(theta, p->num_sets), k, tiebreak, seeds,
                 nullptr, num_seeds, &f));
  R.select_ms = ms_since(t0);
  R.f = f;
  R.total_sets = p->num_sets;
  R.pool_elements = p->num_elems;
  R.rrr_set_bytes = p->num_elems * sizeof(uint32_t);
  R.total_ms = ms_since(t_total);
  if (rec) *rec = R;
  return RIP_OK;
}

extern "C" int rip_imm(rip_ctx *c, rip_graph *g, uint32_t k, double epsilon,
                       double l, uint64_t seed, int tiebreak, int sampler,
                       uint32_t *seeds, uint32_t *num_seeds,
                       rip_imm_record *record) {
  rip_pool *p = nullptr;
  TRY(rip_pool_create(c, g, &p));
  int rc = rip_imm_pool(p, k, epsilon, l, seed, tiebreak, sampler, seeds,
                        num_seeds, record);
  rip_pool_destroy(p);
  return rc;
}

