// opimc_driver.cu -- OPIM-C on the device (host side).
//
// rip_coverage is FindCoverage (include/ripples/opimc.h:101-118) over a
// pool's sets [0, S); rip_opimc_pool is the OPIM-C loop (opimc.h:150-243):
// pools R1 (sets of key `seed`) and R2 (key seed + R2_KEY_OFFSET) of theta_0
// sets each, greedy selection on R1, the seeds' coverage of R2, the bounds of
// opimc.cpp, and theta doubled until lower / upper >= 1 - 1/e - epsilon (or
// theta reaches theta_max, the paper's cap).  Sets are pure functions of
// (key, id), so R1 and R2 equal the oracle's pools and the seeds equal the
// oracle's OPIM-C.
#include "host.h"

namespace {
constexpr uint64_t R2_KEY_OFFSET = 0x9E3779B97F4A7C15ull;
constexpr float OPIMC_A = 0.6321203113733684f;  // 1 - 1/e as the reference writes it
}  // namespace

extern "C" int rip_coverage(rip_pool *p, uint64_t num_sets, const uint32_t *seeds, uint32_t k,
                            uint64_t *covered) {
  if (!p || !covered || (k && !seeds)) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  if (num_sets > p->num_sets)
    return set_err(c, RIP_ERR_INVALID, "rip_coverage: %llu sets asked, the pool holds %llu",
                   (unsigned long long)num_sets, (unsigned long long)p->num_sets);
  const uint32_t n = p->g->n;
  std::vector<uint32_t> bits(((size_t)n + 31) / 32 + 1, 0u);
  for (uint32_t i = 0; i < k; ++i) {
    if (seeds[i] >= n)
      return set_err(c, RIP_ERR_INVALID, "rip_coverage: seed %u out of range (n = %u)",
                     seeds[i], n);
    bits[seeds[i] >> 5] |= 1u << (seeds[i] & 31);
  }
  *covered = 0;
  if (num_sets == 0 || k == 0) return RIP_OK;
  CK(c, cudaSetDevice(c->device));
  struct Buffers {
    rip_ctx *c;
    DevMem marked, ctr;
    ~Buffers() {
      dfree(c, marked);
      dfree(c, ctr);
    }
  } B{c, {}, {}};
  TRY(dalloc(c, B.marked, bits.size() * sizeof(uint32_t)));
  TRY(dalloc(c, B.ctr, sizeof(unsigned long long)));
  CK(c, cudaMemcpyAsync(B.marked.p, bits.data(), bits.size() * sizeof(uint32_t),
                        cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaMemsetAsync(B.ctr.p, 0, sizeof(unsigned long long), c->stream));
  launch_coverage(p->view(), num_sets, ptr<uint32_t>(B.marked),
                  ptr<unsigned long long>(B.ctr), c->num_sms * 8, c->stream);
  CK(c, cudaGetLastError());
  unsigned long long got = 0;
  CK(c, cudaMemcpyAsync(&got, B.ctr.p, sizeof(got), cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  *covered = got;
  return RIP_OK;
}

extern "C" int rip_opimc_pool(rip_pool *r1, rip_pool *r2, uint32_t k, float epsilon,
                              float delta, uint64_t seed, int tiebreak, int sampler,
                              uint32_t *seeds, uint32_t *num_seeds, rip_opimc_record *rec) {
  if (!r1 || !r2 || !num_seeds || (k && !seeds) || !(epsilon > 0) || !(delta > 0))
    return RIP_ERR_INVALID;
  rip_ctx *c = r1->ctx;
  if (r1->g != r2->g || r1 == r2)
    return set_err(c, RIP_ERR_INVALID, "rip_opimc_pool: two distinct pools of one graph");
  const auto t0 = clk::now();
  const uint64_t n = r1->g->n;
  rip_opimc_record R;
  std::memset(&R, 0, sizeof(R));
  uint64_t theta = rip_opimc_theta_zero(n, epsilon, k, delta);
  const uint64_t theta_max = rip_opimc_theta_max(n, epsilon, k, delta);
  R.theta_zero = theta;
  R.theta_max = theta_max;
  TRY(rip_pool_clear(r1));
  TRY(rip_pool_clear(r2));
  TRY(rip_sample(r1, seed, theta, sampler));
  TRY(rip_sample(r2, seed + R2_KEY_OFFSET, theta, sampler));
  const uint64_t i_max = (uint64_t)std::ceil(std::log2(theta_max / theta));
  const float d = delta / (3 * i_max);
  std::vector<uint32_t> picks(std::max<uint32_t>(k, 1));
  uint32_t np = 0;
  for (uint32_t round = 0;; ++round) {
    double f = 0;
    TRY(rip_select(r1, theta, k, tiebreak, picks.data(), nullptr, &np, &f));
    const uint64_t cov1 = (uint64_t)(f * theta);  // the reference scales f back
    uint64_t cov2 = 0;
    TRY(rip_coverage(r2, theta, picks.data(), np, &cov2));
    const float upper = rip_opimc_upper_bound(cov1, d, n, theta);
    const float lower = rip_opimc_lower_bound(cov2, d, n, theta);
    R.rounds = round + 1;
    R.coverage1 = cov1;
    R.coverage2 = cov2;
    R.lower = lower;
    R.upper = upper;
    if (lower / upper >= (OPIMC_A - epsilon)) break;
    if (theta >= theta_max) break;  // the paper's cap; the reference has none
    TRY(rip_sample(r1, seed, theta, sampler));  // sets [theta, 2 theta)
    TRY(rip_sample(r2, seed + R2_KEY_OFFSET, theta, sampler));
    theta *= 2;
  }
  for (uint32_t i = 0; i < np; ++i) seeds[i] = picks[i];
  *num_seeds = np;
  R.theta = theta;
  R.total_ms = ms_since(t0);
  if (rec) *rec = R;
  return RIP_OK;
}
