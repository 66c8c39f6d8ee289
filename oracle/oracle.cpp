// oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the pnnl/ripples IMM hot path, used exclusively as the
// checker by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
// bench.py.  Nothing in the product (ripples_b200/) links, loads or calls this
// file.  The algorithms are scalar C++ on purpose: simple enough to read
// against the reference line by line.  Only loops over independent items
// (sets listed by id, edge draws, per-vertex weights) run on several host
// threads, which leaves every result unchanged.
//
// What it restates (reference paths are relative to the ripples project):
//   * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
//     easy as 1, 2, 3", SC'11): the counter-based generator that keys every
//     random draw of the sampler on (seed, set id, edge id / vertex id).
//   * IC RRR-set sampling: reverse BFS over live in-edges,
//     include/ripples/add_rrrset.h:128-135 (edge live with probability w),
//     output sorted ascending as in add_rrrset.h:156.
//   * LT RRR-set sampling: one threshold per visited vertex, in-edges walked in
//     CSR order until the cumulative weight reaches the threshold, stop on a
//     revisit, include/ripples/add_rrrset.h:136-150.
//   * Roots uniform in [0, n), include/ripples/generate_rrr_sets.h:192-195.
//   * Greedy max coverage with the lazy max-heap and its tie-break:
//     include/ripples/streaming_find_most_influential.h:410-418 (CompareHeap),
//     :546-572 (getNextSeed), :607-643 (find_most_influential_set);
//     sequential twin include/ripples/find_most_influential.h:85-174.
//     The heap IS libstdc++'s std::priority_queue, exactly as in the reference,
//     so equal-count ties resolve identically.
//   * The lowest-id argmax tie-break of the reference's GPU seed selection,
//     src/gpu/find_most_influential.cc:65-72 (thrust::max_element).
//   * OPIM-C: include/ripples/opimc.h:60-98 (sample sizes and bounds, float
//     arithmetic), :101-118 (coverage of a seed set), :150-243 (the driver).
//   * Forward spread of a seed set, replica by replica:
//     include/ripples/diffusion_simulation.h:73-127 (IC) and :129-178 (LT,
//     restated in its live-edge form).
//   * IMM theta math and the martingale loop: include/ripples/imm.h:77-128
//     (ThetaPrime, InvThetaPrime, Theta), :145-260 (Sampling), :768-860 (IMM),
//     include/ripples/utility.h:84-87 (logBinomial).
//
// Sampler specification (shared with the CUDA kernels, restated here
// independently):
//   key                 = (seed & 0xffffffff, seed >> 32)
//   root(s)             = mulhi64(u64(P(s_lo, 0, 0, ROOT<<24 | s_hi)), n)
//   coin(s, e)          = coarse(s, e) << 16 | fine(s, e)
//   coarse(s, e)        = 16-bit half (e & 1) of word (e >> 1) & 3 of
//                         P(b_lo, b_hi, s_lo, IC<<24 | s_hi),  b = e >> 3
//   fine(s, e)          = P(e_lo, e_hi, s_lo, IC_FINE<<24 | s_hi)[0] & 0xffff
//   lt_threshold(s, v)  = P(v, 0, s_lo, LT<<24 | s_hi)[0]
//   IC edge e live for set s  <=>  coin(s, e) < thr[e]
//   thr[e] = clamp(floor(w_e * 2^32), 0, 2^32-1)
//   forward spread, replica r: sim_coin(r, e) as coin(s, e) with r for s
//   and the SIM_IC / SIM_IC_FINE domains
//   LT: first in-edge j of v (CSR order) with threshold < cum[j],
//       W_i = floor(clamp(w_i, 0, 2) * 2^40)            (exact, 64-bit)
//       cum[j] = min(min(sum_{i<=j} W_i, 2^41) >> 8, 2^32-1)
//       (integer sums: any summation order gives the same thresholds)

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <queue>
#include <utility>
#include <vector>
#include <sys/types.h>

#include <omp.h>
#include <parallel/algorithm>

namespace {

enum : uint32_t {
  DOM_ROOT = 1, DOM_IC = 2, DOM_LT = 3, DOM_RMAT = 4, DOM_ER = 5, DOM_WEIGHT = 6,
  DOM_SIM_IC = 7, DOM_SIM_LT = 8, DOM_IC_FINE = 9, DOM_SIM_IC_FINE = 10
};

void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                   uint32_t out[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += W0;
      k1 += W1;
    }
    uint64_t p0 = (uint64_t)M0 * c0;
    uint64_t p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

inline void make_key(uint64_t seed, uint32_t key[2]) {
  key[0] = (uint32_t)seed;
  key[1] = (uint32_t)(seed >> 32);
}

uint32_t root_of(uint64_t seed, uint64_t s, uint32_t n) {
  uint32_t key[2], ctr[4], out[4];
  make_key(seed, key);
  ctr[0] = (uint32_t)s;
  ctr[1] = 0;
  ctr[2] = 0;
  ctr[3] = (DOM_ROOT << 24) | (uint32_t)((s >> 32) & 0xFFFFFFu);
  philox4x32_10(ctr, key, out);
  uint64_t u = (uint64_t)out[0] | ((uint64_t)out[1] << 32);
  return (uint32_t)(((unsigned __int128)u * n) >> 64);
}

uint32_t ic_coarse(uint64_t seed, uint64_t s, uint64_t e) {
  uint32_t key[2], ctr[4], out[4];
  make_key(seed, key);
  const uint64_t b = e >> 3;
  ctr[0] = (uint32_t)b;
  ctr[1] = (uint32_t)(b >> 32);
  ctr[2] = (uint32_t)s;
  ctr[3] = (DOM_IC << 24) | (uint32_t)((s >> 32) & 0xFFFFFFu);
  philox4x32_10(ctr, key, out);
  const uint32_t w = out[(e >> 1) & 3];
  return (e & 1) ? (w >> 16) : (w & 0xFFFFu);
}

uint32_t ic_fine(uint64_t seed, uint64_t s, uint64_t e) {
  uint32_t key[2], ctr[4], out[4];
  make_key(seed, key);
  ctr[0] = (uint32_t)e;
  ctr[1] = (uint32_t)(e >> 32);
  ctr[2] = (uint32_t)s;
  ctr[3] = (DOM_IC_FINE << 24) | (uint32_t)((s >> 32) & 0xFFFFFFu);
  philox4x32_10(ctr, key, out);
  return out[0] & 0xFFFFu;
}

// The full 32-bit coin of edge e for set s.
uint32_t ic_coin(uint64_t seed, uint64_t s, uint64_t e) {
  return (ic_coarse(seed, s, e) << 16) | ic_fine(seed, s, e);
}

// coin(s, e) < thr, drawing the fine half only on a coarse tie.
bool ic_live(uint64_t seed, uint64_t s, uint64_t e, uint32_t thr) {
  const uint32_t c = ic_coarse(seed, s, e), th = thr >> 16;
  return c < th || (c == th && ic_fine(seed, s, e) < (thr & 0xFFFFu));
}

// Forward spread simulation coin of edge e in replica r (its own domains):
// coarse << 16 | fine, as ic_coin.
uint32_t sim_ic_coarse(uint64_t seed, uint64_t r, uint64_t e) {
  uint32_t key[2], ctr[4], out[4];
  make_key(seed, key);
  const uint64_t b = e >> 3;
  ctr[0] = (uint32_t)b;
  ctr[1] = (uint32_t)(b >> 32);
  ctr[2] = (uint32_t)r;
  ctr[3] = (DOM_SIM_IC << 24) | (uint32_t)((r >> 32) & 0xFFFFFFu);
  philox4x32_10(ctr, key, out);
  const uint32_t w = out[(e >> 1) & 3];
  return (e & 1) ? (w >> 16) : (w & 0xFFFFu);
}

uint32_t sim_ic_fine(uint64_t seed, uint64_t r, uint64_t e) {
  uint32_t key[2], ctr[4], out[4];
  make_key(seed, key);
  ctr[0] = (uint32_t)e;
  ctr[1] = (uint32_t)(e >> 32);
  ctr[2] = (uint32_t)r;
  ctr[3] = (DOM_SIM_IC_FINE << 24) | (uint32_t)((r >> 32) & 0xFFFFFFu);
  philox4x32_10(ctr, key, out);
  return out[0] & 0xFFFFu;
}

// sim coin(r, e) < thr, drawing the fine half only on a coarse tie.
bool sim_ic_live(uint64_t seed, uint64_t r, uint64_t e, uint32_t thr) {
  const uint32_t c = sim_ic_coarse(seed, r, e), th = thr >> 16;
  return c < th || (c == th && sim_ic_fine(seed, r, e) < (thr & 0xFFFFu));
}

// Forward LT spread: the threshold of vertex v in replica r (its own domain).
uint32_t sim_lt_threshold(uint64_t seed, uint64_t r, uint32_t v) {
  uint32_t key[2], ctr[4], out[4];
  make_key(seed, key);
  ctr[0] = v;
  ctr[1] = 0;
  ctr[2] = (uint32_t)r;
  ctr[3] = (DOM_SIM_LT << 24) | (uint32_t)((r >> 32) & 0xFFFFFFu);
  philox4x32_10(ctr, key, out);
  return out[0];
}

uint32_t lt_threshold(uint64_t seed, uint64_t s, uint32_t v) {
  uint32_t key[2], ctr[4], out[4];
  make_key(seed, key);
  ctr[0] = v;
  ctr[1] = 0;
  ctr[2] = (uint32_t)s;
  ctr[3] = (DOM_LT << 24) | (uint32_t)((s >> 32) & 0xFFFFFFu);
  philox4x32_10(ctr, key, out);
  return out[0];
}

uint32_t prob_to_u32(double x) {
  double y = x * 4294967296.0;
  if (!(y > 0.0)) return 0u;
  if (y >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)std::floor(y);
}

// ---- theta math: include/ripples/imm.h:77-128, utility.h:84-87 -------------
double logBinomial(size_t n, size_t k) {
  return lgamma(n + 1) - lgamma(n - k + 1) - lgamma(k + 1);
}

ssize_t ThetaPrime(ssize_t x, double epsilonPrime, double l, size_t k,
                   size_t num_nodes) {
  k = std::min(k, num_nodes / 2);
  return (2 + 2. / 3. * epsilonPrime) *
         (l * std::log(num_nodes) + logBinomial(num_nodes, k) +
          std::log(std::log2(num_nodes))) *
         std::pow(2.0, x) / (epsilonPrime * epsilonPrime);
}

ssize_t InvThetaPrime(ssize_t rrsize, double epsilonPrime, double l, size_t k,
                      size_t num_nodes) {
  k = std::min(k, num_nodes / 2);
  return std::log2(rrsize * epsilonPrime * epsilonPrime /
                   ((2 + 2. / 3. * epsilonPrime) *
                    (l * std::log(num_nodes) + logBinomial(num_nodes, k) +
                     std::log(std::log2(num_nodes)))));
}

size_t Theta(double epsilon, double l, size_t k, double LB, size_t num_nodes) {
  if (LB == 0) return 0;
  k = std::min(k, num_nodes / 2);
  double term1 = 0.6321205588285577;  // 1 - 1/e
  double alpha = sqrt(l * std::log(num_nodes) + std::log(2));
  double beta = sqrt(term1 * (logBinomial(num_nodes, k) +
                              l * std::log(num_nodes) + std::log(2)));
  double lamdaStar = 2 * num_nodes * (term1 * alpha + beta) *
                     (term1 * alpha + beta) * pow(epsilon, -2);
  return lamdaStar / LB;
}

// ---- sampling ------------------------------------------------------------
struct Graph {
  uint32_t n;
  const uint64_t *index;
  const uint32_t *src;
  const uint32_t *thr;  // IC thresholds or LT cumulative thresholds
};

struct SampleStats {
  uint64_t edges_scanned = 0;   // in-edges read (IC: all of each member)
  uint64_t expansions = 0;      // vertices expanded
};

// One IC set: reverse BFS from root(s) over live edges.
void sample_ic_one(const Graph &G, uint64_t seed, uint64_t s,
                   std::vector<uint32_t> &stamp, uint32_t tag,
                   std::vector<uint32_t> &out, SampleStats &st) {
  out.clear();
  uint32_t r = root_of(seed, s, G.n);
  out.push_back(r);
  stamp[r] = tag;
  for (size_t head = 0; head < out.size(); ++head) {
    uint32_t v = out[head];
    st.expansions++;
    for (uint64_t e = G.index[v]; e < G.index[v + 1]; ++e) {
      st.edges_scanned++;
      uint32_t u = G.src[e];
      if (stamp[u] == tag) continue;  // coins are pure: skipping is exact
      if (ic_live(seed, s, e, G.thr[e])) {
        stamp[u] = tag;
        out.push_back(u);
      }
    }
  }
  std::sort(out.begin(), out.end());
}

// One LT set: single-predecessor walk from root(s).
void sample_lt_one(const Graph &G, uint64_t seed, uint64_t s,
                   std::vector<uint32_t> &stamp, uint32_t tag,
                   std::vector<uint32_t> &out, SampleStats &st) {
  out.clear();
  uint32_t cur = root_of(seed, s, G.n);
  out.push_back(cur);
  stamp[cur] = tag;
  for (;;) {
    st.expansions++;
    uint32_t t = lt_threshold(seed, s, cur);
    uint64_t sel = UINT64_MAX;
    for (uint64_t e = G.index[cur]; e < G.index[cur + 1]; ++e) {
      st.edges_scanned++;
      if (t < G.thr[e]) {
        sel = e;
        break;
      }
    }
    if (sel == UINT64_MAX) break;
    uint32_t u = G.src[sel];
    if (stamp[u] == tag) break;
    stamp[u] = tag;
    out.push_back(u);
    cur = u;
  }
  std::sort(out.begin(), out.end());
}


// One set (IC or LT) with a visited bitmap the caller owns: the bits of the
// set's members are cleared again before returning, so one bitmap serves any
// number of sets.  Same semantics as sample_ic_one / sample_lt_one.
void sample_one_bits(const Graph &G, int model, uint64_t seed, uint64_t s,
                     std::vector<uint64_t> &bits, std::vector<uint32_t> &out) {
  auto test_set = [&](uint32_t v) {
    uint64_t &w = bits[v >> 6];
    const uint64_t b = 1ull << (v & 63);
    const bool was = (w & b) != 0;
    w |= b;
    return was;
  };
  out.clear();
  uint32_t r = root_of(seed, s, G.n);
  out.push_back(r);
  test_set(r);
  if (model == 0) {
    for (size_t head = 0; head < out.size(); ++head) {
      const uint32_t v = out[head];
      for (uint64_t e = G.index[v]; e < G.index[v + 1]; ++e) {
        const uint32_t u = G.src[e];
        if (bits[u >> 6] & (1ull << (u & 63))) continue;
        if (ic_live(seed, s, e, G.thr[e])) {
          test_set(u);
          out.push_back(u);
        }
      }
    }
  } else {
    uint32_t cur = r;
    for (;;) {
      const uint32_t t = lt_threshold(seed, s, cur);
      uint64_t sel = UINT64_MAX;
      for (uint64_t e = G.index[cur]; e < G.index[cur + 1]; ++e)
        if (t < G.thr[e]) {
          sel = e;
          break;
        }
      if (sel == UINT64_MAX) break;
      const uint32_t u = G.src[sel];
      if (test_set(u)) break;
      out.push_back(u);
      cur = u;
    }
  }
  for (uint32_t v : out) bits[v >> 6] &= ~(1ull << (v & 63));
  std::sort(out.begin(), out.end());
}

// ---- selection: include/ripples/streaming_find_most_influential.h ----------
struct CompareHeap {
  bool operator()(const std::pair<uint32_t, size_t> &a,
                  const std::pair<uint32_t, size_t> &b) const {
    return a.second < b.second;
  }
};

struct SelectResult {
  std::vector<uint32_t> seeds;
  std::vector<uint64_t> gains;
  uint64_t uncovered = 0;
  double f = 0.0;
};

// tiebreak 0: the reference CPU lazy heap; 1: lowest vertex id wins.
SelectResult select_sets(uint32_t n, uint64_t nsets, const uint64_t *off,
                         const uint32_t *vtx, uint32_t k, int tiebreak) {
  SelectResult R;
  std::vector<uint32_t> count(n, 0);
  uint64_t P = off[nsets] - off[0];
  const uint32_t *base = vtx;
  for (uint64_t i = 0; i < P; ++i) count[base[i]]++;
  // inverted index: vertex -> sets containing it
  std::vector<uint64_t> inv_off(n + 1, 0);
  for (uint32_t v = 0; v < n; ++v) inv_off[v + 1] = inv_off[v] + count[v];
  std::vector<uint64_t> inv(P);
  {
    std::vector<uint64_t> cur(inv_off.begin(), inv_off.end() - 1);
    for (uint64_t s = 0; s < nsets; ++s)
      for (uint64_t i = off[s]; i < off[s + 1]; ++i)
        inv[cur[vtx[i - off[0]]]++] = s;
  }
  std::vector<uint8_t> covered(nsets, 0);
  auto cover = [&](uint32_t v) {
    for (uint64_t j = inv_off[v]; j < inv_off[v + 1]; ++j) {
      uint64_t s = inv[j];
      if (covered[s]) continue;
      covered[s] = 1;
      for (uint64_t i = off[s]; i < off[s + 1]; ++i) count[vtx[i - off[0]]] -= 1;
    }
  };

  uint64_t uncovered = nsets;
  if (tiebreak == 0) {
    std::vector<std::pair<uint32_t, size_t>> storage(n);
    for (uint32_t v = 0; v < n; ++v) storage[v] = {v, count[v]};
    std::priority_queue<std::pair<uint32_t, size_t>,
                        std::vector<std::pair<uint32_t, size_t>>, CompareHeap>
        queue(CompareHeap{}, std::move(storage));
    while (R.seeds.size() < k && uncovered != 0) {
      std::pair<uint32_t, size_t> element;
      for (;;) {
        element = queue.top();
        queue.pop();
        if (element.second > count[element.first]) {
          element.second = count[element.first];
          queue.push(element);
          continue;
        }
        break;
      }
      uncovered -= element.second;
      R.seeds.push_back(element.first);
      R.gains.push_back(element.second);
      if (R.seeds.size() == k) break;
      cover(element.first);
    }
  } else {
    while (R.seeds.size() < k && uncovered != 0) {
      uint32_t best = 0;
      for (uint32_t v = 1; v < n; ++v)
        if (count[v] > count[best]) best = v;
      uncovered -= count[best];
      R.seeds.push_back(best);
      R.gains.push_back(count[best]);
      if (R.seeds.size() == k) break;
      cover(best);
    }
  }
  R.uncovered = uncovered;
  R.f = nsets ? double(nsets - uncovered) / nsets : 0.0;
  return R;
}

struct Pool {
  std::vector<uint64_t> off{0};
  std::vector<uint32_t> vtx;
};

void sample_range(const Graph &G, int model, uint64_t seed, uint64_t first,
                  uint64_t count, Pool &pool, SampleStats &st) {
  std::vector<uint32_t> stamp(G.n, 0);
  std::vector<uint32_t> one;
  uint32_t tag = 0;
  for (uint64_t s = first; s < first + count; ++s) {
    if (++tag == 0) {
      std::fill(stamp.begin(), stamp.end(), 0);
      tag = 1;
    }
    if (model == 0)
      sample_ic_one(G, seed, s, stamp, tag, one, st);
    else
      sample_lt_one(G, seed, s, stamp, tag, one, st);
    pool.vtx.insert(pool.vtx.end(), one.begin(), one.end());
    pool.off.push_back(pool.vtx.size());
  }
}

// OPIM-C (include/ripples/opimc.h:150-243; Tang, Tang, Xiao, Yuan, SIGMOD'18)
// over the oracle's samplers and selection.  Pool R1 holds the sets of key
// `seed`, pool R2 those of key seed + R2_KEY_OFFSET, both ids [0, theta).
// Bounds in the reference's float arithmetic (opimc.h:60-98).
constexpr uint64_t R2_KEY_OFFSET = 0x9E3779B97F4A7C15ull;
constexpr float OPIMC_A = 0.6321203113733684f;

float opimc_theta_helper(size_t n, size_t k, float delta) {
  float B = OPIMC_A * std::sqrt(std::log(6.0 / delta));
  float C = std::sqrt(OPIMC_A * (logBinomial(n, k) + std::log(6.0 / delta)));
  float D = (B + C) * (B + C);
  return 2 * D;
}

// (unqualified log / sqrt on float arguments, as the reference calls them)
float opimc_lower(size_t coverage, float delta2, size_t n, size_t theta) {
  float A = log(1 / delta2);
  float B = sqrt(coverage + 2 * A / 9);
  float C = sqrt(A / 2);
  float D = (B - C) * (B - C);
  float E = A / 18;
  return (float(n) / theta) * (D - E);
}

float opimc_upper(size_t coverage, float delta1, size_t n, size_t theta) {
  float B = coverage / OPIMC_A;
  float C = log(1 / delta1) / 2;
  float D = sqrt(B + C);
  double r = std::sqrt((double)C);  // (D + sqrt(C))^2 evaluates in double
  float E = (float)((D + r) * (D + r));
  return (float(n) / theta) * E;
}

uint64_t coverage_of(const Pool &P, uint64_t nsets, const std::vector<uint32_t> &seeds) {
  std::vector<uint32_t> S(seeds);
  std::sort(S.begin(), S.end());
  uint64_t covered = 0;
  for (uint64_t s = 0; s < nsets; ++s)
    for (uint64_t j = P.off[s]; j < P.off[s + 1]; ++j)
      if (std::binary_search(S.begin(), S.end(), P.vtx[j])) {
        ++covered;
        break;
      }
  return covered;
}

}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t *ctr, const uint32_t *key,
                       uint32_t *out) {
  philox4x32_10(ctr, key, out);
}

uint32_t orc_root(uint64_t seed, uint64_t s, uint32_t n) {
  return root_of(seed, s, n);
}

uint32_t orc_ic_coin(uint64_t seed, uint64_t s, uint64_t e) {
  return ic_coin(seed, s, e);
}

uint32_t orc_lt_threshold(uint64_t seed, uint64_t s, uint32_t v) {
  return lt_threshold(seed, s, v);
}

void orc_pack_ic(const float *w, uint64_t m, uint32_t *thr) {
  for (uint64_t e = 0; e < m; ++e) thr[e] = prob_to_u32((double)w[e]);
}

void orc_pack_lt(const uint64_t *index, uint32_t n, const float *w,
                 uint32_t *cum) {
  const uint64_t CAP = 1ull << 41;
  for (uint32_t v = 0; v < n; ++v) {
    uint64_t acc = 0;
    for (uint64_t e = index[v]; e < index[v + 1]; ++e) {
      double x = (double)w[e];
      uint64_t W = !(x > 0.0) ? 0 : x >= 2.0 ? (2ull << 40) : (uint64_t)std::floor(x * 1099511627776.0);
      acc = acc + W > CAP ? CAP : acc + W;
      uint64_t c = acc >> 8;
      cum[e] = c > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)c;
    }
  }
}

// Samples sets [first, first+count).  Returns an opaque pool handle; the
// caller reads it with orc_pool_* and releases it with orc_pool_free.
void *orc_sample(int model, uint32_t n, const uint64_t *index,
                 const uint32_t *src, const uint32_t *thr, uint64_t seed,
                 uint64_t first, uint64_t count, uint64_t *stats /*2*/) {
  Graph G{n, index, src, thr};
  Pool *p = new Pool();
  SampleStats st;
  sample_range(G, model, seed, first, count, *p, st);
  if (stats) {
    stats[0] = st.expansions;
    stats[1] = st.edges_scanned;
  }
  return p;
}

// Forward IC spread: replica r is a BFS from the seeds over the forward CSR
// (index over sources, dst[e] the target of out-edge e) in which edge e fires
// iff sim_ic_live(seed, r, e, thr[e]); sizes[r] = vertices reached, seeds
// included (include/ripples/diffusion_simulation.h:73-127).  Returns the sum
// of the sizes; *edges (optional) = out-edges of reached vertices, summed.
uint64_t orc_spread_ic(uint32_t n, const uint64_t *index, const uint32_t *dst,
                       const uint32_t *thr, const uint32_t *seeds, uint32_t k,
                       uint64_t replicas, uint64_t seed, uint32_t *sizes,
                       uint64_t *edges, uint32_t *levels) {
  uint64_t n_edges = 0;
  std::vector<uint64_t> stamp(n, ~0ull);
  std::vector<uint32_t> queue;
  uint64_t total = 0;
  for (uint64_t r = 0; r < replicas; ++r) {
    queue.clear();
    for (uint32_t i = 0; i < k; ++i)
      if (stamp[seeds[i]] != r) {
        stamp[seeds[i]] = r;
        queue.push_back(seeds[i]);
      }
    uint32_t lev = 0;
    for (size_t head = 0; head < queue.size(); ++lev) {  // one BFS level per pass
      const size_t end = queue.size();
      for (; head < end; ++head) {
        const uint32_t u = queue[head];
        n_edges += index[u + 1] - index[u];
        for (uint64_t e = index[u]; e < index[u + 1]; ++e) {
          const uint32_t v = dst[e];
          if (stamp[v] == r) continue;  // coins are pure: skipping is exact
          if (sim_ic_live(seed, r, e, thr[e])) {
            stamp[v] = r;
            queue.push_back(v);
          }
        }
      }
    }
    if (sizes) sizes[r] = (uint32_t)queue.size();
    if (levels) levels[r] = lev;
    total += queue.size();
  }
  if (edges) *edges = n_edges;
  return total;
}

uint64_t orc_spread_lt(uint32_t n, const uint64_t *findex, const uint32_t *fdst,
                       const uint64_t *bindex, const uint32_t *bsrc, const uint32_t *cum,
                       const uint32_t *seeds, uint32_t k, uint64_t replicas, uint64_t seed,
                       uint32_t *sizes, uint32_t *levels) {
  std::vector<uint64_t> stamp(n, ~0ull);
  std::vector<uint32_t> queue;
  uint64_t total = 0;
  for (uint64_t r = 0; r < replicas; ++r) {
    queue.clear();
    for (uint32_t i = 0; i < k; ++i)
      if (stamp[seeds[i]] != r) {
        stamp[seeds[i]] = r;
        queue.push_back(seeds[i]);
      }
    uint32_t lev = 0;
    for (size_t head = 0; head < queue.size(); ++lev) {
      const size_t end = queue.size();
      for (; head < end; ++head) {
        const uint32_t u = queue[head];
        for (uint64_t e = findex[u]; e < findex[u + 1]; ++e) {
          const uint32_t v = fdst[e];
          if (stamp[v] == r) continue;
          const uint32_t t = sim_lt_threshold(seed, r, v);
          uint64_t j = bindex[v];
          while (j < bindex[v + 1] && !(t < cum[j])) ++j;  // first j, CSR order
          if (j < bindex[v + 1] && bsrc[j] == u) {
            stamp[v] = r;
            queue.push_back(v);
          }
        }
      }
    }
    if (sizes) sizes[r] = (uint32_t)queue.size();
    if (levels) levels[r] = lev;
    total += queue.size();
  }
  return total;
}

// OPIM-C's coverage check (include/ripples/opimc.h:101-118, FindCoverage):
// the number of sets [0, nsets) holding at least one of the k seeds.
uint64_t orc_find_coverage(uint64_t nsets, const uint64_t *off, const uint32_t *vtx,
                           const uint32_t *seeds, uint32_t k) {
  std::vector<uint32_t> S(seeds, seeds + k);
  std::sort(S.begin(), S.end());
  uint64_t covered = 0;
  for (uint64_t s = 0; s < nsets; ++s)
    for (uint64_t j = off[s]; j < off[s + 1]; ++j)
      if (std::binary_search(S.begin(), S.end(), vtx[j])) {
        ++covered;
        break;
      }
  return covered;
}

// OPIM-C driver; returns the number of seeds written.  theta_out: the final
// pool size; rounds: selections run; thetas[0..1] = theta_0, theta_max.
uint32_t orc_opimc(int model, uint32_t n, const uint64_t *index, const uint32_t *src,
                   const uint32_t *thr, uint32_t k, float epsilon, float delta,
                   uint64_t seed, int tiebreak, uint32_t *seeds, uint64_t *theta_out,
                   uint32_t *rounds, uint64_t *thetas) {
  Graph G{n, index, src, thr};
  Pool R1, R2;
  SampleStats st;
  size_t theta = (size_t)std::ceil(opimc_theta_helper(n, k, delta));
  const size_t theta_max =
      (size_t)std::ceil(n * opimc_theta_helper(n, k, delta) / (epsilon * epsilon * k));
  thetas[0] = theta;
  thetas[1] = theta_max;
  sample_range(G, model, seed, 0, theta, R1, st);
  sample_range(G, model, seed + R2_KEY_OFFSET, 0, theta, R2, st);
  const size_t i_max = (size_t)std::ceil(std::log2(theta_max / theta));
  const float d = delta / (3 * i_max);
  std::vector<uint32_t> result;
  uint32_t r = 0;
  for (;; ++r) {
    SelectResult S = select_sets(n, theta, R1.off.data(), R1.vtx.data(), k, tiebreak);
    const size_t cov1 = (size_t)(S.f * theta);  // the reference scales f back
    const size_t cov2 = coverage_of(R2, theta, S.seeds);
    const float upper = opimc_upper(cov1, d, n, theta);
    const float lower = opimc_lower(cov2, d, n, theta);
    result = S.seeds;
    if (lower / upper >= (OPIMC_A - epsilon)) break;
    if (theta >= theta_max) break;  // the paper's cap; the reference has none
    const size_t grow = theta;  // theta doubles
    sample_range(G, model, seed, theta, grow, R1, st);
    sample_range(G, model, seed + R2_KEY_OFFSET, theta, grow, R2, st);
    theta *= 2;
  }
  for (size_t i = 0; i < result.size(); ++i) seeds[i] = result[i];
  *theta_out = theta;
  *rounds = r + 1;
  return (uint32_t)result.size();
}

void orc_opimc_math(uint64_t n, float epsilon, uint64_t k, float delta, uint64_t coverage,
                    uint64_t theta, uint64_t *thetas, float *bounds) {
  thetas[0] = (uint64_t)std::ceil(opimc_theta_helper(n, k, delta));
  thetas[1] = (uint64_t)std::ceil(n * opimc_theta_helper(n, k, delta) / (epsilon * epsilon * k));
  bounds[0] = opimc_lower(coverage, delta, n, theta);
  bounds[1] = opimc_upper(coverage, delta, n, theta);
}

uint64_t orc_pool_elements(void *h) { return ((Pool *)h)->vtx.size(); }
uint64_t orc_pool_sets(void *h) { return ((Pool *)h)->off.size() - 1; }
void orc_pool_copy(void *h, uint64_t *off, uint32_t *vtx) {
  Pool *p = (Pool *)h;
  std::memcpy(off, p->off.data(), p->off.size() * sizeof(uint64_t));
  if (!p->vtx.empty())
    std::memcpy(vtx, p->vtx.data(), p->vtx.size() * sizeof(uint32_t));
}
void orc_pool_free(void *h) { delete (Pool *)h; }

// Greedy max coverage over nsets sets given as CSR (off[0..nsets], vtx).
// Writes up to k seeds and their marginal gains; returns the number of seeds.
uint32_t orc_select(uint32_t n, uint64_t nsets, const uint64_t *off,
                    const uint32_t *vtx, uint32_t k, int tiebreak,
                    uint32_t *seeds, uint64_t *gains, double *f,
                    uint64_t *uncovered) {
  SelectResult R = select_sets(n, nsets, off, vtx, k, tiebreak);
  for (size_t i = 0; i < R.seeds.size(); ++i) {
    seeds[i] = R.seeds[i];
    gains[i] = R.gains[i];
  }
  *f = R.f;
  *uncovered = R.uncovered;
  return (uint32_t)R.seeds.size();
}

int64_t orc_theta_prime(int64_t x, double eps_prime, double l, uint64_t k,
                        uint64_t n) {
  return ThetaPrime(x, eps_prime, l, k, n);
}
int64_t orc_inv_theta_prime(int64_t rrsize, double eps_prime, double l,
                            uint64_t k, uint64_t n) {
  return InvThetaPrime(rrsize, eps_prime, l, k, n);
}
uint64_t orc_theta(double eps, double l, uint64_t k, double LB, uint64_t n) {
  return Theta(eps, l, k, LB, n);
}
double orc_log_binomial(uint64_t n, uint64_t k) { return logBinomial(n, k); }

// Full IMM (omp_parallel_tag flavour of include/ripples/imm.h:768-860) over
// the restated sampler.  Set ids are assigned 0, 1, 2, ... in generation
// order and the final selection runs over sets [0, theta).
// Outputs: seeds (k slots), *nseeds, *theta, deltas (up to 64 slots, one per
// martingale round), *nrounds, *f_final, *total_sets.
int orc_imm(int model, uint32_t n, const uint64_t *index, const uint32_t *src,
            const uint32_t *thr, uint32_t k, double epsilon, uint64_t seed,
            int tiebreak, uint32_t *seeds, uint32_t *nseeds, uint64_t *theta,
            uint64_t *deltas, uint32_t *nrounds, double *f_final,
            uint64_t *total_sets) {
  Graph G{n, index, src, thr};
  Pool pool;
  SampleStats st;
  double l = 1.0;
  l = l * (1 + 1 / std::log2(n));
  double epsilonPrime = 1.4142135623730951 * epsilon;
  double LB = 0;
  ssize_t x = 1;
  uint32_t rounds = 0;
  for (; x < std::log2(n); ++x) {
    ssize_t thetaPrime = ThetaPrime(x, epsilonPrime, l, k, n);
    size_t have = pool.off.size() - 1;
    double f = 0;
    if ((size_t)thetaPrime <= have) {
      if (rounds < 64) deltas[rounds] = 0;
    } else {
      size_t delta = thetaPrime - have;
      if (rounds < 64) deltas[rounds] = delta;
      sample_range(G, model, seed, have, delta, pool, st);
    }
    ++rounds;
    size_t now = pool.off.size() - 1;
    SelectResult S =
        select_sets(n, now, pool.off.data(), pool.vtx.data(), k, tiebreak);
    f = S.f;
    if (f >= std::pow(2, -x)) {
      LB = (n * f) / (1 + epsilonPrime);
      break;
    }
  }
  size_t th = Theta(epsilon, l, k, LB, n);
  size_t have = pool.off.size() - 1;
  if (th > have) sample_range(G, model, seed, have, th - have, pool, st);
  SelectResult S = select_sets(n, th, pool.off.data(), pool.vtx.data(), k,
                               tiebreak);
  for (size_t i = 0; i < S.seeds.size(); ++i) seeds[i] = S.seeds[i];
  *nseeds = (uint32_t)S.seeds.size();
  *theta = th;
  *nrounds = rounds;
  *f_final = S.f;
  *total_sets = pool.off.size() - 1;
  return 0;
}

// Samples the sets whose ids are listed: pool set i is set ids[i].  Sets are
// pure functions of (seed, id), so they are drawn in parallel over the host
// threads (one n-bit visited bitmap per thread).
void *orc_sample_ids(int model, uint32_t n, const uint64_t *index, const uint32_t *src,
                     const uint32_t *thr, uint64_t seed, const uint64_t *ids,
                     uint64_t count) {
  Graph G{n, index, src, thr};
  std::vector<std::vector<uint32_t>> sets(count);
#pragma omp parallel
  {
    std::vector<uint64_t> bits(((size_t)n + 63) / 64, 0);
#pragma omp for schedule(dynamic, 1)
    for (uint64_t i = 0; i < count; ++i) sample_one_bits(G, model, seed, ids[i], bits, sets[i]);
  }
  Pool *p = new Pool();
  for (auto &one : sets) {
    p->vtx.insert(p->vtx.end(), one.begin(), one.end());
    p->off.push_back(p->vtx.size());
  }
  return p;
}

// ---- synthetic input graphs ------------------------------------------------
// The R-MAT (Chakrabarti, Zhan, Faloutsos, SDM'04) and Erdos-Renyi draws and
// weight models the library's host graph builders use, restated so that the
// reference's input files can be written without loading the library:
//   R-MAT draw i, level l: quadrant from P(i_lo, i_hi, l/4, RMAT<<24)[l%4]
//     against the cumulative thresholds of a, a+b, a+b+c (u32 fixed point);
//     bit l of (src, dst) from most significant down; self-loops dropped.
//   keys (dst<<32 | src) sorted and de-duplicated = the backward CSR.
//   weights of CSR edge e from P(e_lo, e_hi, 0, WEIGHT<<24)[0] >> 8 / 2^24.
int orc_rmat_csr(uint32_t scale, uint64_t draws, double a, double b, double c,
                 uint64_t seed, uint64_t **index_out, uint32_t **src_out, uint64_t *m_out) {
  if (scale == 0 || scale > 31) return -1;
  const uint32_t n = 1u << scale;
  const uint32_t TA = prob_to_u32(a), TB = prob_to_u32(a + b), TC = prob_to_u32(a + b + c);
  uint32_t key[2];
  make_key(seed, key);
  std::vector<uint64_t> keys(draws, ~0ull);
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < draws; ++i) {
    uint32_t s = 0, d = 0, rnd[4] = {0, 0, 0, 0};
    for (uint32_t l = 0; l < scale; ++l) {
      if ((l & 3) == 0) {
        const uint32_t ctr[4] = {(uint32_t)i, (uint32_t)(i >> 32), l >> 2, DOM_RMAT << 24};
        philox4x32_10(ctr, key, rnd);
      }
      const uint32_t u = rnd[l & 3];
      const uint32_t row = u >= TB;                          // quadrants c, d
      const uint32_t col = (u >= TA && u < TB) || u >= TC;   // quadrants b, d
      s |= row << (scale - 1 - l);
      d |= col << (scale - 1 - l);
    }
    if (s != d) keys[i] = ((uint64_t)d << 32) | s;
  }
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  if (!keys.empty() && keys.back() == ~0ull) keys.pop_back();  // the dropped self-loops
  const uint64_t m = keys.size();
  uint64_t *index = (uint64_t *)std::calloc((size_t)n + 1, sizeof(uint64_t));
  uint32_t *src = (uint32_t *)std::malloc(sizeof(uint32_t) * (m ? m : 1));
  if (!index || !src) {
    std::free(index);
    std::free(src);
    return -1;
  }
#pragma omp parallel for schedule(static)
  for (uint64_t e = 0; e < m; ++e) src[e] = (uint32_t)keys[e];
  for (uint64_t e = 0; e < m; ++e) index[(keys[e] >> 32) + 1]++;
  for (uint32_t v = 0; v < n; ++v) index[v + 1] += index[v];
  *index_out = index;
  *src_out = src;
  *m_out = m;
  return 0;
}

// kind 0: U(lo, hi) per edge; 1: U(0,1) normalised per destination (sum in
// double over the float draws, CSR order); 2: weighted cascade 1/in-degree.
int orc_make_weights(int kind, uint32_t n, const uint64_t *index, uint64_t seed, double lo,
                     double hi, float *w) {
  uint32_t key[2];
  make_key(seed, key);
  auto unif = [&](uint64_t e) {
    uint32_t rnd[4];
    const uint32_t ctr[4] = {(uint32_t)e, (uint32_t)(e >> 32), 0, DOM_WEIGHT << 24};
    philox4x32_10(ctr, key, rnd);
    return (double)(rnd[0] >> 8) / 16777216.0;
  };
  if (kind < 0 || kind > 2) return -1;
#pragma omp parallel for schedule(dynamic, 4096)
  for (uint64_t v = 0; v < n; ++v) {
    const uint64_t b = index[v], e1 = index[v + 1];
    if (kind == 0) {
      for (uint64_t e = b; e < e1; ++e) w[e] = (float)(lo + (hi - lo) * unif(e));
    } else if (kind == 1) {
      double sum = 0.0;
      for (uint64_t e = b; e < e1; ++e) {
        w[e] = (float)unif(e);
        sum += (double)w[e];
      }
      for (uint64_t e = b; e < e1; ++e) w[e] = sum > 0.0 ? (float)((double)w[e] / sum) : 0.0f;
    } else {
      for (uint64_t e = b; e < e1; ++e) w[e] = (float)(1.0 / (double)(e1 - b));
    }
  }
  return 0;
}

void orc_free(void *p) { std::free(p); }

}  // extern "C"
