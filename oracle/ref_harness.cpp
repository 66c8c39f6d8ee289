// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiled against the unmodified ripples headers (include/ripples/*.h) by
// oracle/ref.mk into oracle/_ref/libref_harness.so.  It exposes the
// reference's own seed selection, theta math and sequential samplers through a
// C ABI so tests can pin the oracle (oracle/oracle.cpp) against the reference
// itself:
//   ref_select      -> ripples::FindMostInfluentialSet, omp_parallel_tag
//                      (include/ripples/find_most_influential.h:176-196) or
//                      sequential_tag (:85-174)
//   ref_theta_*     -> include/ripples/imm.h:77-128
//   ref_sample      -> ripples::AddRRRSet (include/ripples/add_rrrset.h:105-157)
//                      driven like GenerateRRRSets, sequential_tag
//                      (include/ripples/generate_rrr_sets.h:186-198), with the
//                      project's trng interface shim as the random stream.
//   ref_simulate    -> ripples::simulate (include/ripples/diffusion_simulation.h)
//   ref_simulate_parallel -> the replica loop of tools/simulator.cc:139-149
//   ref_opimc_*, ref_find_coverage
//                   -> include/ripples/opimc.h:60-118
//   ref_generate_parallel -> the imm tool's `-p --rrsets N` path
//                      (tools/imm.cc:224-262): an ICStreamingGenerator over
//                      every OpenMP thread and one GenerateRRRSets call,
//                      omp_parallel_tag (generate_rrr_sets.h:214-224)
//   ref_imm_sequential -> the imm tool's sequential path (tools/imm.cc:313-323,
//                      ripples::IMM with sequential_tag) with a chosen seed
//   ref_graph_load_tsv / ref_graph_copy
//                   -> the sequential TSV loader (include/ripples/loaders.h:138-196)
//                      and the GraphBwd constructor (include/ripples/graph.h:506-620)
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "ripples/find_most_influential.h"
#include "ripples/generate_rrr_sets.h"
#include "ripples/graph.h"
#include "ripples/imm.h"
#include "ripples/imm_configuration.h"
#include "ripples/imm_interface.h"
#include "ripples/streaming_rrr_generator.h"
#include "ripples/diffusion_simulation.h"
#include "ripples/loaders.h"
#include "ripples/opimc.h"
#include "spdlog/sinks/stdout_color_sinks.h"

namespace {

struct MiniGraph {
  using vertex_type = uint32_t;
  size_t n;
  size_t num_nodes() const { return n; }
};

struct MiniCFG {
  size_t k;
  size_t seed_select_max_workers;
  size_t seed_select_max_gpu_workers;
};

using RRRsets = std::vector<std::vector<uint32_t>>;

RRRsets make_sets(uint64_t nsets, const uint64_t *off, const uint32_t *vtx) {
  RRRsets RR(nsets);
  for (uint64_t s = 0; s < nsets; ++s)
    RR[s].assign(vtx + off[s], vtx + off[s + 1]);
  return RR;
}

void ensure_console() {
  if (!spdlog::get("console")) spdlog::stdout_color_st("console");
  spdlog::set_level(spdlog::level::warn);
}

}  // namespace

extern "C" {

// Returns the number of seeds written.  omp != 0 selects omp_parallel_tag.
uint32_t ref_select(uint32_t n, uint64_t nsets, const uint64_t *off,
                    const uint32_t *vtx, uint32_t k, int omp, int threads,
                    uint32_t *seeds, double *f) {
  ensure_console();
  MiniGraph G{n};
  MiniCFG CFG{k, (size_t)(threads > 0 ? threads : 1), 0};
  RRRsets RR = make_sets(nsets, off, vtx);
  ripples::FindMostInfluentialSetRecord record;
  std::pair<double, std::vector<uint32_t>> S;
  if (omp) {
    if (threads > 0) omp_set_num_threads(threads);
    S = ripples::FindMostInfluentialSet(G, CFG, RR.begin(), RR.end(), record,
                                        false, ripples::omp_parallel_tag{});
  } else {
    S = ripples::FindMostInfluentialSet(G, CFG, RR.begin(), RR.end(), record,
                                        false, ripples::sequential_tag{});
  }
  for (size_t i = 0; i < S.second.size(); ++i) seeds[i] = S.second[i];
  *f = S.first;
  return (uint32_t)S.second.size();
}

int64_t ref_theta_prime(int64_t x, double eps_prime, double l, uint64_t k,
                        uint64_t n) {
  return ripples::ThetaPrime(x, eps_prime, l, k, n, ripples::sequential_tag{});
}

int64_t ref_inv_theta_prime(int64_t rrsize, double eps_prime, double l,
                            uint64_t k, uint64_t n) {
  return ripples::InvThetaPrime(rrsize, eps_prime, l, k, n,
                                ripples::sequential_tag{});
}

uint64_t ref_theta(double eps, double l, uint64_t k, double LB, uint64_t n) {
  return ripples::Theta(eps, l, k, LB, n);
}

double ref_log_binomial(uint64_t n, uint64_t k) {
  return ripples::logBinomial(n, k);
}

// Loads a reference-format binary graph (backward direction) from `path`.
static ripples::GraphBwd *load(const char *path) {
  auto *G = new ripples::GraphBwd();
  G->load_binary(path);
  return G;
}

void *ref_graph_load(const char *path) {
  ensure_console();
  return load(path);
}
void ref_graph_free(void *g) { delete (ripples::GraphBwd *)g; }
uint64_t ref_graph_nodes(void *g) { return ((ripples::GraphBwd *)g)->num_nodes(); }
uint64_t ref_graph_edges(void *g) { return ((ripples::GraphBwd *)g)->num_edges(); }

// The replica loop of tools/simulator.cc:139-149 (OpenMP over replicas, one
// trng stream per thread split as the tool splits them) without the tool's
// log sink (a rotating sink of max size 0, which the vendored spdlog
// rejects).  Returns the mean activated count.
double ref_simulate_parallel(const char *fwd_path, int model, const uint32_t *seeds,
                             uint32_t nseeds, uint64_t replicas) {
  ensure_console();
  ripples::GraphFwd G;
  G.load_binary(fwd_path);
  std::vector<uint32_t> S(seeds, seeds + nseeds);
  G.transformID(S.begin(), S.end(), S.begin());
  std::vector<trng::lcg64> generator(omp_get_max_threads());
#pragma omp parallel
  {
    generator[omp_get_thread_num()].seed(0UL);
    generator[omp_get_thread_num()].split(2, 1);
    generator[omp_get_thread_num()].split(omp_get_num_threads(), omp_get_thread_num());
  }
  std::vector<size_t> reached(replicas);
#pragma omp parallel for schedule(dynamic)
  for (uint64_t i = 0; i < replicas; ++i) {
    if (model == 0)
      reached[i] = ripples::simulate(G, S.begin(), S.end(), generator[omp_get_thread_num()],
                                     ripples::independent_cascade_tag{}).first;
    else
      reached[i] = ripples::simulate(G, S.begin(), S.end(), generator[omp_get_thread_num()],
                                     ripples::linear_threshold_tag{}).first;
  }
  double acc = 0.0;
  for (size_t x : reached) acc += (double)x;
  return replicas ? acc / (double)replicas : 0.0;
}

// OPIM-C arithmetic (include/ripples/opimc.h:60-98) and FindCoverage
// (:101-118): the number of sets holding at least one seed.
uint64_t ref_opimc_theta_max(uint64_t n, float eps, uint64_t k, float delta) {
  return ripples::ThetaMax(n, eps, k, delta);
}
uint64_t ref_opimc_theta_zero(uint64_t n, float eps, uint64_t k, float delta) {
  return ripples::ThetaZero(n, eps, k, delta);
}
float ref_opimc_lower_bound(uint64_t cov, float delta2, uint64_t n, uint64_t theta) {
  return ripples::LowerBound(cov, delta2, n, theta);
}
float ref_opimc_upper_bound(uint64_t cov, float delta1, uint64_t n, uint64_t theta) {
  return ripples::UpperBound(cov, delta1, n, theta);
}
uint64_t ref_find_coverage(uint64_t nsets, const uint64_t *off, const uint32_t *vtx,
                           const uint32_t *seeds, uint32_t k) {
  RRRsets RR = make_sets(nsets, off, vtx);
  std::vector<uint32_t> S(seeds, seeds + k);
  return ripples::FindCoverage(RR, S);
}

// Loads an unweighted TSV edge list with the reference's sequential loader
// (include/ripples/loaders.h:138-196; weights from the shim's uniform01
// stream, LT weights normalised per source) into the GraphBwd its constructor
// builds (include/ripples/graph.h:506-620), renumbering when `renumber`.
// (The weighted loader, loaders.h:211-296, parses its per-thread chunk buffer
// as an unterminated C string, so it is not used here.)
void *ref_graph_load_tsv(const char *path, int undirected, int lt, int renumber) {
  ensure_console();
  using E = ripples::Edge<uint32_t, float>;
  trng::lcg64 lcg;
  lcg.seed(0UL);
  lcg.split(2, 0);
  ripples::WeightGenerator<trng::lcg64, trng::uniform01_dist<float>, float> gen(lcg, 1.0f);
  std::vector<E> edges;
  if (lt)
    edges = ripples::load<E>(std::string(path), undirected != 0, gen, ripples::edge_list_tsv{},
                             ripples::linear_threshold_tag{});
  else
    edges = ripples::load<E>(std::string(path), undirected != 0, gen, ripples::edge_list_tsv{},
                             ripples::independent_cascade_tag{});
  return new ripples::GraphBwd(edges.begin(), edges.end(), renumber != 0);
}

// The graph's CSR and id map: index u64[n+1], src u32[m], w f32[m],
// reverse_map u32[n] (internal id -> input id, Graph::convertID).
void ref_graph_copy(void *g, uint64_t *index, uint32_t *src, float *w, uint32_t *reverse_map) {
  auto &G = *(ripples::GraphBwd *)g;
  const uint64_t n = G.num_nodes(), m = G.num_edges();
  const auto *idx = G.csr_index();
  for (uint64_t v = 0; v <= n; ++v) index[v] = (uint64_t)idx[v];
  for (uint64_t e = 0; e < m; ++e) {
    src[e] = G.csr_edges()[e];
    w[e] = G.csr_weights()[e];
  }
  for (uint64_t v = 0; v < n; ++v) reverse_map[v] = G.convertID((uint32_t)v);
}

// Samples `count` sets with the reference sequential sampler; model 0 = IC,
// 1 = LT.  Writes the total element count to *nelem and returns a handle to
// read with ref_pool_copy / release with ref_pool_free.
void *ref_sample(void *g, int model, uint64_t count, uint64_t seed,
                 uint64_t *nelem) {
  auto &G = *(ripples::GraphBwd *)g;
  std::vector<trng::lcg64> gen(1);
  gen[0].seed(seed);
  gen[0].split(2, 1);
  auto *RR = new ripples::RRRsets<ripples::GraphBwd>(count);
  ripples::IMMExecutionRecord rec;
  if (model == 0)
    ripples::GenerateRRRSets(G, gen, RR->begin(), RR->end(), rec,
                             ripples::independent_cascade_tag{},
                             ripples::sequential_tag{});
  else
    ripples::GenerateRRRSets(G, gen, RR->begin(), RR->end(), rec,
                             ripples::linear_threshold_tag{},
                             ripples::sequential_tag{});
  uint64_t tot = 0;
  for (auto &s : *RR) tot += s.size();
  *nelem = tot;
  return RR;
}

void ref_pool_copy(void *h, uint64_t *off, uint32_t *vtx) {
  auto &RR = *(ripples::RRRsets<ripples::GraphBwd> *)h;
  off[0] = 0;
  for (size_t s = 0; s < RR.size(); ++s) {
    std::memcpy(vtx + off[s], RR[s].data(), RR[s].size() * sizeof(uint32_t));
    off[s + 1] = off[s] + RR[s].size();
  }
}
void ref_pool_free(void *h) {
  delete (ripples::RRRsets<ripples::GraphBwd> *)h;
}

// Monte Carlo spread of `seeds` (internal ids) on a FORWARD-direction graph
// loaded from `fwd_path`, with the reference simulator: returns the mean
// number of activated vertices over `replicas` runs.
double ref_simulate(const char *fwd_path, int model, const uint32_t *seeds,
                    uint32_t nseeds, uint64_t replicas, uint64_t seed) {
  ensure_console();
  ripples::GraphFwd G;
  G.load_binary(fwd_path);
  std::vector<uint32_t> S(seeds, seeds + nseeds);
  trng::lcg64 gen;
  gen.seed(seed);
  gen.split(2, 1);
  double acc = 0.0;
  for (uint64_t r = 0; r < replicas; ++r) {
    std::pair<size_t, size_t> res;
    if (model == 0)
      res = ripples::simulate(G, S.begin(), S.end(), gen,
                              ripples::independent_cascade_tag{});
    else
      res = ripples::simulate(G, S.begin(), S.end(), gen,
                              ripples::linear_threshold_tag{});
    acc += (double)res.first;
  }
  return acc / (double)replicas;
}

// The mean of the second member of ripples::simulate's result (BFS levels /
// rounds, the seeds' included), replicas as ref_simulate runs them.
double ref_simulate_levels(const char *fwd_path, int model, const uint32_t *seeds,
                           uint32_t nseeds, uint64_t replicas, uint64_t seed) {
  ensure_console();
  ripples::GraphFwd G;
  G.load_binary(fwd_path);
  std::vector<uint32_t> S(seeds, seeds + nseeds);
  trng::lcg64 gen;
  gen.seed(seed);
  gen.split(2, 1);
  double acc = 0.0;
  for (uint64_t r = 0; r < replicas; ++r) {
    std::pair<size_t, size_t> res;
    if (model == 0)
      res = ripples::simulate(G, S.begin(), S.end(), gen,
                              ripples::independent_cascade_tag{});
    else
      res = ripples::simulate(G, S.begin(), S.end(), gen,
                              ripples::linear_threshold_tag{});
    acc += (double)res.second;
  }
  return acc / (double)replicas;
}

// The imm tool's `-p --rrsets N` sampling (tools/imm.cc:224-262 with
// CFG.num_rr_sets = count): master lcg64 seeded `seed` and split(2, 1), an
// ICStreamingGenerator with one CPU worker per OpenMP thread, no GPU workers,
// the default 64-colour CPU batches, then GenerateRRRSets over `count`
// pre-inserted empty sets.  Returns the milliseconds of that call alone (the
// tool's ThetaEstimationGenerateRRR entry) and the element count.
double ref_generate_parallel(void *g, uint64_t count, uint64_t seed, uint64_t *nelem) {
  ensure_console();
  auto &G = *(ripples::GraphBwd *)g;
  trng::lcg64 generator;
  generator.seed(seed);
  generator.split(2, 1);
  const size_t workers = omp_get_max_threads();
  std::unordered_map<size_t, size_t> worker_to_gpu;
  ripples::ICStreamingGenerator se(G, generator, workers, 0, 0, 64, 64, worker_to_gpu, 1.0f);
  ripples::IMMExecutionRecord R;
  ripples::RRRsetAllocator<uint32_t> allocator;
  std::vector<ripples::RRRset<ripples::GraphBwd>> RR;
  const auto t0 = std::chrono::high_resolution_clock::now();
  RR.insert(RR.end(), count, ripples::RRRset<ripples::GraphBwd>(allocator));
  ripples::GenerateRRRSets(G, se, RR.end() - count, RR.end(), R,
                           ripples::independent_cascade_tag{}, ripples::omp_parallel_tag{});
  const auto t1 = std::chrono::high_resolution_clock::now();
  uint64_t tot = 0;
  for (auto &s : RR) tot += s.size();
  *nelem = tot;
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// The imm tool's sequential IMM (tools/imm.cc:313-323) with the master
// lcg64 seeded `seed` instead of 0.  model 0 = IC, 1 = LT.  Writes the seeds
// (input ids) and returns their number.
uint32_t ref_imm_sequential(void *g, int model, uint32_t k, double epsilon, uint64_t seed,
                            uint32_t *seeds_out) {
  ensure_console();
  auto &G = *(ripples::GraphBwd *)g;
  ripples::IMMConfiguration CFG;
  CFG.k = k;
  CFG.epsilon = epsilon;
  trng::lcg64 generator;
  generator.seed(seed);
  generator.split(2, 1);
  ripples::IMMExecutionRecord R;
  std::vector<uint32_t> seeds;
  if (model == 0)
    seeds = ripples::IMM(G, CFG, 1.0, generator, R, ripples::independent_cascade_tag{},
                         ripples::sequential_tag{});
  else
    seeds = ripples::IMM(G, CFG, 1.0, generator, R, ripples::linear_threshold_tag{},
                         ripples::sequential_tag{});
  G.convertID(seeds.begin(), seeds.end(), seeds.begin());
  for (size_t i = 0; i < seeds.size(); ++i) seeds_out[i] = seeds[i];
  return (uint32_t)seeds.size();
}

}  // extern "C"
