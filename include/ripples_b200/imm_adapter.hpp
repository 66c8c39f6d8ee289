// imm_adapter.hpp -- drop-in binding of ripples_b200 for pnnl/ripples C++ code.
//
// Include after the ripples headers.  It adds, in namespace ripples:
//   * b200_tag                    an execution tag, used like omp_parallel_tag
//                                 (include/ripples/utility.h:71-78);
//   * B200RRRGenerator<GraphTy>   the generator object IMM is handed in place
//                                 of StreamingRRRGenerator
//                                 (include/ripples/streaming_rrr_generator.h:833):
//                                 generate(begin, end, record), isGpuEnabled();
//   * GenerateRRRSets(G, gen, begin, end, record, model_tag, b200_tag)
//                                 (include/ripples/generate_rrr_sets.h:186-224):
//                                 fills the caller's pre-inserted empty sets,
//                                 each sorted ascending;
//   * FindMostInfluentialSet(G, CFG, b, e, record, enableGPU, b200_tag)
//                                 (include/ripples/find_most_influential.h:85-196):
//                                 greedy max coverage on the GPU with the
//                                 reference's CPU heap tie-break, returns (f, seeds);
//   * IMM(G, CFG, l, gen, record, model_tag, b200_tag)
//                                 (include/ripples/imm.h:768-860): the whole
//                                 martingale + final selection on the device,
//                                 filling IMMExecutionRecord as the imm tool
//                                 expects for its JSON log.
// Errors from the library are thrown as std::runtime_error with the library's
// message (the reference throws std::logic_error / std::domain_error).
#ifndef RIPPLES_B200_IMM_ADAPTER_HPP
#define RIPPLES_B200_IMM_ADAPTER_HPP

#include <chrono>
#include <cstdint>
#include <iterator>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "ripples_b200.h"

namespace ripples {

struct b200_tag {};

namespace b200_detail {
inline void check(int rc, rip_ctx *ctx, const char *what) {
  if (rc != RIP_OK)
    throw std::runtime_error(std::string(what) + ": " +
                             (ctx ? rip_last_error(ctx) : "error") + " (" +
                             std::to_string(rc) + ")");
}
template <typename Tag>
constexpr int model_of() {
  return std::is_same<std::decay_t<Tag>, linear_threshold_tag>::value ? RIP_MODEL_LT
                                                                      : RIP_MODEL_IC;
}

// Records that carry GenerateRRRSetsRecord::WalkIterations
// (include/ripples/generate_rrr_sets_record.h:69-91) get one iteration entry
// per generate() call; other record types are left alone.
template <typename R, typename = void>
struct has_walk_iterations : std::false_type {};
template <typename R>
struct has_walk_iterations<R, std::void_t<decltype(std::declval<R &>().WalkIterations)>>
    : std::true_type {};

template <typename R>
void record_walk(R &rec, uint64_t sets, double total_ms, double kernel_ms, double d2h_ms,
                 double post_ms) {
  if constexpr (has_walk_iterations<R>::value) {
    using Iter = typename decltype(rec.WalkIterations)::value_type;
    using Gpu = typename decltype(std::declval<Iter &>().GPUWalks)::value_type;
    using ms = std::chrono::duration<double, std::milli>;
    using ns = std::chrono::nanoseconds;
    Iter it;
    it.NumSets = sets;
    it.Total = std::chrono::duration_cast<decltype(it.Total)>(ms(total_ms));
    Gpu g;
    g.NumSets = sets;
    g.Total = std::chrono::duration_cast<decltype(g.Total)>(ms(total_ms));
    g.Kernel = std::chrono::duration_cast<ns>(ms(kernel_ms));
    g.D2H = std::chrono::duration_cast<ns>(ms(d2h_ms));
    g.Post = std::chrono::duration_cast<ns>(ms(post_ms));
    it.GPUWalks.push_back(g);
    rec.WalkIterations.push_back(std::move(it));
  }
}

// One device context per (host thread, device) for FindMostInfluentialSet on
// host-held sets: an edgeless graph of the right vertex count and a pool the
// sets are imported into, kept between calls so a martingale loop driven by
// the reference pays the set-up once.
struct SelectionContext {
  rip_ctx *ctx = nullptr;
  rip_graph *graph = nullptr;
  rip_pool *pool = nullptr;
  int device = -1;
  uint32_t n = 0;
  ~SelectionContext() {
    if (ctx) rip_ctx_destroy(ctx);  // frees the pool and the graph too
  }
  void prepare(int dev, uint32_t nodes) {
    if (ctx && dev != device) {
      rip_ctx_destroy(ctx);
      ctx = nullptr;
    }
    if (!ctx) {
      check(rip_ctx_create(dev, 0, &ctx), nullptr, "rip_ctx_create");
      device = dev;
      graph = nullptr;
      pool = nullptr;
    }
    if (graph && n != nodes) {
      check(rip_graph_destroy(graph), ctx, "rip_graph_destroy");  // its pool goes too
      graph = nullptr;
      pool = nullptr;
    }
    if (!graph) {
      std::vector<uint64_t> index((size_t)nodes + 1, 0);
      check(rip_graph_upload(ctx, index.data(), nullptr, nullptr, nodes, 0, RIP_MODEL_IC,
                             &graph),
            ctx, "rip_graph_upload");
      n = nodes;
    }
    if (!pool) check(rip_pool_create(ctx, graph, &pool), ctx, "rip_pool_create");
    check(rip_pool_clear(pool), ctx, "rip_pool_clear");
  }
};
inline SelectionContext &selection_context() {
  thread_local SelectionContext sc;
  return sc;
}
}  // namespace b200_detail

// Owns a device context, the uploaded backward CSR and a device RRR pool.
// Sets are numbered in generation order; set i depends only on (G, seed, i).
template <typename GraphTy>
class B200RRRGenerator {
 public:
  B200RRRGenerator(const GraphTy &G, int model, uint64_t seed, int device = 0,
                   int sampler = RIP_SAMPLER_AUTO, uint32_t colors = 64)
      : seed_(seed), sampler_(sampler) {
    b200_detail::check(rip_ctx_create(device, 0, &ctx_), nullptr, "rip_ctx_create");
    const uint64_t n = G.num_nodes(), m = G.num_edges();
    const auto *index = reinterpret_cast<const uint64_t *>(&*G.csr_index());
    const auto *src = reinterpret_cast<const uint32_t *>(&*G.csr_edges());
    std::vector<float> w(m);
    const auto weights = G.csr_weights();
    for (uint64_t e = 0; e < m; ++e) w[e] = static_cast<float>(weights[e]);
    b200_detail::check(rip_graph_upload(ctx_, index, src, w.data(), (uint32_t)n, m,
                                        model, &graph_),
                       ctx_, "rip_graph_upload");
    b200_detail::check(rip_pool_create(ctx_, graph_, &pool_), ctx_, "rip_pool_create");
    b200_detail::check(rip_pool_configure(pool_, colors, 0, 0), ctx_, "rip_pool_configure");
  }
  B200RRRGenerator(const B200RRRGenerator &) = delete;
  B200RRRGenerator &operator=(const B200RRRGenerator &) = delete;
  ~B200RRRGenerator() {
    if (ctx_) rip_ctx_destroy(ctx_);  // frees the pool and the graph too
  }

  // Fills [begin, end) -- empty sets the caller inserted -- with new sets, and
  // adds one WalkIterations entry to the record (one GPU walk: sampling
  // kernels, the copy back, filling the caller's sets).
  template <typename ItrTy, typename RecordTy>
  void generate(ItrTy begin, ItrTy end, RecordTy &record) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    const uint64_t count = std::distance(begin, end);
    uint64_t first = 0;
    double k0 = 0, k1 = 0, sel = 0;
    uint64_t launches = 0;
    b200_detail::check(rip_pool_info(pool_, &first, nullptr), ctx_, "rip_pool_info");
    b200_detail::check(rip_pool_timing(pool_, &k0, &launches, &sel), ctx_, "rip_pool_timing");
    b200_detail::check(rip_sample(pool_, seed_, count, sampler_), ctx_, "rip_sample");
    b200_detail::check(rip_sync(ctx_), ctx_, "rip_sync");
    const auto t1 = clk::now();
    std::vector<uint64_t> off(count + 1);
    b200_detail::check(rip_pool_export(pool_, first, count, off.data(), nullptr), ctx_,
                       "rip_pool_export");
    std::vector<uint32_t> vtx(off[count]);
    b200_detail::check(rip_pool_export(pool_, first, count, off.data(), vtx.data()), ctx_,
                       "rip_pool_export");
    const auto t2 = clk::now();
    uint64_t i = 0;
    for (ItrTy it = begin; it != end; ++it, ++i)
      it->assign(vtx.begin() + off[i], vtx.begin() + off[i + 1]);
    const auto t3 = clk::now();
    b200_detail::check(rip_pool_timing(pool_, &k1, &launches, &sel), ctx_, "rip_pool_timing");
    using ms = std::chrono::duration<double, std::milli>;
    b200_detail::record_walk(record, count, ms(t3 - t0).count(), k1 - k0,
                             ms(t2 - t1).count(), ms(t3 - t2).count());
  }

  bool isGpuEnabled() const { return true; }
  rip_ctx *context() const { return ctx_; }
  rip_graph *graph() const { return graph_; }
  rip_pool *pool() const { return pool_; }
  uint64_t seed() const { return seed_; }
  int sampler() const { return sampler_; }

 private:
  rip_ctx *ctx_ = nullptr;
  rip_graph *graph_ = nullptr;
  rip_pool *pool_ = nullptr;
  uint64_t seed_;
  int sampler_;
};

template <typename GraphTy, typename ItrTy, typename ExecRecordTy,
          typename diff_model_tag>
void GenerateRRRSets(const GraphTy &, B200RRRGenerator<GraphTy> &gen, ItrTy begin,
                     ItrTy end, ExecRecordTy &record, diff_model_tag &&, b200_tag &&) {
  gen.generate(begin, end, record);
}

// Seed selection on the GPU over the sets in [rrr_begin, rrr_end), with the
// reference CPU heap's tie-break: the sets are imported into a device pool
// that is kept (with its context) per host thread and device between calls,
// and are not reordered.  The record gets one Counting entry (the device
// selection: counting, heap, picks and count updates) and one Pivoting entry
// of zero (no partitioning), as the sequential reference pushes one of each
// (include/ripples/find_most_influential.h:169-172).  enableGPU and
// CFG.seed_select_max_workers / seed_select_max_gpu_workers are accepted for
// the reference's signature; selection always runs on the device.
template <typename GraphTy, typename ConfTy, typename RRRsetsItr>
std::pair<double, std::vector<typename GraphTy::vertex_type>> FindMostInfluentialSet(
    const GraphTy &G, const ConfTy &CFG, RRRsetsItr rrr_begin, RRRsetsItr rrr_end,
    FindMostInfluentialSetRecord &record, bool, b200_tag &&, int device = 0) {
  using clk = std::chrono::steady_clock;
  b200_detail::SelectionContext &sc = b200_detail::selection_context();
  sc.prepare(device, (uint32_t)G.num_nodes());
  const uint64_t S = std::distance(rrr_begin, rrr_end);
  std::vector<uint64_t> off(S + 1, 0);
  std::vector<uint32_t> vtx;
  uint64_t i = 0;
  for (auto it = rrr_begin; it != rrr_end; ++it, ++i) {
    off[i + 1] = off[i] + it->size();
    vtx.insert(vtx.end(), it->begin(), it->end());
  }
  b200_detail::check(
      rip_pool_import(sc.pool, off.data(), vtx.empty() ? nullptr : vtx.data(), S), sc.ctx,
      "rip_pool_import");
  const uint32_t k = (uint32_t)CFG.k;
  std::vector<uint32_t> seeds(k ? k : 1);
  uint32_t ns = 0;
  double f = 0;
  const auto t0 = clk::now();
  b200_detail::check(
      rip_select(sc.pool, S, k, RIP_TIE_REF_HEAP, seeds.data(), nullptr, &ns, &f), sc.ctx,
      "rip_select");
  using ms = std::chrono::duration<double, std::milli>;
  record.Counting.push_back(
      std::chrono::duration_cast<typename FindMostInfluentialSetRecord::ex_time_ms>(
          ms(clk::now() - t0)));
  record.Pivoting.push_back(typename FindMostInfluentialSetRecord::ex_time_ms(0));
  std::vector<typename GraphTy::vertex_type> result(seeds.begin(), seeds.begin() + ns);
  return {f, result};
}

// IMM on the device (martingale theta estimation, final sampling, final
// selection over sets [0, theta)); fills the record the imm tool logs.
template <typename GraphTy, typename ConfTy, typename diff_model_tag>
std::vector<typename GraphTy::vertex_type> IMM(const GraphTy &G, const ConfTy &CFG,
                                               double l, B200RRRGenerator<GraphTy> &gen,
                                               IMMExecutionRecord &R, diff_model_tag &&,
                                               b200_tag &&) {
  const uint32_t k = (uint32_t)CFG.k;
  std::vector<uint32_t> seeds(k ? k : 1);
  uint32_t ns = 0;
  rip_imm_record rec;
  b200_detail::check(rip_imm_pool(gen.pool(), k, CFG.epsilon, l, gen.seed(),
                                  RIP_TIE_REF_HEAP, gen.sampler(), seeds.data(), &ns, &rec),
                     gen.context(), "rip_imm_pool");
  using ms = std::chrono::duration<double, std::milli>;
  const uint32_t nr = rec.num_rounds < RIP_MAX_ROUNDS ? rec.num_rounds : RIP_MAX_ROUNDS;
  R.ThetaPrimeDeltas.assign(rec.theta_prime_deltas, rec.theta_prime_deltas + nr);
  for (uint32_t i = 0; i < nr; ++i) {
    R.ThetaEstimationGenerateRRR.emplace_back(ms(rec.round_generate_ms[i]));
    R.ThetaEstimationMostInfluential.emplace_back(ms(rec.round_select_ms[i]));
  }
  R.ThetaEstimationTotal =
      std::chrono::duration_cast<decltype(R.ThetaEstimationTotal)>(ms(rec.theta_estimation_ms));
  R.Theta = rec.theta;
  R.GenerateRRRSets =
      std::chrono::duration_cast<decltype(R.GenerateRRRSets)>(ms(rec.generate_ms));
  R.FindMostInfluentialSet =
      std::chrono::duration_cast<decltype(R.FindMostInfluentialSet)>(ms(rec.select_ms));
  R.RRRSetSize = rec.rrr_set_bytes;
  return std::vector<typename GraphTy::vertex_type>(seeds.begin(), seeds.begin() + ns);
}

}  // namespace ripples

#endif  // RIPPLES_B200_IMM_ADAPTER_HPP
