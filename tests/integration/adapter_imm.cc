// adapter_imm.cc -- integration check of include/ripples_b200/imm_adapter.hpp
// against the unmodified ripples headers (built by oracle/ref.mk into
// oracle/_ref/adapter_imm; run by tests/test_gpu_adapter.py).
//
// Loads a reference-format binary graph with ripples::GraphBwd::load_binary,
// then, through the adapter only:
//   1. ripples::IMM(G, CFG, 1, gen, R, <model>_tag{}, b200_tag{})
//   2. ripples::GenerateRRRSets(G, gen2, begin, end, R2, <model>_tag{}, b200_tag{})
//      on caller-inserted empty sets, then
//      ripples::FindMostInfluentialSet(G, CFG, begin, end, R2, true, b200_tag{})
//      on all of them and again on the first half
// and prints one JSON object with the results and the record's entries.
//   usage: adapter_imm <graph.bin> <IC|LT> <k> <epsilon> <seed> <nsets>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "ripples/configuration.h"
#include "ripples/graph.h"
#include "ripples/imm_configuration.h"
#include "ripples/imm_execution_record.h"
#include "ripples/imm_interface.h"
#include "ripples/utility.h"
#include "ripples/diffusion_simulation.h"
#include "ripples/find_most_influential_record.h"

#include "ripples_b200/imm_adapter.hpp"

template <typename Tag>
int run(const ripples::GraphBwd &G, int model, size_t k, double eps, uint64_t seed,
        size_t nsets) {
  ripples::IMMConfiguration CFG;
  CFG.k = k;
  CFG.epsilon = eps;
  ripples::B200RRRGenerator<ripples::GraphBwd> gen(G, model, seed);
  ripples::IMMExecutionRecord R;
  auto seeds = ripples::IMM(G, CFG, 1.0, gen, R, Tag{}, ripples::b200_tag{});

  ripples::B200RRRGenerator<ripples::GraphBwd> gen2(G, model, seed);
  ripples::RRRsets<ripples::GraphBwd> RR(nsets);
  ripples::IMMExecutionRecord R2;
  ripples::GenerateRRRSets(G, gen2, RR.begin(), RR.end(), R2, Tag{}, ripples::b200_tag{});
  auto S = ripples::FindMostInfluentialSet(G, CFG, RR.begin(), RR.end(), R2, true,
                                           ripples::b200_tag{});
  // a second selection in the same process, on the first half of the sets:
  // the adapter's cached device context is reused
  auto S2 = ripples::FindMostInfluentialSet(G, CFG, RR.begin(), RR.begin() + nsets / 2, R2,
                                            true, ripples::b200_tag{});
  uint64_t elems = 0;
  bool sorted = true;
  for (auto &s : RR) {
    elems += s.size();
    for (size_t i = 1; i < s.size(); ++i) sorted &= s[i - 1] < s[i];
  }
  std::printf("{\"imm_seeds\": [");
  for (size_t i = 0; i < seeds.size(); ++i) std::printf("%s%u", i ? ", " : "", seeds[i]);
  std::printf("], \"theta\": %zu, \"deltas\": [", R.Theta);
  for (size_t i = 0; i < R.ThetaPrimeDeltas.size(); ++i)
    std::printf("%s%zu", i ? ", " : "", R.ThetaPrimeDeltas[i]);
  std::printf("], \"sets\": %zu, \"elements\": %llu, \"sorted\": %s, \"f\": %.17g, "
              "\"select_seeds\": [",
              RR.size(), (unsigned long long)elems, sorted ? "true" : "false", S.first);
  for (size_t i = 0; i < S.second.size(); ++i)
    std::printf("%s%u", i ? ", " : "", S.second[i]);
  std::printf("], \"half_f\": %.17g, \"half_seeds\": [", S2.first);
  for (size_t i = 0; i < S2.second.size(); ++i)
    std::printf("%s%u", i ? ", " : "", S2.second[i]);
  std::printf("], \"counting\": %zu, \"pivoting\": %zu, \"walk_iterations\": %zu, "
              "\"walk_sets\": %zu, \"gpu_walks\": %zu}\n",
              R2.Counting.size(), R2.Pivoting.size(), R2.WalkIterations.size(),
              R2.WalkIterations.empty() ? (size_t)0 : R2.WalkIterations[0].NumSets,
              R2.WalkIterations.empty() ? (size_t)0 : R2.WalkIterations[0].GPUWalks.size());
  return 0;
}

int main(int argc, char **argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s graph.bin IC|LT k epsilon seed nsets\n", argv[0]);
    return 2;
  }
  ripples::GraphBwd G;
  G.load_binary(argv[1]);
  const std::string model = argv[2];
  const size_t k = std::strtoull(argv[3], nullptr, 10);
  const double eps = std::strtod(argv[4], nullptr);
  const uint64_t seed = std::strtoull(argv[5], nullptr, 10);
  const size_t nsets = std::strtoull(argv[6], nullptr, 10);
  try {
    if (model == "IC")
      return run<ripples::independent_cascade_tag>(G, RIP_MODEL_IC, k, eps, seed, nsets);
    return run<ripples::linear_threshold_tag>(G, RIP_MODEL_LT, k, eps, seed, nsets);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "adapter_imm: %s\n", e.what());
    return 1;
  }
}
