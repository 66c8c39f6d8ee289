// imm_b200 -- the ripples `imm` tool on one B200.
//
// Same command line and JSON log as tools/imm.cc of pnnl/ripples
// (options: include/ripples/configuration.h:72-149, tim_configuration.h:59-61,
// imm_configuration.h:80-108; log keys: tools/imm.cc:104-134), computing
// through the C ABI of libripples_b200.
//
//   imm_b200 -i graph -k K -e EPS -d IC|LT [-w] [-u] [--reload-binary]
//            [--disable-renumbering] [--distribution uniform|normal|const]
//            [--mean M] [--variance V] [--scale-factor S] [-p] [--rrsets N]
//            [--gpu-batch-size 64|128|256] [--seed S] [--tiebreak heap|lowest]
//            [--sampler auto|plain|fused] [-o log.json]
//
// Input as in include/ripples/loaders.h: a TSV edge list ("src dst" or, with
// -w, "src dst weight"; lines holding '%' or '#' skipped; -u adds the
// reverse of every edge), or with --reload-binary the reference binary format
// (include/ripples/graph.h:854-995, backward direction).  Vertex ids are
// renumbered to 0..n-1 in sorted order unless --disable-renumbering; the log
// reports seeds in the input's ids (Graph::convertID).  Generated weights
// (no -w) are drawn from the library's Philox stream (seed 0): U(0,1),
// truncated normal(mean, variance) on [0,1), or a constant; for LT they are
// normalised per source with an extra random "not taking" mass, as the
// reference loader does (loaders.h:169-191).  Reading is the library's
// (rip_read_tsv / rip_read_binary).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "ripples_b200.h"

namespace {

struct Options {
  std::string input, output = "output.json", model = "IC", distribution = "uniform";
  std::string tiebreak = "heap", sampler = "auto";
  bool weighted = false, undirected = false, reload = false, no_renumber = false,
       parallel = false;
  double epsilon = 0.5, mean = 0.5, variance = 1.0, scale = 1.0;
  uint64_t k = 10, rrsets = 0, seed = 0, colors = 64;
  bool have_k = false, have_eps = false, have_d = false, have_i = false;
};

[[noreturn]] void usage(const char *msg) {
  std::fprintf(stderr, "imm_b200: %s\n", msg);
  std::exit(106);
}

Options parse(int argc, char **argv) {
  Options o;
  auto value = [&](int &i, const std::string &name) -> std::string {
    std::string a = argv[i];
    auto eq = a.find('=');
    if (a.rfind("--", 0) == 0 && eq != std::string::npos) return a.substr(eq + 1);
    if (i + 1 >= argc) usage(("missing value for " + name).c_str());
    return argv[++i];
  };
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i], key = a.substr(0, a.find('='));
    if (key == "-h" || key == "--help") {
      std::printf("usage: imm_b200 -i graph -k K -e EPS -d IC|LT [options]\n");
      std::exit(0);
    } else if (key == "-i" || key == "--input-graph") { o.input = value(i, key); o.have_i = true; }
    else if (key == "-o" || key == "--output") o.output = value(i, key);
    else if (key == "-k" || key == "--seed-set-size") { o.k = std::stoull(value(i, key)); o.have_k = true; }
    else if (key == "-e" || key == "--epsilon") { o.epsilon = std::stod(value(i, key)); o.have_eps = true; }
    else if (key == "-d" || key == "--diffusion-model") { o.model = value(i, key); o.have_d = true; }
    else if (key == "-w" || key == "--weighted") o.weighted = true;
    else if (key == "-u" || key == "--undirected") o.undirected = true;
    else if (key == "-p" || key == "--parallel") o.parallel = true;
    else if (key == "--reload-binary") o.reload = true;
    else if (key == "--disable-renumbering") o.no_renumber = true;
    else if (key == "--distribution") o.distribution = value(i, key);
    else if (key == "--mean") o.mean = std::stod(value(i, key));
    else if (key == "--variance") o.variance = std::stod(value(i, key));
    else if (key == "--scale-factor") o.scale = std::stod(value(i, key));
    else if (key == "--rrsets") o.rrsets = std::stoull(value(i, key));
    else if (key == "--gpu-batch-size") o.colors = std::stoull(value(i, key));
    else if (key == "--seed") o.seed = std::stoull(value(i, key));
    else if (key == "--tiebreak") o.tiebreak = value(i, key);
    else if (key == "--sampler") o.sampler = value(i, key);
    else if (key == "--streaming-cpu-teams" || key == "--streaming-gpu-workers" ||
             key == "--cpu-batch-size" || key == "--pause-threshold" ||
             key == "--streaming-gpu-mapping" || key == "--seed-select-max-workers" ||
             key == "--seed-select-max-gpu-workers" || key == "--metall-store-dir" ||
             key == "--rr-store-dir")
      value(i, key);  // accepted for compatibility; one B200 does all the work
    else usage(("unknown argument: " + a).c_str());
  }
  if (!o.have_i || !o.have_k || !o.have_eps || !o.have_d)
    usage("-i, -k, -e and -d are required");
  if (o.model != "IC" && o.model != "LT") usage("-d must be IC or LT");
  if (o.scale > 1.0) usage("The scale factor must be <= 1.0");
  if (o.colors != 64 && o.colors != 128 && o.colors != 256)
    o.colors = o.colors <= 64 ? 64 : o.colors <= 128 ? 128 : 256;
  return o;
}

struct Graph {  // backward CSR + id map
  uint32_t n = 0;
  std::vector<uint64_t> index;
  std::vector<uint32_t> src;
  std::vector<float> w;
  std::vector<uint32_t> reverse_map;  // internal id -> input id
};

// The graph through the library's readers (rip_read_tsv / rip_read_binary):
// the reference loader's parsing, generated weights and renumbering.
Graph load_graph(const Options &o) {
  uint32_t n = 0;
  uint64_t m = 0, *index = nullptr;
  uint32_t *src = nullptr, *reverse_map = nullptr;
  float *w = nullptr;
  int rc;
  if (o.reload) {
    rc = rip_read_binary(o.input.c_str(), o.scale, &n, &m, &index, &src, &w, &reverse_map);
  } else {
    rip_tsv_options t;
    t.weighted = o.weighted;
    t.undirected = o.undirected;
    t.renumber = !o.no_renumber;
    t.model = o.model == "LT" ? RIP_MODEL_LT : RIP_MODEL_IC;
    t.distribution = o.distribution == "uniform"  ? RIP_DIST_UNIFORM
                     : o.distribution == "normal" ? RIP_DIST_NORMAL
                     : o.distribution == "const"  ? RIP_DIST_CONST
                                                  : -1;
    t.mean = o.mean;
    t.variance = o.variance;
    t.scale = o.scale;
    rc = rip_read_tsv(o.input.c_str(), &t, &n, &m, &index, &src, &w, &reverse_map);
  }
  if (rc != RIP_OK) usage(rip_read_error());
  Graph G;
  G.n = n;
  G.index.assign(index, index + (size_t)n + 1);
  G.src.assign(src, src + m);
  G.w.assign(w, w + m);
  G.reverse_map.assign(reverse_map, reverse_map + n);
  rip_free(index);
  rip_free(src);
  rip_free(w);
  rip_free(reverse_map);
  return G;
}

void check(int rc, rip_ctx *ctx, const char *what) {
  if (rc != RIP_OK) {
    std::fprintf(stderr, "imm_b200: %s failed (%d): %s\n", what, rc,
                 ctx ? rip_last_error(ctx) : "");
    std::exit(1);
  }
}

std::string json_list(const std::vector<double> &v) {
  std::string s = "[";
  for (size_t i = 0; i < v.size(); ++i) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%s%.17g", i ? ", " : "", v[i]);
    s += buf;
  }
  return s + "]";
}

}  // namespace

int main(int argc, char **argv) {
  const Options o = parse(argc, argv);
  using clk = std::chrono::high_resolution_clock;
  auto t0 = clk::now();
  Graph G = load_graph(o);
  const double load_ms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
  std::fprintf(stderr, "[imm_b200] Loading took %.0fms: %u nodes, %zu edges\n", load_ms, G.n,
               G.src.size());

  rip_ctx *ctx = nullptr;
  check(rip_ctx_create(0, 0, &ctx), nullptr, "rip_ctx_create");
  rip_graph *g = nullptr;
  check(rip_graph_upload(ctx, G.index.data(), G.src.data(), G.w.data(), G.n, G.src.size(),
                         o.model == "IC" ? RIP_MODEL_IC : RIP_MODEL_LT, &g),
        ctx, "rip_graph_upload");
  rip_pool *pool = nullptr;
  check(rip_pool_create(ctx, g, &pool), ctx, "rip_pool_create");
  check(rip_pool_configure(pool, (uint32_t)o.colors, 0, 0), ctx, "rip_pool_configure");
  const int sampler = o.sampler == "plain" ? RIP_SAMPLER_PLAIN
                      : o.sampler == "fused" ? RIP_SAMPLER_FUSED : RIP_SAMPLER_AUTO;
  const int tie = o.tiebreak == "lowest" ? RIP_TIE_LOWEST_ID : RIP_TIE_REF_HEAP;

  std::vector<uint32_t> seeds;
  rip_imm_record rec;
  std::memset(&rec, 0, sizeof(rec));
  auto t1 = clk::now();
  if (o.rrsets) {  // tools/imm.cc:247-281: just generate that many sets
    check(rip_sample(pool, o.seed, o.rrsets, sampler), ctx, "rip_sample");
    check(rip_sync(ctx), ctx, "rip_sync");
    rec.theta = o.rrsets;
    rec.num_rounds = 1;
    rec.theta_prime_deltas[0] = o.rrsets;
    rec.round_generate_ms[0] = std::chrono::duration<double, std::milli>(clk::now() - t1).count();
    seeds.assign(o.k, 1);
  } else {
    seeds.resize(o.k ? o.k : 1);
    uint32_t ns = 0;
    check(rip_imm_pool(pool, (uint32_t)o.k, o.epsilon, 1.0, o.seed, tie, sampler, seeds.data(),
                       &ns, &rec),
          ctx, "rip_imm_pool");
    seeds.resize(ns);
  }
  const double total = std::chrono::duration<double, std::milli>(clk::now() - t1).count();
  uint64_t ns = 0, ne = 0;
  rip_pool_info(pool, &ns, &ne);
  std::fprintf(stderr, "[imm_b200] IMM : %.3fms (theta %llu, %llu sets)\n", total,
               (unsigned long long)rec.theta, (unsigned long long)ns);

  std::vector<double> deltas, gen, sel;
  for (uint32_t i = 0; i < rec.num_rounds && i < RIP_MAX_ROUNDS; ++i) {
    deltas.push_back((double)rec.theta_prime_deltas[i]);
    gen.push_back(rec.round_generate_ms[i]);
    sel.push_back(rec.round_select_ms[i]);
  }
  std::string seeds_json = "[";
  for (size_t i = 0; i < seeds.size(); ++i) {
    const uint32_t s = seeds[i] < G.reverse_map.size() ? G.reverse_map[seeds[i]] : seeds[i];
    seeds_json += (i ? ", " : "") + std::to_string(s);
  }
  seeds_json += "]";
  std::string deltas_json = "[";
  for (size_t i = 0; i < deltas.size(); ++i)
    deltas_json += (i ? ", " : "") + std::to_string((unsigned long long)deltas[i]);
  deltas_json += "]";
  FILE *f = std::fopen(o.output.c_str(), "w");
  if (!f) usage(("cannot write " + o.output).c_str());
  std::fprintf(f,
               "[\n  {\n    \"Algorithm\": \"IMM\",\n    \"Input\": \"%s\",\n"
               "    \"Output\": \"%s\",\n    \"DiffusionModel\": \"%s\",\n"
               "    \"Epsilon\": %.17g,\n    \"K\": %llu,\n    \"L\": 1,\n"
               "    \"NumThreads\": 1,\n    \"NumWalkWorkers\": 1,\n"
               "    \"NumCPUTeams\": 0,\n    \"NumGPUWalkWorkers\": 1,\n"
               "    \"PauseThreshold\": 1.0,\n    \"Total\": %.17g,\n"
               "    \"ThetaPrimeDeltas\": %s,\n    \"ThetaEstimation\": %.17g,\n"
               "    \"ThetaEstimationGenerateRRR\": %s,\n"
               "    \"ThetaEstimationMostInfluential\": %s,\n    \"Theta\": %llu,\n"
               "    \"Counting\": [],\n    \"Pivoting\": [],\n    \"Microbenchmarking\": 0,\n"
               "    \"CPUBatchSize\": 0,\n    \"GPUBatchSize\": %llu,\n"
               "    \"RRRSetSizeBytes\": %llu,\n    \"GenerateRRRSets\": %.17g,\n"
               "    \"FindMostInfluentialSet\": %.17g,\n    \"Seeds\": %s\n  }\n]",
               o.input.c_str(), o.output.c_str(), o.model.c_str(), o.epsilon,
               (unsigned long long)o.k, total, deltas_json.c_str(), rec.theta_estimation_ms,
               json_list(gen).c_str(), json_list(sel).c_str(), (unsigned long long)rec.theta,
               (unsigned long long)o.colors, (unsigned long long)(ne * 4), rec.generate_ms,
               rec.select_ms, seeds_json.c_str());
  std::fclose(f);
  rip_ctx_destroy(ctx);
  return 0;
}
