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
// reference loader does (loaders.h:169-191).
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
#include "../csrc/philox.cuh"

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

double unif(uint64_t ctr) {
  rip::u32x4 r = rip::philox((uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 7u << 24, 0u, 0u);
  return (double)(r.x >> 8) * (1.0 / 16777216.0);
}

float gen_weight(const Options &o, uint64_t &ctr) {
  if (o.distribution == "const") return (float)o.mean;
  if (o.distribution == "normal") {
    for (int it = 0; it < 1000; ++it) {
      double u1 = unif(ctr++), u2 = unif(ctr++);
      if (u1 <= 0.0) continue;
      double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
      double x = o.mean + o.variance * z;
      if (x >= 0.0 && x < 1.0) return (float)x;
    }
    return 0.0f;
  }
  if (o.distribution != "uniform") usage("Unsupported distribution");
  return (float)unif(ctr++);
}

struct Edge {
  uint32_t s, d;
  float w;
};

Graph load_tsv(const Options &o) {
  std::ifstream in(o.input);
  if (!in) usage(("cannot open " + o.input).c_str());
  std::vector<Edge> edges;
  uint64_t ctr = 0;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line.find('%') != std::string::npos ||
        line.find('#') != std::string::npos)
      continue;
    std::istringstream ss(line);
    uint64_t s, d;
    float w = 0.0f;
    if (!(ss >> s >> d)) continue;
    if (o.weighted) ss >> w;
    else w = gen_weight(o, ctr);
    edges.push_back({(uint32_t)s, (uint32_t)d, w});
    if (o.undirected) edges.push_back({(uint32_t)d, (uint32_t)s, o.weighted ? w : gen_weight(o, ctr)});
  }
  if (!o.weighted && o.model == "LT") {
    // normalise per source with a random "not taking" mass (loaders.h:169-191)
    std::stable_sort(edges.begin(), edges.end(),
                     [](const Edge &a, const Edge &b) { return a.s < b.s; });
    for (size_t b = 0; b < edges.size();) {
      size_t e = b;
      while (e < edges.size() && edges[e].s == edges[b].s) ++e;
      float total = gen_weight(o, ctr);
      for (size_t i = b; i < e; ++i) total += edges[i].w;
      for (size_t i = b; i < e; ++i) edges[i].w /= total;
      b = e;
    }
  }
  if (o.scale < 1.0)
    for (auto &e : edges) e.w = (float)(e.w * o.scale);
  Graph G;
  std::vector<uint32_t> ids;
  uint32_t maxid = 0;
  for (auto &e : edges) maxid = std::max(maxid, std::max(e.s, e.d));
  if (o.no_renumber) {
    G.n = edges.empty() ? 0 : maxid + 1;
    G.reverse_map.resize(G.n);
    for (uint32_t v = 0; v < G.n; ++v) G.reverse_map[v] = v;
  } else {
    for (auto &e : edges) {
      ids.push_back(e.s);
      ids.push_back(e.d);
    }
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    G.n = (uint32_t)ids.size();
    G.reverse_map = ids;
    auto id = [&](uint32_t x) {
      return (uint32_t)(std::lower_bound(ids.begin(), ids.end(), x) - ids.begin());
    };
    for (auto &e : edges) {
      e.s = id(e.s);
      e.d = id(e.d);
    }
  }
  // backward CSR: in-edges of each destination, by source id
  std::stable_sort(edges.begin(), edges.end(), [](const Edge &a, const Edge &b) {
    return a.d != b.d ? a.d < b.d : a.s < b.s;
  });
  G.index.assign((size_t)G.n + 1, 0);
  for (auto &e : edges) G.index[e.d + 1]++;
  for (uint32_t v = 0; v < G.n; ++v) G.index[v + 1] += G.index[v];
  G.src.resize(edges.size());
  G.w.resize(edges.size());
  for (size_t i = 0; i < edges.size(); ++i) {
    G.src[i] = edges[i].s;
    G.w[i] = edges[i].w;
  }
  return G;
}

Graph load_binary(const Options &o) {
  std::ifstream in(o.input, std::ios::binary);
  if (!in) usage(("cannot open " + o.input).c_str());
  uint64_t hdr[5];
  in.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
  if (!in || hdr[0] != 0xc0ffeeull) usage("The endianess check failed when reloading the input binary.");
  if (hdr[1] != 0xa1ccac0full)
    usage("You are loading a binary that is not compatible with the algorithm you are trying to run.");
  if (hdr[2] != 32ull) usage("The weight type in the binary file is not float.");
  Graph G;
  G.n = (uint32_t)hdr[3];
  const uint64_t m = hdr[4];
  G.reverse_map.resize(G.n);
  G.index.resize((size_t)G.n + 1);
  G.src.resize(m);
  G.w.resize(m);
  in.read(reinterpret_cast<char *>(G.reverse_map.data()), 4ull * G.n);
  in.read(reinterpret_cast<char *>(G.index.data()), 8ull * (G.n + 1));
  in.read(reinterpret_cast<char *>(G.src.data()), 4ull * m);
  in.read(reinterpret_cast<char *>(G.w.data()), 4ull * m);
  if (!in) usage("truncated binary graph");
  if (o.scale < 1.0)
    for (auto &x : G.w) x = (float)(x * o.scale);
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
  Graph G = o.reload ? load_binary(o) : load_tsv(o);
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
