// simulator_b200 -- the ripples `simulator` tool on one B200.
//
// Same command line and JSON output as tools/simulator.cc of pnnl/ripples:
//
//   simulator_b200 -i graph -e experiments.json --replicas R [-w] [-u]
//                  [--reload-binary] [--disable-renumbering]
//                  [--distribution uniform|normal|const] [--mean M]
//                  [--variance V] [--scale-factor S] [--seed S] [-o out.json]
//
// The graph is read as the reference reads it (TSV through rip_read_tsv, or
// with --reload-binary the FORWARD binary format); the diffusion model comes
// from the first experiment record, as in the reference (simulator.cc:117).
// For every record of the experiment file (the imm / opimc tools' JSON log)
// the seeds, given in input ids, are simulated `replicas` times on the device
// (rip_spread_ic / rip_spread_lt), and the record is written back with its
// "Simulations": [[activated, levels], ...] (simulator.cc:83-94, the pairs
// ripples::simulate returns).  Replicas draw from the library's Philox
// streams keyed by --seed, not from trng: the same distributions, not the
// same draws.
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "ripples_b200.h"

namespace {

[[noreturn]] void usage(const std::string &msg) {
  std::fprintf(stderr, "simulator_b200: %s\n", msg.c_str());
  std::exit(106);
}

// ---- a small JSON reader / writer (the experiment logs) --------------------
struct Json {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  std::string text;  // NUM: the literal as written; STR: the decoded string
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;
  const Json *get(const std::string &key) const {
    for (auto &kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

struct Parser {
  const std::string &s;
  size_t i = 0;
  explicit Parser(const std::string &src) : s(src) {}
  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  [[noreturn]] void fail(const char *what) {
    usage(std::string("experiment file: ") + what + " at byte " + std::to_string(i));
  }
  std::string str() {
    if (s[i] != '"') fail("expected a string");
    ++i;
    std::string out;
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\') {
        if (++i >= s.size()) fail("bad escape");
        const char c = s[i];
        if (c == 'n') out += '\n';
        else if (c == 't') out += '\t';
        else if (c == 'r') out += '\r';
        else if (c == 'b') out += '\b';
        else if (c == 'f') out += '\f';
        else if (c == 'u') {  // \uXXXX: ASCII range kept, others replaced
          if (i + 4 >= s.size()) fail("bad \\u escape");
          const unsigned v = (unsigned)std::strtoul(s.substr(i + 1, 4).c_str(), nullptr, 16);
          out += v < 128 ? (char)v : '?';
          i += 4;
        } else out += c;  // " \ /
        ++i;
      } else {
        out += s[i++];
      }
    }
    if (i >= s.size()) fail("unterminated string");
    ++i;
    return out;
  }
  Json value() {
    ws();
    if (i >= s.size()) fail("unexpected end");
    Json v;
    const char c = s[i];
    if (c == '{') {
      v.kind = Json::OBJ;
      ++i;
      ws();
      if (s[i] == '}') {
        ++i;
        return v;
      }
      for (;;) {
        ws();
        std::string key = str();
        ws();
        if (s[i] != ':') fail("expected ':'");
        ++i;
        v.obj.emplace_back(key, value());
        ws();
        if (s[i] == ',') {
          ++i;
          continue;
        }
        if (s[i] == '}') {
          ++i;
          return v;
        }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = Json::ARR;
      ++i;
      ws();
      if (s[i] == ']') {
        ++i;
        return v;
      }
      for (;;) {
        v.arr.push_back(value());
        ws();
        if (s[i] == ',') {
          ++i;
          continue;
        }
        if (s[i] == ']') {
          ++i;
          return v;
        }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind = Json::STR;
      v.text = str();
      return v;
    }
    if (s.compare(i, 4, "true") == 0) {
      v.kind = Json::BOOL;
      v.b = true;
      i += 4;
      return v;
    }
    if (s.compare(i, 5, "false") == 0) {
      v.kind = Json::BOOL;
      i += 5;
      return v;
    }
    if (s.compare(i, 4, "null") == 0) {
      i += 4;
      return v;
    }
    const size_t b = i;
    while (i < s.size() && (std::isdigit((unsigned char)s[i]) || s[i] == '-' || s[i] == '+' ||
                            s[i] == '.' || s[i] == 'e' || s[i] == 'E'))
      ++i;
    if (b == i) fail("unexpected character");
    v.kind = Json::NUM;
    v.text = s.substr(b, i - b);
    return v;
  }
};

void write_json(std::string &out, const Json &v, int indent, int depth) {
  const std::string pad((size_t)indent * (depth + 1), ' '), end((size_t)indent * depth, ' ');
  switch (v.kind) {
    case Json::NUL: out += "null"; break;
    case Json::BOOL: out += v.b ? "true" : "false"; break;
    case Json::NUM: out += v.text; break;
    case Json::STR: {
      out += '"';
      for (char c : v.text) {
        if (c == '"' || c == '\\') out += '\\', out += c;
        else if (c == '\n') out += "\\n";
        else if (c == '\t') out += "\\t";
        else if ((unsigned char)c < 0x20) {
          char buf[8];
          std::snprintf(buf, sizeof(buf), "\\u%04x", (unsigned)c);
          out += buf;
        } else out += c;
      }
      out += '"';
      break;
    }
    case Json::ARR:
      if (v.arr.empty()) {
        out += "[]";
        break;
      }
      out += "[\n";
      for (size_t j = 0; j < v.arr.size(); ++j) {
        out += pad;
        write_json(out, v.arr[j], indent, depth + 1);
        out += j + 1 < v.arr.size() ? ",\n" : "\n";
      }
      out += end + "]";
      break;
    case Json::OBJ:
      if (v.obj.empty()) {
        out += "{}";
        break;
      }
      out += "{\n";
      for (size_t j = 0; j < v.obj.size(); ++j) {
        Json key;
        key.kind = Json::STR;
        key.text = v.obj[j].first;
        out += pad;
        write_json(out, key, indent, depth + 1);
        out += ": ";
        write_json(out, v.obj[j].second, indent, depth + 1);
        out += j + 1 < v.obj.size() ? ",\n" : "\n";
      }
      out += end + "}";
      break;
  }
}

Json num(uint64_t x) {
  Json v;
  v.kind = Json::NUM;
  v.text = std::to_string((unsigned long long)x);
  return v;
}

// ---- options ---------------------------------------------------------------
struct Options {
  std::string input, experiments, output = "output.json", distribution = "uniform";
  bool weighted = false, undirected = false, reload = false, no_renumber = false;
  double mean = 0.5, variance = 1.0, scale = 1.0;
  uint64_t replicas = 0, seed = 0;
  bool have_i = false, have_e = false, have_r = false;
};

Options parse(int argc, char **argv) {
  Options o;
  auto value = [&](int &i, const std::string &name) -> std::string {
    std::string a = argv[i];
    auto eq = a.find('=');
    if (a.rfind("--", 0) == 0 && eq != std::string::npos) return a.substr(eq + 1);
    if (i + 1 >= argc) usage("missing value for " + name);
    return argv[++i];
  };
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i], key = a.substr(0, a.find('='));
    if (key == "-h" || key == "--help") {
      std::printf("usage: simulator_b200 -i graph -e experiments.json --replicas R "
                  "[options]\n");
      std::exit(0);
    } else if (key == "-i" || key == "--input-graph") { o.input = value(i, key); o.have_i = true; }
    else if (key == "-e" || key == "--experiment-file") { o.experiments = value(i, key); o.have_e = true; }
    else if (key == "--replicas") { o.replicas = std::stoull(value(i, key)); o.have_r = true; }
    else if (key == "-o" || key == "--output") o.output = value(i, key);
    else if (key == "-w" || key == "--weighted") o.weighted = true;
    else if (key == "-u" || key == "--undirected") o.undirected = true;
    else if (key == "--reload-binary") o.reload = true;
    else if (key == "--disable-renumbering") o.no_renumber = true;
    else if (key == "--distribution") o.distribution = value(i, key);
    else if (key == "--mean") o.mean = std::stod(value(i, key));
    else if (key == "--variance") o.variance = std::stod(value(i, key));
    else if (key == "--scale-factor") o.scale = std::stod(value(i, key));
    else if (key == "--seed") o.seed = std::stoull(value(i, key));
    else if (key == "-p" || key == "--parallel") continue;  // one B200 does all the work
    else if (key == "--metall-store-dir" || key == "--rr-store-dir")
      value(i, key);  // accepted for compatibility
    else usage("unknown argument: " + a);
  }
  if (!o.have_i || !o.have_e || !o.have_r) usage("-i, -e and --replicas are required");
  if (o.scale > 1.0) usage("The scale factor must be <= 1.0");
  return o;
}

struct Csr {
  uint32_t n = 0;
  uint64_t m = 0;
  uint64_t *index = nullptr;
  uint32_t *adj = nullptr;
  float *w = nullptr;
  ~Csr() {
    rip_free(index);
    rip_free(adj);
    rip_free(w);
  }
};

void check(int rc, rip_ctx *ctx, const char *what) {
  if (rc != RIP_OK) {
    std::fprintf(stderr, "simulator_b200: %s failed (%d): %s\n", what, rc,
                 ctx ? rip_last_error(ctx) : rip_read_error());
    std::exit(1);
  }
}

}  // namespace

int main(int argc, char **argv) {
  const Options o = parse(argc, argv);
  std::ifstream ein(o.experiments);
  if (!ein) usage("cannot open " + o.experiments);
  std::stringstream buf;
  buf << ein.rdbuf();
  const std::string text = buf.str();
  Parser P(text);
  const Json experiments = P.value();
  if (experiments.kind != Json::ARR || experiments.arr.empty())
    usage("the experiment file must hold a non-empty JSON array");
  const Json *dm = experiments.arr[0].get("DiffusionModel");
  if (!dm || dm->kind != Json::STR || (dm->text != "IC" && dm->text != "LT"))
    usage("the first experiment has no DiffusionModel IC or LT");
  const bool lt = dm->text == "LT";

  // backward (in-edges) and forward (out-edges) CSR of the graph, input id map
  Csr bwd, fwd;
  uint32_t *reverse_map = nullptr;
  if (o.reload) {
    check(rip_read_binary_forward(o.input.c_str(), o.scale, &fwd.n, &fwd.m, &fwd.index,
                                  &fwd.adj, &fwd.w, &reverse_map),
          nullptr, "rip_read_binary_forward");
    bwd.n = fwd.n;
    bwd.m = fwd.m;
    check(rip_transpose_csr(fwd.n, fwd.m, fwd.index, fwd.adj, fwd.w, &bwd.index, &bwd.adj,
                            &bwd.w),
          nullptr, "rip_transpose_csr");
  } else {
    rip_tsv_options t;
    t.weighted = o.weighted;
    t.undirected = o.undirected;
    t.renumber = !o.no_renumber;
    t.model = lt ? RIP_MODEL_LT : RIP_MODEL_IC;
    t.distribution = o.distribution == "uniform"  ? RIP_DIST_UNIFORM
                     : o.distribution == "normal" ? RIP_DIST_NORMAL
                     : o.distribution == "const"  ? RIP_DIST_CONST
                                                  : -1;
    t.mean = o.mean;
    t.variance = o.variance;
    t.scale = o.scale;
    check(rip_read_tsv(o.input.c_str(), &t, &bwd.n, &bwd.m, &bwd.index, &bwd.adj, &bwd.w,
                       &reverse_map),
          nullptr, "rip_read_tsv");
    fwd.n = bwd.n;
    fwd.m = bwd.m;
    check(rip_transpose_csr(bwd.n, bwd.m, bwd.index, bwd.adj, bwd.w, &fwd.index, &fwd.adj,
                            &fwd.w),
          nullptr, "rip_transpose_csr");
  }
  std::unordered_map<uint64_t, uint32_t> internal;  // Graph::transformID
  for (uint32_t v = 0; v < bwd.n; ++v) internal[reverse_map[v]] = v;
  rip_free(reverse_map);
  std::fprintf(stderr, "[simulator_b200] Number of Nodes : %u\n[simulator_b200] Number of "
                       "Edges : %llu\n", bwd.n, (unsigned long long)bwd.m);

  // every record's seeds in internal ids, checked before the device is touched
  std::vector<std::vector<uint32_t>> seed_sets;
  for (const Json &record : experiments.arr) {
    const Json *sj = record.get("Seeds");
    if (!sj || sj->kind != Json::ARR) usage("an experiment has no Seeds array");
    std::vector<uint32_t> seeds;
    for (const Json &x : sj->arr) {
      const uint64_t id = std::strtoull(x.text.c_str(), nullptr, 10);
      auto it = internal.find(id);
      if (x.kind != Json::NUM || it == internal.end())
        usage("seed " + x.text + " is not a vertex of the graph");
      seeds.push_back(it->second);
    }
    seed_sets.push_back(std::move(seeds));
  }

  rip_ctx *ctx = nullptr;
  check(rip_ctx_create(0, 0, &ctx), nullptr, "rip_ctx_create");
  rip_graph *gf = nullptr, *gb = nullptr;
  check(rip_graph_upload(ctx, fwd.index, fwd.adj, fwd.w, fwd.n, fwd.m, RIP_MODEL_IC, &gf), ctx,
        "rip_graph_upload");
  if (lt)
    check(rip_graph_upload(ctx, bwd.index, bwd.adj, bwd.w, bwd.n, bwd.m, RIP_MODEL_LT, &gb),
          ctx, "rip_graph_upload");

  Json out;
  out.kind = Json::ARR;
  std::vector<uint32_t> sizes(o.replicas ? o.replicas : 1), levels(sizes.size());
  for (size_t ri = 0; ri < experiments.arr.size(); ++ri) {
    const Json &record = experiments.arr[ri];
    const std::vector<uint32_t> &seeds = seed_sets[ri];
    double spread = 0;
    if (lt)
      check(rip_spread_lt(gf, gb, seeds.data(), (uint32_t)seeds.size(), o.replicas, o.seed,
                          sizes.data(), levels.data(), &spread),
            ctx, "rip_spread_lt");
    else
      check(rip_spread_ic(gf, seeds.data(), (uint32_t)seeds.size(), o.replicas, o.seed,
                          sizes.data(), levels.data(), &spread),
            ctx, "rip_spread_ic");
    Json sims;
    sims.kind = Json::ARR;
    for (uint64_t r = 0; r < o.replicas; ++r) {
      Json pair;
      pair.kind = Json::ARR;
      pair.arr.push_back(num(sizes[r]));
      pair.arr.push_back(num(levels[r]));
      sims.arr.push_back(pair);
    }
    Json rec;  // simulator.cc:83-94
    rec.kind = Json::OBJ;
    for (const char *key : {"Input", "Algorithm"}) {
      const Json *v = record.get(key);
      rec.obj.emplace_back(key, v ? *v : Json());
    }
    rec.obj.emplace_back("DiffusionModel", *dm);
    for (const char *key : {"Epsilon", "K", "Seeds"}) {
      const Json *v = record.get(key);
      rec.obj.emplace_back(key, v ? *v : Json());
    }
    rec.obj.emplace_back("Simulations", sims);
    out.arr.push_back(rec);
    std::fprintf(stderr, "[simulator_b200] %zu seeds, %llu replicas: mean spread %.3f\n",
                 seeds.size(), (unsigned long long)o.replicas, spread);
  }
  std::string text_out;
  write_json(text_out, out, 2, 0);
  FILE *f = std::fopen(o.output.c_str(), "w");
  if (!f) usage("cannot write " + o.output);
  std::fputs(text_out.c_str(), f);
  std::fputc('\n', f);
  std::fclose(f);
  rip_ctx_destroy(ctx);
  return 0;
}
