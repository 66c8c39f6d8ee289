// ingest.cpp -- graph input files, read on the host into the backward CSR
// that rip_graph_upload takes.
//
//   rip_read_tsv     a TSV edge list as include/ripples/loaders.h:138-296
//                    reads it ("src dst" or, weighted, "src dst weight";
//                    lines holding '%' or '#' skipped; undirected adds the
//                    reverse of every edge, with the same weight when the
//                    input is weighted), then the GraphBwd the reference's
//                    Graph constructor builds from it (include/ripples/
//                    graph.h:520-620): ids renumbered to 0..n-1 in sorted
//                    order unless renumbering is off (then n = max id + 1),
//                    in-edges of each vertex ordered by source id.
//                    Generated weights (unweighted input) come from a Philox
//                    stream (seed 0) instead of trng: U(0,1), truncated
//                    normal(mean, variance) on [0,1), or a constant; for LT
//                    they are normalised per source with an extra random
//                    "not taking" mass, as loaders.h:169-191 does.
//   rip_read_binary  the reference binary format (include/ripples/
//                    graph.h:854-995, backward direction): header, id map,
//                    offsets, sources, float weights; rip_read_binary_forward
//                    the forward direction (the simulator's input).
//   rip_transpose_csr  backward <-> forward CSR on the host (graph.h:787-832).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "philox.cuh"
#include "ripples_b200.h"

namespace {

thread_local std::string g_read_error;

int read_fail(const std::string &msg) {
  g_read_error = msg;
  return RIP_ERR_INVALID;
}

// Uniform [0, 1) draw number ctr of the weight stream (24-bit resolution).
double unif(uint64_t ctr) {
  rip::u32x4 r = rip::philox((uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 7u << 24, 0u, 0u);
  return (double)(r.x >> 8) * (1.0 / 16777216.0);
}

float gen_weight(const rip_tsv_options &o, uint64_t &ctr) {
  if (o.distribution == RIP_DIST_CONST) return (float)o.mean;
  if (o.distribution == RIP_DIST_NORMAL) {
    for (int it = 0; it < 1000; ++it) {  // Box-Muller, rejected outside [0, 1)
      double u1 = unif(ctr++), u2 = unif(ctr++);
      if (u1 <= 0.0) continue;
      double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
      double x = o.mean + o.variance * z;
      if (x >= 0.0 && x < 1.0) return (float)x;
    }
    return 0.0f;
  }
  return (float)unif(ctr++);
}

struct Edge {
  uint32_t s, d;
  float w;
};

template <typename T>
T *copy_out(const std::vector<T> &v) {
  T *p = static_cast<T *>(std::malloc(std::max<size_t>(v.size(), 1) * sizeof(T)));
  if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

int hand_out(uint32_t n, const std::vector<uint64_t> &index, const std::vector<uint32_t> &src,
             const std::vector<float> &w, const std::vector<uint32_t> &reverse_map,
             uint32_t *n_out, uint64_t *m_out, uint64_t **index_out, uint32_t **src_out,
             float **w_out, uint32_t **map_out) {
  uint64_t *pi = copy_out(index);
  uint32_t *ps = copy_out(src);
  float *pw = copy_out(w);
  uint32_t *pm = copy_out(reverse_map);
  if (!pi || !ps || !pw || !pm) {
    std::free(pi);
    std::free(ps);
    std::free(pw);
    std::free(pm);
    g_read_error = "out of host memory";
    return RIP_ERR_NOMEM;
  }
  *n_out = n;
  *m_out = src.size();
  *index_out = pi;
  *src_out = ps;
  *w_out = pw;
  *map_out = pm;
  return RIP_OK;
}

}  // namespace

extern "C" const char *rip_read_error(void) { return g_read_error.c_str(); }

namespace {

// The edge list of a TSV file as include/ripples/loaders.h:138-196 reads it:
// parsing, generated weights, undirected doubling, the LT normalisation per
// source and the scale factor -- everything before the Graph constructor.
int parse_tsv(const char *path, const rip_tsv_options *o, std::vector<Edge> &edges) {
  if (o->scale > 1.0) return read_fail("The scale factor must be <= 1.0");
  std::ifstream in(path);
  if (!in) return read_fail(std::string("cannot open ") + path);
  const bool known_dist = o->distribution == RIP_DIST_UNIFORM ||
                          o->distribution == RIP_DIST_NORMAL ||
                          o->distribution == RIP_DIST_CONST;
  uint64_t ctr = 0, lineno = 0;
  std::string line;
  while (std::getline(in, line)) {
    ++lineno;
    if (line.empty() || line.find('%') != std::string::npos ||
        line.find('#') != std::string::npos)
      continue;
    std::istringstream ss(line);
    uint64_t s, d;
    float w = 0.0f;
    if (!(ss >> s >> d)) continue;
    if (s >= 0xFFFFFFFFull || d >= 0xFFFFFFFFull)  // ids are u32 with ~0 reserved
      return read_fail("vertex id above 2^32 - 2 on line " + std::to_string(lineno));
    if (o->weighted) {
      ss >> w;
    } else {
      if (!known_dist) return read_fail("Unsupported distribution");
      w = gen_weight(*o, ctr);
    }
    edges.push_back({(uint32_t)s, (uint32_t)d, w});
    if (o->undirected)
      edges.push_back({(uint32_t)d, (uint32_t)s, o->weighted ? w : gen_weight(*o, ctr)});
  }
  if (!o->weighted && o->model == RIP_MODEL_LT) {
    // normalise per source with a random "not taking" mass (loaders.h:169-191)
    std::stable_sort(edges.begin(), edges.end(),
                     [](const Edge &a, const Edge &b) { return a.s < b.s; });
    for (size_t b = 0; b < edges.size();) {
      size_t e = b;
      while (e < edges.size() && edges[e].s == edges[b].s) ++e;
      float total = gen_weight(*o, ctr);
      for (size_t i = b; i < e; ++i) total += edges[i].w;
      for (size_t i = b; i < e; ++i) edges[i].w /= total;
      b = e;
    }
  }
  if (o->scale < 1.0)
    for (auto &e : edges) e.w = (float)(e.w * o->scale);
  return RIP_OK;
}

}  // namespace

extern "C" int rip_read_tsv_edges(const char *path, const rip_tsv_options *o, uint64_t *m_out,
                                  uint32_t **src_out, uint32_t **dst_out, float **w_out) {
  if (!path || !o || !m_out || !src_out || !dst_out || !w_out)
    return read_fail("rip_read_tsv_edges: null argument");
  std::vector<Edge> edges;
  const int rc = parse_tsv(path, o, edges);
  if (rc != RIP_OK) return rc;
  std::vector<uint32_t> s(edges.size()), d(edges.size());
  std::vector<float> w(edges.size());
  for (size_t i = 0; i < edges.size(); ++i) {
    s[i] = edges[i].s;
    d[i] = edges[i].d;
    w[i] = edges[i].w;
  }
  uint32_t *ps = copy_out(s), *pd = copy_out(d);
  float *pw = copy_out(w);
  if (!ps || !pd || !pw) {
    std::free(ps);
    std::free(pd);
    std::free(pw);
    g_read_error = "out of host memory";
    return RIP_ERR_NOMEM;
  }
  *m_out = edges.size();
  *src_out = ps;
  *dst_out = pd;
  *w_out = pw;
  return RIP_OK;
}

extern "C" int rip_read_tsv(const char *path, const rip_tsv_options *o, uint32_t *n_out,
                            uint64_t *m_out, uint64_t **index_out, uint32_t **src_out,
                            float **w_out, uint32_t **map_out) {
  if (!path || !o || !n_out || !m_out || !index_out || !src_out || !w_out || !map_out)
    return read_fail("rip_read_tsv: null argument");
  std::vector<Edge> edges;
  {
    const int rc = parse_tsv(path, o, edges);
    if (rc != RIP_OK) return rc;
  }
  uint32_t n = 0;
  std::vector<uint32_t> reverse_map;
  uint32_t maxid = 0;
  for (auto &e : edges) maxid = std::max(maxid, std::max(e.s, e.d));
  if (!o->renumber) {
    n = edges.empty() ? 0 : maxid + 1;
    reverse_map.resize(n);
    for (uint32_t v = 0; v < n; ++v) reverse_map[v] = v;
  } else {
    std::vector<uint32_t> ids;
    ids.reserve(2 * edges.size());
    for (auto &e : edges) {
      ids.push_back(e.s);
      ids.push_back(e.d);
    }
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    n = (uint32_t)ids.size();
    auto id = [&](uint32_t x) {
      return (uint32_t)(std::lower_bound(ids.begin(), ids.end(), x) - ids.begin());
    };
    for (auto &e : edges) {
      e.s = id(e.s);
      e.d = id(e.d);
    }
    reverse_map = std::move(ids);
  }
  // backward CSR: in-edges of each destination, by source id
  std::stable_sort(edges.begin(), edges.end(), [](const Edge &a, const Edge &b) {
    return a.d != b.d ? a.d < b.d : a.s < b.s;
  });
  std::vector<uint64_t> index((size_t)n + 1, 0);
  for (auto &e : edges) index[e.d + 1]++;
  for (uint32_t v = 0; v < n; ++v) index[v + 1] += index[v];
  std::vector<uint32_t> src(edges.size());
  std::vector<float> w(edges.size());
  for (size_t i = 0; i < edges.size(); ++i) {
    src[i] = edges[i].s;
    w[i] = edges[i].w;
  }
  return hand_out(n, index, src, w, reverse_map, n_out, m_out, index_out, src_out, w_out,
                  map_out);
}

namespace {

// The reference binary format in one direction: magic 0xa1ccac0f for the
// backward CSR (in-edges), 0xf0cacc1a for the forward one (out-edges).
int read_binary(const char *path, uint64_t magic, double scale, uint32_t *n_out,
                uint64_t *m_out, uint64_t **index_out, uint32_t **src_out, float **w_out,
                uint32_t **map_out) {
  if (!path || !n_out || !m_out || !index_out || !src_out || !w_out || !map_out)
    return read_fail("rip_read_binary: null argument");
  std::ifstream in(path, std::ios::binary);
  if (!in) return read_fail(std::string("cannot open ") + path);
  uint64_t hdr[5];
  in.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
  if (!in || hdr[0] != 0xc0ffeeull)
    return read_fail("The endianess check failed when reloading the input binary.");
  if (hdr[1] != magic)
    return read_fail(
        "You are loading a binary that is not compatible with the algorithm you are trying to "
        "run.");
  if (hdr[2] != 32ull) return read_fail("The weight type in the binary file is not float.");
  if (hdr[3] >= 0xFFFFFFFFull || hdr[4] >= (1ull << 32))
    return read_fail("graph too large: n < 2^32 - 1 and m < 2^32 required");
  const uint32_t n = (uint32_t)hdr[3];
  const uint64_t m = hdr[4];
  std::vector<uint32_t> reverse_map(n);
  std::vector<uint64_t> index((size_t)n + 1);
  std::vector<uint32_t> src(m);
  std::vector<float> w(m);
  in.read(reinterpret_cast<char *>(reverse_map.data()), 4ull * n);
  in.read(reinterpret_cast<char *>(index.data()), 8ull * (n + 1));
  in.read(reinterpret_cast<char *>(src.data()), 4ull * m);
  in.read(reinterpret_cast<char *>(w.data()), 4ull * m);
  if (!in) return read_fail("truncated binary graph");
  if (scale < 1.0)
    for (auto &x : w) x = (float)(x * scale);
  return hand_out(n, index, src, w, reverse_map, n_out, m_out, index_out, src_out, w_out,
                  map_out);
}

}  // namespace

extern "C" int rip_read_binary(const char *path, double scale, uint32_t *n_out,
                               uint64_t *m_out, uint64_t **index_out, uint32_t **src_out,
                               float **w_out, uint32_t **map_out) {
  return read_binary(path, 0xa1ccac0full, scale, n_out, m_out, index_out, src_out, w_out,
                     map_out);
}

extern "C" int rip_read_binary_forward(const char *path, double scale, uint32_t *n_out,
                                       uint64_t *m_out, uint64_t **index_out,
                                       uint32_t **dst_out, float **w_out, uint32_t **map_out) {
  return read_binary(path, 0xf0cacc1aull, scale, n_out, m_out, index_out, dst_out, w_out,
                     map_out);
}

// The CSR of the transposed graph: out-lists become in-lists and back, each
// list ordered by the other endpoint's id (stable: parallel edges keep their
// order), weights carried along.
extern "C" int rip_transpose_csr(uint32_t n, uint64_t m, const uint64_t *index,
                                 const uint32_t *adj, const float *w, uint64_t **index_out,
                                 uint32_t **adj_out, float **w_out) {
  if ((n && !index) || (m && (!adj || !w)) || !index_out || !adj_out || !w_out)
    return read_fail("rip_transpose_csr: null argument");
  std::vector<uint64_t> t_index((size_t)n + 1, 0);
  for (uint64_t e = 0; e < m; ++e) {
    if (adj[e] >= n) return read_fail("rip_transpose_csr: vertex out of range");
    t_index[adj[e] + 1]++;
  }
  for (uint32_t v = 0; v < n; ++v) t_index[v + 1] += t_index[v];
  std::vector<uint64_t> cursor(t_index.begin(), t_index.begin() + n);
  std::vector<uint32_t> t_adj(m);
  std::vector<float> t_w(m);
  for (uint32_t v = 0; v < n; ++v)  // v ascending: each new list is ordered by v
    for (uint64_t e = index[v]; e < index[v + 1]; ++e) {
      const uint64_t at = cursor[adj[e]]++;
      t_adj[at] = v;
      t_w[at] = w[e];
    }
  uint64_t *pi = copy_out(t_index);
  uint32_t *pa = copy_out(t_adj);
  float *pw = copy_out(t_w);
  if (!pi || !pa || !pw) {
    std::free(pi);
    std::free(pa);
    std::free(pw);
    g_read_error = "out of host memory";
    return RIP_ERR_NOMEM;
  }
  *index_out = pi;
  *adj_out = pa;
  *w_out = pw;
  return RIP_OK;
}
