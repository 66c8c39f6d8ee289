// graph.cu -- device graphs behind include/ripples_b200.h: upload and packing of a
// backward CSR, export, thresholds, R-MAT / Erdos-Renyi graphs built on the device.
#include "host.h"

// ---------------------------------------------------------------------------
// graph
// ---------------------------------------------------------------------------

// IC graphs: the per-vertex uniform thresholds, kept when uniform in-lists of
// two or more edges hold at least half of the edges (weighted cascade: all of
// them); the IC samplers then skip the threshold reads of those lists.  The
// same pass measures the branching factor of a reverse BFS, which picks the
// heavy-set default of untuned graphs.
static int setup_vthr(rip_ctx *c, rip_graph *g) {
  if (g->model != RIP_MODEL_IC || g->m == 0) return RIP_OK;
  DevMem sums, lam;
  int rc = dalloc(c, g->vthr, sizeof(uint32_t) * (size_t)g->n);
  if (!rc) rc = dalloc(c, lam, sizeof(float) * (size_t)g->n);
  if (!rc) rc = dalloc(c, sums, 2 * sizeof(unsigned long long));
  if (rc) {  // an optional speed-up: without room for it the graph still works
    dfree(c, g->vthr);
    dfree(c, lam);
    dfree(c, sums);
    return RIP_OK;
  }
  launch_uniform_threshold(ptr<uint32_t>(g->off), ptr<uint2>(g->edges), g->n, g->m,
                           ptr<uint32_t>(g->vthr), ptr<float>(lam),
                           ptr<unsigned long long>(sums), c->stream);
  unsigned long long h[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(h, sums.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  dfree(c, sums);
  dfree(c, lam);
  if (e != cudaSuccess) {
    dfree(c, g->vthr);
    return set_err(c, RIP_ERR_CUDA, "uniform thresholds: %s", cudaGetErrorString(e));
  }
  if (2 * h[0] < g->m) dfree(c, g->vthr);
  g->use_vthr = g->vthr.p != nullptr;
  double total = 0.0;
  std::memcpy(&total, &h[1], sizeof(total));
  g->branching = total / (double)g->m;
  // grid-wide multi-colour BFS for heavy sets only where sets grow large and
  // overlap (a supercritical reverse BFS); else one CTA per heavy set
  g->default_giant_min = g->branching > kSupercritical ? 32u : 0u;
  return RIP_OK;
}

extern "C" int rip_graph_upload(rip_ctx *c, const uint64_t *index,
                                const uint32_t *src, const float *w, uint32_t n,
                                uint64_t m, int model, rip_graph **out) {
  if (!c || !out || !index || n == 0 || (m && (!src || !w)))
    return set_err(c, RIP_ERR_INVALID, "rip_graph_upload: bad arguments");
  if (model != RIP_MODEL_IC && model != RIP_MODEL_LT)
    return set_err(c, RIP_ERR_INVALID, "rip_graph_upload: unknown model %d", model);
  if (n >= 0xFFFFFFFFu || m >= 0xFFFFFFFCull)
    return set_err(c, RIP_ERR_LIMIT, "graph too large: n=%u m=%llu", n,
                   (unsigned long long)m);
  if (index[0] != 0 || index[n] != m)
    return set_err(c, RIP_ERR_INVALID, "index[0] must be 0 and index[n] == m");
  *out = nullptr;
  CK(c, cudaSetDevice(c->device));
  rip_graph *g = new rip_graph();
  g->ctx = c;
  g->n = n;
  g->m = m;
  g->model = model;
  const uint64_t m_pad = ((m + 3) & ~3ull) + 4;
  DevMem d_index, d_src, d_w;
  int rc = RIP_OK;
  do {
    if ((rc = dalloc(c, g->off, sizeof(uint32_t) * ((size_t)n + 1)))) break;
    if ((rc = dalloc(c, g->edges, sizeof(uint2) * m_pad))) break;
    if ((rc = dalloc(c, d_index, sizeof(uint64_t) * ((size_t)n + 1)))) break;
    if ((rc = dalloc(c, d_src, sizeof(uint32_t) * std::max<uint64_t>(m, 1)))) break;
    if ((rc = dalloc(c, d_w, sizeof(float) * std::max<uint64_t>(m, 1)))) break;
    cudaError_t e = cudaMemcpyAsync(d_index.p, index, sizeof(uint64_t) * ((size_t)n + 1),
                                    cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && m)
      e = cudaMemcpyAsync(d_src.p, src, sizeof(uint32_t) * m,
                          cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && m)
      e = cudaMemcpyAsync(d_w.p, w, sizeof(float) * m, cudaMemcpyHostToDevice,
                          c->stream);
    if (e != cudaSuccess) {
      rc = set_err(c, RIP_ERR_CUDA, "graph upload copy failed: %s",
                   cudaGetErrorString(e));
      break;
    }
    // validated on the device before anything indexes by it
    unsigned long long bad = 0;  // counted in the first word of the edge buffer
    launch_validate_csr(ptr<uint64_t>(d_index), ptr<uint32_t>(d_src), n, m,
                        reinterpret_cast<unsigned long long *>(g->edges.p), c->stream);
    e = cudaMemcpyAsync(&bad, g->edges.p, sizeof(bad), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      rc = set_err(c, RIP_ERR_CUDA, "graph validation failed: %s", cudaGetErrorString(e));
      break;
    }
    if (bad) {
      rc = set_err(c, RIP_ERR_INVALID,
                   "CSR not monotone or source id out of range (%llu bad)", bad);
      break;
    }
    if (model == RIP_MODEL_IC)
      launch_pack_ic(ptr<uint64_t>(d_index), ptr<float>(d_w), n, m,
                     ptr<uint32_t>(g->off), ptr<uint2>(g->edges),
                     ptr<uint32_t>(d_src), c->stream);
    else
      launch_pack_lt(ptr<uint64_t>(d_index), ptr<float>(d_w), n, m,
                     ptr<uint32_t>(g->off), ptr<uint2>(g->edges),
                     ptr<uint32_t>(d_src), c->stream);
    e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess)
      rc = set_err(c, RIP_ERR_CUDA, "graph pack failed: %s", cudaGetErrorString(e));
  } while (0);
  dfree(c, d_index);
  dfree(c, d_src);
  dfree(c, d_w);
  if (rc == RIP_OK) rc = setup_vthr(c, g);
  if (rc != RIP_OK) {
    dfree(c, g->off);
    dfree(c, g->edges);
    dfree(c, g->vthr);
    delete g;
    return rc;
  }
  c->graphs.push_back(g);
  *out = g;
  return RIP_OK;
}

// Packs index/src/weights already in device memory into a new graph.
int pack_device_csr(rip_ctx *c, const uint64_t *d_index, const uint32_t *d_src,
                           const float *d_w, uint32_t n, uint64_t m, int model,
                           rip_graph **out) {
  rip_graph *g = new rip_graph();
  g->ctx = c;
  g->n = n;
  g->m = m;
  g->model = model;
  const uint64_t m_pad = ((m + 3) & ~3ull) + 4;
  int rc = dalloc(c, g->off, sizeof(uint32_t) * ((size_t)n + 1));
  if (!rc) rc = dalloc(c, g->edges, sizeof(uint2) * m_pad);
  if (!rc) {
    if (model == RIP_MODEL_IC)
      launch_pack_ic(d_index, d_w, n, m, ptr<uint32_t>(g->off), ptr<uint2>(g->edges), d_src,
                     c->stream);
    else
      launch_pack_lt(d_index, d_w, n, m, ptr<uint32_t>(g->off), ptr<uint2>(g->edges), d_src,
                     c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) rc = set_err(c, RIP_ERR_CUDA, "pack failed: %s", cudaGetErrorString(e));
  }
  if (!rc) rc = setup_vthr(c, g);
  if (rc) {
    dfree(c, g->off);
    dfree(c, g->edges);
    dfree(c, g->vthr);
    delete g;
    return rc;
  }
  c->graphs.push_back(g);
  *out = g;
  return RIP_OK;
}

extern "C" int rip_er_keys_device(rip_ctx *c, uint32_t n, uint64_t first, uint64_t count,
                                  uint64_t seed, uint64_t *d_keys) {
  if (!c || n < 2 || (count && !d_keys)) return RIP_ERR_INVALID;
  CK(c, cudaSetDevice(c->device));
  if (count) launch_er_keys(n, first, count, seed, reinterpret_cast<unsigned long long *>(d_keys),
                            c->stream);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->stream));
  return RIP_OK;
}

extern "C" int rip_rmat_keys_device(rip_ctx *c, uint32_t scale, uint64_t first,
                                    uint64_t count, double a, double b, double cc,
                                    uint64_t seed, uint64_t *d_keys) {
  if (!c || !d_keys || scale == 0 || scale > 31 || a < 0 || b < 0 || cc < 0 ||
      a + b + cc > 1.0)
    return set_err(c, RIP_ERR_INVALID, "rip_rmat_keys_device: bad arguments");
  CK(c, cudaSetDevice(c->device));
  launch_rmat_keys(scale, first, count, a, b, cc, seed,
                   reinterpret_cast<unsigned long long *>(d_keys), c->stream);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->stream));
  return RIP_OK;
}

extern "C" int rip_graph_from_keys(rip_ctx *c, const uint64_t *d_keys, uint64_t m,
                                   uint32_t n, int weights, uint64_t weight_seed, double lo,
                                   double hi, int model, rip_graph **out) {
  if (!c || !out || (m && !d_keys) || n == 0)
    return set_err(c, RIP_ERR_INVALID, "rip_graph_from_keys: bad arguments");
  if (model != RIP_MODEL_IC && model != RIP_MODEL_LT)
    return set_err(c, RIP_ERR_INVALID, "rip_graph_from_keys: unknown model %d", model);
  if (weights != RIP_WEIGHTS_UNIFORM && weights != RIP_WEIGHTS_LT_NORMALIZED &&
      weights != RIP_WEIGHTS_WC)
    return set_err(c, RIP_ERR_INVALID, "rip_graph_from_keys: unknown weight model %d", weights);
  if (n >= 0xFFFFFFFFu || m >= 0xFFFFFFFCull)
    return set_err(c, RIP_ERR_LIMIT, "graph too large: n=%u m=%llu", n, (unsigned long long)m);
  CK(c, cudaSetDevice(c->device));
  DevMem d_index, d_src, d_w;
  int rc = dalloc(c, d_index, sizeof(uint64_t) * ((size_t)n + 1));
  if (!rc) rc = dalloc(c, d_src, sizeof(uint32_t) * std::max<uint64_t>(m, 1));
  if (!rc) rc = dalloc(c, d_w, sizeof(float) * std::max<uint64_t>(m, 1));
  if (!rc) {
    launch_csr_from_keys(reinterpret_cast<const unsigned long long *>(d_keys), m, n,
                         ptr<uint64_t>(d_index), ptr<uint32_t>(d_src), c->stream);
    launch_weights(weights, ptr<uint64_t>(d_index), n, weight_seed, lo, hi, ptr<float>(d_w),
                   c->stream);
    rc = pack_device_csr(c, ptr<uint64_t>(d_index), ptr<uint32_t>(d_src), ptr<float>(d_w), n,
                         m, model, out);
  }
  dfree(c, d_index);
  dfree(c, d_src);
  dfree(c, d_w);
  return rc;
}

extern "C" int rip_graph_export(rip_graph *g, uint64_t *index, uint32_t *src) {
  if (!g || !index || (g->m && !src)) return RIP_ERR_INVALID;
  rip_ctx *c = g->ctx;
  std::vector<uint32_t> off(g->n + 1);
  std::vector<uint2> rec(g->m);
  CK(c, cudaMemcpyAsync(off.data(), g->off.p, sizeof(uint32_t) * (g->n + 1),
                        cudaMemcpyDeviceToHost, c->stream));
  if (g->m)
    CK(c, cudaMemcpyAsync(rec.data(), g->edges.p, sizeof(uint2) * g->m,
                          cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  for (uint64_t v = 0; v <= g->n; ++v) index[v] = off[v];
  for (uint64_t e = 0; e < g->m; ++e) src[e] = rec[e].x;
  return RIP_OK;
}

extern "C" int rip_graph_destroy(rip_graph *g) {
  if (!g) return RIP_ERR_INVALID;
  rip_ctx *c = g->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  server_graph_gone(c, g);
  // pools sample from this graph: they go first
  std::vector<rip_pool *> mine;
  for (rip_pool *p : c->pools)
    if (p->g == g) mine.push_back(p);
  for (rip_pool *p : mine) rip_pool_destroy(p);
  erase_ptr(c->graphs, g);
  dfree(g->ctx, g->off);
  dfree(g->ctx, g->edges);
  dfree(g->ctx, g->vthr);
  delete g;
  return RIP_OK;
}

extern "C" int rip_graph_info(const rip_graph *g, uint32_t *n, uint64_t *m,
                              int *model) {
  if (!g) return RIP_ERR_INVALID;
  if (n) *n = g->n;
  if (m) *m = g->m;
  if (model) *model = g->model;
  return RIP_OK;
}

extern "C" int rip_graph_thresholds(rip_graph *g, uint32_t *thr) {
  if (!g || (!thr && g->m)) return RIP_ERR_INVALID;
  rip_ctx *c = g->ctx;
  std::vector<uint2> rec(g->m);
  if (g->m) {
    CK(c, cudaMemcpyAsync(rec.data(), g->edges.p, sizeof(uint2) * g->m,
                          cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
  }
  for (uint64_t e = 0; e < g->m; ++e) thr[e] = rec[e].y;
  return RIP_OK;
}

extern "C" int rip_graph_uniform_thresholds(rip_graph *g, int enable, int *available) {
  if (!g) return RIP_ERR_INVALID;
  if (available) *available = g->vthr.p != nullptr;
  if (enable >= 0) g->use_vthr = enable && g->vthr.p != nullptr;
  return RIP_OK;
}

extern "C" int rip_graph_branching(const rip_graph *g, double *branching) {
  if (!g || !branching) return RIP_ERR_INVALID;
  *branching = g->branching;
  return RIP_OK;
}
