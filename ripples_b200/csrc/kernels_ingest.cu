// kernels_ingest.cu -- a loaded edge list turned into the packed backward CSR
// on the device.
//
// The reference builds its graph from an edge list on the host: the Graph
// constructor (include/ripples/graph.h:506-620) collects the vertex ids,
// renumbers them to 0..n-1 in sorted order (unless renumbering is off), counts
// in-degrees and fills each in-list under locks; get_transpose
// (graph.h:787-832) turns one direction into the other.  rip_graph_from_edges
// does the same on the GPU for the edge list a TSV file gives
// (rip_read_tsv_edges):
//   1. renumbering: the 2m endpoint ids sorted and de-duplicated (the reverse
//      map), each endpoint replaced by its rank (binary search);
//      without renumbering n = largest id + 1;
//   2. keys (dst << 32 | src) with the edge's position as the value, radix
//      sorted (stable: parallel edges keep their input order) -- each
//      vertex's in-list ordered by source id, as the host reader orders it;
//   3. offsets from the sorted keys, weights gathered through the positions,
//      then the model's packing (thresholds) as for every other graph.
// The sort and de-duplication are CUB's device primitives (input plumbing,
// not the sampling path).
#include <cub/cub.cuh>

#include "host.h"

namespace rip {
namespace {

__global__ void endpoints_kernel(const uint32_t *s, const uint32_t *d, uint64_t m,
                                 uint32_t *ids) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    ids[2 * e] = s[e];
    ids[2 * e + 1] = d[e];
  }
}

// x[e] = rank of x[e] among the n sorted distinct ids
__global__ void rank_kernel(const uint32_t *uniq, uint32_t n, uint32_t *x, uint64_t m) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = x[e];
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (uniq[mid] < v) lo = mid + 1;
      else hi = mid;
    }
    x[e] = lo;
  }
}

__global__ void keys_kernel(const uint32_t *s, const uint32_t *d, uint64_t m,
                            unsigned long long *keys, uint32_t *pos) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    keys[e] = ((unsigned long long)d[e] << 32) | s[e];
    pos[e] = (uint32_t)e;
  }
}

__global__ void max_kernel(const uint32_t *a, const uint32_t *b, uint64_t m, unsigned int *mx) {
  uint32_t x = 0;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    x = max(x, max(a[e], b[e]));
  for (int k = 16; k > 0; k >>= 1) x = max(x, __shfl_xor_sync(FULL, x, k));
  if ((threadIdx.x & 31u) == 0) atomicMax(mx, x);
}

__global__ void gather_kernel(const float *w, const uint32_t *pos, uint64_t m, float *out) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    out[e] = w[pos[e]];
}

constexpr int kGrid = 2368, kBlock = 256;

}  // namespace
}  // namespace rip

using namespace rip;

extern "C" int rip_graph_from_edges(rip_ctx *c, const uint32_t *src, const uint32_t *dst,
                                    const float *w, uint64_t m, int renumber, int model,
                                    rip_graph **out) {
  if (!c || !out || (m && (!src || !dst || !w)))
    return set_err(c, RIP_ERR_INVALID, "rip_graph_from_edges: bad arguments");
  if (model != RIP_MODEL_IC && model != RIP_MODEL_LT)
    return set_err(c, RIP_ERR_INVALID, "rip_graph_from_edges: unknown model %d", model);
  if (m == 0) return set_err(c, RIP_ERR_INVALID, "rip_graph_from_edges: no edges");
  if (m >= 0xFFFFFFFCull)
    return set_err(c, RIP_ERR_LIMIT, "rip_graph_from_edges: at most 2^32 - 5 edges");
  *out = nullptr;
  CK(c, cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  DevMem d_s, d_d, d_w, d_ids, d_uniq, d_num, d_keys, d_keys2, d_pos, d_pos2, d_tmp, d_index,
      d_src, d_w2;
  auto release = [&]() {
    for (DevMem *x : {&d_s, &d_d, &d_w, &d_ids, &d_uniq, &d_num, &d_keys, &d_keys2, &d_pos,
                      &d_pos2, &d_tmp, &d_index, &d_src, &d_w2})
      dfree(c, *x);
  };
  struct Release {
    decltype(release) &r;
    ~Release() { r(); }
  } guard{release};
  TRY(dalloc(c, d_s, 4 * m));
  TRY(dalloc(c, d_d, 4 * m));
  TRY(dalloc(c, d_w, 4 * m));
  CK(c, cudaMemcpyAsync(d_s.p, src, 4 * m, cudaMemcpyHostToDevice, st));
  CK(c, cudaMemcpyAsync(d_d.p, dst, 4 * m, cudaMemcpyHostToDevice, st));
  CK(c, cudaMemcpyAsync(d_w.p, w, 4 * m, cudaMemcpyHostToDevice, st));
  uint32_t n = 0;
  std::vector<uint32_t> reverse_map;
  TRY(dalloc(c, d_num, sizeof(unsigned long long)));
  if (renumber) {
    // the sorted distinct endpoint ids
    const uint64_t m2 = 2 * m;
    TRY(dalloc(c, d_ids, 4 * m2));
    TRY(dalloc(c, d_uniq, 4 * m2));
    count_launches(1);
    endpoints_kernel<<<kGrid, kBlock, 0, st>>>(ptr<uint32_t>(d_s), ptr<uint32_t>(d_d), m,
                                               ptr<uint32_t>(d_ids));
    size_t tb = 0, tb2 = 0;
    CK(c, cub::DeviceRadixSort::SortKeys(nullptr, tb, ptr<uint32_t>(d_ids),
                                         ptr<uint32_t>(d_uniq), (int64_t)m2, 0, 32, st));
    CK(c, cub::DeviceSelect::Unique(nullptr, tb2, ptr<uint32_t>(d_uniq), ptr<uint32_t>(d_ids),
                                    ptr<unsigned long long>(d_num), (int64_t)m2, st));
    TRY(dalloc(c, d_tmp, std::max(tb, tb2)));
    tb = d_tmp.bytes;
    CK(c, cub::DeviceRadixSort::SortKeys(d_tmp.p, tb, ptr<uint32_t>(d_ids),
                                         ptr<uint32_t>(d_uniq), (int64_t)m2, 0, 32, st));
    tb = d_tmp.bytes;
    CK(c, cub::DeviceSelect::Unique(d_tmp.p, tb, ptr<uint32_t>(d_uniq), ptr<uint32_t>(d_ids),
                                    ptr<unsigned long long>(d_num), (int64_t)m2, st));
    unsigned long long nu = 0;
    CK(c, cudaMemcpyAsync(&nu, d_num.p, sizeof(nu), cudaMemcpyDeviceToHost, st));
    CK(c, cudaStreamSynchronize(st));
    if (nu >= 0xFFFFFFFFull)
      return set_err(c, RIP_ERR_LIMIT, "rip_graph_from_edges: too many vertices");
    n = (uint32_t)nu;
    reverse_map.resize(n);
    CK(c, cudaMemcpyAsync(reverse_map.data(), d_ids.p, 4ull * n, cudaMemcpyDeviceToHost, st));
    count_launches(2);
    rank_kernel<<<kGrid, kBlock, 0, st>>>(ptr<uint32_t>(d_ids), n, ptr<uint32_t>(d_s), m);
    rank_kernel<<<kGrid, kBlock, 0, st>>>(ptr<uint32_t>(d_ids), n, ptr<uint32_t>(d_d), m);
    dfree(c, d_uniq);
    dfree(c, d_tmp);
  } else {
    CK(c, cudaMemsetAsync(d_num.p, 0, sizeof(unsigned int), st));
    count_launches(1);
    max_kernel<<<kGrid, kBlock, 0, st>>>(ptr<uint32_t>(d_s), ptr<uint32_t>(d_d), m,
                                         ptr<unsigned int>(d_num));
    unsigned int mx = 0;
    CK(c, cudaMemcpyAsync(&mx, d_num.p, sizeof(mx), cudaMemcpyDeviceToHost, st));
    CK(c, cudaStreamSynchronize(st));
    if (mx >= 0xFFFFFFFEu)
      return set_err(c, RIP_ERR_LIMIT, "rip_graph_from_edges: vertex id too large");
    n = mx + 1;
  }
  // in-lists ordered by source id, parallel edges in input order
  TRY(dalloc(c, d_keys, 8 * m));
  TRY(dalloc(c, d_keys2, 8 * m));
  TRY(dalloc(c, d_pos, 4 * m));
  TRY(dalloc(c, d_pos2, 4 * m));
  count_launches(1);
  keys_kernel<<<kGrid, kBlock, 0, st>>>(ptr<uint32_t>(d_s), ptr<uint32_t>(d_d), m,
                                        ptr<unsigned long long>(d_keys), ptr<uint32_t>(d_pos));
  dfree(c, d_s);
  dfree(c, d_d);
  {
    size_t tb = 0;
    CK(c, cub::DeviceRadixSort::SortPairs(nullptr, tb, ptr<unsigned long long>(d_keys),
                                          ptr<unsigned long long>(d_keys2),
                                          ptr<uint32_t>(d_pos), ptr<uint32_t>(d_pos2),
                                          (int64_t)m, 0, 64, st));
    TRY(dalloc(c, d_tmp, tb));
    tb = d_tmp.bytes;
    CK(c, cub::DeviceRadixSort::SortPairs(d_tmp.p, tb, ptr<unsigned long long>(d_keys),
                                          ptr<unsigned long long>(d_keys2),
                                          ptr<uint32_t>(d_pos), ptr<uint32_t>(d_pos2),
                                          (int64_t)m, 0, 64, st));
    dfree(c, d_tmp);
    dfree(c, d_keys);
    dfree(c, d_pos);
  }
  TRY(dalloc(c, d_index, 8ull * ((size_t)n + 1)));
  TRY(dalloc(c, d_src, 4 * m));
  TRY(dalloc(c, d_w2, 4 * m));
  launch_csr_from_keys(ptr<unsigned long long>(d_keys2), m, n, ptr<uint64_t>(d_index),
                       ptr<uint32_t>(d_src), st);
  count_launches(1);
  gather_kernel<<<kGrid, kBlock, 0, st>>>(ptr<float>(d_w), ptr<uint32_t>(d_pos2), m,
                                          ptr<float>(d_w2));
  CK(c, cudaGetLastError());
  dfree(c, d_keys2);
  dfree(c, d_pos2);
  dfree(c, d_w);
  rip_graph *g = nullptr;
  TRY(pack_device_csr(c, ptr<uint64_t>(d_index), ptr<uint32_t>(d_src), ptr<float>(d_w2), n, m,
                      model, &g));
  g->reverse_map = std::move(reverse_map);
  *out = g;
  return RIP_OK;
}

extern "C" int rip_graph_id_map(const rip_graph *g, uint32_t *map) {
  if (!g || !map) return RIP_ERR_INVALID;
  if (g->reverse_map.empty()) {
    for (uint32_t v = 0; v < g->n; ++v) map[v] = v;
  } else {
    std::memcpy(map, g->reverse_map.data(), 4ull * g->n);
  }
  return RIP_OK;
}
