// host.h -- host runtime internals shared by the C-ABI translation units:
// the context (stream, device-memory budget and block cache, pinned
// buffers), the device graph and the RRR pool objects, error and CUDA-call
// macros.
#pragma once
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <queue>
#include <string>
#include <utility>
#include <vector>

#include <sys/types.h>

#include "launch.h"
#include "ripples_b200.h"

using namespace rip;

using clk = std::chrono::high_resolution_clock;
inline double ms_since(clk::time_point t0) {
  return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

// ---------------------------------------------------------------------------
// context, memory
// ---------------------------------------------------------------------------
struct DevMem {
  void *p = nullptr;
  size_t bytes = 0;
};

// The reference's heap holds std::pair<vertex, size_t count> ordered by count
// alone (CompareHeap, include/ripples/streaming_find_most_influential.h:410-418).
// The heap algorithms only move elements and compare them with the
// comparator, so an 8-byte {vertex, u32 count} item with the same comparison
// yields the same sequence of heaps (counts never exceed the number of sets,
// < 2^32), at half the memory.
struct HeapItem {
  uint32_t first;   // vertex
  uint32_t second;  // count when pushed
  bool operator==(const HeapItem &o) const { return first == o.first && second == o.second; }
};
struct CompareHeap {
  bool operator()(const HeapItem &a, const HeapItem &b) const { return a.second < b.second; }
};
struct PinnedMem;

struct rip_ctx {
  std::vector<rip_graph *> graphs;  // owned: freed by rip_ctx_destroy
  std::vector<rip_pool *> pools;    // owned: freed by rip_ctx_destroy
  std::vector<rip_server *> servers;  // owned: freed by rip_ctx_destroy
  // Device blocks released by graphs/pools, kept for reuse (a graph upload
  // or a new pool then costs no cudaMalloc); counted in `used`.
  std::vector<DevMem> cache;
  size_t cached = 0;
  PinnedMem *h_cand = nullptr;   // mapped: reference-heap candidate ids and counts
  // last epoch a cover-and-gather kernel published in h_cand's first word
  // (unique per context, so a flag left by an earlier pick never matches)
  uint32_t cg_epoch = 0;
  // reference-heap selection storage, shared by the context's pools (one
  // selection runs at a time) and page-locked once
  std::vector<HeapItem> heap_store;
  void *heap_registered = nullptr;
  PinnedMem *h_count = nullptr;  // counts at the start of a selection
  // multi-instance sampler scratch (per warp: bitmap for the largest graph
  // of the launch + queue), instance table, failure pairs
  DevMem m_scratch, m_table, m_fail;
  uint64_t m_bm_words = 0;
  uint32_t m_qcap = 0, m_warps = 0;
  PinnedMem *h_meta = nullptr;  // per-pool meta blocks read back together
  double multi_kernel_ms = 0.0;
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  size_t budget = 0;
  size_t used = 0;
  std::string err;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

inline int set_err(rip_ctx *c, int code, const char *fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

#define CK(c, call)                                                          \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return set_err((c), RIP_ERR_CUDA, "%s failed: %s (%s:%d)", #call,      \
                     cudaGetErrorString(e_), __FILE__, __LINE__);            \
  } while (0)

#define TRY(expr)              \
  do {                         \
    int r_ = (expr);           \
    if (r_ != RIP_OK) return r_; \
  } while (0)

inline void cache_release_all(rip_ctx *c) {
  if (!c->cache.empty()) cudaStreamSynchronize(c->stream);
  for (DevMem &b : c->cache) {
    cudaFree(b.p);
    c->used -= b.bytes;
  }
  c->cache.clear();
  c->cached = 0;
}

// Returns a block to the context cache (or frees it when the cache is full).
inline void cache_put(rip_ctx *c, DevMem m) {
  if (!m.p) return;
  const size_t limit = c->budget / 4;
  if (m.bytes > limit) {
    cudaStreamSynchronize(c->stream);
    cudaFree(m.p);
    c->used -= m.bytes;
    return;
  }
  while (c->cached + m.bytes > limit && !c->cache.empty()) {
    cudaStreamSynchronize(c->stream);
    cudaFree(c->cache.front().p);
    c->used -= c->cache.front().bytes;
    c->cached -= c->cache.front().bytes;
    c->cache.erase(c->cache.begin());
  }
  c->cache.push_back(m);
  c->cached += m.bytes;
}

// Takes the smallest cached block of at least `bytes` (and at most twice that).
inline bool cache_take(rip_ctx *c, size_t bytes, DevMem &out) {
  size_t best = c->cache.size();
  for (size_t i = 0; i < c->cache.size(); ++i) {
    const size_t b = c->cache[i].bytes;
    if (b >= bytes && b <= 2 * bytes + (1u << 20) &&
        (best == c->cache.size() || b < c->cache[best].bytes))
      best = i;
  }
  if (best == c->cache.size()) return false;
  out = c->cache[best];
  c->cached -= out.bytes;
  c->cache.erase(c->cache.begin() + best);
  return true;
}

inline int dalloc(rip_ctx *c, DevMem &m, size_t bytes) {
  if (m.p && m.bytes >= bytes) return RIP_OK;
  bytes = std::max<size_t>((bytes + 255) & ~(size_t)255, 256);
  DevMem fresh;
  if (!cache_take(c, bytes, fresh)) {
    if (c->used + bytes > c->budget) cache_release_all(c);
    if (c->used + bytes > c->budget)
      return set_err(c, RIP_ERR_NOMEM,
                     "device budget exceeded: need %zu more bytes (used %zu of %zu)",
                     bytes, c->used, c->budget);
    cudaError_t e = cudaMalloc(&fresh.p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      cache_release_all(c);
      e = cudaMalloc(&fresh.p, bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, RIP_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes,
                       cudaGetErrorString(e));
      }
    }
    fresh.bytes = bytes;
    c->used += bytes;
  }
  cache_put(c, m);
  m = fresh;
  return RIP_OK;
}

// Grows m to `bytes`, preserving the first `keep` bytes.
inline int dgrow(rip_ctx *c, DevMem &m, size_t bytes, size_t keep) {
  if (m.p && m.bytes >= bytes) return RIP_OK;
  DevMem n;
  TRY(dalloc(c, n, bytes));
  if (m.p && keep) {
    CK(c, cudaMemcpyAsync(n.p, m.p, std::min(keep, m.bytes),
                          cudaMemcpyDeviceToDevice, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
  }
  cache_put(c, m);
  m = n;
  return RIP_OK;
}

inline void dfree(rip_ctx *c, DevMem &m) {
  cache_put(c, m);
  m = DevMem{};
}

template <typename T>
inline T *ptr(DevMem &m) {
  return reinterpret_cast<T *>(m.p);
}

struct PinnedMem {
  void *p = nullptr;
  void *dev = nullptr;  // device alias when mapped
  size_t bytes = 0;
  int ensure(rip_ctx *c, size_t b, bool mapped = false) {
    if (p && bytes >= b) return RIP_OK;
    if (p) cudaFreeHost(p);
    p = dev = nullptr;
    bytes = 0;
    if (cudaHostAlloc(&p, b, mapped ? cudaHostAllocMapped : cudaHostAllocDefault) !=
        cudaSuccess) {
      cudaGetLastError();
      return set_err(c, RIP_ERR_NOMEM, "cudaHostAlloc(%zu) failed", b);
    }
    if (mapped && cudaHostGetDevicePointer(&dev, p, 0) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeHost(p);
      p = nullptr;
      return set_err(c, RIP_ERR_CUDA, "cudaHostGetDevicePointer failed");
    }
    bytes = b;
    return RIP_OK;
  }
  ~PinnedMem() {
    if (p) cudaFreeHost(p);
  }
};


// Branching factor above which untuned IC graphs grow heavy sets with the
// grid-wide multi-colour BFS (sets large and overlapping) rather than one CTA
// per set.
constexpr double kSupercritical = 1.1;

struct rip_graph {
  rip_ctx *ctx;
  uint32_t n;
  uint64_t m;
  int model;
  DevMem off, edges;
  // internal id -> input id when the graph was built from an edge list with
  // renumbering (rip_graph_from_edges); empty: the identity
  std::vector<uint32_t> reverse_map;
  // per-vertex uniform IC thresholds (DevGraph::vthr); allocated only when
  // uniform in-lists hold at least half of the edges, and used while
  // use_vthr is set
  DevMem vthr;
  bool use_vthr = false;
  // IC: branching factor of a reverse BFS -- the expected live in-edges of
  // an edge's source, sum over edges of lambda(src) / m with lambda(u) the
  // sum of u's in-edge probabilities -- and the heavy-set batch size pools of
  // an untuned graph start with (rip_pool_heavy_batch)
  double branching = 0.0;
  uint32_t default_giant_min = 32;
  // IC sampler configuration picked by rip_graph_autotune (pools created
  // afterwards start from it; RIP_SAMPLER_AUTO follows `sampler`)
  struct Tuned {
    bool set = false;
    int sampler = RIP_SAMPLER_PLAIN;
    uint32_t colors = 64, giant_min = 32;
    uint64_t cap_plain = 1ull << 18, cap_fused = 1ull << 23;
    int plain_occupancy = 0;
    uint32_t big_threads = 256;
  } tuned;
  DevGraph view() {
    return DevGraph{n, m, ptr<uint32_t>(off), ptr<uint2>(edges),
                    use_vthr && vthr.p ? ptr<uint32_t>(vthr) : nullptr};
  }
};
// Packs a backward CSR already in device memory (index u64[n+1], src u32[m],
// weights f32[m]) into a new graph of the context (graph.cu).
int pack_device_csr(rip_ctx *c, const uint64_t *d_index, const uint32_t *d_src,
                    const float *d_w, uint32_t n, uint64_t m, int model, rip_graph **out);


// A captured lowest-id pick loop and the addresses it was captured with.
struct SelGraph {
  cudaGraphExec_t exec = nullptr;
  uint32_t k = 0;
  int pick_blocks = 0;
  void *src = nullptr, *dst = nullptr, *desc = nullptr;
  uint64_t nodes = 0;
};

struct ServeSegment {
  DevMem off, inv;  // off u64[n + 1], inv u32[]: set ids in [first, last)
  uint64_t first = 0, last = 0;
};

struct PoolMeta {  // device-side bookkeeping block (one D2H reads it all)
  unsigned long long cursor;
  unsigned long long first_bad;
  unsigned long long stats[8];
  unsigned int fail_count;
  unsigned int next;
  unsigned int fused_dirty;
};

constexpr uint64_t kNoShard = ~0ull;

struct rip_pool {
  rip_ctx *ctx;
  rip_graph *g;
  DevMem vtx, set_off, set_len, meta;
  uint64_t cap = 0, set_cap = 0;
  uint64_t num_sets = 0, num_elems = 0;
  // sampler scratch (one buffer partitioned into per-warp bitmap + queue)
  DevMem scratch, ids_a, ids_b;
  uint64_t bm_words = 0;
  uint32_t qcap = 0;
  uint32_t warps = 0;
  // fused sampler scratch (per slot: colour masks, pending masks, level
  // flags, frontier log); all-zero between batches
  DevMem f_vis, f_pend, f_flag, f_log, f_order;
  uint32_t f_slots = 0, f_cw = 0, f_lcap = 0;
  // CTA-per-set scratch for sets with very large edge work
  DevMem b_scratch, b_ids;
  uint32_t b_slots = 0, b_qcap = 0;
  // grid-wide multi-colour BFS for the heavy sets (all-zero between batches)
  DevMem g_state, g_lists, g_col;
  uint32_t giant_min = 32;  // heavy sets that switch to the grid-wide BFS (0 = never)
  int auto_sampler = RIP_SAMPLER_PLAIN;  // what RIP_SAMPLER_AUTO runs (IC)
  int plain_occupancy = 0;   // IC one-set-per-warp kernel variant (0 or 5)
  uint64_t cap_plain = 1ull << 18;  // in-edges per set before a warp hands it over
  uint64_t cap_fused = 1ull << 23;  // in-edges per fused batch before handing over
  uint64_t big_sets = 0;            // sets grown one CTA each (diagnostic)
  uint32_t big_threads = 256;       // block shape of the CTA-per-set kernel (128-1024)
  uint32_t colors = 64;      // fused colour width (64/128/256)
  uint32_t fused_slots = 0;  // 0 = size from the budget
  uint32_t lcap_pref = 0;    // 0 = default frontier-log capacity
  // selection state
  DevMem count, inv_off, inv_cur, inv, covered,
      scan_sums;
  // vertex -> sets index over sets [0, sv_sets), shared by the served
  // queries drawing from this pool (each filters to its own prefix): one
  // segment per growth step, merged into one past SEL_MAX_SEGMENTS
  std::vector<ServeSegment> sv_segs;
  DevMem sv_count, sv_cur, sv_sums;  // build scratch
  uint64_t sv_sets = 0;
  std::vector<uint32_t> last_counts;
  bool last_counts_on_device = false;  // last_counts still in `count` only
  bool have_last_counts = false;
  uint32_t cand_fixed = 0;           // first-fetch threshold, % of the last gain (0 = adaptive)
  DevMem d_heap;                     // heap built on the device
  DevMem s_cmax, s_dirty, s_best, s_desc;  // device lowest-id picks
  // reference-heap picks: completion ticket of the cover-and-gather kernel
  // (zero between launches)
  DevMem cg_done;
  bool cg_done_zeroed = false;
  PinnedMem h_best;
  SelGraph sel_graph;                // the captured pick loop
  // sharded selection: `count` holds this shard's counts over sets
  // [0, shard_sets) with their index and covered flags (kNoShard: it does not)
  uint64_t shard_sets = kNoShard;
  uint64_t shard_elems = 0;          // elements of those sets (bound of a decrement list)
  const void *shard_sum = nullptr;   // the summed array whose chunk maxima are cached
  bool shard_cache_ok = false;       // shard_cmax + dirty flags describe shard_sum
  DevMem shard_cmax, shard_dirty;    // per kPickChunk counts: max key, changed flag
  DevMem shard_meta;                 // [0] the pick's key, [1] decrement-list cursor
  PinnedMem h_shard_meta;
  // selection profile: [0] count+index kernels and counts D2H, [1] heap build,
  // [2] pick loop, [3] heap pops, [4] picks, [5] candidate counts fetched,
  // [6] selections, [7] ms covering + fetching candidate counts, [8] fetches
  // of the whole count array from a pop outside the candidates, [9] ms in pops,
  // [10] ms collecting candidates on the host, [11] candidate fetch rounds
  double sel_prof[12] = {0};
  // timing of sampler kernels (CUDA events on the context stream)
  double kernel_ms = 0.0;
  uint64_t kernel_launches = 0;
  double select_kernel_ms = 0.0;

  PoolMeta *dmeta() { return ptr<PoolMeta>(meta); }
  DevPool view() {
    return DevPool{ptr<uint32_t>(vtx), &dmeta()->cursor, cap,
                   ptr<uint64_t>(set_off), ptr<uint32_t>(set_len)};
  }
};

// Ends the server queries on graph g and drops the servers' pools on it
// (called before g is destroyed).
void server_graph_gone(rip_ctx *c, rip_graph *g);

template <typename T>
inline void erase_ptr(std::vector<T *> &v, T *x) {
  v.erase(std::remove(v.begin(), v.end(), x), v.end());
}
