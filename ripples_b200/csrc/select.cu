// select.cu -- greedy max-coverage seed selection behind include/ripples_b200.h
// (FindMostInfluentialSet, include/ripples/find_most_influential.h:176):
// counts, inverted index, the reference CPU heap (exact, host pops with
// device-fetched counts) and device-only lowest-id picks.
#include "host.h"

// ---------------------------------------------------------------------------
// selection
// ---------------------------------------------------------------------------
namespace {
using RefQueue = std::priority_queue<HeapItem, std::vector<HeapItem>, CompareHeap>;

// std::priority_queue that adopts an already-heapified container instead of
// running make_heap again (its container and comparator are protected
// members).  pop/push are libstdc++'s own pop_heap/push_heap, as in the
// reference.
struct AdoptedQueue : RefQueue {
  explicit AdoptedQueue(std::vector<HeapItem> &&heap) { this->c = std::move(heap); }
  std::vector<HeapItem> release() { return std::move(this->c); }
  const std::vector<HeapItem> &items() const { return this->c; }
};

// The vertices of every heap item keyed at least T (keys never grow
// downwards, so subtrees whose root is keyed below T are skipped).  Walked
// breadth first: the children of a queued node are prefetched when it is
// queued, so the random reads into the heap array overlap.  Returns the
// count, or cap + 1 when more than cap items qualify.
static uint32_t collect_at_least(const std::vector<HeapItem> &h, uint32_t T, uint32_t cap,
                                 uint32_t *out, std::vector<uint32_t> &queue) {
  const size_t len = h.size();
  uint32_t cnt = 0;
  queue.clear();
  if (len && h[0].second >= T) queue.push_back(0);
  for (size_t head = 0; head < queue.size(); ++head) {
    const size_t i = queue[head];
    if (cnt == cap) return cap + 1;
    out[cnt++] = h[i].first;
    const size_t l = 2 * i + 1;
    for (size_t c = l; c < l + 2 && c < len; ++c)
      if (h[c].second >= T) {
        queue.push_back((uint32_t)c);
        if (2 * c + 1 < len) __builtin_prefetch(&h[2 * c + 1]);
      }
  }
  return cnt;
}

// Open-addressing map vertex -> fetched count for one pick's candidates.
struct CountMap {
  std::vector<uint32_t> key, val;  // key = vertex + 1, 0 = empty
  uint32_t mask = 0;
  void reset(uint32_t items) {
    uint32_t cap = 64;
    while (cap < 2 * items) cap <<= 1;
    if (key.size() < cap) {
      key.assign(cap, 0u);
      val.resize(cap);
    } else {
      std::fill(key.begin(), key.begin() + cap, 0u);
    }
    mask = cap - 1;
  }
  static uint32_t hash(uint32_t v) { return (v * 2654435761u) ^ (v >> 15); }
  void put(uint32_t v, uint32_t c) {
    uint32_t i = hash(v) & mask;
    while (key[i] != 0u && key[i] != v + 1) i = (i + 1) & mask;
    key[i] = v + 1;
    val[i] = c;
  }
  bool get(uint32_t v, uint32_t &c) const {
    uint32_t i = hash(v) & mask;
    while (key[i] != 0u) {
      if (key[i] == v + 1) {
        c = val[i];
        return true;
      }
      i = (i + 1) & mask;
    }
    return false;
  }
};

// Bit-identical to std::make_heap(v.begin(), v.end(), CompareHeap{}), built
// level by level in parallel.  libstdc++'s make_heap runs __adjust_heap on
// every parent from (len-2)/2 down to 0; each call only touches the subtree
// under its parent, and all parents at one depth have disjoint subtrees and
// larger indices than every parent above them, so processing the depths from
// the deepest up -- each depth in any order -- performs the same operations on
// the same data.
void parallel_make_heap(std::vector<HeapItem> &v) {
  const std::ptrdiff_t len = (std::ptrdiff_t)v.size();
  if (len < 2) return;
  const std::ptrdiff_t last_parent = (len - 2) / 2;
  int dmax = 0;
  while ((((std::ptrdiff_t)2) << dmax) - 1 <= last_parent) ++dmax;
  for (int d = dmax; d >= 0; --d) {
    const std::ptrdiff_t lo = (((std::ptrdiff_t)1) << d) - 1;
    const std::ptrdiff_t hi = std::min(last_parent, (((std::ptrdiff_t)2) << d) - 2);
#pragma omp parallel for schedule(static) if (hi - lo > 8192)
    for (std::ptrdiff_t p = hi; p >= lo; --p) {
      HeapItem val = std::move(v[p]);
      std::__adjust_heap(v.begin(), p, len, std::move(val),
                         __gnu_cxx::__ops::_Iter_comp_iter<CompareHeap>(CompareHeap{}));
    }
  }
}
}  // namespace

// Diagnostic: the device heap build against std::make_heap on n random
// {vertex, count} items with counts in [0, max_count); 1 when identical.
extern "C" int rip_selftest_heap_device(rip_ctx *c, uint64_t n, uint32_t max_count,
                                        uint64_t seed) {
  if (!c || n == 0 || n >= 0xFFFFFFFFull) return RIP_ERR_INVALID;
  std::vector<uint32_t> cnt(n);
  uint64_t x = seed * 6364136223846793005ull + 1442695040888963407ull;
  for (uint64_t i = 0; i < n; ++i) {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    cnt[i] = (uint32_t)((x >> 33) % (max_count ? max_count : 1));
  }
  std::vector<HeapItem> ref(n), got(n);
  for (uint64_t i = 0; i < n; ++i) ref[i] = {(uint32_t)i, cnt[i]};
  std::make_heap(ref.begin(), ref.end(), CompareHeap{});
  DevMem d_cnt, d_heap;
  int rc = dalloc(c, d_cnt, 4 * n);
  if (!rc) rc = dalloc(c, d_heap, 8 * n);
  if (!rc) {
    cudaMemcpyAsync(d_cnt.p, cnt.data(), 4 * n, cudaMemcpyHostToDevice, c->stream);
    launch_make_heap(ptr<uint32_t>(d_cnt), (uint32_t)n, ptr<uint2>(d_heap), c->stream);
    cudaMemcpyAsync(got.data(), d_heap.p, 8 * n, cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) rc = set_err(c, RIP_ERR_CUDA, "heap selftest: %s", cudaGetErrorString(e));
  }
  dfree(c, d_cnt);
  dfree(c, d_heap);
  if (rc) return rc;
  return ref == got ? 1 : 0;
}

// Diagnostic: checks parallel_make_heap against std::make_heap on n random
// counts drawn from [0, max_count) (many ties); returns 1 when identical.
extern "C" int rip_selftest_heap(uint64_t n, uint32_t max_count, uint64_t seed) {
  std::vector<HeapItem> a(n), b;
  uint64_t x = seed * 6364136223846793005ull + 1442695040888963407ull;
  for (uint64_t i = 0; i < n; ++i) {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    a[i] = {(uint32_t)i, (uint32_t)((x >> 33) % (max_count ? max_count : 1))};
  }
  b = a;
  std::make_heap(b.begin(), b.end(), CompareHeap{});
  parallel_make_heap(a);
  return a == b ? 1 : 0;
}

// The counts left by the last selection still sit in the count buffer; bring
// them to the host before anything overwrites that buffer.
static int settle_last_counts(rip_pool *p) {
  if (!p->have_last_counts || !p->last_counts_on_device) return RIP_OK;
  rip_ctx *c = p->ctx;
  p->last_counts.resize(p->g->n);
  CK(c, cudaMemcpyAsync(p->last_counts.data(), p->count.p, sizeof(uint32_t) * (size_t)p->g->n,
                        cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  p->last_counts_on_device = false;
  return RIP_OK;
}

static int count_sets(rip_pool *p, uint64_t S) {
  rip_ctx *c = p->ctx;
  const uint32_t n = p->g->n;
  TRY(settle_last_counts(p));
  p->shard_sets = kNoShard;  // the count buffer no longer holds a shard's counts
  // padded to whole chunks of the device picks (the tail stays zero)
  const size_t chunk = sel_chunk_vertices();
  const size_t padded = ((size_t)n + chunk - 1) / chunk * chunk;
  TRY(dalloc(c, p->count, sizeof(uint32_t) * padded));
  CK(c, cudaMemsetAsync(p->count.p, 0, sizeof(uint32_t) * padded, c->stream));
  launch_count(p->view(), S, ptr<uint32_t>(p->count), c->num_sms * 8, c->stream);
  CK(c, cudaGetLastError());
  return RIP_OK;
}

extern "C" int rip_count(rip_pool *p, uint64_t num_sets, uint32_t *counts) {
  if (!p || !counts || num_sets > p->num_sets) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  CK(c, cudaSetDevice(c->device));
  TRY(count_sets(p, num_sets));
  CK(c, cudaMemcpyAsync(counts, p->count.p, sizeof(uint32_t) * p->g->n,
                        cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  return RIP_OK;
}

// Counts left by the last rip_select (after its last update step).
extern "C" int rip_select_counts(rip_pool *p, uint32_t *counts) {
  if (!p || !counts) return RIP_ERR_INVALID;
  if (!p->have_last_counts)
    return set_err(p->ctx, RIP_ERR_STATE, "no selection has run on this pool");
  TRY(settle_last_counts(p));
  std::memcpy(counts, p->last_counts.data(), sizeof(uint32_t) * p->g->n);
  return RIP_OK;
}

// Counts sets [0, S) into `count`, builds the vertex -> sets index over them
// (inv_off, inv) and clears their covered flags; *P_out = index length.
static int prepare_cover(rip_pool *p, uint64_t S, uint64_t *P_out) {
  rip_ctx *c = p->ctx;
  const uint32_t n = p->g->n;
  TRY(count_sets(p, S));
  TRY(dalloc(c, p->inv_off, sizeof(uint64_t) * ((size_t)n + 1)));
  TRY(dalloc(c, p->inv_cur, sizeof(uint64_t) * ((size_t)n + 1)));
  TRY(dalloc(c, p->scan_sums, sizeof(uint64_t) * scan_block_sums_needed(n)));
  launch_exclusive_scan(ptr<uint32_t>(p->count), ptr<uint64_t>(p->inv_off), n,
                        ptr<uint64_t>(p->scan_sums), c->stream);
  uint64_t P = 0;
  CK(c, cudaMemcpyAsync(&P, ptr<uint64_t>(p->inv_off) + n, sizeof(uint64_t),
                        cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaMemcpyAsync(p->inv_cur.p, p->inv_off.p, sizeof(uint64_t) * ((size_t)n + 1),
                        cudaMemcpyDeviceToDevice, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  TRY(dalloc(c, p->inv, sizeof(uint32_t) * std::max<uint64_t>(P, 1)));
  launch_build_inverted(p->view(), S, ptr<uint64_t>(p->inv_cur), ptr<uint32_t>(p->inv),
                        c->num_sms * 8, c->stream);
  CK(c, cudaGetLastError());
  TRY(dalloc(c, p->covered, std::max<uint64_t>(S, 1)));
  CK(c, cudaMemsetAsync(p->covered.p, 0, std::max<uint64_t>(S, 1), c->stream));
  *P_out = P;
  return RIP_OK;
}

static CoverLaunch cover_launch(rip_pool *p) {
  CoverLaunch C;
  C.P = p->view();
  C.inv_off = ptr<uint64_t>(p->inv_off);
  C.inv = ptr<uint32_t>(p->inv);
  C.covered = ptr<uint8_t>(p->covered);
  C.count = ptr<uint32_t>(p->count);
  C.blocks = p->ctx->num_sms * 4;
  return C;
}

extern "C" int rip_select(rip_pool *p, uint64_t S, uint32_t k, int tiebreak,
                          uint32_t *seeds, uint64_t *gains, uint32_t *num_seeds,
                          double *f) {
  if (!p || (k && !seeds) || !num_seeds) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  if (S > p->num_sets)
    return set_err(c, RIP_ERR_INVALID, "rip_select: %llu sets requested, pool has %llu",
                   (unsigned long long)S, (unsigned long long)p->num_sets);
  if (tiebreak != RIP_TIE_REF_HEAP && tiebreak != RIP_TIE_LOWEST_ID)
    return set_err(c, RIP_ERR_INVALID, "rip_select: unknown tie-break %d", tiebreak);
  if (S >= (1ull << 32))
    return set_err(c, RIP_ERR_LIMIT, "rip_select: at most 2^32-1 sets");
  CK(c, cudaSetDevice(c->device));
  const uint32_t n = p->g->n;
  *num_seeds = 0;
  if (f) *f = 0.0;
  CK(c, cudaEventRecord(c->ev0, c->stream));
  const auto t_sel0 = clk::now();
  // 1. histogram, 2. vertex -> sets index
  p->have_last_counts = false;  // superseded by this selection
  uint64_t P = 0;
  TRY(prepare_cover(p, S, &P));
  CoverLaunch C = cover_launch(p);

  // whole-array count fetches land in the context's page-locked buffer and
  // are read there (no second host copy)
  const uint32_t *hcount = nullptr;
  if (!c->h_cand) c->h_cand = new PinnedMem();
  if (!c->h_count) c->h_count = new PinnedMem();
  // mapped: candidate vertex ids in, their counts out (reference-heap picks)
  constexpr uint32_t CAND_CAP = 1u << 16;
  TRY(c->h_cand->ensure(c, 16 + 2 * sizeof(uint32_t) * (size_t)CAND_CAP, true));
  TRY(c->h_count->ensure(c, sizeof(uint32_t) * (size_t)n));
  PinnedMem &h_cand = *c->h_cand, &h_count = *c->h_count;

  uint64_t uncovered = S;
  std::vector<uint32_t> out_seeds;
  std::vector<uint64_t> out_gains;

  p->sel_prof[0] += ms_since(t_sel0);
  p->sel_prof[6] += 1;
  const int max_blocks = c->num_sms * 4;
  unsigned char *hb = static_cast<unsigned char *>(h_cand.p);
  unsigned char *db = static_cast<unsigned char *>(h_cand.dev);
  // One pick: mark v's uncovered sets covered and decrement their members, one
  // warp per set of v's inverted list (`gain` of them are still uncovered).
  auto cover = [&](uint32_t v, uint64_t gain) -> int {
    C.vertex = v;
    C.blocks = (int)std::min<uint64_t>(max_blocks * 4, std::max<uint64_t>(1, (gain + 7) / 8));
    launch_cover(C, c->stream);
    CK(c, cudaGetLastError());
    return RIP_OK;
  };

  if (tiebreak == RIP_TIE_REF_HEAP) {
    const auto t_h0 = clk::now();
    // InitHeapStorage + std::priority_queue(cmp, std::move(storage)), as the
    // reference builds its heap (streaming_find_most_influential.h:541-544;
    // counting.h:196-206): the same heap, built level-parallel on the device
    // and downloaded into page-locked storage the queue adopts as is.
    // The storage is the context's (page-locked once, reused by every pool);
    // the guards hand it back on every way out of this block.
    struct Lease {
      rip_ctx *c;
      std::vector<HeapItem> v;
      explicit Lease(rip_ctx *c_) : c(c_), v(std::move(c_->heap_store)) {}
      ~Lease() {
        if (v.capacity()) c->heap_store = std::move(v);
      }
    } lease(c);
    std::vector<HeapItem> &storage = lease.v;
    if (storage.capacity() < n || !c->heap_registered) {
      if (c->heap_registered) cudaHostUnregister(c->heap_registered);
      c->heap_registered = nullptr;
      std::vector<HeapItem>().swap(storage);
      storage.reserve(n);
      storage.resize(n);
      if (cudaHostRegister(storage.data(), sizeof(HeapItem) * storage.capacity(), 0) ==
          cudaSuccess) {
        c->heap_registered = storage.data();
      } else {
        cudaGetLastError();  // pageable copy still works, only slower
      }
    }
    storage.resize(n);
    TRY(dalloc(c, p->d_heap, sizeof(uint2) * (size_t)n));
    launch_make_heap(ptr<uint32_t>(p->count), n, ptr<uint2>(p->d_heap), c->stream);
    CK(c, cudaGetLastError());
    CK(c, cudaMemcpyAsync(storage.data(), p->d_heap.p, sizeof(uint2) * (size_t)n,
                          cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    AdoptedQueue queue(std::move(storage));
    struct Return {
      rip_ctx *c;
      AdoptedQueue &q;
      ~Return() { c->heap_store = q.release(); }
    } give_back{c, queue};
    p->sel_prof[1] += ms_since(t_h0);
    const auto t_p0 = clk::now();
    // The lazy pops of a pick only read the current counts of heap items keyed
    // at least the pick's gain m (keys are stale upper bounds of the counts and
    // m is the largest count).  After each cover the host fetches the counts
    // of the items keyed >= T for a guess T below the previous gain; if one of
    // them still counts >= T, then m >= T and the fetch covers every item the
    // pops can reach.  Otherwise their largest count c is a lower bound of m
    // and a second fetch with T = c is exact.  A pop outside the fetched items
    // (not expected) falls back to the whole count array.
    uint32_t *h_ids = reinterpret_cast<uint32_t *>(hb + 16);
    uint32_t *h_cnt = h_ids + CAND_CAP;
    const uint32_t *d_ids = reinterpret_cast<const uint32_t *>(db + 16);
    uint32_t *d_cnt = reinterpret_cast<uint32_t *>(db + 16) + CAND_CAP;
    CountMap cmap;
    std::vector<uint32_t> stack;
    // First pick: every key is still exact, so only the top is examined.
    bool fresh_all = false, first = true;
    if (!queue.empty()) {
      cmap.reset(1);
      cmap.put(queue.top().first, queue.top().second);
    }
    double ratio = 0.9;   // recent gain ratio g_i / g_{i-1}
    double margin = 0.9;  // guess = margin * ratio: lowered when a guess misses
    auto fetch_all = [&]() -> int {
      CK(c, cudaMemcpyAsync(h_count.p, p->count.p, sizeof(uint32_t) * (size_t)n,
                            cudaMemcpyDeviceToHost, c->stream));
      CK(c, cudaStreamSynchronize(c->stream));
      hcount = static_cast<const uint32_t *>(h_count.p);
      fresh_all = true;
      p->sel_prof[8] += 1;
      return RIP_OK;
    };
    // The next pick's first candidate fetch rides on the cover: its items are
    // collected before the cover is launched (the heap and the last gain are
    // final once the seed is chosen) and, when few enough, the cover kernel's
    // last block gathers their counts and raises a flag the host polls.
    constexpr uint32_t FUSED_MAX = 2048;  // one block reads the ids over the bus
    TRY(dalloc(c, p->cg_done, sizeof(unsigned int)));
    if (!p->cg_done_zeroed) {
      CK(c, cudaMemsetAsync(p->cg_done.p, 0, sizeof(unsigned int), c->stream));
      p->cg_done_zeroed = true;
    }
    volatile unsigned int *h_flag = reinterpret_cast<volatile unsigned int *>(hb);
    unsigned int *d_flag = reinterpret_cast<unsigned int *>(db);
    bool prefetched = false;  // h_ids / h_cnt hold round 0 of the next pick
    uint32_t pre_T = 0, pre_nc = 0;
    auto first_T = [&](uint64_t g_prev) {
      const double guess = p->cand_fixed ? p->cand_fixed / 100.0 : margin * ratio;
      return (uint32_t)std::max<double>(1.0, std::floor((double)g_prev * guess));
    };
    // round-0 collect at T (raised once while too many items qualify);
    // returns the count, CAND_CAP + 1 when still too many
    auto collect0 = [&](uint64_t g_prev, uint32_t &T) -> uint32_t {
      for (;;) {
        const auto t_c0 = clk::now();
        const uint32_t nc = collect_at_least(queue.items(), T, CAND_CAP, h_ids, stack);
        p->sel_prof[10] += ms_since(t_c0);
        if (nc > CAND_CAP && T < g_prev) {
          T = (uint32_t)std::min<uint64_t>(g_prev, (uint64_t)T + (g_prev - T + 1) / 2);
          continue;
        }
        return nc;
      }
    };
    while (out_seeds.size() < k && uncovered != 0) {
      const auto t_g0 = clk::now();
      if (!first) {
        const uint64_t g_prev = out_gains.back();
        uint32_t T = prefetched ? pre_T : first_T(g_prev);
        for (int round = 0;; ++round) {
          uint32_t nc;
          if (round == 0 && prefetched) {
            nc = pre_nc;
          } else if (round == 0) {
            nc = collect0(g_prev, T);
          } else {
            const auto t_c0 = clk::now();
            nc = collect_at_least(queue.items(), T, CAND_CAP, h_ids, stack);
            p->sel_prof[10] += ms_since(t_c0);
          }
          p->sel_prof[11] += 1;
          if (nc > CAND_CAP) {
            TRY(fetch_all());
            break;
          }
          if (!(round == 0 && prefetched)) {
            launch_gather_counts(ptr<uint32_t>(p->count), d_ids, nc, d_cnt, c->stream);
            CK(c, cudaGetLastError());
            CK(c, cudaStreamSynchronize(c->stream));
          }
          p->sel_prof[5] += nc;
          cmap.reset(nc);
          uint32_t mc = 0;
          for (uint32_t i = 0; i < nc; ++i) {
            const uint32_t cv = *reinterpret_cast<volatile uint32_t *>(h_cnt + i);
            cmap.put(h_ids[i], cv);
            mc = std::max(mc, cv);
          }
          if (mc >= T || nc == queue.size()) {
            if (round == 0) margin = std::min(0.97, margin + 0.01);
            break;
          }
          T = std::max<uint32_t>(mc, 1u);  // mc <= m < T: exact next round
          margin = std::max(0.5, margin - 0.05);
        }
        prefetched = false;
      }
      p->sel_prof[7] += ms_since(t_g0);
      HeapItem element;
      const auto t_q0 = clk::now();
      for (;;) {  // getNextSeed, streaming_find_most_influential.h:560-571
        if (queue.empty())
          return set_err(c, RIP_ERR_STATE, "selection heap exhausted");
        element = queue.top();
        uint32_t cur = 0;
        if (fresh_all) {
          cur = hcount[element.first];
        } else if (!cmap.get(element.first, cur)) {
          TRY(fetch_all());
          cur = hcount[element.first];
        }
        queue.pop();
        p->sel_prof[3] += 1;
        if (element.second > cur) {
          element.second = cur;
          queue.push(element);
          continue;
        }
        break;
      }
      p->sel_prof[9] += ms_since(t_q0);
      if (!out_gains.empty() && out_gains.back())
        ratio = std::min(1.0, (double)element.second / (double)out_gains.back());
      uncovered -= element.second;
      out_seeds.push_back(element.first);
      out_gains.push_back(element.second);
      if (out_seeds.size() == k) break;
      const auto t_f0 = clk::now();
      pre_T = first_T(element.second);
      pre_nc = collect0(element.second, pre_T);
      if (pre_nc <= FUSED_MAX) {
        C.vertex = element.first;
        C.blocks = (int)std::min<uint64_t>(max_blocks * 4,
                                           std::max<uint64_t>(1, (element.second + 7) / 8));
        // epochs count per context: the mapped buffer is the context's
        const unsigned int epoch = ++c->cg_epoch;
        *h_flag = 0u;  // the buffer's first word may hold anything before this
        launch_cover_gather(C, d_ids, pre_nc, d_cnt, ptr<unsigned int>(p->cg_done), d_flag,
                            epoch, c->stream);
        CK(c, cudaGetLastError());
        // poll the flag; a stream synchronise covers the (unexpected) case of
        // a flag that does not arrive within a second
        const auto t_w0 = clk::now();
        while (*h_flag != epoch) {
          if (ms_since(t_w0) > 1000.0) {
            CK(c, cudaStreamSynchronize(c->stream));
            if (*h_flag != epoch)
              return set_err(c, RIP_ERR_DEVICE, "pick flag not raised after the cover");
            break;
          }
        }
        std::atomic_thread_fence(std::memory_order_acquire);
        prefetched = true;
      } else {
        TRY(cover(element.first, element.second));
      }
      p->sel_prof[7] += ms_since(t_f0);
      fresh_all = first = false;
    }
    p->sel_prof[2] += ms_since(t_p0);
    p->sel_prof[4] += out_seeds.size();
  } else if (k > 0 && S > 0) {
    // Lowest-id picks entirely on the device: k pick launches (cached chunk
    // maxima, lowest id on ties) and k - 1 cover launches, one read-back.
    const uint32_t chunk = sel_chunk_vertices();
    const uint32_t nchunks = (uint32_t)(((uint64_t)n + chunk - 1) / chunk);
    TRY(dalloc(c, p->s_cmax, (size_t)nchunks * 8));
    TRY(dalloc(c, p->s_dirty, (size_t)nchunks));
    TRY(dalloc(c, p->s_best, (size_t)k * 8 + 256));
    TRY(dalloc(c, p->s_desc, sizeof(SelDesc)));
    TRY(p->h_best.ensure(c, (size_t)k * 8));
    SelDesc d{};
    d.P = p->view();
    d.seg_off[0] = ptr<uint64_t>(p->inv_off);
    d.seg_inv[0] = ptr<uint32_t>(p->inv);
    d.seg_first[0] = 0;
    d.nseg = 1;
    d.S = S;
    d.n = n;
    d.nchunks = nchunks;
    d.k = k;
    d.keep_counts = 1;
    d.count = ptr<uint32_t>(p->count);
    d.cmax = ptr<unsigned long long>(p->s_cmax);
    d.dirty = ptr<uint8_t>(p->s_dirty);
    d.covered = ptr<uint8_t>(p->covered);
    d.best = ptr<unsigned long long>(p->s_best);
    d.done_blocks = reinterpret_cast<unsigned int *>(ptr<uint8_t>(p->s_best) + (size_t)k * 8);
    d.acc = reinterpret_cast<unsigned long long *>(ptr<uint8_t>(p->s_best) + (size_t)k * 8 + 64);
    d.total_elems = P;
    CK(c, cudaMemcpyAsync(p->s_desc.p, &d, sizeof(d), cudaMemcpyHostToDevice, c->stream));
    const SelDesc *dd = ptr<SelDesc>(p->s_desc);
    const int pick_blocks = (int)std::max<uint32_t>(1, std::min<uint32_t>((nchunks + 7) / 8,
                                                                          c->num_sms * 4));
    // The pick loop runs as one CUDA graph, captured once per (k, buffers):
    // kernels read everything through the descriptor; the final copy node
    // holds the best / h_best addresses, so moving those drops the graph.
    SelGraph &sg = p->sel_graph;
    if (sg.exec && (sg.k != k || sg.src != p->s_best.p || sg.dst != p->h_best.p ||
                    sg.desc != p->s_desc.p || sg.pick_blocks != pick_blocks)) {
      cudaGraphExecDestroy(sg.exec);
      sg.exec = nullptr;
    }
    if (!sg.exec) {
      const uint64_t before = launch_counter();
      cudaGraph_t graph = nullptr;
      CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      launch_sel_init(dd, c->num_sms, c->stream);
      for (uint32_t i = 0; i < k; ++i) {
        launch_sel_pick(dd, i, pick_blocks, c->stream);
        if (i + 1 < k) launch_sel_cover(dd, i, max_blocks, c->stream);
      }
      cudaMemcpyAsync(p->h_best.p, p->s_best.p, (size_t)k * 8, cudaMemcpyDeviceToHost,
                      c->stream);
      const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
      sg.nodes = launch_counter() - before;
      uncount_launches(sg.nodes);
      if (ce != cudaSuccess)
        return set_err(c, RIP_ERR_CUDA, "pick graph capture failed: %s", cudaGetErrorString(ce));
      const cudaError_t ie = cudaGraphInstantiate(&sg.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) {
        sg.exec = nullptr;
        return set_err(c, RIP_ERR_CUDA, "pick graph instantiate failed: %s",
                       cudaGetErrorString(ie));
      }
      sg.k = k;
      sg.src = p->s_best.p;
      sg.dst = p->h_best.p;
      sg.desc = p->s_desc.p;
      sg.pick_blocks = pick_blocks;
    }
    CK(c, cudaGraphLaunch(sg.exec, c->stream));
    count_launches(sg.nodes);
    CK(c, cudaStreamSynchronize(c->stream));
    const unsigned long long *hb8 = static_cast<const unsigned long long *>(p->h_best.p);
    for (uint32_t i = 0; i < k && uncovered != 0; ++i) {
      const uint64_t cnt = hb8[i] >> 32;
      if (cnt == 0) break;
      uncovered -= cnt;
      out_seeds.push_back(~(uint32_t)(hb8[i] & 0xFFFFFFFFull));
      out_gains.push_back(cnt);
    }
  }
  CK(c, cudaEventRecord(c->ev1, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  float sms = 0.f;
  cudaEventElapsedTime(&sms, c->ev0, c->ev1);
  p->select_kernel_ms += sms;
  p->have_last_counts = true;
  p->last_counts_on_device = true;  // read back on demand (rip_select_counts)
  for (size_t i = 0; i < out_seeds.size(); ++i) {
    seeds[i] = out_seeds[i];
    if (gains) gains[i] = out_gains[i];
  }
  *num_seeds = (uint32_t)out_seeds.size();
  if (f) *f = S ? double(S - uncovered) / (double)S : 0.0;
  return RIP_OK;
}

// ---------------------------------------------------------------------------
// sharded selection: one shard's part of a pick over sets split between
// devices or processes (MPI FindMostInfluentialSet,
// include/ripples/mpi/find_most_influential.h:449-690).  The caller sums the
// shards' counts into d_sum once (an all-reduce across ranks), then per pick
// either sums the shards' updated counts again (rip_shard_cover) or applies
// every shard's decrement list to d_sum (rip_shard_cover_list +
// rip_shard_apply).  Picks keep the maximum of each kPickChunk counts of
// d_sum; the next pick on the same array recomputes only the chunks that
// rip_shard_apply calls touched since, and all of them when none ran (the
// array may have been rewritten, or be a new one at the same address).
// ---------------------------------------------------------------------------

static int check_sum_buffer(rip_ctx *c, const void *d, const char *where) {
  if (!d || (reinterpret_cast<uintptr_t>(d) & 15))
    return set_err(c, RIP_ERR_INVALID, "%s: device array missing or not 16-byte aligned", where);
  return RIP_OK;
}

static int shard_state(rip_pool *p, const char *where) {
  if (p->shard_sets == kNoShard)
    return set_err(p->ctx, RIP_ERR_STATE, "%s: no rip_shard_begin on this pool's current counts",
                   where);
  return RIP_OK;
}

extern "C" int rip_shard_begin(rip_pool *p, uint64_t num_sets, uint32_t *d_sum,
                               uint64_t *elements) {
  if (!p) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  TRY(check_sum_buffer(c, d_sum, "rip_shard_begin"));
  if (num_sets > p->num_sets)
    return set_err(c, RIP_ERR_INVALID, "rip_shard_begin: %llu sets requested, pool has %llu",
                   (unsigned long long)num_sets, (unsigned long long)p->num_sets);
  if (num_sets >= (1ull << 32))
    return set_err(c, RIP_ERR_LIMIT, "rip_shard_begin: at most 2^32-1 sets");
  CK(c, cudaSetDevice(c->device));
  p->have_last_counts = false;
  uint64_t P = 0;
  TRY(prepare_cover(p, num_sets, &P));
  const uint32_t nchunks = (p->g->n + kPickChunk - 1) / kPickChunk;
  TRY(dalloc(c, p->shard_cmax, (size_t)nchunks * 8));
  TRY(dalloc(c, p->shard_dirty, nchunks));
  TRY(dalloc(c, p->shard_meta, 16));
  TRY(p->h_shard_meta.ensure(c, 16));
  p->shard_sets = num_sets;
  p->shard_elems = P;
  p->shard_cache_ok = false;
  CK(c, cudaMemcpyAsync(d_sum, p->count.p, sizeof(uint32_t) * (size_t)p->g->n,
                        cudaMemcpyDeviceToDevice, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  if (elements) *elements = P;
  return RIP_OK;
}

extern "C" int rip_shard_pick(rip_pool *p, const uint32_t *d_sum, uint32_t *vertex,
                              uint64_t *gain) {
  if (!p || !vertex || !gain) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  TRY(check_sum_buffer(c, d_sum, "rip_shard_pick"));
  TRY(shard_state(p, "rip_shard_pick"));
  CK(c, cudaSetDevice(c->device));
  const uint32_t n = p->g->n;
  const uint32_t nchunks = (n + kPickChunk - 1) / kPickChunk;
  if (!p->shard_cache_ok || d_sum != p->shard_sum)
    CK(c, cudaMemsetAsync(p->shard_dirty.p, 1, nchunks, c->stream));
  unsigned long long *meta = ptr<unsigned long long>(p->shard_meta);
  launch_chunk_pick(d_sum, n, ptr<uint8_t>(p->shard_dirty), ptr<unsigned long long>(p->shard_cmax),
                    meta, c->stream);
  CK(c, cudaGetLastError());
  CK(c, cudaMemcpyAsync(p->h_shard_meta.p, meta, 8, cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  p->shard_sum = d_sum;
  p->shard_cache_ok = false;  // until a rip_shard_apply on this array
  const unsigned long long key = *static_cast<const unsigned long long *>(p->h_shard_meta.p);
  *vertex = ~(uint32_t)(key & 0xFFFFFFFFull);
  *gain = key >> 32;
  return RIP_OK;
}

static CoverLaunch shard_cover_launch(rip_pool *p, uint32_t vertex, uint64_t gain) {
  CoverLaunch C = cover_launch(p);
  C.vertex = vertex;
  C.blocks = (int)std::min<uint64_t>((uint64_t)p->ctx->num_sms * 16,
                                     std::max<uint64_t>(1, (gain + 7) / 8));
  return C;
}

extern "C" int rip_shard_cover(rip_pool *p, uint32_t vertex, uint64_t gain, uint32_t *d_sum) {
  if (!p) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  TRY(check_sum_buffer(c, d_sum, "rip_shard_cover"));
  TRY(shard_state(p, "rip_shard_cover"));
  if (vertex >= p->g->n)
    return set_err(c, RIP_ERR_INVALID, "rip_shard_cover: vertex %u out of range", vertex);
  CK(c, cudaSetDevice(c->device));
  launch_cover(shard_cover_launch(p, vertex, gain), c->stream);
  CK(c, cudaGetLastError());
  CK(c, cudaMemcpyAsync(d_sum, p->count.p, sizeof(uint32_t) * (size_t)p->g->n,
                        cudaMemcpyDeviceToDevice, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  p->shard_cache_ok = false;  // the caller rewrites d_sum with the new sums
  return RIP_OK;
}

extern "C" int rip_shard_cover_list(rip_pool *p, uint32_t vertex, uint64_t gain,
                                    uint32_t *d_dec, uint64_t capacity, uint64_t *count) {
  if (!p || !count) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  TRY(shard_state(p, "rip_shard_cover_list"));
  if (vertex >= p->g->n)
    return set_err(c, RIP_ERR_INVALID, "rip_shard_cover_list: vertex %u out of range", vertex);
  if (capacity < p->shard_elems || (p->shard_elems && !d_dec))
    return set_err(c, RIP_ERR_INVALID,
                   "rip_shard_cover_list: capacity %llu below the shard's %llu elements",
                   (unsigned long long)capacity, (unsigned long long)p->shard_elems);
  CK(c, cudaSetDevice(c->device));
  unsigned long long *cursor = ptr<unsigned long long>(p->shard_meta) + 1;
  CK(c, cudaMemsetAsync(cursor, 0, 8, c->stream));
  if (p->shard_elems) {
    launch_cover_list(shard_cover_launch(p, vertex, gain), d_dec, cursor, c->stream);
    CK(c, cudaGetLastError());
  }
  unsigned long long *h = static_cast<unsigned long long *>(p->h_shard_meta.p);
  CK(c, cudaMemcpyAsync(h + 1, cursor, 8, cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  *count = h[1];
  return RIP_OK;
}

extern "C" int rip_shard_apply(rip_pool *p, uint32_t *d_sum, const uint32_t *d_dec,
                               uint64_t count) {
  if (!p || (count && !d_dec)) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  TRY(check_sum_buffer(c, d_sum, "rip_shard_apply"));
  TRY(shard_state(p, "rip_shard_apply"));
  CK(c, cudaSetDevice(c->device));
  // the cached chunk maxima describe d_sum once this apply's chunks are marked
  p->shard_cache_ok = d_sum == p->shard_sum;
  if (count) {
    const int blocks = (int)std::min<uint64_t>((uint64_t)c->num_sms * 8, (count + 255) / 256);
    launch_apply_decrements(d_sum, p->g->n, d_dec, count, ptr<uint8_t>(p->shard_dirty), blocks,
                            c->stream);
    CK(c, cudaGetLastError());
  }
  CK(c, cudaStreamSynchronize(c->stream));
  return RIP_OK;
}
