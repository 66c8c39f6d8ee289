// server.cu -- IMM queries served in continuous batches.
//
// A server keeps graphs' RRR pools resident between queries: queries on the
// same graph with the same sampler seed draw from one pool, which only grows
// (a later query that needs a larger theta extends it; a smaller one reads a
// prefix).  Every query behaves exactly as a fresh IMM run
// (include/ripples/imm.h:145-260 Sampling, :768-860 IMM): its martingale
// starts at x = 1, round x selects over the first max(theta'_x, previous)
// sets and the final selection over the first theta sets -- sets are pure
// functions of (seed, set id), so a prefix of a shared pool is the pool a
// fresh run would have built, and a query's seeds do not depend on what it
// is batched with.
//
// One tick advances every admitted query by one round:
//   1. admit queued queries while slots are free and their estimated
//      footprint (new sets x mean set size + selection buffers) fits; past
//      a query that must wait, only queries whose resident pool already
//      holds their estimated theta;
//   2. sample every pool's shortfall in one multi-instance launch;
//   3. extend each pool's vertex -> sets index to the sets it now holds;
//   4. run each lowest-id query's round as one CUDA graph on its slot's
//      stream (init, count, k x (pick, cover)), all slots concurrently;
//      reference-heap queries use the host-heap selection;
//   5. advance each query's martingale; finished queries are written back.
#include <deque>
#include <map>
#include <set>

#include "host.h"

namespace {

struct SelSlot {
  cudaStream_t st = nullptr;
  DevMem desc, count, cmax, dirty, covered, best, ctr;
  PinnedMem h_desc, h_best;
  uint32_t nchunk_cap = 0, k_cap = 0;
  uint64_t s_cap = 0;
  // captured rounds by k and grid class: (graph, kernel nodes), oldest first.  Kernels read
  // every buffer through the descriptor, but the final copy node holds the
  // best / h_best addresses: reallocating those drops the captured rounds.
  std::vector<std::pair<uint64_t, std::pair<cudaGraphExec_t, uint64_t>>> execs;
};
constexpr size_t MAX_GRAPHS_PER_SLOT = 8;
// rounds over more elements than this run on full-occupancy grids
constexpr double WIDE_ROUND_ELEMENTS = 64.0 * 1024 * 1024;
// queued queries looked at per tick for admission
constexpr size_t MAX_ADMISSION_SCAN = 1024;

struct Active {
  rip_imm_query *q = nullptr;
  rip_pool *pool = nullptr;
  int slot = -1;
  int phase = 0;  // 0 estimating theta, 1 final selection
  int64_t x = 1;
  uint64_t n = 0;
  double lp = 0, epsP = 0, LB = 0;
  uint64_t theta = 0;
  uint64_t fresh = 0;  // sets a fresh run would hold before this round
  uint64_t S = 0;      // this round's selection prefix
  uint64_t delta = 0;  // sets a fresh run would sample this round
  uint64_t footprint = 0;
  bool stalled = false;  // this tick: its pool could not grow; retried next tick
  clk::time_point t_sub, t_start, t_round;
  rip_imm_record R{};
  std::vector<uint32_t> picks;
  std::vector<uint64_t> gains;
};

}  // namespace

struct rip_server {
  rip_ctx *c = nullptr;
  size_t budget = 0;
  uint32_t max_active = 0;
  std::vector<std::pair<std::pair<rip_graph *, uint64_t>, rip_pool *>> pools;
  std::deque<std::pair<rip_imm_query *, clk::time_point>> queue;
  std::vector<Active> active;
  std::vector<SelSlot> slots;
  std::vector<int> free_slots;
  uint64_t admitted_bytes = 0;
  uint64_t ticks = 0, completed = 0, graph_launches = 0, suspended = 0;
  double tick_ms = 0, sample_ms = 0, index_ms = 0, select_ms = 0;
  std::map<rip_pool *, double> last_lb;  // per pool: LB of the last finished query
  bool pressure = false;  // the last tick had a query waiting for memory
  std::set<rip_imm_query *> resumed;  // suspended once: admitted only in arrival order
};

namespace {

int pool_for(rip_server *s, rip_graph *g, uint64_t seed, rip_pool **out) {
  for (auto &e : s->pools)
    if (e.first.first == g && e.first.second == seed) {
      *out = e.second;
      return RIP_OK;
    }
  rip_pool *p = nullptr;
  TRY(rip_pool_create(s->c, g, &p));
  s->pools.push_back({{g, seed}, p});
  *out = p;
  return RIP_OK;
}

double mean_set_size(rip_pool *p) {
  return p->num_sets ? (double)p->num_elems / (double)p->num_sets : 16.0;
}

// Estimated device bytes a query adds: the sets its theta may add to the pool
// (elements + offsets + index entries) and its selection buffers.
uint64_t estimate_footprint(rip_server *s, rip_imm_query *q, rip_pool *p) {
  const uint64_t n = q->graph->n;
  const double lp = q->l * (1 + 1 / std::log2((double)n));
  uint64_t theta;
  auto it = s->last_lb.find(p);
  if (it != s->last_lb.end() && it->second > 0) {
    theta = rip_theta(q->epsilon, lp, q->k, it->second, n);
  } else {
    // no finished query on this pool yet: a few martingale rounds' worth
    const double epsP = 1.4142135623730951 * q->epsilon;
    theta = 8 * (uint64_t)std::max<int64_t>(0, rip_theta_prime(1, epsP, lp, q->k, n));
  }
  const double per_set = mean_set_size(p) * 8.0 + 12.0 + 1.0;
  const uint64_t grow = theta > p->num_sets ? theta - p->num_sets : 0;
  return (uint64_t)(per_set * (double)grow) + (uint64_t)n * 4 + theta + 8ull * q->k;
}

// The server's pool for (graph, seed) when one is resident, else null.
rip_pool *resident_pool(rip_server *s, rip_graph *g, uint64_t seed) {
  for (auto &e : s->pools)
    if (e.first.first == g && e.first.second == seed) return e.second;
  return nullptr;
}

// True when the pool already holds the theta the query is estimated to need
// (from the lower bound of the last query that finished on the pool).
bool holds_estimate(rip_server *s, rip_imm_query *q, rip_pool *p) {
  auto it = s->last_lb.find(p);
  if (it == s->last_lb.end() || !(it->second > 0)) return false;
  const uint64_t n = q->graph->n;
  const double lp = q->l * (1 + 1 / std::log2((double)n));
  const uint64_t theta = rip_theta(q->epsilon, lp, q->k, it->second, n);
  return theta + theta / 4 <= p->num_sets;  // a margin: the bound came from another k
}

int slot_buffers(rip_server *s, SelSlot &sl, uint32_t nchunks, uint64_t S, uint32_t k) {
  rip_ctx *c = s->c;
  const uint32_t chunk = sel_chunk_vertices();
  if (!sl.st) CK(c, cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking));
  if (!sl.desc.p) {
    TRY(dalloc(c, sl.desc, sizeof(SelDesc)));
    TRY(dalloc(c, sl.ctr, 256));
    CK(c, cudaMemsetAsync(sl.ctr.p, 0, 256, c->stream));
    TRY(sl.h_desc.ensure(c, sizeof(SelDesc)));
  }
  if (nchunks > sl.nchunk_cap) {
    TRY(dalloc(c, sl.count, (size_t)nchunks * chunk * 4));
    TRY(dalloc(c, sl.cmax, (size_t)nchunks * 8));
    TRY(dalloc(c, sl.dirty, (size_t)nchunks));
    sl.nchunk_cap = nchunks;
  }
  const uint64_t sb = ((S + 15) & ~15ull) + 16;
  if (sb > sl.s_cap) {
    const uint64_t cap = std::max<uint64_t>(sb, sl.s_cap * 3 / 2);
    TRY(dalloc(c, sl.covered, cap));
    sl.s_cap = cap;
  }
  if (k > sl.k_cap) {
    // the captured rounds copy best -> h_best through the old buffers: drop them
    for (auto &e : sl.execs) cudaGraphExecDestroy(e.second.first);
    sl.execs.clear();
    TRY(dalloc(c, sl.best, (size_t)k * 8));
    TRY(sl.h_best.ensure(c, (size_t)k * 8));
    sl.k_cap = k;
  }
  return RIP_OK;
}

// The vertex -> sets index of a pool over all the sets it holds: the sets
// added since the last call get a segment of their own (count, scan and
// scatter over that range only); past SEL_MAX_SEGMENTS segments everything
// is re-indexed as one.
int extend_index(rip_pool *p) {
  rip_ctx *c = p->ctx;
  if (p->sv_sets == p->num_sets) return RIP_OK;
  if (p->sv_segs.size() == SEL_MAX_SEGMENTS) {
    for (ServeSegment &g : p->sv_segs) {
      dfree(c, g.off);
      dfree(c, g.inv);
    }
    p->sv_segs.clear();
    p->sv_sets = 0;
  }
  const uint32_t n = p->g->n;
  const uint64_t first = p->sv_sets, S = p->num_sets - first;
  // the pool viewed from set `first` on: set_off / set_len shifted
  DevPool view = p->view();
  view.set_off += first;
  view.set_len += first;
  ServeSegment seg;
  seg.first = first;
  seg.last = p->num_sets;
  TRY(dalloc(c, p->sv_count, sizeof(uint32_t) * (size_t)n));
  CK(c, cudaMemsetAsync(p->sv_count.p, 0, sizeof(uint32_t) * (size_t)n, c->stream));
  launch_count(view, S, ptr<uint32_t>(p->sv_count), c->num_sms * 8, c->stream);
  TRY(dalloc(c, seg.off, sizeof(uint64_t) * ((size_t)n + 1)));
  TRY(dalloc(c, p->sv_cur, sizeof(uint64_t) * ((size_t)n + 1)));
  TRY(dalloc(c, p->sv_sums, sizeof(uint64_t) * scan_block_sums_needed(n)));
  launch_exclusive_scan(ptr<uint32_t>(p->sv_count), ptr<uint64_t>(seg.off), n,
                        ptr<uint64_t>(p->sv_sums), c->stream);
  uint64_t P = 0;
  CK(c, cudaMemcpyAsync(&P, ptr<uint64_t>(seg.off) + n, sizeof(uint64_t),
                        cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaMemcpyAsync(p->sv_cur.p, seg.off.p, sizeof(uint64_t) * ((size_t)n + 1),
                        cudaMemcpyDeviceToDevice, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  int rc = dalloc(c, seg.inv, sizeof(uint32_t) * std::max<uint64_t>(P, 1));
  if (rc != RIP_OK) {
    dfree(c, seg.off);
    return rc;
  }
  launch_build_inverted(view, S, ptr<uint64_t>(p->sv_cur), ptr<uint32_t>(seg.inv),
                        c->num_sms * 8, c->stream, first);
  CK(c, cudaGetLastError());
  p->sv_segs.push_back(seg);
  p->sv_sets = p->num_sets;
  return RIP_OK;
}

// Launches one round of a lowest-id query on its slot: the slot's graph
// (captured once per k) reads the descriptor written just before it.
int launch_round(rip_server *s, Active &a) {
  rip_ctx *c = s->c;
  SelSlot &sl = s->slots[a.slot];
  rip_pool *p = a.pool;
  const uint32_t chunk = sel_chunk_vertices();
  const uint32_t nchunks = (uint32_t)(((uint64_t)a.n + chunk - 1) / chunk);
  const uint32_t k = a.q->k;
  SelDesc *hd = static_cast<SelDesc *>(sl.h_desc.p);
  hd->P = p->view();
  hd->nseg = (uint32_t)p->sv_segs.size();
  for (uint32_t g = 0; g < hd->nseg; ++g) {
    hd->seg_off[g] = ptr<uint64_t>(p->sv_segs[g].off);
    hd->seg_inv[g] = ptr<uint32_t>(p->sv_segs[g].inv);
    hd->seg_first[g] = p->sv_segs[g].first;
  }
  hd->S = a.S;
  hd->n = (uint32_t)a.n;
  hd->nchunks = nchunks;
  hd->k = k;
  hd->keep_counts = 0;
  hd->count = ptr<uint32_t>(sl.count);
  hd->cmax = ptr<unsigned long long>(sl.cmax);
  hd->dirty = ptr<uint8_t>(sl.dirty);
  hd->covered = ptr<uint8_t>(sl.covered);
  hd->best = ptr<unsigned long long>(sl.best);
  hd->done_blocks = ptr<unsigned int>(sl.ctr);
  hd->acc = reinterpret_cast<unsigned long long *>(ptr<uint8_t>(sl.ctr) + 64);
  hd->total_elems = 0;
  CK(c, cudaMemcpyAsync(sl.desc.p, hd, sizeof(SelDesc), cudaMemcpyHostToDevice, sl.st));
  // Rounds over many elements take full-occupancy grids for the count and
  // the covers (one such round fills the device by itself); small rounds
  // keep small grids so that many slots' rounds share the device.  The
  // captured rounds are keyed by k and the grid class.
  const bool wide = mean_set_size(p) * (double)a.S > WIDE_ROUND_ELEMENTS;
  const uint64_t key = (uint64_t)k | (wide ? 1ull << 32 : 0ull);
  size_t gi = 0;
  while (gi < sl.execs.size() && sl.execs[gi].first != key) ++gi;
  if (gi == sl.execs.size()) {
    if (sl.execs.size() == MAX_GRAPHS_PER_SLOT) {
      cudaGraphExecDestroy(sl.execs.front().second.first);
      sl.execs.erase(sl.execs.begin());
    }
    const SelDesc *d = ptr<SelDesc>(sl.desc);
    const int blocks = std::max(8, c->num_sms / 2);
    const int count_blocks = wide ? c->num_sms * 8 : blocks * 2;
    const int cover_blocks = wide ? c->num_sms * 4 : blocks;
    const uint64_t before = launch_counter();
    cudaGraph_t g = nullptr;
    CK(c, cudaStreamBeginCapture(sl.st, cudaStreamCaptureModeThreadLocal));
    launch_sel_init(d, blocks, sl.st);
    launch_sel_count(d, count_blocks, sl.st);
    for (uint32_t i = 0; i < k; ++i) {
      launch_sel_pick(d, i, blocks, sl.st);
      if (i + 1 < k) launch_sel_cover(d, i, cover_blocks, sl.st);
    }
    cudaMemcpyAsync(sl.h_best.p, sl.best.p, (size_t)k * 8, cudaMemcpyDeviceToHost, sl.st);
    const cudaError_t e = cudaStreamEndCapture(sl.st, &g);
    const uint64_t nodes = launch_counter() - before;
    uncount_launches(nodes);
    if (e != cudaSuccess)
      return set_err(c, RIP_ERR_CUDA, "selection graph capture failed: %s",
                     cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess)
      return set_err(c, RIP_ERR_CUDA, "selection graph instantiate failed: %s",
                     cudaGetErrorString(ie));
    sl.execs.push_back({key, {exec, nodes}});
    gi = sl.execs.size() - 1;
  }
  CK(c, cudaGraphLaunch(sl.execs[gi].second.first, sl.st));
  count_launches(sl.execs[gi].second.second);
  s->graph_launches++;
  return RIP_OK;
}

// Decodes the picks of a finished device round: seeds in pick order until
// the first pick that covers nothing (then every set is covered).
void read_round(SelSlot &sl, uint32_t k, std::vector<uint32_t> &seeds,
                std::vector<uint64_t> &gains) {
  const unsigned long long *b = static_cast<const unsigned long long *>(sl.h_best.p);
  seeds.clear();
  gains.clear();
  for (uint32_t i = 0; i < k; ++i) {
    const uint64_t cnt = b[i] >> 32;
    if (cnt == 0) break;
    seeds.push_back(~(uint32_t)(b[i] & 0xFFFFFFFFull));
    gains.push_back(cnt);
  }
}

void finish(rip_server *s, Active &a, int status) {
  rip_imm_query *q = a.q;
  q->status = status;
  if (status == RIP_OK) {
    for (size_t i = 0; i < a.picks.size(); ++i) q->seeds[i] = a.picks[i];
    q->num_seeds = (uint32_t)a.picks.size();
    a.R.total_sets = std::max(a.fresh, a.theta);
    a.R.pool_elements = a.pool->num_elems;
    a.R.rrr_set_bytes = a.pool->num_elems * sizeof(uint32_t);
    a.R.total_ms = ms_since(a.t_start);
    q->record = a.R;
    if (a.LB > 0) s->last_lb[a.pool] = a.LB;
  } else {
    q->num_seeds = 0;
  }
  q->latency_ms = ms_since(a.t_sub);
  q->done = 1;
  s->resumed.erase(q);
  s->completed++;
  s->admitted_bytes -= std::min(s->admitted_bytes, a.footprint);
  if (a.slot >= 0) s->free_slots.push_back(a.slot);
}

// Takes an admitted query back to the end of the queue (it restarts from its
// first round when admitted again) and frees its pool unless another admitted
// query draws from it: the way out when every admitted query waits for memory.
void suspend(rip_server *s, Active &a) {
  s->admitted_bytes -= std::min(s->admitted_bytes, a.footprint);
  if (a.slot >= 0) s->free_slots.push_back(a.slot);
  s->queue.push_back({a.q, a.t_sub});
  s->resumed.insert(a.q);
  s->suspended++;
  for (const Active &b : s->active)
    if (&b != &a && b.pool == a.pool) return;
  for (size_t i = 0; i < s->pools.size(); ++i)
    if (s->pools[i].second == a.pool) {
      s->last_lb.erase(a.pool);
      rip_pool_destroy(a.pool);
      s->pools.erase(s->pools.begin() + i);
      return;
    }
}

// Moves a query past the round just selected (imm.h:214-225 and :233-235).
void advance(Active &a, double f) {
  if (a.phase == 0) {
    const uint32_t r = a.R.num_rounds;
    if (r < RIP_MAX_ROUNDS) {
      a.R.theta_prime_deltas[r] = a.delta;
      a.R.round_select_ms[r] = ms_since(a.t_round);
    }
    a.R.num_rounds++;
    a.fresh = a.S;
    bool done = false;
    if (f >= std::pow(2, -a.x)) {
      a.LB = ((double)a.n * f) / (1 + a.epsP);
      done = true;
    } else {
      ++a.x;
      done = !((double)a.x < std::log2((double)a.n));
    }
    if (done) {
      a.theta = rip_theta(a.q->epsilon, a.lp, a.q->k, a.LB, a.n);
      a.R.theta = a.theta;
      a.R.theta_estimation_ms = ms_since(a.t_start);
      a.phase = 1;
    }
  }
}

bool pool_in_use(rip_server *s, rip_pool *p) {
  for (Active &a : s->active)
    if (a.pool == p) return true;
  return false;
}

// Frees the pools no admitted query draws from (a queued query re-creates
// its pool when admitted): called only when a pool cannot grow.
void evict_idle_pools(rip_server *s) {
  std::vector<std::pair<std::pair<rip_graph *, uint64_t>, rip_pool *>> keep;
  for (auto &e : s->pools) {
    if (pool_in_use(s, e.second)) {
      keep.push_back(e);
    } else {
      s->last_lb.erase(e.second);
      rip_pool_destroy(e.second);
    }
  }
  s->pools.swap(keep);
}

bool out_of_room(int rc) { return rc == RIP_ERR_NOMEM || rc == RIP_ERR_LIMIT; }

// Device bytes held by live allocations (the block cache is reusable).
size_t in_use(rip_ctx *c) { return c->used - std::min(c->used, c->cached); }

}  // namespace

// A graph is going away: its queued and admitted queries end with
// RIP_ERR_STATE and the server's pools on it are destroyed.
void server_graph_gone(rip_ctx *c, rip_graph *g) {
  for (rip_server *s : c->servers) {
    for (SelSlot &sl : s->slots)
      if (sl.st) cudaStreamSynchronize(sl.st);
    std::deque<std::pair<rip_imm_query *, clk::time_point>> q2;
    for (auto &e : s->queue) {
      if (e.first->graph != g) {
        q2.push_back(e);
        continue;
      }
      Active a;
      a.q = e.first;
      a.t_sub = e.second;
      a.t_start = clk::now();
      finish(s, a, RIP_ERR_STATE);
    }
    s->queue.swap(q2);
    std::vector<Active> keep;
    for (Active &a : s->active) {
      if (a.q->graph == g) finish(s, a, RIP_ERR_STATE);
      else keep.push_back(std::move(a));
    }
    s->active.swap(keep);
    std::vector<std::pair<std::pair<rip_graph *, uint64_t>, rip_pool *>> pk;
    for (auto &e : s->pools) {
      if (e.first.first == g) {
        s->last_lb.erase(e.second);
        rip_pool_destroy(e.second);
      } else {
        pk.push_back(e);
      }
    }
    s->pools.swap(pk);
  }
}

extern "C" int rip_server_create(rip_ctx *c, size_t footprint_budget, uint32_t max_active,
                                 rip_server **out) {
  if (!c || !out || max_active == 0) return set_err(c, RIP_ERR_INVALID, "rip_server_create: bad arguments");
  rip_server *s = new rip_server();
  s->c = c;
  s->budget = footprint_budget ? footprint_budget : c->budget / 2;
  s->max_active = max_active;
  s->slots.resize(max_active);
  for (int i = (int)max_active - 1; i >= 0; --i) s->free_slots.push_back(i);
  c->servers.push_back(s);
  *out = s;
  return RIP_OK;
}

extern "C" int rip_server_destroy(rip_server *s) {
  if (!s) return RIP_ERR_INVALID;
  rip_ctx *c = s->c;
  cudaSetDevice(c->device);
  for (SelSlot &sl : s->slots) {
    if (sl.st) cudaStreamSynchronize(sl.st);
    for (auto &e : sl.execs) cudaGraphExecDestroy(e.second.first);
    DevMem *m[] = {&sl.desc, &sl.count, &sl.cmax, &sl.dirty, &sl.covered, &sl.best, &sl.ctr};
    for (DevMem *x : m) dfree(c, *x);
    if (sl.st) cudaStreamDestroy(sl.st);
  }
  for (auto &e : s->pools) rip_pool_destroy(e.second);
  c->servers.erase(std::find(c->servers.begin(), c->servers.end(), s));
  delete s;
  return RIP_OK;
}

extern "C" int rip_server_submit(rip_server *s, rip_imm_query *q) {
  if (!s || !q) return RIP_ERR_INVALID;
  q->done = 0;
  q->status = RIP_OK;
  q->num_seeds = 0;
  q->f = 0;
  q->queue_ms = q->latency_ms = 0;
  std::memset(&q->record, 0, sizeof(q->record));
  s->queue.push_back({q, clk::now()});
  return RIP_OK;
}

extern "C" int rip_server_pending(const rip_server *s, uint32_t *active, uint32_t *queued) {
  if (!s) return RIP_ERR_INVALID;
  if (active) *active = (uint32_t)s->active.size();
  if (queued) *queued = (uint32_t)s->queue.size();
  return RIP_OK;
}

extern "C" int rip_server_stats(const rip_server *s, uint64_t out[10]) {
  if (!s || !out) return RIP_ERR_INVALID;
  out[0] = s->ticks;
  out[1] = s->completed;
  out[2] = s->graph_launches;
  out[3] = (uint64_t)s->pools.size();
  out[4] = s->admitted_bytes;
  out[5] = (uint64_t)(s->tick_ms * 1000.0);
  out[6] = s->suspended;
  out[7] = (uint64_t)(s->sample_ms * 1000.0);
  out[8] = (uint64_t)(s->index_ms * 1000.0);
  out[9] = (uint64_t)(s->select_ms * 1000.0);
  return RIP_OK;
}

extern "C" int rip_server_tick(rip_server *s, uint32_t *completed) {
  if (!s) return RIP_ERR_INVALID;
  rip_ctx *c = s->c;
  CK(c, cudaSetDevice(c->device));
  const auto t_tick = clk::now();
  uint32_t done_now = 0;
  // 1. admission, in arrival order.  Once a query has to wait (no room for
  // its pool to grow), later queries are still admitted when their pool is
  // resident and already holds the theta their estimate asks for: they add
  // selection buffers only, so they cannot delay the waiting query's growth.
  // Not while the last tick had a query waiting for memory: the waiting
  // queries drain first (suspension frees pools), so a suspended query is
  // not taken straight back.
  bool head_waits = false;
  size_t scanned = 0;
  for (auto it = s->queue.begin();
       it != s->queue.end() && !s->free_slots.empty() && scanned < MAX_ADMISSION_SCAN;
       ++scanned) {
    rip_imm_query *q = it->first;
    const bool bad = !q->graph || q->graph->ctx != c || q->k == 0 || !q->seeds ||
                     !(q->epsilon > 0) || q->graph->n < 2 ||
                     (q->tiebreak != RIP_TIE_LOWEST_ID && q->tiebreak != RIP_TIE_REF_HEAP);
    Active a;
    a.q = q;
    a.t_sub = it->second;
    if (bad) {
      it = s->queue.erase(it);
      a.t_start = clk::now();
      finish(s, a, RIP_ERR_INVALID);
      ++done_now;
      continue;
    }
    rip_pool *p = nullptr;
    uint64_t fp = 0;
    if (!head_waits) {
      // admitted while its estimated footprint fits and the device is not
      // already mostly in use (resident pools stay: later queries reuse
      // them); always when nothing else is admitted
      if (!s->active.empty() && in_use(c) > c->budget / 20 * 17) {
        head_waits = true;
        ++it;
        continue;
      }
      TRY(pool_for(s, q->graph, q->seed, &p));
      if (p->num_sets == 0) {  // a first slice of the pool measures its mean set size
        const int r = rip_sample(p, q->seed, 256, RIP_SAMPLER_AUTO);
        if (out_of_room(r) && !s->active.empty()) {
          head_waits = true;
          ++it;
          continue;
        }
        if (r != RIP_OK && !out_of_room(r)) return r;
      }
      fp = estimate_footprint(s, q, p);
      if (!s->active.empty() && s->admitted_bytes + fp > s->budget) {
        head_waits = true;
        ++it;
        continue;
      }
    } else {
      if (s->pressure) break;
      p = resident_pool(s, q->graph, q->seed);
      if (!p || s->resumed.count(q) || !holds_estimate(s, q, p)) {
        ++it;
        continue;
      }
      fp = estimate_footprint(s, q, p);
      if (s->admitted_bytes + fp > s->budget) {
        ++it;
        continue;
      }
    }
    it = s->queue.erase(it);
    a.pool = p;
    a.slot = s->free_slots.back();
    s->free_slots.pop_back();
    a.footprint = fp;
    s->admitted_bytes += fp;
    a.n = q->graph->n;
    a.lp = q->l * (1 + 1 / std::log2((double)a.n));
    a.epsP = 1.4142135623730951 * q->epsilon;
    a.t_start = clk::now();
    q->queue_ms = std::chrono::duration<double, std::milli>(a.t_start - a.t_sub).count();
    if (!(1.0 < std::log2((double)a.n))) {  // no estimation round (imm.h:179)
      a.theta = rip_theta(q->epsilon, a.lp, q->k, 0.0, a.n);
      a.phase = 1;
    }
    s->active.push_back(std::move(a));
  }
  if (s->active.empty()) {
    if (completed) *completed = done_now;
    return RIP_OK;
  }
  // 2. this round's prefixes and the pools' shortfalls, sampled in one launch
  std::vector<rip_pool *> mp;
  std::vector<uint64_t> need;
  for (Active &a : s->active) {
    if (a.phase == 0) {
      const int64_t tp = rip_theta_prime(a.x, a.epsP, a.lp, a.q->k, a.n);
      const uint64_t t = (uint64_t)std::max<int64_t>(tp, 0);
      a.delta = t > a.fresh ? t - a.fresh : 0;
      a.S = std::max(a.fresh, t);
    } else {
      a.delta = a.theta > a.fresh ? a.theta - a.fresh : 0;
      a.S = a.theta;
    }
    size_t i = 0;
    while (i < mp.size() && mp[i] != a.pool) ++i;
    if (i == mp.size()) {
      mp.push_back(a.pool);
      need.push_back(0);
    }
    need[i] = std::max(need[i], a.S);
  }
  // A round whose pool would not fit the device even with nothing else on it
  // ends its query now (RIP_ERR_LIMIT) instead of waiting for memory.
  {
    std::vector<Active> keep;
    for (Active &a : s->active) {
      const double per_set = mean_set_size(a.pool) * 8.0 + 13.0;
      const double bytes = per_set * (double)a.S + (double)a.n * 96.0;
      if (bytes > 0.9 * (double)c->budget) {
        finish(s, a, RIP_ERR_LIMIT);
        ++done_now;
      } else {
        keep.push_back(std::move(a));
      }
    }
    s->active.swap(keep);
    mp.clear();
    need.clear();
    for (Active &a : s->active) {
      size_t i = 0;
      while (i < mp.size() && mp[i] != a.pool) ++i;
      if (i == mp.size()) {
        mp.push_back(a.pool);
        need.push_back(0);
      }
      need[i] = std::max(need[i], a.S);
    }
  }
  std::vector<rip_pool *> sp;
  std::vector<uint64_t> sseed, scnt;
  for (size_t i = 0; i < mp.size(); ++i)
    if (need[i] > mp[i]->num_sets) {
      sp.push_back(mp[i]);
      for (auto &e : s->pools)
        if (e.second == mp[i]) sseed.push_back(e.first.second);
      scnt.push_back(need[i] - mp[i]->num_sets);
    }
  const auto t_gen = clk::now();
  if (!sp.empty()) {
    const int rc = rip_sample_multi(c, sp.data(), sseed.data(), scnt.data(), (uint32_t)sp.size());
    if (out_of_room(rc)) {
      // Free idle pools, then grow the pools one by one.  A pool grows to its
      // largest remaining request; when that does not fit, the queries asking
      // for it wait for the next tick (other queries' pools may become idle
      // and be freed by then) and the next largest request is tried.
      evict_idle_pools(s);
      for (size_t i = 0; i < sp.size(); ++i) {
        for (;;) {
          uint64_t target = 0;
          for (Active &a : s->active)
            if (a.pool == sp[i] && !a.stalled) target = std::max(target, a.S);
          const uint64_t cnt = target > sp[i]->num_sets ? target - sp[i]->num_sets : 0;
          const int r = cnt ? rip_sample_multi(c, &sp[i], &sseed[i], &cnt, 1) : RIP_OK;
          if (!out_of_room(r)) {
            TRY(r);
            break;
          }
          for (Active &a : s->active)
            if (a.pool == sp[i] && a.S == target) a.stalled = true;
        }
      }
    } else {
      TRY(rc);
    }
  }
  const double gen_ms = ms_since(t_gen);
  s->sample_ms += gen_ms;
  for (Active &a : s->active) {
    a.t_round = clk::now();
    if (a.phase == 0 && a.R.num_rounds < RIP_MAX_ROUNDS)
      a.R.round_generate_ms[a.R.num_rounds] = a.delta ? gen_ms : 0.0;
    if (a.phase == 1) a.R.generate_ms = a.delta ? gen_ms : 0.0;
  }
  // 3. indexes, 4. selections
  const auto t_idx = clk::now();
  bool any_dev = false;
  for (Active &a : s->active) {
    if (a.stalled || a.q->tiebreak != RIP_TIE_LOWEST_ID) continue;
    const int r = extend_index(a.pool);
    if (out_of_room(r)) {
      for (Active &b : s->active)
        if (b.pool == a.pool) b.stalled = true;
      continue;
    }
    TRY(r);
    any_dev = true;
  }
  if (any_dev) {
    const uint32_t chunk = sel_chunk_vertices();
    for (Active &a : s->active) {
      if (a.stalled || a.q->tiebreak != RIP_TIE_LOWEST_ID) continue;
      const int r = slot_buffers(s, s->slots[a.slot], (uint32_t)((a.n + chunk - 1) / chunk),
                                 a.S, a.q->k);
      if (out_of_room(r)) a.stalled = true;
      else TRY(r);
    }
    CK(c, cudaStreamSynchronize(c->stream));
    s->index_ms += ms_since(t_idx);
    for (Active &a : s->active)
      if (!a.stalled && a.q->tiebreak == RIP_TIE_LOWEST_ID) TRY(launch_round(s, a));
  }
  std::vector<double> fs(s->active.size(), 0.0);
  for (size_t i = 0; i < s->active.size(); ++i) {
    Active &a = s->active[i];
    if (a.stalled || a.q->tiebreak != RIP_TIE_REF_HEAP) continue;
    a.picks.assign(a.q->k, 0);
    uint32_t ns = 0;
    TRY(rip_select(a.pool, a.S, a.q->k, RIP_TIE_REF_HEAP, a.picks.data(), nullptr, &ns,
                   &fs[i]));
    a.picks.resize(ns);
  }
  for (size_t i = 0; i < s->active.size(); ++i) {
    Active &a = s->active[i];
    if (a.stalled || a.q->tiebreak != RIP_TIE_LOWEST_ID) continue;
    SelSlot &sl = s->slots[a.slot];
    CK(c, cudaStreamSynchronize(sl.st));
    read_round(sl, a.q->k, a.picks, a.gains);
    uint64_t cov = 0;
    for (uint64_t g : a.gains) cov += g;
    fs[i] = a.S ? (double)cov / (double)a.S : 0.0;
  }
  s->select_ms += ms_since(t_idx);
  // 5. martingale steps, completions.  When every admitted query waited for
  // memory, the one asking for the most sets is suspended (or, alone, ends).
  bool progress = false;
  size_t worst = 0;
  s->pressure = false;
  for (size_t i = 0; i < s->active.size(); ++i) {
    if (!s->active[i].stalled) progress = true;
    else s->pressure = true;
    if (s->active[i].S > s->active[worst].S) worst = i;
  }
  std::vector<Active> keep;
  const size_t n_active = s->active.size();
  for (size_t i = 0; i < s->active.size(); ++i) {
    Active &a = s->active[i];
    if (a.stalled) {
      a.stalled = false;
      if (!progress && i == worst) {
        if (n_active > 1) {
          suspend(s, a);  // frees memory for the others; it runs again later
        } else {
          finish(s, a, RIP_ERR_NOMEM);  // does not fit even alone
          ++done_now;
        }
      } else {
        keep.push_back(std::move(a));
      }
      continue;
    }
    if (a.phase == 1) {
      a.R.select_ms = ms_since(a.t_round);
      a.q->f = fs[i];
      a.R.f = fs[i];
      finish(s, a, RIP_OK);
      ++done_now;
      continue;
    }
    advance(a, fs[i]);
    keep.push_back(std::move(a));
  }
  s->active.swap(keep);
  s->ticks++;
  s->tick_ms += ms_since(t_tick);
  if (completed) *completed = done_now;
  return RIP_OK;
}

extern "C" int rip_imm_batch(rip_ctx *c, rip_imm_query *queries, uint32_t n) {
  if (!c || (n && !queries)) return RIP_ERR_INVALID;
  if (n == 0) return RIP_OK;
  rip_server *s = nullptr;
  TRY(rip_server_create(c, 0, n, &s));
  int rc = RIP_OK;
  for (uint32_t i = 0; i < n && rc == RIP_OK; ++i) rc = rip_server_submit(s, queries + i);
  uint32_t left = n;
  while (rc == RIP_OK && left) {
    uint32_t done = 0;
    rc = rip_server_tick(s, &done);
    left -= std::min(left, done);
  }
  rip_server_destroy(s);
  return rc;
}
