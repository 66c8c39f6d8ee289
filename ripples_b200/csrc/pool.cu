// pool.cu -- RRR pools behind include/ripples_b200.h: growth, export/import,
// the sampler launch / retry / hand-over loop (one set per warp, fused
// multi-colour, heavy sets one CTA each or grid-wide), many pools in one
// launch, tuning knobs and the per-graph autotuner.
#include "host.h"

// ---------------------------------------------------------------------------
// pool
// ---------------------------------------------------------------------------

static int read_meta(rip_pool *p, PoolMeta &m) {
  rip_ctx *c = p->ctx;
  CK(c, cudaMemcpyAsync(&m, p->meta.p, sizeof(PoolMeta), cudaMemcpyDeviceToHost,
                        c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  return RIP_OK;
}

extern "C" int rip_pool_create(rip_ctx *c, rip_graph *g, rip_pool **out) {
  if (!c || !g || !out || g->ctx != c) return set_err(c, RIP_ERR_INVALID, "rip_pool_create: bad arguments");
  CK(c, cudaSetDevice(c->device));
  rip_pool *p = new rip_pool();
  p->ctx = c;
  p->g = g;
  int rc = dalloc(c, p->meta, sizeof(PoolMeta));
  if (rc) {
    delete p;
    return rc;
  }
  cudaMemsetAsync(p->meta.p, 0, sizeof(PoolMeta), c->stream);
  p->giant_min = g->default_giant_min;
  if (g->tuned.set) {
    p->auto_sampler = g->tuned.sampler;
    p->colors = g->tuned.colors;
    p->cap_plain = g->tuned.cap_plain;
    p->cap_fused = g->tuned.cap_fused;
    p->giant_min = g->tuned.giant_min;
    p->plain_occupancy = g->tuned.plain_occupancy;
    p->big_threads = g->tuned.big_threads;
  }
  c->pools.push_back(p);
  *out = p;
  return RIP_OK;
}

extern "C" int rip_pool_destroy(rip_pool *p) {
  if (!p) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  DevMem *all[] = {&p->vtx,     &p->set_off,   &p->set_len,  &p->meta,
                   &p->scratch, &p->ids_a,     &p->ids_b,    &p->f_vis,
                   &p->f_pend,  &p->f_flag,    &p->f_log,    &p->f_order,
                   &p->b_scratch, &p->b_ids,   &p->d_heap,
                   &p->g_state, &p->g_lists,   &p->g_col,
                   &p->s_cmax,  &p->s_dirty,   &p->s_best,   &p->s_desc,

                   &p->count,   &p->inv_off,   &p->inv_cur,  &p->inv,
                   &p->covered, &p->shard_cmax, &p->shard_dirty, &p->shard_meta,
                   &p->scan_sums, &p->sv_count, &p->sv_cur, &p->sv_sums};
  for (ServeSegment &g : p->sv_segs) {
    dfree(c, g.off);
    dfree(c, g.inv);
  }
  for (DevMem *m : all) dfree(c, *m);
  if (p->sel_graph.exec) cudaGraphExecDestroy(p->sel_graph.exec);
  erase_ptr(c->pools, p);
  delete p;
  return RIP_OK;
}

extern "C" int rip_pool_clear(rip_pool *p) {
  if (!p) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  CK(c, cudaMemsetAsync(p->meta.p, 0, sizeof(PoolMeta), c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  p->num_sets = p->num_elems = 0;
  p->kernel_ms = p->select_kernel_ms = 0.0;
  for (double &x : p->sel_prof) x = 0.0;
  p->kernel_launches = 0;
  p->have_last_counts = false;
  p->shard_sets = kNoShard;
  for (ServeSegment &g : p->sv_segs) {
    dfree(c, g.off);
    dfree(c, g.inv);
  }
  p->sv_segs.clear();
  p->sv_sets = 0;
  return RIP_OK;
}

extern "C" int rip_pool_info(const rip_pool *p, uint64_t *num_sets,
                             uint64_t *num_elements) {
  if (!p) return RIP_ERR_INVALID;
  if (num_sets) *num_sets = p->num_sets;
  if (num_elements) *num_elements = p->num_elems;
  return RIP_OK;
}

extern "C" int rip_pool_stats(rip_pool *p, uint64_t stats[8]) {
  if (!p || !stats) return RIP_ERR_INVALID;
  PoolMeta m;
  TRY(read_meta(p, m));
  for (int i = 0; i < 8; ++i) stats[i] = m.stats[i];
  return RIP_OK;
}

// Kernel-time accounting of the sampler launches (CUDA events on the stream).
extern "C" int rip_pool_timing(rip_pool *p, double *sample_kernel_ms,
                               uint64_t *launches, double *select_kernel_ms) {
  if (!p) return RIP_ERR_INVALID;
  if (sample_kernel_ms) *sample_kernel_ms = p->kernel_ms;
  if (launches) *launches = p->kernel_launches;
  if (select_kernel_ms) *select_kernel_ms = p->select_kernel_ms;
  return RIP_OK;
}

static int ensure_sets(rip_pool *p, uint64_t need) {
  rip_ctx *c = p->ctx;
  if (need <= p->set_cap) return RIP_OK;
  uint64_t nc = std::max<uint64_t>(need, std::max<uint64_t>(p->set_cap * 2, 4096));
  TRY(dgrow(c, p->set_off, nc * sizeof(uint64_t), p->num_sets * sizeof(uint64_t)));
  TRY(dgrow(c, p->set_len, nc * sizeof(uint32_t), p->num_sets * sizeof(uint32_t)));
  p->set_cap = nc;
  return RIP_OK;
}

static int ensure_elems(rip_pool *p, uint64_t need) {
  rip_ctx *c = p->ctx;
  if (need <= p->cap) return RIP_OK;
  uint64_t nc = std::max<uint64_t>(need, std::max<uint64_t>(p->cap + p->cap / 2, 1 << 16));
  TRY(dgrow(c, p->vtx, nc * sizeof(uint32_t), p->num_elems * sizeof(uint32_t)));
  p->cap = nc;
  return RIP_OK;
}

// Partitions the sampler scratch into `warps` x (bitmap + queue of qcap).  LT
// walks need no bitmap (revisits are found in the queue).
static uint64_t scratch_bm_words(const rip_pool *p) {
  return p->g->model == RIP_MODEL_LT ? 0 : (((uint64_t)p->g->n + 31) / 32 + 7) & ~7ull;
}

static int ensure_scratch(rip_pool *p, uint32_t warps, uint32_t qcap) {
  rip_ctx *c = p->ctx;
  const uint64_t bm_words = scratch_bm_words(p);
  const uint64_t per = bm_words * 4 + (uint64_t)qcap * 4;
  const uint64_t bytes = per * warps;
  if (p->scratch.p && p->bm_words == bm_words && p->qcap == qcap &&
      p->warps == warps)
    return RIP_OK;
  TRY(dalloc(c, p->scratch, bytes));
  // bitmaps must start all-zero; queue contents are don't-care
  if (bm_words) CK(c, cudaMemsetAsync(p->scratch.p, 0, bm_words * 4 * warps, c->stream));
  p->bm_words = bm_words;
  p->qcap = qcap;
  p->warps = warps;
  return RIP_OK;
}

static uint32_t default_warps(rip_pool *p, uint32_t qcap) {
  rip_ctx *c = p->ctx;
  const uint64_t bm_bytes = scratch_bm_words(p) * 4;
  const uint64_t per = bm_bytes + (uint64_t)qcap * 4;
  // LT walks: 32 resident warps per SM -- a launch lasts about as long as its
  // longest walk either way (a chain of dependent loads), and half the SMs'
  // warp slots stay free for other queries' pick launches; IC: 32, or 40
  // with the register-capped kernel variant
  uint64_t want = (uint64_t)c->num_sms *
                  (p->g->model == RIP_MODEL_LT ? 32 : p->plain_occupancy == 5 ? 40 : 32);
  size_t avail = c->budget > c->used ? c->budget - c->used : 0;
  uint64_t fit = (avail / 4) / per;  // scratch gets at most a quarter
  uint64_t w = std::min<uint64_t>(want, std::max<uint64_t>(fit, 8));
  return (uint32_t)std::max<uint64_t>(8, w & ~7ull);
}

static int sample_fused(rip_pool *p, uint64_t seed, uint64_t first, uint32_t count);
static int sample_big(rip_pool *p, uint64_t seed, uint64_t first,
                      const std::vector<uint32_t> &ids);

// One set per warp (IC BFS / LT walk).  IC sets whose edge work exceeds the
// per-set cap are handed to the CTA-per-set sampler; sets that outgrow the warp
// queues or the pool are re-run with larger buffers.
static int sample_warp_per_set(rip_pool *p, uint64_t seed, uint64_t first,
                               uint32_t count, const std::vector<uint32_t> *only) {
  rip_ctx *c = p->ctx;
  rip_graph *g = p->g;
  uint32_t qcap = std::min<uint32_t>(g->n, 1u << 14);
  if (p->qcap > qcap && p->scratch.p) qcap = p->qcap;
  uint32_t warps = p->warps && p->qcap == qcap ? p->warps : default_warps(p, qcap);
  TRY(ensure_scratch(p, warps, qcap));
  TRY(dalloc(c, p->ids_a, sizeof(uint32_t) * (size_t)count));
  TRY(dalloc(c, p->ids_b, sizeof(uint32_t) * (size_t)count));
  PoolMeta *dm = p->dmeta();
  const uint32_t *ids = nullptr;
  uint32_t todo = count;
  if (only) {  // run just these indices (relative to first)
    todo = (uint32_t)only->size();
    if (todo == 0) return RIP_OK;
    CK(c, cudaMemcpyAsync(p->ids_b.p, only->data(), sizeof(uint32_t) * todo,
                          cudaMemcpyHostToDevice, c->stream));
    ids = ptr<uint32_t>(p->ids_b);
  }
  const bool capped = g->model == RIP_MODEL_IC && p->cap_plain != 0;
  std::vector<uint32_t> big, retry;
  for (int attempt = 0; attempt < 64; ++attempt) {
    CK(c, cudaMemsetAsync(&dm->fail_count, 0, sizeof(unsigned int), c->stream));
    CK(c, cudaMemsetAsync(&dm->next, 0, sizeof(unsigned int), c->stream));
    CK(c, cudaMemsetAsync(&dm->first_bad, 0xFF, sizeof(unsigned long long), c->stream));
    SampleLaunch L;
    L.G = g->view();
    L.P = p->view();
    L.key = make_key(seed);
    L.first = first;
    L.count = todo;
    L.ids = ids;
    L.next = &dm->next;
    L.bitmaps = ptr<uint32_t>(p->scratch);
    L.bm_words = p->bm_words;
    L.queues = ptr<uint32_t>(p->scratch) + (size_t)p->bm_words * p->warps;
    L.qcap = p->qcap;
    L.work_cap = capped ? p->cap_plain : 0;
    L.F = FailList{ptr<uint32_t>(p->ids_a), &dm->fail_count, &dm->first_bad};
    L.st = Stats{dm->stats};
    L.threads = 256;
    L.occupancy = p->plain_occupancy;
    const uint32_t active = std::min<uint32_t>(p->warps, todo);
    L.blocks = (int)std::max<uint32_t>(1, (active + 7) / 8);
    CK(c, cudaEventRecord(c->ev0, c->stream));
    if (g->model == RIP_MODEL_IC)
      launch_ic_plain(L, c->stream);
    else
      launch_lt_walk(L, c->stream);
    CK(c, cudaGetLastError());
    CK(c, cudaEventRecord(c->ev1, c->stream));
    PoolMeta m;
    TRY(read_meta(p, m));
    float kms = 0.f;
    cudaEventElapsedTime(&kms, c->ev0, c->ev1);
    p->kernel_ms += kms;
    p->kernel_launches++;
    if (m.fail_count == 0) {
      p->num_elems = m.cursor;
      break;
    }
    // Roll the bump pointer back to the end of the last stored set.
    unsigned long long cur = std::min<unsigned long long>(m.cursor, m.first_bad);
    CK(c, cudaMemcpyAsync(&dm->cursor, &cur, sizeof(cur), cudaMemcpyHostToDevice, c->stream));
    p->num_elems = cur;
    std::vector<uint32_t> failed(m.fail_count);
    CK(c, cudaMemcpyAsync(failed.data(), p->ids_a.p, sizeof(uint32_t) * m.fail_count,
                          cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    retry.clear();
    bool queue_overflow = false;
    for (uint32_t f : failed) {
      if (f & FAIL_BIG) big.push_back(f & ~FAIL_BIG);
      else retry.push_back(f);
    }
    if (retry.empty()) break;
    if (m.first_bad != ~0ull) {
      double mean = m.stats[2] ? (double)m.stats[3] / (double)m.stats[2] : 16.0;
      uint64_t need = cur + (uint64_t)(mean * 2.0 * retry.size()) + 4096;
      TRY(ensure_elems(p, std::max<uint64_t>(need, p->cap * 2)));
    } else {
      queue_overflow = true;
    }
    if (queue_overflow && p->qcap < g->n) {
      // widen the queues (fewer warps) so the worst case, a set holding every
      // vertex, fits eventually
      uint32_t nq = (uint32_t)std::min<uint64_t>(g->n, (uint64_t)p->qcap * 4);
      uint32_t nw = std::max<uint32_t>(8, std::min(default_warps(p, nq), p->warps));
      TRY(ensure_scratch(p, nw, nq));
    }
    CK(c, cudaMemcpyAsync(p->ids_b.p, retry.data(), sizeof(uint32_t) * retry.size(),
                          cudaMemcpyHostToDevice, c->stream));
    ids = ptr<uint32_t>(p->ids_b);
    todo = (uint32_t)retry.size();
    if (attempt == 63) return set_err(c, RIP_ERR_DEVICE, "sampler did not converge after retries");
  }
  if (!big.empty()) {
    std::sort(big.begin(), big.end());
    TRY(sample_big(p, seed, first, big));
  }
  return RIP_OK;
}

// ---------------------------------------------------------------------------
// heavy-tail IC sets: one CTA per set
// ---------------------------------------------------------------------------
static int ensure_big_scratch(rip_pool *p, uint32_t slots, uint32_t qcap) {
  rip_ctx *c = p->ctx;
  const uint64_t bm_words = (((uint64_t)p->g->n + 31) / 32 + 7) & ~7ull;
  if (p->b_scratch.p && p->b_slots == slots && p->b_qcap == qcap) return RIP_OK;
  const size_t bytes = (size_t)slots * (bm_words * 4 + (size_t)qcap * 4);
  TRY(dalloc(c, p->b_scratch, bytes));
  CK(c, cudaMemsetAsync(p->b_scratch.p, 0, (size_t)slots * bm_words * 4, c->stream));
  p->b_slots = slots;
  p->b_qcap = qcap;
  return RIP_OK;
}

// Grows the sets first+ids[i] 64*cw at a time, each batch by the whole grid
// (kernels_giant.cu): one host round trip per BFS level for the frontier size.
static int sample_giant(rip_pool *p, uint64_t seed, uint64_t first,
                        const std::vector<uint32_t> &ids) {
  rip_ctx *c = p->ctx;
  rip_graph *g = p->g;
  const size_t n = g->n;
  constexpr uint32_t MAXCOL = 256, CWMAX = 4;
  // state: vis | pend (n * 4 words each) | pflag (n); zero between batches
  const size_t st_bytes = n * CWMAX * 8 * 2 + n * 4;
  if (!p->g_state.p || p->g_state.bytes < st_bytes) {
    TRY(dalloc(c, p->g_state, st_bytes));
    CK(c, cudaMemsetAsync(p->g_state.p, 0, st_bytes, c->stream));
  }
  // lists: front | next | touched | ng (n u32 each) | masks (n * 4 words) |
  // goff (n + 1) | scan sums
  const size_t sums = scan_block_sums_needed((uint32_t)n);
  const size_t li_bytes = n * 4 * 4 + n * CWMAX * 8 + (n + 1) * 8 + sums * 8;
  TRY(dalloc(c, p->g_lists, li_bytes));
  // per colour: set ids (u64) | starts (u64) | sizes | fill (u32) | counters
  TRY(dalloc(c, p->g_col, MAXCOL * 24 + 256));
  uint8_t *st = ptr<uint8_t>(p->g_state), *li = ptr<uint8_t>(p->g_lists),
          *co = ptr<uint8_t>(p->g_col);
  GiantLaunch L;
  L.G = g->view();
  L.P = p->view();
  L.key = make_key(seed);
  L.vis = reinterpret_cast<uint64_t *>(st);
  L.pend = reinterpret_cast<uint64_t *>(st + n * CWMAX * 8);
  L.pflag = reinterpret_cast<uint32_t *>(st + n * CWMAX * 16);
  L.front = reinterpret_cast<uint32_t *>(li);
  L.front_next = reinterpret_cast<uint32_t *>(li + n * 4);
  L.touched = reinterpret_cast<uint32_t *>(li + n * 8);
  L.ng = reinterpret_cast<uint32_t *>(li + n * 12);
  L.masks = reinterpret_cast<uint64_t *>(li + n * 16);
  L.goff = reinterpret_cast<uint64_t *>(li + n * 16 + n * CWMAX * 8);
  uint64_t *d_sums = reinterpret_cast<uint64_t *>(li + n * 16 + n * CWMAX * 8 + (n + 1) * 8);
  L.set_ids = reinterpret_cast<const uint64_t *>(co);
  L.starts = reinterpret_cast<unsigned long long *>(co + MAXCOL * 8);
  L.sizes = reinterpret_cast<uint32_t *>(co + MAXCOL * 16);
  L.fill = reinterpret_cast<uint32_t *>(co + MAXCOL * 20);
  L.ctr = reinterpret_cast<unsigned int *>(co + MAXCOL * 24);
  L.stats = p->dmeta()->stats;
  const int blocks = c->num_sms * 8;
  std::vector<uint64_t> sid(MAXCOL);
  std::vector<uint32_t> sizes(MAXCOL);
  std::vector<unsigned long long> starts(MAXCOL);
  // A batch left unfinished by an error would leave masks and level stamps
  // set: every error return clears the whole state first.
  struct Clear {
    rip_ctx *c;
    void *p;
    size_t bytes;
    bool armed = true;
    ~Clear() {
      if (armed) {
        cudaMemsetAsync(p, 0, bytes, c->stream);
        cudaStreamSynchronize(c->stream);
      }
    }
  } clear_on_error{c, p->g_state.p, st_bytes};
  for (size_t b0 = 0; b0 < ids.size(); b0 += MAXCOL) {
    const uint32_t ncol = (uint32_t)std::min<size_t>(MAXCOL, ids.size() - b0);
    const int cw = ncol <= 64 ? 1 : ncol <= 128 ? 2 : 4;
    L.ncol = ncol;
    for (uint32_t i = 0; i < ncol; ++i) sid[i] = first + ids[b0 + i];
    CK(c, cudaEventRecord(c->ev0, c->stream));
    CK(c, cudaMemcpyAsync(co, sid.data(), 8 * ncol, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemsetAsync(L.ctr, 0, 16, c->stream));
    CK(c, cudaMemsetAsync(L.sizes, 0, 4 * MAXCOL, c->stream));
    launch_giant(0, cw, L, 0, 0, 1, c->stream);
    unsigned int hc[2] = {0, 0};
    CK(c, cudaMemcpyAsync(hc, L.ctr, 8, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    uint32_t nf = hc[0];
    for (uint32_t level = 1; nf > 0; ++level) {
      launch_giant(1, cw, L, nf, level, blocks, c->stream);
      launch_exclusive_scan(L.ng, L.goff, nf, d_sums, c->stream);
      CK(c, cudaMemsetAsync(L.ctr, 0, 4, c->stream));
      launch_giant(2, cw, L, nf, level, blocks, c->stream);
      CK(c, cudaGetLastError());
      CK(c, cudaMemcpyAsync(hc, L.ctr, 8, cudaMemcpyDeviceToHost, c->stream));
      CK(c, cudaStreamSynchronize(c->stream));
      std::swap(L.front, L.front_next);
      nf = hc[0];
    }
    const uint32_t nt = hc[1];
    launch_giant(3, cw, L, nt, 0, blocks, c->stream);
    CK(c, cudaMemcpyAsync(sizes.data(), L.sizes, 4 * ncol, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    uint64_t total = 0;
    for (uint32_t i = 0; i < ncol; ++i) {
      starts[i] = p->num_elems + total;
      total += sizes[i];
    }
    TRY(ensure_elems(p, p->num_elems + total));
    L.P = p->view();
    CK(c, cudaMemcpyAsync(L.starts, starts.data(), 8 * ncol, cudaMemcpyHostToDevice,
                          c->stream));
    launch_giant(5, cw, L, 0, 0, 1, c->stream);
    launch_giant(4, cw, L, nt, 0, blocks, c->stream);
    CK(c, cudaGetLastError());
    const unsigned long long cur = p->num_elems + total;
    CK(c, cudaMemcpyAsync(&p->dmeta()->cursor, &cur, sizeof(cur), cudaMemcpyHostToDevice,
                          c->stream));
    CK(c, cudaEventRecord(c->ev1, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    p->num_elems = cur;
    float kms = 0.f;
    cudaEventElapsedTime(&kms, c->ev0, c->ev1);
    p->kernel_ms += kms;
    p->kernel_launches++;
    p->big_sets += ncol;
  }
  clear_on_error.armed = false;
  return RIP_OK;
}

// Grows the sets first+ids[i], one 1024-thread CTA each.
static int sample_big(rip_pool *p, uint64_t seed, uint64_t first,
                      const std::vector<uint32_t> &ids_in) {
  if (ids_in.empty()) return RIP_OK;
  if (p->giant_min && ids_in.size() >= p->giant_min) return sample_giant(p, seed, first, ids_in);
  rip_ctx *c = p->ctx;
  rip_graph *g = p->g;
  const uint64_t bm_words = (((uint64_t)g->n + 31) / 32 + 7) & ~7ull;
  uint32_t qcap = p->b_qcap ? p->b_qcap : std::min<uint32_t>(g->n, 1u << 20);
  auto slots_for = [&](uint32_t q) {
    const size_t per = bm_words * 4 + (size_t)q * 4;
    size_t avail = c->budget > c->used ? c->budget - c->used : 0;
    avail += p->b_scratch.bytes;
    // one slot per resident CTA
    const uint64_t max_slots = (uint64_t)c->num_sms * kBigCtasPerSm((int)p->big_threads);
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(max_slots, (avail / 4) / per));
  };
  TRY(ensure_big_scratch(p, slots_for(qcap), qcap));
  std::vector<uint32_t> ids = ids_in;
  PoolMeta *dm = p->dmeta();
  for (int attempt = 0; attempt < 32 && !ids.empty(); ++attempt) {
    TRY(dalloc(c, p->b_ids, sizeof(uint32_t) * ids.size() * 2));
    CK(c, cudaMemcpyAsync(p->b_ids.p, ids.data(), sizeof(uint32_t) * ids.size(),
                          cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemsetAsync(&dm->fail_count, 0, sizeof(unsigned int), c->stream));
    CK(c, cudaMemsetAsync(&dm->next, 0, sizeof(unsigned int), c->stream));
    CK(c, cudaMemsetAsync(&dm->first_bad, 0xFF, sizeof(unsigned long long), c->stream));
    BigLaunch L;
    L.G = g->view();
    L.P = p->view();
    L.key = make_key(seed);
    L.first = first;
    L.count = (uint32_t)ids.size();
    L.ids = ptr<uint32_t>(p->b_ids);
    L.next = &dm->next;
    L.bitmaps = ptr<uint32_t>(p->b_scratch);
    L.bm_words = bm_words;
    L.queues = ptr<uint32_t>(p->b_scratch) + (size_t)p->b_slots * bm_words;
    L.qcap = p->b_qcap;
    L.F = FailList{ptr<uint32_t>(p->b_ids) + ids.size(), &dm->fail_count, &dm->first_bad};
    L.st = Stats{dm->stats};
    L.blocks = (int)std::min<uint32_t>(p->b_slots, (uint32_t)ids.size());
    L.threads = (int)p->big_threads;
    CK(c, cudaEventRecord(c->ev0, c->stream));
    launch_ic_bigset(L, c->stream);
    CK(c, cudaGetLastError());
    CK(c, cudaEventRecord(c->ev1, c->stream));
    PoolMeta m;
    TRY(read_meta(p, m));
    float kms = 0.f;
    cudaEventElapsedTime(&kms, c->ev0, c->ev1);
    p->kernel_ms += kms;
    p->kernel_launches++;
    p->big_sets += ids.size() - m.fail_count;
    if (m.fail_count == 0) {
      p->num_elems = m.cursor;
      return RIP_OK;
    }
    const unsigned long long cur = std::min<unsigned long long>(m.cursor, m.first_bad);
    CK(c, cudaMemcpyAsync(&dm->cursor, &cur, sizeof(cur), cudaMemcpyHostToDevice, c->stream));
    p->num_elems = cur;
    std::vector<uint32_t> failed(m.fail_count);
    CK(c, cudaMemcpyAsync(failed.data(), ptr<uint32_t>(p->b_ids) + ids.size(),
                          sizeof(uint32_t) * m.fail_count, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    if (m.first_bad != ~0ull) {
      TRY(ensure_elems(p, std::max<uint64_t>(p->cap * 2, cur + (1u << 20))));
    } else if (p->b_qcap < g->n) {
      const uint32_t nq = (uint32_t)std::min<uint64_t>(g->n, (uint64_t)p->b_qcap * 4);
      TRY(ensure_big_scratch(p, std::min(slots_for(nq), p->b_slots), nq));
    } else {
      return set_err(c, RIP_ERR_DEVICE, "big-set sampler failed with full-size queues");
    }
    ids.swap(failed);
  }
  return ids.empty() ? RIP_OK : set_err(c, RIP_ERR_DEVICE, "big-set sampler did not converge");
}

// ---------------------------------------------------------------------------
// fused multi-colour sampler (IC)
// ---------------------------------------------------------------------------
static int ensure_fused_scratch(rip_pool *p, uint32_t slots, uint32_t cw,
                                uint32_t lcap) {
  rip_ctx *c = p->ctx;
  const size_t n = p->g->n;
  if (p->f_vis.p && p->f_slots == slots && p->f_cw == cw && p->f_lcap == lcap)
    return RIP_OK;
  const size_t mask_bytes = (size_t)slots * n * cw * sizeof(uint64_t);
  TRY(dalloc(c, p->f_vis, mask_bytes));
  TRY(dalloc(c, p->f_pend, mask_bytes));
  TRY(dalloc(c, p->f_flag, (size_t)slots * n * sizeof(uint32_t)));
  TRY(dalloc(c, p->f_log, (size_t)slots * lcap * sizeof(uint32_t)));
  CK(c, cudaMemsetAsync(p->f_vis.p, 0, mask_bytes, c->stream));
  CK(c, cudaMemsetAsync(p->f_pend.p, 0, mask_bytes, c->stream));
  CK(c, cudaMemsetAsync(p->f_flag.p, 0, (size_t)slots * n * sizeof(uint32_t), c->stream));
  p->f_slots = slots;
  p->f_cw = cw;
  p->f_lcap = lcap;
  return RIP_OK;
}

static int clear_fused_scratch(rip_pool *p) {
  rip_ctx *c = p->ctx;
  const size_t n = p->g->n;
  const size_t mask_bytes = (size_t)p->f_slots * n * p->f_cw * sizeof(uint64_t);
  CK(c, cudaMemsetAsync(p->f_vis.p, 0, mask_bytes, c->stream));
  CK(c, cudaMemsetAsync(p->f_pend.p, 0, mask_bytes, c->stream));
  CK(c, cudaMemsetAsync(p->f_flag.p, 0, (size_t)p->f_slots * n * sizeof(uint32_t), c->stream));
  return RIP_OK;
}

static int sample_fused(rip_pool *p, uint64_t seed, uint64_t first,
                        uint32_t count) {
  rip_ctx *c = p->ctx;
  rip_graph *g = p->g;
  const uint32_t colors = p->colors;
  const uint32_t cw = colors / 64;
  uint32_t lcap = p->lcap_pref ? p->lcap_pref
                 : p->f_lcap  ? p->f_lcap
                              : (uint32_t)std::min<uint64_t>(
                                    std::max<uint64_t>((uint64_t)g->n * 2, 4096), 1u << 20);
  // slots: one per resident CTA, limited by what the masks cost
  const size_t per_slot = (size_t)g->n * (cw * 16 + 4) + (size_t)lcap * 4;
  size_t avail = c->budget > c->used ? c->budget - c->used : 0;
  avail += p->f_vis.bytes + p->f_pend.bytes + p->f_flag.bytes + p->f_log.bytes;
  uint64_t fit = (avail / 2) / std::max<size_t>(per_slot, 1);
  uint64_t want = p->fused_slots ? p->fused_slots
                                 : (uint64_t)c->num_sms * fused_ctas_per_sm(colors);
  uint32_t slots = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, fit));
  if (p->f_vis.p && p->f_cw == cw && p->f_lcap == lcap && p->f_slots >= 1 &&
      p->f_slots <= slots)
    slots = p->f_slots;  // reuse the existing partition
  TRY(ensure_fused_scratch(p, slots, cw, lcap));
  TRY(dalloc(c, p->ids_a, sizeof(uint32_t) * ((size_t)count / 64 + 2)));
  PoolMeta *dm = p->dmeta();
  std::vector<uint32_t> order;  // empty: identity over [0, count)
  std::vector<uint32_t> big;    // sets of batches that outgrew their edge budget
  uint32_t todo = count;
  for (int attempt = 0; attempt < 4 && todo; ++attempt) {
    const uint32_t nb = (todo + colors - 1) / colors;
    if (!order.empty()) {
      TRY(dalloc(c, p->f_order, sizeof(uint32_t) * order.size()));
      CK(c, cudaMemcpyAsync(p->f_order.p, order.data(), sizeof(uint32_t) * order.size(),
                            cudaMemcpyHostToDevice, c->stream));
    }
    CK(c, cudaMemsetAsync(&dm->fail_count, 0, sizeof(unsigned int), c->stream));
    CK(c, cudaMemsetAsync(&dm->next, 0, sizeof(unsigned int), c->stream));
    CK(c, cudaMemsetAsync(&dm->fused_dirty, 0, sizeof(unsigned int), c->stream));
    CK(c, cudaMemsetAsync(&dm->first_bad, 0xFF, sizeof(unsigned long long), c->stream));
    FusedLaunch L;
    L.G = g->view();
    L.P = p->view();
    L.key = make_key(seed);
    L.first = first;
    L.count = todo;
    L.order = order.empty() ? nullptr : ptr<uint32_t>(p->f_order);
    L.num_batches = nb;
    L.colors = colors;
    L.next = &dm->next;
    L.vis = ptr<uint64_t>(p->f_vis);
    L.pend = ptr<uint64_t>(p->f_pend);
    L.pflag = ptr<uint32_t>(p->f_flag);
    L.log = ptr<uint32_t>(p->f_log);
    L.lcap = p->f_lcap;
    L.dirty = &dm->fused_dirty;
    L.work_cap = p->cap_fused;
    L.F = FailList{ptr<uint32_t>(p->ids_a), &dm->fail_count, &dm->first_bad};
    L.st = Stats{dm->stats};
    L.blocks = (int)std::min<uint32_t>(p->f_slots, nb);
    CK(c, cudaEventRecord(c->ev0, c->stream));
    launch_ic_fused(L, c->stream);
    CK(c, cudaGetLastError());
    CK(c, cudaEventRecord(c->ev1, c->stream));
    PoolMeta m;
    TRY(read_meta(p, m));
    float kms = 0.f;
    cudaEventElapsedTime(&kms, c->ev0, c->ev1);
    p->kernel_ms += kms;
    p->kernel_launches++;
    const uint32_t claimed = std::min<uint32_t>(m.next, nb);
    if (m.fail_count == 0 && claimed == nb) {
      p->num_elems = m.cursor;
      todo = 0;
      break;
    }
    unsigned long long cur = std::min<unsigned long long>(m.cursor, m.first_bad);
    CK(c, cudaMemcpyAsync(&dm->cursor, &cur, sizeof(cur), cudaMemcpyHostToDevice,
                          c->stream));
    p->num_elems = cur;
    std::vector<uint32_t> failed(m.fail_count);
    if (m.fail_count)
      CK(c, cudaMemcpyAsync(failed.data(), p->ids_a.p, sizeof(uint32_t) * m.fail_count,
                            cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    for (uint32_t b = claimed; b < nb; ++b) failed.push_back(b);
    std::vector<uint32_t> next_order;
    for (uint32_t fb : failed) {
      const uint32_t b = fb & ~FAIL_BIG;
      for (uint32_t i = b * colors; i < std::min<uint32_t>((b + 1) * colors, todo); ++i)
        ((fb & FAIL_BIG) ? big : next_order).push_back(order.empty() ? i : order[i]);
    }
    order.swap(next_order);
    todo = (uint32_t)order.size();
    if (m.first_bad != ~0ull) {
      double mean = m.stats[2] ? (double)m.stats[3] / (double)m.stats[2] : 16.0;
      TRY(ensure_elems(p, std::max<uint64_t>(cur + (uint64_t)(mean * 2.0 * todo) + 4096,
                                             p->cap * 2)));
    }
    if (m.fused_dirty) {
      // a frontier log overflowed: clear the masks and give the logs more room
      TRY(clear_fused_scratch(p));
      const uint32_t nl = (uint32_t)std::min<uint64_t>((uint64_t)p->f_lcap * 4,
                                                       (uint64_t)g->n * colors);
      const uint32_t ns = std::max<uint32_t>(1, p->f_slots / 2);
      TRY(ensure_fused_scratch(p, ns, cw, nl));
    }
  }
  // Whatever still failed runs set by set (same sets, bit for bit); sets of
  // batches that outgrew their edge budget are grown one CTA each.
  if (todo) TRY(sample_warp_per_set(p, seed, first, todo, &order));
  if (!big.empty()) {
    std::sort(big.begin(), big.end());
    TRY(sample_big(p, seed, first, big));
  }
  return RIP_OK;
}

// Fused-sampler configuration (the autotuner's knobs): colour width 64, 128
// or 256, number of CTA slots (0 = size from the budget) and frontier-log
// capacity per slot (0 = default).  Takes effect at the next rip_sample.
// Diagnostic breakdown of rip_select since the pool was created (see
// rip_pool::sel_prof).
extern "C" int rip_select_profile(rip_pool *p, double out[12]) {
  if (!p || !out) return RIP_ERR_INVALID;
  for (int i = 0; i < 12; ++i) out[i] = p->sel_prof[i];
  return RIP_OK;
}

// Edge-work budgets before a warp (plain) or a CTA batch (fused) hands its
// set(s) to the CTA-per-set sampler; 0 disables the hand-over.
extern "C" int rip_pool_work_caps(rip_pool *p, uint64_t plain_cap, uint64_t fused_cap) {
  if (!p) return RIP_ERR_INVALID;
  p->cap_plain = plain_cap;
  p->cap_fused = fused_cap;
  return RIP_OK;
}

// Per-graph sampler autotuner: times a pilot of sets under each IC sampler
// configuration on a scratch pool and keeps the fastest for the graph.
extern "C" int rip_graph_autotune(rip_graph *g, uint64_t seed, uint32_t pilot, double *ms,
                                  int *choice) {
  if (!g) return RIP_ERR_INVALID;
  rip_ctx *c = g->ctx;
  struct Cand {
    int sampler;
    uint32_t colors;
    uint64_t cap_plain, cap_fused;
    uint32_t giant_min;
    int occupancy;
    uint32_t big_threads;
  };
  static const Cand cands[RIP_TUNE_CANDIDATES] = {
      {RIP_SAMPLER_PLAIN, 64, 1ull << 18, 1ull << 23, 32, 0, 1024},
      {RIP_SAMPLER_PLAIN, 64, 1ull << 14, 1ull << 23, 32, 0, 1024},
      {RIP_SAMPLER_PLAIN, 64, 1ull << 18, 1ull << 23, 0, 0, 1024},
      {RIP_SAMPLER_FUSED, 64, 1ull << 18, 1ull << 23, 32, 0, 1024},
      {RIP_SAMPLER_FUSED, 128, 1ull << 18, 1ull << 23, 32, 0, 1024},
      {RIP_SAMPLER_FUSED, 256, 1ull << 18, 1ull << 23, 32, 0, 1024},
      {RIP_SAMPLER_PLAIN, 64, 1ull << 18, 1ull << 23, 32, 5, 256},
      {RIP_SAMPLER_PLAIN, 64, 1ull << 18, 1ull << 23, 0, 5, 256},
      {RIP_SAMPLER_PLAIN, 64, 1ull << 18, 1ull << 23, 0, 0, 256},
      {RIP_SAMPLER_PLAIN, 64, 1ull << 16, 1ull << 23, 0, 0, 256},
  };
  if (ms)
    for (int i = 0; i < RIP_TUNE_CANDIDATES; ++i) ms[i] = -1.0;
  if (g->model != RIP_MODEL_IC) {  // one LT sampler: nothing to choose
    g->tuned = rip_graph::Tuned{};
    g->tuned.set = true;
    if (choice) *choice = 0;
    return RIP_OK;
  }
  // Two phases: every candidate on a short screen of the pilot's first sets,
  // then those within twice the best screen time on the whole pilot (on large
  // graphs the heavy sets of a short run are too few to fill the GPU, which
  // hides what the heavy-set paths cost at full size).  Each timing is the
  // faster of two runs after a warm-up that sizes every scratch buffer.
  pilot = std::max<uint32_t>(pilot ? pilot : 2048, 64);
  const uint32_t screen = std::min<uint32_t>(pilot, 2048);
  auto time_cand = [&](int i, uint32_t sets, double *out) -> int {
    rip_pool *p = nullptr;
    TRY(rip_pool_create(c, g, &p));
    p->auto_sampler = cands[i].sampler;
    p->colors = cands[i].colors;
    p->cap_plain = cands[i].cap_plain;
    p->cap_fused = cands[i].cap_fused;
    p->giant_min = cands[i].giant_min;
    p->plain_occupancy = cands[i].occupancy;
    p->big_threads = cands[i].big_threads;
    int rc = rip_sample(p, seed, sets, RIP_SAMPLER_AUTO);
    if (rc == RIP_OK) rc = rip_sync(c);
    double t = 1e300;
    for (int rep = 0; rep < 2 && rc == RIP_OK; ++rep) {
      rc = rip_pool_clear(p);
      const auto t0 = clk::now();
      if (rc == RIP_OK) rc = rip_sample(p, seed, sets, RIP_SAMPLER_AUTO);
      if (rc == RIP_OK) rc = rip_sync(c);
      t = std::min(t, ms_since(t0));
    }
    rip_pool_destroy(p);
    *out = t;
    return rc;
  };
  double t_screen[RIP_TUNE_CANDIDATES];
  double screen_best = 1e300;
  for (int i = 0; i < RIP_TUNE_CANDIDATES; ++i) {
    TRY(time_cand(i, screen, &t_screen[i]));
    screen_best = std::min(screen_best, t_screen[i]);
    if (ms) ms[i] = t_screen[i];
  }
  int best = 0;
  double best_ms = 1e300;
  for (int i = 0; i < RIP_TUNE_CANDIDATES; ++i) {
    double t = t_screen[i];
    if (pilot > screen) {
      if (t_screen[i] > 2.0 * screen_best) continue;  // out after the screen
      TRY(time_cand(i, pilot, &t));
      if (ms) ms[i] = t;
    }
    if (t < best_ms) {
      best = i;
      best_ms = t;
    }
  }
  g->tuned.set = true;
  g->tuned.sampler = cands[best].sampler;
  g->tuned.colors = cands[best].colors;
  g->tuned.cap_plain = cands[best].cap_plain;
  g->tuned.cap_fused = cands[best].cap_fused;
  g->tuned.giant_min = cands[best].giant_min;
  g->tuned.plain_occupancy = cands[best].occupancy;
  g->tuned.big_threads = cands[best].big_threads;
  if (choice) *choice = best;
  return RIP_OK;
}

// Register/occupancy variant of the one-set-per-warp IC kernel (0 or 5).
extern "C" int rip_pool_plain_occupancy(rip_pool *p, int blocks_per_sm) {
  if (!p || (blocks_per_sm != 0 && blocks_per_sm != 5)) return RIP_ERR_INVALID;
  if (p->plain_occupancy != blocks_per_sm) {
    p->plain_occupancy = blocks_per_sm;
    p->warps = 0;  // re-size the per-warp scratch for the new warp count
  }
  return RIP_OK;
}

// Number of heavy IC sets from which they are grown by the grid-wide
// multi-colour BFS instead of one CTA each (0 = never).
extern "C" int rip_pool_heavy_batch(rip_pool *p, uint32_t min_sets) {
  if (!p) return RIP_ERR_INVALID;
  p->giant_min = min_sets;
  return RIP_OK;
}

// Block shape of the CTA-per-set kernel for heavy IC sets.
extern "C" int rip_pool_heavy_block(rip_pool *p, uint32_t threads) {
  if (!p || (threads != 128 && threads != 256 && threads != 512 && threads != 1024))
    return RIP_ERR_INVALID;
  p->big_threads = threads;
  return RIP_OK;
}

// First-fetch threshold of reference-heap picks as a percentage of the
// previous gain (0 = adaptive); the seeds do not depend on it.
extern "C" int rip_pool_select_guess(rip_pool *p, uint32_t percent) {
  if (!p || percent > 100) return RIP_ERR_INVALID;
  p->cand_fixed = percent;
  return RIP_OK;
}

extern "C" int rip_pool_configure(rip_pool *p, uint32_t colors, uint32_t slots,
                                  uint32_t log_capacity) {
  if (!p) return RIP_ERR_INVALID;
  if (colors != 64 && colors != 128 && colors != 256)
    return set_err(p->ctx, RIP_ERR_INVALID, "colors must be 64, 128 or 256");
  p->colors = colors;
  p->fused_slots = slots;
  p->lcap_pref = log_capacity;
  return RIP_OK;
}

extern "C" int rip_sample(rip_pool *p, uint64_t seed, uint64_t count,
                          int sampler) {
  if (!p) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  if (count == 0) return RIP_OK;
  if (count >= (1ull << 31))
    return set_err(c, RIP_ERR_LIMIT, "rip_sample: at most 2^31-1 sets per call");
  if (p->num_sets + count >= (1ull << 56))
    return set_err(c, RIP_ERR_LIMIT, "rip_sample: set ids are limited to 2^56");
  CK(c, cudaSetDevice(c->device));
  const uint64_t first = p->num_sets;
  TRY(ensure_sets(p, first + count));
  PoolMeta m;
  TRY(read_meta(p, m));
  if (m.stats[2] == 0 && count > 4096) {
    // Fresh pool: sample a pilot of 1024 sets first so the pool is sized from
    // a measured mean set size (the sets are the same either way).
    TRY(rip_sample(p, seed, 1024, sampler));
    return rip_sample(p, seed, count - 1024, sampler);
  }
  double mean = m.stats[2] ? (double)m.stats[3] / (double)m.stats[2] : 8.0;
  TRY(ensure_elems(p, p->num_elems + (uint64_t)(mean * 1.25 * count) + 1024));
  int rc;
  const bool fused = sampler == RIP_SAMPLER_FUSED ||
                     (sampler == RIP_SAMPLER_AUTO && p->auto_sampler == RIP_SAMPLER_FUSED);
  if (p->g->model == RIP_MODEL_IC && fused)
    rc = sample_fused(p, seed, first, (uint32_t)count);
  else
    rc = sample_warp_per_set(p, seed, first, (uint32_t)count, nullptr);
  if (rc != RIP_OK) return rc;
  p->num_sets += count;
  p->have_last_counts = false;
  return RIP_OK;
}

extern "C" int rip_pool_export(rip_pool *p, uint64_t first, uint64_t count,
                               uint64_t *offsets, uint32_t *vertices) {
  if (!p || !offsets) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  if (first + count > p->num_sets)
    return set_err(c, RIP_ERR_INVALID, "export range beyond the pool (%llu sets)",
                   (unsigned long long)p->num_sets);
  std::vector<uint32_t> lens(count);
  if (count) {
    CK(c, cudaMemcpyAsync(lens.data(), ptr<uint32_t>(p->set_len) + first,
                          sizeof(uint32_t) * count, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
  }
  offsets[0] = 0;
  for (uint64_t i = 0; i < count; ++i) offsets[i + 1] = offsets[i] + lens[i];
  if (!vertices || offsets[count] == 0) return RIP_OK;
  DevMem d_csr, d_out;
  int rc = RIP_OK;
  do {
    if ((rc = dalloc(c, d_csr, sizeof(uint64_t) * (count + 1)))) break;
    if ((rc = dalloc(c, d_out, sizeof(uint32_t) * offsets[count]))) break;
    cudaMemcpyAsync(d_csr.p, offsets, sizeof(uint64_t) * (count + 1),
                    cudaMemcpyHostToDevice, c->stream);
    launch_gather_sets(p->view(), first, count, ptr<uint64_t>(d_csr),
                       ptr<uint32_t>(d_out), c->stream);
    cudaMemcpyAsync(vertices, d_out.p, sizeof(uint32_t) * offsets[count],
                    cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) rc = set_err(c, RIP_ERR_CUDA, "export failed: %s", cudaGetErrorString(e));
  } while (0);
  dfree(c, d_csr);
  dfree(c, d_out);
  if (rc) return rc;
#pragma omp parallel for schedule(dynamic, 256)
  for (long long i = 0; i < (long long)count; ++i)
    std::sort(vertices + offsets[i], vertices + offsets[i + 1]);
  return RIP_OK;
}

extern "C" int rip_pool_import(rip_pool *p, const uint64_t *offsets,
                               const uint32_t *vertices, uint64_t count) {
  if (!p || !offsets || (offsets[count] && !vertices)) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  if (offsets[0] != 0)
    return set_err(c, RIP_ERR_INVALID, "rip_pool_import: offsets[0] must be 0");
  const uint64_t P = offsets[count];
  for (uint64_t i = 0; i < count; ++i) {
    if (offsets[i + 1] < offsets[i])
      return set_err(c, RIP_ERR_INVALID, "rip_pool_import: offsets not monotone");
    if (offsets[i + 1] - offsets[i] > p->g->n)
      return set_err(c, RIP_ERR_INVALID, "rip_pool_import: set larger than n");
  }
  for (uint64_t i = 0; i < P; ++i)
    if (vertices[i] >= p->g->n)
      return set_err(c, RIP_ERR_INVALID, "rip_pool_import: vertex %u out of range",
                     vertices[i]);
  CK(c, cudaSetDevice(c->device));
  TRY(ensure_sets(p, p->num_sets + count));
  TRY(ensure_elems(p, p->num_elems + P));
  std::vector<uint64_t> so(count);
  std::vector<uint32_t> sl(count);
  for (uint64_t i = 0; i < count; ++i) {
    so[i] = p->num_elems + offsets[i];
    sl[i] = (uint32_t)(offsets[i + 1] - offsets[i]);
  }
  if (P)
    CK(c, cudaMemcpyAsync(ptr<uint32_t>(p->vtx) + p->num_elems, vertices,
                          sizeof(uint32_t) * P, cudaMemcpyHostToDevice, c->stream));
  if (count) {
    CK(c, cudaMemcpyAsync(ptr<uint64_t>(p->set_off) + p->num_sets, so.data(),
                          sizeof(uint64_t) * count, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaMemcpyAsync(ptr<uint32_t>(p->set_len) + p->num_sets, sl.data(),
                          sizeof(uint32_t) * count, cudaMemcpyHostToDevice, c->stream));
  }
  unsigned long long cur = p->num_elems + P;
  CK(c, cudaMemcpyAsync(&p->dmeta()->cursor, &cur, sizeof(cur),
                        cudaMemcpyHostToDevice, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  p->num_elems += P;
  p->num_sets += count;
  p->have_last_counts = false;
  return RIP_OK;
}

// Appends `count` empty sets: the ids another shard samples.  An empty set
// adds nothing to any count and is never covered, so a pool that holds its
// own ids' sets and empty placeholders for the rest counts exactly its share.
extern "C" int rip_pool_skip(rip_pool *p, uint64_t count) {
  if (!p) return RIP_ERR_INVALID;
  rip_ctx *c = p->ctx;
  if (count == 0) return RIP_OK;
  if (p->num_sets + count >= (1ull << 56))
    return set_err(c, RIP_ERR_LIMIT, "rip_pool_skip: set ids are limited to 2^56");
  CK(c, cudaSetDevice(c->device));
  TRY(ensure_sets(p, p->num_sets + count));
  CK(c, cudaMemsetAsync(ptr<uint64_t>(p->set_off) + p->num_sets, 0, sizeof(uint64_t) * count,
                        c->stream));
  CK(c, cudaMemsetAsync(ptr<uint32_t>(p->set_len) + p->num_sets, 0, sizeof(uint32_t) * count,
                        c->stream));
  p->num_sets += count;
  p->have_last_counts = false;
  return RIP_OK;
}


// ---------------------------------------------------------------------------
// many pools in one launch
// ---------------------------------------------------------------------------
// Sets of every pool come from the same one-set-per-warp bodies as rip_sample
// (same set ids, same Philox streams), so a pool extended here holds exactly
// the sets rip_sample would have put there.  Sets that fail in the shared
// launch (queue or pool overflow, IC edge work over the cap) are finished per
// pool by the single-pool paths.
extern "C" int rip_sample_multi(rip_ctx *c, rip_pool *const *pools, const uint64_t *seeds,
                                const uint64_t *counts, uint32_t n_pools) {
  if (!c || (n_pools && (!pools || !seeds || !counts))) return RIP_ERR_INVALID;
  uint64_t total = 0;
  for (uint32_t i = 0; i < n_pools; ++i) {
    if (!pools[i] || pools[i]->ctx != c)
      return set_err(c, RIP_ERR_INVALID, "rip_sample_multi: pool %u is not of this context", i);
    for (uint32_t j = 0; j < i; ++j)
      if (pools[j] == pools[i] && counts[i] && counts[j])
        return set_err(c, RIP_ERR_INVALID, "rip_sample_multi: pool %u listed twice", i);
    if (counts[i] >= (1ull << 31))
      return set_err(c, RIP_ERR_LIMIT, "rip_sample_multi: at most 2^31-1 sets per pool");
    if (pools[i]->num_sets + counts[i] >= (1ull << 56))
      return set_err(c, RIP_ERR_LIMIT, "rip_sample_multi: set ids are limited to 2^56");
    total += counts[i];
  }
  if (total == 0) return RIP_OK;
  if (total >= (1ull << 32) - 1)
    return set_err(c, RIP_ERR_LIMIT, "rip_sample_multi: at most 2^32-2 sets per call");
  CK(c, cudaSetDevice(c->device));
  std::vector<uint32_t> act;  // pools with work
  for (uint32_t i = 0; i < n_pools; ++i)
    if (counts[i]) act.push_back(i);
  // per-pool meta (set-size means for the pool sizing), read in one sync
  if (!c->h_meta) c->h_meta = new PinnedMem();
  TRY(c->h_meta->ensure(c, sizeof(PoolMeta) * act.size()));
  PoolMeta *hm = reinterpret_cast<PoolMeta *>(c->h_meta->p);
  for (size_t a = 0; a < act.size(); ++a)
    CK(c, cudaMemcpyAsync(hm + a, pools[act[a]]->meta.p, sizeof(PoolMeta),
                          cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  {
    // Fresh pools with large requests first take a pilot of 1024 sets (as
    // rip_sample does) so they are sized from a measured mean set size.
    std::vector<rip_pool *> pp;
    std::vector<uint64_t> ps, pc;
    for (size_t a = 0; a < act.size(); ++a)
      if (hm[a].stats[2] == 0 && counts[act[a]] > 4096) {
        pp.push_back(pools[act[a]]);
        ps.push_back(seeds[act[a]]);
        pc.push_back(1024);
      }
    if (!pp.empty()) {
      TRY(rip_sample_multi(c, pp.data(), ps.data(), pc.data(), (uint32_t)pp.size()));
      std::vector<uint64_t> rest(counts, counts + n_pools);
      for (uint32_t i = 0; i < n_pools; ++i)
        for (rip_pool *q : pp)
          if (pools[i] == q && rest[i]) {
            rest[i] -= 1024;
            break;
          }
      return rip_sample_multi(c, pools, seeds, rest.data(), n_pools);
    }
  }
  uint64_t max_n = 1;
  std::vector<uint64_t> firsts(act.size());
  for (size_t a = 0; a < act.size(); ++a) {
    rip_pool *p = pools[act[a]];
    const uint64_t cnt = counts[act[a]];
    max_n = std::max<uint64_t>(max_n, p->g->n);
    firsts[a] = p->num_sets;
    TRY(ensure_sets(p, p->num_sets + cnt));
    const double mean = hm[a].stats[2] ? (double)hm[a].stats[3] / (double)hm[a].stats[2] : 8.0;
    TRY(ensure_elems(p, p->num_elems + (uint64_t)(mean * 1.25 * cnt) + 1024));
  }
  // shared per-warp scratch, sized for the largest graph of the launch
  const uint64_t bm_words = ((max_n + 31) / 32 + 7) & ~7ull;
  const uint32_t qcap = (uint32_t)std::min<uint64_t>(max_n, 1u << 14);
  if (!c->m_scratch.p || c->m_bm_words < bm_words || c->m_qcap < qcap) {
    const uint64_t per = bm_words * 4 + (uint64_t)qcap * 4;
    const size_t avail = c->budget > c->used ? c->budget - c->used : 0;
    uint64_t w = std::min<uint64_t>((uint64_t)c->num_sms * 32,
                                    std::max<uint64_t>((avail / 4) / per, 8));
    w = std::max<uint64_t>(8, w & ~7ull);
    TRY(dalloc(c, c->m_scratch, per * w));
    CK(c, cudaMemsetAsync(c->m_scratch.p, 0, per * w, c->stream));
    c->m_bm_words = bm_words;
    c->m_qcap = qcap;
    c->m_warps = (uint32_t)w;
  }
  // instance table | prefix | launch counters, one upload
  const size_t n_act = act.size();
  const size_t desc_bytes = sizeof(InstanceDesc) * n_act;
  const size_t pre_off = (desc_bytes + 15) & ~(size_t)15;
  const size_t ctr_off = (pre_off + sizeof(uint32_t) * (n_act + 1) + 15) & ~(size_t)15;
  const size_t table_bytes = ctr_off + 16;
  std::vector<uint8_t> table(table_bytes, 0);
  InstanceDesc *desc = reinterpret_cast<InstanceDesc *>(table.data());
  uint32_t *prefix = reinterpret_cast<uint32_t *>(table.data() + pre_off);
  prefix[0] = 0;
  for (size_t a = 0; a < n_act; ++a) {
    rip_pool *p = pools[act[a]];
    InstanceDesc &D = desc[a];
    D.G = p->g->view();
    D.P = p->view();
    D.key = make_key(seeds[act[a]]);
    D.first = firsts[a];
    D.work_cap = p->g->model == RIP_MODEL_IC ? p->cap_plain : 0;
    D.first_bad = &p->dmeta()->first_bad;
    D.stats = p->dmeta()->stats;
    D.model = (uint32_t)p->g->model;
    prefix[a + 1] = prefix[a] + (uint32_t)counts[act[a]];
    CK(c, cudaMemsetAsync(&p->dmeta()->first_bad, 0xFF, sizeof(unsigned long long), c->stream));
  }
  TRY(dalloc(c, c->m_table, table_bytes));
  TRY(dalloc(c, c->m_fail, sizeof(uint32_t) * 2 * (size_t)total));
  CK(c, cudaMemcpyAsync(c->m_table.p, table.data(), table_bytes, cudaMemcpyHostToDevice,
                        c->stream));
  uint8_t *dt = ptr<uint8_t>(c->m_table);
  MultiLaunch L;
  L.inst = reinterpret_cast<const InstanceDesc *>(dt);
  L.prefix = reinterpret_cast<const uint32_t *>(dt + pre_off);
  L.n_inst = (uint32_t)n_act;
  L.total = (uint32_t)total;
  L.next = reinterpret_cast<unsigned int *>(dt + ctr_off);
  L.fail_count = reinterpret_cast<unsigned int *>(dt + ctr_off + 4);
  L.bitmaps = ptr<uint32_t>(c->m_scratch);
  L.bm_words = c->m_bm_words;
  L.queues = ptr<uint32_t>(c->m_scratch) + (size_t)c->m_bm_words * c->m_warps;
  L.qcap = c->m_qcap;
  L.fail = ptr<uint32_t>(c->m_fail);
  L.blocks = (int)std::max<uint64_t>(1, (std::min<uint64_t>(c->m_warps, total) + 7) / 8);
  CK(c, cudaEventRecord(c->ev0, c->stream));
  launch_multi_sample(L, c->stream);
  CK(c, cudaGetLastError());
  CK(c, cudaEventRecord(c->ev1, c->stream));
  uint32_t n_fail = 0;
  CK(c, cudaMemcpyAsync(&n_fail, L.fail_count, sizeof(n_fail), cudaMemcpyDeviceToHost,
                        c->stream));
  for (size_t a = 0; a < n_act; ++a)
    CK(c, cudaMemcpyAsync(hm + a, pools[act[a]]->meta.p, sizeof(PoolMeta),
                          cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  float kms = 0.f;
  cudaEventElapsedTime(&kms, c->ev0, c->ev1);
  c->multi_kernel_ms += kms;
  std::vector<uint32_t> fails(2 * (size_t)n_fail);
  if (n_fail) {
    CK(c, cudaMemcpyAsync(fails.data(), L.fail, sizeof(uint32_t) * 2 * n_fail,
                          cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
  }
  std::vector<std::vector<uint32_t>> retry(n_act), big(n_act);
  for (uint32_t f = 0; f < n_fail; ++f) {
    const uint32_t a = fails[2 * f], r = fails[2 * f + 1];
    if (r & FAIL_BIG) big[a].push_back(r & ~FAIL_BIG);
    else retry[a].push_back(r);
  }
  for (size_t a = 0; a < n_act; ++a) {
    rip_pool *p = pools[act[a]];
    const double share = (double)counts[act[a]] / (double)total;
    p->kernel_ms += kms * share;
    p->kernel_launches++;
    // roll the bump pointer back to the end of the last stored set
    const unsigned long long cur = std::min<unsigned long long>(hm[a].cursor, hm[a].first_bad);
    if (cur != hm[a].cursor)
      CK(c, cudaMemcpyAsync(&p->dmeta()->cursor, &cur, sizeof(cur), cudaMemcpyHostToDevice,
                            c->stream));
    p->num_elems = cur;
    if (!retry[a].empty()) {
      if (hm[a].first_bad != ~0ull) {
        const double mean =
            hm[a].stats[2] ? (double)hm[a].stats[3] / (double)hm[a].stats[2] : 16.0;
        TRY(ensure_elems(p, std::max<uint64_t>(
                                cur + (uint64_t)(mean * 2.0 * retry[a].size()) + 4096,
                                p->cap * 2)));
      }
      std::sort(retry[a].begin(), retry[a].end());
      TRY(sample_warp_per_set(p, seeds[act[a]], firsts[a], (uint32_t)counts[act[a]],
                              &retry[a]));
    }
    if (!big[a].empty()) {
      std::sort(big[a].begin(), big[a].end());
      TRY(sample_big(p, seeds[act[a]], firsts[a], big[a]));
    }
    p->num_sets += counts[act[a]];
    p->have_last_counts = false;
  }
  CK(c, cudaStreamSynchronize(c->stream));
  return RIP_OK;
}

