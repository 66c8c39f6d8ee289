// spread.cu -- forward Monte Carlo spread of a seed set (host side).
//
// rip_spread_ic / rip_spread_lt replace the replica loop of
// tools/simulator.cc:139-149 over ripples::simulate
// (include/ripples/diffusion_simulation.h:73-178): the expected number of
// vertices a seed set reaches, averaged over replicas, with every replica's
// reached count available for variance estimates.
#include "host.h"

namespace {

int spread_run(rip_graph *g, rip_graph *b, const uint32_t *seeds, uint32_t k,
               uint64_t replicas, uint64_t seed, uint32_t *sizes, uint32_t *levels,
               double *spread, const char *who) {
  rip_ctx *c = g->ctx;
  if ((k && !seeds) || !spread) return set_err(c, RIP_ERR_INVALID, "%s: null argument", who);
  for (uint32_t i = 0; i < k; ++i)
    if (seeds[i] >= g->n)
      return set_err(c, RIP_ERR_INVALID, "%s: seed %u out of range (n = %u)", who, seeds[i],
                     g->n);
  if (replicas >= (1ull << 56))
    return set_err(c, RIP_ERR_LIMIT, "%s: at most 2^56 replicas", who);
  *spread = 0.0;
  if (replicas == 0 || g->n == 0) return RIP_OK;
  CK(c, cudaSetDevice(c->device));

  // per CTA slot: an n-bit visited bitmap and an n-entry queue (a replica
  // queues every vertex at most once); at most one slot per resident CTA,
  // fewer when the slots would take more than a quarter of the free budget
  const uint64_t bm_words = ((uint64_t)g->n + 31) / 32;
  const uint64_t per_slot = 4 * bm_words + 4 * (uint64_t)g->n;
  uint64_t slots = std::min<uint64_t>(replicas, (uint64_t)c->num_sms * kSpreadCtasPerSm);
  const uint64_t room = c->budget > c->used ? (c->budget - c->used) / 4 : 0;
  while (slots > 1 && slots * per_slot > room) slots /= 2;

  struct Buffers {
    rip_ctx *c;
    DevMem scratch, ctr, d_seeds, d_sizes, d_levels;
    ~Buffers() {
      dfree(c, scratch);
      dfree(c, ctr);
      dfree(c, d_seeds);
      dfree(c, d_sizes);
      dfree(c, d_levels);
    }
  } B{c, {}, {}, {}, {}, {}};
  TRY(dalloc(c, B.scratch, slots * per_slot));
  TRY(dalloc(c, B.ctr, 2 * sizeof(unsigned long long)));
  TRY(dalloc(c, B.d_seeds, sizeof(uint32_t) * std::max<uint32_t>(k, 1)));
  if (sizes) TRY(dalloc(c, B.d_sizes, sizeof(uint32_t) * replicas));
  if (levels) TRY(dalloc(c, B.d_levels, sizeof(uint32_t) * replicas));
  CK(c, cudaMemsetAsync(B.scratch.p, 0, slots * bm_words * 4, c->stream));
  CK(c, cudaMemsetAsync(B.ctr.p, 0, 2 * sizeof(unsigned long long), c->stream));
  if (k)
    CK(c, cudaMemcpyAsync(B.d_seeds.p, seeds, sizeof(uint32_t) * k, cudaMemcpyHostToDevice,
                          c->stream));

  SpreadLaunch L;
  L.G = g->view();
  if (b) L.B = b->view();
  L.key = make_key(seed);
  L.seeds = ptr<uint32_t>(B.d_seeds);
  L.k = k;
  L.replicas = replicas;
  L.next = ptr<unsigned long long>(B.ctr);
  L.total = L.next + 1;
  L.sizes = sizes ? ptr<uint32_t>(B.d_sizes) : nullptr;
  L.levels = levels ? ptr<uint32_t>(B.d_levels) : nullptr;
  L.bitmaps = ptr<uint32_t>(B.scratch);
  L.bm_words = bm_words;
  L.queues = L.bitmaps + slots * bm_words;
  L.qcap = g->n;
  L.blocks = (int)slots;
  launch_spread(L, b != nullptr, c->stream);
  CK(c, cudaGetLastError());
  unsigned long long total = 0;
  CK(c, cudaMemcpyAsync(&total, L.total, sizeof(total), cudaMemcpyDeviceToHost, c->stream));
  if (sizes)
    CK(c, cudaMemcpyAsync(sizes, B.d_sizes.p, sizeof(uint32_t) * replicas,
                          cudaMemcpyDeviceToHost, c->stream));
  if (levels)
    CK(c, cudaMemcpyAsync(levels, B.d_levels.p, sizeof(uint32_t) * replicas,
                          cudaMemcpyDeviceToHost, c->stream));
  CK(c, cudaStreamSynchronize(c->stream));
  *spread = (double)total / (double)replicas;
  return RIP_OK;
}

}  // namespace

extern "C" int rip_spread_ic(rip_graph *g, const uint32_t *seeds, uint32_t k,
                             uint64_t replicas, uint64_t seed, uint32_t *sizes,
                             uint32_t *levels, double *spread) {
  if (!g) return RIP_ERR_INVALID;
  if (g->model != RIP_MODEL_IC)
    return set_err(g->ctx, RIP_ERR_INVALID,
                   "rip_spread_ic: the graph must be an IC graph holding the forward CSR");
  return spread_run(g, nullptr, seeds, k, replicas, seed, sizes, levels, spread,
                    "rip_spread_ic");
}

extern "C" int rip_spread_lt(rip_graph *fwd, rip_graph *bwd, const uint32_t *seeds,
                             uint32_t k, uint64_t replicas, uint64_t seed, uint32_t *sizes,
                             uint32_t *levels, double *spread) {
  if (!fwd || !bwd) return RIP_ERR_INVALID;
  if (bwd->model != RIP_MODEL_LT || fwd->ctx != bwd->ctx)
    return set_err(fwd->ctx, RIP_ERR_INVALID,
                   "rip_spread_lt: bwd must be the graph's LT upload in the same context");
  if (fwd->n != bwd->n || fwd->m != bwd->m)
    return set_err(fwd->ctx, RIP_ERR_INVALID,
                   "rip_spread_lt: forward and backward CSR differ in size");
  return spread_run(fwd, bwd, seeds, k, replicas, seed, sizes, levels, spread,
                    "rip_spread_lt");
}
