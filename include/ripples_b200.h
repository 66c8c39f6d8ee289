/*
 * ripples_b200.h -- C ABI of the B200-native IMM hot path.
 *
 * The reference (pnnl/ripples) exposes this path as header-only C++ templates:
 *   ripples::IMM                      include/ripples/imm.h:671,768
 *   ripples::GenerateRRRSets          include/ripples/generate_rrr_sets.h:186,217
 *   StreamingRRRGenerator::generate   include/ripples/streaming_rrr_generator.h:1026
 *   ripples::FindMostInfluentialSet   include/ripples/find_most_influential.h:85,176
 * and its CUDA side through GPU<R>::device_malloc/h2d/d2h
 * (include/ripples/gpu/gpu_runtime_trait.h:64-320).  This header is the plain
 * C boundary those templates call instead: plain pointers and sizes, no C++ or
 * torch types.
 *
 * Conventions
 *   - Every entry point returns an int status: RIP_OK (0) or a negative
 *     RIP_ERR_* code.  A human-readable message for the last failure on a
 *     context is returned by rip_last_error().  Nothing aborts the process.
 *     (The reference prints CUDA errors and continues, src/gpu/cuda_utils.cu:53-59,
 *     or calls exit(-1), include/ripples/graph.h:866-935.)
 *   - Host arrays passed in are read during the call and never retained.
 *   - Vertex ids are uint32 in [0, n); in-edge lists follow the reference's
 *     backward CSR (GraphBwd, include/ripples/graph.h:107-130): the in-neighbours
 *     of v are src[index[v] .. index[v+1]).
 *   - One context = one CUDA device + one stream.  A context is not re-entrant;
 *     use one context per host thread (the reference is single-threaded at this
 *     boundary too, include/ripples/imm.h:768).
 */
#ifndef RIPPLES_B200_H
#define RIPPLES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define RIP_OK 0
#define RIP_ERR_INVALID (-1)   /* bad argument (null pointer, id out of range) */
#define RIP_ERR_CUDA (-2)      /* a CUDA runtime call failed                    */
#define RIP_ERR_NOMEM (-3)     /* device or host allocation failed / budget     */
#define RIP_ERR_STATE (-4)     /* call not valid in the object's current state  */
#define RIP_ERR_LIMIT (-5)     /* input beyond a documented size limit          */
#define RIP_ERR_DEVICE (-6)    /* a kernel reported an internal error flag      */

/* ---- enums ---------------------------------------------------------------- */
/* Diffusion models: independent_cascade_tag / linear_threshold_tag
 * (include/ripples/diffusion_simulation.h). */
#define RIP_MODEL_IC 0
#define RIP_MODEL_LT 1

/* Seed-selection tie-break.  REF_HEAP reproduces the reference CPU lazy
 * max-heap order (include/ripples/streaming_find_most_influential.h:410-418,
 * 546-572); LOWEST_ID reproduces the reference GPU selection, which takes
 * thrust::max_element (src/gpu/find_most_influential.cc:65-72). */
#define RIP_TIE_REF_HEAP 0
#define RIP_TIE_LOWEST_ID 1

/* IC sampler variants (LT always uses the walk kernel). */
#define RIP_SAMPLER_AUTO 0   /* the graph's autotuned choice (default: plain) */
#define RIP_SAMPLER_PLAIN 1  /* one set per warp                              */
#define RIP_SAMPLER_FUSED 2  /* fused multi-colour reverse BFS                */

/* Synthetic edge-weight models (for graph construction helpers). */
#define RIP_WEIGHTS_UNIFORM 0       /* U(lo, hi) per edge                       */
#define RIP_WEIGHTS_LT_NORMALIZED 1 /* U(0,1) then normalised per destination   */
#define RIP_WEIGHTS_WC 2            /* weighted cascade: 1 / in-degree(dst)     */

typedef struct rip_ctx rip_ctx;
typedef struct rip_graph rip_graph;
typedef struct rip_pool rip_pool;

/* ---- context -------------------------------------------------------------- */
/* Replaces the per-GPU runtime set-up of the streaming engine
 * (include/ripples/streaming_rrr_generator.h:866-872, gpu_runtime_trait.h:64-160).
 * hbm_budget: bytes this context may allocate on the device (0 = 90% of free). */
int rip_ctx_create(int device, size_t hbm_budget, rip_ctx **out);
int rip_ctx_destroy(rip_ctx *ctx);
const char *rip_last_error(const rip_ctx *ctx);
int rip_sync(rip_ctx *ctx);
/* Device bytes currently held by the context (graphs, pools, scratch). */
int rip_ctx_memory(rip_ctx *ctx, size_t *used, size_t *budget);
/* Library version string, e.g. "ripples_b200 0.1.0 sm_100a". */
const char *rip_version(void);
/* The context's CUDA stream (a cudaStream_t), so callers can order their own
 * work or record timing events on it.  No reference counterpart (the reference
 * keeps one stream per GPU worker internally, streaming_rrr_generator.h:369). */
int rip_ctx_stream(rip_ctx *ctx, void **stream);
/* Number of kernels this library has launched in the process so far. */
uint64_t rip_kernel_launches(void);
/* Measured ceiling of the IC coin function on this device: coins per second
 * of a kernel that only draws coins (Philox4x32-10, four per block) the way a
 * uniform-threshold in-list is expanded, at full occupancy, no memory
 * traffic.  The roofline of the samplers on weighted-cascade graphs, which
 * are bound by this arithmetic rather than by HBM.  No reference counterpart. */
int rip_coin_rate(rip_ctx *ctx, double *coins_per_s);

/* ---- graph ---------------------------------------------------------------- */
/* Uploads a backward CSR (GraphBwd) and packs it for the kernels: weights are
 * converted once to uint32 thresholds (IC: floor(w*2^32); LT: cumulative
 * in-weight in CSR order).  Replaces make_gpu_context / gpu_graph upload
 * (include/ripples/gpu/gpu_graph.h:47-96, src/gpu/gpu_graph.cc:48-84).
 * Limits: n < 2^32 - 1, m < 2^32. */
int rip_graph_upload(rip_ctx *ctx, const uint64_t *index, const uint32_t *src,
                     const float *weights, uint32_t n, uint64_t m, int model,
                     rip_graph **out);
int rip_graph_destroy(rip_graph *g);
int rip_graph_info(const rip_graph *g, uint32_t *n, uint64_t *m, int *model);
/* Copies the packed per-edge thresholds (m values) back to the host. */
int rip_graph_thresholds(rip_graph *g, uint32_t *thr);

/* Copies the graph's backward CSR (index u64[n+1], src u32[m]) to the host. */
int rip_graph_export(rip_graph *g, uint64_t *index, uint32_t *src);

/* Device-side R-MAT draws for graphs too large to build on the host:
 * d_keys[j] = (dst << 32) | src of draw first+j, ~0 for a self-loop -- the same
 * draws as rip_rmat_csr.  d_keys is caller-owned device memory (count u64). */
int rip_rmat_keys_device(rip_ctx *ctx, uint32_t scale, uint64_t first,
                         uint64_t count, double a, double b, double c,
                         uint64_t seed, uint64_t *d_keys);
/* The same for Erdos-Renyi draws (uniform source and destination), the draws
 * of rip_er_csr. */
int rip_er_keys_device(rip_ctx *ctx, uint32_t n, uint64_t first, uint64_t count,
                       uint64_t seed, uint64_t *d_keys);
/* Builds a packed graph on the device from m sorted, unique (dst << 32 | src)
 * keys in device memory (no self-loops), with one of the RIP_WEIGHTS_* models
 * computed on the device exactly as rip_make_weights computes them. */
int rip_graph_from_keys(rip_ctx *ctx, const uint64_t *d_keys, uint64_t m,
                        uint32_t n, int weights, uint64_t weight_seed, double lo,
                        double hi, int model, rip_graph **out);

/* Builds a packed graph on the device from a host edge list -- m directed
 * edges src[e] -> dst[e] with weight w[e], as a TSV file gives them
 * (rip_read_tsv_edges) -- doing on the GPU what the reference's Graph
 * constructor and get_transpose do on the host (include/ripples/graph.h:
 * 506-620, 787-832): with `renumber`, ids become 0..n-1 in sorted order of
 * the distinct endpoints (rip_graph_id_map gives the map back), else
 * n = largest id + 1; each vertex's in-list is ordered by source id, parallel
 * edges in input order; weights are packed for `model` as rip_graph_upload
 * packs them.  The result equals rip_graph_upload of rip_read_tsv's CSR for
 * the same file.  Limits: m < 2^32 - 4, n < 2^32 - 1. */
int rip_graph_from_edges(rip_ctx *ctx, const uint32_t *src, const uint32_t *dst,
                         const float *w, uint64_t m, int renumber, int model,
                         rip_graph **out);
/* Internal id -> input id of a graph's vertices (n entries; the identity for
 * graphs not renumbered by rip_graph_from_edges), Graph::convertID's map. */
int rip_graph_id_map(const rip_graph *g, uint32_t *map);

/* ---- RRR pool --------------------------------------------------------------- */
/* A device-resident, growable flat pool of RRR sets, addressed by set id
 * 0, 1, 2, ...  Replaces RRRsets = std::vector<std::vector<uint32_t>>
 * (include/ripples/rrr_sets.h:84-105). */
int rip_pool_create(rip_ctx *ctx, rip_graph *g, rip_pool **out);
int rip_pool_destroy(rip_pool *p);
/* Drops every set (keeps the allocation). */
int rip_pool_clear(rip_pool *p);
int rip_pool_info(const rip_pool *p, uint64_t *num_sets, uint64_t *num_elements);

/* Appends `count` sets with ids num_sets .. num_sets+count-1 sampled under the
 * graph's model with the given seed.  Set contents depend only on
 * (graph, seed, set id), never on batching, sampler variant or stream order.
 * Replaces GenerateRRRSets(G, gen, begin, end, record, model_tag, ex_tag)
 * (include/ripples/generate_rrr_sets.h:186-224), whose sets were pre-inserted
 * by the caller (include/ripples/imm.h:199-200). */
int rip_sample(rip_pool *p, uint64_t seed, uint64_t count, int sampler);

/* Copies sets [first, first+count) to host buffers: offsets has count+1
 * entries (offsets[0] = 0), vertices has offsets[count] entries.  Each set is
 * sorted ascending, as AddRRRSet leaves it (include/ripples/add_rrrset.h:156).
 * Call with vertices == NULL to learn the sizes (offsets still written). */
int rip_pool_export(rip_pool *p, uint64_t first, uint64_t count,
                    uint64_t *offsets, uint32_t *vertices);
/* Appends `count` host sets (CSR: offsets[count+1], vertices).  Lets tests feed
 * the reference's own sets to the device selection. */
int rip_pool_import(rip_pool *p, const uint64_t *offsets,
                    const uint32_t *vertices, uint64_t count);
/* Appends `count` empty sets: the ids that other shards of a sharded
 * selection sample (rip_shard_*).  An empty set adds to no count and is never
 * covered.  The reference's MPI IMM gives each rank its own sets instead
 * (include/ripples/mpi/imm.h:181-190). */
int rip_pool_skip(rip_pool *p, uint64_t count);

/* Device counters of the sampling kernels since the pool was created/cleared:
 * stats[0] = vertex expansions (a vertex's in-edge list read once, whatever
 * number of sets it served), stats[1] = in-edges read, stats[2] = sets
 * written, stats[3] = pool elements written, stats[4] = per-set expansions
 * (sum over sets of vertices expanded), stats[5] = per-set in-edges
 * (sum over sets of in-edges of the expanded vertices), stats[6] = in-edges
 * of uniform-threshold lists (coins drawn against the vertex's threshold,
 * records not read; see rip_graph_uniform_thresholds), stats[7] = live edges
 * of those lists (their source id read). */
int rip_pool_stats(rip_pool *p, uint64_t stats[8]);

/* Kernel time (CUDA events on the context stream) spent in the sampler
 * launches and in rip_select since the pool was created/cleared. */
int rip_pool_timing(rip_pool *p, double *sample_kernel_ms, uint64_t *launches,
                    double *select_ms);

/* Fused-sampler knobs (what the autotuner sets): colour width 64/128/256,
 * CTA slots (0 = size from the budget), frontier-log entries per slot
 * (0 = default).  No reference counterpart: the reference fixes the colour
 * width per run (--gpu-batch-size, include/ripples/imm_configuration.h:67). */
int rip_pool_configure(rip_pool *p, uint32_t colors, uint32_t slots,
                       uint32_t log_capacity);

/* Edge-work budgets (in-edges read) after which a one-set-per-warp set, or a
 * fused CTA batch, is handed to the CTA-per-set sampler, whose 32 warps split
 * each level's edge groups (the heavy tail of IC sampling on skewed graphs);
 * 0 disables the hand-over.  Defaults 2^18 and 2^23.  Results do not depend on
 * these values. */
int rip_pool_work_caps(rip_pool *p, uint64_t plain_cap, uint64_t fused_cap);

/* Per-graph sampler autotuner.  Times sets of `seed` on a scratch pool under
 * each of RIP_TUNE_CANDIDATES IC configurations (after a warm-up run, the
 * faster of two timed runs): every candidate on the first min(pilot, 2048)
 * sets, then the candidates within twice the best of that screen on all
 * `pilot` sets (0 = 2048; large graphs want tens of thousands, so that the
 * heavy sets fill the GPU as they do at full size):
 *   0 plain (one set per warp), heavy sets past 2^18 in-edges -> grid-wide BFS
 *   1 plain, heavy past 2^14 in-edges -> grid-wide BFS
 *   2 plain, heavy past 2^18 -> one CTA per set
 *   3/4/5 fused 64/128/256 colours, batches past 2^23 -> heavy path
 *   6/7 as 0/2 with the one-set-per-warp kernel capped at 48 registers
 *       (40 resident warps per SM instead of 32)
 *   8 as 2 with 256-thread CTAs for the heavy sets (5 sets growing per SM
 *       instead of 1: the block-shape axis; candidates 0-2 use 1024-thread
 *       CTAs, 6-7 256-thread ones), 9 the same with heavy sets from 2^16
 *       in-edges
 * writes the wall times to ms[] (may be null; a candidate dropped after the
 * screen keeps its screen time) and the fastest to *choice, and
 * keeps it for the graph: pools created afterwards start from it and
 * RIP_SAMPLER_AUTO runs it.  Untuned graphs run configuration 0 for AUTO.  LT
 * graphs have one sampler (choice 0).  Sets never depend on the choice.  No
 * reference counterpart (the reference fixes its GPU colour width). */
#define RIP_TUNE_CANDIDATES 10
int rip_graph_autotune(rip_graph *g, uint64_t seed, uint32_t pilot, double *ms, int *choice);

/* Per-vertex uniform IC thresholds.  When every in-edge of a vertex has the
 * same threshold (weighted cascade, p = 1/in-degree, makes all of them so),
 * the IC samplers draw that vertex's coins against the one value and read the
 * source id of a live edge only -- not the 8-byte record of every in-edge.
 * rip_graph_upload / rip_graph_from_keys build the per-vertex array when such
 * in-lists (two or more edges) hold at least half of the edges, and turn it
 * on.  enable: 1 on, 0 off, -1 leave as is; *available (may be null): 1 when
 * the array exists.  Sets never depend on it.  No reference counterpart (the
 * reference reads each edge's weight, include/ripples/add_rrrset.h:128-135). */
int rip_graph_uniform_thresholds(rip_graph *g, int enable, int *available);
/* The branching factor of a reverse BFS on an IC graph, measured at upload:
 * the expected number of live in-edges of an edge's source,
 * sum over edges (u->v) of sum_{w->u} p(w->u), divided by m (0 for LT graphs).
 * Above 1.1 sets grow large and overlap, and untuned pools grow heavy sets with
 * the grid-wide BFS (rip_pool_heavy_batch).  No reference counterpart. */
int rip_graph_branching(const rip_graph *g, double *branching);

/* Variant of the one-set-per-warp IC kernel: 0 = no register cap (32 resident
 * warps per SM), 5 = at most 48 registers (40 warps per SM).  Results do not
 * depend on it; rip_graph_autotune chooses it per graph.  No reference
 * counterpart. */
int rip_pool_plain_occupancy(rip_pool *p, int blocks_per_sm);

/* IC sets whose edge work passes the caps above are grown either one
 * 1024-thread CTA per set or, when at least `min_sets` of them are pending,
 * 256 at a time by a multi-colour reverse BFS spread over the whole GPU (the
 * regime of supercritical graphs, where many sets hold a large share of the
 * graph and overlap).  Default 32 on IC graphs whose reverse BFS is
 * supercritical -- the expected live in-edges of an edge's source,
 * sum over edges (u->v) of sum_{w->u} p(w->u) / m, above 1.1 -- else 0
 * (weighted cascade: at most 1); 0 = always one CTA per set.  An autotuned graph's pools start from its
 * tuned value.  Results do not depend on it.  No reference counterpart (the reference's GPU BFS,
 * include/ripples/gpu/bfs.h:1338-1680, has one colour-batched path). */
int rip_pool_heavy_batch(rip_pool *p, uint32_t min_sets);

/* Block shape of the one-CTA-per-set kernel for heavy IC sets: 128, 256, 512
 * or 1024 threads, 10, 5, 2 or 1 of them resident per SM (default 256; an
 * autotuned graph's pools start from its tuned value).  Smaller CTAs grow
 * more sets per SM at once, each with fewer threads.  Results do not depend on it.  No reference counterpart. */
int rip_pool_heavy_block(rip_pool *p, uint32_t threads);

/* Reference-heap selection (RIP_TIE_REF_HEAP): after each pick the host
 * fetches the current counts of the heap items keyed at least a threshold,
 * first `percent` % of the previous gain (0 = adaptive, from the recent gain
 * ratio), then -- if no fetched item still counts that much -- the largest
 * fetched count, which covers every item the lazy pops can examine.  The seeds
 * never depend on it.  No reference counterpart: the reference keeps every
 * count on the host (streaming_find_most_influential.h:560-571). */
int rip_pool_select_guess(rip_pool *p, uint32_t percent);

/* ---- seed selection ------------------------------------------------------- */
/* Greedy max coverage over sets [0, num_sets) of the pool.  Writes up to k
 * seeds (internal ids) and their marginal coverage, *num_seeds and
 * f = covered / num_sets.  Stops early when every set is covered.  Sets are
 * not reordered.  Replaces FindMostInfluentialSet (omp_parallel_tag,
 * include/ripples/find_most_influential.h:176-196 ->
 * streaming_find_most_influential.h:607-643). */
int rip_select(rip_pool *p, uint64_t num_sets, uint32_t k, int tiebreak,
               uint32_t *seeds, uint64_t *gains, uint32_t *num_seeds,
               double *f);

/* Coverage counts (n values) as the last rip_select left them: after the
 * update that followed its last-but-one seed.  For checking the update step
 * (the reference's known-answer test, test/cuda_find_most_influential.cc:84-167). */
int rip_select_counts(rip_pool *p, uint32_t *counts);

/* Diagnostic breakdown of the rip_select calls on this pool: out[0] ms
 * enqueueing the counting/indexing kernels, out[1] ms until the heap is on
 * the host (includes those kernels), out[2] ms in the pick loop, out[3] heap
 * pops, out[4] seeds picked, out[5] candidate counts fetched, out[6]
 * selections, out[7] ms covering and fetching candidate counts (includes
 * out[10]), out[8] fetches of the whole count array, out[9] ms in heap pops,
 * out[10] ms collecting candidates on the host, out[11] fetch rounds.  The
 * heap fields are those of the reference-heap tie-break. */
int rip_select_profile(rip_pool *p, double out[12]);

/* Diagnostic: builds a heap of n random (vertex, count) entries, counts in
 * [0, max_count), with the library's level-parallel heap construction and with
 * std::make_heap; returns 1 when the two are identical element for element. */
int rip_selftest_heap(uint64_t n, uint32_t max_count, uint64_t seed);
/* Same check for the device heap build that rip_select uses. */
int rip_selftest_heap_device(rip_ctx *ctx, uint64_t n, uint32_t max_count, uint64_t seed);

/* Vertex occurrence counts over sets [0, num_sets) (n values), the first
 * step of selection (CountOccurrencies, include/ripples/counting.h:65-97). */
int rip_count(rip_pool *p, uint64_t num_sets, uint32_t *counts);

/* ---- sharded selection ------------------------------------------------------ */
/* One shard's part of a greedy lowest-id selection whose sets are split
 * across pools (one per GPU or process).  Replaces the MPI
 * FindMostInfluentialSet (include/ripples/mpi/find_most_influential.h:449-690:
 * per-pick reduction of the vertex counters, the maximum picked, every rank
 * updating its own sets).  d_sum is a device array of n uint32 (16-byte
 * aligned) on the pool's device that holds the summed counts; every call
 * returns once its work on the context stream is done, so the caller may
 * combine the shards' arrays on any stream (an all-reduce, an all-gather),
 * and must finish that before the next call reads them.
 *   rip_shard_begin: counts this pool's sets [0, num_sets) into d_sum (the
 *     caller then sums the shards' arrays) and builds its vertex -> sets
 *     index; *elements = those sets' element count.
 *   rip_shard_pick: *vertex = the largest entry of the summed d_sum, the
 *     lowest id among equal ones; *gain = its value (0: nothing left).  The
 *     maximum of every 2048 entries is kept: a pick that follows
 *     rip_shard_apply calls on the same array rescans only the entries they
 *     changed (so change it between those picks only through
 *     rip_shard_apply), any other pick rescans the whole array.
 *   Then per pick, one of two exchanges:
 *   rip_shard_cover (dense): covers this pool's uncovered sets holding
 *     `vertex` and writes its updated counts to d_sum, which the caller sums
 *     again (n values per pick, as the reference's MPI_Reduce);
 *   rip_shard_cover_list (sparse): covers them and writes their members to
 *     d_dec (capacity >= *elements of rip_shard_begin), *count of them; the
 *     caller gathers every shard's list and rip_shard_apply subtracts one per
 *     entry from the summed d_sum (the decrements only, not n values).
 *   `gain` (the pick's summed count) only sizes the cover launch.
 * Any other rip_count / rip_select on the pool ends the sharded selection. */
int rip_shard_begin(rip_pool *p, uint64_t num_sets, uint32_t *d_sum, uint64_t *elements);
int rip_shard_pick(rip_pool *p, const uint32_t *d_sum, uint32_t *vertex, uint64_t *gain);
int rip_shard_cover(rip_pool *p, uint32_t vertex, uint64_t gain, uint32_t *d_sum);
int rip_shard_cover_list(rip_pool *p, uint32_t vertex, uint64_t gain, uint32_t *d_dec,
                         uint64_t capacity, uint64_t *count);
int rip_shard_apply(rip_pool *p, uint32_t *d_sum, const uint32_t *d_dec, uint64_t count);

/* ---- IMM driver ----------------------------------------------------------- */
/* Fields mirror IMMExecutionRecord (include/ripples/imm_execution_record.h:55-92)
 * and the JSON keys of the imm tool (tools/imm.cc:104-134).  Times in ms. */
#define RIP_MAX_ROUNDS 64
typedef struct rip_imm_record {
  uint64_t theta;
  uint32_t num_rounds;
  uint64_t theta_prime_deltas[RIP_MAX_ROUNDS];
  double round_generate_ms[RIP_MAX_ROUNDS];
  double round_select_ms[RIP_MAX_ROUNDS];
  double theta_estimation_ms;
  double generate_ms;
  double select_ms;
  double total_ms;
  double f;
  uint64_t total_sets;
  uint64_t pool_elements;
  uint64_t rrr_set_bytes;
} rip_imm_record;

/* Runs IMM (martingale theta estimation, final sampling, final selection over
 * sets [0, theta)) on the device.  l is the reference's `l` argument (the imm
 * tool passes 1; the driver applies l *= 1 + 1/log2(n) as imm.h:815 does).
 * Replaces ripples::IMM (include/ripples/imm.h:768-860). */
int rip_imm(rip_ctx *ctx, rip_graph *g, uint32_t k, double epsilon, double l,
            uint64_t seed, int tiebreak, int sampler, uint32_t *seeds,
            uint32_t *num_seeds, rip_imm_record *record);

/* IMM on an existing pool: reuses the sets it holds (extending it when theta
 * needs more), as Sampling does when RR is non-empty (include/ripples/imm.h:173-177). */
int rip_imm_pool(rip_pool *p, uint32_t k, double epsilon, double l,
                 uint64_t seed, int tiebreak, int sampler, uint32_t *seeds,
                 uint32_t *num_seeds, rip_imm_record *record);

/* ---- spread of a seed set ------------------------------------------------- */
/* Forward Monte Carlo spread under IC: the mean number of vertices a seed set
 * reaches (seeds included) over `replicas` independent cascades, as the
 * replica loop of tools/simulator.cc:139-149 over ripples::simulate
 * (include/ripples/diffusion_simulation.h:73-127) measures it.
 *   g       : an IC graph uploaded with the FORWARD CSR -- index over source
 *             vertices, src[] holding each out-edge's target, weights p(u->v)
 *             (rip_graph_upload's arrays for the transposed graph).
 *   seeds   : k vertex ids < n (a repeated id counts once).
 *   sizes   : optional host array of `replicas` entries: the reached count of
 *             each replica.  Replica r is a pure function of (seed, r).
 *   levels  : optional host array of `replicas` entries: the BFS levels of
 *             each replica, the seeds' level included (the second member of
 *             the pair ripples::simulate returns).
 * Edge e fires in replica r iff P(e>>2, r; seed, SIM_IC)[e&3] < threshold(e):
 * the same distribution as the reference's uniform01 <= p(u->v) draws, not the
 * same draws.  Returns RIP_ERR_INVALID for an LT graph or a seed >= n. */
int rip_spread_ic(rip_graph *g, const uint32_t *seeds, uint32_t k,
                  uint64_t replicas, uint64_t seed, uint32_t *sizes, uint32_t *levels,
                  double *spread);
/* Forward Monte Carlo spread under LT, the live-edge form of
 * include/ripples/diffusion_simulation.h:129-178's threshold model: in replica
 * r vertex v keeps the first in-edge j (CSR order of `bwd`) with
 * P(v, 0, r; seed, SIM_LT)[0] < cum[j] (the LT sampler's cumulative
 * thresholds), or none; v is reached iff that edge's source is.
 *   fwd : the forward CSR, uploaded as an IC graph (its weights are unused).
 *   bwd : the same graph's backward CSR uploaded with RIP_MODEL_LT (the graph
 *         IMM runs on).
 * Other arguments and results as rip_spread_ic. */
int rip_spread_lt(rip_graph *fwd, rip_graph *bwd, const uint32_t *seeds, uint32_t k,
                  uint64_t replicas, uint64_t seed, uint32_t *sizes, uint32_t *levels,
                  double *spread);

/* ---- OPIM-C --------------------------------------------------------------- */
/* FindCoverage (include/ripples/opimc.h:101-118): the number of sets among the
 * pool's first num_sets holding at least one of the k seeds. */
int rip_coverage(rip_pool *p, uint64_t num_sets, const uint32_t *seeds, uint32_t k,
                 uint64_t *covered);

typedef struct rip_opimc_record {
  uint64_t theta_zero, theta_max;  /* eq. (17), (16) */
  uint64_t theta;                  /* final sets per pool */
  uint32_t rounds;                 /* selections run */
  uint64_t coverage1, coverage2;   /* of the last round: greedy on R1, seeds on R2 */
  float lower, upper;              /* the last round's bounds (eq. 5, 8) */
  double total_ms;
} rip_opimc_record;

/* OPIM-C (include/ripples/opimc.h:150-243) on two pools of one graph: R1 holds
 * the sets of key `seed`, R2 those of key seed + 0x9E3779B97F4A7C15, both
 * cleared first and grown from theta_0 sets, doubling, until the lower bound
 * of the seeds' spread (their coverage of R2) reaches (1 - 1/e - epsilon)
 * times the upper bound of the optimum (the greedy coverage of R1), or theta
 * reaches theta_max (the paper's cap; the reference has none).  Seeds are
 * picked on R1 with `tiebreak`. */
int rip_opimc_pool(rip_pool *r1, rip_pool *r2, uint32_t k, float epsilon, float delta,
                   uint64_t seed, int tiebreak, int sampler, uint32_t *seeds,
                   uint32_t *num_seeds, rip_opimc_record *record);

/* ---- batching and serving --------------------------------------------------- */
/* No counterpart in the reference (its GenerateRRRSets, include/ripples/
 * generate_rrr_sets.h:60-120, fills one instance's sets per call).  Extends
 * n_pools pools (all of this context, each listed once) by counts[i] sets of
 * seeds[i] in ONE persistent launch whose warps pull (pool, set) work items
 * from a single device counter; sets are identical to rip_sample's. */
int rip_sample_multi(rip_ctx *ctx, rip_pool *const *pools, const uint64_t *seeds,
                     const uint64_t *counts, uint32_t n_pools);

/* One IMM query for rip_imm_batch / rip_server_*.  The answer equals a fresh
 * rip_imm(graph, k, epsilon, l, seed, tiebreak) whatever it is batched with;
 * queries with equal (graph, seed) share one resident pool. */
typedef struct rip_imm_query {
  rip_graph *graph;       /* in: the graph (its model: IC or LT) */
  uint32_t k;             /* in */
  double epsilon;         /* in */
  double l;               /* in: the reference's l (the imm tool passes 1) */
  uint64_t seed;          /* in: sampler seed */
  int tiebreak;           /* in: RIP_TIE_LOWEST_ID (picks on the device, in a
                             CUDA graph) or RIP_TIE_REF_HEAP (host heap) */
  uint32_t *seeds;        /* in: caller buffer of k entries; out: the seeds */
  uint32_t num_seeds;     /* out */
  int status;             /* out: RIP_OK or an error code, once done != 0 */
  int done;               /* out: set when the query has finished */
  double f;               /* out: covered fraction of the final selection */
  double queue_ms;        /* out: submit -> admission */
  double latency_ms;      /* out: submit -> done */
  rip_imm_record record;  /* out; pool_elements/rrr_set_bytes describe the
                             shared pool */
} rip_imm_query;

/* Runs n queries to completion as one continuous batch. */
int rip_imm_batch(rip_ctx *ctx, rip_imm_query *queries, uint32_t n);

/* Request loop: queries are submitted at any time and admitted at the next
 * tick while one of max_active slots is free and the sum of the admitted
 * queries' estimated footprints (theta x mean set size, selection buffers)
 * stays within footprint_budget bytes (0 = half the context budget; a query
 * is always admitted when none is active).  Each tick samples every pool's
 * shortfall in one launch and runs one martingale round (or the final
 * selection) of every admitted query, their device picks concurrently on
 * per-slot streams.  The query struct must stay valid until done != 0. */
typedef struct rip_server rip_server;
int rip_server_create(rip_ctx *ctx, size_t footprint_budget, uint32_t max_active,
                      rip_server **out);
int rip_server_destroy(rip_server *s);
int rip_server_submit(rip_server *s, rip_imm_query *q);
int rip_server_tick(rip_server *s, uint32_t *completed);
int rip_server_pending(const rip_server *s, uint32_t *active, uint32_t *queued);
/* [0] ticks, [1] completed, [2] selection-graph launches, [3] resident pools,
 * [4] admitted footprint bytes, [5] microseconds spent in ticks, [6] times a
 * query was suspended (every admitted query waited for memory: the largest
 * went back to the queue, its pool freed, to restart later).  A query ends
 * with RIP_ERR_NOMEM only when it does not fit even alone.  [7] microseconds
 * sampling, [8] building the pools' vertex -> sets indexes, [9] indexing plus
 * selecting (host-timed, with the synchronisations they need). */
int rip_server_stats(const rip_server *s, uint64_t out[10]);

/* ---- sampling without allocation ------------------------------------------- */
/* No counterpart in the reference.  A variant of rip_sample's one-set-per-warp
 * samplers (IC BFS / LT walk) for callers that cannot allocate device memory
 * when they sample -- e.g. a serving process whose HBM is reserved up front by
 * its own arena allocator, a latency-critical loop where cudaMalloc/cudaFree
 * would synchronise the device, or a plugin host that forbids allocations
 * outside its allocator.  It calls no cudaMalloc/cudaFree: all scratch comes
 * from one file-scope device array of RIP_STATIC_SCRATCH_BYTES that every GPU
 * loading the library holds until exit.
 *   Inputs : the packed graph in caller-owned device memory -- d_off, u32[n+1]
 *            edge offsets, and d_edges, 8-byte {u32 source, u32 threshold}
 *            records, padded with zero records to a multiple of 4 plus 4 and
 *            32-byte aligned (the layout rip_graph_upload builds; thresholds as
 *            rip_graph_thresholds returns them).
 *   Outputs: caller-owned device buffers -- set s = first+i (i < count) is
 *            d_vertices[d_set_offsets[i] .. + d_set_lengths[i]) (members in
 *            discovery order, not sorted); *num_elements = elements written.
 *            Sets are bit-identical to rip_sample's for the same seed and ids.
 *   Limits : count <= RIP_STATIC_MAX_SETS per call.  IC: n such that eight
 *            warps' n-bit bitmaps plus queues fit in the array (about 24
 *            million vertices); LT walks keep no bitmap (any n; a walk may
 *            reach about 786 000 vertices).  Larger requests return
 *            RIP_ERR_LIMIT, as does a vertex_capacity too small for the sets
 *            (message from rip_static_last_error()).
 *   Speed  : the array is split into as many warps as fit (at most 32 per SM):
 *            IC gets 120 warps at n = 2^20 and 8 at n = 2^24, against the
 *            4 736 rip_sample runs on a B200, so large graphs sample far more
 *            slowly here.
 *   Rules  : the first call on a device looks up the array's address with
 *            cudaGetSymbolAddress and the device's SM count and caches
 *            both.  The cached address belongs to
 *            the device's primary context: do not call again after a
 *            cudaDeviceReset of that device.  Every call shares the array and
 *            it keeps the last call's contents (each call re-zeroes what must
 *            start at zero); calls that overlap on the GPU race, so serialise
 *            them.  `stream` is a cudaStream_t (NULL = legacy default stream);
 *            every call synchronises it before returning. */
#define RIP_STATIC_SCRATCH_BYTES (32u << 20)
#define RIP_STATIC_MAX_SETS (1u << 20)
int rip_sample_static(const uint32_t *d_off, const void *d_edges, uint32_t n,
                      uint64_t m, int model, uint64_t seed, uint64_t first,
                      uint32_t count, uint32_t *d_vertices, uint64_t vertex_capacity,
                      uint64_t *d_set_offsets, uint32_t *d_set_lengths,
                      uint64_t *num_elements, void *stream);
/* Message for the last rip_sample_static failure on the calling thread. */
const char *rip_static_last_error(void);

/* ---- theta math (host) ------------------------------------------------------ */
/* Exactly include/ripples/imm.h:77-128 and utility.h:84-87, including the
 * ssize_t / size_t truncations. */
int64_t rip_theta_prime(int64_t x, double epsilon_prime, double l, uint64_t k,
                        uint64_t n);
int64_t rip_inv_theta_prime(int64_t rr_size, double epsilon_prime, double l,
                            uint64_t k, uint64_t n);
uint64_t rip_theta(double epsilon, double l, uint64_t k, double lower_bound,
                   uint64_t n);
double rip_log_binomial(uint64_t n, uint64_t k);
/* OPIM-C sample sizes and bounds, exactly include/ripples/opimc.h:60-98 in its
 * float arithmetic: theta_max (eq. 16), theta_0 (eq. 17), the lower bound of a
 * seed set's spread from its coverage of R2 (eq. 5) and the upper bound of the
 * optimum from the greedy coverage of R1 (eq. 8). */
uint64_t rip_opimc_theta_max(uint64_t n, float epsilon, uint64_t k, float delta);
uint64_t rip_opimc_theta_zero(uint64_t n, float epsilon, uint64_t k, float delta);
float rip_opimc_lower_bound(uint64_t coverage, float delta2, uint64_t n, uint64_t theta);
float rip_opimc_upper_bound(uint64_t coverage, float delta1, uint64_t n, uint64_t theta);

/* ---- graph construction helpers (host) ------------------------------------- */
/* R-MAT (Chakrabarti, Zhan, Faloutsos, SDM'04) edge sampling with quadrant
 * probabilities a, b, c (d = 1-a-b-c), `num_edges` draws on 2^scale vertices,
 * self-loops and duplicate edges removed; returns the backward CSR in buffers
 * allocated by the library (free with rip_free).  Deterministic in seed. */
int rip_rmat_csr(uint32_t scale, uint64_t num_edges, double a, double b,
                 double c, uint64_t seed, uint64_t **index, uint32_t **src,
                 uint64_t *m);
/* Erdos-Renyi G(n, M): M directed edge draws, self-loops and duplicates
 * removed, backward CSR as above. */
int rip_er_csr(uint32_t n, uint64_t num_edges, uint64_t seed, uint64_t **index,
               uint32_t **src, uint64_t *m);
/* Fills w[m] for a backward CSR under one of RIP_WEIGHTS_*. */
int rip_make_weights(int kind, uint32_t n, const uint64_t *index, uint64_t m,
                     uint64_t seed, double lo, double hi, float *w);
/* Writes the reference binary graph format (include/ripples/graph.h:700-771)
 * for the backward CSR (backward != 0) or its transpose (backward == 0). */
int rip_write_binary(const char *path, uint32_t n, uint64_t m,
                     const uint64_t *index, const uint32_t *src,
                     const float *w, int backward);
void rip_free(void *ptr);

/* ---- graph input files (host) ---------------------------------------------- */
/* Weight distributions for unweighted TSV input (--distribution). */
enum { RIP_DIST_UNIFORM = 0, RIP_DIST_NORMAL = 1, RIP_DIST_CONST = 2 };

typedef struct rip_tsv_options {
  int weighted;     /* third column holds the weight (-w) */
  int undirected;   /* also add the reverse of every edge (-u) */
  int renumber;     /* ids to 0..n-1 in sorted order (0: --disable-renumbering) */
  int model;        /* RIP_MODEL_LT: generated weights normalised per source */
  int distribution; /* RIP_DIST_* for generated weights */
  double mean, variance, scale;  /* normal / const parameters; scale factor <= 1 */
} rip_tsv_options;

/* Reads a TSV edge list into the backward CSR (GraphBwd) the reference builds
 * from it: include/ripples/loaders.h:138-296 (parsing, generated weights and
 * their LT normalisation per source with a "not taking" mass, loaders.h:
 * 169-191) and the Graph constructor (include/ripples/graph.h:520-620:
 * renumbering, in-edges by source id).  Generated weights come from a Philox
 * stream, not trng (same distributions, not the same draws).  Outputs are
 * malloc'd arrays released with rip_free: index u64[n+1], src u32[m],
 * w f32[m], reverse_map u32[n] (internal id -> input id, Graph::convertID).
 * Returns RIP_ERR_INVALID with rip_read_error() text for an unreadable file
 * or bad options. */
int rip_read_tsv(const char *path, const rip_tsv_options *opt, uint32_t *n, uint64_t *m,
                 uint64_t **index, uint32_t **src, float **w, uint32_t **reverse_map);
/* The edge list of a TSV file before any CSR is built: parsing, generated
 * weights, undirected doubling, the LT per-source normalisation and the scale
 * factor exactly as rip_read_tsv applies them (include/ripples/loaders.h:
 * 138-196), in input ids.  Outputs are malloc'd arrays of m entries released
 * with rip_free; rip_graph_from_edges builds the graph from them on the
 * device. */
int rip_read_tsv_edges(const char *path, const rip_tsv_options *opt, uint64_t *m,
                       uint32_t **src, uint32_t **dst, float **w);
/* Reads the reference binary format (include/ripples/graph.h:854-995,
 * backward direction, float weights), weights multiplied by `scale` when it
 * is below 1.  Outputs as rip_read_tsv. */
int rip_read_binary(const char *path, double scale, uint32_t *n, uint64_t *m,
                    uint64_t **index, uint32_t **src, float **w, uint32_t **reverse_map);
/* The forward direction of the same format (the simulator's input: index
 * over sources, dst u32[m] the out-edge targets). */
int rip_read_binary_forward(const char *path, double scale, uint32_t *n, uint64_t *m,
                            uint64_t **index, uint32_t **dst, float **w, uint32_t **reverse_map);
/* The CSR of the transposed graph (include/ripples/graph.h:787-832): in-lists
 * become out-lists and back, each ordered by the other endpoint (stable),
 * weights carried along; malloc'd outputs released with rip_free. */
int rip_transpose_csr(uint32_t n, uint64_t m, const uint64_t *index, const uint32_t *adj,
                      const float *w, uint64_t **index_out, uint32_t **adj_out, float **w_out);
/* Message for the last failed rip_read_* call on the calling thread. */
const char *rip_read_error(void);

#ifdef __cplusplus
}
#endif

#endif /* RIPPLES_B200_H */
