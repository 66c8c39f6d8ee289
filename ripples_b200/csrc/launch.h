// launch.h -- host-side launchers of the device kernels (one per .cu file).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "device.cuh"

namespace rip {

// Process-wide count of kernel launches issued by this library.
uint64_t launch_counter();
void count_launches(uint64_t n);
void uncount_launches(uint64_t n);  // launches recorded into a CUDA graph, not run

// Failure ids carry this bit when a set (or fused batch) was abandoned for
// exceeding its edge-work cap rather than for lack of room.
constexpr uint32_t FAIL_BIG = 0x80000000u;

struct SampleLaunch {
  DevGraph G{};
  DevPool P{};
  Key key{};
  uint64_t first = 0;        // set id of the launch's first set (== pool set index)
  uint32_t count = 0;        // number of set indices to process
  const uint32_t *ids = nullptr;  // optional list of indices relative to `first`
  unsigned int *next = nullptr;   // work counter (zeroed by the host)
  uint32_t *bitmaps = nullptr;
  uint64_t bm_words = 0;
  uint32_t *queues = nullptr;
  uint32_t qcap = 0;
  uint64_t work_cap = 0;     // IC: abandon a set after this many in-edges (0 = none)
  FailList F{};
  Stats st{};
  int blocks = 0, threads = 0;
  int occupancy = 0;         // IC: 5 = the 48-register variant (40 warps per SM)
};

void launch_ic_plain(const SampleLaunch &L, cudaStream_t stream);

// A batch of up to 64*cw IC sets grown by the whole grid (kernels_giant.cu).
struct GiantLaunch {
  DevGraph G;
  DevPool P;
  Key key;
  RoundKeys rk{};                      // round_keys(key), filled by launch_giant
  const uint64_t *set_ids = nullptr;   // ncol set ids (colour c = set_ids[c])
  uint32_t ncol = 0;
  uint64_t *vis = nullptr, *pend = nullptr;  // n * cw words each, zero between batches
  uint32_t *pflag = nullptr;           // n, zero between batches
  uint32_t *front = nullptr, *front_next = nullptr, *touched = nullptr;  // n each
  uint64_t *masks = nullptr;           // n * cw: the current level's colours per entry
  uint32_t *ng = nullptr;              // n: coin blocks per entry
  uint64_t *goff = nullptr;            // n + 1: exclusive scan of ng
  unsigned int *ctr = nullptr;         // [0] next-frontier tail, [1] touched count
  uint32_t *sizes = nullptr, *fill = nullptr;  // per colour
  unsigned long long *starts = nullptr;        // per colour: pool offset
  unsigned long long *stats = nullptr;         // the pool's counters
};
// what: 0 seed roots, 1 level prep (n_items = frontier size), 2 expand
// (n_items = frontier size, level), 3 per-colour sizes, 4 scatter (n_items =
// touched), 5 set offsets/lengths
void launch_giant(int what, int cw, const GiantLaunch &L, uint32_t n_items, uint32_t level,
                  int blocks, cudaStream_t s);

// One IMM instance of a multi-instance launch.
struct InstanceDesc {
  DevGraph G;
  DevPool P;
  Key key;
  uint64_t first;                 // set id of the instance's first set in this launch
  uint64_t work_cap;              // IC edge-work cap per set (0 = none)
  unsigned long long *first_bad;  // the instance pool's failure bookkeeping
  unsigned long long *stats;      // the instance pool's counters [8]
  uint32_t model;
};
struct MultiLaunch {
  const InstanceDesc *inst = nullptr;
  const uint32_t *prefix = nullptr;  // n_inst + 1 exclusive prefix of the set counts
  uint32_t n_inst = 0, total = 0;
  unsigned int *next = nullptr;
  uint32_t *bitmaps = nullptr;       // per warp, bm_words (sized for the largest graph)
  uint64_t bm_words = 0;
  uint32_t *queues = nullptr;
  uint32_t qcap = 0;
  uint32_t *fail = nullptr;          // pairs (instance, rel | FAIL_BIG)
  unsigned int *fail_count = nullptr;
  int blocks = 0;
};
void launch_multi_sample(const MultiLaunch &L, cudaStream_t stream);
void launch_lt_walk(const SampleLaunch &L, cudaStream_t stream);

// Fused multi-colour IC BFS: one CTA (slot) per batch of `colors` sets.
struct FusedLaunch {
  DevGraph G;
  DevPool P;
  Key key;
  uint64_t first;
  uint32_t count;        // number of sets
  const uint32_t *order; // set indices relative to `first`, batch-major (or null)
  uint32_t num_batches;
  uint32_t colors;       // 64, 128 or 256
  unsigned int *next;    // batch counter
  uint64_t *vis;         // per slot: n * (colors/64) words, all-zero between batches
  uint64_t *pend;        // per slot: n * (colors/64) words, all-zero between batches
  uint32_t *pflag;       // per slot: n level flags, all-zero between batches
  uint32_t *log;         // per slot: lcap frontier-log entries
  uint32_t lcap;
  unsigned int *dirty;   // slots abandoned with scratch left dirty
  uint64_t work_cap = 0; // abandon a batch after this many in-edges (0 = none)
  FailList F;            // failed batch indices
  Stats st;
  int blocks;            // slots
};

// IC sets with very large edge work: one 1024-thread CTA per set, the CTA's
// warps splitting every level's edge groups (kernels_bigset.cu).
struct BigLaunch {
  DevGraph G{};
  DevPool P{};
  Key key{};
  RoundKeys rk{};                 // round_keys(key), filled by launch_ic_bigset
  uint64_t first = 0;
  uint32_t count = 0;             // entries of ids
  const uint32_t *ids = nullptr;  // set indices relative to first
  unsigned int *next = nullptr;
  uint32_t *bitmaps = nullptr;    // per CTA slot, bm_words words, all-zero between sets
  uint64_t bm_words = 0;
  uint32_t *queues = nullptr;     // per CTA slot, qcap entries
  uint32_t qcap = 0;
  FailList F{};
  Stats st{};
  int blocks = 0;
  int threads = 1024;             // block shape: 128, 256, 512 or 1024
};
// Resident CTAs per SM of each heavy-set block shape (the kernel's launch
// bounds and the number of heavy-set scratch slots per SM).
constexpr int kBigCtasPerSm(int threads) {
  return threads == 128 ? 10 : threads == 256 ? 5 : threads == 512 ? 2 : 1;
}
void launch_ic_bigset(const BigLaunch &L, cudaStream_t stream);

// Forward spread simulation (kernels_spread.cu): one CTA per replica.
struct SpreadLaunch {
  DevGraph G{};                   // forward CSR: edges[e] = {target, IC threshold}
  DevGraph B{};                   // LT only: backward CSR, edges[j] = {source, cumulative}
  Key key{};
  const uint32_t *seeds = nullptr;  // k vertex ids < n
  uint32_t k = 0;
  uint64_t replicas = 0;
  unsigned long long *next = nullptr;   // replica counter (zeroed)
  unsigned long long *total = nullptr;  // sum of reached counts (zeroed)
  uint32_t *sizes = nullptr;      // per replica reached count, or null
  uint32_t *levels = nullptr;     // per replica BFS levels (seeds' included), or null
  uint32_t *bitmaps = nullptr;    // per CTA slot, bm_words words, all-zero
  uint64_t bm_words = 0;
  uint32_t *queues = nullptr;     // per CTA slot, qcap = n entries
  uint32_t qcap = 0;
  int blocks = 0;
};
// Resident spread CTAs (one replica each at a time) per SM.
constexpr int kSpreadCtasPerSm = 4;
void launch_spread(const SpreadLaunch &L, bool lt, cudaStream_t stream);
void launch_ic_fused(const FusedLaunch &L, cudaStream_t stream);
// Resident fused CTAs per SM for a colour width (occupancy API).
int fused_ctas_per_sm(uint32_t colors);

// Synthetic graphs on the device (kernels_graphgen.cu).
inline uint32_t prob_u32_host(double p) {
  const double y = p * 4294967296.0;
  if (!(y > 0.0)) return 0u;
  if (y >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)(uint64_t)y;
}
void launch_er_keys(uint32_t n, uint64_t first, uint64_t count, uint64_t seed,
                    unsigned long long *keys, cudaStream_t stream);
void launch_rmat_keys(uint32_t scale, uint64_t first, uint64_t count, double a, double b,
                      double c, uint64_t seed, unsigned long long *keys, cudaStream_t stream);
void launch_csr_from_keys(const unsigned long long *keys, uint64_t m, uint32_t n,
                          uint64_t *index, uint32_t *src, cudaStream_t stream);
void launch_weights(int kind, const uint64_t *index, uint32_t n, uint64_t seed, double lo,
                    double hi, float *w, cudaStream_t stream);

// Graph packing.
void launch_pack_ic(const uint64_t *index, const float *w, uint32_t n,
                    uint64_t m, uint32_t *off, uint2 *edges, const uint32_t *src,
                    cudaStream_t stream);
void launch_validate_csr(const uint64_t *index, const uint32_t *src, uint32_t n, uint64_t m,
                         unsigned long long *bad, cudaStream_t stream);
void launch_pack_lt(const uint64_t *index, const float *w, uint32_t n,
                    uint64_t m, uint32_t *off, uint2 *edges, const uint32_t *src,
                    cudaStream_t stream);
// Per-vertex uniform IC thresholds (DevGraph::vthr); sums[0] = the edges they
// cover, sums[1] holds a double whose value / m is the branching factor of a
// reverse BFS (zero bits are 0.0).  lam is n floats of scratch.
void launch_uniform_threshold(const uint32_t *off, const uint2 *edges, uint32_t n, uint64_t m,
                              uint32_t *vthr, float *lam, unsigned long long *sums,
                              cudaStream_t stream);

// Selection.
void launch_count(const DevPool &P, uint64_t num_sets, uint32_t *count,
                  int blocks, cudaStream_t stream);
void launch_exclusive_scan(const uint32_t *in, uint64_t *out, uint32_t n,
                           uint64_t *block_sums, cudaStream_t stream);
size_t scan_block_sums_needed(uint32_t n);
// inv receives base + (set index in P) for every element of sets [0, num_sets)
void launch_build_inverted(const DevPool &P, uint64_t num_sets,
                           uint64_t *cursor, uint32_t *inv, int blocks,
                           cudaStream_t stream, uint64_t base = 0);
struct CoverLaunch {
  DevPool P;
  const uint64_t *inv_off;
  const uint32_t *inv;
  uint32_t vertex;
  uint8_t *covered;
  uint32_t *count;
  int blocks;
};
void launch_cover(const CoverLaunch &C, cudaStream_t stream);
// Sharded picks (keys count << 32 | ~v: the largest count, the lowest id on
// ties; counts 16-byte aligned).  cover_list: the cover, with the
// members of the newly covered sets appended to out[*cursor ...] instead of
// decremented.  apply_decrements: count[dec[i]] -= 1 (dec[i] < n), marking
// dirty[dec[i] / kPickChunk].  chunk_pick: recomputes the dirty chunks'
// maxima into cmax (clearing their flags), then *best = max over cmax.
constexpr uint32_t kPickChunk = 2048;
void launch_cover_list(const CoverLaunch &C, uint32_t *out, unsigned long long *cursor,
                       cudaStream_t stream);
void launch_apply_decrements(uint32_t *count, uint32_t n, const uint32_t *dec, uint64_t m,
                             uint8_t *dirty, int blocks, cudaStream_t stream);
void launch_chunk_pick(const uint32_t *count, uint32_t n, uint8_t *dirty,
                       unsigned long long *cmax, unsigned long long *best, cudaStream_t stream);
// The cover, then the last block gathers count[ids[i]] (i < nids) into out
// (ids and out 16-byte aligned), resets *done (a zeroed device word) and
// writes epoch to *flag (mapped).
void launch_cover_gather(const CoverLaunch &C, const uint32_t *ids, uint32_t nids,
                         uint32_t *out, unsigned int *done, unsigned int *flag,
                         unsigned int epoch, cudaStream_t stream);
// Builds the selection max-heap of {vertex, count} on the device, element for
// element the heap std::make_heap builds (level-parallel).
void launch_make_heap(const uint32_t *count, uint32_t n, uint2 *heap, cudaStream_t stream);


// Device-only lowest-id picks of one served query (lives in device memory).
constexpr uint32_t SEL_MAX_SEGMENTS = 8;
struct SelDesc {
  DevPool P;                       // the pool the query draws from
  // vertex -> sets index of the pool, as up to SEL_MAX_SEGMENTS segments, each
  // over a range of set ids [seg_first[g], ...): v's sets in segment g are
  // seg_inv[g][seg_off[g][v] .. seg_off[g][v + 1])
  const uint64_t *seg_off[SEL_MAX_SEGMENTS];
  const uint32_t *seg_inv[SEL_MAX_SEGMENTS];
  uint64_t seg_first[SEL_MAX_SEGMENTS];
  uint32_t nseg;
  uint64_t S;                      // select over sets [0, S)
  uint32_t n, nchunks;             // vertices; chunks of sel_chunk_vertices()
  uint32_t k;                      // picks
  uint32_t keep_counts;            // 1: count and covered are already set up
  uint32_t *count;                 // nchunks * chunk entries (tail stays 0)
  unsigned long long *cmax;        // per chunk: max key
  uint8_t *dirty;                  // per chunk
  uint8_t *covered;                // >= S rounded up to 16 bytes
  unsigned long long *best;        // k keys: count << 32 | ~vertex
  unsigned int *done_blocks;       // last-block counter of sel_pick
  unsigned long long *acc;         // [2] elements of the sets still uncovered,
                                   // [3] sets still uncovered, [4] cover mode
                                   // of the current pick (1 = recount)
  uint64_t total_elems;            // elements of sets [0, S) (keep_counts)
};
// Sets of [0, S) holding a vertex whose bit is set in `marked` (n bits).
void launch_coverage(const DevPool &P, uint64_t S, const uint32_t *marked,
                     unsigned long long *covered, int blocks, cudaStream_t stream);
void launch_sel_init(const SelDesc *d, int blocks, cudaStream_t stream);
void launch_sel_count(const SelDesc *d, int blocks, cudaStream_t stream);
void launch_sel_pick(const SelDesc *d, uint32_t i, int blocks, cudaStream_t stream);
// Covers pick i's sets: marks them and decrements their members' counts or --
// when they hold more elements than every set still uncovered -- recounts the
// uncovered sets (2 launches; the pick decides which, on the device).
void launch_sel_cover(const SelDesc *d, uint32_t i, int blocks, cudaStream_t stream);
uint32_t sel_chunk_vertices();
// out[i] = count[ids[i]], i < m (ids and out 16-byte aligned)
void launch_gather_counts(const uint32_t *count, const uint32_t *ids, uint32_t m,
                          uint32_t *out, cudaStream_t stream);

// Copies sets [first, first+count) into out[csr[i] ..] in set-id order.
void launch_gather_sets(const DevPool &P, uint64_t first, uint64_t count,
                        const uint64_t *csr, uint32_t *out, cudaStream_t s);

}  // namespace rip
