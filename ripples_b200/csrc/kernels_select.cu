// kernels_select.cu -- greedy max-coverage building blocks for sm_100a.
//
// count_kernel      vertex-occurrence histogram over sets [0, S)
//                   (CountOccurrencies, include/ripples/counting.h:65-97;
//                   reference GPU kernel_count, src/gpu/find_most_influential.cc:56-63)
//                   with warp-aggregated atomics: __match_any_sync groups
//                   lanes holding the same vertex and one leader adds the
//                   group size.
// inverted_kernel   vertex -> sets index (a CSR transpose of the pool), built
//                   once per selection so each pick touches only the sets that
//                   contain the seed, instead of re-scanning the pool
//                   (update_mask_kernel + count_uncovered_kernel,
//                   src/gpu/find_most_influential.cc:74-98).
// cover_kernel      after a reference-heap pick: marks the seed's
//                   still-uncovered sets covered and decrements the counts of
//                   their members (UpdateCounters,
//                   include/ripples/counting.h:141-151).
// gather_counts     the counts of the heap items a reference-heap pick can
//                   examine, into mapped host memory.
// heap kernels      the selection max-heap built on the device, level by
//                   level, element for element the one std::make_heap builds.
// sel_* kernels     lowest-id picks entirely on the device (max count, lowest
//                   vertex id on ties, as thrust::max_element in
//                   src/gpu/find_most_influential.cc:65-72): cached chunk
//                   maxima, cover by decrement or recount.
//
// All per-set loops use the same warp-level load balancing: a warp takes 32
// sets, scans their lengths and walks the concatenated elements 32 at a time,
// each lane finding its set with a 5-step shuffle search.
#include <algorithm>

#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

constexpr uint32_t NONE = 0xFFFFFFFFu;

// Iterates the elements of 32 sets per warp.  `set_of(i)` returns the set
// index for lane i of the current 32-set window (or a value >= limit for
// none); `fn(set, vertex, valid)` is called by ALL lanes (valid says whether
// the lane holds an element) so it may use warp collectives.
template <typename SetOf, typename Fn>
__device__ __forceinline__ void for_each_element(const DevPool &P,
                                                 uint64_t window_base,
                                                 uint64_t limit, SetOf set_of,
                                                 Fn fn) {
  const uint32_t lane = lane_id();
  const uint64_t sidx = window_base + lane;
  uint64_t s = 0;
  uint32_t len = 0;
  uint64_t off = 0;
  if (sidx < limit) {
    s = set_of(sidx);
    if (s != ~0ull) {
      len = P.set_len[s];
      off = P.set_off[s];
    }
  }
  const uint32_t incl = warp_incl_scan(len);
  const uint32_t total = __shfl_sync(FULL, incl, 31);
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t j = base + lane;
    const bool valid = j < total;
    const uint32_t owner = warp_find_owner(incl, valid ? j : total - 1);
    const uint64_t ooff = __shfl_sync(FULL, off, owner);
    const uint32_t oexcl =
        __shfl_sync(FULL, incl, owner) - __shfl_sync(FULL, len, owner);
    const uint64_t os = __shfl_sync(FULL, s, owner);
    const uint32_t v = valid ? P.vtx[ooff + (j - oexcl)] : NONE;
    fn(os, v, valid);
  }
}

// One occurrence per valid lane, called by all lanes of the warp.  When the
// warp's 32 elements come from one set they are distinct vertices (a set
// holds each vertex once) and every lane adds 1; otherwise lanes holding the
// same vertex are grouped with __match_any_sync and one leader adds the group
// size.  Lanes past the last element carry the last set's id.
__device__ __forceinline__ void add_occurrence(uint32_t *count, uint64_t s, uint32_t v,
                                               bool valid) {
  if (__shfl_sync(FULL, s, 0) == __shfl_sync(FULL, s, 31)) {
    if (valid) atomicAdd(count + v, 1u);
    return;
  }
  const uint32_t peers = __match_any_sync(FULL, v);
  if (valid && (__ffs(peers) - 1) == (int)lane_id())
    atomicAdd(count + v, (uint32_t)__popc(peers));
}

__global__ void __launch_bounds__(256)
count_kernel(DevPool P, uint64_t S, uint32_t *count) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t wb = gw * 32; wb < S; wb += nw * 32) {
    for_each_element(
        P, wb, S, [](uint64_t i) { return i; },
        [&](uint64_t s, uint32_t v, bool valid) { add_occurrence(count, s, v, valid); });
  }
}

// Sets of [0, S) holding at least one marked vertex (OPIM-C's FindCoverage,
// include/ripples/opimc.h:101-118): bit (s - window) of `hit` is set when a
// member of set s is marked; each warp adds the covered sets of its window.
__global__ void __launch_bounds__(256)
coverage_kernel(DevPool P, uint64_t S, const uint32_t *marked, unsigned long long *covered) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long mine = 0;
  for (uint64_t wb = gw * 32; wb < S; wb += nw * 32) {
    uint32_t hit = 0;
    for_each_element(
        P, wb, S, [](uint64_t i) { return i; },
        [&](uint64_t s, uint32_t v, bool valid) {
          const bool m = valid && ((__ldg(marked + (v >> 5)) >> (v & 31)) & 1u);
          hit |= __reduce_or_sync(FULL, m ? 1u << (uint32_t)(s - wb) : 0u);
        });
    mine += __popc(hit);
  }
  if (lane_id() == 0 && mine) atomicAdd(covered, mine);
}

__global__ void __launch_bounds__(256)
inverted_kernel(DevPool P, uint64_t S, uint64_t *cursor, uint32_t *inv, uint64_t base) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t wb = gw * 32; wb < S; wb += nw * 32) {
    for_each_element(
        P, wb, S, [](uint64_t i) { return i; },
        [&](uint64_t s, uint32_t v, bool valid) {
          if (__shfl_sync(FULL, s, 0) == __shfl_sync(FULL, s, 31)) {  // distinct vertices
            if (valid)
              inv[atomicAdd((unsigned long long *)cursor + v, 1ull)] = (uint32_t)(base + s);
            return;
          }
          const uint32_t peers = __match_any_sync(FULL, v);
          const uint32_t leader = __ffs(peers) - 1;
          unsigned long long b = 0;
          if (valid && leader == lane_id())
            b = atomicAdd((unsigned long long *)cursor + v,
                          (unsigned long long)__popc(peers));
          b = __shfl_sync(FULL, b, leader);
          if (valid) inv[b + __popc(peers & lanemask_lt())] = (uint32_t)(base + s);
        });
  }
}

// One warp per set of the seed's inverted list.  A set holds each vertex
// once, so its members are decremented with plain reductions (no result
// needed, nothing to aggregate).
__global__ void __launch_bounds__(256) cover_kernel(CoverLaunch C) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = lane_id();
  const uint64_t lo = C.inv_off[C.vertex], hi = C.inv_off[C.vertex + 1];
  for (uint64_t i = lo + gw; i < hi; i += nw) {
    const uint32_t s = C.inv[i];
    if (C.covered[s]) continue;  // covered by an earlier seed (warp-uniform)
    const uint32_t len = C.P.set_len[s];
    const uint64_t off = C.P.set_off[s];
    if (lane == 0) C.covered[s] = 1;  // s holds the vertex once: no other warp has s
    for (uint32_t j = lane; j < len; j += 32) atomicSub(C.count + C.P.vtx[off + j], 1u);
  }
}

// The pick of a sharded selection over the summed counts: the largest
// count << 32 | ~v, i.e. the largest count and the lowest vertex id among
// equal counts (thrust::max_element over the reduced counters,
// include/ripples/mpi/find_most_influential.h:505-511).
__device__ __forceinline__ unsigned long long pick_key(uint32_t c, uint32_t v) {
  return (unsigned long long)c << 32 | (uint32_t)~v;
}

// A sharded pick's cover with its decrements listed instead of applied:
// marks this shard's uncovered sets holding the vertex covered and appends
// their members to `out` (each entry: that vertex's summed count drops by
// one), a warp per set as cover_kernel.  At most the shard's element count
// is written.
__global__ void __launch_bounds__(256) cover_list_kernel(CoverLaunch C, uint32_t *out,
                                                         unsigned long long *cursor) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = lane_id();
  const uint64_t lo = C.inv_off[C.vertex], hi = C.inv_off[C.vertex + 1];
  for (uint64_t i = lo + gw; i < hi; i += nw) {
    const uint32_t s = C.inv[i];
    if (C.covered[s]) continue;  // warp-uniform
    const uint32_t len = C.P.set_len[s];
    const uint64_t off = C.P.set_off[s];
    unsigned long long b = 0;
    if (lane == 0) {
      C.covered[s] = 1;
      b = atomicAdd(cursor, (unsigned long long)len);
    }
    b = __shfl_sync(FULL, b, 0);
    for (uint32_t j = lane; j < len; j += 32) out[b + j] = C.P.vtx[off + j];
  }
}

// Summed counts minus the listed decrements; marks the chunks they touch for
// the next pick (entries >= n are skipped).
__global__ void __launch_bounds__(256) apply_decrements_kernel(uint32_t *count, uint32_t n,
                                                               const uint32_t *dec, uint64_t m,
                                                               uint8_t *dirty) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint32_t v = dec[i];
    if (v < n) {
      atomicSub(count + v, 1u);
      dirty[v / kPickChunk] = 1;
    }
  }
}

// The pick key maximum of every dirty chunk of kPickChunk counts, one block
// per chunk (clean chunks return at once); clears the chunk's flag.
__global__ void __launch_bounds__(256) chunk_max_kernel(const uint32_t *__restrict__ count,
                                                        uint32_t n, uint8_t *dirty,
                                                        unsigned long long *cmax) {
  const uint32_t chunk = blockIdx.x;
  if (!dirty[chunk]) return;
  const uint32_t lo = chunk * kPickChunk;
  const uint32_t hi = min(n, lo + kPickChunk);
  unsigned long long key = 0;
  if (hi - lo == kPickChunk) {  // whole chunk: 16-byte loads (count 16-byte aligned)
    const uint4 *c4 = reinterpret_cast<const uint4 *>(count + lo);
    for (uint32_t i = threadIdx.x; i < kPickChunk / 4; i += blockDim.x) {
      const uint4 q = c4[i];
      const uint32_t v = lo + i * 4;
      key = max(key, pick_key(q.x, v));
      key = max(key, pick_key(q.y, v + 1));
      key = max(key, pick_key(q.z, v + 2));
      key = max(key, pick_key(q.w, v + 3));
    }
  } else {
    for (uint32_t v = lo + threadIdx.x; v < hi; v += blockDim.x) key = max(key, pick_key(count[v], v));
  }
  for (int o = 16; o; o >>= 1) key = max(key, __shfl_xor_sync(FULL, key, o));
  __shared__ unsigned long long s_key[8];
  const uint32_t warp = threadIdx.x >> 5;
  if (lane_id() == 0) s_key[warp] = key;
  __syncthreads();
  if (warp == 0) {
    key = lane_id() < (blockDim.x >> 5) ? s_key[lane_id()] : 0ull;
    for (int o = 4; o; o >>= 1) key = max(key, __shfl_xor_sync(FULL, key, o));
    if (lane_id() == 0) {
      cmax[chunk] = key;
      dirty[chunk] = 0;
    }
  }
}

// *best = the maximum of cmax[0, nchunks) (one block).
__global__ void __launch_bounds__(1024) cmax_max_kernel(const unsigned long long *cmax,
                                                        uint32_t nchunks,
                                                        unsigned long long *best) {
  unsigned long long key = 0;
  for (uint32_t i = threadIdx.x; i < nchunks; i += blockDim.x) key = max(key, cmax[i]);
  for (int o = 16; o; o >>= 1) key = max(key, __shfl_xor_sync(FULL, key, o));
  __shared__ unsigned long long s_key[32];
  const uint32_t warp = threadIdx.x >> 5;
  if (lane_id() == 0) s_key[warp] = key;
  __syncthreads();
  if (warp == 0) {
    key = lane_id() < (blockDim.x >> 5) ? s_key[lane_id()] : 0ull;
    for (int o = 16; o; o >>= 1) key = max(key, __shfl_xor_sync(FULL, key, o));
    if (lane_id() == 0) *best = key;
  }
}

// A reference-heap pick in one launch: cover_kernel's work, then the last
// block to finish (a completion ticket in *done) gathers the current counts of
// the host's candidates for the next pick into `out` (mapped host memory),
// resets the ticket and publishes `epoch` in *flag after a system-wide fence,
// so the host polls one word instead of synchronising the stream.
__global__ void __launch_bounds__(256) cover_gather_kernel(CoverLaunch C, const uint32_t *ids,
                                                           uint32_t nids, uint32_t *out,
                                                           unsigned int *done,
                                                           volatile unsigned int *flag,
                                                           unsigned int epoch) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = lane_id();
  const uint64_t lo = C.inv_off[C.vertex], hi = C.inv_off[C.vertex + 1];
  for (uint64_t i = lo + gw; i < hi; i += nw) {
    const uint32_t s = C.inv[i];
    if (C.covered[s]) continue;
    const uint32_t len = C.P.set_len[s];
    const uint64_t off = C.P.set_off[s];
    if (lane == 0) C.covered[s] = 1;
    for (uint32_t j = lane; j < len; j += 32) atomicSub(C.count + C.P.vtx[off + j], 1u);
  }
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // this block's decrements before its ticket
    s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();  // every other block's decrements are visible from here
  // ids and out sit in mapped host memory (16-byte aligned): four ids a
  // read, so that a 2048-id gather is two rounds over the bus per thread
  const uint32_t n4 = nids >> 2;
  const uint4 *ids4 = reinterpret_cast<const uint4 *>(ids);
  uint4 *out4 = reinterpret_cast<uint4 *>(out);
  for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) {
    const uint4 v = ids4[i];
    out4[i] = make_uint4(__ldcg(C.count + v.x), __ldcg(C.count + v.y), __ldcg(C.count + v.z),
                         __ldcg(C.count + v.w));
  }
  for (uint32_t i = (n4 << 2) + threadIdx.x; i < nids; i += blockDim.x)
    out[i] = __ldcg(C.count + ids[i]);
  __syncthreads();
  if (threadIdx.x == 0) {
    *done = 0u;
    __threadfence_system();
    *flag = epoch;
  }
}

// ---- device-only picks (served queries) -----------------------------------
// Every kernel reads its buffers from a SelDesc in device memory, so one
// captured CUDA graph serves every round of a query: the host rewrites the
// descriptor (S, buffers) and replays the graph.  Picks keep the lowest-id
// tie-break: key(v) = count[v] << 32 | ~v, the maximum key wins.  The count
// array is split into chunks of SEL_CHUNK vertices with a cached maximum key
// each; a cover marks the chunks it decrements dirty and the next pick
// re-reads only those, then reduces the chunk maxima in the last block.
constexpr uint32_t SEL_CHUNK = 1024;

__device__ __forceinline__ unsigned long long sel_key(uint32_t c, uint32_t v) {
  return ((unsigned long long)c << 32) | (unsigned long long)(~v);
}
__device__ __forceinline__ unsigned long long umax64(unsigned long long a,
                                                     unsigned long long b) {
  return a > b ? a : b;
}

__global__ void __launch_bounds__(256) sel_init_kernel(const SelDesc *__restrict__ dp) {
  const SelDesc d = *dp;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  if (!d.keep_counts) {
    const uint64_t n4 = (uint64_t)d.nchunks * (SEL_CHUNK / 4);
    uint4 *c4 = reinterpret_cast<uint4 *>(d.count);
    for (uint64_t i = tid; i < n4; i += stride) c4[i] = make_uint4(0, 0, 0, 0);
    const uint64_t s16 = (d.S + 15) / 16;
    uint4 *cv = reinterpret_cast<uint4 *>(d.covered);
    for (uint64_t i = tid; i < s16; i += stride) cv[i] = make_uint4(0, 0, 0, 0);
  }
  for (uint64_t i = tid; i < d.nchunks; i += stride) d.dirty[i] = 1;
  for (uint64_t i = tid; i < d.k; i += stride) d.best[i] = 0ull;
  if (tid == 0) {
    *d.done_blocks = 0;
    d.acc[2] = d.keep_counts ? d.total_elems : 0ull;
    d.acc[3] = d.S;  // sets still uncovered
    d.acc[4] = 0ull;
  }
}

__global__ void __launch_bounds__(256) sel_count_kernel(const SelDesc *__restrict__ dp) {
  const SelDesc d = *dp;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long elems = 0;
  for (uint64_t wb = gw * 32; wb < d.S; wb += nw * 32) {
    for_each_element(
        d.P, wb, d.S, [](uint64_t i) { return i; },
        [&](uint64_t s, uint32_t v, bool valid) {
          add_occurrence(d.count, s, v, valid);
          elems += valid ? 1 : 0;
        });
  }
  elems = warp_sum_u64(elems);
  if (lane_id() == 0 && elems) atomicAdd(d.acc + 2, elems);
}

// Pick i: refresh the dirty chunk maxima (one warp per chunk), then the last
// block to finish reduces all chunk maxima into best[i].
__global__ void __launch_bounds__(256) sel_pick_kernel(const SelDesc *__restrict__ dp,
                                                       uint32_t i) {
  __shared__ unsigned long long s_red[8];
  __shared__ bool s_last;
  const SelDesc d = *dp;
  if (i > 0 && (d.best[i - 1] >> 32) == 0) return;  // everything covered
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t c = gw; c < d.nchunks; c += nw) {
    if (!d.dirty[c]) continue;  // warp-uniform
    const uint4 *src = reinterpret_cast<const uint4 *>(d.count + c * SEL_CHUNK);
    unsigned long long key = 0;
#pragma unroll
    for (uint32_t j = 0; j < SEL_CHUNK / 128; ++j) {
      const uint32_t q = j * 32 + lane;
      const uint4 x = __ldcg(src + q);
      const uint32_t v = (uint32_t)(c * SEL_CHUNK) + 4 * q;
      key = umax64(key, umax64(umax64(sel_key(x.x, v), sel_key(x.y, v + 1)),
                               umax64(sel_key(x.z, v + 2), sel_key(x.w, v + 3))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) key = umax64(key, __shfl_xor_sync(FULL, key, o));
    if (lane == 0) {
      d.cmax[c] = key;
      d.dirty[c] = 0;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(d.done_blocks, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  unsigned long long key = 0;
  for (uint64_t c = threadIdx.x; c < d.nchunks; c += blockDim.x)
    key = umax64(key, __ldcg(d.cmax + c));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) key = umax64(key, __shfl_xor_sync(FULL, key, o));
  if (lane == 0) s_red[wid] = key;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = umax64(b, s_red[w]);
    d.best[i] = b;
    *d.done_blocks = 0;
    // how the cover of this pick runs: its g sets hold about g x the mean
    // uncovered set size; when that outweighs the rest, recounting the rest
    // is less work than decrementing (either way the counts are exact)
    const unsigned long long g = b >> 32, left = d.acc[2], sets = d.acc[3];
    const unsigned long long est = sets ? (unsigned long long)((double)g * (double)left /
                                                               (double)sets)
                                        : 0ull;
    d.acc[4] = (est > (left > est ? left - est : 0ull) + d.n / 4) ? 1ull : 0ull;
    d.acc[3] = sets > g ? sets - g : 0ull;
  }
}

// After pick i: mark the seed's still-uncovered sets in [0, S) covered (every
// index segment).  Decrement mode (the pick's choice in acc[4] = 0): one warp
// per set decrements its members and marks their chunks dirty.  Recount
// mode: the sets are only marked, every count is cleared and every chunk
// marked dirty, and sel_recount_kernel counts the sets left.  Both subtract
// the covered sets' elements from acc[2] (elements of uncovered sets).
__global__ void __launch_bounds__(256) sel_cover_kernel(const SelDesc *__restrict__ dp,
                                                        uint32_t i) {
  const SelDesc d = *dp;
  const unsigned long long b = d.best[i];
  if ((b >> 32) == 0) return;
  const uint32_t v = ~(uint32_t)(b & 0xFFFFFFFFull);
  const bool recount = d.acc[4] != 0ull;
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t gw = tid >> 5, nw = stride >> 5;
  const uint32_t lane = lane_id();
  unsigned long long elems = 0;
  if (recount) {
    uint4 *c4 = reinterpret_cast<uint4 *>(d.count);
    const uint64_t n4 = (uint64_t)d.nchunks * (SEL_CHUNK / 4);
    for (uint64_t x = tid; x < n4; x += stride) c4[x] = make_uint4(0, 0, 0, 0);
    for (uint64_t x = tid; x < d.nchunks; x += stride) d.dirty[x] = 1;
  }
  for (uint32_t g = 0; g < d.nseg; ++g) {
    if (d.seg_first[g] >= d.S) continue;  // the segment's sets are all >= S
    const uint64_t lo = d.seg_off[g][v], hi = d.seg_off[g][v + 1];
    if (recount) {  // one thread per entry: mark only
      for (uint64_t j = lo + tid; j < hi; j += stride) {
        const uint32_t s = d.seg_inv[g][j];
        if (s < d.S && !d.covered[s]) {  // s holds v once: no other thread has s
          d.covered[s] = 1;
          elems += d.P.set_len[s];
        }
      }
      continue;
    }
    for (uint64_t j = lo + gw; j < hi; j += nw) {  // one warp per entry
      const uint32_t s = d.seg_inv[g][j];
      if (s >= d.S || d.covered[s]) continue;  // warp-uniform
      const uint32_t len = d.P.set_len[s];
      const uint64_t so = d.P.set_off[s];
      if (lane == 0) {
        d.covered[s] = 1;
        elems += len;
      }
      for (uint32_t e = lane; e < len; e += 32) {
        const uint32_t u = d.P.vtx[so + e];
        atomicSub(d.count + u, 1u);
        d.dirty[u / SEL_CHUNK] = 1;
      }
    }
  }
  elems = warp_sum_u64(elems);
  if (lane == 0 && elems) atomicAdd(d.acc + 2, (unsigned long long)0 - elems);  // acc[2] -= elems
}

// Recount mode only: count the members of every set in [0, S) still
// uncovered.
__global__ void __launch_bounds__(256) sel_recount_kernel(const SelDesc *__restrict__ dp) {
  const SelDesc d = *dp;
  if (d.acc[4] == 0ull) return;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t wb = gw * 32; wb < d.S; wb += nw * 32) {
    for_each_element(
        d.P, wb, d.S, [&](uint64_t x) { return d.covered[x] ? ~0ull : x; },
        [&](uint64_t s, uint32_t v, bool valid) { add_occurrence(d.count, s, v, valid); });
  }
}

// out[i] = count[ids[i]] (ids and out may live in mapped host memory)
__global__ void gather_counts_kernel(const uint32_t *__restrict__ count,
                                     const uint32_t *ids, uint32_t m, uint32_t *out) {
  // ids and out in mapped host memory (16-byte aligned): four ids a read
  const uint32_t m4 = m >> 2;
  const uint4 *ids4 = reinterpret_cast<const uint4 *>(ids);
  uint4 *out4 = reinterpret_cast<uint4 *>(out);
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m4; i += stride) {
    const uint4 v = ids4[i];
    out4[i] = make_uint4(count[v.x], count[v.y], count[v.z], count[v.w]);
  }
  for (uint32_t i = (m4 << 2) + blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    out[i] = count[ids[i]];
}

// ---- exclusive scan of u32 counts into u64 offsets (n+1 outputs) ----------
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr uint32_t SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ unsigned long long block_excl_scan(unsigned long long x,
                                              unsigned long long *warp_tot,
                                              unsigned long long *total) {
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
  unsigned long long incl = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long y = __shfl_up_sync(FULL, incl, d);
    if (lane >= (uint32_t)d) incl += y;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    unsigned long long t = lane < (blockDim.x >> 5) ? warp_tot[lane] : 0;
    unsigned long long ti = t;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long y = __shfl_up_sync(FULL, ti, d);
      if (lane >= (uint32_t)d) ti += y;
    }
    warp_tot[lane] = ti - t;
    if (lane == 31) *total = ti;
  }
  __syncthreads();
  const unsigned long long r = warp_tot[wid] + incl - x;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(SCAN_THREADS)
scan_tiles_kernel(const uint32_t *in, uint32_t n, uint64_t *tile_sums) {
  __shared__ unsigned long long wt[32];
  __shared__ unsigned long long tot;
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  unsigned long long s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i)
    if (base + i < n) s += in[base + i];
  block_excl_scan(s, wt, &tot);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS)
scan_sums_kernel(uint64_t *tile_sums, uint32_t tiles) {
  __shared__ unsigned long long wt[32];
  __shared__ unsigned long long tot;
  unsigned long long carry = 0;
  for (uint32_t b = 0; b < tiles; b += SCAN_THREADS) {
    const uint32_t i = b + threadIdx.x;
    const unsigned long long x = i < tiles ? tile_sums[i] : 0;
    const unsigned long long ex = block_excl_scan(x, wt, &tot);
    if (i < tiles) tile_sums[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_sums[tiles] = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS)
scan_apply_kernel(const uint32_t *in, uint32_t n, const uint64_t *tile_sums,
                  uint64_t *out) {
  __shared__ unsigned long long wt[32];
  __shared__ unsigned long long tot;
  const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  unsigned long long s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    v[i] = base + i < n ? in[base + i] : 0u;
    s += v[i];
  }
  unsigned long long ex = block_excl_scan(s, wt, &tot) + tile_sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    if (base + i < n) out[base + i] = ex;
    ex += v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
    const uint32_t tiles = gridDim.x;
    out[n] = tile_sums[tiles];
  }
}

// libstdc++-compatible sift of make_heap: the hole at `hole` sinks to a leaf
// along the larger child (the right one unless the left is strictly larger),
// then `value` rises from there while its parent compares less.  Elements are
// {vertex, count}; only counts are compared.
__device__ void adjust_heap_dev(uint2 *h, int64_t hole, int64_t len, uint2 value) {
  const int64_t top = hole;
  int64_t child = hole;
  while (child < (len - 1) / 2) {
    child = 2 * (child + 1);
    if (h[child].y < h[child - 1].y) child--;
    h[hole] = h[child];
    hole = child;
  }
  if ((len & 1) == 0 && child == (len - 2) / 2) {
    child = 2 * (child + 1);
    h[hole] = h[child - 1];
    hole = child - 1;
  }
  int64_t parent = (hole - 1) / 2;
  while (hole > top && h[parent].y < value.y) {
    h[hole] = h[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  h[hole] = value;
}

// heap[v] = {v, count[v]}
__global__ void heap_fill_kernel(const uint32_t *count, uint32_t n, uint2 *heap) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    heap[v] = make_uint2(v, count[v]);
}

// make_heap's parents [lo, hi] (one depth) in parallel: disjoint subtrees.
__global__ void heap_level_kernel(uint2 *heap, int64_t len, int64_t lo, int64_t hi) {
  for (int64_t p = hi - (int64_t)(blockIdx.x * blockDim.x + threadIdx.x); p >= lo;
       p -= (int64_t)gridDim.x * blockDim.x)
    adjust_heap_dev(heap, p, len, heap[p]);
}

}  // namespace

void launch_make_heap(const uint32_t *count, uint32_t n, uint2 *heap, cudaStream_t stream) {
  count_launches(1);
  heap_fill_kernel<<<592, 256, 0, stream>>>(count, n, heap);
  const int64_t len = n;
  if (len < 2) return;
  const int64_t last_parent = (len - 2) / 2;
  int dmax = 0;
  while ((((int64_t)2) << dmax) - 1 <= last_parent) ++dmax;
  for (int d = dmax; d >= 0; --d) {
    const int64_t lo = (((int64_t)1) << d) - 1;
    const int64_t hi = std::min<int64_t>(last_parent, (((int64_t)2) << d) - 2);
    const int blocks = (int)std::min<int64_t>(1184, (hi - lo + 1 + 255) / 256);
    count_launches(1);
    heap_level_kernel<<<blocks, 256, 0, stream>>>(heap, len, lo, hi);
  }
}

void launch_count(const DevPool &P, uint64_t num_sets, uint32_t *count,
                  int blocks, cudaStream_t stream) {
  count_launches(1);
  count_kernel<<<blocks, 256, 0, stream>>>(P, num_sets, count);
}

size_t scan_block_sums_needed(uint32_t n) {
  return (size_t)((uint64_t)n + SCAN_TILE - 1) / SCAN_TILE + 1;
}

void launch_exclusive_scan(const uint32_t *in, uint64_t *out, uint32_t n,
                           uint64_t *block_sums, cudaStream_t stream) {
  count_launches(3);
  const uint32_t tiles = (uint32_t)((n + (uint64_t)SCAN_TILE - 1) / SCAN_TILE);
  if (tiles == 0) {
    cudaMemsetAsync(out, 0, sizeof(uint64_t), stream);
    return;
  }
  scan_tiles_kernel<<<tiles, SCAN_THREADS, 0, stream>>>(in, n, block_sums);
  scan_sums_kernel<<<1, SCAN_THREADS, 0, stream>>>(block_sums, tiles);
  scan_apply_kernel<<<tiles, SCAN_THREADS, 0, stream>>>(in, n, block_sums, out);
}

void launch_build_inverted(const DevPool &P, uint64_t num_sets,
                           uint64_t *cursor, uint32_t *inv, int blocks,
                           cudaStream_t stream, uint64_t base) {
  count_launches(1);
  inverted_kernel<<<blocks, 256, 0, stream>>>(P, num_sets, cursor, inv, base);
}

void launch_cover(const CoverLaunch &C, cudaStream_t stream) {
  count_launches(1);
  cover_kernel<<<C.blocks, 256, 0, stream>>>(C);
}

void launch_cover_list(const CoverLaunch &C, uint32_t *out, unsigned long long *cursor,
                       cudaStream_t stream) {
  count_launches(1);
  cover_list_kernel<<<C.blocks, 256, 0, stream>>>(C, out, cursor);
}

void launch_apply_decrements(uint32_t *count, uint32_t n, const uint32_t *dec, uint64_t m,
                             uint8_t *dirty, int blocks, cudaStream_t stream) {
  count_launches(1);
  apply_decrements_kernel<<<blocks, 256, 0, stream>>>(count, n, dec, m, dirty);
}

void launch_chunk_pick(const uint32_t *count, uint32_t n, uint8_t *dirty,
                       unsigned long long *cmax, unsigned long long *best, cudaStream_t stream) {
  const uint32_t nchunks = (n + kPickChunk - 1) / kPickChunk;
  count_launches(2);
  chunk_max_kernel<<<nchunks, 256, 0, stream>>>(count, n, dirty, cmax);
  cmax_max_kernel<<<1, 1024, 0, stream>>>(cmax, nchunks, best);
}

void launch_cover_gather(const CoverLaunch &C, const uint32_t *ids, uint32_t nids,
                         uint32_t *out, unsigned int *done, unsigned int *flag,
                         unsigned int epoch, cudaStream_t stream) {
  count_launches(1);
  cover_gather_kernel<<<C.blocks, 256, 0, stream>>>(C, ids, nids, out, done, flag, epoch);
}

void launch_coverage(const DevPool &P, uint64_t S, const uint32_t *marked,
                     unsigned long long *covered, int blocks, cudaStream_t stream) {
  count_launches(1);
  coverage_kernel<<<blocks, 256, 0, stream>>>(P, S, marked, covered);
}

void launch_sel_init(const SelDesc *d, int blocks, cudaStream_t stream) {
  count_launches(1);
  sel_init_kernel<<<blocks, 256, 0, stream>>>(d);
}
void launch_sel_count(const SelDesc *d, int blocks, cudaStream_t stream) {
  count_launches(1);
  sel_count_kernel<<<blocks, 256, 0, stream>>>(d);
}
void launch_sel_pick(const SelDesc *d, uint32_t i, int blocks, cudaStream_t stream) {
  count_launches(1);
  sel_pick_kernel<<<blocks, 256, 0, stream>>>(d, i);
}
void launch_sel_cover(const SelDesc *d, uint32_t i, int blocks, cudaStream_t stream) {
  count_launches(2);
  sel_cover_kernel<<<blocks, 256, 0, stream>>>(d, i);
  sel_recount_kernel<<<blocks, 256, 0, stream>>>(d);
}
uint32_t sel_chunk_vertices() { return SEL_CHUNK; }

void launch_gather_counts(const uint32_t *count, const uint32_t *ids, uint32_t m,
                          uint32_t *out, cudaStream_t stream) {
  if (m == 0) return;
  count_launches(1);
  gather_counts_kernel<<<std::min<uint32_t>((m + 255) / 256, 148), 256, 0, stream>>>(count, ids,
                                                                                     m, out);
}


}  // namespace rip
