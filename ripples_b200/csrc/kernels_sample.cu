// kernels_sample.cu -- RRR-set sampling kernels for sm_100a.
//
// ic_plain_kernel   one IC set per warp: reverse BFS over live in-edges
//                   (semantics of include/ripples/add_rrrset.h:128-135, with
//                   the per-edge coin keyed on (set, edge) instead of drawn
//                   from a sequential trng stream).
// lt_walk_kernel    one LT set per warp: single-predecessor walk
//                   (include/ripples/add_rrrset.h:136-150) with no length cap
//                   and no host fallback (the reference GPU walk stops at 8
//                   vertices and redoes longer walks on the CPU,
//                   include/ripples/gpu/lt_kernel.h:59-130,
//                   streaming_rrr_generator.h:492-520).
//
// Both are persistent: each warp pulls set indices from an atomic counter
// until the range is exhausted.  A warp owns an n-bit visited bitmap and a
// queue (the set's members in discovery order) in global scratch; at the end
// of a set it reserves room in the pool with one atomicAdd, copies the queue
// out and clears exactly the bitmap words it touched.  A set that outgrows
// the queue, or does not fit in the pool, is recorded in the failure list and
// the host re-runs it with larger buffers -- the result does not change,
// because every draw is a pure function of (seed, set id, edge / vertex id).
#include "device.cuh"
#include "launch.h"
#include "ripples_b200.h"

namespace rip {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// In-lists of at least this many 8-edge coin blocks are swept by a whole
// warp at a time instead of sharing it with other lists.
constexpr uint32_t kLongBlocks = 32;

struct WarpCtx {
  uint32_t *bm;  // visited bitmap, ceil(n/32) words
  uint32_t *q;   // queue, qcap entries
  uint32_t qcap;
};

// Writes the finished set to the pool (unless it overflowed) and clears the
// warp's bitmap.  Returns true when the set was stored; on a pool overflow
// the reservation's offset is recorded in *first_bad.
__device__ bool store_set(const WarpCtx &W, uint32_t qlen, bool overflow, uint64_t s,
                          const DevPool &P, unsigned long long *first_bad,
                          bool clear_bitmap = true) {
  const uint32_t lane = lane_id();
  bool stored = false;
  if (!overflow) {
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(P.cursor, (unsigned long long)qlen);
    b = __shfl_sync(FULL, b, 0);
    if (b + qlen <= P.cap) {
      for (uint32_t i = lane; i < qlen; i += 32) P.vtx[b + i] = W.q[i];
      if (lane == 0) {
        P.set_off[s] = b;
        P.set_len[s] = qlen;
      }
      stored = true;
    } else if (lane == 0) {
      atomicMin(first_bad, b);
    }
  }
  if (clear_bitmap)
    for (uint32_t i = lane; i < qlen; i += 32) W.bm[W.q[i] >> 5] = 0u;
  __syncwarp();
  return stored;
}

__device__ bool finish_set(const WarpCtx &W, uint32_t qlen, bool overflow,
                           uint64_t s, uint32_t rel, const DevPool &P,
                           const FailList &F, bool big = false, bool clear_bitmap = true) {
  const bool stored = store_set(W, qlen, overflow, s, P, F.first_bad_base, clear_bitmap);
  if (!stored && lane_id() == 0) F.ids[atomicAdd(F.count, 1u)] = big ? (rel | FAIL_BIG) : rel;
  __syncwarp();
  return stored;
}

struct SetOutcome {
  uint32_t qlen;
  bool overflow, big;
  unsigned long long exp, edges;  // per-set work (valid on lane 0 / summed over lanes)
  // IC, summed over lanes: in-edges of uniform-threshold lists (coins drawn,
  // records not read) and live edges of those lists (source id read)
  unsigned long long uedges = 0, usrc = 0;
};

// One IC set: reverse BFS from root(s) over live in-edges, warp-cooperative,
// members in discovery order in W.q.  Sets past `work_cap` in-edges (when
// nonzero) are abandoned with big = true.
template <class Coins>
__device__ __forceinline__ SetOutcome ic_plain_set(const DevGraph &G, Key key, const Coins &coins,
                                                   uint64_t s, const WarpCtx &W,
                                                   uint64_t work_cap) {
  const uint32_t lane = lane_id();
  const uint32_t root = root_of(key, s, G.n);
  if (lane == 0) {
    W.q[0] = root;
    atomicOr(&W.bm[root >> 5], 1u << (root & 31));
  }
  __syncwarp();
  uint32_t qlen = 1, head = 0;
  bool overflow = false, big = false;
  unsigned long long set_exp = 0, set_edges = 0, warp_edges = 0;
  uint32_t set_uedges = 0, set_usrc = 0;  // a set's edges are fewer than m < 2^32

  // Appends this lane's newly reached vertex (if any) to the queue,
  // warp-wide in lane order; on queue overflow the set is abandoned and the
  // bits of vertices that will never be queued cleared.
  auto append_one = [&](bool isnew, uint32_t nu) {
    const uint32_t bal = __ballot_sync(FULL, isnew);
    if (bal == 0) return;
    const uint32_t cnt = __popc(bal);
    if (overflow || qlen + cnt > W.qcap) {
      if (isnew) W.bm[nu >> 5] = 0u;
      overflow = true;
      return;
    }
    if (isnew) W.q[qlen + __popc(bal & lanemask_lt())] = nu;
    qlen += cnt;
  };
  auto block_live = [&](uint32_t b, uint32_t ob, uint32_t oe, uint32_t ovt) -> uint32_t {
    return ic_block_live(G, key, s, b, ob, oe, ovt, coins.block(b, s));
  };
  // Marks the sources of a block's live edges in the bitmap and queues the
  // new ones: one live edge per lane per pass, every lane voting (live edges
  // are few; a record's source is read again, from L1).
  auto take_live = [&](uint32_t b, uint32_t live, bool uniform) {
    while (__any_sync(FULL, live != 0)) {
      bool isnew = false;
      uint32_t nu = 0;
      if (live) {
        const uint32_t e = (b << 3) + (__ffs(live) - 1);
        live &= live - 1;
        nu = __ldg(&G.edges[e].x);
        if (uniform) ++set_usrc;
        const uint32_t bit = 1u << (nu & 31);
        isnew = !(atomicOr(&W.bm[nu >> 5], bit) & bit);
      }
      append_one(isnew, nu);
    }
  };

  while (head < qlen && !overflow) {
    const uint32_t take = min(32u, qlen - head);
    uint32_t beg = 0, end = 0, nb = 0, vt = 0;
    if (lane < take) {
      const uint32_t v = W.q[head + lane];
      beg = __ldg(G.off + v);
      end = __ldg(G.off + v + 1);
      if (G.vthr) vt = __ldg(G.vthr + v);
      nb = block_count(beg, end);
      set_edges += end - beg;
      if (vt) set_uedges += end - beg;
    }
    set_exp += (lane == 0) ? take : 0;
    {
      const uint32_t all = warp_incl_scan(nb);
      warp_edges += (unsigned long long)__shfl_sync(FULL, all, 31) * 8;
    }
    if (work_cap && warp_edges > work_cap) {
      // too much edge work for one warp: leave the set to a whole CTA
      overflow = big = true;
      break;
    }
    // Long in-lists (hubs) are swept by the whole warp, one list at a time:
    // lane j takes coin blocks j, j + 32, ... of the list, no owner search.
    uint32_t longs = __ballot_sync(FULL, nb >= kLongBlocks);
    while (longs && !overflow) {
      const uint32_t L = __ffs(longs) - 1;
      longs &= longs - 1;
      const uint32_t lb = __shfl_sync(FULL, beg, L), le = __shfl_sync(FULL, end, L);
      const uint32_t lvt = __shfl_sync(FULL, vt, L);
      const uint32_t b_last = (le - 1) >> 3;
      for (uint32_t base = lb >> 3; base <= b_last && !overflow; base += 32) {
        const uint32_t b = base + lane;
        const uint32_t live = b <= b_last ? block_live(b, lb, le, lvt) : 0u;
        take_live(b, live, lvt != 0);
        __syncwarp();
      }
    }
    // The shorter lists share the warp through their concatenated coin
    // blocks: block j belongs to the lane whose scanned range holds it.
    const uint32_t nbs = nb >= kLongBlocks ? 0u : nb;
    const uint32_t incl = warp_incl_scan(nbs);
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    for (uint32_t base = 0; base < total && !overflow; base += 32) {
      const uint32_t j = base + lane;
      const bool valid = j < total;
      const uint32_t owner = warp_find_owner(incl, valid ? j : total - 1);
      const uint32_t ob = __shfl_sync(FULL, beg, owner);
      const uint32_t oe = __shfl_sync(FULL, end, owner);
      const uint32_t oexcl = __shfl_sync(FULL, incl, owner) - __shfl_sync(FULL, nbs, owner);
      const uint32_t ovt = __shfl_sync(FULL, vt, owner);
      const uint32_t b = (ob >> 3) + (j - oexcl);
      const uint32_t live = valid ? block_live(b, ob, oe, ovt) : 0u;
      take_live(b, live, ovt != 0);
      __syncwarp();
    }
    head += take;
  }
  return SetOutcome{qlen, overflow, big, set_exp, set_edges, set_uedges, set_usrc};
}

// One LT set: the single-predecessor walk from root(s) (see lt_walk_kernel).
// A revisit is found by scanning the walk so far (the warp's queue, 32
// entries per load, L1-resident): walks are short (tens of steps), so this
// costs less than a visited-bitmap atomic and needs no bitmap at all.  After a
// pick, the next vertex's offsets and (degree <= 32) its in-edges are
// requested before the scan.
__device__ __forceinline__ SetOutcome lt_walk_set(const DevGraph &G, Key key, uint64_t s,
                                                  const WarpCtx &W) {
  const uint32_t lane = lane_id();
  uint32_t cur = root_of(key, s, G.n);
  if (lane == 0) W.q[0] = cur;
  __syncwarp();
  uint32_t qlen = 1;
  bool overflow = false;
  unsigned long long set_exp = 0, set_edges = 0;
  uint32_t lo = __ldg(G.off + cur), hi = __ldg(G.off + cur + 1);
  // the current vertex's in-edges when it has at most 32 (lane j: edge lo + j)
  bool have = false;
  uint2 rec = make_uint2(0u, 0u);
  for (;;) {
    set_exp += (lane == 0);
    if (hi == lo) break;
    const uint32_t t = lt_threshold(key, s, cur);
    if (!have) {
      // 32-ary search for the first edge whose cumulative threshold exceeds t
      bool none = false;
      while (hi - lo > 32) {
        const uint32_t stride = (hi - lo + 31) / 32;
        const uint32_t p = min(lo + (lane + 1) * stride - 1, hi - 1);
        const bool pred = t < __ldg(&G.edges[p].y);
        const uint32_t bal = __ballot_sync(FULL, pred);
        set_edges += (lane == 0) ? 32 : 0;
        if (bal == 0) {  // even the last edge's cumulative weight is <= t
          none = true;
          break;
        }
        const uint32_t L = __ffs(bal) - 1;
        const uint32_t nlo = lo + L * stride;
        hi = min(hi, lo + (L + 1) * stride);
        lo = nlo;
      }
      if (none) break;
      const uint32_t e = lo + lane;
      rec = make_uint2(0u, 0u);
      if (e < hi) rec = __ldg(&G.edges[e]);
    }
    const uint32_t bal = __ballot_sync(FULL, lo + lane < hi && t < rec.y);
    set_edges += (lane == 0) ? (hi - lo) : 0;
    if (bal == 0) break;  // no in-edge picked: the walk ends here
    const uint32_t u = __shfl_sync(FULL, rec.x, __ffs(bal) - 1);
    const uint32_t lo2 = __ldg(G.off + u), hi2 = __ldg(G.off + u + 1);
    // u's in-edges, requested before the revisit scan
    have = hi2 - lo2 <= 32;
    if (have) {
      const uint32_t e = lo2 + lane;
      rec = make_uint2(0u, 0u);
      if (e < hi2) rec = __ldg(&G.edges[e]);
    }
    bool seen = false;
    for (uint32_t b = 0; b < qlen && !seen; b += 32) {
      const uint32_t j = b + lane;
      seen = __any_sync(FULL, j < qlen && W.q[j] == u);
    }
    if (seen) break;
    if (qlen + 1 > W.qcap) {
      overflow = true;
      break;
    }
    if (lane == 0) W.q[qlen] = u;
    __syncwarp();
    ++qlen;
    cur = u;
    lo = lo2;
    hi = hi2;
  }
  __syncwarp();
  return SetOutcome{qlen, overflow, false, set_exp, set_edges};
}

}  // namespace

// MINB: resident blocks per SM the compiler must allow (4: at most 64
// registers, 32 warps per SM; 5: at most 48 registers, 40 warps per SM -- the
// autotuner picks per graph).
template <int MINB>
__global__ void __launch_bounds__(256, MINB)
ic_plain_kernel(DevGraph G, DevPool P, Key key, const __grid_constant__ RoundKeys rk,
                uint64_t first, uint32_t count,
                const uint32_t *ids, unsigned int *next, uint32_t *bitmaps,
                uint64_t bm_words, uint32_t *queues, uint32_t qcap,
                uint64_t work_cap, FailList F, Stats st) {
  const uint32_t lane = lane_id();
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  WarpCtx W{bitmaps + w * bm_words, queues + w * (uint64_t)qcap, qcap};
  unsigned long long n_exp = 0, n_edges = 0, n_sets = 0, n_elems = 0, n_uedges = 0, n_usrc = 0;

  for (;;) {
    uint32_t idx = 0;
    if (lane == 0) idx = atomicAdd(next, 1u);
    idx = __shfl_sync(FULL, idx, 0);
    if (idx >= count) break;
    const uint32_t rel = ids ? ids[idx] : idx;
    const uint64_t s = first + rel;
    const SetOutcome o = ic_plain_set(G, key, RoundKeyCoins{rk}, s, W, work_cap);
    if (finish_set(W, o.qlen, o.overflow, s, rel, P, F, o.big)) {
      n_sets += (lane == 0);
      n_elems += (lane == 0) ? o.qlen : 0;
      n_exp += o.exp;
      n_edges += o.edges;
      n_uedges += o.uedges;
      n_usrc += o.usrc;
    }
  }
  n_exp = warp_sum_u64(n_exp);
  n_edges = warp_sum_u64(n_edges);
  n_sets = warp_sum_u64(n_sets);
  n_elems = warp_sum_u64(n_elems);
  n_uedges = warp_sum_u64(n_uedges);
  n_usrc = warp_sum_u64(n_usrc);
  if (lane == 0) {
    atomicAdd(st.v + 0, n_exp);
    atomicAdd(st.v + 1, n_edges);
    atomicAdd(st.v + 2, n_sets);
    atomicAdd(st.v + 3, n_elems);
    atomicAdd(st.v + 4, n_exp);
    atomicAdd(st.v + 5, n_edges);
    if (n_uedges) atomicAdd(st.v + 6, n_uedges);
    if (n_usrc) atomicAdd(st.v + 7, n_usrc);
  }
}

// One walk per warp.  Each step needs the chosen in-edge of the current
// vertex: a 32-ary search over the cumulative thresholds (one probe per lane
// per round, log32(in-degree) rounds), finishing with one 8-byte load per lane
// so the lane that holds the pick also holds its source id.  Walks are chains
// of dependent loads; the kernel is bound to 32 registers (up to 64 resident
// warps per SM) and the host launches 32 warps per SM: a launch lasts about
// as long as its longest walk either way, and the free warp slots serve
// other queries' kernels.
__global__ void __launch_bounds__(256, 8)
lt_walk_kernel(DevGraph G, DevPool P, Key key, uint64_t first, uint32_t count,
               const uint32_t *ids, unsigned int *next, uint32_t *bitmaps,
               uint64_t bm_words, uint32_t *queues, uint32_t qcap, FailList F,
               Stats st) {
  const uint32_t lane = lane_id();
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  WarpCtx W{bitmaps + w * bm_words, queues + w * (uint64_t)qcap, qcap};
  unsigned long long n_exp = 0, n_edges = 0, n_sets = 0, n_elems = 0;

  for (;;) {
    uint32_t idx = 0;
    if (lane == 0) idx = atomicAdd(next, 1u);
    idx = __shfl_sync(FULL, idx, 0);
    if (idx >= count) break;
    const uint32_t rel = ids ? ids[idx] : idx;
    const uint64_t s = first + rel;
    const SetOutcome o = lt_walk_set(G, key, s, W);
    if (finish_set(W, o.qlen, o.overflow, s, rel, P, F, false, false)) {
      n_sets += (lane == 0);
      n_elems += (lane == 0) ? o.qlen : 0;
      n_exp += o.exp;
      n_edges += o.edges;
    }
  }
  n_exp = warp_sum_u64(n_exp);
  n_edges = warp_sum_u64(n_edges);
  n_sets = warp_sum_u64(n_sets);
  n_elems = warp_sum_u64(n_elems);
  if (lane == 0) {
    atomicAdd(st.v + 0, n_exp);
    atomicAdd(st.v + 1, n_edges);
    atomicAdd(st.v + 2, n_sets);
    atomicAdd(st.v + 3, n_elems);
    atomicAdd(st.v + 4, n_exp);
    atomicAdd(st.v + 5, n_edges);
  }
}

// Many IMM instances in one persistent launch: warps pull global work indices
// from one counter; index i belongs to the instance a with
// prefix[a] <= i < prefix[a+1] and is that instance's set first_a + i -
// prefix[a], grown with that instance's graph, model and seed into its pool.
__global__ void __launch_bounds__(256)
multi_sample_kernel(MultiLaunch L) {
  const uint32_t lane = lane_id();
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  WarpCtx W{L.bitmaps + w * L.bm_words, L.queues + w * (uint64_t)L.qcap, L.qcap};
  // counters of the instance the warp is on, flushed when it moves on
  uint32_t cur = ~0u;
  unsigned long long n_exp = 0, n_edges = 0, n_sets = 0, n_elems = 0, n_uedges = 0, n_usrc = 0;
  auto flush = [&]() {
    const unsigned long long e = warp_sum_u64(n_exp), d = warp_sum_u64(n_edges);
    const unsigned long long ue = warp_sum_u64(n_uedges), us = warp_sum_u64(n_usrc);
    if (lane == 0 && cur != ~0u && n_sets) {
      unsigned long long *st = L.inst[cur].stats;
      atomicAdd(st + 0, e);
      atomicAdd(st + 1, d);
      atomicAdd(st + 2, n_sets);
      atomicAdd(st + 3, n_elems);
      atomicAdd(st + 4, e);
      atomicAdd(st + 5, d);
      if (ue) atomicAdd(st + 6, ue);
      if (us) atomicAdd(st + 7, us);
    }
    n_exp = n_edges = n_sets = n_elems = n_uedges = n_usrc = 0;
  };
  for (;;) {
    uint32_t idx = 0;
    if (lane == 0) idx = atomicAdd(L.next, 1u);
    idx = __shfl_sync(FULL, idx, 0);
    if (idx >= L.total) break;
    uint32_t a = 0, b = L.n_inst;  // prefix[a] <= idx < prefix[b]
    while (b - a > 1) {
      const uint32_t mid = (a + b) >> 1;
      if (L.prefix[mid] <= idx) a = mid;
      else b = mid;
    }
    if (a != cur) {
      flush();
      cur = a;
    }
    const InstanceDesc &D = L.inst[a];
    const uint32_t rel = idx - L.prefix[a];
    const uint64_t s = D.first + rel;
    const SetOutcome o = D.model == RIP_MODEL_IC ? ic_plain_set(D.G, D.key, KeyCoins{D.key}, s, W, D.work_cap)
                                                 : lt_walk_set(D.G, D.key, s, W);
    if (store_set(W, o.qlen, o.overflow, s, D.P, D.first_bad, D.model == RIP_MODEL_IC)) {
      n_sets += 1;
      n_elems += o.qlen;
      n_exp += o.exp;
      n_edges += o.edges;
      n_uedges += o.uedges;
      n_usrc += o.usrc;
    } else if (lane == 0) {
      const unsigned int f = atomicAdd(L.fail_count, 1u);
      L.fail[2 * f] = a;
      L.fail[2 * f + 1] = o.big ? (rel | FAIL_BIG) : rel;
    }
    __syncwarp();
  }
  flush();
}

void launch_multi_sample(const MultiLaunch &L, cudaStream_t stream) {
  count_launches(1);
  multi_sample_kernel<<<L.blocks, 256, 0, stream>>>(L);
}

void launch_ic_plain(const SampleLaunch &L, cudaStream_t stream) {
  count_launches(1);
  const RoundKeys rk = round_keys(L.key);
  if (L.occupancy == 5)
    ic_plain_kernel<5><<<L.blocks, L.threads, 0, stream>>>(
        L.G, L.P, L.key, rk, L.first, L.count, L.ids, L.next, L.bitmaps, L.bm_words,
        L.queues, L.qcap, L.work_cap, L.F, L.st);
  else
    ic_plain_kernel<4><<<L.blocks, L.threads, 0, stream>>>(
        L.G, L.P, L.key, rk, L.first, L.count, L.ids, L.next, L.bitmaps, L.bm_words,
        L.queues, L.qcap, L.work_cap, L.F, L.st);
}

void launch_lt_walk(const SampleLaunch &L, cudaStream_t stream) {
  count_launches(1);
  lt_walk_kernel<<<L.blocks, L.threads, 0, stream>>>(
      L.G, L.P, L.key, L.first, L.count, L.ids, L.next, L.bitmaps, L.bm_words,
      L.queues, L.qcap, L.F, L.st);
}

}  // namespace rip
