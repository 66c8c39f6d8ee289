// kernels_bigset.cu -- IC sets with very large edge work, one CTA each.
//
// Under weighted-cascade probabilities on skewed graphs a few RRR sets reach
// many hubs and read millions of in-edge records each (on an R-MAT graph with
// 2^20 vertices 1% of the sets carry ~40% of the edge work).  One warp per set
// (ic_plain_kernel) or one warp per frontier entry (ic_fused_kernel) walks a
// hub's in-list alone, so those sets set the kernel's length.  Here one CTA
// grows one such set: level by level, the level's entries are taken a CTA's
// width at a time; in-lists of at least that many 8-edge coin blocks (hubs)
// are swept by all threads one list at a time, and the others through their
// concatenated blocks (a block scan turns block counts into offsets; each
// thread finds its entry with a forward-only cursor in shared memory).
// Levels are separated by __syncthreads only.  Coins are the same
// (set, edge)-keyed Philox draws as every other sampler; a thread takes
// whole 8-edge coin blocks (one Philox block each).
#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

// Block shapes: 128, 256, 512 or 1024 threads, kBigCtasPerSm of them
// resident per SM (10, 5, 2 or 1: at most 48, 48, 64 or 64 registers a
// thread), each growing its own set -- more resident CTAs let one set's
// barrier waits overlap another's work; the autotuner picks the shape per
// graph.  In-lists of at least BIG_THREADS coin blocks are swept by the
// whole CTA, one list at a time.

// Exclusive block scan of one u32 per thread; returns the exclusive value and
// writes the block total to *total.  Uses `warp_tot` (BIG_WARPS entries).
template <int BIG_THREADS>
__device__ uint32_t big_block_scan(uint32_t x, uint32_t *warp_tot, uint32_t *total) {
  constexpr int BIG_WARPS = BIG_THREADS / 32;
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
  const uint32_t incl = warp_incl_scan(x);
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const uint32_t t = lane < BIG_WARPS ? warp_tot[lane] : 0u;
    const uint32_t ti = warp_incl_scan(t);
    if (lane < BIG_WARPS) warp_tot[lane] = ti - t;
    if (lane == 31) *total = ti;
  }
  __syncthreads();
  const uint32_t r = warp_tot[wid] + incl - x;
  __syncthreads();
  return r;
}

template <int BIG_THREADS>
__global__ void __launch_bounds__(BIG_THREADS, kBigCtasPerSm(BIG_THREADS))
ic_bigset_kernel(const __grid_constant__ BigLaunch L) {
  constexpr int BIG_WARPS = BIG_THREADS / 32;
  constexpr uint32_t kLongCTA = BIG_THREADS;
  __shared__ uint32_t s_off[BIG_THREADS + 1];  // exclusive coin-block offsets of the chunk
  __shared__ uint32_t s_beg[BIG_THREADS], s_end[BIG_THREADS], s_vt[BIG_THREADS];
  __shared__ uint32_t s_warp[BIG_WARPS];
  __shared__ uint32_t s_long[BIG_THREADS];  // entries of the chunk with long in-lists
  __shared__ uint32_t s_idx, s_qlen, s_overflow, s_total, s_nlong;
  __shared__ unsigned long long s_edges, s_uedges, s_usrc, s_base;

  const uint32_t tid = threadIdx.x;
  uint32_t *bm = L.bitmaps + (size_t)blockIdx.x * L.bm_words;
  uint32_t *q = L.queues + (size_t)blockIdx.x * L.qcap;
  unsigned long long n_exp = 0, n_edges = 0, n_sets = 0, n_elems = 0, n_uedges = 0, n_usrc = 0;

  for (;;) {
    if (tid == 0) s_idx = atomicAdd(L.next, 1u);
    __syncthreads();
    const uint32_t idx = s_idx;
    if (idx >= L.count) break;
    const uint32_t rel = L.ids[idx];
    const uint64_t s = L.first + rel;
    if (tid == 0) {
      const uint32_t root = root_of(L.key, s, L.G.n);
      q[0] = root;
      atomicOr(&bm[root >> 5], 1u << (root & 31));
      s_qlen = 1;
      s_overflow = 0;
      s_edges = 0;
      s_uedges = 0;
      s_usrc = 0;
    }
    __syncthreads();
    uint32_t lo = 0, hi = 1;
    // Source u of a live edge joins the set (and the queue) unless there.
    auto reach = [&](uint32_t u) {
      const uint32_t bit = 1u << (u & 31);
      if (!(atomicOr(&bm[u >> 5], bit) & bit)) {
        const uint32_t pos = atomicAdd(&s_qlen, 1u);
        if (pos < L.qcap) q[pos] = u;
        else s_overflow = 1;
      }
    };
    // The live edges of 8-edge coin block b of the in-list [ob, oe) given its
    // coarse coins c; their sources are read then and reached.
    auto expand_block = [&](uint32_t b, uint32_t ob, uint32_t oe, uint32_t ovt, const u32x4 &c) {
      uint32_t live = ic_block_live(L.G, L.key, s, b, ob, oe, ovt, c);
      while (live) {
        const uint32_t ed = (b << 3) + (__ffs(live) - 1);
        live &= live - 1;
        if (ovt) atomicAdd(&s_usrc, 1ull);
        reach(__ldg(&L.G.edges[ed].x));
      }
    };
    while (lo < hi && !s_overflow) {
      for (uint32_t cb = lo; cb < hi; cb += BIG_THREADS) {
        const uint32_t e = cb + tid;
        uint32_t beg = 0, end = 0, vt = 0;
        if (tid == 0) s_nlong = 0;
        if (e < hi) {
          const uint32_t v = q[e];
          beg = __ldg(L.G.off + v);
          end = __ldg(L.G.off + v + 1);
          if (L.G.vthr) vt = __ldg(L.G.vthr + v);
          atomicAdd(&s_edges, (unsigned long long)(end - beg));
          if (vt) atomicAdd(&s_uedges, (unsigned long long)(end - beg));
        }
        s_beg[tid] = beg;
        s_end[tid] = end;
        s_vt[tid] = vt;
        const uint32_t nb = block_count(beg, end);
        const bool lng = nb >= kLongCTA;
        s_off[tid] = big_block_scan<BIG_THREADS>(lng ? 0u : nb, s_warp, &s_total);  // syncs
        if (tid == 0) s_off[BIG_THREADS] = s_total;
        if (lng) s_long[atomicAdd(&s_nlong, 1u)] = tid;
        __syncthreads();
        // long in-lists (hubs): all threads sweep one list at a time, a
        // thread taking whole coin blocks, two in flight so that their
        // dependent Philox rounds interleave
        const uint32_t nlong = s_nlong;
        for (uint32_t li = 0; li < nlong; ++li) {
          const uint32_t a = s_long[li];
          const uint32_t ob = s_beg[a], oe = s_end[a], ovt = s_vt[a];
          const uint32_t b_last = (oe - 1) >> 3;
          uint32_t b = (ob >> 3) + tid;
          for (; b + BIG_THREADS <= b_last; b += 2 * BIG_THREADS) {
            const u32x4 c0 = ic_block_rk(L.rk, b, s);
            const u32x4 c1 = ic_block_rk(L.rk, b + BIG_THREADS, s);
            expand_block(b, ob, oe, ovt, c0);
            expand_block(b + BIG_THREADS, ob, oe, ovt, c1);
          }
          if (b <= b_last) expand_block(b, ob, oe, ovt, ic_block_rk(L.rk, b, s));
        }
        // the other lists through their concatenated coin blocks: entry a
        // holds block j when s_off[a] <= j < s_off[a + 1]; a thread's j only
        // grows, so its entry cursor only moves forward
        const uint32_t total = s_off[BIG_THREADS];
        uint32_t a = 0;
        for (uint32_t j = tid; j < total; j += BIG_THREADS) {
          if (s_off[a + 1] <= j) {
            uint32_t hi2 = BIG_THREADS;
            while (hi2 - a > 1) {
              const uint32_t mid = (a + hi2) >> 1;
              if (s_off[mid] <= j) a = mid;
              else hi2 = mid;
            }
          }
          const uint32_t ob = s_beg[a];
          const uint32_t b = (ob >> 3) + (j - s_off[a]);
          expand_block(b, ob, s_end[a], s_vt[a], ic_block_rk(L.rk, b, s));
        }
        __syncthreads();
      }
      lo = hi;
      hi = min(s_qlen, L.qcap);
      __syncthreads();
    }
    const uint32_t qlen = min(s_qlen, L.qcap);
    bool stored = false;
    if (!s_overflow) {
      if (tid == 0) {
        const unsigned long long b = atomicAdd(L.P.cursor, (unsigned long long)qlen);
        if (b + qlen <= L.P.cap) {
          s_base = b;
          L.P.set_off[s] = b;
          L.P.set_len[s] = qlen;
        } else {
          atomicMin(L.F.first_bad_base, b);
          s_base = ~0ull;
        }
      }
      __syncthreads();
      stored = s_base != ~0ull;
      if (stored)
        for (uint32_t i = tid; i < qlen; i += BIG_THREADS) L.P.vtx[s_base + i] = q[i];
    }
    __syncthreads();
    // clear the bitmap: every set bit belongs to a queued vertex -- except on
    // queue overflow, where discovered vertices past the queue also set bits
    if (s_overflow) {
      for (uint64_t w = tid; w < L.bm_words; w += BIG_THREADS) bm[w] = 0u;
    } else {
      for (uint32_t i = tid; i < qlen; i += BIG_THREADS) bm[q[i] >> 5] = 0u;
    }
    if (tid == 0) {
      if (stored) {
        n_sets += 1;
        n_elems += qlen;
        n_exp += qlen;
        n_edges += s_edges;
        n_uedges += s_uedges;
        n_usrc += s_usrc;
      } else {
        L.F.ids[atomicAdd(L.F.count, 1u)] = rel;
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    atomicAdd(L.st.v + 0, n_exp);
    atomicAdd(L.st.v + 1, n_edges);
    atomicAdd(L.st.v + 2, n_sets);
    atomicAdd(L.st.v + 3, n_elems);
    atomicAdd(L.st.v + 4, n_exp);
    atomicAdd(L.st.v + 5, n_edges);
    if (n_uedges) atomicAdd(L.st.v + 6, n_uedges);
    if (n_usrc) atomicAdd(L.st.v + 7, n_usrc);
  }
}

}  // namespace

void launch_ic_bigset(const BigLaunch &L0, cudaStream_t stream) {
  count_launches(1);
  BigLaunch L = L0;
  L.rk = round_keys(L.key);
  if (L.threads == 128)
    ic_bigset_kernel<128><<<L.blocks, 128, 0, stream>>>(L);
  else if (L.threads == 256)
    ic_bigset_kernel<256><<<L.blocks, 256, 0, stream>>>(L);
  else if (L.threads == 512)
    ic_bigset_kernel<512><<<L.blocks, 512, 0, stream>>>(L);
  else
    ic_bigset_kernel<1024><<<L.blocks, 1024, 0, stream>>>(L);
}

}  // namespace rip
