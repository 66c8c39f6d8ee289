// kernels_bigset.cu -- IC sets with very large edge work, one CTA each.
//
// Under weighted-cascade probabilities on skewed graphs a few RRR sets reach
// many hubs and read millions of in-edge records each (on an R-MAT graph with
// 2^20 vertices 1% of the sets carry ~40% of the edge work).  One warp per set
// (ic_plain_kernel) or one warp per frontier entry (ic_fused_kernel) walks a
// hub's in-list alone, so those sets set the kernel's length.  Here one CTA
// grows one such set: level by level, the level's entries are taken a CTA's
// width at a time; in-lists of at least that many 4-edge groups (hubs) are
// swept by all threads one list at a time, and the others through their
// concatenated groups (a block scan turns group counts into offsets; each
// thread finds its entry with a forward-only cursor in shared memory).
// Levels are separated by __syncthreads only.  Coins are the same
// (set, edge)-keyed Philox draws as every other sampler; on lists with a
// uniform threshold a thread takes whole 8-edge coin blocks.
#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

// Block shapes: 128, 256, 512 or 1024 threads (at 64 registers a thread: 8,
// 4, 2 or 1 CTA per SM, each growing its own set -- smaller CTAs let one set's barrier
// waits overlap another's work; the autotuner picks per graph).  In-lists of
// at least BIG_THREADS 4-edge groups are swept by the whole CTA, one list at
// a time.

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
__global__ void __launch_bounds__(BIG_THREADS, 1024 / BIG_THREADS)
ic_bigset_kernel(BigLaunch L) {
  constexpr int BIG_WARPS = BIG_THREADS / 32;
  constexpr uint32_t kLongCTA = BIG_THREADS;
  __shared__ uint32_t s_off[BIG_THREADS + 1];  // exclusive group offsets of the chunk
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
    // Coins of group g of the in-list [ob, oe) (uniform threshold ovt, or 0:
    // each record's own); newly reached sources go to the queue.
    // Source u of a live edge joins the set (and the queue) unless there.
    auto reach = [&](uint32_t u) {
      const uint32_t bit = 1u << (u & 31);
      if (!(atomicOr(&bm[u >> 5], bit) & bit)) {
        const uint32_t pos = atomicAdd(&s_qlen, 1u);
        if (pos < L.qcap) q[pos] = u;
        else s_overflow = 1;
      }
    };
    // The live edges of group g given its coin block c (the group is half
    // of the 8-edge block g >> 1) and, for a list without a uniform
    // threshold, its records.
    auto apply_coins = [&](uint32_t g, uint32_t ob, uint32_t oe, uint32_t ovt, const u32x4 &c,
                           const uint2 rec[4]) {
      const uint32_t hb = (g & 1u) << 2;
      uint32_t live = 0, tie = 0;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const uint32_t ed = (g << 2) + t;
        const uint32_t th = (ovt ? ovt : rec[t].y) >> 16, cc = coarse_of(c, hb + t);
        if (ed >= ob && ed < oe) {
          if (cc < th) live |= 1u << t;
          else if (cc == th) tie |= 1u << t;
        }
      }
      while (tie) {  // a coarse tie, one edge in 65 536: the fine half decides
        const uint32_t t = __ffs(tie) - 1;
        tie &= tie - 1;
        const uint32_t thr = ovt ? ovt
                                 : (t == 0 ? rec[0].y : t == 1 ? rec[1].y : t == 2 ? rec[2].y : rec[3].y);
        if (ic_fine_call(L.key, (g << 2) + t, s) < (thr & 0xFFFFu)) live |= 1u << t;
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const uint32_t ed = (g << 2) + t;
        if (live & (1u << t)) {
          uint32_t u = rec[t].x;
          if (ovt) {
            u = __ldg(&L.G.edges[ed].x);
            atomicAdd(&s_usrc, 1ull);
          }
          reach(u);
        }
      }
    };
    // The live edges of the 8-edge block b of a uniform-threshold list.
    auto apply_block = [&](uint32_t b, uint32_t ob, uint32_t oe, uint32_t ovt, const u32x4 &c) {
      const uint32_t th = ovt >> 16;
      if (block_min16(c) > th) return;  // nothing live, no tie
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const uint32_t cc = coarse_of(c, h), ed = (b << 3) + h;
        if (cc <= th && ed >= ob && ed < oe &&
            (cc < th || ic_fine_call(L.key, ed, s) < (ovt & 0xFFFFu))) {
          atomicAdd(&s_usrc, 1ull);
          reach(__ldg(&L.G.edges[ed].x));
        }
      }
    };
    auto expand_group = [&](uint32_t g, uint32_t ob, uint32_t oe, uint32_t ovt) {
      uint2 rec[4] = {};
      if (!ovt) load_group(L.G.edges, g, rec);  // else: uniform threshold
      apply_coins(g, ob, oe, ovt, ic_block(L.key, g >> 1, s), rec);
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
        const uint32_t ng = group_count(beg, end);
        const bool lng = ng >= kLongCTA;
        s_off[tid] = big_block_scan<BIG_THREADS>(lng ? 0u : ng, s_warp, &s_total);  // syncs
        if (tid == 0) s_off[BIG_THREADS] = s_total;
        if (lng) s_long[atomicAdd(&s_nlong, 1u)] = tid;
        __syncthreads();
        // long in-lists (hubs): all threads sweep one list at a time
        const uint32_t nlong = s_nlong;
        for (uint32_t li = 0; li < nlong; ++li) {
          const uint32_t a = s_long[li];
          const uint32_t ob = s_beg[a], oe = s_end[a], ovt = s_vt[a];
          const uint32_t g_last = (oe - 1) >> 2;
          if (ovt) {
            // uniform threshold: nothing to load; a thread takes whole
            // 8-edge coin blocks, two in flight so their dependent Philox
            // rounds interleave
            const uint32_t b_last = (oe - 1) >> 3;
            uint32_t b = (ob >> 3) + tid;
            for (; b + BIG_THREADS <= b_last; b += 2 * BIG_THREADS) {
              const u32x4 c0 = ic_block(L.key, b, s);
              const u32x4 c1 = ic_block(L.key, b + BIG_THREADS, s);
              apply_block(b, ob, oe, ovt, c0);
              apply_block(b + BIG_THREADS, ob, oe, ovt, c1);
            }
            if (b <= b_last) apply_block(b, ob, oe, ovt, ic_block(L.key, b, s));
          } else {
            for (uint32_t g = (ob >> 2) + tid; g <= g_last; g += BIG_THREADS)
              expand_group(g, ob, oe, ovt);
          }
        }
        // the other lists through their concatenated groups: entry a holds
        // group j when s_off[a] <= j < s_off[a + 1]; a thread's j only grows,
        // so its entry cursor only moves forward
        const uint32_t total = s_off[BIG_THREADS];
        uint32_t a = 0;
        for (uint32_t j = tid; j < total; j += BIG_THREADS) {
          if (s_off[a + 1] <= j) {
            uint32_t b = BIG_THREADS;
            while (b - a > 1) {
              const uint32_t mid = (a + b) >> 1;
              if (s_off[mid] <= j) a = mid;
              else b = mid;
            }
          }
          const uint32_t ob = s_beg[a];
          expand_group((ob >> 2) + (j - s_off[a]), ob, s_end[a], s_vt[a]);
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

void launch_ic_bigset(const BigLaunch &L, cudaStream_t stream) {
  count_launches(1);
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
