// kernels_spread.cu -- forward Monte Carlo spread of a seed set (IC, LT).
//
// The reference measures the quality of a seed set with ripples::simulate
// (include/ripples/diffusion_simulation.h:73-178, driven replica by replica
// by tools/simulator.cc); the spread is the number of vertices reached,
// seeds included.  Here one 512-thread CTA runs one replica at a time with
// the level loop of the one-CTA-per-heavy-set sampler: a level's entries are
// taken a CTA's width at a time, a block scan turns their out-edge unit counts into
// offsets and all warps stride over the concatenated units (IC: 8-edge coin
// blocks, one Philox block each; LT: 4-edge record groups).
//   IC: out-edge e of a reached vertex fires in replica r iff its coin
//       (coarse half from sim_ic_block(key, e >> 3, r), fine half from
//       sim_ic_fine on a coarse tie) is below threshold(e) (BFS over live
//       edges, diffusion_simulation.h:73-127).
//   LT: the live-edge form of the threshold model (Kempe, Kleinberg, Tardos,
//       KDD'03): vertex v keeps at most one in-edge -- the first j of its
//       in-list with sim_lt_threshold(key, r, v) < cum[j], cum being the
//       fixed-point cumulative in-weights the LT sampler uses -- and v is
//       reached iff the source of that in-edge is reached.  The reached set
//       has the distribution of diffusion_simulation.h:129-178's.
// Either way a replica's reached set is a pure function of (seed, r),
// whatever the visiting order.
#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

// four 512-thread CTAs per SM (32 registers a thread: 64 resident warps).
// The kernel waits on L2 latency, so replicas in flight are what move it:
// one 1024-thread CTA per SM (32 warps) ran 19.3 K replicas/s on the 2^20
// bench, two of 768 threads 23.1 K, three of 640 25.6 K, four of 512 26.5 K.
constexpr int SIM_THREADS = 512;
constexpr int SIM_WARPS = SIM_THREADS / 32;

__device__ uint32_t sim_block_scan(uint32_t x, uint32_t *warp_tot, uint32_t *total) {
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
  const uint32_t incl = warp_incl_scan(x);
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const uint32_t t = lane < SIM_WARPS ? warp_tot[lane] : 0u;
    const uint32_t ti = warp_incl_scan(t);
    if (lane < SIM_WARPS) warp_tot[lane] = ti - t;
    if (lane == 31) *total = ti;
  }
  __syncthreads();
  const uint32_t r = warp_tot[wid] + incl - x;
  __syncthreads();
  return r;
}

constexpr uint32_t NO_VERTEX = 0xFFFFFFFFu;

// LT: the source of the in-edge vertex v keeps in replica r, or NO_VERTEX.
// cum is non-decreasing along the in-list, so the first j with t < cum[j] is
// found by binary search.
__device__ __forceinline__ uint32_t lt_kept_source(const DevGraph &B, Key key, uint64_t r,
                                                   uint32_t v) {
  const uint32_t lo = __ldg(B.off + v), hi = __ldg(B.off + v + 1);
  if (lo == hi) return NO_VERTEX;
  const uint32_t t = sim_lt_threshold(key, r, v);
  if (!(t < __ldg(B.edges + (hi - 1)).y)) return NO_VERTEX;  // keeps no in-edge
  uint32_t a = lo, b = hi - 1;  // cum[b] > t
  while (a < b) {
    const uint32_t mid = a + ((b - a) >> 1);  // edge ids reach 2^32: no a + b
    if (__ldg(B.edges + mid).y > t) b = mid;
    else a = mid + 1;
  }
  return __ldg(B.edges + a).x;
}

template <bool LT>
__global__ void __launch_bounds__(SIM_THREADS, kSpreadCtasPerSm)
spread_kernel(SpreadLaunch L) {
  __shared__ uint32_t s_off[SIM_THREADS + 1];
  __shared__ uint32_t s_beg[SIM_THREADS], s_end[SIM_THREADS];
  __shared__ uint32_t s_v[LT ? SIM_THREADS : 1];  // LT: the entry's vertex
  __shared__ uint32_t s_warp[SIM_WARPS];
  __shared__ uint32_t s_qlen, s_total;
  __shared__ unsigned long long s_rep;

  const uint32_t tid = threadIdx.x;
  uint32_t *bm = L.bitmaps + (size_t)blockIdx.x * L.bm_words;
  uint32_t *q = L.queues + (size_t)blockIdx.x * L.qcap;
  unsigned long long reached = 0;

  for (;;) {
    if (tid == 0) {
      s_rep = atomicAdd(L.next, 1ull);
      s_qlen = 0;
    }
    __syncthreads();
    const uint64_t r = s_rep;
    if (r >= L.replicas) break;
    // the seeds are the first level (a repeated seed is queued once)
    for (uint32_t i = tid; i < L.k; i += SIM_THREADS) {
      const uint32_t v = L.seeds[i];
      const uint32_t bit = 1u << (v & 31);
      if (!(atomicOr(&bm[v >> 5], bit) & bit)) {
        const uint32_t pos = atomicAdd(&s_qlen, 1u);
        if (pos < L.qcap) q[pos] = v;
      }
    }
    __syncthreads();
    uint32_t lo = 0, hi = min(s_qlen, L.qcap), levels = 0;
    while (lo < hi) {
      ++levels;  // one BFS level (the seeds are the first)
      for (uint32_t cb = lo; cb < hi; cb += SIM_THREADS) {
        const uint32_t e = cb + tid;
        uint32_t beg = 0, end = 0;
        if (e < hi) {
          const uint32_t v = q[e];
          beg = __ldg(L.G.off + v);
          end = __ldg(L.G.off + v + 1);
          if (LT) s_v[tid] = v;
        }
        s_beg[tid] = beg;
        s_end[tid] = end;
        const uint32_t ng = LT ? group_count(beg, end) : block_count(beg, end);
        s_off[tid] = sim_block_scan(ng, s_warp, &s_total);
        if (tid == 0) s_off[SIM_THREADS] = s_total;
        __syncthreads();
        const uint32_t total = s_off[SIM_THREADS];
        for (uint32_t j = tid; j < total; j += SIM_THREADS) {
          uint32_t a = 0, b = SIM_THREADS;  // entry a: s_off[a] <= j < s_off[a + 1]
          while (b - a > 1) {
            const uint32_t mid = (a + b) >> 1;
            if (s_off[mid] <= j) a = mid;
            else b = mid;
          }
          const uint32_t ob = s_beg[a], oe = s_end[a];
          if (LT) {
            const uint32_t g = (ob >> 2) + (j - s_off[a]);
            uint2 rec[4];
            load_group(L.G.edges, g, rec);
            const uint32_t from = s_v[a];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              const uint32_t ed = (g << 2) + t;
              if (ed < ob || ed >= oe) continue;
              const uint32_t u = rec[t].x;
              const uint32_t bit = 1u << (u & 31);
              // a plain read first: reached bits are only ever set
              if ((__ldcg(&bm[u >> 5]) & bit) || lt_kept_source(L.B, L.key, r, u) != from)
                continue;
              if (!(atomicOr(&bm[u >> 5], bit) & bit)) {
                const uint32_t pos = atomicAdd(&s_qlen, 1u);
                if (pos < L.qcap) q[pos] = u;
              }
            }
          } else {
            // an 8-edge coin block: records two at a time (a pair past the
            // list's end is not read: the record array ends on a 4-edge
            // boundary), coarse coins first, the fine half on a tie
            const uint32_t b = (ob >> 3) + (j - s_off[a]);
            const u32x4 c = sim_ic_block(L.key, b, r);
            const uint4 *rp = reinterpret_cast<const uint4 *>(L.G.edges + ((size_t)b << 3));
            uint32_t live = 0, tie = 0;
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
              const uint32_t e0 = (b << 3) + 2 * qq;
              if (e0 < oe && e0 + 1 >= ob) {
                const uint4 rr = __ldg(rp + qq);
                const uint32_t c0 = coarse_of(c, 2 * qq), c1 = coarse_of(c, 2 * qq + 1);
                if (e0 >= ob) {
                  if (c0 < (rr.y >> 16)) live |= 1u << (2 * qq);
                  else if (c0 == (rr.y >> 16)) tie |= 1u << (2 * qq);
                }
                if (e0 + 1 < oe) {
                  if (c1 < (rr.w >> 16)) live |= 2u << (2 * qq);
                  else if (c1 == (rr.w >> 16)) tie |= 2u << (2 * qq);
                }
              }
            }
            while (tie) {
              const uint32_t h = __ffs(tie) - 1;
              tie &= tie - 1;
              const uint32_t ed = (b << 3) + h;
              if (sim_ic_fine(L.key, ed, r) < (__ldg(&L.G.edges[ed].y) & 0xFFFFu))
                live |= 1u << h;
            }
            while (live) {
              const uint32_t u = __ldg(&L.G.edges[(b << 3) + (__ffs(live) - 1)].x);
              live &= live - 1;
              const uint32_t bit = 1u << (u & 31);
              if (!(atomicOr(&bm[u >> 5], bit) & bit)) {
                const uint32_t pos = atomicAdd(&s_qlen, 1u);
                if (pos < L.qcap) q[pos] = u;
              }
            }
          }
        }
        __syncthreads();
      }
      lo = hi;
      hi = min(s_qlen, L.qcap);
      __syncthreads();
    }
    // every vertex is queued at most once, so qlen <= n = qcap
    const uint32_t qlen = min(s_qlen, L.qcap);
    if (tid == 0) {
      if (L.sizes) L.sizes[r] = qlen;
      if (L.levels) L.levels[r] = levels;
      reached += qlen;
    }
    for (uint32_t i = tid; i < qlen; i += SIM_THREADS) bm[q[i] >> 5] = 0u;
    __syncthreads();
  }
  if (tid == 0 && reached) atomicAdd(L.total, reached);
}

}  // namespace

void launch_spread(const SpreadLaunch &L, bool lt, cudaStream_t stream) {
  count_launches(1);
  if (lt) spread_kernel<true><<<L.blocks, SIM_THREADS, 0, stream>>>(L);
  else spread_kernel<false><<<L.blocks, SIM_THREADS, 0, stream>>>(L);
}

}  // namespace rip
