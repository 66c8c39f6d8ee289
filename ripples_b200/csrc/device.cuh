// device.cuh -- device data views and warp-level helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "philox.cuh"

namespace rip {

constexpr uint32_t FULL = 0xFFFFFFFFu;

// Backward CSR packed for the sampler.  edges[e] = {source vertex, threshold}:
//   IC: threshold = floor(p_e * 2^32)  (edge live iff coin < threshold)
//   LT: threshold = floor(cumulative in-weight up to e * 2^32)
// off has n+1 entries; edges is padded with {0, 0} records to a multiple of 4
// and 32-byte aligned so a 4-edge group is one aligned 32-byte read.
// vthr (IC graphs, optional): vthr[v] != 0 when every in-edge of v has the
// threshold vthr[v] (weighted cascade: p = 1/in-degree); the IC samplers then
// compare v's coins against it and read only the sources of live edges.
// 0 means "read each edge's own threshold" (a uniform threshold of 0, an
// in-list that never fires, is stored as 0 too: still exact, only slower).
struct DevGraph {
  uint32_t n;
  uint64_t m;
  const uint32_t *off;
  const uint2 *edges;
  const uint32_t *vthr = nullptr;
};

// Flat RRR pool: set s occupies vtx[set_off[s] .. set_off[s] + set_len[s]).
struct DevPool {
  uint32_t *vtx;
  unsigned long long *cursor;  // next free element (atomic bump pointer)
  uint64_t cap;                // element capacity
  uint64_t *set_off;
  uint32_t *set_len;
};

// Failure list for sets that did not fit their scratch or the pool; the host
// re-runs them with larger buffers (results do not depend on the retry).
struct FailList {
  uint32_t *ids;          // indices relative to the launch's first set
  unsigned int *count;
  unsigned long long *first_bad_base;  // lowest pool offset of a failed reservation
};

// Counters for roofline accounting (see rip_pool_stats in ripples_b200.h).
struct Stats {
  unsigned long long *v;  // [8]
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(FULL, x, d);
    if (lane_id() >= (uint32_t)d) x += y;
  }
  return x;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(FULL, x, d);
  return x;
}

// Given an inclusive warp scan `incl` (held per lane) of per-lane item
// counts, returns the lane whose range holds item j (0 <= j < total):
// the smallest lane i with incl[i] > j.  Five shuffle steps.
__device__ __forceinline__ uint32_t warp_find_owner(uint32_t incl, uint32_t j) {
  uint32_t lo = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    uint32_t probe = __shfl_sync(FULL, incl, lo + step - 1);
    if (probe <= j) lo += step;
  }
  return lo;
}

// Lane-wise minimum of two pairs of 16-bit halves.
__device__ __forceinline__ uint32_t vmin_u16x2(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}

// Smallest of the eight coarse coins of a block: when it exceeds a uniform
// threshold's coarse half, no edge of the block is live and none ties.
__device__ __forceinline__ uint32_t block_min16(const u32x4 &c) {
  const uint32_t m = vmin_u16x2(vmin_u16x2(c.x, c.y), vmin_u16x2(c.z, c.w));
  return min(m & 0xFFFFu, m >> 16);
}

// Number of 4-edge groups covering [beg, end).
__device__ __forceinline__ uint32_t group_count(uint32_t beg, uint32_t end) {
  return end > beg ? ((end - 1) >> 2) - (beg >> 2) + 1 : 0;
}

// Number of 8-edge coin blocks covering [beg, end).
__device__ __forceinline__ uint32_t block_count(uint32_t beg, uint32_t end) {
  return end > beg ? ((end - 1) >> 3) - (beg >> 3) + 1 : 0;
}

// Coin blocks of a launch: from the key (its schedule added in registers)
// or from round keys the kernel keeps in parameter space.
struct KeyCoins {
  Key k;
  __device__ __forceinline__ u32x4 block(uint64_t b, uint64_t s) const { return ic_block(k, b, s); }
};
struct RoundKeyCoins {
  const RoundKeys &rk;
  __device__ __forceinline__ u32x4 block(uint64_t b, uint64_t s) const {
    return ic_block_rk(rk, b, s);
  }
};

// Live edges (bit h: edge 8b + h) of 8-edge coin block b of the in-list
// [ob, oe) for set s, given the block's coarse coins c: compared with the
// list's uniform threshold ovt (a whole block usually cleared by its smallest
// coin) or, when ovt is 0, with each record's own threshold (records read two
// at a time; a pair past the list's end is not read: the record array ends
// on a 4-edge boundary, not an 8-edge one).  A coarse tie (one edge in
// 65 536) draws the fine half.
__device__ __forceinline__ uint32_t ic_block_live(const DevGraph &G, Key key, uint64_t s,
                                                  uint32_t b, uint32_t ob, uint32_t oe,
                                                  uint32_t ovt, const u32x4 &c) {
  uint32_t live = 0, tie = 0;
  if (ovt) {
    const uint32_t th = ovt >> 16;
    if (block_min16(c) > th) return 0u;
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      const uint32_t cc = coarse_of(c, h), e = (b << 3) + h;
      if (cc <= th && e >= ob && e < oe) {
        if (cc < th) live |= 1u << h;
        else tie |= 1u << h;
      }
    }
  } else {
    const uint4 *rp = reinterpret_cast<const uint4 *>(G.edges + ((size_t)b << 3));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t e0 = (b << 3) + 2 * q;
      if (e0 < oe && e0 + 1 >= ob) {
        const uint4 r = __ldg(rp + q);
        const uint32_t c0 = coarse_of(c, 2 * q), c1 = coarse_of(c, 2 * q + 1);
        if (e0 >= ob) {
          if (c0 < (r.y >> 16)) live |= 1u << (2 * q);
          else if (c0 == (r.y >> 16)) tie |= 1u << (2 * q);
        }
        if (e0 + 1 < oe) {
          if (c1 < (r.w >> 16)) live |= 2u << (2 * q);
          else if (c1 == (r.w >> 16)) tie |= 2u << (2 * q);
        }
      }
    }
  }
  while (tie) {
    const uint32_t h = __ffs(tie) - 1;
    tie &= tie - 1;
    const uint32_t e = (b << 3) + h;
    const uint32_t thr = ovt ? ovt : __ldg(&G.edges[e].y);
    if (ic_fine_call(key, e, s) < (thr & 0xFFFFu)) live |= 1u << h;
  }
  return live;
}

// Loads the 4 edge records of group g (32-byte aligned).
__device__ __forceinline__ void load_group(const uint2 *edges, uint32_t g,
                                           uint2 rec[4]) {
  const uint4 *p = reinterpret_cast<const uint4 *>(edges + ((size_t)g << 2));
  uint4 a = __ldg(p), b = __ldg(p + 1);
  rec[0] = make_uint2(a.x, a.y);
  rec[1] = make_uint2(a.z, a.w);
  rec[2] = make_uint2(b.x, b.y);
  rec[3] = make_uint2(b.z, b.w);
}

}  // namespace rip
