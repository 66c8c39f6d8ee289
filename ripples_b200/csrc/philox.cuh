// philox.cuh -- counter-based random draws of the sampler (host + device).
//
// Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw, "Parallel
// random numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of two 32x32->64
// multiplies (constants 0xD2511F53, 0xCD9E8D57) with a Weyl key schedule
// (0x9E3779B9, 0xBB67AE85).
//
// Every random decision of the sampler is a pure function of
// (seed, set id, edge id / vertex id), which is what lets the fused
// multi-colour BFS, the one-set-per-warp BFS and the CPU oracle produce
// bit-identical RRR sets whatever order they visit edges in.
//   key                = (seed_lo, seed_hi)
//   root(s)            = mulhi64(P(s_lo, 0, 0, ROOT<<24 | s_hi)[0..1], n)
//   coin(s, e)         = coarse(s, e) << 16 | fine(s, e)   (32 bits)
//   coarse(s, e)       = 16-bit half (e & 1) of word (e >> 1) & 3 of
//                        P(b_lo, b_hi, s_lo, IC<<24 | s_hi),  b = e >> 3
//   fine(s, e)         = low 16 bits of P(e_lo, e_hi, s_lo, IC_FINE<<24 | s_hi)[0]
//   lt_threshold(s, v) = P(v, 0, s_lo, LT<<24 | s_hi)[0]
// An IC edge is live iff coin < threshold: coarse < thr >> 16, or
// coarse == thr >> 16 and fine < thr & 0xFFFF.  One Philox block thus
// carries the coarse halves of eight edges, and the fine half is drawn for
// one edge in 65 536 (a coarse tie); the coin is still an exactly uniform
// 32-bit draw per (set, edge), compared with the same threshold.
// (s_hi = bits 32..55 of the set id; set ids are limited to 2^56.)
// Forward Monte Carlo spread simulation draws from domains of its own, keyed
// by the replica id r instead of a set id:
//   sim_coin(r, e)     = coarse << 16 | fine as coin(s, e), from
//                        P(b_lo, b_hi, r_lo, SIM_IC<<24 | r_hi) and
//                        P(e_lo, e_hi, r_lo, SIM_IC_FINE<<24 | r_hi)[0]
//   sim_lt_thr(r, v)   = P(v, 0, r_lo, SIM_LT<<24 | r_hi)[0]
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define RIP_HD __host__ __device__ __forceinline__
#else
#define RIP_HD inline
#endif

namespace rip {

enum : uint32_t {
  DOM_ROOT = 1,
  DOM_IC = 2,
  DOM_LT = 3,
  DOM_SIM_IC = 7,
  DOM_SIM_LT = 8,
  DOM_IC_FINE = 9,
  DOM_SIM_IC_FINE = 10
};

RIP_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
#if defined(__CUDA_ARCH__)
  hi = __umulhi(a, b);
  lo = a * b;
#else
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
#endif
}

struct u32x4 {
  uint32_t x, y, z, w;
};

RIP_HD u32x4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                    uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, hi0, lo0);
    mulhilo32(0xCD9E8D57u, c2, hi1, lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  return u32x4{c0, c1, c2, c3};
}

RIP_HD void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2],
                          uint32_t out[4]) {
  u32x4 r = philox(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  out[3] = r.w;
}

struct Key {
  uint32_t k0, k1;
};

RIP_HD Key make_key(uint64_t seed) {
  return Key{(uint32_t)seed, (uint32_t)(seed >> 32)};
}

// Round keys of the Weyl schedule, k + r * (0x9E3779B9, 0xBB67AE85) for
// r = 0..9, computed once per launch: a kernel that keeps them in its
// parameter space (__grid_constant__) XORs them in from there instead of
// adding the schedule in registers every round.
struct RoundKeys {
  uint32_t k0[10], k1[10];
};

RIP_HD RoundKeys round_keys(Key k) {
  RoundKeys rk;
  for (int r = 0; r < 10; ++r) {
    rk.k0[r] = k.k0 + (uint32_t)r * 0x9E3779B9u;
    rk.k1[r] = k.k1 + (uint32_t)r * 0xBB67AE85u;
  }
  return rk;
}

// philox() with the round keys given.
RIP_HD u32x4 philox_rk(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                       const RoundKeys &rk) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, hi0, lo0);
    mulhilo32(0xCD9E8D57u, c2, hi1, lo1);
    const uint32_t n0 = hi1 ^ c1 ^ rk.k0[r];
    const uint32_t n2 = hi0 ^ c3 ^ rk.k1[r];
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  return u32x4{c0, c1, c2, c3};
}

RIP_HD uint32_t set_hi(uint64_t s, uint32_t dom) {
  return (dom << 24) | (uint32_t)((s >> 32) & 0xFFFFFFu);
}

RIP_HD uint32_t root_of(Key k, uint64_t s, uint32_t n) {
  u32x4 r = philox((uint32_t)s, 0u, 0u, set_hi(s, DOM_ROOT), k.k0, k.k1);
  uint64_t u = (uint64_t)r.x | ((uint64_t)r.y << 32);
#if defined(__CUDA_ARCH__)
  return (uint32_t)__umul64hi(u, (uint64_t)n);
#else
  return (uint32_t)(((unsigned __int128)u * n) >> 64);
#endif
}

// Coarse coins of the 8 edges 8b .. 8b+7 of set s: edge 8b + h is half
// h & 1 of word h >> 1 (coarse_of).
RIP_HD u32x4 ic_block(Key k, uint64_t b, uint64_t s) {
  return philox((uint32_t)b, (uint32_t)(b >> 32), (uint32_t)s,
                set_hi(s, DOM_IC), k.k0, k.k1);
}

// ic_block() with the launch's round keys.
RIP_HD u32x4 ic_block_rk(const RoundKeys &rk, uint64_t b, uint64_t s) {
  return philox_rk((uint32_t)b, (uint32_t)(b >> 32), (uint32_t)s, set_hi(s, DOM_IC), rk);
}

// Fine (low) 16 bits of the coin of edge e of set s.
RIP_HD uint32_t ic_fine(Key k, uint64_t e, uint64_t s) {
  return philox((uint32_t)e, (uint32_t)(e >> 32), (uint32_t)s,
                set_hi(s, DOM_IC_FINE), k.k0, k.k1).x & 0xFFFFu;
}

#if defined(__CUDACC__)
// The fine half is drawn on one coarse tie in 65 536: out of line on the
// device, so the samplers' hot loops carry one Philox body, not two.
static __device__ __noinline__ uint32_t ic_fine_call(Key k, uint64_t e, uint64_t s) {
  return ic_fine(k, e, s);
}
#endif

// Live test of edge e with coarse coin `coarse` against threshold thr.
RIP_HD bool ic_live(Key k, uint64_t s, uint64_t e, uint32_t coarse, uint32_t thr) {
  const uint32_t th = thr >> 16;
#if defined(__CUDA_ARCH__)
  return coarse < th || (coarse == th && ic_fine_call(k, e, s) < (thr & 0xFFFFu));
#else
  return coarse < th || (coarse == th && ic_fine(k, e, s) < (thr & 0xFFFFu));
#endif
}

// Coarse coins of the 8 forward edges 8b .. 8b+7 in spread replica r.
RIP_HD u32x4 sim_ic_block(Key k, uint64_t b, uint64_t r) {
  return philox((uint32_t)b, (uint32_t)(b >> 32), (uint32_t)r,
                set_hi(r, DOM_SIM_IC), k.k0, k.k1);
}

// Fine (low) 16 bits of the coin of forward edge e in spread replica r.
RIP_HD uint32_t sim_ic_fine(Key k, uint64_t e, uint64_t r) {
  return philox((uint32_t)e, (uint32_t)(e >> 32), (uint32_t)r,
                set_hi(r, DOM_SIM_IC_FINE), k.k0, k.k1).x & 0xFFFFu;
}

// Threshold of vertex v in LT spread replica r.
RIP_HD uint32_t sim_lt_threshold(Key k, uint64_t r, uint32_t v) {
  return philox(v, 0u, (uint32_t)r, set_hi(r, DOM_SIM_LT), k.k0, k.k1).x;
}

RIP_HD uint32_t lt_threshold(Key k, uint64_t s, uint32_t v) {
  return philox(v, 0u, (uint32_t)s, set_hi(s, DOM_LT), k.k0, k.k1).x;
}

RIP_HD uint32_t lane_of(const u32x4 &r, uint32_t i) {
  return i == 0 ? r.x : i == 1 ? r.y : i == 2 ? r.z : r.w;
}

// Coarse coin h (0..7) of a block.
RIP_HD uint32_t coarse_of(const u32x4 &blk, uint32_t h) {
  const uint32_t w = lane_of(blk, h >> 1);
  return (h & 1) ? (w >> 16) : (w & 0xFFFFu);
}

}  // namespace rip
