// kernels_giant.cu -- IC sets too large for one warp or one CTA, grown 64*CW
// at a time by the whole GPU.
//
// On graphs where IC is supercritical (R-MAT with p ~ U(0, 0.1) and average
// degree 16: a giant component), a tenth or more of all RRR sets each hold a
// sizeable fraction of the graph and overlap heavily.  A batch of up to 64*CW
// such sets is grown as one multi-colour reverse BFS spread over the whole
// grid: every vertex carries a visited and a pending colour mask, and each
// level runs as
//   prep    : the level's frontier entries take their pending masks (for the
//             colours that reached them last level) and count their 8-edge
//             coin blocks;
//   scan    : exclusive scan of the group counts (one global work list);
//   expand  : one thread per aligned 8-edge coin block, its owner found by
//             one binary search per warp in the scan and a short walk per
//             lane; for every colour of the owner's mask one Philox block
//             gives the eight edges' coarse coins; live edges OR the
//             colour into the source's visited mask, and colours new to it go
//             to its pending mask and put it on the next level's frontier
//             (once per level: a per-vertex level stamp).
// A hub's in-edge list is therefore split over the whole grid, and a vertex
// reached by many sets in the same level is read once for all of them.  When
// the frontier is empty the members are counted per colour, placed in the
// pool (host-reserved range), and the masks cleared -- only for vertices the
// batch touched (a first-touch list).  Coins are the same (set, edge) Philox
// draws as every other sampler, so the sets are bit-identical to theirs.
#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt_g() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Appends x (for lanes with want) to list[*tail ...], one atomic per warp.
__device__ __forceinline__ void warp_append(bool want, uint32_t x, uint32_t *list,
                                            unsigned int *tail) {
  const uint32_t bal = __ballot_sync(FULL, want);
  if (!bal) return;
  const uint32_t leader = __ffs(bal) - 1;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(tail, (unsigned int)__popc(bal));
  base = __shfl_sync(FULL, base, leader);
  if (want) list[base + __popc(bal & lanemask_lt_g())] = x;
}

template <int CW>
__global__ void __launch_bounds__(256) giant_seed_kernel(GiantLaunch L) {
  const uint32_t lane = lane_id();
  for (uint32_t base = blockIdx.x * blockDim.x; base < L.ncol; base += gridDim.x * blockDim.x) {
    const uint32_t c = base + threadIdx.x;
    const bool valid = c < L.ncol;
    uint32_t r = 0, old = 1;
    if (valid) {
      r = root_of(L.key, L.set_ids[c], L.G.n);
      const unsigned long long bit = 1ull << (c & 63);
      atomicOr((unsigned long long *)&L.vis[(size_t)r * CW + (c >> 6)], bit);
      atomicOr((unsigned long long *)&L.pend[(size_t)r * CW + (c >> 6)], bit);
      old = atomicExch(&L.pflag[r], 1u);
    }
    (void)lane;
    warp_append(valid && old == 0u, r, L.touched, L.ctr + 1);
    warp_append(valid && old != 1u, r, L.front, L.ctr + 0);
  }
}

// Level prep: entry i of the frontier takes its vertex's pending colours and
// counts its 8-edge coin blocks.
template <int CW>
__global__ void __launch_bounds__(256) giant_prep_kernel(GiantLaunch L, uint32_t nf) {
  unsigned long long exp = 0, edges = 0, sexp = 0, sedges = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
    const uint32_t v = L.front[i];
    uint32_t pc = 0;
#pragma unroll
    for (int w = 0; w < CW; ++w) {
      const uint64_t m = L.pend[(size_t)v * CW + w];
      L.pend[(size_t)v * CW + w] = 0ull;
      L.masks[(size_t)i * CW + w] = m;
      pc += __popcll(m);
    }
    uint32_t ng = 0;
    if (pc) {
      const uint32_t beg = __ldg(L.G.off + v), end = __ldg(L.G.off + v + 1);
      ng = block_count(beg, end);
      exp += 1;
      edges += end - beg;
      sexp += pc;
      sedges += (unsigned long long)pc * (end - beg);
    }
    L.ng[i] = ng;
  }
  exp = warp_sum_u64(exp);
  edges = warp_sum_u64(edges);
  sexp = warp_sum_u64(sexp);
  sedges = warp_sum_u64(sedges);
  if (lane_id() == 0 && exp) {
    atomicAdd(L.stats + 0, exp);
    atomicAdd(L.stats + 1, edges);
    atomicAdd(L.stats + 4, sexp);
    atomicAdd(L.stats + 5, sedges);
  }
}

template <int CW>
__global__ void __launch_bounds__(256) giant_expand_kernel(const __grid_constant__ GiantLaunch L,
                                                           uint32_t nf, uint32_t level) {
  const uint64_t total = L.goff[nf];
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
    const uint64_t j = base + threadIdx.x;
    const bool valid = j < total;
    uint32_t u[8], thr[8];
#pragma unroll
    for (int h = 0; h < 8; ++h) u[h] = thr[h] = 0;
    uint32_t addm = 0;  // edges whose source gained a colour
    // owner of j: the last entry i with goff[i] <= j.  One binary search per
    // warp (for its first j), then each lane walks forward from there: the
    // warp's 32 consecutive blocks span few entries
    uint32_t wlo = 0;
    {
      const uint64_t j0 = __shfl_sync(FULL, j, 0);
      if (lane_id() == 0 && j0 < total) {
        uint32_t lo = 0, hi = nf;
        while (hi - lo > 1) {
          const uint32_t mid = lo + ((hi - lo) >> 1);
          if (L.goff[mid] <= j0) lo = mid;
          else hi = mid;
        }
        wlo = lo;
      }
      wlo = __shfl_sync(FULL, wlo, 0);
    }
    if (valid) {
      uint32_t lo = wlo;
      while (lo + 1 < nf && L.goff[lo + 1] <= j) ++lo;
      const uint32_t v = L.front[lo];
      const uint32_t beg = __ldg(L.G.off + v), end = __ldg(L.G.off + v + 1);
      // an 8-edge coin block: its two 4-edge record groups (the second only
      // when it holds an edge of this list: the record array ends on a
      // 4-edge boundary)
      const uint32_t b = (beg >> 3) + (uint32_t)(j - L.goff[lo]);
      uint2 rec[8];
      load_group(L.G.edges, 2 * b, rec);
      if (((2 * b + 1) << 2) < end) {
        load_group(L.G.edges, 2 * b + 1, rec + 4);
      } else {
#pragma unroll
        for (int h = 4; h < 8; ++h) rec[h] = make_uint2(0u, 0u);
      }
      uint32_t inr = 0;
#pragma unroll
      for (int h = 0; h < 8; ++h) {
        const uint32_t e = (b << 3) + h;
        if (e >= beg && e < end && rec[h].y != 0u) inr |= 1u << h;
        u[h] = rec[h].x;
        thr[h] = rec[h].y;
      }
      if (inr) {
#pragma unroll
        for (int w = 0; w < CW; ++w) {
          // one Philox block per colour gives the eight edges' coarse coins
          uint64_t live[8];
#pragma unroll
          for (int h = 0; h < 8; ++h) live[h] = 0;
          uint64_t mm = L.masks[(size_t)lo * CW + w];
          while (mm) {
            const int bi = __ffsll((long long)mm) - 1;
            mm &= mm - 1;
            const uint64_t sid = L.set_ids[w * 64 + bi];
            const u32x4 cb = ic_block_rk(L.rk, b, sid);
            const uint64_t bit = 1ull << bi;
            uint32_t tie = 0;
#pragma unroll
            for (int h = 0; h < 8; ++h) {
              const uint32_t th = thr[h] >> 16, cc = coarse_of(cb, h);
              if (inr & (1u << h)) {
                if (cc < th) live[h] |= bit;
                else if (cc == th) tie |= 1u << h;
              }
            }
            while (tie) {  // a coarse tie, one edge in 65 536: the fine half decides
              const uint32_t h = __ffs(tie) - 1;
              tie &= tie - 1;
              uint32_t t = thr[0];
#pragma unroll
              for (int q = 1; q < 8; ++q)
                if (h == (uint32_t)q) t = thr[q];
              if (ic_fine_call(L.key, (b << 3) + h, sid) < (t & 0xFFFFu)) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                  if (h == (uint32_t)q) live[q] |= bit;
              }
            }
          }
#pragma unroll
          for (int h = 0; h < 8; ++h) {
            // a plain read first: visited bits only get set, so colours it
            // shows need no atomic (most live edges late in a giant BFS)
            if (live[h] && (live[h] & ~__ldcg(&L.vis[(size_t)u[h] * CW + w]))) {
              const uint64_t old =
                  atomicOr((unsigned long long *)&L.vis[(size_t)u[h] * CW + w], live[h]);
              const uint64_t add = live[h] & ~old;
              if (add) {
                atomicOr((unsigned long long *)&L.pend[(size_t)u[h] * CW + w], add);
                addm |= 1u << h;
              }
            }
          }
        }
      }
    }
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      const bool added = (addm >> h) & 1u;
      uint32_t oldf = level + 1;
      if (added) oldf = atomicExch(&L.pflag[u[h]], level + 1);
      warp_append(added && oldf == 0u, u[h], L.touched, L.ctr + 1);
      warp_append(added && oldf != level + 1, u[h], L.front_next, L.ctr + 0);
    }
  }
}

constexpr uint32_t GIANT_CHUNK = 2048;  // touched vertices per block in compaction

// Members per colour (block-local histograms, one global add per colour).
template <int CW>
__global__ void __launch_bounds__(256) giant_sizes_kernel(GiantLaunch L, uint32_t nt) {
  __shared__ uint32_t s_cnt[64 * CW];
  for (uint32_t c = threadIdx.x; c < 64 * CW; c += blockDim.x) s_cnt[c] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
    const uint32_t v = L.touched[i];
#pragma unroll
    for (int w = 0; w < CW; ++w) {
      uint64_t m = L.vis[(size_t)v * CW + w];
      while (m) {
        const int bi = __ffsll((long long)m) - 1;
        m &= m - 1;
        atomicAdd(&s_cnt[w * 64 + bi], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t c = threadIdx.x; c < L.ncol; c += blockDim.x)
    if (s_cnt[c]) atomicAdd(L.sizes + c, s_cnt[c]);
}

// Writes each member into its set's pool range and clears the batch's state.
// A block takes GIANT_CHUNK touched vertices: counts them per colour,
// reserves a slice of every colour's range with one atomic each, then places
// them; positions inside a set are arbitrary (set contents are compared as
// sets).
template <int CW>
__global__ void __launch_bounds__(256) giant_scatter_kernel(GiantLaunch L, uint32_t nt) {
  __shared__ uint32_t s_cnt[64 * CW];
  __shared__ unsigned long long s_at[64 * CW];
  for (uint32_t c0 = blockIdx.x * GIANT_CHUNK; c0 < nt; c0 += gridDim.x * GIANT_CHUNK) {
    const uint32_t c1 = min(nt, c0 + GIANT_CHUNK);
    for (uint32_t c = threadIdx.x; c < 64 * CW; c += blockDim.x) s_cnt[c] = 0;
    __syncthreads();
    for (uint32_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
      const uint32_t v = L.touched[i];
#pragma unroll
      for (int w = 0; w < CW; ++w) {
        uint64_t m = L.vis[(size_t)v * CW + w];
        while (m) {
          const int bi = __ffsll((long long)m) - 1;
          m &= m - 1;
          atomicAdd(&s_cnt[w * 64 + bi], 1u);
        }
      }
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < L.ncol; c += blockDim.x) {
      s_at[c] = s_cnt[c] ? L.starts[c] + atomicAdd(L.fill + c, s_cnt[c]) : 0ull;
      s_cnt[c] = 0;
    }
    __syncthreads();
    for (uint32_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
      const uint32_t v = L.touched[i];
#pragma unroll
      for (int w = 0; w < CW; ++w) {
        uint64_t m = L.vis[(size_t)v * CW + w];
        L.vis[(size_t)v * CW + w] = 0ull;
        while (m) {
          const int bi = __ffsll((long long)m) - 1;
          m &= m - 1;
          const uint32_t c = w * 64 + bi;
          L.P.vtx[s_at[c] + atomicAdd(&s_cnt[c], 1u)] = v;
        }
      }
      L.pflag[v] = 0u;
    }
    __syncthreads();
  }
}

// set_off / set_len of the batch's sets (starts computed on the host).
__global__ void giant_meta_kernel(GiantLaunch L) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < L.ncol;
       c += gridDim.x * blockDim.x) {
    const uint64_t s = L.set_ids[c];
    L.P.set_off[s] = L.starts[c];
    L.P.set_len[s] = L.sizes[c];
    L.fill[c] = 0;
    atomicAdd(L.stats + 2, 1ull);
    atomicAdd(L.stats + 3, (unsigned long long)L.sizes[c]);
  }
}

}  // namespace

template <int CW>
static void giant_launch(int what, const GiantLaunch &L, uint32_t n_items, uint32_t level,
                         int blocks, cudaStream_t s) {
  count_launches(1);
  switch (what) {
    case 0: giant_seed_kernel<CW><<<1, 256, 0, s>>>(L); break;
    case 1: giant_prep_kernel<CW><<<blocks, 256, 0, s>>>(L, n_items); break;
    case 2: giant_expand_kernel<CW><<<blocks, 256, 0, s>>>(L, n_items, level); break;
    case 3: giant_sizes_kernel<CW><<<blocks, 256, 0, s>>>(L, n_items); break;
    case 4: giant_scatter_kernel<CW><<<blocks, 256, 0, s>>>(L, n_items); break;
    default: giant_meta_kernel<<<1, 256, 0, s>>>(L); break;
  }
}

void launch_giant(int what, int cw, const GiantLaunch &L0, uint32_t n_items, uint32_t level,
                  int blocks, cudaStream_t s) {
  GiantLaunch L = L0;
  L.rk = round_keys(L.key);
  if (cw == 1) giant_launch<1>(what, L, n_items, level, blocks, s);
  else if (cw == 2) giant_launch<2>(what, L, n_items, level, blocks, s);
  else giant_launch<4>(what, L, n_items, level, blocks, s);
}

}  // namespace rip
