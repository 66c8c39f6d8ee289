// kernels_wide.cu -- grid-wide fused multi-colour reverse BFS (IC), sm_100a.
//
// For the heavy tail of IC sampling: under weighted-cascade probabilities on
// skewed graphs a few RRR sets reach many hubs and read millions of in-edge
// records each (1% of the sets can carry ~40% of the edge work), which one
// warp (ic_plain_kernel) or one CTA (ic_fused_kernel, whose warps split the
// frontier entry by entry) walks alone.  Here a batch of up to 64*CW such
// sets is grown level by level by the WHOLE GPU:
//   1. wide_prepare_kernel: every frontier entry of the level consumes its
//      pending colour mask and records (first edge group, #groups, mask);
//   2. an exclusive scan of the group counts (launch_exclusive_scan);
//   3. wide_expand_kernel: one thread per 4-edge group of the level -- a
//      binary search over the scanned counts finds its entry -- evaluates the
//      colours' coins, ORs discoveries into the visited masks, and appends
//      newly pending vertices to the frontier log (once per level, through
//      the per-vertex level flag);
//   4. the host reads the log tail and starts the next level.
// Coins, colour masks and compaction are those of ic_fused_kernel, so the
// sets are bit-identical to every other sampler's.
#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt_w() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <int CW>
__global__ void wide_seed_kernel(WideLaunch L) {
  for (uint32_t c = threadIdx.x; c < L.ncol; c += blockDim.x) {
    const uint32_t r = root_of(L.key, L.sets[c], L.G.n);
    const uint64_t bit = 1ull << (c & 63);
    atomicOr((unsigned long long *)&L.vis[(size_t)r * CW + (c >> 6)], bit);
    atomicOr((unsigned long long *)&L.pend[(size_t)r * CW + (c >> 6)], bit);
    atomicAdd(&L.sizes[c], 1u);
    if (atomicExch(&L.pflag[r], 1u) != 1u) {
      const uint32_t pos = atomicAdd(L.tail, 1u);
      if (pos < L.lcap) L.log[pos] = r;
      else atomicExch(L.overflow, 1u);
    }
  }
}

// Entries log[lo, hi) of the current level -> ent_* arrays (index i - lo).
template <int CW>
__global__ void wide_prepare_kernel(WideLaunch L, uint32_t lo, uint32_t hi) {
  unsigned long long n_exp = 0, n_edges = 0, n_sexp = 0, n_sedges = 0;
  for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi;
       i += gridDim.x * blockDim.x) {
    const uint32_t v = L.log[i];
    uint32_t any = 0, pc = 0;
#pragma unroll
    for (int w = 0; w < CW; ++w) {
      const uint64_t m = atomicExch((unsigned long long *)&L.pend[(size_t)v * CW + w], 0ull);
      L.ent_mask[(size_t)(i - lo) * CW + w] = m;
      any |= m != 0;
      pc += __popcll(m);
    }
    uint32_t beg = 0, end = 0;
    if (any) {
      beg = __ldg(L.G.off + v);
      end = __ldg(L.G.off + v + 1);
      n_exp += 1;
      n_edges += end - beg;
      n_sexp += pc;
      n_sedges += (unsigned long long)pc * (end - beg);
    }
    L.ent_beg[i - lo] = beg;
    L.ent_end[i - lo] = end;
    L.ent_groups[i - lo] = group_count(beg, end);
  }
  n_exp = warp_sum_u64(n_exp);
  n_edges = warp_sum_u64(n_edges);
  n_sexp = warp_sum_u64(n_sexp);
  n_sedges = warp_sum_u64(n_sedges);
  if (lane_id() == 0 && (n_exp | n_sexp)) {
    atomicAdd(L.batch_stats + 0, n_exp);
    atomicAdd(L.batch_stats + 1, n_edges);
    atomicAdd(L.batch_stats + 2, n_sexp);
    atomicAdd(L.batch_stats + 3, n_sedges);
  }
}

// One thread per 4-edge group of the level's entries (nent entries whose
// exclusive group prefix is ent_prefix[0..nent], ent_prefix[nent] = total).
template <int CW>
__global__ void __launch_bounds__(256)
wide_expand_kernel(WideLaunch L, uint32_t nent, uint32_t level) {
  const uint64_t total = L.ent_prefix[nent];
  const uint32_t lane = lane_id();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  // all lanes iterate together so the appends below can use warp collectives
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
       base < total; base += stride) {
    const uint64_t j = base + lane;
    const bool valid = j < total;
    uint64_t live[4][CW];
    uint32_t u[4] = {0, 0, 0, 0};
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
      for (int w = 0; w < CW; ++w) live[t][w] = 0;
    if (valid) {
      // entry: last index whose prefix <= j
      uint32_t a = 0, b = nent;  // invariant: prefix[a] <= j < prefix[b]
      while (b - a > 1) {
        const uint32_t mid = (a + b) >> 1;
        if (L.ent_prefix[mid] <= j) a = mid;
        else b = mid;
      }
      const uint32_t ob = L.ent_beg[a], oe = L.ent_end[a];
      const uint32_t g = (ob >> 2) + (uint32_t)(j - L.ent_prefix[a]);
      uint2 rec[4];
      load_group(L.G.edges, g, rec);
      bool inr[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const uint32_t e = (g << 2) + t;
        inr[t] = e >= ob && e < oe && rec[t].y != 0u;
        u[t] = rec[t].x;
      }
      if (inr[0] | inr[1] | inr[2] | inr[3]) {
#pragma unroll
        for (int w = 0; w < CW; ++w) {
          uint64_t mm = L.ent_mask[(size_t)a * CW + w];
          while (mm) {
            const int bi = __ffsll((long long)mm) - 1;
            mm &= mm - 1;
            const u32x4 cn = ic_coins(L.key, g, L.sets[w * 64 + bi]);
            const uint64_t bit = 1ull << bi;
            if (inr[0] && cn.x < rec[0].y) live[0][w] |= bit;
            if (inr[1] && cn.y < rec[1].y) live[1][w] |= bit;
            if (inr[2] && cn.z < rec[2].y) live[2][w] |= bit;
            if (inr[3] && cn.w < rec[3].y) live[3][w] |= bit;
          }
        }
      }
    }
    bool push[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      bool added = false;
#pragma unroll
      for (int w = 0; w < CW; ++w) {
        if (live[t][w]) {
          const uint64_t old =
              atomicOr((unsigned long long *)&L.vis[(size_t)u[t] * CW + w], live[t][w]);
          uint64_t add = live[t][w] & ~old;
          if (add) {
            atomicOr((unsigned long long *)&L.pend[(size_t)u[t] * CW + w], add);
            added = true;
            while (add) {
              const int bi = __ffsll((long long)add) - 1;
              add &= add - 1;
              atomicAdd(&L.sizes[w * 64 + bi], 1u);
            }
          }
        }
      }
      push[t] = added && atomicExch(&L.pflag[u[t]], level + 1) != level + 1;
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const uint32_t bal = __ballot_sync(FULL, push[t]);
      if (!bal) continue;
      uint32_t pos0 = 0;
      if (lane == (uint32_t)(__ffs(bal) - 1)) pos0 = atomicAdd(L.tail, __popc(bal));
      pos0 = __shfl_sync(FULL, pos0, __ffs(bal) - 1);
      if (push[t]) {
        const uint32_t pos = pos0 + __popc(bal & lanemask_lt_w());
        if (pos < L.lcap) L.log[pos] = u[t];
        else atomicExch(L.overflow, 1u);
      }
    }
  }
}

// Reserves pool room for the batch (one thread) and records the sets.
__global__ void wide_reserve_kernel(WideLaunch L) {
  unsigned long long tot = 0;
  for (uint32_t c = 0; c < L.ncol; ++c) tot += L.sizes[c];
  const unsigned long long base = atomicAdd(L.P.cursor, tot);
  if (base + tot > L.P.cap) {
    atomicMin(L.F.first_bad_base, base);
    *L.overflow = 2u;
    return;
  }
  unsigned long long run = base;
  for (uint32_t c = 0; c < L.ncol; ++c) {
    L.starts[c] = run;
    L.P.set_off[L.sets[c]] = run;
    L.P.set_len[L.sets[c]] = L.sizes[c];
    run += L.sizes[c];
  }
}

// Writes members (when `store`) and clears the masks and level flags of every
// vertex the batch reached; resets the batch counters.
template <int CW>
__global__ void wide_emit_kernel(WideLaunch L, uint32_t tail, int store) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < tail;
       i += gridDim.x * blockDim.x) {
    const uint32_t v = L.log[i];
#pragma unroll
    for (int w = 0; w < CW; ++w) {
      uint64_t mm = atomicExch((unsigned long long *)&L.vis[(size_t)v * CW + w], 0ull);
      L.pend[(size_t)v * CW + w] = 0ull;
      while (mm && store) {
        const int bi = __ffsll((long long)mm) - 1;
        mm &= mm - 1;
        const uint32_t c = w * 64 + bi;
        const uint32_t pos = atomicAdd(&L.fill[c], 1u);
        L.P.vtx[L.starts[c] + pos] = v;
      }
    }
    L.pflag[v] = 0u;
  }
}

// Adds a stored batch's work to the pool counters.
__global__ void wide_commit_kernel(WideLaunch L, Stats st) {
  unsigned long long tot = 0;
  for (uint32_t c = 0; c < L.ncol; ++c) tot += L.sizes[c];
  atomicAdd(st.v + 0, L.batch_stats[0]);
  atomicAdd(st.v + 1, L.batch_stats[1]);
  atomicAdd(st.v + 4, L.batch_stats[2]);
  atomicAdd(st.v + 5, L.batch_stats[3]);
  atomicAdd(st.v + 2, (unsigned long long)L.ncol);
  atomicAdd(st.v + 3, tot);
}

}  // namespace

void launch_wide_commit(const WideLaunch &L, Stats st, cudaStream_t s) {
  count_launches(1);
  wide_commit_kernel<<<1, 1, 0, s>>>(L, st);
}

void launch_wide_seed(const WideLaunch &L, cudaStream_t s) {
  count_launches(1);
  if (L.cw == 1) wide_seed_kernel<1><<<1, 256, 0, s>>>(L);
  else if (L.cw == 2) wide_seed_kernel<2><<<1, 256, 0, s>>>(L);
  else wide_seed_kernel<4><<<1, 256, 0, s>>>(L);
}

void launch_wide_prepare(const WideLaunch &L, uint32_t lo, uint32_t hi, cudaStream_t s) {
  count_launches(1);
  const int blocks = (int)std::min<uint32_t>(1184, (hi - lo + 255) / 256 + 1);
  if (L.cw == 1) wide_prepare_kernel<1><<<blocks, 256, 0, s>>>(L, lo, hi);
  else if (L.cw == 2) wide_prepare_kernel<2><<<blocks, 256, 0, s>>>(L, lo, hi);
  else wide_prepare_kernel<4><<<blocks, 256, 0, s>>>(L, lo, hi);
}

void launch_wide_expand(const WideLaunch &L, uint32_t nent, uint32_t level, int blocks,
                        cudaStream_t s) {
  count_launches(1);
  if (L.cw == 1) wide_expand_kernel<1><<<blocks, 256, 0, s>>>(L, nent, level);
  else if (L.cw == 2) wide_expand_kernel<2><<<blocks, 256, 0, s>>>(L, nent, level);
  else wide_expand_kernel<4><<<blocks, 256, 0, s>>>(L, nent, level);
}

void launch_wide_reserve(const WideLaunch &L, cudaStream_t s) {
  count_launches(1);
  wide_reserve_kernel<<<1, 1, 0, s>>>(L);
}

void launch_wide_emit(const WideLaunch &L, uint32_t tail, bool store, cudaStream_t s) {
  count_launches(1);
  const int blocks = (int)std::min<uint32_t>(1184, tail / 256 + 1);
  if (L.cw == 1) wide_emit_kernel<1><<<blocks, 256, 0, s>>>(L, tail, store ? 1 : 0);
  else if (L.cw == 2) wide_emit_kernel<2><<<blocks, 256, 0, s>>>(L, tail, store ? 1 : 0);
  else wide_emit_kernel<4><<<blocks, 256, 0, s>>>(L, tail, store ? 1 : 0);
}

}  // namespace rip
