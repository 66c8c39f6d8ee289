// kernels_fused.cu -- fused multi-colour reverse BFS for IC sampling (sm_100a).
//
// One CTA grows a batch of W = 64*CW RRR sets (CW = 1, 2, 4 -> 64/128/256
// colours) in a single traversal: every vertex carries a W-bit colour mask, so
// a vertex reached by several sets in the same level reads its in-edge list
// once for all of them.  The reference's GPU sampler does the same colour
// batching (GPUBatchedBFSMultiColorFused, include/ripples/gpu/bfs.h:1338-1680;
// kernels include/ripples/gpu/bfs_kernels.h:442-666) but rescans all n
// vertices every level, syncs the host per level and copies the whole
// n x colour matrix back for a host-side scan after each batch.  Here:
//   * frontiers are sparse: a per-CTA log of (vertex) entries, one level
//     after the other; a vertex enters a level's list once, when its pending
//     mask first gains a colour for that level (per-vertex level flag); the
//     log's first kSharedLog entries are staged in shared memory (most
//     batches never leave it), the rest in the CTA's global log;
//   * levels are separated by __syncthreads only -- no grid sync, no host
//     round trip; CTAs are persistent and pull batches from an atomic counter;
//   * the coin of (set s, edge e) is the same pure function of (seed, s, e)
//     as every sampler's (coarse halves from an 8-edge Philox block, the fine
//     half on a tie), so the sets equal those of the one-set-per-warp kernel
//     and of the CPU restatement bit for bit;
//   * in-edges are read in aligned 4-edge groups (one 32-byte load, one Philox
//     block per colour per group) with warp-level load balancing across
//     entries;
//   * the finished batch is compacted straight into the flat pool: one
//     atomicAdd reserves all W sets, per-colour shared cursors place members,
//     and the same pass clears the colour masks (atomicExch) for the next
//     batch, touching only vertices the batch reached.
// A batch whose frontier log overflows is abandoned; the CTA marks its slot
// dirty and leaves, and the host clears the scratch and re-runs the batch's
// sets with the one-set-per-warp kernel (identical results).
#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

constexpr int FUSED_THREADS = 512;
constexpr int FUSED_WARPS = FUSED_THREADS / 32;
constexpr uint32_t kSharedLog = 4096;  // frontier-log entries staged in shared memory

template <int CW>
__global__ void __launch_bounds__(FUSED_THREADS)
ic_fused_kernel(FusedLaunch L) {
  constexpr int W = 64 * CW;
  __shared__ uint64_t s_set[W];
  __shared__ unsigned long long s_start[W];
  __shared__ uint32_t s_size[W];
  __shared__ uint32_t s_fill[W];
  __shared__ uint32_t s_batch, s_ncol, s_tail, s_overflow;
  __shared__ uint32_t s_log[kSharedLog];  // log entries [0, kSharedLog)
  __shared__ unsigned long long s_base, s_work;

  const uint32_t tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
  const uint32_t slot = blockIdx.x;
  const uint32_t n = L.G.n;
  uint64_t *vis = L.vis + (size_t)slot * n * CW;
  uint64_t *pend = L.pend + (size_t)slot * n * CW;
  uint32_t *pflag = L.pflag + (size_t)slot * n;
  uint32_t *log = L.log + (size_t)slot * L.lcap;
  const uint32_t lcap = L.lcap;
  unsigned long long n_exp = 0, n_edges = 0, n_sexp = 0, n_sedges = 0,
                     n_sets = 0, n_elems = 0;
  // per-batch work, folded into the totals only when the batch is stored
  unsigned long long b_exp = 0, b_edges = 0, b_sexp = 0, b_sedges = 0;

  for (;;) {
    if (tid == 0) {
      s_batch = atomicAdd(L.next, 1u);
      s_tail = 0;
      s_overflow = 0;
      s_work = 0;
    }
    __syncthreads();
    const uint32_t b = s_batch;
    if (b >= L.num_batches) break;
    const uint32_t c0 = b * W;
    const uint32_t ncol = min((uint32_t)W, L.count - c0);
    if (tid == 0) s_ncol = ncol;
    for (uint32_t c = tid; c < W; c += FUSED_THREADS) {
      s_size[c] = 0;
      s_fill[c] = 0;
      if (c < ncol) {
        const uint32_t rel = L.order ? L.order[c0 + c] : c0 + c;
        s_set[c] = L.first + rel;
      }
    }
    __syncthreads();
    // seed the roots: level 1
    for (uint32_t c = tid; c < ncol; c += FUSED_THREADS) {
      const uint32_t r = root_of(L.key, s_set[c], n);
      const uint64_t bit = 1ull << (c & 63);
      atomicOr((unsigned long long *)&vis[(size_t)r * CW + (c >> 6)], bit);
      atomicOr((unsigned long long *)&pend[(size_t)r * CW + (c >> 6)], bit);
      atomicAdd(&s_size[c], 1u);
      if (atomicExch(&pflag[r], 1u) != 1u) {
        const uint32_t pos = atomicAdd(&s_tail, 1u);
        if (pos < lcap) {
          if (pos < kSharedLog) s_log[pos] = r;
          else log[pos] = r;
        }
        else s_overflow = 1;
      }
    }
    __syncthreads();
    b_exp = b_edges = b_sexp = b_sedges = 0;
    uint32_t lvl_start = 0, lvl_end = min(s_tail, lcap), level = 1;
    while (lvl_start < lvl_end && !s_overflow) {
      // ---- expand level `level`: entries log[lvl_start, lvl_end) ----------
      for (uint32_t eb = lvl_start + wid * 32; eb < lvl_end; eb += FUSED_WARPS * 32) {
        const uint32_t ei = eb + lane;
        uint64_t mask[CW];
        uint32_t beg = 0, end = 0, ng = 0;
#pragma unroll
        for (int w = 0; w < CW; ++w) mask[w] = 0;
        if (ei < lvl_end) {
          const uint32_t v = ei < kSharedLog ? s_log[ei] : log[ei];
          uint32_t any = 0;
#pragma unroll
          for (int w = 0; w < CW; ++w) {
            mask[w] = atomicExch((unsigned long long *)&pend[(size_t)v * CW + w], 0ull);
            any |= mask[w] != 0;
          }
          if (any) {
            beg = __ldg(L.G.off + v);
            end = __ldg(L.G.off + v + 1);
            ng = group_count(beg, end);
            uint32_t pc = 0;
#pragma unroll
            for (int w = 0; w < CW; ++w) pc += __popcll(mask[w]);
            b_exp += 1;
            b_edges += end - beg;
            if (L.work_cap) atomicAdd(&s_work, (unsigned long long)(end - beg));
            b_sexp += pc;
            b_sedges += (unsigned long long)pc * (end - beg);
          }
        }
        const uint32_t incl = warp_incl_scan(ng);
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        for (uint32_t base = 0; base < total; base += 32) {
          const uint32_t j = base + lane;
          const bool valid = j < total;
          const uint32_t owner = warp_find_owner(incl, valid ? j : total - 1);
          const uint32_t ob = __shfl_sync(FULL, beg, owner);
          const uint32_t oe = __shfl_sync(FULL, end, owner);
          const uint32_t oexcl = __shfl_sync(FULL, incl, owner) -
                                 __shfl_sync(FULL, ng, owner);
          uint64_t om[CW];
#pragma unroll
          for (int w = 0; w < CW; ++w) om[w] = __shfl_sync(FULL, mask[w], owner);
          uint64_t live[4][CW];
          uint32_t u[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            u[t] = 0;
#pragma unroll
            for (int w = 0; w < CW; ++w) live[t][w] = 0;
          }
          if (valid) {
            const uint32_t g = (ob >> 2) + (j - oexcl);
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
                uint64_t mm = om[w];
                while (mm) {
                  const int bi = __ffsll((long long)mm) - 1;
                  mm &= mm - 1;
                  const uint64_t sid = s_set[w * 64 + bi];
                  // this group's four coarse coins: half of the 8-edge block
                  const u32x4 cb = ic_block(L.key, g >> 1, sid);
                  const uint32_t hb = (g & 1u) << 2;
                  const uint64_t bit = 1ull << bi;
                  uint32_t tie = 0;
#pragma unroll
                  for (int t = 0; t < 4; ++t) {
                    const uint32_t th = rec[t].y >> 16, cc = coarse_of(cb, hb + t);
                    if (inr[t]) {
                      if (cc < th) live[t][w] |= bit;
                      else if (cc == th) tie |= 1u << t;
                    }
                  }
                  while (tie) {  // a coarse tie, one edge in 65 536: the fine half decides
                    const uint32_t t = __ffs(tie) - 1;
                    tie &= tie - 1;
                    const uint32_t thr = t == 0 ? rec[0].y : t == 1 ? rec[1].y : t == 2 ? rec[2].y : rec[3].y;
                    if (ic_fine_call(L.key, (g << 2) + t, sid) < (thr & 0xFFFFu)) {
                      if (t == 0) live[0][w] |= bit;
                      else if (t == 1) live[1][w] |= bit;
                      else if (t == 2) live[2][w] |= bit;
                      else live[3][w] |= bit;
                    }
                  }
                }
              }
            }
          }
          // apply discoveries
          bool push[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            bool added = false;
#pragma unroll
            for (int w = 0; w < CW; ++w) {
              if (live[t][w]) {
                const uint64_t old = atomicOr(
                    (unsigned long long *)&vis[(size_t)u[t] * CW + w], live[t][w]);
                uint64_t add = live[t][w] & ~old;
                if (add) {
                  atomicOr((unsigned long long *)&pend[(size_t)u[t] * CW + w], add);
                  added = true;
                  while (add) {
                    const int bi = __ffsll((long long)add) - 1;
                    add &= add - 1;
                    atomicAdd(&s_size[w * 64 + bi], 1u);
                  }
                }
              }
            }
            push[t] = added && atomicExch(&pflag[u[t]], level + 1) != level + 1;
          }
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const uint32_t bal = __ballot_sync(FULL, push[t]);
            if (!bal) continue;
            uint32_t pos0 = 0;
            if (lane == (uint32_t)(__ffs(bal) - 1)) pos0 = atomicAdd(&s_tail, __popc(bal));
            pos0 = __shfl_sync(FULL, pos0, __ffs(bal) - 1);
            if (push[t]) {
              const uint32_t pos = pos0 + __popc(bal & lanemask_lt());
              if (pos < lcap) {
                if (pos < kSharedLog) s_log[pos] = u[t];
                else log[pos] = u[t];
              }
              else s_overflow = 1;
            }
          }
        }
      }
      __syncthreads();
      lvl_start = lvl_end;
      lvl_end = min(s_tail, lcap);
      ++level;
      // a batch that outgrows its edge budget goes to the CTA-per-set sampler
      if (tid == 0 && L.work_cap && s_work > L.work_cap && !s_overflow) s_overflow = 3;
      __syncthreads();
    }
    if (s_overflow == 1) {
      // Abandon: the scratch may now hold colours of vertices that never
      // reached the log.  Record the batch, mark the slot dirty and stop.
      if (tid == 0) {
        L.F.ids[atomicAdd(L.F.count, 1u)] = b;
        atomicAdd(L.dirty, 1u);
      }
      break;
    }
    // ---- compaction into the pool ----------------------------------------
    if (tid == 0 && s_overflow == 0) {
      unsigned long long tot = 0;
      for (uint32_t c = 0; c < ncol; ++c) tot += s_size[c];
      const unsigned long long base = atomicAdd(L.P.cursor, tot);
      s_base = base;
      if (base + tot > L.P.cap) {
        atomicMin(L.F.first_bad_base, base);
        s_overflow = 2;
      } else {
        unsigned long long run = base;
        for (uint32_t c = 0; c < ncol; ++c) {
          s_start[c] = run;
          run += s_size[c];
        }
      }
    }
    __syncthreads();
    const bool store = s_overflow == 0;
    if (store) {
      n_exp += b_exp;
      n_edges += b_edges;
      n_sexp += b_sexp;
      n_sedges += b_sedges;
      for (uint32_t c = tid; c < ncol; c += FUSED_THREADS) {
        L.P.set_off[s_set[c]] = s_start[c];
        L.P.set_len[s_set[c]] = s_size[c];
      }
    }
    const uint32_t tail = min(s_tail, lcap);
    const bool aborted = s_overflow == 3;  // frontier left unexpanded: clear pend too
    for (uint32_t i = tid; i < tail; i += FUSED_THREADS) {
      const uint32_t v = i < kSharedLog ? s_log[i] : log[i];
#pragma unroll
      for (int w = 0; w < CW; ++w) {
        if (aborted) pend[(size_t)v * CW + w] = 0ull;
        uint64_t mm = atomicExch((unsigned long long *)&vis[(size_t)v * CW + w], 0ull);
        while (mm && store) {
          const int bi = __ffsll((long long)mm) - 1;
          mm &= mm - 1;
          const uint32_t c = w * 64 + bi;
          const uint32_t pos = atomicAdd(&s_fill[c], 1u);
          L.P.vtx[s_start[c] + pos] = v;
        }
      }
      pflag[v] = 0;
    }
    if (tid == 0) {
      if (store) {
        unsigned long long tot = 0;
        for (uint32_t c = 0; c < ncol; ++c) tot += s_size[c];
        n_sets += ncol;
        n_elems += tot;
      } else {
        L.F.ids[atomicAdd(L.F.count, 1u)] = aborted ? (b | FAIL_BIG) : b;
      }
    }
    __syncthreads();
  }
  n_exp = warp_sum_u64(n_exp);
  n_edges = warp_sum_u64(n_edges);
  n_sexp = warp_sum_u64(n_sexp);
  n_sedges = warp_sum_u64(n_sedges);
  if (lane == 0) {
    atomicAdd(L.st.v + 0, n_exp);
    atomicAdd(L.st.v + 1, n_edges);
    atomicAdd(L.st.v + 4, n_sexp);
    atomicAdd(L.st.v + 5, n_sedges);
  }
  if (tid == 0) {
    atomicAdd(L.st.v + 2, n_sets);
    atomicAdd(L.st.v + 3, n_elems);
  }
}

}  // namespace

void launch_ic_fused(const FusedLaunch &L, cudaStream_t stream) {
  count_launches(1);
  if (L.colors == 64)
    ic_fused_kernel<1><<<L.blocks, FUSED_THREADS, 0, stream>>>(L);
  else if (L.colors == 128)
    ic_fused_kernel<2><<<L.blocks, FUSED_THREADS, 0, stream>>>(L);
  else
    ic_fused_kernel<4><<<L.blocks, FUSED_THREADS, 0, stream>>>(L);
}

int fused_ctas_per_sm(uint32_t colors) {
  int nb = 0;
  if (colors == 64)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ic_fused_kernel<1>, FUSED_THREADS, 0);
  else if (colors == 128)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ic_fused_kernel<2>, FUSED_THREADS, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ic_fused_kernel<4>, FUSED_THREADS, 0);
  return nb > 0 ? nb : 1;
}

// ---- export gather: sets [first, first+count) -> out, in set-id order -----
namespace {
__global__ void __launch_bounds__(256)
gather_sets_kernel(DevPool P, uint64_t first, uint64_t count,
                   const uint64_t *csr, uint32_t *out) {
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = lane_id();
  for (uint64_t i = gw; i < count; i += nw) {
    const uint64_t s = first + i;
    const uint64_t off = P.set_off[s];
    const uint32_t len = P.set_len[s];
    const uint64_t o = csr[i];
    for (uint32_t j = lane; j < len; j += 32) out[o + j] = P.vtx[off + j];
  }
}
}  // namespace

void launch_gather_sets(const DevPool &P, uint64_t first, uint64_t count,
                        const uint64_t *csr, uint32_t *out, cudaStream_t s) {
  count_launches(1);
  if (count == 0) return;
  gather_sets_kernel<<<1184, 256, 0, s>>>(P, first, count, csr, out);
}

}  // namespace rip
