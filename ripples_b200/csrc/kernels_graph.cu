// kernels_graph.cu -- packs a backward CSR into the sampler's layout.
//
// The reference keeps index u64[n+1], edges u32[m], weights f32[m] as three
// arrays (include/ripples/graph.h:364-1086; device copy in
// src/gpu/gpu_graph.cc:48-84) and compares a fresh uniform01 draw with the
// float weight on every coin flip.  Here the weight is converted once into an
// integer threshold and interleaved with the source id, so one aligned 8-byte
// record serves an edge and the coin test is an integer compare:
//   IC : thr = clamp(floor(w * 2^32), 0, 2^32-1)   live iff coin < thr
//   LT : thr = min(min(sum_{i<=e} W_i, 2^41) >> 8, 2^32-1) over the vertex's
//        in-edges in CSR order, W_i = floor(clamp(w_i, 0, 2) * 2^40): exact
//        64-bit fixed point, so the prefix sum may run in any order (here a
//        warp-parallel scan) and still equal a left-to-right sum bit for bit
// Offsets shrink to u32 (m < 2^32 is required).
#include <atomic>

#include "device.cuh"
#include "launch.h"

namespace rip {

namespace {

__device__ __forceinline__ uint32_t prob_u32(double p) {
  const double y = p * 4294967296.0;
  if (!(y > 0.0)) return 0u;
  if (y >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)floor(y);
}

__global__ void pack_off_kernel(const uint64_t *index, uint32_t n,
                                uint32_t *off) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= n;
       v += (uint64_t)gridDim.x * blockDim.x)
    off[v] = (uint32_t)index[v];
}

__global__ void pack_ic_kernel(const uint32_t *src, const float *w, uint64_t m,
                               uint64_t m_pad, uint2 *edges) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m_pad;
       e += (uint64_t)gridDim.x * blockDim.x)
    edges[e] = e < m ? make_uint2(src[e], prob_u32((double)w[e]))
                     : make_uint2(0u, 0u);
}

__device__ __forceinline__ uint64_t lt_fixed(float w) {
  const double x = (double)w;
  if (!(x > 0.0)) return 0ull;
  if (x >= 2.0) return 2ull << 40;
  return (uint64_t)floor(x * 1099511627776.0);  // exact: w has a 24-bit mantissa
}

__device__ __forceinline__ uint64_t sat_add(uint64_t a, uint64_t b) {
  const uint64_t s = a + b;  // a, b <= 2^41: no wrap
  return s > (1ull << 41) ? (1ull << 41) : s;
}

// One warp per vertex: coalesced 32-edge chunks, a saturating integer warp
// scan per chunk, carried across chunks.
__global__ void pack_lt_kernel(const uint64_t *index, const uint32_t *src,
                               const float *w, uint32_t n, uint64_t m,
                               uint64_t m_pad, uint2 *edges) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  // 32 consecutive vertices per warp: a lane scans its own vertex when it has
  // at most 32 in-edges (most vertices); the warp scans each larger one
  // together, 32 edges per step with a shuffle scan
  for (uint64_t v0 = gw * 32; v0 < n; v0 += nw * 32) {
    const uint64_t v = v0 + lane;
    uint64_t beg = 0, end = 0;
    if (v < n) {
      beg = index[v];
      end = index[v + 1];
    }
    if (end - beg <= 32) {
      uint64_t run = 0;
      for (uint64_t e = beg; e < end; ++e) {
        run = sat_add(run, lt_fixed(w[e]));
        const uint64_t c = run >> 8;
        edges[e] = make_uint2(src[e], c > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)c);
      }
    }
    uint32_t big = __ballot_sync(0xFFFFFFFFu, end - beg > 32);
    while (big) {
      const uint32_t L = __ffs(big) - 1;
      big &= big - 1;
      const uint64_t b = __shfl_sync(0xFFFFFFFFu, beg, L), t = __shfl_sync(0xFFFFFFFFu, end, L);
      uint64_t carry = 0;
      for (uint64_t base = b; base < t; base += 32) {
        const uint64_t e = base + lane;
        uint64_t x = e < t ? lt_fixed(w[e]) : 0ull;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
          if (lane >= (uint32_t)d) x = sat_add(x, y);
        }
        x = sat_add(x, carry);
        if (e < t) {
          const uint64_t c = x >> 8;
          edges[e] = make_uint2(src[e], c > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)c);
        }
        carry = __shfl_sync(0xFFFFFFFFu, x, 31);
      }
    }
  }
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = m + tid; e < m_pad; e += stride) edges[e] = make_uint2(0u, 0u);
}

}  // namespace

static std::atomic<uint64_t> g_launches{0};
uint64_t launch_counter() { return g_launches.load(); }
void count_launches(uint64_t n) { g_launches.fetch_add(n); }
void uncount_launches(uint64_t n) { g_launches.fetch_sub(n); }

static uint64_t pad4(uint64_t m) { return (m + 3) & ~uint64_t(3); }

void launch_pack_ic(const uint64_t *index, const float *w, uint32_t n,
                    uint64_t m, uint32_t *off, uint2 *edges, const uint32_t *src,
                    cudaStream_t stream) {
  count_launches(2);
  pack_off_kernel<<<1184, 256, 0, stream>>>(index, n, off);
  pack_ic_kernel<<<2368, 256, 0, stream>>>(src, w, m, pad4(m) + 4, edges);
}

// *bad = entries with index[v + 1] < index[v] plus sources >= n
__global__ void validate_csr_kernel(const uint64_t *index, const uint32_t *src, uint32_t n,
                                    uint64_t m, unsigned long long *bad) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long b = 0;
  for (uint64_t v = tid; v < n; v += stride) b += index[v + 1] < index[v];
  for (uint64_t e = tid; e < m; e += stride) b += src[e] >= n;
  for (int d = 16; d > 0; d >>= 1) b += __shfl_xor_sync(0xFFFFFFFFu, b, d);
  if ((threadIdx.x & 31u) == 0 && b) atomicAdd(bad, b);
}

void launch_validate_csr(const uint64_t *index, const uint32_t *src, uint32_t n, uint64_t m,
                         unsigned long long *bad, cudaStream_t stream) {
  count_launches(1);
  cudaMemsetAsync(bad, 0, sizeof(*bad), stream);
  validate_csr_kernel<<<2368, 256, 0, stream>>>(index, src, n, m, bad);
}

// vthr[v] = the threshold every in-edge of v shares, else 0; lam[v] = the
// expected number of live in-edges of v (sum of its thresholds / 2^32).  One
// warp per vertex.  sums[0] += in-degrees of the uniform vertices with at
// least two in-edges (the edge reads the IC samplers can skip).
__global__ void uniform_threshold_kernel(const uint32_t *off, const uint2 *edges, uint32_t n,
                                         uint32_t *vthr, float *lam, unsigned long long *sums) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long cov = 0;
  for (uint64_t v = warp; v < n; v += warps) {
    const uint32_t beg = off[v], end = off[v + 1];
    const uint32_t t = end > beg ? edges[beg].y : 0u;
    bool same = true;
    unsigned long long tsum = 0;
    for (uint32_t e = beg + lane; e < end; e += 32) {
      const uint32_t x = edges[e].y;
      same = same && x == t;
      tsum += x;
    }
    same = __all_sync(0xFFFFFFFFu, same);
    for (int d = 16; d > 0; d >>= 1) tsum += __shfl_xor_sync(0xFFFFFFFFu, tsum, d);
    if (lane == 0) {
      vthr[v] = same ? t : 0u;
      lam[v] = (float)((double)tsum * (1.0 / 4294967296.0));
      if (same && t && end - beg >= 2) cov += end - beg;
    }
  }
  if (lane == 0 && cov) atomicAdd(sums, cov);
}

// *total (a double) += lam[source] over every edge: divided by m it is the
// branching factor of a reverse BFS (the expected live in-edges of the vertex
// an edge leads to).
__global__ void branching_kernel(const uint2 *edges, uint64_t m, const float *lam,
                                 double *total) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  double acc = 0.0;
  for (uint64_t e = tid; e < m; e += stride) acc += (double)lam[edges[e].x];
  for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, d);
  if ((threadIdx.x & 31u) == 0 && acc != 0.0) atomicAdd(total, acc);
}

void launch_uniform_threshold(const uint32_t *off, const uint2 *edges, uint32_t n, uint64_t m,
                              uint32_t *vthr, float *lam, unsigned long long *sums,
                              cudaStream_t stream) {
  count_launches(2);
  cudaMemsetAsync(sums, 0, 2 * sizeof(*sums), stream);
  uniform_threshold_kernel<<<2368, 256, 0, stream>>>(off, edges, n, vthr, lam, sums);
  branching_kernel<<<2368, 256, 0, stream>>>(edges, m, lam, reinterpret_cast<double *>(sums + 1));
}

void launch_pack_lt(const uint64_t *index, const float *w, uint32_t n,
                    uint64_t m, uint32_t *off, uint2 *edges, const uint32_t *src,
                    cudaStream_t stream) {
  count_launches(2);
  pack_off_kernel<<<1184, 256, 0, stream>>>(index, n, off);
  pack_lt_kernel<<<2368, 256, 0, stream>>>(index, src, w, n, m, pad4(m) + 4,
                                           edges);
}

}  // namespace rip
