// kernels_graphgen.cu -- synthetic graph construction on the device.
//
// The same R-MAT draws as the host generator (graphgen.cpp), produced on the
// GPU for graphs too large to build on the host quickly (2^24 vertices and
// 2^29 edge draws), and a CSR builder that turns sorted, unique (dst, src)
// keys into a packed rip_graph with the synthetic weight models.
//   key of edge draw i = (dst << 32) | src, ~0 for a self-loop
//   weights of CSR edge e: Philox(seed; e, WEIGHT) as in graphgen.cpp
#include "device.cuh"
#include "launch.h"
#include "ripples_b200.h"

namespace rip {

namespace {

constexpr uint32_t DOM_RMAT = 4, DOM_ER = 5, DOM_WEIGHT = 6;

__global__ void rmat_keys_kernel(uint32_t scale, uint64_t first, uint64_t count,
                                 uint32_t TA, uint32_t TB, uint32_t TC, Key key,
                                 unsigned long long *keys) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = first + j;
    uint32_t s = 0, d = 0;
    u32x4 r{0, 0, 0, 0};
    for (uint32_t l = 0; l < scale; ++l) {
      if ((l & 3) == 0) r = philox((uint32_t)i, (uint32_t)(i >> 32), l >> 2, DOM_RMAT << 24,
                                   key.k0, key.k1);
      const uint32_t u = lane_of(r, l & 3);
      const uint32_t rb = u >= TB ? 1u : 0u;
      const uint32_t cb = ((u >= TA && u < TB) || u >= TC) ? 1u : 0u;
      s |= rb << (scale - 1 - l);
      d |= cb << (scale - 1 - l);
    }
    keys[j] = s == d ? ~0ull : (((unsigned long long)d << 32) | s);
  }
}

// Erdos-Renyi draw i: src = mulhi(P(i; ER)[0], n), dst = mulhi(P(i; ER)[1], n),
// as graphgen.cpp draws it.
__global__ void er_keys_kernel(uint32_t n, uint64_t first, uint64_t count, Key key,
                               unsigned long long *keys) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = first + j;
    const u32x4 r = philox((uint32_t)i, (uint32_t)(i >> 32), 0u, DOM_ER << 24, key.k0, key.k1);
    const uint32_t s = (uint32_t)(((uint64_t)r.x * n) >> 32);
    const uint32_t d = (uint32_t)(((uint64_t)r.y * n) >> 32);
    keys[j] = s == d ? ~0ull : (((unsigned long long)d << 32) | s);
  }
}

// index[v] = first position whose key >= v << 32 (keys sorted, unique, no ~0)
__global__ void csr_index_kernel(const unsigned long long *keys, uint64_t m,
                                 uint32_t n, uint64_t *index, uint32_t *src) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v <= n; v += stride) {
    const unsigned long long target = (unsigned long long)v << 32;
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (keys[mid] < target) lo = mid + 1;
      else hi = mid;
    }
    index[v] = lo;
  }
  for (uint64_t e = tid; e < m; e += stride) src[e] = (uint32_t)keys[e];
}

__device__ __forceinline__ double weight_unif(Key k, uint64_t e) {
  const u32x4 r = philox((uint32_t)e, (uint32_t)(e >> 32), 0u, DOM_WEIGHT << 24, k.k0, k.k1);
  return (double)(r.x >> 8) * (1.0 / 16777216.0);
}

// Weight models of rip_make_weights (graphgen.cpp), on the device.  LT
// normalisation sums in double, left to right per vertex, like the host.
__global__ void weights_kernel(int kind, const uint64_t *index, uint32_t n, Key k,
                               double lo, double hi, float *w) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = tid; v < n; v += stride) {
    const uint64_t b = index[v], e1 = index[v + 1];
    if (kind == RIP_WEIGHTS_UNIFORM) {
      for (uint64_t e = b; e < e1; ++e) w[e] = (float)(lo + (hi - lo) * weight_unif(k, e));
    } else if (kind == RIP_WEIGHTS_WC) {
      const float x = (float)(1.0 / (double)(e1 - b));
      for (uint64_t e = b; e < e1; ++e) w[e] = x;
    } else {
      double sum = 0.0;
      for (uint64_t e = b; e < e1; ++e) {
        const float r = (float)weight_unif(k, e);
        w[e] = r;
        sum += (double)r;
      }
      for (uint64_t e = b; e < e1; ++e)
        w[e] = sum > 0.0 ? (float)((double)w[e] / sum) : 0.0f;
    }
  }
}

}  // namespace

void launch_rmat_keys(uint32_t scale, uint64_t first, uint64_t count, double a, double b,
                      double c, uint64_t seed, unsigned long long *keys,
                      cudaStream_t stream) {
  count_launches(1);
  rmat_keys_kernel<<<2368, 256, 0, stream>>>(scale, first, count, prob_u32_host(a),
                                             prob_u32_host(a + b), prob_u32_host(a + b + c),
                                             make_key(seed), keys);
}

void launch_er_keys(uint32_t n, uint64_t first, uint64_t count, uint64_t seed,
                    unsigned long long *keys, cudaStream_t stream) {
  count_launches(1);
  er_keys_kernel<<<2368, 256, 0, stream>>>(n, first, count, make_key(seed), keys);
}

void launch_csr_from_keys(const unsigned long long *keys, uint64_t m, uint32_t n,
                          uint64_t *index, uint32_t *src, cudaStream_t stream) {
  count_launches(1);
  csr_index_kernel<<<2368, 256, 0, stream>>>(keys, m, n, index, src);
}

void launch_weights(int kind, const uint64_t *index, uint32_t n, uint64_t seed, double lo,
                    double hi, float *w, cudaStream_t stream) {
  count_launches(1);
  weights_kernel<<<1184, 128, 0, stream>>>(kind, index, n, make_key(seed), lo, hi, w);
}

}  // namespace rip
