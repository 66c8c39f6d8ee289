// graphgen.cpp -- host-side synthetic graph construction for ripples_b200.
//
// R-MAT and Erdos-Renyi edge sampling, backward-CSR assembly, the synthetic
// edge-weight models, and the reference's binary graph writer.  These produce
// the INPUTS of the hot path; they are deterministic in their seeds so the
// same graph can be rebuilt anywhere (and fed to the reference through its
// --reload-binary path, include/ripples/graph.h:854-995).
//
// Random draws come from Philox4x32-10 (Salmon et al., SC'11) in counter mode:
//   R-MAT edge i, level l : P(key=seed, ctr=(i_lo, i_hi, l/4, RMAT<<24))[l%4]
//   ER edge i             : P(key=seed, ctr=(i_lo, i_hi, 0, ER<<24))[0..1]
//   weight of CSR edge e  : P(key=seed, ctr=(e_lo, e_hi, 0, WEIGHT<<24))[0]
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <parallel/algorithm>
#include <vector>

#include <omp.h>

#include "ripples_b200.h"
#include "philox.cuh"

namespace {

using rip::philox4x32_10;

constexpr uint32_t DOM_RMAT = 4, DOM_ER = 5, DOM_WEIGHT = 6;

inline uint32_t prob_u32(double p) {
  double y = p * 4294967296.0;
  if (!(y > 0.0)) return 0u;
  if (y >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)std::floor(y);
}

// keys are (dst << 32 | src); sorted + unique gives the backward CSR directly.
int keys_to_csr(std::vector<uint64_t> &keys, uint32_t n, uint64_t **index_out,
                uint32_t **src_out, uint64_t *m_out) {
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  uint64_t m = keys.size();
  uint64_t *index = (uint64_t *)std::malloc(sizeof(uint64_t) * ((size_t)n + 1));
  uint32_t *src = (uint32_t *)std::malloc(sizeof(uint32_t) * (m ? m : 1));
  if (!index || !src) {
    std::free(index);
    std::free(src);
    return RIP_ERR_NOMEM;
  }
  std::memset(index, 0, sizeof(uint64_t) * ((size_t)n + 1));
#pragma omp parallel for schedule(static)
  for (uint64_t e = 0; e < m; ++e) src[e] = (uint32_t)keys[e];
  // index[v] = first position whose dst >= v (keys are sorted by dst)
  for (uint64_t e = 0; e < m; ++e) index[(keys[e] >> 32) + 1]++;
  for (uint64_t v = 0; v < n; ++v) index[v + 1] += index[v];
  *index_out = index;
  *src_out = src;
  *m_out = m;
  return RIP_OK;
}

}  // namespace

extern "C" {

int rip_rmat_csr(uint32_t scale, uint64_t num_edges, double a, double b,
                 double c, uint64_t seed, uint64_t **index, uint32_t **src,
                 uint64_t *m) {
  if (!index || !src || !m || scale == 0 || scale > 31) return RIP_ERR_INVALID;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return RIP_ERR_INVALID;
  const uint32_t n = 1u << scale;
  const uint32_t TA = prob_u32(a), TB = prob_u32(a + b), TC = prob_u32(a + b + c);
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  std::vector<uint64_t> keys(num_edges);
  size_t kept = 0;
#pragma omp parallel
  {
    std::vector<uint64_t> local;
    local.reserve(num_edges / omp_get_num_threads() + 16);
#pragma omp for schedule(static)
    for (uint64_t i = 0; i < num_edges; ++i) {
      uint32_t s = 0, d = 0;
      uint32_t out[4];
      for (uint32_t l = 0; l < scale; ++l) {
        if ((l & 3) == 0) {
          const uint32_t ctr[4] = {(uint32_t)i, (uint32_t)(i >> 32), l >> 2,
                                   DOM_RMAT << 24};
          philox4x32_10(ctr, key, out);
        }
        uint32_t u = out[l & 3];
        uint32_t rb = (u >= TB) ? 1u : 0u;                 // row: quadrants c, d
        uint32_t cb = (u >= TA && u < TB) || (u >= TC) ? 1u : 0u;  // col: b, d
        s |= rb << (scale - 1 - l);
        d |= cb << (scale - 1 - l);
      }
      if (s != d) local.push_back(((uint64_t)d << 32) | s);
    }
    size_t off;
#pragma omp atomic capture
    {
      off = kept;
      kept += local.size();
    }
    std::copy(local.begin(), local.end(), keys.begin() + off);
  }
  keys.resize(kept);
  return keys_to_csr(keys, n, index, src, m);
}

int rip_er_csr(uint32_t n, uint64_t num_edges, uint64_t seed, uint64_t **index,
               uint32_t **src, uint64_t *m) {
  if (!index || !src || !m || n < 2) return RIP_ERR_INVALID;
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  std::vector<uint64_t> keys(num_edges);
  size_t kept = 0;
#pragma omp parallel
  {
    std::vector<uint64_t> local;
#pragma omp for schedule(static)
    for (uint64_t i = 0; i < num_edges; ++i) {
      uint32_t out[4];
      const uint32_t ctr[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0, DOM_ER << 24};
      philox4x32_10(ctr, key, out);
      uint32_t s = (uint32_t)(((uint64_t)out[0] * n) >> 32);
      uint32_t d = (uint32_t)(((uint64_t)out[1] * n) >> 32);
      if (s != d) local.push_back(((uint64_t)d << 32) | s);
    }
    size_t off;
#pragma omp atomic capture
    {
      off = kept;
      kept += local.size();
    }
    std::copy(local.begin(), local.end(), keys.begin() + off);
  }
  keys.resize(kept);
  return keys_to_csr(keys, n, index, src, m);
}

int rip_make_weights(int kind, uint32_t n, const uint64_t *index, uint64_t m,
                     uint64_t seed, double lo, double hi, float *w) {
  if (!index || (!w && m) || index[n] != m) return RIP_ERR_INVALID;
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  auto unif = [&](uint64_t e) {
    uint32_t out[4];
    const uint32_t ctr[4] = {(uint32_t)e, (uint32_t)(e >> 32), 0, DOM_WEIGHT << 24};
    philox4x32_10(ctr, key, out);
    return (double)(out[0] >> 8) * (1.0 / 16777216.0);  // [0, 1), 24 bits
  };
  if (kind == RIP_WEIGHTS_UNIFORM) {
#pragma omp parallel for schedule(static)
    for (uint64_t e = 0; e < m; ++e) w[e] = (float)(lo + (hi - lo) * unif(e));
  } else if (kind == RIP_WEIGHTS_LT_NORMALIZED) {
#pragma omp parallel for schedule(dynamic, 1024)
    for (uint64_t v = 0; v < n; ++v) {
      double sum = 0.0;
      for (uint64_t e = index[v]; e < index[v + 1]; ++e) {
        float r = (float)unif(e);
        w[e] = r;
        sum += (double)r;
      }
      for (uint64_t e = index[v]; e < index[v + 1]; ++e)
        w[e] = sum > 0.0 ? (float)((double)w[e] / sum) : 0.0f;
    }
  } else if (kind == RIP_WEIGHTS_WC) {
#pragma omp parallel for schedule(dynamic, 1024)
    for (uint64_t v = 0; v < n; ++v) {
      uint64_t d = index[v + 1] - index[v];
      for (uint64_t e = index[v]; e < index[v + 1]; ++e)
        w[e] = (float)(1.0 / (double)d);
    }
  } else {
    return RIP_ERR_INVALID;
  }
  return RIP_OK;
}

// Reference binary layout (include/ripples/graph.h:700-771): five uint64
// header words (0xc0ffee endianness check, direction 0xa1ccac0f backward /
// 0xf0cacc1a forward, weight type 32 = float, n, m), then reverseMap u32[n]
// (identity), index u64[n+1], edges u32[m], weights f32[m].
int rip_write_binary(const char *path, uint32_t n, uint64_t m,
                     const uint64_t *index, const uint32_t *src, const float *w,
                     int backward) {
  if (!path || !index || (m && (!src || !w))) return RIP_ERR_INVALID;
  std::vector<uint64_t> tindex;
  std::vector<uint32_t> tsrc;
  std::vector<float> tw;
  const uint64_t *I = index;
  const uint32_t *S = src;
  const float *W = w;
  if (!backward) {  // transpose the backward CSR into the forward CSR
    tindex.assign((size_t)n + 1, 0);
    tsrc.resize(m);
    tw.resize(m);
    for (uint64_t e = 0; e < m; ++e) tindex[src[e] + 1]++;
    for (uint64_t v = 0; v < n; ++v) tindex[v + 1] += tindex[v];
    std::vector<uint64_t> pos(tindex.begin(), tindex.end() - 1);
    for (uint32_t v = 0; v < n; ++v)
      for (uint64_t e = index[v]; e < index[v + 1]; ++e) {
        uint64_t p = pos[src[e]]++;
        tsrc[p] = v;
        tw[p] = w[e];
      }
    I = tindex.data();
    S = tsrc.data();
    W = tw.data();
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) return RIP_ERR_INVALID;
  uint64_t hdr[5] = {0xc0ffeeull, backward ? 0xa1ccac0full : 0xf0cacc1aull,
                     32ull, (uint64_t)n, m};
  bool ok = std::fwrite(hdr, sizeof(hdr), 1, f) == 1;
  std::vector<uint32_t> rmap(n);
  for (uint32_t v = 0; v < n; ++v) rmap[v] = v;
  ok = ok && std::fwrite(rmap.data(), sizeof(uint32_t), n, f) == n;
  ok = ok && std::fwrite(I, sizeof(uint64_t), (size_t)n + 1, f) == (size_t)n + 1;
  ok = ok && (m == 0 || std::fwrite(S, sizeof(uint32_t), m, f) == m);
  ok = ok && (m == 0 || std::fwrite(W, sizeof(float), m, f) == m);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? RIP_OK : RIP_ERR_INVALID;
}

void rip_free(void *ptr) { std::free(ptr); }

}  // extern "C"
