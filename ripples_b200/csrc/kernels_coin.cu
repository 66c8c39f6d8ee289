// kernels_coin.cu -- the throughput ceiling of the sampler's coin function.
//
// On uniform-threshold in-lists (weighted cascade: p = 1/in-degree) the IC
// samplers read almost nothing: per eight in-edges they draw one
// Philox4x32-10 block and compare the smallest of its eight 16-bit halves
// against the vertex's threshold (each half, and the fine half of a coin on
// a tie, only when that passes), so the SM's integer issue rate bounds them,
// not HBM.
// coin_rate_kernel draws coins the way a hub expansion does -- consecutive
// coin blocks of one set against one threshold -- with no memory traffic and
// full occupancy; its coins per second (rip_coin_rate) is the measured
// ceiling the sampler's coin rate is reported against.
#include "host.h"

namespace rip {
namespace {

__global__ void __launch_bounds__(256)
coin_rate_kernel(const __grid_constant__ RoundKeys rk, Key key, uint32_t blocks_per_thread,
                 uint32_t thr, unsigned long long *live) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t s = tid;                                 // one set per thread
  const uint64_t b0 = tid * (uint64_t)blocks_per_thread;  // its own coin blocks
  uint32_t cnt = 0;
  for (uint32_t i = 0; i < blocks_per_thread; ++i) {
    const u32x4 c = ic_block_rk(rk, b0 + i, s);
    if (block_min16(c) <= (thr >> 16)) {  // as the samplers: most blocks stop here
#pragma unroll
      for (int h = 0; h < 8; ++h)
        cnt += ic_live(key, s, ((b0 + i) << 3) + h, coarse_of(c, h), thr);
    }
  }
  for (int d = 16; d > 0; d >>= 1) cnt += __shfl_xor_sync(FULL, cnt, d);
  if ((threadIdx.x & 31u) == 0 && cnt) atomicAdd(live, (unsigned long long)cnt);
}

}  // namespace
}  // namespace rip

using namespace rip;

extern "C" int rip_coin_rate(rip_ctx *c, double *coins_per_s) {
  if (!c || !coins_per_s) return RIP_ERR_INVALID;
  CK(c, cudaSetDevice(c->device));
  DevMem live;
  TRY(dalloc(c, live, sizeof(unsigned long long)));
  const int blocks = c->num_sms * 8;  // 64 resident warps per SM
  const uint32_t cblocks = 1024;
  const Key key = make_key(0x5EEDull);
  const RoundKeys rk = round_keys(key);
  CK(c, cudaMemsetAsync(live.p, 0, sizeof(unsigned long long), c->stream));
  count_launches(2);
  coin_rate_kernel<<<blocks, 256, 0, c->stream>>>(rk, key, cblocks, 1u << 20,
                                                  ptr<unsigned long long>(live));
  CK(c, cudaEventRecord(c->ev0, c->stream));
  coin_rate_kernel<<<blocks, 256, 0, c->stream>>>(rk, key, cblocks, 1u << 20,
                                                  ptr<unsigned long long>(live));
  CK(c, cudaEventRecord(c->ev1, c->stream));
  CK(c, cudaEventSynchronize(c->ev1));
  CK(c, cudaGetLastError());
  float ms = 0.f;
  CK(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  dfree(c, live);
  *coins_per_s = ms > 0.f ? (double)blocks * 256.0 * cblocks * 8.0 / (ms * 1e-3) : 0.0;
  return RIP_OK;
}
