// sample_static.cu -- RRR sampling that allocates nothing.
//
// rip_sample_static() runs the one-set-per-warp samplers (ic_plain_kernel /
// lt_walk_kernel) with all of their scratch -- per-warp visited bitmaps and
// queues, the work/failure counters and the retry lists -- carved out of one
// file-scope device array, g_static_scratch, instead of memory from
// cudaMalloc.  It exists for callers that cannot allocate device memory at
// the moment they sample: a serving process whose HBM is reserved up front
// by its own arena allocator (a stray cudaMalloc fails or fragments it), code
// on a latency-critical path where cudaMalloc/cudaFree would synchronise the
// device, and plugin hosts that forbid allocations outside their allocator.
// The caller passes the packed graph and the output buffers; the library
// touches no other memory.
//
// Limits and rules:
//   * g_static_scratch is RIP_STATIC_SCRATCH_BYTES (32 MiB); every GPU that
//     loads this library holds it until the process exits.
//   * At most RIP_STATIC_MAX_SETS sets per call, and n small enough that
//     eight warps' scratch fits in the array: IC needs an n-bit bitmap plus a
//     queue per warp (n up to about 24 million vertices), LT only the queue
//     (its walks find revisits by scanning it).  Larger requests are rejected
//     with RIP_ERR_LIMIT and a message.
//   * Throughput follows the array size: the scratch is split into as many
//     warps as fit, at most 32 per SM.  With 24 MiB left after the id lists,
//     IC on n = 2^20 gets 120 warps (192 KiB each; rip_sample runs 4 736 on a
//     B200) and on n = 2^24 the minimum of 8, so large graphs sample far
//     slower than through rip_sample.  LT warps hold a 64 KiB queue each
//     (376 warps at any n); a walk may grow to about 786 000 vertices.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and the device's SM
//     count, and caches both.  Every call synchronises `stream` before it
//     returns.
//   * The cached address belongs to the device's primary context: after a
//     cudaDeviceReset on that device the process must not call this entry
//     point again.
//   * All calls share the one array and it keeps the last call's contents;
//     each call re-zeroes what must start at zero (counters, bitmaps).  Calls
//     whose work overlaps on the GPU (other streams, other host threads on the
//     same device) race on the array and must be serialised by the caller.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "launch.h"
#include "ripples_b200.h"

namespace rip {
namespace {

constexpr size_t kMetaBytes = 4096;
constexpr size_t kIdsBytes = (size_t)RIP_STATIC_MAX_SETS * sizeof(uint32_t);

// In host code this name is only a host-side stand-in for the device array;
// kernels get the address that cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_static_scratch[RIP_STATIC_SCRATCH_BYTES];

struct StaticMeta {  // at the start of g_static_scratch
  unsigned long long cursor;
  unsigned long long first_bad;
  unsigned long long stats[8];
  unsigned int fail_count;
  unsigned int next;
};

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};
int g_sms[kMaxDevices] = {};
thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// Device address of g_static_scratch on the current device and the device's
// SM count (set up once per device).
int scratch_address(unsigned char **out, int *sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(RIP_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(RIP_ERR_LIMIT, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      return fail(RIP_ERR_CUDA, "cudaGetSymbolAddress(g_static_scratch): %s",
                  cudaGetErrorString(e));
    int count = 0;
    e = cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || count <= 0)
      return fail(RIP_ERR_CUDA, "cudaDeviceGetAttribute(SM count): %s", cudaGetErrorString(e));
    g_sms[dev] = count;
    g_addr[dev] = p;
  }
  *out = static_cast<unsigned char *>(g_addr[dev]);
  *sms = g_sms[dev];
  return RIP_OK;
}

}  // namespace
}  // namespace rip

using namespace rip;

extern "C" const char *rip_static_last_error(void) { return g_err.c_str(); }

extern "C" int rip_sample_static(const uint32_t *d_off, const void *d_edges,
                                 uint32_t n, uint64_t m, int model, uint64_t seed,
                                 uint64_t first, uint32_t count, uint32_t *d_vertices,
                                 uint64_t vertex_capacity, uint64_t *d_set_offsets,
                                 uint32_t *d_set_lengths, uint64_t *num_elements,
                                 void *stream) {
  g_err.clear();
  if (!d_off || !d_edges || !d_vertices || !d_set_offsets || !d_set_lengths ||
      !num_elements || n == 0)
    return fail(RIP_ERR_INVALID, "rip_sample_static: null pointer or n == 0");
  if (model != RIP_MODEL_IC && model != RIP_MODEL_LT)
    return fail(RIP_ERR_INVALID, "rip_sample_static: unknown model %d", model);
  if (count > RIP_STATIC_MAX_SETS)
    return fail(RIP_ERR_LIMIT, "rip_sample_static: %u sets requested, at most %u per call",
                count, (unsigned)RIP_STATIC_MAX_SETS);
  if (first + count >= (1ull << 56))
    return fail(RIP_ERR_LIMIT, "rip_sample_static: set ids are limited to 2^56");
  *num_elements = 0;
  if (count == 0) return RIP_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char *base = nullptr;
  int sms = 0;
  int rc = scratch_address(&base, &sms);
  if (rc != RIP_OK) return rc;

  StaticMeta *meta = reinterpret_cast<StaticMeta *>(base);
  uint32_t *ids[2] = {reinterpret_cast<uint32_t *>(base + kMetaBytes),
                      reinterpret_cast<uint32_t *>(base + kMetaBytes + kIdsBytes)};
  unsigned char *work = base + kMetaBytes + 2 * kIdsBytes;
  const size_t work_bytes = RIP_STATIC_SCRATCH_BYTES - kMetaBytes - 2 * kIdsBytes;
  // IC warps keep an n-bit visited bitmap; LT walks need none
  const uint64_t bm_words = model == RIP_MODEL_IC ? (((uint64_t)n + 31) / 32 + 7) & ~7ull : 0;
  const uint64_t bm_bytes = bm_words * 4;

  // Partition: as many warps as fit (multiple of 8, at most 32 per SM of this
  // device), each with its bitmap and a queue of qcap entries.
  uint32_t qcap = n < (1u << 14) ? n : (1u << 14);
  auto warps_for = [&](uint32_t q) -> uint64_t {
    uint64_t w = work_bytes / (bm_bytes + 4ull * q);
    if (w > (uint64_t)sms * 32) w = (uint64_t)sms * 32;
    return w & ~7ull;
  };
  if (warps_for(qcap) < 8)
    return fail(RIP_ERR_LIMIT,
                "rip_sample_static: n = %u needs %llu bytes of scratch for 8 warps, the "
                "static array has %zu",
                n, (unsigned long long)(8 * (bm_bytes + 4ull * qcap)), work_bytes);

  if (cudaMemsetAsync(meta, 0, sizeof(StaticMeta), s) != cudaSuccess)
    return fail(RIP_ERR_CUDA, "cudaMemsetAsync(meta) failed");
  SampleLaunch L;
  L.G = DevGraph{n, m, d_off, static_cast<const uint2 *>(d_edges)};
  // The kernels index the set arrays by absolute set id, so they get the
  // caller's buffers moved back by `first` entries: entry `first` is then the
  // caller's index 0, and only ids in [first, first + count) are written.  The
  // moved addresses are formed in integer arithmetic (the pointer arithmetic
  // would leave the buffers' bounds) and are never dereferenced below `first`.
  auto moved_back = [first](void *ptr, size_t elem) {
    return reinterpret_cast<uintptr_t>(ptr) - (uintptr_t)(first * elem);
  };
  L.P = DevPool{d_vertices, &meta->cursor, vertex_capacity,
                reinterpret_cast<uint64_t *>(moved_back(d_set_offsets, sizeof(uint64_t))),
                reinterpret_cast<uint32_t *>(moved_back(d_set_lengths, sizeof(uint32_t)))};
  L.key = make_key(seed);
  L.first = first;
  L.next = &meta->next;
  L.st = Stats{meta->stats};
  const uint32_t *todo_ids = nullptr;
  uint32_t todo = count;
  for (int attempt = 0; attempt < 16; ++attempt) {
    const uint64_t warps = warps_for(qcap);
    if (warps < 8)
      return fail(RIP_ERR_LIMIT,
                  "rip_sample_static: a set outgrew the queues the static scratch can hold "
                  "for n = %u", n);
    // bitmaps must start all-zero; this region may have held queues before
    if ((bm_bytes && cudaMemsetAsync(work, 0, warps * bm_bytes, s) != cudaSuccess) ||
        cudaMemsetAsync(&meta->fail_count, 0, sizeof(unsigned int), s) != cudaSuccess ||
        cudaMemsetAsync(&meta->next, 0, sizeof(unsigned int), s) != cudaSuccess ||
        cudaMemsetAsync(&meta->first_bad, 0xFF, sizeof(unsigned long long), s) != cudaSuccess)
      return fail(RIP_ERR_CUDA, "cudaMemsetAsync(scratch) failed");
    L.count = todo;
    L.ids = todo_ids;
    L.bitmaps = reinterpret_cast<uint32_t *>(work);
    L.bm_words = bm_words;
    L.queues = reinterpret_cast<uint32_t *>(work + warps * bm_bytes);
    L.qcap = qcap;
    L.F = FailList{ids[attempt & 1], &meta->fail_count, &meta->first_bad};
    L.threads = 256;
    const uint64_t active = todo < warps ? ((uint64_t)todo + 7) & ~7ull : warps;
    L.blocks = (int)(active / 8);
    if (model == RIP_MODEL_IC)
      launch_ic_plain(L, s);
    else
      launch_lt_walk(L, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(RIP_ERR_CUDA, "sampler launch: %s", cudaGetErrorString(e));
    StaticMeta h;
    e = cudaMemcpyAsync(&h, meta, sizeof(StaticMeta), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(RIP_ERR_CUDA, "sampler: %s", cudaGetErrorString(e));
    if (h.fail_count == 0) {
      *num_elements = h.cursor;
      return RIP_OK;
    }
    if (h.first_bad != ~0ull)
      return fail(RIP_ERR_LIMIT,
                  "rip_sample_static: vertex_capacity %llu is too small for these sets",
                  (unsigned long long)vertex_capacity);
    // queue overflow only: widen the queues (fewer warps) and re-run the
    // failed sets; their results do not depend on the retry
    if (qcap == n)
      return fail(RIP_ERR_DEVICE, "rip_sample_static: sets failed with full-size queues");
    qcap = (uint64_t)qcap * 4 < n ? qcap * 4 : n;
    todo = h.fail_count;
    todo_ids = ids[attempt & 1];
  }
  return fail(RIP_ERR_DEVICE, "rip_sample_static: did not converge");
}
