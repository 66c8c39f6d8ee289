// api.cu -- host runtime behind include/ripples_b200.h: the context (one
// device, one stream, a device-memory budget with a block cache).  The other
// parts of the C ABI live beside it:
//   graph.cu   device graphs (upload, packing, device-built R-MAT / ER)
//   pool.cu    RRR pools and every sampler path, many pools in one launch,
//              the sampler autotuner
//   select.cu  seed selection under both reference tie-breaks
//   imm.cu     theta math and the IMM driver
//   server.cu  batched IMM queries and the request loop
#include "host.h"

extern "C" {

const char *rip_version(void) { return "ripples_b200 0.1.0 sm_100a"; }

int rip_ctx_create(int device, size_t hbm_budget, rip_ctx **out) {
  if (!out) return RIP_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RIP_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return RIP_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return RIP_ERR_CUDA;
  rip_ctx *c = new rip_ctx();
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    delete c;
    return RIP_ERR_CUDA;
  }
  c->num_sms = prop.multiProcessorCount;
  if (prop.major < 10) {
    delete c;
    return RIP_ERR_CUDA;  // built for sm_100a only
  }
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  c->budget = hbm_budget ? hbm_budget : (size_t)(0.9 * (double)fr);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess ||
      cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return RIP_ERR_CUDA;
  }
  *out = c;
  return RIP_OK;
}

int rip_ctx_destroy(rip_ctx *c) {
  if (!c) return RIP_ERR_INVALID;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  while (!c->servers.empty()) rip_server_destroy(c->servers.back());
  while (!c->pools.empty()) rip_pool_destroy(c->pools.back());
  while (!c->graphs.empty()) rip_graph_destroy(c->graphs.back());
  cache_release_all(c);
  dfree(c, c->m_scratch);
  dfree(c, c->m_table);
  dfree(c, c->m_fail);
  if (c->heap_registered) cudaHostUnregister(c->heap_registered);
  delete c->h_cand;
  delete c->h_count;
  delete c->h_meta;
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return RIP_OK;
}

const char *rip_last_error(const rip_ctx *c) {
  return c ? c->err.c_str() : "null context";
}

int rip_sync(rip_ctx *c) {
  if (!c) return RIP_ERR_INVALID;
  CK(c, cudaStreamSynchronize(c->stream));
  return RIP_OK;
}

int rip_ctx_stream(rip_ctx *c, void **stream) {
  if (!c || !stream) return RIP_ERR_INVALID;
  *stream = (void *)c->stream;
  return RIP_OK;
}

uint64_t rip_kernel_launches(void) { return rip::launch_counter(); }

int rip_ctx_memory(rip_ctx *c, size_t *used, size_t *budget) {
  if (!c) return RIP_ERR_INVALID;
  if (used) *used = c->used;
  if (budget) *budget = c->budget;
  return RIP_OK;
}

}  // extern "C"
