// felog_build_alias_noalloc: the alias-table builder for callers that cannot
// allocate device memory.
//
// Some callers can't call cudaMalloc: a host application whose device memory
// is owned by its own pooling allocator (or by another runtime), a process
// that must not grow its device footprint after start-up, or code running
// where the CUDA allocator is off limits.  They already hold the graph and the
// output tables in device memory; this entry point needs no more than that.
// Its only working memory, the Vose small/large worklists of felog_build_alias,
// lives in the file-scope device array below, sized for at most
// kNoAllocMaxEntries CSR entries (16 MiB of worklist words).  Every GPU that
// loads this library holds that array until the process exits.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress and caches it; make that
// first call before any stream capture.  All calls share the one array and it
// keeps the last call's contents; calls that overlap on the GPU (on different
// streams, or from different threads) race on it, so callers serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "alias.cuh"
#include "felog_gpu.h"

namespace {

using namespace felog;

// Words 0..63: header (word 0 = device error code, cleared by every call);
// words 64.. : worklists indexed like the CSR entries.
constexpr uint64_t kHeaderWords = 64;
constexpr uint64_t kNoAllocMaxEntries = FELOG_NOALLOC_MAX_ENTRIES;
static __device__ __align__(256) uint32_t g_alias_scratch[kHeaderWords + kNoAllocMaxEntries];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
uint32_t *g_scratch_ptr[kMaxDevices] = {nullptr};

__global__ void k_build_alias_weights(const uint64_t *__restrict__ row_ptr, const float *__restrict__ weight_of,
                                      uint32_t v_num, float *__restrict__ prob, uint32_t *__restrict__ alias,
                                      uint32_t *__restrict__ scratch) {
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  int *err = reinterpret_cast<int *>(scratch);
  uint32_t *work = scratch + kHeaderWords;
  auto weight = [weight_of](uint64_t j) { return weight_of[j]; };
  for (uint32_t v = warp; v < v_num; v += nwarps)
    alias_build_vertex(row_ptr[v], row_ptr[v + 1], weight, prob, alias, work, err);
}

}  // namespace

extern "C" felog_status felog_build_alias_noalloc(const uint64_t *d_row_ptr, const float *d_weight,
                                                 uint32_t v_num, uint64_t e_num, float *d_prob,
                                                 uint32_t *d_alias, void *stream) {
  // status codes: FELOG_INVALID_ARG for a null buffer, more than
  // FELOG_NOALLOC_MAX_ENTRIES entries (rejected before any device work) or a
  // negative / non-finite weight; FELOG_CUDA_ERROR for a failed CUDA call.
  if (!d_row_ptr || (e_num && (!d_weight || !d_prob || !d_alias))) return FELOG_INVALID_ARG;
  if (e_num > kNoAllocMaxEntries) return FELOG_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FELOG_CUDA_ERROR;
  uint32_t *scratch;
  {
    std::lock_guard<std::mutex> g(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
      // a host-side use of g_alias_scratch names a host shadow, not device memory
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, g_alias_scratch) != cudaSuccess) return FELOG_CUDA_ERROR;
      g_scratch_ptr[dev] = static_cast<uint32_t *>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  if (v_num == 0 || e_num == 0) return FELOG_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(scratch, 0, sizeof(uint32_t), st) != cudaSuccess) return FELOG_CUDA_ERROR;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint64_t want = ((uint64_t)v_num * 32 + 255) / 256;
  int blocks = (int)(want < (uint64_t)sms * 8 ? (want ? want : 1) : (uint64_t)sms * 8);
  k_build_alias_weights<<<blocks, 256, 0, st>>>(d_row_ptr, d_weight, v_num, d_prob, d_alias, scratch);
  if (cudaGetLastError() != cudaSuccess) return FELOG_CUDA_ERROR;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, scratch, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return FELOG_CUDA_ERROR;
  if (h == kErrBadWeight) return FELOG_INVALID_ARG;
  return h == 0 ? FELOG_OK : FELOG_INTERNAL;
}
