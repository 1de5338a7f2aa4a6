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
// Set-up: every call looks up the array's device address on the current
// device with cudaGetSymbolAddress (nothing is cached, so a call after a
// device reset sees the reloaded module).  With CUDA's lazy module loading
// the array is mapped on a device by the first call there, not when the
// library is loaded: make one call at start-up, before the caller's own pool
// reserves the free memory, and before any stream capture.  A first call that
// finds no room for the array returns FELOG_OOM.  All calls share the one
// array and it keeps the last call's contents; calls that overlap on the GPU
// (on different streams, or from different threads) race on it, so callers
// serialise them.
//
// The kernel checks every vertex's CSR range against e_num before touching
// the worklists, so a row_ptr that is out of order or points past e_num is
// reported as FELOG_INVALID_ARG and never indexes past the array.
#include <cuda_runtime.h>

#include "alias.cuh"
#include "felog_gpu.h"

namespace {

using namespace felog;

// Words 0..63: header (word 0 = device error code, cleared by every call);
// words 64.. : worklists indexed like the CSR entries.
constexpr uint64_t kHeaderWords = 64;
constexpr uint64_t kNoAllocMaxEntries = FELOG_NOALLOC_MAX_ENTRIES;
static __device__ __align__(256) uint32_t g_alias_scratch[kHeaderWords + kNoAllocMaxEntries];

// device error code of a CSR range outside [0, e_num] or out of order
constexpr int kErrBadRowPtr = 64;

__global__ void k_build_alias_weights(const uint64_t *__restrict__ row_ptr, const float *__restrict__ weight_of,
                                      uint32_t v_num, uint64_t e_num, float *__restrict__ prob,
                                      uint32_t *__restrict__ alias, uint32_t *__restrict__ scratch) {
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  int *err = reinterpret_cast<int *>(scratch);
  uint32_t *work = scratch + kHeaderWords;
  auto weight = [weight_of](uint64_t j) { return weight_of[j]; };
  for (uint32_t v = warp; v < v_num; v += nwarps) {
    const uint64_t b = row_ptr[v], e = row_ptr[v + 1];
    if (e < b || e > e_num || e - b > 0xFFFFFFFFull) {
      if (lane_id() == 0) set_error(err, kErrBadRowPtr);
      continue;  // uniform across the warp: b and e are the same in every lane
    }
    alias_build_vertex(b, e, weight, prob, alias, work, err);
  }
}

}  // namespace

extern "C" felog_status felog_build_alias_noalloc(const uint64_t *d_row_ptr, const float *d_weight,
                                                 uint32_t v_num, uint64_t e_num, float *d_prob,
                                                 uint32_t *d_alias, void *stream) {
  // status codes: FELOG_INVALID_ARG for a null buffer, more than
  // FELOG_NOALLOC_MAX_ENTRIES entries (rejected before any device work), edges
  // without vertices, a CSR range outside [0, e_num] or a negative /
  // non-finite weight; FELOG_OOM when the array cannot be mapped on this
  // device; FELOG_CUDA_ERROR for a failed CUDA call.
  if (!d_row_ptr || (e_num && (!d_weight || !d_prob || !d_alias))) return FELOG_INVALID_ARG;
  if (e_num > kNoAllocMaxEntries) return FELOG_INVALID_ARG;
  if (v_num == 0) return e_num ? FELOG_INVALID_ARG : FELOG_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FELOG_CUDA_ERROR;
  // host code must not hand g_alias_scratch itself to a kernel: on the host
  // that name is a shadow variable, not device memory
  void *p = nullptr;
  const cudaError_t ge = cudaGetSymbolAddress(&p, g_alias_scratch);
  if (ge != cudaSuccess) {
    cudaGetLastError();
    return ge == cudaErrorMemoryAllocation ? FELOG_OOM : FELOG_CUDA_ERROR;
  }
  uint32_t *scratch = static_cast<uint32_t *>(p);
  if (e_num == 0) return FELOG_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(scratch, 0, sizeof(uint32_t), st) != cudaSuccess) return FELOG_CUDA_ERROR;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint64_t want = ((uint64_t)v_num * 32 + 255) / 256;
  int blocks = (int)(want < (uint64_t)sms * 8 ? (want ? want : 1) : (uint64_t)sms * 8);
  k_build_alias_weights<<<blocks, 256, 0, st>>>(d_row_ptr, d_weight, v_num, e_num, d_prob, d_alias, scratch);
  if (cudaGetLastError() != cudaSuccess) return FELOG_CUDA_ERROR;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, scratch, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return FELOG_CUDA_ERROR;
  if (h == kErrBadWeight || h == kErrBadRowPtr) return FELOG_INVALID_ARG;
  return h == 0 ? FELOG_OK : FELOG_INTERNAL;
}
