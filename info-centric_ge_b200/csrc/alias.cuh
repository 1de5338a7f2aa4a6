// Vose's alias method for one vertex's adjacency list, run by one warp.
//
// prob[j] is the probability of keeping slot j, alias[j] the slot taken
// otherwise, both indexed like the CSR entries b..e-1.  The warp sums the
// weights in FP64; lane 0 then builds the table in order (tables are built
// once per graph).  The small and large worklists live in scratch[b..e):
// small grows up from b, large grows down from e-1 (an index is in at most
// one list, so they never meet).  A uniform list gives prob = 1 everywhere.
#pragma once

#include "common.cuh"

namespace felog {

template <class WeightAt>
__device__ __forceinline__ void alias_build_vertex(uint64_t b, uint64_t e, WeightAt weight, float *prob,
                                                   uint32_t *alias, uint32_t *scratch, int *err) {
  const int lane = lane_id();
  const uint32_t n = (uint32_t)(e - b);
  if (n == 0) return;
  double tot = 0.0;
  for (uint32_t j = lane; j < n; j += 32) {
    float w = weight(b + j);
    if (!(w >= 0.0f) || isinf(w)) set_error(err, kErrBadWeight);
    tot += (double)w;
  }
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
  if (lane == 0) {
    uint32_t *small = scratch + b;
    uint32_t ns = 0, nl = 0;
    for (uint32_t j = 0; j < n; j++) {
      float w = weight(b + j);
      double q = tot > 0.0 ? (double)w * n / tot : 1.0;
      prob[b + j] = (float)q;
      if (q < 1.0) small[ns++] = j;
      else scratch[e - 1 - nl++] = j;
    }
    while (ns > 0 && nl > 0) {
      uint32_t s = small[--ns];
      uint32_t l = scratch[e - nl];
      nl--;
      alias[b + s] = l;
      float pl = prob[b + l] - (1.0f - prob[b + s]);
      prob[b + l] = pl;
      if (pl < 1.0f) small[ns++] = l;
      else scratch[e - 1 - nl++] = l;
    }
    while (nl > 0) {
      uint32_t l = scratch[e - nl];
      nl--;
      prob[b + l] = 1.0f;
      alias[b + l] = l;
    }
    while (ns > 0) {
      uint32_t s = small[--ns];
      prob[b + s] = 1.0f;
      alias[b + s] = s;
    }
  }
  __syncwarp();
}

}  // namespace felog
