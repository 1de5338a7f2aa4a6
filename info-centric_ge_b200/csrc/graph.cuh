// Device CSR construction and per-vertex alias tables.
//
// CSR order follows graph.hpp:531-575: the record list is doubled when the
// graph is undirected (record i -> entries 2i = e, 2i+1 = e^T,
// graph.hpp:741-772) and each entry is appended to its source's bucket in
// list order.  That order is what a candidate index draw addresses, so the
// build is a stable sort of entries by source (a stable LSD radix sort).
#pragma once

#include "common.cuh"

namespace felog {

// Expand records to directed entries: key = source, value = entry index.
__global__ void k_expand_edges(const uint32_t *__restrict__ rec /* 3 words per record */, uint64_t n_rec,
                               int undirected, uint32_t v_num, uint32_t *__restrict__ keys,
                               uint32_t *__restrict__ vals, uint32_t *__restrict__ deg, int *err) {
  uint64_t m = undirected ? 2 * n_rec : n_rec;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = undirected ? (i >> 1) : i;
    uint32_t s = rec[3 * r], d = rec[3 * r + 1];
    if (undirected && (i & 1)) {
      uint32_t t = s;
      s = d;
      d = t;
    }
    if (s >= v_num || d >= v_num) {
      set_error(err, kErrBadVertex);
      s = 0;
    }
    keys[i] = s;
    vals[i] = (uint32_t)i;
    atomicAdd(&deg[s], 1u);
  }
}

// Walker entries: wadj[j] = {neighbour, data bits, the neighbour's first CSR
// entry, its degree}.  A walk step reads its candidate's entry and, from the
// same 16 bytes, where the candidate's own list starts and how long it is, so
// a step costs one dependent random read instead of two (adj[b + r], then
// row_ptr[dst], row_ptr[dst + 1]).  Entry indices are below 2^32.
__global__ void k_fuse_adj(const uint64_t *__restrict__ row_ptr, const uint2 *__restrict__ adj, uint64_t m,
                           uint4 *__restrict__ wadj) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 e = adj[j];
    const uint64_t b = row_ptr[e.x];
    wadj[j] = make_uint4(e.x, e.y, (uint32_t)b, (uint32_t)(row_ptr[e.x + 1] - b));
  }
}

// Gather entries into CSR order: adj[j] = {neighbour, data bits}.
__global__ void k_gather_adj(const uint32_t *__restrict__ rec, const uint32_t *__restrict__ order, uint64_t m,
                             int undirected, uint2 *__restrict__ adj) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t i = order[j];
    uint64_t r = undirected ? (i >> 1) : i;
    uint32_t s = rec[3 * r], d = rec[3 * r + 1], w = rec[3 * r + 2];
    uint32_t nb = (undirected && (i & 1)) ? s : d;
    adj[j] = make_uint2(nb, w);
  }
}

// ------------------------------------------------------------- alias
// Vose's alias method per vertex over the entries' data (weights).  One warp
// per vertex for short lists; the warp builds the table sequentially in lane
// 0 for clarity of order (alias tables are built once per graph).  prob[j] is
// the probability of keeping slot j, alias[j] the slot taken otherwise, both
// indexed like adj.  A uniform list gives prob = 1 everywhere.
__global__ void k_build_alias(const uint64_t *__restrict__ row_ptr, const uint2 *__restrict__ adj, uint32_t v_num,
                              float *__restrict__ prob, uint32_t *__restrict__ alias,
                              uint32_t *__restrict__ scratch /* m: small/large worklists */, int *err) {
  int lane = lane_id();
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = warp; v < v_num; v += nwarps) {
    uint64_t b = row_ptr[v], e = row_ptr[v + 1];
    uint32_t n = (uint32_t)(e - b);
    if (n == 0) continue;
    // total weight (FP64, lane-strided then reduced)
    double tot = 0.0;
    for (uint32_t j = lane; j < n; j += 32) {
      float w = __uint_as_float(adj[b + j].y);
      if (!(w >= 0.0f) || isinf(w)) set_error(err, kErrBadWeight);
      tot += (double)w;
    }
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (lane == 0) {
      uint32_t *small = scratch + b;  // grows up from b
      uint32_t ns = 0, nl = 0;        // large list grows down from e-1
      for (uint32_t j = 0; j < n; j++) {
        float w = __uint_as_float(adj[b + j].y);
        double q = tot > 0.0 ? (double)w * n / tot : 1.0;
        prob[b + j] = (float)q;
        if (q < 1.0) small[ns++] = j;
        else scratch[e - 1 - nl++] = j;
      }
      while (ns > 0 && nl > 0) {
        uint32_t s = small[--ns];
        uint32_t l = scratch[e - nl];  // most recently pushed large
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
  }
}

}  // namespace felog
