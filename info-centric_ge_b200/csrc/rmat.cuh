// Seeded R-MAT graph generated on the device, for the synthetic stand-ins of
// the reference's datasets at sizes the host generator cannot reach (1.6 B
// undirected edges).  The edge list equals felog_synth_generate's (host,
// felog_tools.cpp) with no held-out split:
//   * candidate i draws, per level l < scale, r = unit01(draw(seed, i, l))
//     and picks the quadrant (a | b | c | d); u >= V, v >= V and u == v are
//     void;
//   * the edges are the first e_target distinct unordered pairs in candidate
//     order, each kept at its first candidate (orientation as drawn);
//   * vertex ids are optionally permuted (the host's Fisher-Yates), untouched
//     vertices dropped and the rest renumbered in increasing order;
//   * weights from draw(seed ^ 0x77, i, .) as on the host.
// The device keeps the candidates as (pair key, index): a stable radix sort
// by key puts each pair's first candidate first, the first candidates of all
// pairs are selected, sorted by index, cut at e_target and expanded again.
#pragma once

#include "common.cuh"

namespace felog {

__host__ __device__ __forceinline__ uint64_t rmat_mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
// value k of the counter-based stream (seed, id); hs = rmat_mix64(seed ^ 0x5DEECE66D)
__host__ __device__ __forceinline__ uint64_t rmat_draw(uint64_t hs, uint64_t id, uint64_t k) {
  return rmat_mix64(hs + rmat_mix64(id * 0xD1B54A32D192ED03ULL + k));
}
__host__ __device__ __forceinline__ double rmat_unit(uint64_t r) {
  return (double)(r >> 11) * (1.0 / 9007199254740992.0);
}

struct RmatArgs {
  uint64_t hs;        // rmat_mix64(seed ^ 0x5DEECE66D)
  uint64_t hw;        // rmat_mix64((seed ^ 0x77) ^ 0x5DEECE66D): weight stream
  int scale;          // levels: smallest s with 2^s >= V
  uint64_t V;
  double ta, tab, tabc;  // a, a + b, a + b + c
  int lognormal;
  double mu, sigma;
};

__device__ __forceinline__ void rmat_pair(const RmatArgs &a, uint64_t id, uint64_t &u, uint64_t &v) {
  u = 0;
  v = 0;
  for (int l = 0; l < a.scale; l++) {
    const double r = rmat_unit(rmat_draw(a.hs, id, (uint64_t)l));
    const uint64_t bu = r < a.tab ? 0 : 1;
    const uint64_t bv = (r < a.ta || (r >= a.tab && r < a.tabc)) ? 0 : 1;
    u = (u << 1) | bu;
    v = (v << 1) | bv;
  }
}

constexpr uint64_t kRmatVoid = ~0ULL;

// candidates i0 .. i0 + n - 1: key = (min << 32) | max, or void
__global__ void k_rmat_candidates(RmatArgs a, uint64_t i0, uint64_t n, uint64_t *__restrict__ key,
                                  uint32_t *__restrict__ idx) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t u, v;
    rmat_pair(a, i0 + i, u, v);
    key[i] = (u >= a.V || v >= a.V || u == v) ? kRmatVoid : ((u < v ? u : v) << 32) | (u < v ? v : u);
    idx[i] = (uint32_t)(i0 + i);
  }
}

// first candidate of each distinct pair in a key-sorted run (stable: index order within a key)
__global__ void k_rmat_first(const uint64_t *__restrict__ key, uint64_t n, uint8_t *__restrict__ flag) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    flag[j] = key[j] != kRmatVoid && (j == 0 || key[j] != key[j - 1]);
}

// touched[perm(u)] = touched[perm(v)] = 1 for the kept candidates
__global__ void k_rmat_touch(RmatArgs a, const uint32_t *__restrict__ idx, uint64_t E,
                             const uint32_t *__restrict__ perm, uint8_t *__restrict__ touched) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t u, v;
    rmat_pair(a, idx[i], u, v);
    if (perm) {
      u = perm[u];
      v = perm[v];
    }
    touched[u] = 1;
    touched[v] = 1;
  }
}

// 12-byte records {newid[perm(u)], newid[perm(v)], weight} in index order
__global__ void k_rmat_records(RmatArgs a, const uint32_t *__restrict__ idx, uint64_t E,
                               const uint32_t *__restrict__ perm, const uint32_t *__restrict__ newid,
                               uint32_t *__restrict__ rec) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = idx[i];
    uint64_t u, v;
    rmat_pair(a, k, u, v);
    if (perm) {
      u = perm[u];
      v = perm[v];
    }
    float w;
    if (a.lognormal) {
      // Box-Muller on two stream values (FP64 device log / cos / exp / sqrt)
      double u1 = rmat_unit(rmat_draw(a.hw, k, 1));
      const double u2 = rmat_unit(rmat_draw(a.hw, k, 2));
      if (u1 < 1e-300) u1 = 1e-300;
      const double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
      w = (float)exp(a.mu + a.sigma * z);
    } else {
      const uint32_t r24 = (uint32_t)(rmat_draw(a.hw, k, 0) >> 40);
      w = (float)(r24 + 1) * (1.0f / 16777216.0f);
    }
    rec[3 * i] = newid[u];
    rec[3 * i + 1] = newid[v];
    rec[3 * i + 2] = __float_as_uint(w);
  }
}

__global__ void k_u8_to_u32(const uint8_t *__restrict__ x, uint64_t n, uint32_t *__restrict__ y) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    y[i] = x[i];
}

__global__ void k_max_u32(const uint32_t *__restrict__ x, uint64_t n, unsigned int *out) {
  unsigned int m = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    m = max(m, x[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

}  // namespace felog
