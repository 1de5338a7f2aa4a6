// Common neighbours per input edge: the reference's offline tool
// (src/tools/gcn.cpp:248-357) on the GPU.
//
// The tool sorts every CSR row by neighbour and, for an edge (s, d), keeps
// the elements of the shorter neighbour list (N(s) on a size tie) that occur
// in the longer one, in order - its galloping search matches a repeated
// short element again against the same long element - then takes the count
// down by one for a leading s or d and, while more than one is left, by one
// for every later element equal to its predecessor or to s or d.  Edges are
// visited in input order and an edge whose (s, d) entry already holds a count
// (set by an earlier copy of the edge or by the mirror (d, s)) keeps it, so
// every edge of an unordered pair reports the count of the pair's first edge
// in its own orientation.
//
// Here: the rows are sorted with one radix sort of (s << 32 | d) keys; every
// edge computes its own orientation's count (a thread per edge with a
// monotone binary search per short element, or a warp per edge when the
// short list is long); a stable sort of the edges by unordered pair and a max
// scan of the group heads then hand every edge its group's first count.
#pragma once

#include <stdint.h>

#include "common.cuh"

namespace felog {

constexpr uint32_t kGcnWarpMin = 17;  // short lists at least this long take the warp path

__global__ void k_gcn_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t n,
                           uint32_t v_num, int undirected, unsigned long long *__restrict__ keys, int *err) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s = src[e], d = dst[e];
    if (s >= v_num || d >= v_num) {  // the host checks ids first; a bad one never indexes a row here
      set_error(err, kErrBadVertex);
      s = d = 0;
    }
    if (undirected) {
      keys[2 * e] = ((unsigned long long)s << 32) | d;
      keys[2 * e + 1] = ((unsigned long long)d << 32) | s;
    } else {
      keys[e] = ((unsigned long long)s << 32) | d;
    }
  }
}

// row_ptr from the sorted keys; nbr = low halves.  row_ptr has v_num + 1 entries.
__global__ void k_gcn_rows(const unsigned long long *__restrict__ keys, uint64_t m, uint32_t v_num,
                           uint64_t *__restrict__ row_ptr, uint32_t *__restrict__ nbr) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += stride) {
    const uint32_t v = (uint32_t)(keys[i] >> 32);
    nbr[i] = (uint32_t)keys[i];
    const long long pv = i ? (long long)(keys[i - 1] >> 32) : -1;
    for (long long u = pv + 1; u <= (long long)v; u++) row_ptr[u] = i;
    if (i == m - 1)
      for (uint64_t u = (uint64_t)v + 1; u <= v_num; u++) row_ptr[u] = m;
  }
  if (m == 0)
    for (uint64_t u = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u <= v_num; u += stride) row_ptr[u] = 0;
}

__device__ __forceinline__ uint64_t gcn_lower(const uint32_t *__restrict__ v, uint64_t lo, uint64_t hi, uint32_t key) {
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (v[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// The tool's count from the matched short elements: total matches, whether the
// first is s or d, and the number of later matches equal to their
// predecessor or to s or d.
__device__ __forceinline__ int32_t gcn_count(uint32_t total, bool first_sd, uint32_t dec) {
  uint32_t c = total;
  if (c > 0) {
    if (first_sd) c--;
    if (c > 1) c -= dec;
  }
  return (int32_t)c;
}

struct GcnLists {
  uint64_t sb, sn;  // short list: start, length
  uint64_t lb, ln;  // long list
};

__device__ __forceinline__ GcnLists gcn_lists(const uint64_t *__restrict__ row_ptr, uint32_t s, uint32_t d) {
  const uint64_t b1 = row_ptr[s], n1 = row_ptr[s + 1] - b1;
  const uint64_t b2 = row_ptr[d], n2 = row_ptr[d + 1] - b2;
  GcnLists g;
  if (n1 > n2) {
    g.lb = b1; g.ln = n1; g.sb = b2; g.sn = n2;
  } else {
    g.lb = b2; g.ln = n2; g.sb = b1; g.sn = n1;
  }
  return g;
}

// Thread per edge; edges with long short lists go to the warp list.
__global__ void k_gcn_edges(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t n,
                            const uint64_t *__restrict__ row_ptr, const uint32_t *__restrict__ nbr,
                            int32_t *__restrict__ cn, uint32_t *__restrict__ heavy,
                            unsigned long long *__restrict__ n_heavy) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[e], d = dst[e];
    const GcnLists g = gcn_lists(row_ptr, s, d);
    if (g.sn >= kGcnWarpMin) {
      heavy[atomicAdd(n_heavy, 1ULL)] = (uint32_t)e;
      continue;
    }
    uint32_t total = 0, dec = 0, prev = 0;
    bool first_sd = false;
    uint64_t lo = g.lb;
    const uint64_t hi = g.lb + g.ln;
    for (uint64_t j = 0; j < g.sn; j++) {
      const uint32_t x = nbr[g.sb + j];
      lo = gcn_lower(nbr, lo, hi, x);
      if (lo < hi && nbr[lo] == x) {
        if (total == 0) first_sd = x == s || x == d;
        else dec += (x == prev || x == s || x == d) ? 1u : 0u;
        prev = x;
        total++;
      }
    }
    cn[e] = gcn_count(total, first_sd, dec);
  }
}

// Warp per listed edge; a match that equals the previous short element or s
// or d is one decrement, except at the first match, where only s or d counts
// (and then separately).  Lists of comparable length (long <= kGcnMergeRatio x
// short) are merged: each lane takes an equal share of the merge steps (its
// start found by a diagonal binary search), and the merge takes the short
// element first on ties, so a short element is matched exactly when the long
// element in front of it is equal, and a repeated short element matches
// again.  Otherwise lanes take short elements j = lane, lane + 32, ... with a
// binary search of the long list each.
constexpr uint64_t kGcnMergeRatio = 4;
__global__ void k_gcn_heavy(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            const uint32_t *__restrict__ heavy, const unsigned long long *__restrict__ n_heavy,
                            const uint64_t *__restrict__ row_ptr, const uint32_t *__restrict__ nbr,
                            int32_t *__restrict__ cn) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t nh = *n_heavy;
  for (uint64_t h = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; h < nh; h += warps) {
    const uint32_t e = heavy[h];
    const uint32_t s = src[e], d = dst[e];
    const GcnLists g = gcn_lists(row_ptr, s, d);
    uint32_t total = 0, flagged = 0;
    uint64_t j0 = ~0ULL;
    if (g.ln <= kGcnMergeRatio * g.sn) {
      const uint32_t *S = nbr + g.sb, *L = nbr + g.lb;
      const uint64_t ns = g.sn, nl = g.ln, seg = (ns + nl + 31) / 32;
      const uint64_t dg = lane * seg < ns + nl ? lane * seg : ns + nl;
      // i = short elements among the first dg merged ones
      uint64_t lo = dg > nl ? dg - nl : 0, hi = dg < ns ? dg : ns;
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (S[mid] <= L[dg - mid - 1]) lo = mid + 1;
        else hi = mid;
      }
      uint64_t i = lo, j = dg - lo;
      uint32_t prev = i > 0 ? S[i - 1] : 0;
      for (uint64_t step = 0; step < seg && (i < ns || j < nl); step++) {
        if (i < ns && (j >= nl || S[i] <= L[j])) {
          const uint32_t x = S[i];
          if (j < nl && L[j] == x) {
            total++;
            if (i < j0) j0 = i;
            flagged += ((i > 0 && prev == x) || x == s || x == d) ? 1u : 0u;
          }
          prev = x;
          i++;
        } else {
          j++;
        }
      }
    } else {
      for (uint64_t j = lane; j < g.sn; j += 32) {
        const uint32_t x = nbr[g.sb + j];
        const uint64_t p = gcn_lower(nbr, g.lb, g.lb + g.ln, x);
        if (p < g.lb + g.ln && nbr[p] == x) {
          total++;
          if (j < j0) j0 = j;
          const bool dup = j > 0 && nbr[g.sb + j - 1] == x;
          flagged += (dup || x == s || x == d) ? 1u : 0u;
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      total += __shfl_xor_sync(0xffffffffu, total, o);
      flagged += __shfl_xor_sync(0xffffffffu, flagged, o);
      const uint64_t oj = __shfl_xor_sync(0xffffffffu, j0, o);
      j0 = oj < j0 ? oj : j0;
    }
    if (lane == 0) {
      bool first_sd = false;
      if (total) {
        const uint32_t x0 = nbr[g.sb + j0];
        first_sd = x0 == s || x0 == d;
      }
      cn[e] = gcn_count(total, first_sd, flagged - (first_sd ? 1u : 0u));
    }
  }
}

// Unordered-pair keys, values = edge index (stable sort keeps input order).
__global__ void k_gcn_pair_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst, uint64_t n,
                                unsigned long long *__restrict__ keys, uint32_t *__restrict__ idx) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = src[e], b = dst[e];
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    keys[e] = ((unsigned long long)lo << 32) | hi;
    idx[e] = (uint32_t)e;
  }
}

__global__ void k_gcn_heads(const unsigned long long *__restrict__ keys, uint64_t n, uint64_t *__restrict__ head) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? i : 0;
}

__global__ void k_gcn_scatter(const uint32_t *__restrict__ idx, const uint64_t *__restrict__ head, uint64_t n,
                              const int32_t *__restrict__ cn_own, int32_t *__restrict__ cn) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    cn[idx[i]] = cn_own[idx[head[i]]];
}

struct GcnMax {
  __device__ __forceinline__ uint64_t operator()(uint64_t a, uint64_t b) const { return a > b ? a : b; }
};

}  // namespace felog
