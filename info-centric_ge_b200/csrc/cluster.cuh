// Spherical K-means over the resident syn0 rows (the -classes output; the
// reference's interface is word2vec.cu:2128-2175: one class id per vocabulary
// row, written as "<vertex> <class>").
//
// Objective: maximise sum_v x_v . c_{label(v)} over unit centroids c.  Each
// iteration is one assignment pass (every row takes the centroid with the
// largest dot product, ties to the lower index) and one update pass (every
// centroid becomes the normalised sum of its rows; a centroid without rows
// keeps its direction).  Both passes can only raise the objective, so it is
// non-decreasing over iterations and a pass without label changes is a fixed
// point.  Initial centroids are the normalised rows at evenly spaced
// vocabulary positions (rows are in degree-descending order, so the seeds
// span the degree range).
//
// Layout: centroids live in the rows' interleaved order (physical lane * J + j
// holds logical lane + 32 j), so dot products never un-permute a row.  The
// update is deterministic: rows are sorted by label (stable radix sort), one
// block sums each centroid's rows in FP64 in row order, warps combined in a
// fixed order.
#pragma once

#include "common.cuh"
#include "sgns.cuh"

namespace felog {

struct KmArgs {
  SgArgs rows;          // syn0 rows (FP32, or BF16 with FP32 master rows)
  uint64_t n_rows;      // vocabulary rows
  int k;                // centroids
  float *cent;          // k x DIM, interleaved, unit length (or zero)
  int32_t *labels;      // per row
  double *obj_partial;  // per block: sum of the best dot products of its rows
  unsigned long long *changed;  // rows whose label changed in this pass
  int first;            // first pass: every row counts as changed
};

template <int DIM>
__device__ __forceinline__ float km_lane_dot(const float (&x)[DIM / 32], const float *__restrict__ c) {
  constexpr int J = DIM / 32;
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < J; j++) s = __fmaf_rn(x[j], __ldg(&c[j]), s);
  return s;
}

// Assignment: one warp per row.  Centroids are scored eight at a time; the
// eight lane partials go through a transposing butterfly (xor 16, 8, 4 keep
// half, a quarter, an eighth of the candidates; xor 2 and 1 finish the sums),
// after which lane l holds the full dot of candidate ((l >> 2) & 7) in a
// fixed bit order.  Each lane keeps its own best; one warp argmax at the end.
template <int DIM, class P>
__global__ void __launch_bounds__(256) k_km_assign(KmArgs a) {
  constexpr int J = DIM / 32;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  const int mine = ((lane >> 4) & 1) | (((lane >> 3) & 1) << 1) | (((lane >> 2) & 1) << 2);
  double obj = 0.0;
  unsigned long long changed = 0;
  for (uint64_t r = warp; r < a.n_rows; r += nwarps) {
    float x[J];
    row_load<DIM, P>(a.rows, 0, (long long)r, x);
    float best = -INFINITY;
    int bi = 0x7FFFFFFF;
    for (int c0 = 0; c0 < a.k; c0 += 8) {
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; q++)
        v[q] = c0 + q < a.k ? km_lane_dot<DIM>(x, a.cent + (size_t)(c0 + q) * DIM + lane * J) : 0.0f;
      // level 16: lanes with bit 4 keep odd candidates, the others even ones
      const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
      float w[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        const float keep = b4 ? v[2 * t + 1] : v[2 * t], send = b4 ? v[2 * t] : v[2 * t + 1];
        w[t] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
      }
      float u[2];
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const float keep = b3 ? w[2 * t + 1] : w[2 * t], send = b3 ? w[2 * t] : w[2 * t + 1];
        u[t] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
      }
      float z = (b2 ? u[1] : u[0]) + __shfl_xor_sync(0xffffffffu, b2 ? u[0] : u[1], 4);
      z += __shfl_xor_sync(0xffffffffu, z, 2);
      z += __shfl_xor_sync(0xffffffffu, z, 1);
      // candidate index held by this lane: bit 0 from b4, bit 1 from b3, bit 2 from b2
      const int ci = c0 + mine;
      if (ci < a.k && (z > best || (z == best && ci < bi))) {
        best = z;
        bi = ci;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) {
      changed += (a.first || a.labels[r] != bi) ? 1 : 0;
      a.labels[r] = bi;
      obj += (double)best;
    }
  }
  // block sum of the objective in warp order (deterministic)
  __shared__ double s_obj[32];
  __shared__ unsigned long long s_ch[32];
  const int wib = threadIdx.x >> 5;
  if (lane == 0) {
    s_obj[wib] = obj;
    s_ch[wib] = changed;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    unsigned long long ch = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
      t += s_obj[i];
      ch += s_ch[i];
    }
    a.obj_partial[blockIdx.x] = t;
    if (ch) atomicAdd(a.changed, ch);
  }
}

// Rows sorted by label: seg[c] .. seg[c + 1] are centroid c's rows (ascending
// row index).  One block per centroid sums them in FP64: warp w takes rows
// w, w + 8, ... of the segment, the warps' sums are added in warp order, and
// the centroid becomes the sum divided by its norm.  An empty centroid (or a
// zero sum) keeps its previous value.
template <int DIM, class P>
__global__ void __launch_bounds__(256) k_km_update(KmArgs a, const uint32_t *__restrict__ sorted_rows,
                                                   const uint64_t *__restrict__ seg) {
  constexpr int J = DIM / 32;
  constexpr int kWarps = 8;
  __shared__ double s_sum[kWarps][DIM];
  __shared__ double s_norm;
  const int lane = lane_id(), w = threadIdx.x >> 5;
  for (int c = blockIdx.x; c < a.k; c += gridDim.x) {
    const uint64_t b = seg[c], e = seg[c + 1];
    double acc[J];
#pragma unroll
    for (int j = 0; j < J; j++) acc[j] = 0.0;
    for (uint64_t i = b + w; i < e; i += kWarps) {
      float x[J];
      row_load<DIM, P>(a.rows, 0, (long long)sorted_rows[i], x);
#pragma unroll
      for (int j = 0; j < J; j++) acc[j] += (double)x[j];
    }
#pragma unroll
    for (int j = 0; j < J; j++) s_sum[w][lane * J + j] = acc[j];
    __syncthreads();
    if (w == 0) {
      double sq = 0.0;
      for (int i = lane; i < DIM; i += 32) {
        double t = 0.0;
        for (int ww = 0; ww < kWarps; ww++) t += s_sum[ww][i];
        s_sum[0][i] = t;
        sq += t * t;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
      if (lane == 0) s_norm = sqrt(sq);
    }
    __syncthreads();
    const double nrm = s_norm;
    if (e > b && nrm > 0.0)
      for (int i = threadIdx.x; i < DIM; i += blockDim.x) a.cent[(size_t)c * DIM + i] = (float)(s_sum[0][i] / nrm);
    __syncthreads();
  }
}

// Seeds: centroid c is the normalised row floor((c + 0.5) n_rows / k).
template <int DIM, class P>
__global__ void __launch_bounds__(32) k_km_seed(KmArgs a) {
  constexpr int J = DIM / 32;
  const int lane = lane_id();
  for (int c = blockIdx.x; c < a.k; c += gridDim.x) {
    const uint64_t r = (uint64_t)(((double)c + 0.5) * (double)a.n_rows / (double)a.k);
    float x[J];
    row_load<DIM, P>(a.rows, 0, (long long)(r < a.n_rows ? r : a.n_rows - 1), x);
    double sq = 0.0;
#pragma unroll
    for (int j = 0; j < J; j++) sq += (double)x[j] * x[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    const double nrm = sqrt(sq);
#pragma unroll
    for (int j = 0; j < J; j++) a.cent[(size_t)c * DIM + lane * J + j] = nrm > 0.0 ? (float)(x[j] / nrm) : 0.0f;
  }
}

__global__ void k_km_count(const int32_t *__restrict__ labels, uint64_t n, uint32_t *__restrict__ keys,
                           uint32_t *__restrict__ vals, unsigned long long *__restrict__ count) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t l = (uint32_t)labels[i];
    keys[i] = l;
    vals[i] = (uint32_t)i;
    atomicAdd(&count[l], 1ULL);
  }
}

}  // namespace felog
