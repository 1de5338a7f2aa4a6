// Walk-budget kernels: the per-vertex convergence check that stops a
// vertex's walkers, and the round relative entropy.
//
// Convergence restates word2vec.cu:2016-2080 with the pair kernel
// batch_similarity_direct_index_optimized_kernel (word2vec.cu:1448-1506)
// fused in: one warp per unconverged vertex gathers at most 30 neighbours
// (all of them in CSR order when the degree is <= 30, else the first 30 of a
// random permutation), computes each cosine in the reference's reduction
// order (products, then pairwise halving over a 128- or 256-thread tree),
// averages them in FP32 in neighbour order and sets the stop flag when the
// mean exceeds 0.65.  No host round trip: flags stay on the device.
// Vertices outside the vocabulary (possible with -min-count > 0, where the
// reference indexes past its id2offset table) are skipped, and such
// neighbours are left out of the mean.
#pragma once

#include "common.cuh"
#include "sgns.cuh"

namespace felog {

struct ConvArgs {
  SgArgs rows;  // syn0 rows (FP32 and, in BF16 mode, BF16 parts), interleaved
  const uint32_t *id2offset;
  const uint64_t *row_ptr;
  const uint2 *adj;
  uint32_t v_num;
  uint8_t *stop;
  float *sim;
  uint64_t seed;
  uint32_t round;
  unsigned long long *counters;  // [evaluated, unconverged, stopped_total, predicted, audited, overruled,
                                 //  audited_unconverged, evaluated_unconverged]
  uint8_t *stop_round;           // round whose check stopped v (label recording)
  // learned budget (pred_count == nullptr: plain criterion for every vertex)
  const uint8_t *pred_count;
  const float *pred_conf;
  float conf_min;
  uint32_t audit_threshold;      // audited when hash(seed, round, v) < this
};

// audit draw of vertex v in round r (uniform 32 bits)
__device__ __forceinline__ uint32_t audit_hash(uint64_t seed, uint32_t round, uint32_t v) {
  const uint4 o = philox4x32_10(make_uint4(v, round, 0x41554454u, 0u),
                                make_uint2((uint32_t)seed ^ 0x9E3779B9u, (uint32_t)(seed >> 32)));
  return o.x;
}

// First 30 positions of a partial Fisher-Yates shuffle of 0..deg-1 driven by
// Philox (v, round, i); the same sequence as the oracle's orc_eval_choose.
__device__ void eval_choose(uint64_t seed, uint32_t round, uint32_t v, uint32_t deg, uint32_t *chosen) {
  uint32_t pos[30], val[30];
  int nsw = 0;
  for (uint32_t i = 0; i < 30; i++) {
    uint4 o = philox4x32_10(make_uint4(v, round, i, 0x45564C31u),
                            make_uint2((uint32_t)seed ^ 0x2545F491u, (uint32_t)(seed >> 32)));
    uint32_t j = i + mulhi64_u32(((uint64_t)o.y << 32) | o.x, deg - i);
    uint32_t vi = i, vj = j;
    int hi = -1, hj = -1;
    for (int k = 0; k < nsw; k++) {
      if (pos[k] == i) hi = k;
      if (pos[k] == j) hj = k;
    }
    if (hi >= 0) vi = val[hi];
    if (hj >= 0) vj = val[hj];
    chosen[i] = vj;
    if (hj >= 0) val[hj] = vi;
    else {
      pos[nsw] = j;
      val[nsw] = vi;
      nsw++;
    }
  }
}

template <int J>
__device__ __forceinline__ float tree_sum(float (&p)[J]) {
#pragma unroll
  for (int h = J / 2; h >= 1; h >>= 1)
#pragma unroll
    for (int j = 0; j < h; j++) p[j] = __fadd_rn(p[j], p[j + h]);
  float r = p[0];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r = __fadd_rn(r, __shfl_xor_sync(0xffffffffu, r, o));
  return r;
}

template <int DIM, class P>
__global__ void __launch_bounds__(256) k_converge(ConvArgs a) {
  constexpr int J = DIM / 32;
  __shared__ uint32_t s_choice[8][30];
  const int lane = lane_id();
  const int wib = threadIdx.x >> 5;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long evaluated = 0, unconv = 0, predicted = 0, audited = 0, overruled = 0, aud_unconv = 0,
                     eval_unconv = 0;
  for (uint32_t v = warp; v < a.v_num; v += nwarps) {
    // vertices outside the vocabulary (-min-count) have no row: not evaluated
    if (a.stop[v] || a.id2offset[v] == 0xFFFFFFFFu) continue;
    // learned budget: a confident prediction decides unless v is audited
    bool confident = false, learned_stop = false, audit = false;
    if (a.pred_count) {
      confident = a.pred_conf[v] >= a.conf_min;
      learned_stop = a.round + 1 >= (uint32_t)a.pred_count[v];
      audit = confident && audit_hash(a.seed, a.round, v) < a.audit_threshold;
      if (confident && !audit) {
        if (lane == 0) {
          predicted++;
          if (learned_stop) {
            a.stop[v] = 1;
            if (a.stop_round) a.stop_round[v] = (uint8_t)min(a.round, 254u);
          } else {
            unconv++;
          }
        }
        continue;
      }
    }
    evaluated++;
    const uint64_t b = a.row_ptr[v];
    const uint32_t deg = (uint32_t)(a.row_ptr[v + 1] - b);
    const int n = deg > 30 ? 30 : (int)deg;
    if (deg > 30) {
      if (lane == 0) eval_choose(a.seed, a.round, v, deg, s_choice[wib]);
      __syncwarp();
    }
    float x[J];
    row_load<DIM, P>(a.rows, 0, a.id2offset[v], x);
    float px[J];
#pragma unroll
    for (int j = 0; j < J; j++) px[j] = __fmul_rn(x[j], x[j]);
    const float nx = __fsqrt_rn(tree_sum<J>(px));
    float sum = 0.0f;
    int used = 0;
    for (int i = 0; i < n; i++) {
      const uint32_t idx = deg > 30 ? s_choice[wib][i] : (uint32_t)i;
      const uint32_t u = a.adj[b + idx].x;
      if (a.id2offset[u] == 0xFFFFFFFFu) continue;  // neighbour without a row
      used++;
      float y[J];
      row_load<DIM, P>(a.rows, 0, a.id2offset[u], y);
      float pd[J], py[J];
#pragma unroll
      for (int j = 0; j < J; j++) {
        pd[j] = __fmul_rn(x[j], y[j]);
        py[j] = __fmul_rn(y[j], y[j]);
      }
      const float dot = tree_sum<J>(pd);
      const float ny = __fsqrt_rn(tree_sum<J>(py));
      const float cs = (nx == 0.0f || ny == 0.0f) ? 0.0f : __fdiv_rn(dot, __fmul_rn(nx, ny));
      sum = __fadd_rn(sum, cs);
    }
    __syncwarp();
    const float s = used > 0 ? __fdiv_rn(sum, (float)used) : 0.0f;
    if (lane == 0) {
      a.sim[v] = s;
      const bool plain_stop = (double)s > 0.65;
      if (plain_stop) {
        a.stop[v] = 1;
        if (a.stop_round) a.stop_round[v] = (uint8_t)min(a.round, 254u);
      } else {
        unconv++;
        eval_unconv++;
      }
      if (audit) {
        audited++;
        overruled += plain_stop != learned_stop;
        aud_unconv += !plain_stop;
      }
    }
  }
  if (lane == 0) {
    if (evaluated) atomicAdd(&a.counters[0], evaluated);
    if (unconv) atomicAdd(&a.counters[1], unconv);
    if (predicted) atomicAdd(&a.counters[3], predicted);
    if (audited) atomicAdd(&a.counters[4], audited);
    if (overruled) atomicAdd(&a.counters[5], overruled);
    if (aud_unconv) atomicAdd(&a.counters[6], aud_unconv);
    if (eval_unconv) atomicAdd(&a.counters[7], eval_unconv);
  }
}

__global__ void k_count_stopped(const uint8_t *stop, uint32_t v_num, unsigned long long *out) {
  unsigned long long c = 0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < v_num; v += gridDim.x * blockDim.x) c += stop[v] != 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// Round relative entropy KL(p || q), p_v = deg_v / sum deg, q_v = freq_v / sum
// freq (walk.hpp:767-787), FP64, deterministic two-pass reduction.
__global__ void __launch_bounds__(256) k_kl_partial(const uint32_t *deg, const unsigned int *freq, uint32_t v_num,
                                                    double deg_sum, double words_sum, double *partial) {
  __shared__ double sh[256];
  double h = 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < v_num; v += gridDim.x * blockDim.x) {
    double pi = (double)deg[v] / deg_sum;
    double qi = (double)freq[v] / words_sum;
    h += pi * (log(pi) - log(qi));
  }
  sh[threadIdx.x] = h;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_kl_final(const double *partial, int n, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double h = 0.0;
    for (int i = 0; i < n; i++) h += partial[i];
    *out = h;
  }
}

}  // namespace felog
