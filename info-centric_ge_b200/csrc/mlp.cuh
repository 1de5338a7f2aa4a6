// Learned walk budget: per-vertex features, a 6 -> 64 -> 64 -> (9 + 1) MLP
// (ReLU hidden layers; 9 logits for the walk count 2..10, one regression
// output for the walk length 20..80) with hand-written forward, backward and
// Adam kernels, and batched inference.  No reference counterpart: the plain
// information-centric criterion (convergence check, word2vec.cu:2016-2080,
// and the correlation stop, walk.hpp:945-951) produces the training labels,
// stays the fallback for low-confidence vertices and audits a random sample.
//
// Parameter vector (FP32, kMlpParams):
//   W1[64][6] b1[64] W2[64][64] b2[64] W3[10][64] b3[10]
// Loss of one sample: softmax cross-entropy of the 9 count logits against
// the label (walk count - 2) plus (out[9] - (length - 50) / 30)^2 / 2.
#pragma once

#include "common.cuh"

namespace felog {

constexpr int kMlpIn = 6, kMlpH = 64, kMlpC = 9, kMlpOut = kMlpC + 1;
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpH * kMlpIn, kMlpW2 = kMlpB1 + kMlpH, kMlpB2 = kMlpW2 + kMlpH * kMlpH,
              kMlpW3 = kMlpB2 + kMlpH, kMlpB3 = kMlpW3 + kMlpOut * kMlpH, kMlpParams = kMlpB3 + kMlpOut;
constexpr int kMlpBatch = 256;                 // samples per block in the gradient kernel
constexpr int kMlpPad = kMlpH + 1;             // shared-memory row stride (no bank conflicts)
constexpr float kLenMid = 50.0f, kLenScale = 30.0f;

// --------------------------------------------------------------- features
// Per vertex v (row_ptr / adj in CSR; data = edge weight bits):
//   f0 = log1p(deg)             f1 = log1p(sum of weights)
//   f2 = entropy of w / sum w   (the transition distribution the alias
//                                table encodes; 0 for degree <= 1)
//   f3 = log1p(sum of the neighbours' degrees)
//   f4 = log1p(visits in the walks so far)
//   f5 = log1p(length of v's walk in the first round)
// One warp per vertex; sums in FP64 over the adjacency in CSR order, lane
// partials combined by a fixed xor tree.
__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__global__ void __launch_bounds__(256) k_budget_features(const uint64_t *row_ptr, const uint2 *adj, uint32_t v_num,
                                                         const unsigned int *visits, const uint32_t *first_len,
                                                         float *feat) {
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  for (uint64_t v = warp; v < v_num; v += nw) {
    const uint64_t b = row_ptr[v], e = row_ptr[v + 1];
    double ws = 0.0, hop2 = 0.0;
    for (uint64_t i = b + lane; i < e; i += 32) {
      const uint2 u = adj[i];
      ws += (double)__uint_as_float(u.y);
      hop2 += (double)(row_ptr[u.x + 1] - row_ptr[u.x]);
    }
    ws = warp_sum_d(ws);
    hop2 = warp_sum_d(hop2);
    double h = 0.0;
    if (ws > 0.0) {
      for (uint64_t i = b + lane; i < e; i += 32) {
        const double p = (double)__uint_as_float(adj[i].y) / ws;
        if (p > 0.0) h -= p * log(p);
      }
    }
    h = warp_sum_d(h);
    if (lane == 0) {
      float *f = feat + v * kMlpIn;
      f[0] = (float)log1p((double)(e - b));
      f[1] = (float)log1p(ws);
      f[2] = (float)h;
      f[3] = (float)log1p(hop2);
      f[4] = (float)log1p((double)visits[v]);
      f[5] = (float)log1p((double)first_len[v]);
    }
  }
}

// standardize features in place with the model's (mean, inv_std)
__global__ void k_budget_standardize(float *feat, uint64_t n, const float *mean, const float *inv_std) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n * kMlpIn;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % kMlpIn);
    feat[i] = __fmul_rn(__fsub_rn(feat[i], mean[k]), inv_std[k]);
  }
}

// ---------------------------------------------------------------- forward
// Each product sum runs over its inputs in index order with fmaf (the oracle
// follows the same order in FP64).
__device__ __forceinline__ void mlp_hidden1(const float *P, const float *x, float *h1) {
  for (int u = 0; u < kMlpH; u++) {
    float a = P[kMlpB1 + u];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) a = __fmaf_rn(P[kMlpW1 + u * kMlpIn + i], x[i], a);
    h1[u] = fmaxf(a, 0.0f);
  }
}

__device__ __forceinline__ float mlp_hidden2_unit(const float *P, const float *h1, int u) {
  float a = P[kMlpB2 + u];
#pragma unroll 8
  for (int k = 0; k < kMlpH; k++) a = __fmaf_rn(P[kMlpW2 + u * kMlpH + k], h1[k], a);
  return fmaxf(a, 0.0f);
}

// logits of the 9 count classes and the length output for one sample
__device__ __forceinline__ void mlp_forward(const float *P, const float *x, float *h1, float *out) {
  mlp_hidden1(P, x, h1);
  for (int c = 0; c < kMlpOut; c++) out[c] = P[kMlpB3 + c];
  for (int u = 0; u < kMlpH; u++) {
    const float h2 = mlp_hidden2_unit(P, h1, u);
    for (int c = 0; c < kMlpOut; c++) out[c] = __fmaf_rn(P[kMlpW3 + c * kMlpH + u], h2, out[c]);
  }
}

// --------------------------------------------------------------- training
// One block of kMlpBatch threads, one sample per thread: forward with the
// activations kept in shared memory, per-sample deltas, then the weight
// gradients summed over the block's samples in sample order (each thread
// owns a set of weights), written as this block's partial.  Samples past n
// contribute nothing.
struct MlpGradArgs {
  const float *params;
  const float *X;           // standardized features, row per vertex
  const uint8_t *y_count;   // walk count label (2..10)
  const float *y_len;       // walk length label
  const uint32_t *idx;      // sample -> vertex
  uint64_t n;
  float *partial;           // gridDim.x x kMlpParams
  double *loss_partial;     // gridDim.x
};

__device__ __forceinline__ int mlp_smem_floats() {
  return kMlpParams + kMlpBatch * (2 * kMlpPad + kMlpOut + kMlpIn);
}

__global__ void __launch_bounds__(kMlpBatch) k_mlp_grad(MlpGradArgs a) {
  extern __shared__ float sm[];
  float *P = sm;
  float *H1 = P + kMlpParams;                 // [t][kMlpPad]: h1, then delta1
  float *H2 = H1 + kMlpBatch * kMlpPad;       // [t][kMlpPad]: h2, then delta2
  float *D3 = H2 + kMlpBatch * kMlpPad;       // [t][kMlpOut]
  float *XS = D3 + kMlpBatch * kMlpOut;       // [t][kMlpIn]
  __shared__ double s_loss[kMlpBatch];
  const int t = threadIdx.x;
  for (int i = t; i < kMlpParams; i += kMlpBatch) P[i] = a.params[i];
  const uint64_t sidx = (uint64_t)blockIdx.x * kMlpBatch + t;
  const bool live = sidx < a.n;
  float x[kMlpIn];
  const uint32_t v = live ? a.idx[sidx] : 0u;
#pragma unroll
  for (int i = 0; i < kMlpIn; i++) {
    x[i] = live ? a.X[(uint64_t)v * kMlpIn + i] : 0.0f;
    XS[t * kMlpIn + i] = x[i];
  }
  __syncthreads();
  float *h1 = H1 + t * kMlpPad;
  float *h2 = H2 + t * kMlpPad;
  float out[kMlpOut];
  mlp_hidden1(P, x, h1);
  for (int c = 0; c < kMlpOut; c++) out[c] = P[kMlpB3 + c];
  for (int u = 0; u < kMlpH; u++) {
    h2[u] = mlp_hidden2_unit(P, h1, u);
    for (int c = 0; c < kMlpOut; c++) out[c] = __fmaf_rn(P[kMlpW3 + c * kMlpH + u], h2[u], out[c]);
  }
  // output deltas: softmax cross-entropy (count) and squared error (length)
  double loss = 0.0;
  {
    float m = out[0];
    for (int c = 1; c < kMlpC; c++) m = fmaxf(m, out[c]);
    float e[kMlpC], se = 0.0f;
    for (int c = 0; c < kMlpC; c++) {
      e[c] = expf(out[c] - m);
      se += e[c];
    }
    const int yc = live ? (int)a.y_count[v] - 2 : 0;
    const float yl = live ? (a.y_len[v] - kLenMid) / kLenScale : 0.0f;
    for (int c = 0; c < kMlpC; c++) D3[t * kMlpOut + c] = live ? e[c] / se - (c == yc ? 1.0f : 0.0f) : 0.0f;
    const float dl = out[kMlpC] - yl;
    D3[t * kMlpOut + kMlpC] = live ? dl : 0.0f;
    if (live) loss = (double)logf(se) + (double)m - (double)out[yc] + 0.5 * (double)dl * (double)dl;
  }
  s_loss[t] = loss;
  __syncthreads();
  float *G = a.partial + (uint64_t)blockIdx.x * kMlpParams;
  // dW3, db3
  for (int w = t; w < kMlpOut * (kMlpH + 1); w += kMlpBatch) {
    const int c = w / (kMlpH + 1), u = w % (kMlpH + 1);
    float g = 0.0f;
    for (int s = 0; s < kMlpBatch; s++) g += D3[s * kMlpOut + c] * (u < kMlpH ? H2[s * kMlpPad + u] : 1.0f);
    if (u < kMlpH) G[kMlpW3 + c * kMlpH + u] = g;
    else G[kMlpB3 + c] = g;
  }
  __syncthreads();
  // delta2 = W3^T d3 * relu'(h2), in place
  for (int u = 0; u < kMlpH; u++) {
    float d = 0.0f;
    for (int c = 0; c < kMlpOut; c++) d = __fmaf_rn(P[kMlpW3 + c * kMlpH + u], D3[t * kMlpOut + c], d);
    h2[u] = h2[u] > 0.0f ? d : 0.0f;
  }
  __syncthreads();
  // dW2, db2
  for (int w = t; w < kMlpH * (kMlpH + 1); w += kMlpBatch) {
    const int u = w / (kMlpH + 1), k = w % (kMlpH + 1);
    float g = 0.0f;
    for (int s = 0; s < kMlpBatch; s++) g += H2[s * kMlpPad + u] * (k < kMlpH ? H1[s * kMlpPad + k] : 1.0f);
    if (k < kMlpH) G[kMlpW2 + u * kMlpH + k] = g;
    else G[kMlpB2 + u] = g;
  }
  __syncthreads();
  // delta1 = W2^T d2 * relu'(h1), in place
  for (int k = 0; k < kMlpH; k++) {
    float d = 0.0f;
    for (int u = 0; u < kMlpH; u++) d = __fmaf_rn(P[kMlpW2 + u * kMlpH + k], h2[u], d);
    h1[k] = h1[k] > 0.0f ? d : 0.0f;
  }
  __syncthreads();
  // dW1, db1
  for (int w = t; w < kMlpH * (kMlpIn + 1); w += kMlpBatch) {
    const int k = w / (kMlpIn + 1), i = w % (kMlpIn + 1);
    float g = 0.0f;
    for (int s = 0; s < kMlpBatch; s++) g += H1[s * kMlpPad + k] * (i < kMlpIn ? XS[s * kMlpIn + i] : 1.0f);
    if (i < kMlpIn) G[kMlpW1 + k * kMlpIn + i] = g;
    else G[kMlpB1 + k] = g;
  }
  if (t == 0) {
    double l = 0.0;
    for (int s = 0; s < kMlpBatch; s++) l += s_loss[s];
    a.loss_partial[blockIdx.x] = l;
  }
}

// sum the block partials in block order, divide by the batch size, Adam step
// Bias corrections: bc1 / bc2, or, with bc_tab, entry *step_base + j of the
// per-step table (a captured epoch replays with the step offset in device
// memory).
__global__ void k_mlp_adam(float *params, float *m1, float *m2, const float *partial, int blocks, float inv_n,
                           float lr, float beta1, float beta2, float eps, float bc1, float bc2, float *grad_out,
                           const float2 *bc_tab = nullptr, const uint32_t *step_base = nullptr, uint32_t j = 0) {
  if (bc_tab) {
    const float2 bc = bc_tab[*step_base + j];
    bc1 = bc.x;
    bc2 = bc.y;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
    float g = 0.0f;
    for (int b = 0; b < blocks; b++) g += partial[(uint64_t)b * kMlpParams + i];
    g *= inv_n;
    if (grad_out) grad_out[i] = g;
    if (lr > 0.0f) {
      m1[i] = beta1 * m1[i] + (1.0f - beta1) * g;
      m2[i] = beta2 * m2[i] + (1.0f - beta2) * g * g;
      params[i] -= lr * (m1[i] / bc1) / (sqrtf(m2[i] / bc2) + eps);
    }
  }
}

// -------------------------------------------------------------- inference
// Per vertex: count class = argmax of the logits (+2), confidence = its
// softmax probability, length = clamp(50 + 30 out[9], 20, 80).
__global__ void __launch_bounds__(128) k_mlp_infer(const float *params, const float *X, uint32_t n, uint8_t *count,
                                                   float *conf, float *len) {
  __shared__ float P[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    float x[kMlpIn], h1[kMlpH], out[kMlpOut];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) x[i] = X[(uint64_t)v * kMlpIn + i];
    mlp_forward(P, x, h1, out);
    int best = 0;
    float m = out[0];
    for (int c = 1; c < kMlpC; c++)
      if (out[c] > m) {
        m = out[c];
        best = c;
      }
    float se = 0.0f;
    for (int c = 0; c < kMlpC; c++) se += expf(out[c] - m);
    count[v] = (uint8_t)(best + 2);
    conf[v] = 1.0f / se;
    len[v] = fminf(fmaxf(kLenMid + kLenScale * out[kMlpC], 20.0f), 80.0f);
  }
}

}  // namespace felog
