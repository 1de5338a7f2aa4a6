// Skip-gram negative-sampling kernels.
//
// One warp per sentence (Hogwild across warps, like the reference's one block
// per sentence).  Row layout is interleaved: for a row of DIM = 32 * J floats,
// physical position lane * J + j holds logical dimension lane + 32 j, so each
// lane moves its J values with one vector load / one vector reduction and the
// dot product below sums the products in exactly the order of the reference's
// shared-memory tree (word2vec.cu:510-518: pair t with t + DIM/2 via a*b + c,
// then halve).  Every multiply-add that the reference kernel fuses is written
// as an explicit fmaf and every other operation as a rounded intrinsic, so a
// single warp reproduces the reference's sequential semantics bit for bit.
#pragma once

#include "common.cuh"

namespace felog {

constexpr int kMaxNeg = 15;
constexpr int kChunk = 8;  // targets whose rows are loaded together
constexpr unsigned long long kUnigramSlots = 100000000ULL;  // table_size, word2vec.cu:171

// x % d for a 64-bit x and a fixed 32-bit d, by a precomputed reciprocal
// m = floor(2^64 / d): q = mulhi(x, m) is floor(x / d) or one less, so one
// correction step gives the exact remainder.
struct FastMod {
  unsigned long long m;
  uint32_t d;
};

inline FastMod make_fastmod(uint32_t d) {
  FastMod f;
  f.d = d;
  f.m = d <= 1 ? 0ULL : (unsigned long long)(((unsigned __int128)1 << 64) / d);
  return f;
}

__device__ __forceinline__ uint32_t fastmod(unsigned long long x, const FastMod &f) {
  if (f.d <= 1) return 0;
  unsigned long long q = __umul64hi(x, f.m);
  unsigned long long r = x - q * (unsigned long long)f.d;
  return (uint32_t)(r >= f.d ? r - f.d : r);
}

struct SgArgs {
  float *syn0;
  float *syn1;
  const int32_t *sen;
  const uint64_t *sent_start;  // n_sent + 1
  const uint32_t *blk;         // index of the sentence in its batch
  const int32_t *negs;         // reuse-neg: negative per sentence (sentence-major)
  uint64_t n_sent;
  const int32_t *table;
  uint64_t table_size;
  long long vocab_size;
  const float *exp_table;
  int window;
  int negative;
  float alpha;
  unsigned long long *next_sent;
  unsigned long long *pairs;
  FastMod fm_window;  // % window
  FastMod fm_vocab1;  // % (vocab_size - 1)
};

template <int J>
__device__ __forceinline__ void ld_row(const float *row, float (&r)[J]) {
  const float *p = row + lane_id() * J;
  if constexpr (J == 8) {
    float4 u = __ldcg(reinterpret_cast<const float4 *>(p));
    float4 v = __ldcg(reinterpret_cast<const float4 *>(p) + 1);
    r[0] = u.x; r[1] = u.y; r[2] = u.z; r[3] = u.w; r[4] = v.x; r[5] = v.y; r[6] = v.z; r[7] = v.w;
  } else if constexpr (J == 4) {
    float4 u = __ldcg(reinterpret_cast<const float4 *>(p));
    r[0] = u.x; r[1] = u.y; r[2] = u.z; r[3] = u.w;
  } else if constexpr (J == 2) {
    float2 u = __ldcg(reinterpret_cast<const float2 *>(p));
    r[0] = u.x; r[1] = u.y;
  } else {
    r[0] = __ldcg(p);
  }
}

__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d) {
  asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c),
               "f"(d)
               : "memory");
}
__device__ __forceinline__ void red_add_v2(float *p, float a, float b) {
  asm volatile("red.relaxed.gpu.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b) : "memory");
}

template <int J>
__device__ __forceinline__ void red_row(float *row, const float (&u)[J]) {
  float *p = row + lane_id() * J;
  if constexpr (J == 8) {
    red_add_v4(p, u[0], u[1], u[2], u[3]);
    red_add_v4(p + 4, u[4], u[5], u[6], u[7]);
  } else if constexpr (J == 4) {
    red_add_v4(p, u[0], u[1], u[2], u[3]);
  } else if constexpr (J == 2) {
    red_add_v2(p, u[0], u[1]);
  } else {
    atomicAdd(p, u[0]);
  }
}

// dot product in the reference tree order (FSIZE = DIM / 2)
template <int J>
__device__ __forceinline__ float sg_dot(const float (&x)[J], const float (&y)[J]) {
  if constexpr (J == 1) {
    float xs = __shfl_down_sync(0xffffffffu, x[0], 16);
    float ys = __shfl_down_sync(0xffffffffu, y[0], 16);
    float s = __fmaf_rn(xs, ys, __fmul_rn(x[0], y[0]));  // meaningful in lanes 0..15
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) s = __fadd_rn(s, __shfl_xor_sync(0xffffffffu, s, o));
    return __shfl_sync(0xffffffffu, s, 0);
  } else {
    float s[J / 2];
#pragma unroll
    for (int j = 0; j < J / 2; j++) s[j] = __fmaf_rn(x[j + J / 2], y[j + J / 2], __fmul_rn(x[j], y[j]));
#pragma unroll
    for (int h = J / 4; h >= 1; h >>= 1)
#pragma unroll
      for (int j = 0; j < h; j++) s[j] = __fadd_rn(s[j], s[j + h]);
    float r = s[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = __fadd_rn(r, __shfl_xor_sync(0xffffffffu, r, o));
    return r;
  }
}

// g = (label - sigma(f)) * alpha with the reference's quantized sigmoid
// (word2vec.cu:519-526; index (f + 6) * 83, EXP_TABLE_SIZE / MAX_EXP / 2 = 83).
__device__ __forceinline__ float sg_grad(float f, int label, const float *s_exp, float alpha) {
  if (f > 6.0f) return __fmul_rn((float)(label - 1), alpha);
  if (f < -6.0f) return __fmul_rn((float)label, alpha);
  int idx = (int)__fmul_rn(__fadd_rn(f, 6.0f), 83.0f);
  return __fmul_rn(__fsub_rn((float)label, s_exp[idx]), alpha);
}

// skip_gram_kernel semantics (word2vec.cu:442-536, hs = 0) per warp, any
// number of negatives (chunks of kChunk targets).
template <int DIM>
__global__ void __launch_bounds__(256) k_sgns_skipgram_any(SgArgs a) {
  constexpr int J = DIM / 32;
  __shared__ float s_exp[1000];
  for (int i = threadIdx.x; i < 1000; i += blockDim.x) s_exp[i] = a.exp_table[i];
  __syncthreads();
  const int lane = lane_id();
  unsigned long long my_pairs = 0;
  for (;;) {
    unsigned long long s = 0;
    if (lane == 0) s = atomicAdd(a.next_sent, 1ULL);
    s = __shfl_sync(0xffffffffu, s, 0);
    if (s >= a.n_sent) break;
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    unsigned long long nr = a.blk[s];
    for (long long pos = sb; pos < se; pos++) {
      const int word = a.sen[pos];
      nr = nr * 2514903917ULL + 11ULL;  // the reference's window LCG (word2vec.cu:458)
      const int b = (int)(nr % (unsigned long long)a.window);
      for (int aa = b; aa < a.window * 2 + 1 - b; aa++) {
        if (aa == a.window) continue;
        const long long c = pos - a.window + aa;
        if (c < sb || c >= se) continue;
        const int l1 = a.sen[c];
        float *xrow = a.syn0 + (long long)l1 * DIM;
        float x[J];
        ld_row<J>(xrow, x);
        float neu[J];
#pragma unroll
        for (int j = 0; j < J; j++) neu[j] = 0.0f;
        my_pairs++;
        for (int d0 = 0; d0 <= a.negative; d0 += kChunk) {
          int tg[kChunk];
          int lab[kChunk];
          float y[kChunk][J];
          const int nd = min(kChunk, a.negative + 1 - d0);
          // targets of this chunk, in the reference's draw order
#pragma unroll
          for (int q = 0; q < kChunk; q++) {
            tg[q] = -1;
            if (q < nd) {
              const int d = d0 + q;
              if (d == 0) {
                tg[q] = word;
                lab[q] = 1;
              } else {
                nr = nr * 25214903917ULL + 11ULL;
                int t = a.table[(nr >> 16) % a.table_size];
                if (t == 0) t = (int)(nr % (unsigned long long)(a.vocab_size - 1) + 1);
                tg[q] = t == word ? -1 : t;
                lab[q] = 0;
              }
            }
          }
#pragma unroll
          for (int q = 0; q < kChunk; q++)
            if (tg[q] >= 0) ld_row<J>(a.syn1 + (long long)tg[q] * DIM, y[q]);
#pragma unroll
          for (int q = 0; q < kChunk; q++) {
            if (tg[q] < 0) continue;
            const float f = sg_dot<J>(x, y[q]);
            const float g = sg_grad(f, lab[q], s_exp, a.alpha);
            float upd[J];
#pragma unroll
            for (int j = 0; j < J; j++) {
              neu[j] = __fmaf_rn(g, y[q][j], neu[j]);
              upd[j] = __fmul_rn(g, x[j]);
            }
            red_row<J>(a.syn1 + (long long)tg[q] * DIM, upd);
            // a later target with the same row sees this update
#pragma unroll
            for (int r = q + 1; r < kChunk; r++)
              if (tg[r] == tg[q])
#pragma unroll
                for (int j = 0; j < J; j++) y[r][j] = __fadd_rn(y[q][j], upd[j]);
          }
        }
        red_row<J>(xrow, neu);
      }
    }
  }
  if (lane == 0 && my_pairs) atomicAdd(a.pairs, my_pairs);
}

// skip_gram_kernel semantics for a fixed number of negatives NK, pipelined:
// the draw sequence of the reference's LCG does not depend on the rows, so
// the next (center, context) pair and its K unigram-table slots are produced
// while the current pair is trained, and the table loads of the next pair are
// in flight during the current pair's row loads and updates.  The LCG steps
// happen in the reference's order: one window draw per center
// (word2vec.cu:458-459), then K negative draws per context in range
// (:502-505).
template <int DIM, int NK>
__global__ void __launch_bounds__(256) k_sgns_skipgram(SgArgs a) {
  constexpr int J = DIM / 32;
  constexpr int NT = NK + 1;
  __shared__ float s_exp[1000];
  for (int i = threadIdx.x; i < 1000; i += blockDim.x) s_exp[i] = a.exp_table[i];
  __syncthreads();
  const int lane = lane_id();
  unsigned long long my_pairs = 0;
  for (;;) {
    unsigned long long s = 0;
    if (lane == 0) s = atomicAdd(a.next_sent, 1ULL);
    s = __shfl_sync(0xffffffffu, s, 0);
    if (s >= a.n_sent) break;
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    unsigned long long nr = a.blk[s];
    long long pos = sb - 1;
    int aa = 0, hi = 0, word = 0;
    // next valid pair: center word, context row, K table slots and fallbacks
    auto advance = [&](int &w_out, int &l1_out, int32_t (&tv)[NK], int (&fb)[NK]) -> bool {
      for (;;) {
        if (aa >= hi) {
          pos++;
          if (pos >= se) return false;
          word = __ldg(&a.sen[pos]);
          nr = nr * 2514903917ULL + 11ULL;
          const int b = (int)fastmod(nr, a.fm_window);
          aa = b;
          hi = a.window * 2 + 1 - b;
        }
        const int ca = aa++;
        if (ca == a.window) continue;
        const long long c = pos - a.window + ca;
        if (c < sb || c >= se) continue;
        w_out = word;
        l1_out = __ldg(&a.sen[c]);
#pragma unroll
        for (int q = 0; q < NK; q++) {
          nr = nr * 25214903917ULL + 11ULL;
          tv[q] = __ldg(&a.table[(nr >> 16) % kUnigramSlots]);
          fb[q] = (int)fastmod(nr, a.fm_vocab1) + 1;
        }
        return true;
      }
    };
    int c_word = 0, c_l1 = 0;
    int32_t c_tv[NK];
    int c_fb[NK];
    bool have = advance(c_word, c_l1, c_tv, c_fb);
    while (have) {
      int n_word = 0, n_l1 = 0;
      int32_t n_tv[NK];
      int n_fb[NK];
      const bool nhave = advance(n_word, n_l1, n_tv, n_fb);
      // targets of the current pair (word2vec.cu:496-507)
      int tg[NT];
      tg[0] = c_word;
#pragma unroll
      for (int q = 0; q < NK; q++) {
        const int t = c_tv[q] == 0 ? c_fb[q] : c_tv[q];
        tg[q + 1] = t == c_word ? -1 : t;
      }
      float *xrow = a.syn0 + (long long)c_l1 * DIM;
      float x[J];
      ld_row<J>(xrow, x);
      float y[NT][J];
#pragma unroll
      for (int q = 0; q < NT; q++)
        if (tg[q] >= 0) ld_row<J>(a.syn1 + (long long)tg[q] * DIM, y[q]);
      float neu[J];
#pragma unroll
      for (int j = 0; j < J; j++) neu[j] = 0.0f;
#pragma unroll
      for (int q = 0; q < NT; q++) {
        if (tg[q] < 0) continue;
        const float f = sg_dot<J>(x, y[q]);
        const float g = sg_grad(f, q == 0 ? 1 : 0, s_exp, a.alpha);
        float upd[J];
#pragma unroll
        for (int j = 0; j < J; j++) {
          neu[j] = __fmaf_rn(g, y[q][j], neu[j]);
          upd[j] = __fmul_rn(g, x[j]);
        }
        red_row<J>(a.syn1 + (long long)tg[q] * DIM, upd);
#pragma unroll
        for (int r = q + 1; r < NT; r++)
          if (tg[r] == tg[q])
#pragma unroll
            for (int j = 0; j < J; j++) y[r][j] = __fadd_rn(y[q][j], upd[j]);
      }
      red_row<J>(xrow, neu);
      my_pairs++;
      c_word = n_word;
      c_l1 = n_l1;
#pragma unroll
      for (int q = 0; q < NK; q++) {
        c_tv[q] = n_tv[q];
        c_fb[q] = n_fb[q];
      }
      have = nhave;
    }
  }
  if (lane == 0 && my_pairs) atomicAdd(a.pairs, my_pairs);
}

// cbow_kernel semantics (word2vec.cu:538-646, hs = 0) per warp: the mean of
// the window's context rows (summed in window order, then divided by the
// count) is scored against the positive and K negatives; every context row
// then receives the accumulated error.
template <int DIM>
__global__ void __launch_bounds__(256) k_sgns_cbow(SgArgs a) {
  constexpr int J = DIM / 32;
  __shared__ float s_exp[1000];
  for (int i = threadIdx.x; i < 1000; i += blockDim.x) s_exp[i] = a.exp_table[i];
  __syncthreads();
  const int lane = lane_id();
  unsigned long long my_pairs = 0;
  for (;;) {
    unsigned long long s = 0;
    if (lane == 0) s = atomicAdd(a.next_sent, 1ULL);
    s = __shfl_sync(0xffffffffu, s, 0);
    if (s >= a.n_sent) break;
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    unsigned long long nr = a.blk[s];
    for (long long pos = sb; pos < se; pos++) {
      const int word = a.sen[pos];
      nr = nr * 2514903917ULL + 11ULL;
      const int b = (int)(nr % (unsigned long long)a.window);
      float neu1[J], neu1e[J];
#pragma unroll
      for (int j = 0; j < J; j++) neu1[j] = neu1e[j] = 0.0f;
      int cw = 0;
      for (int aa = b; aa < a.window * 2 + 1 - b; aa++) {
        if (aa == a.window) continue;
        const long long c = pos - a.window + aa;
        if (c < sb || c >= se) continue;
        float x[J];
        ld_row<J>(a.syn0 + (long long)a.sen[c] * DIM, x);
#pragma unroll
        for (int j = 0; j < J; j++) neu1[j] = __fadd_rn(neu1[j], x[j]);
        cw++;
      }
      if (!cw) continue;
#pragma unroll
      for (int j = 0; j < J; j++) neu1[j] = __fdiv_rn(neu1[j], (float)cw);
      my_pairs += cw;
      for (int d0 = 0; d0 <= a.negative; d0 += kChunk) {
        int tg[kChunk];
        int lab[kChunk];
        float y[kChunk][J];
        const int nd = min(kChunk, a.negative + 1 - d0);
#pragma unroll
        for (int q = 0; q < kChunk; q++) {
          tg[q] = -1;
          if (q < nd) {
            const int d = d0 + q;
            if (d == 0) {
              tg[q] = word;
              lab[q] = 1;
            } else {
              nr = nr * 25214903917ULL + 11ULL;
              int t = a.table[(nr >> 16) % a.table_size];
              if (t == 0) t = (int)(nr % (unsigned long long)(a.vocab_size - 1) + 1);
              tg[q] = t == word ? -1 : t;
              lab[q] = 0;
            }
          }
        }
#pragma unroll
        for (int q = 0; q < kChunk; q++)
          if (tg[q] >= 0) ld_row<J>(a.syn1 + (long long)tg[q] * DIM, y[q]);
#pragma unroll
        for (int q = 0; q < kChunk; q++) {
          if (tg[q] < 0) continue;
          const float f = sg_dot<J>(neu1, y[q]);
          const float g = sg_grad(f, lab[q], s_exp, a.alpha);
          float upd[J];
#pragma unroll
          for (int j = 0; j < J; j++) {
            neu1e[j] = __fmaf_rn(g, y[q][j], neu1e[j]);
            upd[j] = __fmul_rn(g, neu1[j]);
          }
          red_row<J>(a.syn1 + (long long)tg[q] * DIM, upd);
#pragma unroll
          for (int r = q + 1; r < kChunk; r++)
            if (tg[r] == tg[q])
#pragma unroll
              for (int j = 0; j < J; j++) y[r][j] = __fadd_rn(y[q][j], upd[j]);
        }
      }
      for (int aa = b; aa < a.window * 2 + 1 - b; aa++) {
        if (aa == a.window) continue;
        const long long c = pos - a.window + aa;
        if (c < sb || c >= se) continue;
        red_row<J>(a.syn0 + (long long)a.sen[c] * DIM, neu1e);
      }
    }
  }
  if (lane == 0 && my_pairs) atomicAdd(a.pairs, my_pairs);
}

}  // namespace felog
