// Skip-gram / CBOW negative-sampling kernels.
//
// One warp per sentence (Hogwild across warps, like the reference's one block
// per sentence).  Row layout is interleaved: for a row of DIM = 32 * J values,
// physical position lane * J + j holds logical dimension lane + 32 j, so each
// lane moves its J values with one vector load / one vector reduction and the
// dot product below sums the products in exactly the order of the reference's
// shared-memory tree (word2vec.cu:510-518: pair t with t + DIM/2 via a*b + c,
// then halve).  Every multiply-add that the reference kernel fuses is written
// as an explicit fmaf and every other operation as a rounded intrinsic, so a
// single warp reproduces the reference's sequential semantics bit for bit.
//
// Row storage policies (template parameter P):
//   RowsF32  - every row FP32; updates are vector reductions (the reference's
//              atomicAdd, word2vec.cu:530, :533).
//   RowsBF16 - the n_hot most frequent vocabulary rows (rows 0..n_hot-1: the
//              vocabulary is sorted by degree) are FP32 master rows updated by
//              reductions; every other row is stored in BF16, computed on in
//              FP32 and written back as the stochastically rounded new value
//              with a plain store (Hogwild).  The rounding bits come from a
//              hash of (seed, sentence, pair, slot, lane), not from the
//              schedule, so one warp is still deterministic.
#pragma once

#include <cstring>

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
  float *syn0;  // FP32 rows: all rows, or the n_hot master rows (RowsBF16)
  float *syn1;
  uint16_t *syn0_bf;  // RowsBF16: rows n_hot.. as BF16 bits, row r at (r - n_hot) * DIM
  uint16_t *syn1_bf;
  long long n_hot;
  uint32_t sr_seed;
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
  // the negative-draw LCG advanced by q + 1 steps: x -> lcg_a[q] x + lcg_c[q]
  unsigned long long lcg_a[kMaxNeg];
  unsigned long long lcg_c[kMaxNeg];
  // lost-update count (diagnostic pair-trainer variant only): per-row store
  // versions of syn0 / syn1 and the totals [cold-row updates, overwritten ones]
  uint32_t *ver0, *ver1;
  unsigned long long *lost;
  // BF16 rows are read again right before their store, so a concurrent
  // update lands in the stored value unless it falls in that last round trip
  int reread;
  // window tiles (-reuse-neg 4): the unigram table's coarse buckets, % slots,
  // and the negative LCG advanced by K j steps (j = 0 .. 2 window)
  const uint32_t *coarse;
  FastMod fm_table;
  const unsigned long long *jump_a, *jump_c;
  int *err;  // device error code (bounded waits that give up)
  uint64_t s_first;  // tile kernels: the first sentence of this launch (claims count from it)
};

// ------------------------------------------------------------ row access
template <int J>
__device__ __forceinline__ void ld_f32(const float *p, float (&r)[J]) {
  if constexpr (J % 4 == 0) {
#pragma unroll
    for (int k = 0; k < J / 4; k++) {
      float4 u = __ldcg(reinterpret_cast<const float4 *>(p) + k);
      r[4 * k] = u.x; r[4 * k + 1] = u.y; r[4 * k + 2] = u.z; r[4 * k + 3] = u.w;
    }
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
__device__ __forceinline__ void red_f32(float *p, const float (&u)[J]) {
  if constexpr (J % 4 == 0) {
#pragma unroll
    for (int k = 0; k < J / 4; k++) red_add_v4(p + 4 * k, u[4 * k], u[4 * k + 1], u[4 * k + 2], u[4 * k + 3]);
  } else if constexpr (J == 2) {
    red_add_v2(p, u[0], u[1]);
  } else {
    atomicAdd(p, u[0]);
  }
}

// 32-bit integer mixer (multiply / xor-shift), the source of the rounding bits
__host__ __device__ __forceinline__ uint32_t sr_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}

// Rounding bits.  One hash per (sentence, pair) gives the pair's key
// kp = H(seed ^ (s * 0x9E3779B1 + pair * 0x85EBCA77)); lane L mixes it to
// x = kp ^ (L * 0xC2B2AE3D).  Word k (two values) of row slot `slot` (target
// index d = 0..K for syn1 rows, kSlotCtx (+ window position for CBOW) for
// syn0 rows) takes the bits (x + slot * 0x27D4EB2F + k * 0x165667B1) *
// 0x9E3779B1 mod 2^32: the low 16 bits round the lane's value 2k, the high 16
// bits value 2k + 1.  kp is uniform, so every value's 16 bits are uniform and
// each rounding is unbiased; the bits depend on (seed, sentence, pair, slot,
// lane) only.  A word costs one multiply-add once x is known, so a kernel
// short of registers recomputes bits cheaply (the pair trainer reads kp from
// its pair record instead of hashing).
constexpr uint32_t kSlotCtx = 256;
__host__ __device__ __forceinline__ uint32_t pair_key(uint32_t seed, uint64_t s, uint32_t pair) {
  return sr_hash(seed ^ ((uint32_t)s * 0x9E3779B1u + pair * 0x85EBCA77u));
}
__host__ __device__ __forceinline__ uint32_t lane_mix(uint32_t kp, uint32_t lane) { return kp ^ (lane * 0xC2B2AE3Du); }
__host__ __device__ __forceinline__ uint32_t sr_bits(uint32_t x, uint32_t slot, uint32_t k) {
  return (x + slot * 0x27D4EB2Fu + k * 0x165667B1u) * 0x9E3779B1u;
}
// Two FP32 values to packed BF16 by stochastic rounding in one instruction
// (sm_100a cvt.rs): hi goes to the upper half with random bits r >> 16, lo to
// the lower half with r & 0xFFFF; each is (FP32 bits + 16 random bits) >> 16,
// i.e. the magnitude rounds up with probability equal to the dropped
// fraction.  (.satfinite only matters beyond the BF16 range.)
__device__ __forceinline__ uint32_t sr_bf16x2(float hi, float lo, uint32_t r) {
  uint32_t d;
  asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(r));
  return d;
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

struct RowsF32 {
  static constexpr bool kBF16 = false;
};
struct RowsBF16 {
  static constexpr bool kBF16 = true;
};

// load row `row` of table `which` (0: syn0, 1: syn1) into the lane's J values
template <int DIM, class P>
__device__ __forceinline__ void row_load(const SgArgs &a, int which, long long row, float (&r)[DIM / 32]) {
  constexpr int J = DIM / 32;
  const int lane = lane_id();
  if constexpr (P::kBF16) {
    if (row >= a.n_hot) {
      const uint16_t *b = (which ? a.syn1_bf : a.syn0_bf) + (row - a.n_hot) * DIM + lane * J;
      if constexpr (J == 8) {
        uint4 u = __ldcg(reinterpret_cast<const uint4 *>(b));
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
          r[2 * k] = bf16_lo(w[k]);
          r[2 * k + 1] = bf16_hi(w[k]);
        }
      } else if constexpr (J == 4) {
        uint2 u = __ldcg(reinterpret_cast<const uint2 *>(b));
        r[0] = bf16_lo(u.x); r[1] = bf16_hi(u.x); r[2] = bf16_lo(u.y); r[3] = bf16_hi(u.y);
      } else if constexpr (J == 2) {
        uint32_t u = __ldcg(reinterpret_cast<const unsigned int *>(b));
        r[0] = bf16_lo(u); r[1] = bf16_hi(u);
      } else {
        r[0] = __uint_as_float((uint32_t)__ldcg(reinterpret_cast<const unsigned short *>(b)) << 16);
      }
      return;
    }
  }
  ld_f32<J>((which ? a.syn1 : a.syn0) + row * DIM + lane * J, r);
}

// Add u to row `row` whose value, as this warp read it, is cur.  FP32 rows:
// vector reduction, cur unchanged, returns false.  BF16 rows: cur becomes the
// stored value SR(cur + u) (plain store), returns true.
template <int DIM, class P>
__device__ __forceinline__ bool row_update(const SgArgs &a, int which, long long row, const float (&u)[DIM / 32],
                                           float (&cur)[DIM / 32], uint32_t x, uint32_t slot) {
  constexpr int J = DIM / 32;
  const int lane = lane_id();
  if constexpr (P::kBF16) {
    if (row >= a.n_hot) {
      constexpr int W = (J + 1) / 2;
      if (a.reread) {
        float now[J];
        row_load<DIM, P>(a, which, row, now);
#pragma unroll
        for (int j = 0; j < J; j++) cur[j] = now[j];
      }
      uint32_t w[W];
#pragma unroll
      for (int k = 0; k < W; k++) {
        const float lo = __fadd_rn(cur[2 * k], u[2 * k]);
        const float hi = 2 * k + 1 < J ? __fadd_rn(cur[2 * k + 1], u[2 * k + 1]) : 0.0f;
        w[k] = sr_bf16x2(hi, lo, sr_bits(x, slot, (uint32_t)k));
        cur[2 * k] = bf16_lo(w[k]);
        if (2 * k + 1 < J) cur[2 * k + 1] = bf16_hi(w[k]);
      }
      uint16_t *b = (which ? a.syn1_bf : a.syn0_bf) + (row - a.n_hot) * DIM + lane * J;
      if constexpr (J == 8) {
        *reinterpret_cast<uint4 *>(b) = make_uint4(w[0], w[1], w[2], w[3]);
      } else if constexpr (J == 4) {
        *reinterpret_cast<uint2 *>(b) = make_uint2(w[0], w[1]);
      } else if constexpr (J == 2) {
        *reinterpret_cast<unsigned int *>(b) = w[0];
      } else {
        *reinterpret_cast<unsigned short *>(b) = (unsigned short)w[0];
      }
      return true;
    }
  }
  red_f32<J>((which ? a.syn1 : a.syn0) + row * DIM + lane * J, u);
  return false;
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

// Dot products of x against up to 8 rows y[0..NT) at once, each bit-identical
// to sg_dot.  Every lane first folds its J products per target as sg_dot does;
// then a transposing butterfly: at xor distance 16 a lane keeps the partial
// sums of half of the targets and hands the other half to its partner, at 8 a
// quarter, at 4 an eighth, then plain xor 2 and 1.  Each partial is the sum
// of the same two halves as in sg_dot (IEEE addition commutes), so the values
// are identical, for 7 shuffles instead of 5 per target.  Lane l ends with
// the dot of target butterfly_target(l).
__device__ __forceinline__ int butterfly_target(int lane) {
  return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}
__device__ __forceinline__ int butterfly_lane(int target) {
  return ((target >> 2) & 1) * 16 + ((target >> 1) & 1) * 8 + (target & 1) * 4;
}

template <int J, int NT>
__device__ __forceinline__ float multi_dot(const float (&x)[J], const float (&y)[NT][J]) {
  static_assert(NT <= 8 && J >= 2, "up to 8 targets, at least two values per lane");
  const int lane = lane_id();
  float v[8];
#pragma unroll
  for (int q = 0; q < 8; q++) {
    if (q < NT) {
      float s[J / 2];
#pragma unroll
      for (int j = 0; j < J / 2; j++) s[j] = __fmaf_rn(x[j + J / 2], y[q][j + J / 2], __fmul_rn(x[j], y[q][j]));
#pragma unroll
      for (int h = J / 4; h >= 1; h >>= 1)
#pragma unroll
        for (int j = 0; j < h; j++) s[j] = __fadd_rn(s[j], s[j + h]);
      v[q] = s[0];
    } else {
      v[q] = 0.0f;
    }
  }
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  float w[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float keep = b4 ? v[k + 4] : v[k], send = b4 ? v[k] : v[k + 4];
    w[k] = __fadd_rn(keep, __shfl_xor_sync(0xffffffffu, send, 16));
  }
  float u[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const float keep = b3 ? w[k + 2] : w[k], send = b3 ? w[k] : w[k + 2];
    u[k] = __fadd_rn(keep, __shfl_xor_sync(0xffffffffu, send, 8));
  }
  float z = __fadd_rn(b2 ? u[1] : u[0], __shfl_xor_sync(0xffffffffu, b2 ? u[0] : u[1], 4));
  z = __fadd_rn(z, __shfl_xor_sync(0xffffffffu, z, 2));
  z = __fadd_rn(z, __shfl_xor_sync(0xffffffffu, z, 1));
  return z;
}

// g = (label - sigma(f)) * alpha with the reference's quantized sigmoid
// (word2vec.cu:519-526; index (f + 6) * 83, EXP_TABLE_SIZE / MAX_EXP / 2 = 83).
__device__ __forceinline__ float sg_grad(float f, int label, const float *s_exp, float alpha) {
  if (f > 6.0f) return __fmul_rn((float)(label - 1), alpha);
  if (f < -6.0f) return __fmul_rn((float)label, alpha);
  int idx = (int)__fmul_rn(__fadd_rn(f, 6.0f), 83.0f);
  return __fmul_rn(__fsub_rn((float)label, s_exp[idx]), alpha);
}

__device__ __forceinline__ void load_exp(const SgArgs &a, float *s_exp) {
  for (int i = threadIdx.x; i < 1000; i += blockDim.x) s_exp[i] = a.exp_table[i];
  __syncthreads();
}

__device__ __forceinline__ bool claim_sentence(const SgArgs &a, unsigned long long &s) {
  unsigned long long v = 0;
  if (lane_id() == 0) v = atomicAdd(a.next_sent, 1ULL);
  s = __shfl_sync(0xffffffffu, v, 0);
  return s < a.n_sent;
}

// skip_gram_kernel semantics (word2vec.cu:442-536, hs = 0) per warp, any
// number of negatives (chunks of kChunk targets).
template <int DIM, class P>
__global__ void __launch_bounds__(256) k_sgns_skipgram_any(SgArgs a) {
  constexpr int J = DIM / 32;
  __shared__ float s_exp[1000];
  load_exp(a, s_exp);
  unsigned long long my_pairs = 0;
  unsigned long long s;
  while (claim_sentence(a, s)) {
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    unsigned long long nr = a.blk[s];
    uint32_t pair = 0;
    for (long long pos = sb; pos < se; pos++) {
      const int word = a.sen[pos];
      nr = nr * 2514903917ULL + 11ULL;  // the reference's window LCG (word2vec.cu:458)
      const int b = (int)(nr % (unsigned long long)a.window);
      for (int aa = b; aa < a.window * 2 + 1 - b; aa++) {
        if (aa == a.window) continue;
        const long long c = pos - a.window + aa;
        if (c < sb || c >= se) continue;
        const int l1 = a.sen[c];
        const uint32_t key = P::kBF16 ? lane_mix(pair_key(a.sr_seed, s, pair), lane_id()) : 0u;
        float x[J];
        row_load<DIM, P>(a, 0, l1, x);
        float neu[J];
#pragma unroll
        for (int j = 0; j < J; j++) neu[j] = 0.0f;
        my_pairs++;
        pair++;
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
            if (tg[q] >= 0) row_load<DIM, P>(a, 1, tg[q], y[q]);
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
            const bool stored = row_update<DIM, P>(a, 1, tg[q], upd, y[q], key, d0 + q);
            // a later target with the same row sees this update
#pragma unroll
            for (int r = q + 1; r < kChunk; r++)
              if (tg[r] == tg[q])
#pragma unroll
                for (int j = 0; j < J; j++) y[r][j] = stored ? y[q][j] : __fadd_rn(y[q][j], upd[j]);
          }
        }
        row_update<DIM, P>(a, 0, l1, neu, x, key, kSlotCtx);
      }
    }
  }
  if (lane_id() == 0 && my_pairs) atomicAdd(a.pairs, my_pairs);
}

// cbow_kernel semantics (word2vec.cu:538-646, hs = 0) per warp: the mean of
// the window's context rows (summed in window order, then divided by the
// count) is scored against the positive and K negatives; every context row
// then receives the accumulated error.  Rounding streams (RowsBF16) are keyed
// by the center's position in the sentence.
template <int DIM, class P>
__global__ void __launch_bounds__(256) k_sgns_cbow(SgArgs a) {
  constexpr int J = DIM / 32;
  __shared__ float s_exp[1000];
  load_exp(a, s_exp);
  unsigned long long my_pairs = 0;
  unsigned long long s;
  while (claim_sentence(a, s)) {
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    unsigned long long nr = a.blk[s];
    for (long long pos = sb; pos < se; pos++) {
      const int word = a.sen[pos];
      const uint32_t key = P::kBF16 ? lane_mix(pair_key(a.sr_seed, s, (uint32_t)(pos - sb)), lane_id()) : 0u;
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
        row_load<DIM, P>(a, 0, a.sen[c], x);
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
          if (tg[q] >= 0) row_load<DIM, P>(a, 1, tg[q], y[q]);
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
          const bool stored = row_update<DIM, P>(a, 1, tg[q], upd, y[q], key, d0 + q);
#pragma unroll
          for (int r = q + 1; r < kChunk; r++)
            if (tg[r] == tg[q])
#pragma unroll
              for (int j = 0; j < J; j++) y[r][j] = stored ? y[q][j] : __fadd_rn(y[q][j], upd[j]);
        }
      }
      // every context row receives neu1e; a BF16 row is re-read so that a
      // context that occurs twice in the window sees its first update
      for (int aa = b; aa < a.window * 2 + 1 - b; aa++) {
        if (aa == a.window) continue;
        const long long c = pos - a.window + aa;
        if (c < sb || c >= se) continue;
        float x[J];
        if constexpr (P::kBF16) row_load<DIM, P>(a, 0, a.sen[c], x);
        row_update<DIM, P>(a, 0, a.sen[c], neu1e, x, key, kSlotCtx + aa);
      }
    }
  }
  if (lane_id() == 0 && my_pairs) atomicAdd(a.pairs, my_pairs);
}

// Scores of (context, target, label) triples for the precision study: the
// dot of syn0[ctx] and syn1[target] exactly as the trainer forms it (FP32
// products and tree from the stored rows) and each triple's negative-sampling
// loss -log sigma(+-f) in FP64, summed per batch in FP64.
template <int DIM, class P>
__global__ void __launch_bounds__(256) k_score_pairs(SgArgs a, const int32_t *ctx, const int32_t *tgt,
                                                     const int8_t *label, const uint64_t *batch_of, uint64_t n,
                                                     float *dots, double *batch_loss) {
  constexpr int J = DIM / 32;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  for (uint64_t i = warp; i < n; i += nw) {
    float x[J], y[J];
    row_load<DIM, P>(a, 0, ctx[i], x);
    row_load<DIM, P>(a, 1, tgt[i], y);
    const float f = sg_dot<J>(x, y);
    if (lane_id() == 0) {
      dots[i] = f;
      const double z = label[i] ? (double)f : -(double)f;
      const double l = z > 0 ? log1p(exp(-z)) : -z + log1p(exp(z));  // -log sigma(z)
      atomicAdd(&batch_loss[batch_of[i]], l);
    }
  }
}

}  // namespace felog
