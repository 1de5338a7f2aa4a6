// Pair stream of one skip-gram round: for every (center, context) pair of the
// batch plan, in the reference's draw order, the context row, the positive
// target (the center word) and the K negative targets of skip_gram_kernel
// (word2vec.cu:442-536, hs = 0):
//   per center (in sentence order): next = next * 2514903917 + 11,
//     b = next % window (the window shrink, :458-459);
//   per context a in [b, 2 window + 1 - b), a != window, inside the sentence:
//     K draws next = next * 25214903917 + 11, target = table[(next >> 16) %
//     1e8], 0 -> next % (vocab - 1) + 1, skipped when equal to the word
//     (:496-507);
// with next seeded by the sentence's index in its batch (blockIdx.x, :446).
// With -reuse-neg 1 (__sgNegReuse, word2vec.cu:368-440) the window is the full
// window and the K negatives are the sentence's plan negatives.
// The draws depend only on the plan, never on the rows, so one scalar thread
// per sentence produces them ahead of training; the trainer's warps then do
// row work only.
//
// Record of one pair (int32 x stride, stride = K + 3 rounded up to 4):
//   [0] context row, top bit set when two non-skipped negatives hit the same
//       row, [1] positive target, [2 .. K+1] negatives (-1: skipped),
//   [K+2] the pair's rounding key pair_key(seed, sentence, pair) (sgns.cuh).
#pragma once

#include "common.cuh"
#include "sgns.cuh"

namespace felog {

constexpr uint32_t kPairDup = 0x80000000u;  // in word 0, over the context row

__host__ __device__ constexpr int pair_stride(int negative) { return (negative + 3 + 3) & ~3; }

struct PairArgs {
  const int32_t *sen;
  const uint64_t *sent_start;  // plan sentence starts (n_sent + 1)
  const uint32_t *blk;         // index of each sentence in its batch
  uint64_t s0, s1;             // sentences of this chunk
  const int32_t *table;
  FastMod fm_window;
  FastMod fm_vocab1;
  FastMod fm_table;      // % unigram table slots
  int window;
  int negative;
  int stride;
  uint64_t *count;       // pairs per sentence (count kernel: sentences s0..s1)
  const uint64_t *off;   // exclusive scan of count over the round's sentences
  uint64_t base;         // off[s0]: the first pair of the chunk
  int32_t *rec;          // records of the chunk (pair off[s] - base at rec + (off[s] - base) * stride)
  unsigned long long *cstate;  // per center (plan token): LCG state after its window draw
  uint32_t *cfirst;            // per center: pairs of its sentence before it
  const unsigned long long *jump_a, *jump_c;  // the negative LCG advanced by K j steps, j < 2 window
  int reuse;             // -reuse-neg 1: full window, negatives from negs
  const int32_t *negs;   // plan negatives, K per sentence
  const uint32_t *coarse;  // per 64-slot bucket of the unigram table (see k_unigram_coarse)
  uint32_t sr_seed;        // rounding seed of the round (the pair's key goes into its record)
};

// The unigram table is nondecreasing (word2vec.cu:683-690), so a bucket of 64
// slots holds one word iff its first and last slots agree.  coarse[k] is the
// first slot's word, with the top bit set when the whole bucket is that word;
// those slots are answered from this 6-MB array (L2-resident) instead of a
// random read of the 400-MB table.
constexpr int kCoarseShift = 6;
constexpr uint32_t kCoarseUniform = 0x80000000u;

__global__ void k_unigram_coarse(const int32_t *table, uint64_t table_size, uint32_t *coarse) {
  const uint64_t nb = (table_size + (1u << kCoarseShift) - 1) >> kCoarseShift;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nb; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t first = k << kCoarseShift;
    const uint64_t last = min(first + (1u << kCoarseShift), table_size) - 1;
    const int32_t w = table[first];
    coarse[k] = (uint32_t)w | (table[last] == w ? kCoarseUniform : 0u);
  }
}

__device__ __forceinline__ int32_t unigram_lookup(const int32_t *table, const uint32_t *coarse, uint64_t slot) {
  const uint32_t c = __ldg(&coarse[slot >> kCoarseShift]);
  return (c & kCoarseUniform) ? (int32_t)(c & ~kCoarseUniform) : __ldg(&table[slot]);
}

// number of valid contexts of the center at pos with window shrink b
__device__ __forceinline__ int contexts_of(long long pos, long long sb, long long se, int window, int b) {
  long long lo = pos - window + b, hi = pos + window - b;  // inclusive context positions
  if (lo < sb) lo = sb;
  if (hi > se - 1) hi = se - 1;
  if (hi < lo) return 0;
  return (int)(hi - lo + 1) - 1;  // minus the center itself (always inside)
}

__global__ void k_pair_count(PairArgs a) {
  for (uint64_t s = a.s0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < a.s1;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    unsigned long long nr = a.blk[s];
    uint64_t n = 0;
    for (long long pos = sb; pos < se; pos++) {
      int b = 0;
      if (!a.reuse) {
        nr = nr * 2514903917ULL + 11ULL;
        b = (int)fastmod(nr, a.fm_window);
      }
      const int c = contexts_of(pos, sb, se, a.window, b);
      a.cstate[pos] = nr;
      a.cfirst[pos] = (uint32_t)n;
      n += (uint64_t)c;
      if (c && !a.reuse) nr = a.jump_a[c] * nr + a.jump_c[c];
    }
    a.count[s] = n;
  }
}

// One warp per sentence; lane i expands pairs p0 + i + 32 u (u < kEmitUnroll,
// interleaved so that their table loads are in flight together).  A pair's
// center is the last one whose first pair is <= p, its context the
// (p - first)-th valid window position, and its K draws start from the
// center's post-window state advanced by K (p - first) steps.  Lanes write
// consecutive records (coalesced).
constexpr int kEmitUnroll = 4;

template <int K>
__global__ void __launch_bounds__(256) k_pair_emit(PairArgs a) {
  constexpr int S = pair_stride(K);
  constexpr int U = kEmitUnroll;
  const int lane = lane_id();
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  for (uint64_t s = a.s0 + warp; s < a.s1; s += nwarps) {
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    const uint64_t np = a.off[s + 1] - a.off[s];
    int32_t *r0 = a.rec + (a.off[s] - a.base) * (uint64_t)S;
    for (uint64_t p0 = 0; p0 < np; p0 += 32 * U) {
      long long pos[U], lo[U], hi[U];
      bool live[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        live[u] = p0 + lane + 32 * u < np;
        lo[u] = sb;
        hi[u] = se - 1;
      }
      // centers: largest pos in [sb, se) with cfirst[pos] <= p (binary searches side by side)
      while (true) {
        bool any = false;
#pragma unroll
        for (int u = 0; u < U; u++) any |= lo[u] < hi[u];
        if (!any) break;
#pragma unroll
        for (int u = 0; u < U; u++) {
          if (lo[u] < hi[u]) {
            const long long mid = (lo[u] + hi[u] + 1) >> 1;
            if ((uint64_t)a.cfirst[mid] <= p0 + lane + 32 * u) lo[u] = mid;
            else hi[u] = mid - 1;
          }
        }
      }
      unsigned long long nr[U];
      int word[U], ctx[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        pos[u] = lo[u];
        const uint64_t p = p0 + lane + 32 * u;
        const uint32_t j = live[u] ? (uint32_t)(p - a.cfirst[pos[u]]) : 0u;
        nr[u] = a.cstate[pos[u]];
        const int b = a.reuse ? 0 : (int)fastmod(nr[u], a.fm_window);
        long long c = pos[u] - a.window + b;
        if (c < sb) c = sb;
        c += j;
        if (c >= pos[u]) c++;
        if (c >= se) c = se - 1;  // only for lanes past the end (not written)
        word[u] = a.sen[pos[u]];
        ctx[u] = a.sen[c];
        if (!a.reuse) nr[u] = a.jump_a[j] * nr[u] + a.jump_c[j];
      }
      int32_t t[U][K];
      if (a.reuse) {
#pragma unroll
        for (int q = 0; q < K; q++)
#pragma unroll
          for (int u = 0; u < U; u++) t[u][q] = __ldg(&a.negs[s * (uint64_t)K + q]);
      } else {
#pragma unroll
        for (int q = 0; q < K; q++)
#pragma unroll
          for (int u = 0; u < U; u++) {
            nr[u] = nr[u] * 25214903917ULL + 11ULL;
            t[u][q] = unigram_lookup(a.table, a.coarse, fastmod(nr[u] >> 16, a.fm_table));
            if (t[u][q] == 0) t[u][q] = -2 - (int)fastmod(nr[u], a.fm_vocab1);  // fallback, resolved below
          }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (!live[u]) continue;
        uint32_t flags = 0;
        int32_t rv[S];
        rv[1] = word[u];
#pragma unroll
        for (int q = 0; q < K; q++) {
          int v = t[u][q];
          if (v < 0) v = -2 - v + 1;  // next % (vocab - 1) + 1
          v = v == word[u] ? -1 : v;
#pragma unroll
          for (int q2 = 0; q2 < q; q2++) flags |= (v >= 0 && rv[2 + q2] == v) ? kPairDup : 0u;
          rv[2 + q] = v;
        }
        rv[0] = (int32_t)((uint32_t)ctx[u] | flags);
        rv[2 + K] = (int32_t)pair_key(a.sr_seed, s, (uint32_t)(p0 + lane + 32 * u));
#pragma unroll
        for (int q = K + 3; q < S; q++) rv[q] = 0;
        int4 *dst = reinterpret_cast<int4 *>(r0 + (p0 + lane + 32 * u) * S);
#pragma unroll
        for (int k = 0; k < S / 4; k++) dst[k] = make_int4(rv[4 * k], rv[4 * k + 1], rv[4 * k + 2], rv[4 * k + 3]);
      }
    }
  }
}

// ---- row access for the pair trainer (DIM >= 64, J = DIM / 32 >= 2): each
// lane's J values as J / 2 float2, so the elementwise work runs on the packed
// FP32 pipe (one instruction per two values, each value rounded as in the
// scalar form).  RR: read a BF16 row again right before its store (1), never
// (0), or as SgArgs::reread says (-1); the fixed forms keep the branch out of
// the pair trainer.
template <int DIM, class P, int RR = -1>
struct LaneRows {
  static constexpr int J = DIM / 32;
  static constexpr int H = J / 2;
  const float *f[2];     // FP32 rows of syn0 / syn1 with this lane's offset
  const uint16_t *b[2];  // BF16 rows with this lane's offset, shifted so row r is at b + r * DIM
  uint32_t n_hot;
  bool reread;           // RR < 0: SgArgs::reread

  __device__ __forceinline__ void init(const SgArgs &a) {
    const int lo = lane_id() * J;
    f[0] = a.syn0 + lo;
    f[1] = a.syn1 + lo;
    n_hot = 0;
    reread = RR < 0 ? a.reread != 0 : RR > 0;
    b[0] = b[1] = nullptr;
    if constexpr (P::kBF16) {
      n_hot = (uint32_t)a.n_hot;
      const uintptr_t shift = (uintptr_t)a.n_hot * DIM * sizeof(uint16_t);
      b[0] = reinterpret_cast<const uint16_t *>(reinterpret_cast<uintptr_t>(a.syn0_bf + lo) - shift);
      b[1] = reinterpret_cast<const uint16_t *>(reinterpret_cast<uintptr_t>(a.syn1_bf + lo) - shift);
    }
  }

  template <int W>
  __device__ __forceinline__ void load(uint32_t row, float2 (&r)[H]) const {
    const float *pf = f[W] + (size_t)row * DIM;
    if constexpr (!P::kBF16) {
      load_f32(pf, r);
    } else {
      if (row < n_hot) {
        load_f32(pf, r);
      } else {
        uint32_t hv[H];
        load_b16(b[W] + (size_t)row * DIM, hv);
#pragma unroll
        for (int k = 0; k < H; k++) r[k] = make_float2(bf16_lo(hv[k]), bf16_hi(hv[k]));
      }
    }
  }

  // row += u.  FP32 rows: vector reduction (cur unchanged, returns false).
  // BF16 rows: cur becomes SR(cur + u), stored with a plain store (returns true).
  // x: the lane's mixed rounding key (lane_mix), slot: the row slot
  template <int W>
  __device__ __forceinline__ bool update(uint32_t row, const float2 (&u)[H], float2 (&cur)[H], uint32_t x,
                                         uint32_t slot) const {
    float *pf = const_cast<float *>(f[W]) + (size_t)row * DIM;
    if constexpr (!P::kBF16) {
      red_f32x2(pf, u);
      return false;
    } else {
      const bool hot = row < n_hot;
      if (!hot && (RR < 0 ? reread : RR > 0)) {
        uint32_t hv[H];
        load_b16(b[W] + (size_t)row * DIM, hv);
#pragma unroll
        for (int k = 0; k < H; k++) cur[k] = make_float2(bf16_lo(hv[k]), bf16_hi(hv[k]));
      }
      uint32_t w[H];
#pragma unroll
      for (int k = 0; k < H; k++) {
        const float2 nv = __fadd2_rn(cur[k], u[k]);
        w[k] = sr_bf16x2(nv.y, nv.x, sr_bits(x, slot, (uint32_t)k));
      }
      if (hot) {
        red_f32x2(pf, u);
      } else {
        store_b16(const_cast<uint16_t *>(b[W]) + (size_t)row * DIM, w);
#pragma unroll
        for (int k = 0; k < H; k++) cur[k] = make_float2(bf16_lo(w[k]), bf16_hi(w[k]));
      }
      return !hot;
    }
  }

  static __device__ __forceinline__ void load_f32(const float *p, float2 (&r)[H]) {
    if constexpr (H % 2 == 0) {
#pragma unroll
      for (int k = 0; k < H / 2; k++) {
        const float4 v = __ldcg(reinterpret_cast<const float4 *>(p) + k);
        r[2 * k] = make_float2(v.x, v.y);
        r[2 * k + 1] = make_float2(v.z, v.w);
      }
    } else {
      r[0] = __ldcg(reinterpret_cast<const float2 *>(p));
    }
  }
  static __device__ __forceinline__ void load_b16(const uint16_t *p, uint32_t (&h)[H]) {
    if constexpr (H == 4) {
      const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(p));
      h[0] = v.x; h[1] = v.y; h[2] = v.z; h[3] = v.w;
    } else if constexpr (H == 2) {
      const uint2 v = __ldcg(reinterpret_cast<const uint2 *>(p));
      h[0] = v.x; h[1] = v.y;
    } else {
      h[0] = __ldcg(reinterpret_cast<const unsigned int *>(p));
    }
  }
  static __device__ __forceinline__ void store_b16(uint16_t *p, const uint32_t (&w)[H]) {
    if constexpr (H == 4) *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    else if constexpr (H == 2) *reinterpret_cast<uint2 *>(p) = make_uint2(w[0], w[1]);
    else *reinterpret_cast<unsigned int *>(p) = w[0];
  }
  static __device__ __forceinline__ void red_f32x2(float *p, const float2 (&u)[H]) {
    if constexpr (H % 2 == 0) {
#pragma unroll
      for (int k = 0; k < H / 2; k++) red_add_v4(p + 4 * k, u[2 * k].x, u[2 * k].y, u[2 * k + 1].x, u[2 * k + 1].y);
    } else {
      red_add_v2(p, u[0].x, u[0].y);
    }
  }
};

// lost-update count of one store to a BF16 row (lane 0 of the warp)
__device__ __forceinline__ void count_store(uint32_t *ver, uint32_t row, uint32_t seen, uint32_t n_hot,
                                            unsigned long long &n_cold, unsigned long long &n_lost) {
  if (row < n_hot || lane_id() != 0) return;
  n_cold++;
  if (atomicAdd(&ver[row], 1u) != seen) n_lost++;
}

// in-lane part of the reference tree (pair t with t + DIM/2 via a*b + c, then
// halve) on packed values; lane value j is element j % 2 of pair j / 2
template <int H>
__device__ __forceinline__ float fold2(const float2 (&x)[H], const float2 (&y)[H]) {
  if constexpr (H == 1) {
    return __fmaf_rn(x[0].y, y[0].y, __fmul_rn(x[0].x, y[0].x));
  } else {
    float2 s[H / 2];
#pragma unroll
    for (int k = 0; k < H / 2; k++) s[k] = __ffma2_rn(x[k + H / 2], y[k + H / 2], __fmul2_rn(x[k], y[k]));
#pragma unroll
    for (int h = H / 4; h >= 1; h >>= 1)
#pragma unroll
      for (int k = 0; k < h; k++) s[k] = __fadd2_rn(s[k], s[k + h]);
    return __fadd_rn(s[0].x, s[0].y);
  }
}

template <int H>
__device__ __forceinline__ float sg_dot2(const float2 (&x)[H], const float2 (&y)[H]) {
  float r = fold2<H>(x, y);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) r = __fadd_rn(r, __shfl_xor_sync(0xffffffffu, r, o));
  return r;
}

// multi_dot on packed values: the same butterfly over the in-lane folds
template <int H, int NT>
__device__ __forceinline__ float multi_dot2(const float2 (&x)[H], const float2 (&y)[NT][H]) {
  static_assert(NT <= 8, "up to 8 targets");
  const int lane = lane_id();
  float v[8];
#pragma unroll
  for (int q = 0; q < 8; q++) v[q] = q < NT ? fold2<H>(x, y[q]) : 0.0f;
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

template <int S>
__device__ __forceinline__ int rec_at(const int4 (&v)[S / 4], int i) {
  const int4 q = v[i / 4];
  return (i & 3) == 0 ? q.x : (i & 3) == 1 ? q.y : (i & 3) == 2 ? q.z : q.w;
}

// skip_gram_kernel semantics (word2vec.cu:442-536, hs = 0) over the pair
// stream: one warp per sentence, the sentence's pairs in order.  The record of
// the next pair is loaded one pair ahead (every lane reads the same 16-byte
// words: one broadcast request).  The pair count of the chunk is known on the
// host, so the kernel counts nothing.  With distinct targets the K + 1 scores come
// from one multi_dot and each lane evaluates one gradient; a pair whose
// negatives repeat a row takes the sequential path, where the later target
// sees the earlier update as in the reference.
// MINB: resident 256-thread blocks per SM the register budget is built for
// (the launch-shape autotuner picks among 2, 3, 4 and 5 for DIM <= 128).
// RR (BF16 rows): every cold row is read again right before its store.
// CNT (diagnostic, BF16 rows): every cold-row store bumps the row's version;
// a store whose row changed version since this warp read it overwrote another
// warp's update, which is counted as lost.
template <int DIM, int NK, class P, int MINB = (DIM >= 256 ? 2 : 4), bool RR = false, bool CNT = false>
__global__ void __launch_bounds__(256, MINB)
    k_sgns_train_pairs(SgArgs a, const int32_t *__restrict__ rec, const uint64_t *__restrict__ off, uint64_t base,
                       uint64_t s0) {
  static_assert(DIM >= 64, "two or more values per lane");
  constexpr int H = DIM / 64;
  constexpr int NT = NK + 1;
  constexpr int S = pair_stride(NK);
  constexpr bool kMulti = NT <= 8;
  __shared__ float s_exp[1000];
  load_exp(a, s_exp);
  const int lane = lane_id();
  LaneRows<DIM, P, RR ? 1 : 0> rows;
  rows.init(a);
  unsigned long long n_cold = 0, n_lost = 0;  // CNT only
  unsigned long long sc;
  while (claim_sentence(a, sc)) {
    const uint64_t gs = s0 + sc;  // sentence index in the round's plan
    // pair indices relative to the chunk (a chunk holds at most 2^27 pairs)
    const uint32_t pb = (uint32_t)(off[gs] - base), pe = (uint32_t)(off[gs + 1] - base);
    if (pb == pe) continue;
    int4 nxt[S / 4];
#pragma unroll
    for (int k = 0; k < S / 4; k++) nxt[k] = __ldg(reinterpret_cast<const int4 *>(rec + (size_t)pb * S) + k);
    for (uint32_t p = pb; p < pe; p++) {
      int4 cur[S / 4];
#pragma unroll
      for (int k = 0; k < S / 4; k++) cur[k] = nxt[k];
      if (p + 1 < pe) {
#pragma unroll
        for (int k = 0; k < S / 4; k++) nxt[k] = __ldg(reinterpret_cast<const int4 *>(rec + (size_t)(p + 1) * S) + k);
      }
      const uint32_t r0 = (uint32_t)rec_at<S>(cur, 0);
      const uint32_t l1 = r0 & ~kPairDup;
      int tg[NT];
#pragma unroll
      for (int q = 0; q < NT; q++) tg[q] = rec_at<S>(cur, 1 + q);
      const bool dup = (r0 & kPairDup) != 0;
      float2 x[H];
      uint32_t seen[NT + 1];
      if constexpr (CNT) {
        seen[NT] = __ldcg(&a.ver0[l1]);
#pragma unroll
        for (int q = 0; q < NT; q++) seen[q] = tg[q] >= 0 ? __ldcg(&a.ver1[tg[q]]) : 0u;
      }
      rows.template load<0>(l1, x);
      float2 y[NT][H];
#pragma unroll
      for (int q = 0; q < NT; q++)
        if (tg[q] >= 0) rows.template load<1>((uint32_t)tg[q], y[q]);
      float2 neu[H];
#pragma unroll
      for (int k = 0; k < H; k++) neu[k] = make_float2(0.0f, 0.0f);
      const uint32_t key = P::kBF16 ? lane_mix((uint32_t)rec_at<S>(cur, NK + 2), lane) : 0u;
      bool done = false;
      if constexpr (kMulti) {
        if (!dup) {
          const float z = multi_dot2<H, NT>(x, y);
          const int tq = butterfly_target(lane);
          const float gv = tq < NT ? sg_grad(z, tq == 0 ? 1 : 0, s_exp, a.alpha) : 0.0f;
#pragma unroll
          for (int q = 0; q < NT; q++) {
            const float g = __shfl_sync(0xffffffffu, gv, butterfly_lane(q));
            if (tg[q] < 0) continue;
            const float2 g2 = make_float2(g, g);
            float2 upd[H];
#pragma unroll
            for (int k = 0; k < H; k++) {
              neu[k] = __ffma2_rn(g2, y[q][k], neu[k]);
              upd[k] = __fmul2_rn(g2, x[k]);
            }
            if constexpr (CNT && RR) seen[q] = __ldcg(&a.ver1[tg[q]]);  // the window starts at the re-read
            rows.template update<1>((uint32_t)tg[q], upd, y[q], key, (uint32_t)q);
            if constexpr (CNT) count_store(a.ver1, (uint32_t)tg[q], seen[q], rows.n_hot, n_cold, n_lost);
          }
          done = true;
        }
      }
      if (!done) {
#pragma unroll
        for (int q = 0; q < NT; q++) {
          if (tg[q] < 0) continue;
          const float f = sg_dot2<H>(x, y[q]);
          const float g = sg_grad(f, q == 0 ? 1 : 0, s_exp, a.alpha);
          const float2 g2 = make_float2(g, g);
          float2 upd[H];
#pragma unroll
          for (int k = 0; k < H; k++) {
            neu[k] = __ffma2_rn(g2, y[q][k], neu[k]);
            upd[k] = __fmul2_rn(g2, x[k]);
          }
          const bool stored = rows.template update<1>((uint32_t)tg[q], upd, y[q], key, (uint32_t)q);
          if constexpr (CNT) {
            count_store(a.ver1, (uint32_t)tg[q], seen[q], rows.n_hot, n_cold, n_lost);
#pragma unroll
            for (int r = q + 1; r < NT; r++) seen[r] += tg[r] == tg[q] ? 1u : 0u;  // this warp's own store
          }
#pragma unroll
          for (int r = q + 1; r < NT; r++)
            if (tg[r] == tg[q])
#pragma unroll
              for (int k = 0; k < H; k++) y[r][k] = stored ? y[q][k] : __fadd2_rn(y[q][k], upd[k]);
        }
      }
      if constexpr (CNT && RR) seen[NT] = __ldcg(&a.ver0[l1]);
      rows.template update<0>(l1, neu, x, key, kSlotCtx);
      if constexpr (CNT) count_store(a.ver0, l1, seen[NT], rows.n_hot, n_cold, n_lost);
    }
  }
  if constexpr (CNT) {
    if (lane == 0 && n_cold) atomicAdd(&a.lost[0], n_cold);
    if (lane == 0 && n_lost) atomicAdd(&a.lost[1], n_lost);
  }
}

// -reuse-neg 2: __sgNegReuse's work (word2vec.cu:368-440: full window, the
// sentence's K plan negatives) as one tile per center.  The K + 1 target rows
// (the center word as positive, the negatives not equal to it) are read once
// at the center; every context in window order is read fresh, scored against
// them, and updated at once (syn0[c] += sum_j g_j y_j); the targets' updates
// sum over the center's contexts and are applied once at the end of the
// center (a negative that occurs twice gets the sum of both).  Per center this
// reads and writes n + K + 1 rows instead of 2 (K + 1) n for the pair-by-pair
// order, n being the number of contexts.
//
// WIN (-reuse-neg 4, window tiles): the same tile over skip_gram_kernel's own
// windows (word2vec.cu:442-536): the window shrink b comes from the
// sentence's LCG (:458-459) and the center's shared negatives are the K draws
// the reference makes for its first context (:496-507); the LCG then jumps
// past the K draws of every context of the center, so every center's window
// is the reference's.  Lane q < K makes draw q; one table lookup per lane.
// MINB: resident 256-thread blocks per SM the register budget is built for
// (the autotuner picks among 4, 3 and 2 at DIM 128).
template <int DIM, int NK, class P, bool WIN = false, int MINB = 4>
__global__ void __launch_bounds__(256, MINB) k_sgns_reuse_tile(SgArgs a) {
  static_assert(DIM >= 64, "two or more values per lane");
  constexpr int H = DIM / 64;
  constexpr int NT = NK + 1;
  static_assert(NT <= 8, "up to 8 targets");
  __shared__ float s_exp[1000];
  load_exp(a, s_exp);
  const int lane = lane_id();
  LaneRows<DIM, P> rows;
  rows.init(a);
  unsigned long long my_pairs = 0;
  unsigned long long s_rel;
  while (claim_sentence(a, s_rel)) {
    const unsigned long long s = a.s_first + s_rel;
    const long long sb = (long long)a.sent_start[s], se = (long long)a.sent_start[s + 1];
    int neg[NK];
    unsigned long long nr = 0;  // WIN: the sentence's LCG, seeded by its index in the batch (word2vec.cu:446)
    if constexpr (WIN) {
      nr = a.blk[s];
    } else {
#pragma unroll
      for (int q = 0; q < NK; q++) neg[q] = __ldg(&a.negs[s * (uint64_t)NK + q]);
    }
    for (long long pos = sb; pos < se; pos++) {
      const int word = __ldg(&a.sen[pos]);
      int b = 0;
      if constexpr (WIN) {
        nr = nr * 2514903917ULL + 11ULL;
        b = (int)fastmod(nr, a.fm_window);
      }
      long long c0 = pos - a.window + b, c1 = pos + a.window - b;
      if (c0 < sb) c0 = sb;
      if (c1 > se - 1) c1 = se - 1;
      if (c1 - c0 < 1) continue;  // no context, no draws
      if constexpr (WIN) {
        int v = 0;
        if (lane < NK) {
          const unsigned long long r = a.lcg_a[lane] * nr + a.lcg_c[lane];
          v = unigram_lookup(a.table, a.coarse, fastmod(r >> 16, a.fm_table));
          if (v == 0) v = (int)fastmod(r, a.fm_vocab1) + 1;
        }
#pragma unroll
        for (int q = 0; q < NK; q++) neg[q] = __shfl_sync(0xffffffffu, v, q);
        const int n = (int)(c1 - c0);
        nr = __ldg(&a.jump_a[n]) * nr + __ldg(&a.jump_c[n]);
      }
      int tg[NT];
      tg[0] = word;
#pragma unroll
      for (int q = 0; q < NK; q++) tg[q + 1] = neg[q] == word ? -1 : neg[q];
      float2 y[NT][H], dy[NT][H];
#pragma unroll
      for (int q = 0; q < NT; q++) {
#pragma unroll
        for (int k = 0; k < H; k++) {
          y[q][k] = make_float2(0.0f, 0.0f);
          dy[q][k] = make_float2(0.0f, 0.0f);
        }
        if (tg[q] >= 0) rows.template load<1>((uint32_t)tg[q], y[q]);
      }
      const uint32_t center = (uint32_t)(pos - sb);
      const uint32_t key = P::kBF16 ? lane_mix(pair_key(a.sr_seed, s, center), lane) : 0u;
      const int tq = butterfly_target(lane);
      uint32_t vmask = 0;
#pragma unroll
      for (int q = 0; q < NT; q++) vmask |= (tg[q] >= 0 ? 1u : 0u) << q;
      const bool lane_scores = tq < NT && ((vmask >> tq) & 1u);
      for (long long c = c0; c <= c1; c++) {
        if (c == pos) continue;
        const uint32_t l1 = (uint32_t)__ldg(&a.sen[c]);
        float2 x[H];
        rows.template load<0>(l1, x);
        const float z = multi_dot2<H, NT>(x, y);
        const float gv = lane_scores ? sg_grad(z, tq == 0 ? 1 : 0, s_exp, a.alpha) : 0.0f;
        float2 neu[H];
#pragma unroll
        for (int k = 0; k < H; k++) neu[k] = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < NT; q++) {
          const float g = __shfl_sync(0xffffffffu, gv, butterfly_lane(q));
          if (tg[q] < 0) continue;
          const float2 g2 = make_float2(g, g);
#pragma unroll
          for (int k = 0; k < H; k++) {
            neu[k] = __ffma2_rn(g2, y[q][k], neu[k]);
            dy[q][k] = __ffma2_rn(g2, x[k], dy[q][k]);
          }
        }
        rows.template update<0>(l1, neu, x, key, kSlotCtx + (uint32_t)(c - pos + a.window));
        my_pairs++;
      }
      // targets: a repeated negative adds its sum into the first occurrence
#pragma unroll
      for (int q = 2; q < NT; q++) {
        bool merged = false;
#pragma unroll
        for (int r = 1; r < q; r++) {
          const bool hit = !merged && tg[q] >= 0 && tg[r] == tg[q];
#pragma unroll
          for (int k = 0; k < H; k++) dy[r][k] = hit ? __fadd2_rn(dy[r][k], dy[q][k]) : dy[r][k];
          merged |= hit;
        }
        if (merged) tg[q] = -2;  // applied through its first occurrence
      }
#pragma unroll
      for (int q = 0; q < NT; q++)
        if (tg[q] >= 0) rows.template update<1>((uint32_t)tg[q], dy[q], y[q], key, (uint32_t)q);
    }
  }
  if (lane == 0 && my_pairs) atomicAdd(a.pairs, my_pairs);
}

// Center tiles of -reuse-neg 3 hold at most kTileRows contexts per center
// (window <= kTileRows / 2); their staging rounds to nearest BF16.
constexpr int kTileRows = 32;

__device__ __forceinline__ uint32_t bf16x2_rn(float hi, float lo) {
  uint32_t d;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

// Row references of a chunk of pair records: per pair its context row and
// every target row that is trained (a skipped negative is -1), and how many of
// them are FP32 master rows (row < n_hot).  out[0] += references, out[1] +=
// master-row references.
__global__ void k_pair_row_mix(const int32_t *__restrict__ rec, uint64_t n, int stride, int nt, uint32_t n_hot,
                               unsigned long long *out) {
  unsigned long long refs = 0, hot = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t *r = rec + i * (uint64_t)stride;
    refs++;
    hot += ((uint32_t)r[0] & ~kPairDup) < n_hot;
    for (int q = 0; q < nt; q++) {
      const int32_t t = r[1 + q];
      refs += t >= 0;
      hot += t >= 0 && (uint32_t)t < n_hot;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    refs += __shfl_down_sync(0xffffffffu, refs, o);
    hot += __shfl_down_sync(0xffffffffu, hot, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (refs) atomicAdd(&out[0], refs);
    if (hot) atomicAdd(&out[1], hot);
  }
}

}  // namespace felog
