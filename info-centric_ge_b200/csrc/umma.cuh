// Fifth-generation tensor cores (tcgen05) for the center tiles of -reuse-neg 3.
//
// -reuse-neg 3 scores, per center, the window's contexts against the center's
// K + 1 targets (the center word and the sentence's shared negatives,
// __sgNegReuse's work, word2vec.cu:368-440) as one [contexts x DIM] x
// [DIM x (K + 1)] product.  One center is far below one tcgen05.mma (M = 128
// rows), so the four warps of a CTA share one A operand, one quarter each,
// and every warp walks its own sentence in order:
//   rows 32 w .. 32 w + 31 of A  = the contexts of warp w's center (BF16)
//   rows  8 w ..  8 w + 7  of B  = its K + 1 <= 8 targets (BF16)
// Warps do not wait for one another: when warp w has staged its center, one
// of its lanes issues D_w = A B_w^T (M = 128, N = 16, K = DIM) into its own
// 16 tensor-memory columns, B_w being B rows 8 w .. 8 w + 15, and commits to
// its own mbarrier.  The warp reads back D_w[32 w + t][q], q < 8, with
// tcgen05.ld (TMEM lanes 32 w .. 32 w + 31 are the lanes warp w may access).
// The other rows and columns of D_w mix in other warps' operands, possibly
// half written, and are never read: each D value depends only on its own row
// of A and row of B.  Everything after the
// scores is per warp: per center, all n <= 32 contexts and the K + 1 targets
// are read at the start of the center and staged as BF16 (FP32 master rows
// rounded to nearest), scored with FP32 accumulation; a context word that
// occurs twice in the window gets the sum of its rows of G, a negative that
// occurs twice the sum of its columns, so every row receives one update per
// center: syn0[c] += sum_j G_cj y_j (y in FP32), syn1[t_j] += sum_c G_cj x_c
// (x as staged).
//
// Shared-memory operands use the K-major 128-byte-swizzle layout: rows of 64
// BF16 (128 B), 8-row atoms of 1 KB (16-byte chunk c of row r stored at chunk
// c ^ (r & 7)), atoms stacked along M/N (stride 1 KB), and the second 64 K
// values of every row in a second such region.  K runs over the rows'
// physical (interleaved) order: a dot product does not depend on the order of
// its terms, and contexts and targets share the layout.
#pragma once

#include "pairs.cuh"

namespace felog {

constexpr int kUmmaWarps = 4;                 // centers (warps) per CTA
constexpr int kUmmaM = 32 * kUmmaWarps;       // A rows: 32 contexts per warp
constexpr int kUmmaN = 16;                    // N of one warp's product: its 8 target rows and the next 8
constexpr int kUmmaBRows = 8 * kUmmaWarps + 8;  // B rows: 8 targets per warp + 8 rows read by the last warp
constexpr uint32_t kUmmaTmemCols = kUmmaN * kUmmaWarps;  // FP32 accumulator columns, 16 per warp
constexpr uint32_t kUmmaWaitLimit = 1u << 22; // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major with 128-byte swizzle: start
// address >> 4 (bits 0-13), leading byte offset 16 B (bits 16-29, unused by
// this layout), stride byte offset 1024 B between 8-row atoms (bits 32-45),
// descriptor version 1 (bits 46-47), base offset 0 (atoms 1-KB aligned),
// layout type 2 = 128-byte swizzle (bits 61-63).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 (bits
// 17-22), M >> 4 (bits 24-28); dense, no negation, no saturation.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory become visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D (tensor memory) = A B^T (+ D when acc != 0), one elected thread
__device__ __forceinline__ void umma_bf16_ss(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                             uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
// the mbarrier completes one phase when every tcgen05.mma issued before by
// this thread has finished
__device__ __forceinline__ void umma_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(mbar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(mbar)), "r"(parity)
      : "memory");
  return done != 0;
}
// 8 consecutive FP32 columns of this thread's TMEM lane (warp w: lanes 32 w ..)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// Asynchronous copy of this lane's BF16 values of a row (DIM / 32 values:
// 8 B at DIM 128, 4 B at DIM 64) from global to shared memory.
template <int DIM>
__device__ __forceinline__ void cp_async_row(uint8_t *dst, const uint16_t *src) {
  constexpr int kBytes = DIM / 32 * 2;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src), "n"(kBytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Byte offset of this lane's BF16 values of row `row` in a swizzled operand
// region of `rows` rows: the lane holds physical values lane J .. lane J + J - 1
// (J = DIM / 32), which stay inside one 16-byte chunk.
template <int DIM>
__device__ __forceinline__ uint32_t sw128_offset(int rows, int row, int lane) {
  constexpr int J = DIM / 32;
  const int p0 = lane * J;
  const int half = p0 >> 6, kk = p0 & 63;
  const int chunk = kk >> 3;
  return (uint32_t)(half * rows * 128 + (row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4) +
                    (kk & 7) * 2);
}

template <int DIM>
__device__ __forceinline__ void stage_row(uint8_t *base, int rows, int row, int lane, const float2 (&x)[DIM / 64]) {
  constexpr int W = DIM / 64;
  uint8_t *p = base + sw128_offset<DIM>(rows, row, lane);
  if constexpr (W == 2) {
    *reinterpret_cast<uint2 *>(p) = make_uint2(bf16x2_rn(x[0].y, x[0].x), bf16x2_rn(x[1].y, x[1].x));
  } else {
    *reinterpret_cast<uint32_t *>(p) = bf16x2_rn(x[0].y, x[0].x);
  }
}

template <int DIM>
__device__ __forceinline__ void unstage_row(const uint8_t *base, int rows, int row, int lane,
                                            float2 (&x)[DIM / 64]) {
  constexpr int W = DIM / 64;
  const uint8_t *p = base + sw128_offset<DIM>(rows, row, lane);
  if constexpr (W == 2) {
    const uint2 w = *reinterpret_cast<const uint2 *>(p);
    x[0] = make_float2(bf16_lo(w.x), bf16_hi(w.x));
    x[1] = make_float2(bf16_lo(w.y), bf16_hi(w.y));
  } else {
    const uint32_t w = *reinterpret_cast<const uint32_t *>(p);
    x[0] = make_float2(bf16_lo(w), bf16_hi(w));
  }
}

template <int DIM>
struct UmmaSmem {
  static constexpr int KH = DIM / 64;                       // 128-byte K slices per row
  static constexpr uint32_t kA = (uint32_t)KH * kUmmaM * 128;  // A operand bytes
  static constexpr uint32_t kB = (uint32_t)KH * kUmmaBRows * 128;  // B operand bytes
  static constexpr uint32_t kG = kUmmaWarps * 32 * 8 * 4;   // gradients
  static constexpr uint32_t kIdx = kUmmaWarps * 32 * 4 * 2; // context words and first occurrences
  static constexpr uint32_t kBytes = kA + kB + kG + kIdx + 8 * kUmmaWarps + 16;
  static constexpr uint32_t kDynamic = kBytes + 1024;      // + alignment slack for the 1-KB atoms
};

// k_sgns_tile_umma<DIM, NK>: -reuse-neg 3 with tcgen05.  n_workers warps of
// each CTA take sentences (1 in the one-warp deterministic mode, so that
// sentences are trained in order; 4 otherwise).  Every mbarrier wait is
// bounded; a wait that gives up records kErrWaitTimeout and the warp stops;
// the CTA frees its tensor memory once all warps have stopped.
template <int DIM, int NK>
__global__ void __launch_bounds__(32 * kUmmaWarps, 4) k_sgns_tile_umma(SgArgs a, int n_workers) {
  static_assert(DIM == 64 || DIM == 128, "staged tile sizes");
  constexpr int H = DIM / 64;
  constexpr int NT = NK + 1;
  static_assert(NT <= 8, "eight target columns per warp");
  using P = RowsBF16;
  using L = UmmaSmem<DIM>;
  __shared__ float s_exp[1000];
  extern __shared__ uint8_t dsm_raw[];
  uint8_t *dsm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dsm_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t *sA = dsm;
  uint8_t *sB = dsm + L::kA;
  float(*sg)[32][8] = reinterpret_cast<float(*)[32][8]>(sB + L::kB);
  int(*sword)[32] = reinterpret_cast<int(*)[32]>(dsm + L::kA + L::kB + L::kG);
  int(*sfirst)[32] = sword + kUmmaWarps;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(dsm + L::kA + L::kB + L::kG + L::kIdx);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + kUmmaWarps);

  load_exp(a, s_exp);  // ends with __syncthreads
  const int warp = threadIdx.x >> 5, lane = lane_id();
  if (warp == 0) {
    tmem_alloc(tmem_slot, kUmmaTmemCols);
    tmem_relinquish();
  }
  if (threadIdx.x == 32) {
    for (int w = 0; w < kUmmaWarps; w++) mbar_init(mbar + w, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t idesc = umma_idesc_bf16(kUmmaM, kUmmaN);

  LaneRows<DIM, P> rows;
  rows.init(a);
  unsigned long long my_pairs = 0;
  bool worker = warp < n_workers, have = false;
  unsigned long long s = 0;
  long long sb = 0, se = 0, pos = 0;
  int neg[NK];
#pragma unroll
  for (int q = 0; q < NK; q++) neg[q] = 0;
  uint32_t phase = 0;
  uint8_t *wA = sA;  // this warp's context rows are rows 32 warp .. of A
  uint8_t *wB = sB;  // its targets rows 8 warp .. of B
  for (;;) {
    // this warp's next center with at least one context
    bool active = false;
    int n = 0, word = 0;
    long long c0 = 0;
    while (worker) {
      if (!have) {
        if (!claim_sentence(a, s)) {
          worker = false;
          break;
        }
        have = true;
        sb = (long long)a.sent_start[s];
        se = (long long)a.sent_start[s + 1];
        pos = sb;
#pragma unroll
        for (int q = 0; q < NK; q++) neg[q] = __ldg(&a.negs[s * (uint64_t)NK + q]);
      }
      if (pos >= se) {
        have = false;
        continue;
      }
      word = __ldg(&a.sen[pos]);
      c0 = pos - a.window;
      long long c1 = pos + a.window;
      if (c0 < sb) c0 = sb;
      if (c1 > se - 1) c1 = se - 1;
      n = (int)(c1 - c0);
      if (n < 1) {
        pos++;
        continue;
      }
      active = true;
      break;
    }
    int tg[NT];
    float2 y[NT][H];
    if (active) {
      tg[0] = word;
#pragma unroll
      for (int q = 0; q < NK; q++) tg[q + 1] = neg[q] == word ? -1 : neg[q];
      // targets: FP32 in registers, BF16 in B rows 8 warp + q (unused columns keep old values; never read)
#pragma unroll
      for (int q = 0; q < NT; q++) {
#pragma unroll
        for (int k = 0; k < H; k++) y[q][k] = make_float2(0.0f, 0.0f);
        if (tg[q] >= 0) rows.template load<1>((uint32_t)tg[q], y[q]);
        stage_row<DIM>(wB, kUmmaBRows, 8 * warp + q, lane, y[q]);
      }
      // contexts in window order into A rows 32 warp + i, i < n: lane i reads
      // the i-th context word; BF16 rows go to shared memory by asynchronous
      // copies (all in flight at once), FP32 master rows through registers,
      // rounded to nearest, four at a time
      int cw = -1;
      if (lane < n) {
        long long c = c0 + lane;
        if (c >= pos) c++;
        cw = __ldg(&a.sen[c]);
      }
      sword[warp][lane] = cw;
      const unsigned hot = __ballot_sync(0xffffffffu, lane < n && (uint32_t)cw < rows.n_hot);
      for (int i = 0; i < n; i++) {
        const int w = __shfl_sync(0xffffffffu, cw, i);
        if ((hot >> i) & 1u) continue;
        cp_async_row<DIM>(wA + sw128_offset<DIM>(kUmmaM, 32 * warp + i, lane), rows.b[0] + (size_t)w * DIM);
      }
      cp_async_commit();
      for (unsigned hm = hot; hm;) {
        int idx[4];
        float2 x[4][H];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          idx[u] = hm ? __ffs(hm) - 1 : -1;
          hm &= hm ? hm - 1 : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (idx[u] >= 0) rows.template load<0>((uint32_t)__shfl_sync(0xffffffffu, cw, idx[u]), x[u]);
#pragma unroll
        for (int u = 0; u < 4; u++)
          if (idx[u] >= 0) stage_row<DIM>(wA, kUmmaM, 32 * warp + idx[u], lane, x[u]);
      }
      cp_async_wait_all();
      __syncwarp();
      // first occurrence of each context word in the window: the lowest lane
      // holding the same word (lanes past n hold distinct negative keys)
      const unsigned same = __match_any_sync(0xffffffffu, lane < n ? cw : -1 - lane);
      sfirst[warp][lane] = __ffs(same) - 1;
    }
    if (!active) break;  // this warp has no sentence left
    // the staged operands go to the tensor core once every lane has written its part
    fence_async_smem();
    tc_fence_before();
    __syncwarp();
    tc_fence_after();
    if (lane == 0) {
      const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB) + (uint32_t)warp * 1024;  // B rows 8 warp ..
#pragma unroll
      for (int ks = 0; ks < DIM / 16; ks++) {
        const uint32_t koff = (uint32_t)(ks & 3) * 32;  // K = 16 BF16 values = 32 B inside a 128-byte row
        const uint32_t ah = (uint32_t)(ks >> 2) * (kUmmaM * 128), bh = (uint32_t)(ks >> 2) * (kUmmaBRows * 128);
        umma_bf16_ss(tmem + (uint32_t)(kUmmaN * warp), umma_desc_sw128(a0 + ah + koff),
                     umma_desc_sw128(b0 + bh + koff), idesc, ks > 0 ? 1u : 0u);
      }
      umma_commit(mbar + warp);
    }
    __syncwarp();
    // bounded wait for the product
    uint32_t polls = 0;
    bool ok = true;
    while (!mbar_try_wait(mbar + warp, phase)) {
      if (++polls > kUmmaWaitLimit) {
        ok = false;
        break;
      }
    }
    phase ^= 1u;
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) set_error(a.err, kErrWaitTimeout);
      break;
    }
    tc_fence_after();
    if (active) {
      float v[8];
      tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(kUmmaN * warp), v);
      uint32_t vmask = 0;
#pragma unroll
      for (int q = 0; q < NT; q++) vmask |= (tg[q] >= 0 ? 1u : 0u) << q;
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const bool okq = lane < n && q < NT && ((vmask >> q) & 1u);
        sg[warp][lane][q] = okq ? sg_grad(v[q], q == 0 ? 1 : 0, s_exp, a.alpha) : 0.0f;
      }
      __syncwarp();
      // rows of a repeated context word go into its first occurrence
      if (lane < 8) {
        for (int i = 1; i < n; i++) {
          const int fi = sfirst[warp][i];
          if (fi != i) {
            sg[warp][fi][lane] = __fadd_rn(sg[warp][fi][lane], sg[warp][i][lane]);
            sg[warp][i][lane] = 0.0f;
          }
        }
      }
      __syncwarp();
      const uint32_t center = (uint32_t)(pos - sb);
      const uint32_t key = lane_mix(pair_key(a.sr_seed, s, center), lane);
      float2 dy[NT][H];
#pragma unroll
      for (int q = 0; q < NT; q++)
#pragma unroll
        for (int k = 0; k < H; k++) dy[q][k] = make_float2(0.0f, 0.0f);
      for (int i = 0; i < n; i++) {
        float2 xs[H];  // the context as the tensor core saw it
        unstage_row<DIM>(wA, kUmmaM, 32 * warp + i, lane, xs);
        float2 neu[H];
#pragma unroll
        for (int k = 0; k < H; k++) neu[k] = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < NT; q++) {
          const float g = sg[warp][i][q];
          const float2 g2 = make_float2(g, g);
#pragma unroll
          for (int k = 0; k < H; k++) {
            neu[k] = __ffma2_rn(g2, y[q][k], neu[k]);
            dy[q][k] = __ffma2_rn(g2, xs[k], dy[q][k]);
          }
        }
        if (sfirst[warp][i] == i) {
          const uint32_t wi = (uint32_t)sword[warp][i];
          const long long c = c0 + i + (c0 + i >= pos ? 1 : 0);
          rows.template update<0>(wi, neu, xs, key, kSlotCtx + (uint32_t)(c - pos + a.window));
        }
      }
      my_pairs += (unsigned long long)n;
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
        if (merged) tg[q] = -2;
      }
#pragma unroll
      for (int q = 0; q < NT; q++)
        if (tg[q] >= 0) rows.template update<1>((uint32_t)tg[q], dy[q], y[q], key, (uint32_t)q);
      pos++;
      __syncwarp();
    }
    tc_fence_before();
  }
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, kUmmaTmemCols);
  if (lane == 0 && my_pairs) atomicAdd(a.pairs, my_pairs);
}

}  // namespace felog
