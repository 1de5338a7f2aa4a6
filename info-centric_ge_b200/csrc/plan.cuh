// Trainer batch plan on the device (word2vec.cu:1133-1248).
//
// The reference packs sentences on the host into batches of at most 15000
// sentences, closing a batch after the sentence that brings it to 299,980
// kept tokens; a sentence stops at vocabulary index 0 and after 1000 kept
// tokens; tokens whose subsampling threshold is below 65535 draw a 16-bit
// value from one LCG stream (re-seeded every round) and are dropped when the
// value exceeds the threshold; after each batch the same stream draws
// cnt * negative host negatives.  Inside a batch the kernel's LCG is seeded
// with the sentence's index in the batch (blockIdx.x).
//
// Because the draws a sentence consumes do not depend on the drawn values
// (unless a sentence reaches the 1000-token cap), the stream offset of every
// sentence is known from prefix sums, and the LCG's jump-ahead turns the
// sequential host loop into: (A) a per-sentence scan, (B) one block that walks
// the batches, each step resolving up to 15000 sentences in parallel, (C) a
// parallel emit of kept tokens, (D) a parallel draw of the negatives.
#pragma once

#include "common.cuh"

namespace felog {

constexpr int kMaxSentence = 15000;        // MAX_SENTENCE, word2vec.cu:49
constexpr int kMaxSentenceLen = 1000;      // MAX_SENTENCE_LENGTH, word2vec.cu:42
constexpr uint64_t kBatchTokens = (uint64_t)(kMaxSentence - 1) * 20;  // word2vec.cu:1234
constexpr uint32_t kOov = 0xFFFFFFFFu;

struct PlanArgs {
  const uint32_t *arena;
  const uint64_t *sent_ptr;
  const uint32_t *sent_len;
  uint64_t n_sent;
  const uint32_t *id2offset;
  const uint16_t *thr;   // NULL when the reference would not subsample
  const int32_t *table;
  uint64_t table_size;
  long long vocab_size;
  int negative;
  unsigned long long seed;
  // per sentence
  uint32_t *cand;        // candidate tokens before the first vocabulary-0 token
  uint32_t *draws;       // candidates with threshold < 65535
  uint32_t *considered;  // tokens counted by word_count
  uint32_t *kept;
  unsigned long long *state;  // LCG state at the sentence's first draw
  uint32_t *blk;         // index within its batch
  uint64_t *out_off;     // exclusive scan of kept (sent_start)
  // per batch
  uint64_t *batch_first;
  unsigned long long *neg_state;
  uint64_t max_batches;
  // outputs
  int32_t *sen;
  int32_t *negs;
  unsigned long long *counters;  // [n_batches, long_sentences]
  const LcgJump *jump;
  int *err;
};

// (A) per-sentence scan
__global__ void k_plan_scan(PlanArgs a) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < a.n_sent;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t *t = a.arena + a.sent_ptr[j];
    uint32_t n = a.sent_len[j], c = 0, d = 0, cons = 0;
    for (uint32_t i = 0; i < n; i++) {
      uint32_t off = a.id2offset[t[i]];
      if (off == kOov) continue;
      cons++;
      if (off == 0) break;
      c++;
      if (a.thr && a.thr[off] < 65535) d++;
    }
    a.cand[j] = c;
    a.draws[j] = d;
    a.considered[j] = cons;
  }
}

// Kept tokens of sentence j given the stream state at its first draw; also
// returns the number of draws actually consumed (differs from draws[j] only
// when the 1000-token cap ends the sentence early).
__device__ uint32_t plan_simulate(const PlanArgs &a, uint64_t j, unsigned long long st, uint32_t *used) {
  const uint32_t *t = a.arena + a.sent_ptr[j];
  uint32_t n = a.sent_len[j], kept = 0, u = 0;
  for (uint32_t i = 0; i < n; i++) {
    uint32_t off = a.id2offset[t[i]];
    if (off == kOov) continue;
    if (off == 0) break;
    if (a.thr) {
      uint16_t keep = a.thr[off];
      if (keep < 65535) {
        st = lcg_next(st);
        u++;
        uint16_t r16 = (uint16_t)(((uint32_t)(st >> 16)) >> 16);
        if (r16 > keep) continue;
      }
    }
    kept++;
    if (kept >= (uint32_t)kMaxSentenceLen) break;
  }
  *used = u;
  return kept;
}

template <int NT>
__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long v, unsigned long long *sh,
                                                              unsigned long long *total) {
  // Hillis-Steele over NT threads in shared memory
  int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int o = 1; o < NT; o <<= 1) {
    unsigned long long x = t >= o ? sh[t - o] : 0ULL;
    __syncthreads();
    sh[t] += x;
    __syncthreads();
  }
  unsigned long long incl = sh[t];
  *total = sh[NT - 1];
  __syncthreads();
  return incl - v;
}

// (B) walk the batches; one block of NT threads.
template <int NT>
__global__ void __launch_bounds__(NT) k_plan_batches(PlanArgs a) {
  __shared__ unsigned long long sh[NT];
  __shared__ unsigned long long s_end;
  __shared__ int s_long;
  constexpr int SPT = (kMaxSentence + NT - 1) / NT;
  const LcgJump &J = *a.jump;
  uint64_t s = 0, nb = 0;
  unsigned long long state = a.seed;
  unsigned long long n_long = 0;
  while (s < a.n_sent) {
    uint64_t W = a.n_sent - s < (uint64_t)kMaxSentence ? a.n_sent - s : (uint64_t)kMaxSentence;
    uint64_t j0 = s + (uint64_t)threadIdx.x * SPT;
    uint64_t j1 = j0 + SPT < s + W ? j0 + SPT : s + W;
    if (j0 > j1) j0 = j1;
    // draws of this thread's sentences, and whether any may hit the cap
    unsigned long long dsum = 0;
    int has_long = 0;
    for (uint64_t j = j0; j < j1; j++) {
      dsum += a.draws[j];
      has_long |= a.cand[j] >= (uint32_t)kMaxSentenceLen;
    }
    if (threadIdx.x == 0) s_long = 0;
    __syncthreads();
    if (has_long) s_long = 1;
    unsigned long long dtot;
    unsigned long long doff = block_excl_scan<NT>(dsum, sh, &dtot);
    unsigned long long ksum = 0;
    if (!s_long) {
      unsigned long long st = lcg_jump(J, state, doff);
      for (uint64_t j = j0; j < j1; j++) {
        a.state[j] = st;
        uint32_t used;
        uint32_t k = a.draws[j] ? plan_simulate(a, j, st, &used) : (a.cand[j] < (uint32_t)kMaxSentenceLen ? a.cand[j] : (uint32_t)kMaxSentenceLen);
        if (!a.draws[j]) used = 0;
        a.kept[j] = k;
        ksum += k;
        st = lcg_jump(J, st, used);
      }
    } else if (threadIdx.x == 0) {
      // a sentence may stop at the cap: resolve the window in order
      n_long++;
      unsigned long long st = state;
      for (uint64_t j = s; j < s + W; j++) {
        a.state[j] = st;
        uint32_t used;
        a.kept[j] = plan_simulate(a, j, st, &used);
        st = lcg_jump(J, st, used);
      }
    }
    __syncthreads();
    if (s_long) {
      ksum = 0;
      for (uint64_t j = j0; j < j1; j++) ksum += a.kept[j];
    }
    unsigned long long ktot;
    unsigned long long koff = block_excl_scan<NT>(ksum, sh, &ktot);
    // first sentence whose running kept total reaches the batch limit
    if (threadIdx.x == 0) s_end = s + W - 1;
    __syncthreads();
    {
      unsigned long long run = koff;
      for (uint64_t j = j0; j < j1; j++) {
        run += a.kept[j];
        if (run >= kBatchTokens) {
          atomicMin(&s_end, (unsigned long long)j);
          break;
        }
      }
    }
    __syncthreads();
    uint64_t e = s_end + 1;  // exclusive end of this batch
    // draws consumed by the batch's sentences
    unsigned long long du = 0;
    for (uint64_t j = j0; j < j1 && j < e; j++) {
      if (a.cand[j] >= (uint32_t)kMaxSentenceLen && a.draws[j]) {
        uint32_t used;
        plan_simulate(a, j, a.state[j], &used);
        du += used;
      } else {
        du += a.draws[j];
      }
      a.blk[j] = (uint32_t)(j - s);
    }
    unsigned long long dbatch;
    block_excl_scan<NT>(du, sh, &dbatch);
    if (threadIdx.x == 0) {
      if (nb < a.max_batches) {
        a.batch_first[nb] = s;
        a.neg_state[nb] = lcg_jump(J, state, dbatch);
      } else {
        set_error(a.err, kErrPlanOverflow);
      }
    }
    state = lcg_jump(J, lcg_jump(J, state, dbatch), (e - s) * (unsigned long long)a.negative);
    s = e;
    nb++;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (nb < a.max_batches + 1) a.batch_first[nb < a.max_batches ? nb : a.max_batches] = a.n_sent;
    a.counters[0] = nb;
    a.counters[1] = n_long;
  }
}

// (C) emit kept vocabulary indices of every sentence at out_off[j]
__global__ void k_plan_emit(PlanArgs a) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < a.n_sent;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t *t = a.arena + a.sent_ptr[j];
    uint32_t n = a.sent_len[j], kept = 0;
    unsigned long long st = a.state[j];
    int32_t *o = a.sen + a.out_off[j];
    for (uint32_t i = 0; i < n; i++) {
      uint32_t off = a.id2offset[t[i]];
      if (off == kOov) continue;
      if (off == 0) break;
      if (a.thr) {
        uint16_t keep = a.thr[off];
        if (keep < 65535) {
          st = lcg_next(st);
          uint16_t r16 = (uint16_t)(((uint32_t)(st >> 16)) >> 16);
          if (r16 > keep) continue;
        }
      }
      o[kept++] = (int32_t)off;
      if (kept >= (uint32_t)kMaxSentenceLen) break;
    }
  }
}

// (D) host-style negatives of every batch (word2vec.cu:1240-1248), sentence-major
__global__ void k_plan_negs(PlanArgs a, uint64_t n_batches) {
  uint64_t total = a.n_sent * (uint64_t)a.negative;
  const LcgJump &J = *a.jump;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = i / a.negative;
    // batch of sentence j: first sentence = j - blk[j]
    uint64_t first = j - a.blk[j];
    // locate the batch record by binary search on batch_first
    uint64_t lo = 0, hi = n_batches;
    while (hi - lo > 1) {
      uint64_t mid = (lo + hi) / 2;
      if (a.batch_first[mid] <= first) lo = mid;
      else hi = mid;
    }
    uint64_t pos = i - first * (uint64_t)a.negative;  // draw index within the batch
    unsigned long long st = lcg_jump(J, a.neg_state[lo], pos + 1);
    uint32_t randd = (uint32_t)(st >> 16);
    int32_t ts = a.table[randd % a.table_size];
    a.negs[i] = ts == 0 ? (int32_t)(randd % (uint64_t)(a.vocab_size - 1)) + 1 : ts;
  }
}

}  // namespace felog
