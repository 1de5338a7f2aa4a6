// Walker engine: one lane per walker, persistent grid sized to residency;
// each warp claims 32 consecutive walkers with one atomic, so uneven walks keep
// every warp busy.  The round's counters are summed per warp before the
// single atomic per counter: same-address atomics from every thread at exit
// serialize in L2 and once cost more than the walks themselves.
//
// Per walker it restates walk.hpp:926-1101 at np = 1:
//   * step 0 is the start vertex; the first visit seeds the correlation state
//     (H=0, S=1, E[H]=0, E[S]=1, E[HS]=0, E[HH]=0, E[SS]=1, N=1, R=1);
//   * each iteration draws a candidate index in [0, deg(cur)) (walk.hpp:976),
//     ends the walk if deg == 2 and the first neighbour is cur itself
//     (:977-979), redraws self-loops at step 0 (:981-983), then draws p and
//     computes p_accept = (1/(deg_s - cn)) * max(deg_s, deg_d) / min(...) with
//     cn = (int) edge data, tracing back iff tanh(p_accept) <= p (:997-1019);
//   * each appended token updates the FP64 entropy-length correlation with
//     fi = earlier visits of that vertex; the walk stops once step > min_L and
//     R^2 < 0.999 or R < 0 (:945-951, :1056-1062, :1088-1093).
// The +,-,*,/ of the correlation update are IEEE intrinsics so the compiler
// cannot contract them; pow/log2/tanh/sqrt are the FP64 device functions.
// Three exact shortcuts keep the per-token FP64 work small:
//   * E[S], E[S^2] and D_S depend only on S, so they come from a table built
//     once with the same operations (k_corr_series);
//   * a division by the integer S + 1 is Markstein's correction of the
//     product with the correctly rounded reciprocal (the table holds it),
//     which is the correctly rounded quotient; tiny dividends take __ddiv_rn;
//   * R is formed only when the stop test can fire (step > min_L).
// The trace test tanh(p_accept) <= p first runs in FP32: tanhf of the FP32
// p_accept is within 3e-7 of the FP64 tanh while degrees stay below 2^24, so
// a gap of more than 2^-16 to p decides it; otherwise the FP64 test runs.
//
// Tokens go to a per-walker slot of slot_len tokens; a walk that outgrows it
// moves to a doubled chunk of the spill arena.  The first kSmemPath tokens of
// each walk are also kept in shared memory.  fi lookups use a 64-bit Bloom
// word per walker (no scan for first visits) and a scan of the walk's own
// tokens otherwise (shared memory first, the global tail after it); the
// return step of a trace uses a running count of the current vertex.
#pragma once

#include "common.cuh"

namespace felog {

struct WalkArgs {
  const uint64_t *row_ptr;
  const uint2 *adj;
  const uint4 *wadj;        // walker entries {neighbour, data, its row start, its degree} (k_fuse_adj), or NULL
  const float *alias_prob;  // weighted mode only
  const uint32_t *alias_idx;
  uint32_t v_num;
  uint32_t n_active;
  const uint32_t *active;   // walker ids, ascending
  uint32_t min_len;
  uint32_t round;
  uint64_t seed;
  int weighted;
  // injected draws (parity mode)
  int injected;
  const uint64_t *inj_idx_off;
  const uint32_t *inj_idx;
  const uint64_t *inj_p_off;
  const double *inj_p;
  // output
  uint32_t *arena;               // [n_active * slot_len | spill region]
  uint32_t slot_len;
  unsigned long long *spill_cursor;  // tokens used in the spill region
  uint64_t spill_base;           // first token of the spill region
  uint64_t arena_cap;            // total tokens
  uint64_t *sent_ptr;            // per sentence: token offset in arena
  uint32_t *sent_len;
  unsigned int *visit_freq;      // cumulative visits per vertex (KL)
  const double *corr_tab;        // t(S, fi) table (k_corr_table), or NULL
  const double4 *corr_series;    // S-only moments and reciprocals (k_corr_series)
  unsigned int *next_walker;     // claim counter: next unclaimed walker index
  unsigned long long *stats;     // [tokens, traces, iterations, long]
  int *err;
};

struct Corr {
  double H, EH, ES, EHS, EHH, ESS, S;  // N == S throughout (both count tokens)
};

// ES and ESS are only kept current once S leaves the series table.
__device__ __forceinline__ void corr_init(Corr &c) {
  c.H = 0.0; c.EH = 0.0; c.ES = 1.0; c.EHS = 0.0; c.EHH = 0.0; c.ESS = 1.0; c.S = 1.0;
}

// The entropy increment t(S, fi) of Correlation::iterateHn with step_k = 1
// (walk.hpp:296-316): log2 of SnSn_div_Snp1Snp1(S) times, for a revisit,
// FjFj_div_FiFi(fi).  It depends only on the integers S and fi.
__device__ __forceinline__ double corr_t(double Sn, double fi) {
  const double Snp1 = __dadd_rn(Sn, 1.0);
  double ss = __dmul_rn(pow(__ddiv_rn(Sn, Snp1), Sn), pow(__ddiv_rn(1.0, Snp1), 1.0));
  if (fi == 0.0) return log2(ss);
  double fj = __dadd_rn(fi, 1.0);
  double ff = __dmul_rn(pow(__ddiv_rn(fj, fi), fi), pow(fj, 1.0));
  return log2(__dmul_rn(ss, ff));
}

// t(S, fi) for 1 <= S <= kCorrTableS and 0 <= fi <= S, computed once by
// k_corr_table with corr_t itself, so a table entry is bit-identical to the
// value the walker would compute; larger S falls back to corr_t.
constexpr int kCorrTableS = 127;
__device__ __forceinline__ uint32_t corr_tab_index(uint32_t S, uint32_t fi) { return S * (kCorrTableS + 1) + fi; }

__global__ void k_corr_table(double *tab) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (kCorrTableS + 1) * (kCorrTableS + 1);
       i += gridDim.x * blockDim.x) {
    uint32_t S = i / (kCorrTableS + 1), fi = i % (kCorrTableS + 1);
    tab[i] = (S >= 1 && fi <= S) ? corr_t((double)S, (double)fi) : 0.0;
  }
}

// Series of the S-only moments: entry s = {E[S], E[S^2], D_S, RN(1/(s+1))}
// after the update that takes S from s to s + 1 (walk.hpp:322-366 with
// step_k = 1), for 1 <= s < kCorrSeries; one thread, the walker's operations.
constexpr uint32_t kCorrSeries = 256;

__global__ void k_corr_series(double4 *ser) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double ES = 1.0, ESS = 1.0;
  ser[0] = make_double4(ES, ESS, 0.0, 1.0);
  for (uint32_t s = 1; s < kCorrSeries; s++) {
    const double Snp1 = __dadd_rn((double)s, 1.0);
    ES = __dadd_rn(ES, __ddiv_rn(__dsub_rn(Snp1, ES), Snp1));
    ESS = __dadd_rn(ESS, __ddiv_rn(__dsub_rn(__dmul_rn(Snp1, Snp1), ESS), Snp1));
    ser[s] = make_double4(ES, ESS, __dsub_rn(ESS, __dmul_rn(ES, ES)), __drcp_rn(Snp1));
  }
}

// x / n rounded to nearest for n an integer-valued double and y = RN(1/n):
// q0 = RN(x y) is within one ulp of x / n, r = x - q0 n is exact (FMA), and
// RN(q0 + r y) is the correctly rounded quotient (P. Markstein, IBM J. Res.
// Dev. 34(1), 1990).  The theorem needs a normal quotient, so dividends near
// the underflow range take the IEEE division.
__device__ __forceinline__ double div_int(double x, double n, double y) {
  if (fabs(x) < 0x1p-900) return __ddiv_rn(x, n);
  const double q0 = __dmul_rn(x, y);
  const double r = __fma_rn(-q0, n, x);
  return __fma_rn(r, y, q0);
}

// Correlation::iterate with step_k = 1 (walk.hpp:309-366) followed by the stop
// test of walk.hpp:945-951 (step > min_L and R^2 < 0.999 or R < 0); returns
// true when the walk stops after this token.
__device__ __forceinline__ bool corr_step(Corr &c, uint32_t fi_u, const double *__restrict__ tab,
                                          const double4 *s_ser, uint32_t step, uint32_t min_len) {
  const double Sn = c.S;
  const double Snp1 = __dadd_rn(Sn, 1.0);
  const uint32_t S_u = (uint32_t)Sn;
  const double t = (tab && S_u <= (uint32_t)kCorrTableS) ? __ldg(&tab[corr_tab_index(S_u, fi_u)])
                                                         : corr_t(Sn, (double)fi_u);
  double ES, DS, y;
  if (S_u < kCorrSeries) {
    const double4 q = s_ser[S_u];
    ES = q.x;
    DS = q.z;
    y = q.w;
  } else {
    const double ES0 = S_u == kCorrSeries ? s_ser[kCorrSeries - 1].x : c.ES;
    const double ESS0 = S_u == kCorrSeries ? s_ser[kCorrSeries - 1].y : c.ESS;
    ES = __dadd_rn(ES0, __ddiv_rn(__dsub_rn(Snp1, ES0), Snp1));
    const double ESS = __dadd_rn(ESS0, __ddiv_rn(__dsub_rn(__dmul_rn(Snp1, Snp1), ESS0), Snp1));
    DS = __dsub_rn(ESS, __dmul_rn(ES, ES));
    y = __drcp_rn(Snp1);
    c.ES = ES;
    c.ESS = ESS;
  }
  const double H1 = div_int(__dsub_rn(__dmul_rn(Sn, c.H), t), Snp1, y);
  // N + 1 == S + 1
  const double EH = __dadd_rn(c.EH, div_int(__dsub_rn(H1, c.EH), Snp1, y));
  const double EHS = __dadd_rn(c.EHS, div_int(__dsub_rn(__dmul_rn(H1, Snp1), c.EHS), Snp1, y));
  const double EHH = __dadd_rn(c.EHH, div_int(__dsub_rn(__dmul_rn(H1, H1), c.EHH), Snp1, y));
  c.H = H1; c.EH = EH; c.EHS = EHS; c.EHH = EHH; c.S = Snp1;
  if (step <= min_len) return false;
  const double DH = __dsub_rn(EHH, __dmul_rn(EH, EH));
  const double ex = __dsub_rn(EHS, __dmul_rn(EH, ES));
  const double R = ex == 0.0 ? 0.0 : __ddiv_rn(ex, __dsqrt_rn(__dmul_rn(DH, DS)));
  return __dmul_rn(R, R) < 0.999 || R < 0.0;
}

// The trace test of walk.hpp:997-1019: tanh(p_accept) <= p with
// p_accept = (1 / (deg_s - cn)) * max(deg_s, deg_d) / min(deg_s, deg_d).
__device__ __forceinline__ bool trace_test(int sd, int cn, int mx, int mn, double p) {
  const int dn = sd - cn;
  if (mx < (1 << 24) && dn < (1 << 24) && dn > -(1 << 24)) {
    const float tf = tanhf((1.0f / (float)dn) * (float)mx / (float)mn);
    const float pf = (float)p;
    if (fabsf(tf - pf) > 0x1p-16f) return tf < pf;
  }
  const double p_accept = __ddiv_rn(__dmul_rn(__ddiv_rn(1.0, (double)dn), (double)mx), (double)mn);
  return tanh(p_accept) <= p;
}

__device__ __forceinline__ uint64_t bloom_bit(uint32_t v) { return 1ULL << ((v * 0x9E3779B1u) >> 26); }

// Number of occurrences of v among the first n tokens of p.
__device__ __forceinline__ uint32_t count_in_path(const uint32_t *p, uint32_t n, uint32_t v) {
  uint32_t c = 0;
  uint32_t i = 0;
  for (; i + 4 <= n; i += 4) {
    uint4 q = *reinterpret_cast<const uint4 *>(p + i);
    c += (q.x == v) + (q.y == v) + (q.z == v) + (q.w == v);
  }
  for (; i < n; i++) c += p[i] == v;
  return c;
}

constexpr uint32_t kWalkThreads = 256;  // block size of k_walk
constexpr uint32_t kSmemPath = 32;      // leading tokens of each walk kept in shared memory

struct PathBuf {
  uint32_t *p;    // token storage of this walk
  uint32_t len;
  uint32_t cap;
  uint32_t *s;    // this lane's column of the block's shared token rows
};

// Occurrences of v in the walk so far: the shared-memory rows, then the tail.
__device__ __forceinline__ uint32_t count_in_walk(const PathBuf &pb, uint32_t v) {
  const uint32_t m = pb.len < kSmemPath ? pb.len : kSmemPath;
  uint32_t c = 0;
  for (uint32_t i = 0; i < m; i++) c += pb.s[i * kWalkThreads] == v;
  if (pb.len > kSmemPath) c += count_in_path(pb.p + kSmemPath, pb.len - kSmemPath, v);
  return c;
}

// Append one token, moving the walk to a larger spill chunk when full.
__device__ __forceinline__ bool path_push(const WalkArgs &a, PathBuf &pb, uint32_t v) {
  if (pb.len == pb.cap) {
    uint32_t ncap = pb.cap * 2;
    unsigned long long off = atomicAdd(a.spill_cursor, (unsigned long long)ncap);
    if (a.spill_base + off + ncap > a.arena_cap) {
      set_error(a.err, kErrArenaFull);
      return false;
    }
    uint32_t *np = a.arena + a.spill_base + off;
    for (uint32_t i = 0; i < pb.len; i++) np[i] = pb.p[i];
    pb.p = np;
    pb.cap = ncap;
  }
  if (pb.len < kSmemPath) pb.s[pb.len * kWalkThreads] = v;
  pb.p[pb.len++] = v;
  atomicAdd(&a.visit_freq[v], 1u);
  return true;
}

// INJ: parity mode with injected draws; WEIGHTED: alias-table candidates;
// FUSED: candidates read from the walker entries (one dependent random read
// per step; the walk is the same).
template <bool INJ, bool WEIGHTED, bool FUSED>
__global__ void __launch_bounds__(kWalkThreads, 3) k_walk(WalkArgs a) {
  __shared__ uint32_t s_path[kSmemPath * kWalkThreads];
  __shared__ double4 s_ser[kCorrSeries];
  for (uint32_t i = threadIdx.x; i < kCorrSeries; i += kWalkThreads) s_ser[i] = a.corr_series[i];
  __syncthreads();
  unsigned long long my_tok = 0, my_tr = 0, my_it = 0, my_long = 0;
  const uint32_t lane = threadIdx.x & 31;
  for (;;) {
    // the whole warp claims walkers base .. base + 31; once base is past the
    // end every lane leaves together
    __syncwarp();
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(a.next_walker, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= a.n_active) break;
    const uint32_t k = base + lane;
    if (k >= a.n_active) continue;
    const uint32_t w = a.active[k];
    const uint32_t start = w % a.v_num, replica = w / a.v_num;
    PathBuf pb{a.arena + (uint64_t)k * a.slot_len, 0, a.slot_len, s_path + threadIdx.x};
    bool ok = path_push(a, pb, start);
    Corr c;
    corr_init(c);
    uint32_t cur = start;
    uint64_t b = a.row_ptr[cur];
    uint32_t deg = (uint32_t)(a.row_ptr[cur + 1] - b);
    uint32_t step = 0, iter = 0, cnt_cur = 1;
    uint64_t bloom = bloom_bit(start);
    uint64_t di = 0, di_end = 0, dp = 0, dp_end = 0;
    if (INJ) {
      di = a.inj_idx_off[k];
      di_end = a.inj_idx_off[k + 1];
      dp = a.inj_p_off[k];
      dp_end = a.inj_p_off[k + 1];
    }
    while (ok) {
      if (deg == 0) break;
      uint32_t r;
      double p = 0.0;
      if (INJ) {
        if (di >= di_end) {
          set_error(a.err, kErrDrawsExhausted);
          break;
        }
        r = a.inj_idx[di++];
        if (r >= deg) {
          set_error(a.err, kErrDrawsExhausted);
          break;
        }
      } else {
        walk_draw(a.seed, start, a.round, iter, replica, deg, r, p);
        if (WEIGHTED) {
          // alias draw: keep slot r with probability prob[r], else take its
          // alias; the coin comes from a second Philox block of this iteration.
          uint4 o = philox4x32_10(make_uint4(start, a.round, iter, replica ^ 0x80000000u),
                                  make_uint2((uint32_t)a.seed, (uint32_t)(a.seed >> 32)));
          float u = (float)(o.x >> 8) * (1.0f / 16777216.0f);
          if (u >= a.alias_prob[b + r]) r = a.alias_idx[b + r];
        }
      }
      iter++;
      if (iter > kWalkIterLimit) {
        set_error(a.err, kErrWalkLimit);
        break;
      }
      if (deg == 2 && (FUSED ? a.wadj[b].x : a.adj[b].x) == cur) break;
      uint2 cand;
      uint64_t bd;
      uint32_t dd;
      if constexpr (FUSED) {
        const uint4 e = a.wadj[b + r];
        cand = make_uint2(e.x, e.y);
        bd = e.z;
        dd = e.w;
      } else {
        cand = a.adj[b + r];
      }
      if (step == 0 && cand.x == cur) continue;
      if (INJ) {
        if (dp >= dp_end) {
          set_error(a.err, kErrDrawsExhausted);
          break;
        }
        p = a.inj_p[dp++];
      }
      const int cn = (int)__uint_as_float(cand.y);
      const uint32_t dst = cand.x;
      if constexpr (!FUSED) {
        bd = a.row_ptr[dst];
        dd = (uint32_t)(a.row_ptr[dst + 1] - bd);
      }
      const int sd = (int)deg, ddi = (int)dd;
      const int mx = sd > ddi ? sd : ddi, mn = sd < ddi ? sd : ddi;
      const bool trace = trace_test(sd, cn, mx, mn, p);
      my_tr += trace;
      // forward token
      step++;
      uint32_t fi;
      if (dst == cur) fi = cnt_cur;
      else if (bloom & bloom_bit(dst)) fi = count_in_walk(pb, dst);
      else fi = 0;
      if (!path_push(a, pb, dst)) { ok = false; break; }
      bloom |= bloom_bit(dst);
      if (dst == cur) cnt_cur++;
      if (corr_step(c, fi, a.corr_tab, s_ser, step, a.min_len)) break;
      if (trace) {
        step++;
        if (!path_push(a, pb, cur)) { ok = false; break; }
        const bool stop = corr_step(c, cnt_cur, a.corr_tab, s_ser, step, a.min_len);
        cnt_cur++;
        if (stop) break;
      } else {
        if (dst != cur) cnt_cur = fi + 1;
        cur = dst;
        b = bd;
        deg = dd;
      }
    }
    my_it += iter;
    my_tok += pb.len;
    my_long += pb.cap > a.slot_len;
    a.sent_ptr[k] = (uint64_t)(pb.p - a.arena);
    a.sent_len[k] = pb.len;
  }
  __syncwarp();
  for (int o = 16; o > 0; o >>= 1) {
    my_tok += __shfl_down_sync(0xffffffffu, my_tok, o);
    my_tr += __shfl_down_sync(0xffffffffu, my_tr, o);
    my_it += __shfl_down_sync(0xffffffffu, my_it, o);
    my_long += __shfl_down_sync(0xffffffffu, my_long, o);
  }
  if (lane == 0) {
    if (my_tok) atomicAdd(&a.stats[0], my_tok);
    if (my_tr) atomicAdd(&a.stats[1], my_tr);
    if (my_it) atomicAdd(&a.stats[2], my_it);
    if (my_long) atomicAdd(&a.stats[3], my_long);
  }
}

// Memory skeleton of a finished walk round, for its attainable-rate ceiling:
// every walker of the round emits as many tokens as its walk had; a token is
// a dependent uniform-neighbour gather (the candidate's adjacency entry, then
// the neighbour's row_ptr pair; with FUSED the candidate's walker entry alone,
// as the walker reads it) with probability gather_frac (the round's
// forward steps per token), else a repeat of the current vertex (the return
// token of a trace, which loads nothing).  Same block size and warp claims
// as k_walk, at its own full residency (no shared memory and few registers
// give 8 blocks per SM, where k_walk holds 3); no FP64, no trace test, no
// revisit counts and no visit counters.  Tokens go to a scratch buffer at
// the walk's offsets.
template <bool FUSED>
__global__ void __launch_bounds__(kWalkThreads, 3)
    k_walk_skeleton(const uint64_t *__restrict__ row_ptr, const uint2 *__restrict__ adj,
                    const uint4 *__restrict__ wadj, uint32_t v_num,
                    uint32_t n_active, const uint32_t *__restrict__ active, const uint64_t *__restrict__ sent_ptr,
                    const uint32_t *__restrict__ sent_len, uint32_t gather_frac, uint32_t *out,
                    unsigned int *next_walker) {
  const uint32_t lane = threadIdx.x & 31;
  for (;;) {
    __syncwarp();
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(next_walker, 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n_active) break;
    const uint32_t k = base + lane;
    if (k >= n_active) continue;
    uint32_t cur = active[k] % v_num;
    uint64_t b = row_ptr[cur];
    uint32_t deg = (uint32_t)(row_ptr[cur + 1] - b);
    uint32_t *o = out + sent_ptr[k];
    const uint32_t len = sent_len[k];
    if (len) o[0] = cur;
    uint32_t h = k * 0x9E3779B1u;
    for (uint32_t t = 1; t < len; t++) {
      h = h * 1664525u + 1013904223u;
      if (deg && (h >> 8) < (gather_frac >> 8)) {
        const uint32_t r = (uint32_t)(((uint64_t)(h ^ (h >> 13)) * deg) >> 32);
        if constexpr (FUSED) {
          const uint4 e = wadj[b + r];
          cur = e.x;
          b = e.z;
          deg = e.w;
        } else {
          const uint32_t dst = adj[b + r].x;
          b = row_ptr[dst];
          deg = (uint32_t)(row_ptr[dst + 1] - b);
          cur = dst;
        }
      }
      o[t] = cur;
    }
  }
}

}  // namespace felog
