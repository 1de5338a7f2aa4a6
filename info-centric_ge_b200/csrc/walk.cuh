// Walker engine: one lane per walker, persistent grid, walkers claimed from a
// global counter so uneven walks keep every lane busy.
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
//
// Tokens go to a per-walker slot of slot_len tokens; a walk that outgrows it
// moves to a doubled chunk of the spill arena.  fi lookups use a 64-bit
// Bloom word per walker (no scan for first visits) and a scan of the walk's
// own tokens otherwise; the return step of a trace uses a running count of
// the current vertex.
#pragma once

#include "common.cuh"

namespace felog {

struct WalkArgs {
  const uint64_t *row_ptr;
  const uint2 *adj;
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
  unsigned int *next_walker;     // kWalkClaimers claim counters (walker i + kWalkClaimers j)
  unsigned long long *stats;     // [tokens, traces, iterations, long]
  int *err;
};

constexpr uint32_t kWalkClaimers = 64;  // claim counters: walkers i, i + 64, i + 128, ... share counter i

struct Corr {
  double H, EH, ES, EHS, EHH, ESS, R, S;  // N == S throughout (both count tokens)
};

__device__ __forceinline__ void corr_init(Corr &c) {
  c.H = 0.0; c.EH = 0.0; c.ES = 1.0; c.EHS = 0.0; c.EHH = 0.0; c.ESS = 1.0; c.R = 1.0; c.S = 1.0;
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

// Correlation::iterate with step_k = 1 (walk.hpp:309-366).
__device__ __forceinline__ void corr_iterate(Corr &c, uint32_t fi_u, const double *__restrict__ tab) {
  const double Sn = c.S;
  const double Snp1 = __dadd_rn(Sn, 1.0);
  const double fi = (double)fi_u;
  const uint32_t S_u = (uint32_t)Sn;
  const double t = (tab && S_u <= (uint32_t)kCorrTableS) ? __ldg(&tab[corr_tab_index(S_u, fi_u)]) : corr_t(Sn, fi);
  const double H1 = __ddiv_rn(__dsub_rn(__dmul_rn(Sn, c.H), t), Snp1);
  const double Np1 = Snp1;  // N + 1 with N == S
  const double EH = __dadd_rn(c.EH, __ddiv_rn(__dsub_rn(H1, c.EH), Np1));
  const double ES = __dadd_rn(c.ES, __ddiv_rn(__dsub_rn(Snp1, c.ES), Np1));
  const double EHS = __dadd_rn(c.EHS, __ddiv_rn(__dsub_rn(__dmul_rn(H1, Snp1), c.EHS), Np1));
  const double EHH = __dadd_rn(c.EHH, __ddiv_rn(__dsub_rn(__dmul_rn(H1, H1), c.EHH), Np1));
  const double ESS = __dadd_rn(c.ESS, __ddiv_rn(__dsub_rn(__dmul_rn(Snp1, Snp1), c.ESS), Np1));
  const double DH = __dsub_rn(EHH, __dmul_rn(EH, EH));
  const double DS = __dsub_rn(ESS, __dmul_rn(ES, ES));
  const double ex = __dsub_rn(EHS, __dmul_rn(EH, ES));
  c.R = ex == 0.0 ? 0.0 : __ddiv_rn(ex, __dsqrt_rn(__dmul_rn(DH, DS)));
  c.H = H1; c.EH = EH; c.ES = ES; c.EHS = EHS; c.EHH = EHH; c.ESS = ESS; c.S = Snp1;
}

__device__ __forceinline__ bool corr_stop(const Corr &c, uint32_t step, uint32_t min_len) {
  return step > min_len && (__dmul_rn(c.R, c.R) < 0.999 || c.R < 0.0);
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

struct PathBuf {
  uint32_t *p;    // token storage of this walk
  uint32_t len;
  uint32_t cap;
};

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
  pb.p[pb.len++] = v;
  atomicAdd(&a.visit_freq[v], 1u);
  return true;
}

// INJ: parity mode with injected draws; WEIGHTED: alias-table candidates.
template <bool INJ, bool WEIGHTED>
__global__ void __launch_bounds__(256, 3) k_walk(WalkArgs a) {
  unsigned long long my_tok = 0, my_tr = 0, my_it = 0, my_long = 0;
  // walkers are claimed through kWalkClaimers counters so that claims do not
  // serialize on one address
  const uint32_t claimer = (blockIdx.x * blockDim.x + threadIdx.x) % kWalkClaimers;
  for (;;) {
    const uint32_t k = claimer + kWalkClaimers * atomicAdd(&a.next_walker[claimer], 1u);
    if (k >= a.n_active) break;
    const uint32_t w = a.active[k];
    const uint32_t start = w % a.v_num, replica = w / a.v_num;
    PathBuf pb{a.arena + (uint64_t)k * a.slot_len, 0, a.slot_len};
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
      if (deg == 2 && a.adj[b].x == cur) break;
      const uint2 cand = a.adj[b + r];
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
      const uint64_t bd = a.row_ptr[dst];
      const uint32_t dd = (uint32_t)(a.row_ptr[dst + 1] - bd);
      const int sd = (int)deg, ddi = (int)dd;
      const int mx = sd > ddi ? sd : ddi, mn = sd < ddi ? sd : ddi;
      const double p_accept = __ddiv_rn(__dmul_rn(__ddiv_rn(1.0, (double)(sd - cn)), (double)mx), (double)mn);
      const bool trace = tanh(p_accept) <= p;
      my_tr += trace;
      // forward token
      step++;
      uint32_t fi;
      if (dst == cur) fi = cnt_cur;
      else if (bloom & bloom_bit(dst)) fi = count_in_path(pb.p, pb.len, dst);
      else fi = 0;
      if (!path_push(a, pb, dst)) { ok = false; break; }
      bloom |= bloom_bit(dst);
      if (dst == cur) cnt_cur++;
      corr_iterate(c, fi, a.corr_tab);
      if (corr_stop(c, step, a.min_len)) break;
      if (trace) {
        step++;
        if (!path_push(a, pb, cur)) { ok = false; break; }
        corr_iterate(c, cnt_cur, a.corr_tab);
        cnt_cur++;
        if (corr_stop(c, step, a.min_len)) break;
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
  atomicAdd(&a.stats[0], my_tok);
  atomicAdd(&a.stats[1], my_tr);
  atomicAdd(&a.stats[2], my_it);
  atomicAdd(&a.stats[3], my_long);
}

}  // namespace felog
