/*
 * felog_oracle.c - CPU restatement of FeLoG's graph-embedding hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see felog_oracle.h).  Plain C, single-threaded,
 * written for small cases.  Floating-point expressions keep the reference's
 * operation order; a*b+c is not contracted (built with -ffp-contract=off)
 * except where the reference's CUDA kernels fuse it, which is written out
 * with fmaf().
 */
#include "felog_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ CSR */

/* graph.hpp:741-772 (undirected doubling, e then its transpose),
 * graph.hpp:781-785 (out-degree), graph.hpp:531-575 (bucket by src in order). */
int orc_build_csr(const orc_edge12 *edges, uint64_t n, uint32_t v_num, int undirected, orc_csr *out) {
  uint64_t m = undirected ? 2 * n : n;
  memset(out, 0, sizeof(*out));
  out->v_num = v_num;
  out->e_num = m;
  out->row_ptr = (uint64_t *)calloc((size_t)v_num + 1, sizeof(uint64_t));
  out->nbr = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
  out->data = (float *)malloc((m ? m : 1) * sizeof(float));
  uint64_t *fill = (uint64_t *)calloc((size_t)v_num + 1, sizeof(uint64_t));
  if (!out->row_ptr || !out->nbr || !out->data || !fill) return -1;
  for (uint64_t i = 0; i < m; i++) {
    const orc_edge12 *e = &edges[undirected ? i / 2 : i];
    uint32_t src = (undirected && (i & 1)) ? e->dst : e->src;
    if (src >= v_num) { free(fill); return -2; }
    out->row_ptr[src + 1]++;
  }
  for (uint32_t v = 0; v < v_num; v++) out->row_ptr[v + 1] += out->row_ptr[v];
  for (uint32_t v = 0; v < v_num; v++) fill[v] = out->row_ptr[v];
  for (uint64_t i = 0; i < m; i++) {
    const orc_edge12 *e = &edges[undirected ? i / 2 : i];
    int t = undirected && (i & 1);
    uint32_t src = t ? e->dst : e->src, dst = t ? e->src : e->dst;
    uint64_t pos = fill[src]++;
    out->nbr[pos] = dst;
    out->data[pos] = e->data;
  }
  free(fill);
  return 0;
}

void orc_free_csr(orc_csr *c) {
  free(c->row_ptr);
  free(c->nbr);
  free(c->data);
  memset(c, 0, sizeof(*c));
}

/* ---------------------------------------------------------- Correlation */

/* SetProperty(0,1,0,1,0,0,1,1,1) at the first visit, walk.hpp:928-933 */
void orc_corr_init(orc_corr *c) {
  c->Hn = 0.0; c->Sn = 1.0; c->EnH = 0.0; c->EnS = 1.0; c->EnHS = 0.0;
  c->EnHH = 0.0; c->EnSS = 1.0; c->N = 1.0; c->R = 1.0;
}

/* Correlation::iterate with step_k = 1, walk.hpp:296-366 */
void orc_corr_iterate(orc_corr *c, double fi) {
  const double step_k = 1.0;
  double Sn = c->Sn, Hn = c->Hn;
  /* SnSn_div_Snp1Snp1, walk.hpp:296-301 */
  double Snp1a = Sn + step_k;
  double ss = pow(Sn / Snp1a, Sn) * pow(1.0 / Snp1a, step_k);
  double t;
  if (fi == 0.0) {
    t = log2(ss);
  } else {
    /* FjFj_div_FiFi, walk.hpp:303-307 */
    double fj = fi + step_k;
    double ff = pow(fj / fi, fi) * pow(fj, step_k);
    t = log2(ss * ff);
  }
  double Hnp1 = (Sn * Hn - t) / (Sn + step_k); /* walk.hpp:314 */
  double Snp1 = c->Sn + step_k;
  double Np1 = c->N + 1.0;
  double EH = c->EnH + (Hnp1 - c->EnH) / Np1; /* iterateEX, walk.hpp:322-324 */
  double ES = c->EnS + (Snp1 - c->EnS) / Np1;
  double EHS = c->EnHS + (Hnp1 * Snp1 - c->EnHS) / Np1;
  double EHH = c->EnHH + (Hnp1 * Hnp1 - c->EnHH) / Np1;
  double ESS = c->EnSS + (Snp1 * Snp1 - c->EnSS) / Np1;
  double DH = EHH - EH * EH;
  double DS = ESS - ES * ES;
  double ex = EHS - EH * ES;
  c->R = ex == 0.0 ? 0.0 : ex / sqrt(DH * DS);
  c->Hn = Hnp1; c->Sn = Snp1; c->EnH = EH; c->EnS = ES; c->EnHS = EHS;
  c->EnHH = EHH; c->EnSS = ESS; c->N = Np1;
}

/* walk.hpp:945-951, :1056-1062: stop once step > minLength and R^2 < 0.999 or R < 0 */
int orc_corr_stop(const orc_corr *c, uint32_t step, uint32_t min_len) {
  if (step > min_len) {
    if (pow(c->R, 2) < 0.999 || c->R < 0) return 1;
  }
  return 0;
}

/* ---------------------------------------------------------------- RNG */

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline uint32_t mulhi64_u32(uint64_t r, uint32_t n) {
  return (uint32_t)(((unsigned __int128)r * n) >> 64);
}

void orc_walk_draw(uint64_t seed, uint32_t start, uint32_t round, uint32_t iter, uint32_t replica,
                   uint32_t deg, uint32_t *index, double *p) {
  uint32_t ctr[4] = {start, round, iter, replica};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  orc_philox4x32_10(ctr, key, o);
  *index = mulhi64_u32(((uint64_t)o[3] << 32) | o[0], deg);
  *p = (double)((((uint64_t)o[1] << 32) | o[2]) >> 11) * (1.0 / 9007199254740992.0);
}

/* --------------------------------------------------------------- walk */

static uint64_t count_in(const uint32_t *path, uint64_t n, uint32_t v) {
  uint64_t c = 0;
  for (uint64_t i = 0; i < n; i++) c += path[i] == v;
  return c;
}

int orc_walk_round(const orc_csr *g, uint32_t walker_num, const uint8_t *stop_flags, uint32_t min_len,
                   uint64_t seed, uint32_t round, const orc_draws *inj, uint32_t *tokens,
                   uint64_t tok_cap, uint64_t *sent_off, uint32_t *sent_walker, orc_walk_stats *st) {
  const uint32_t V = g->v_num;
  memset(st, 0, sizeof(*st));
  uint64_t ntok = 0, k = 0;
  sent_off[0] = 0;
  for (uint32_t w = 0; w < walker_num; w++) {
    uint32_t start = w % V; /* walk.hpp:519-527 */
    if (stop_flags && stop_flags[start]) continue; /* walk.hpp:570 */
    uint32_t replica = w / V;
    uint64_t di = 0, dp = 0; /* consumed injected draws */
    uint32_t iter = 0;
    uint32_t *path = tokens + ntok;
    uint64_t len = 0;
    if (ntok + 1 > tok_cap) return -1;
    path[len++] = start; /* step-0 footprint, walk.hpp:691-699 */
    orc_corr c;
    orc_corr_init(&c); /* first visit: fi = 0 consumed, walk.hpp:926-933 */
    uint32_t cur = start, step = 0;
    for (;;) {
      uint64_t b = g->row_ptr[cur];
      uint32_t deg = (uint32_t)(g->row_ptr[cur + 1] - b);
      if (deg == 0) break; /* walk.hpp:964-969 */
      uint32_t r;
      double p = 0.0;
      if (inj) {
        if (inj->idx_off[k] + di >= inj->idx_off[k + 1]) return -2;
        r = inj->idx[inj->idx_off[k] + di++];
      } else {
        orc_walk_draw(seed, start, round, iter, replica, deg, &r, &p);
      }
      iter++;
      st->n_iterations++;
      if (iter > (1u << 24)) return -3; /* same limit as the device walker */
      if (deg == 2 && g->nbr[b] == cur) break;               /* walk.hpp:977-979 */
      uint64_t cand = b + r;
      if (step == 0 && g->nbr[cand] == cur) continue;        /* walk.hpp:981-983 */
      int cn = (int)g->data[cand];                          /* walk.hpp:997 */
      if (inj) {
        if (inj->p_off[k] + dp >= inj->p_off[k + 1]) return -2;
        p = inj->p[inj->p_off[k] + dp++];
      }
      int sd = (int)deg;
      uint32_t dst = g->nbr[cand];
      int dd = (int)(g->row_ptr[dst + 1] - g->row_ptr[dst]);
      int mx = sd > dd ? sd : dd, mn = sd < dd ? sd : dd;
      double p_accept = (1 / ((double)(sd - cn)) * ((double)mx) / mn); /* walk.hpp:1010 */
      double p_norm = tanh(p_accept);
      int trace = p_norm <= p;                                        /* walk.hpp:1015 */
      st->n_traces += trace;
      step++;
      if (ntok + len + 1 > tok_cap) return -1;
      path[len++] = dst;                                              /* walk.hpp:1038-1041 */
      orc_corr_iterate(&c, (double)count_in(path, len - 1, dst));
      if (orc_corr_stop(&c, step, min_len)) break;
      if (trace) {                                                    /* walk.hpp:1063-1094 */
        step++;
        if (ntok + len + 1 > tok_cap) return -1;
        path[len++] = cur;
        orc_corr_iterate(&c, (double)count_in(path, len - 1, cur));
        if (orc_corr_stop(&c, step, min_len)) break;
      } else {
        cur = dst;
      }
    }
    ntok += len;
    if (len > 64) st->n_long++;
    sent_off[k + 1] = ntok;
    if (sent_walker) sent_walker[k] = w;
    k++;
  }
  st->n_sentences = k;
  st->n_tokens = ntok;
  return 0;
}

/* walk.hpp:754-787 */
double orc_round_kl(const uint32_t *deg, const uint64_t *freq, uint32_t v_num) {
  uint64_t words_sum = 0, degree_sum = 0;
  for (uint32_t i = 0; i < v_num; i++) {
    words_sum += freq[i];
    degree_sum += deg[i];
  }
  double h = 0.0;
  for (uint32_t i = 0; i < v_num; i++) {
    double pi = (double)deg[i] / degree_sum;
    double qi = (double)freq[i] / words_sum;
    h += pi * (log(pi) - log(qi));
  }
  return h;
}

float orc_lr(float initial, float decay, int r) { return initial * expf(-decay * r); }

/* ------------------------------------------------------------ trainer */

typedef struct {
  long long cn;
  uint32_t v;
} vw;

static int vw_cmp(const void *a, const void *b) {
  const vw *x = (const vw *)a, *y = (const vw *)b;
  if (x->cn != y->cn) return x->cn < y->cn ? 1 : -1;
  return x->v < y->v ? -1 : (x->v > y->v ? 1 : 0); /* stable: keeps id order */
}

int orc_vocab(const uint32_t *deg, uint32_t v_num, long long min_count, uint32_t *vocab_vertex,
              long long *vocab_cn, uint32_t *id2offset, long long *vocab_size, long long *train_words) {
  vw *a = (vw *)malloc(sizeof(vw) * (v_num ? v_num : 1));
  if (!a) return -1;
  for (uint32_t v = 0; v < v_num; v++) {
    a[v].cn = deg[v];
    a[v].v = v;
  }
  qsort(a, v_num, sizeof(vw), vw_cmp);
  long long size = v_num, tw = 0;
  for (uint32_t i = 0; i < v_num; i++) { /* SortVocab, word2vec.cu:740-748 */
    if (a[i].cn < min_count && i != 0) size--;
    else tw += a[i].cn;
  }
  for (uint32_t v = 0; v < v_num; v++) id2offset[v] = 0xFFFFFFFFu;
  for (long long i = 0; i < size; i++) {
    vocab_vertex[i] = a[i].v;
    vocab_cn[i] = a[i].cn;
    id2offset[a[i].v] = (uint32_t)i;
  }
  *vocab_size = size;
  *train_words = tw;
  free(a);
  return 0;
}

void orc_unigram_table(const long long *cn, long long vocab_size, int32_t *table, int64_t table_size) {
  double train_words_pow = 0, d1, power = 0.75;
  long long a, i;
  for (a = 0; a < vocab_size; a++) train_words_pow += pow((double)cn[a], power);
  i = 0;
  d1 = pow((double)cn[i], power) / train_words_pow;
  for (a = 0; a < table_size; a++) {
    table[a] = (int32_t)i;
    if (a / (double)table_size > d1) {
      i++;
      d1 += pow((double)cn[i < vocab_size ? i : vocab_size - 1], power) / train_words_pow;
    }
    if (i >= vocab_size) i = vocab_size - 1;
  }
}

int orc_subsample_thresholds(const long long *cn, long long vocab_size, double sample,
                             long long train_words, uint16_t *thr) {
  if (sample <= 0.0 || train_words <= 0) return 0;
  const double stw = sample * (double)train_words;
  if (stw <= 0.0 || vocab_size <= 0) return 0;
  for (long long i = 0; i < vocab_size; i++) {
    long long count = cn[i];
    if (count <= 0) {
      thr[i] = 65535;
      continue;
    }
    double prob = (sqrt(count / stw) + 1.0) * (stw / (double)count);
    if (prob > 1.0) prob = 1.0;
    else if (prob < 0.0) prob = 0.0;
    thr[i] = prob >= 1.0 ? 65535 : (uint16_t)(prob * 65535.0 + 0.5);
  }
  return 1;
}

void orc_exp_table(float *t) {
  for (int i = 0; i < 1000; i++) {
    t[i] = expf((i / (float)1000 * 2 - 1) * 6);
    t[i] = t[i] / (t[i] + 1);
  }
}

/* FastRandomState, word2vec.cu:134-152 */
typedef struct {
  unsigned long long state;
} fast_rng;
static uint32_t rng_next32(fast_rng *r) {
  r->state = r->state * 25214903917ULL + 11ULL;
  return (uint32_t)(r->state >> 16);
}

int orc_plan_batches(const uint32_t *tokens, const uint64_t *sent_off, uint64_t n_corpus_sent,
                     const uint32_t *id2offset, const uint16_t *thr, int use_thr, const int32_t *table,
                     int64_t table_size, long long vocab_size, int negative, int rank, orc_plan_out *out) {
  fast_rng rng;
  unsigned long long seed = 0x9E3779B97F4A7C15ULL ^ (((unsigned long long)rank + 1ULL) << 1) ^ 0x2ULL;
  rng.state = seed ? seed : 1ULL;
  uint64_t ci = 0, total = 0, s_out = 0, nb = 0;
  long long word = 0;
  out->words_considered = 0;
  out->sent_start[0] = 0;
  while (ci < n_corpus_sent) {
    uint64_t batch_base = total;
    int cnt = 0;
    out->batch_first[nb] = s_out;
    while (cnt < 15000 && ci < n_corpus_sent) { /* word2vec.cu:1193-1235 */
      int temp = 0;
      for (uint64_t t = sent_off[ci]; t < sent_off[ci + 1]; t++) {
        uint32_t off = id2offset[tokens[t]];
        if (off == 0xFFFFFFFFu) continue; /* out of vocabulary */
        word = (long long)off;
        out->words_considered++;
        if (word == 0) break;
        if (use_thr) {
          uint16_t keep = thr[word];
          if (keep < 65535) {
            uint16_t r16 = (uint16_t)(rng_next32(&rng) >> 16);
            if (r16 > keep) continue;
          }
        }
        if (total >= out->sen_cap) return -1;
        out->sen[total++] = (int32_t)word;
        temp++;
        if (temp >= 1000) break;
      }
      cnt++;
      s_out++;
      out->sent_start[s_out] = total;
      ci++;
      if (total - batch_base >= (uint64_t)(15000 - 1) * 20) break;
    }
    if (cnt == 0) break;
    for (int i = 0; i < cnt * negative; i++) { /* word2vec.cu:1240-1248 */
      uint32_t randd = rng_next32(&rng);
      int32_t ts = table[randd % (uint64_t)table_size];
      out->negs[(out->batch_first[nb]) * negative + i] =
          ts == 0 ? (int32_t)(randd % (uint64_t)(vocab_size - 1)) + 1 : ts;
    }
    nb++;
  }
  out->batch_first[nb] = s_out;
  out->n_sentences = s_out;
  out->n_batches = nb;
  out->n_sen = total;
  return (int)s_out;
}

/* dot product in skip_gram_kernel's order (FSIZE = dim / 2, word2vec.cu:510-518) */
static float sg_dot(const float *x, const float *y, int dim) {
  int fs = dim / 2;
  float f[512];
  for (int t = 0; t < fs; t++) f[t] = x[t] * y[t];
  for (int t = fs; t < dim; t++) f[t % fs] = fmaf(x[t], y[t], f[t % fs]);
  for (int i = fs / 2; i > 0; i /= 2)
    for (int t = 0; t < i; t++) f[t] += f[i + t];
  return f[0];
}

static float sg_gradient(float f, int label, const float *exp_table, float alpha) {
  if (f > 6) return (label - 1) * alpha;
  if (f < -6) return (label - 0) * alpha;
  return (label - exp_table[(int)((f + 6) * (1000 / 6 / 2))]) * alpha;
}

void orc_skipgram_batch(float *syn0, float *syn1, const float *exp_table, const int32_t *table,
                        int64_t table_size, long long vocab_size, const int32_t *sen,
                        const uint64_t *sent_start, uint64_t first_sentence, uint64_t n_sentences,
                        int window, int dim, int negative, float alpha) {
  float neu1e[512];
  for (uint64_t blk = 0; blk < n_sentences; blk++) {
    uint64_t s = first_sentence + blk;
    long long sidx_s = (long long)sent_start[s], sidx_e = (long long)sent_start[s + 1];
    unsigned long next_random = (unsigned long)blk; /* blockIdx.x within the batch */
    for (long long pos = sidx_s; pos < sidx_e; pos++) {
      int word = sen[pos];
      if (word == -1) continue;
      next_random = next_random * (unsigned long)2514903917 + 11;
      int b = (int)(next_random % (unsigned long)window);
      for (int a = b; a < window * 2 + 1 - b; a++) {
        if (a == window) continue;
        long long c = pos - window + a;
        if (c < sidx_s || c >= sidx_e) continue;
        int last_word = sen[c];
        if (last_word == -1) continue;
        float *x = syn0 + (long long)last_word * dim;
        for (int t = 0; t < dim; t++) neu1e[t] = 0;
        for (int d = 0; d < negative + 1; d++) {
          int target, label;
          if (d == 0) {
            target = word;
            label = 1;
          } else {
            next_random = next_random * (unsigned long)25214903917 + 11;
            target = table[(next_random >> 16) % (unsigned long)table_size];
            if (target == 0) target = (int)(next_random % (unsigned long)(vocab_size - 1) + 1);
            if (target == word) continue;
            label = 0;
          }
          float *y = syn1 + (long long)target * dim;
          float f = sg_dot(x, y, dim);
          float g = sg_gradient(f, label, exp_table, alpha);
          for (int t = 0; t < dim; t++) {
            neu1e[t] = fmaf(g, y[t], neu1e[t]);
            y[t] += g * x[t];
          }
        }
        for (int t = 0; t < dim; t++) x[t] += neu1e[t];
      }
    }
  }
}

/* __sgNegReuse (word2vec.cu:368-440) restated with a true dot product: per
 * sentence K negatives drawn by the host plan, the full window (no shrink), and
 * for every (center, context) pair the positive (the center word) and the
 * negatives not equal to it.  The reference's warp reduction
 * (reduceInWarp, word2vec.cu:214-219, __shfl_sync(f, i) reads lane i) does not
 * form a dot product; here each score is the skip-gram tree dot.  Targets are
 * taken in the order positive, negative 0..K-1, each scored against the rows
 * as they are at that point (targets with distinct rows do not see each
 * other's updates, as in the reference where all K + 1 warps score before
 * they update); sigma is the expTable lookup (the reference recomputes the
 * same quantized sigmoid with exp). */
void orc_negreuse_batch(float *syn0, float *syn1, const float *exp_table, const int32_t *sen,
                        const uint64_t *sent_start, uint64_t first_sentence, uint64_t n_sentences,
                        const int32_t *negs, int window, int dim, int negative, float alpha) {
  float neu1e[512];
  for (uint64_t blk = 0; blk < n_sentences; blk++) {
    uint64_t s = first_sentence + blk;
    long long ss = (long long)sent_start[s], se = (long long)sent_start[s + 1];
    const int32_t *neg = negs + s * (uint64_t)negative;
    for (long long pos = ss; pos < se; pos++) {
      int word = sen[pos];
      if (word == -1) continue;
      for (int a = 0; a < window * 2 + 1; a++) {
        if (a == window) continue;
        long long c = pos - window + a;
        if (c < ss || c >= se || sen[c] == -1) continue;
        float *x = syn0 + (long long)sen[c] * dim;
        for (int t = 0; t < dim; t++) neu1e[t] = 0;
        for (int d = 0; d <= negative; d++) {
          int target = d == 0 ? word : neg[d - 1];
          if (d > 0 && target == word) continue;
          int label = d == 0 ? 1 : 0;
          float *y = syn1 + (long long)target * dim;
          float f = sg_dot(x, y, dim);
          float g = sg_gradient(f, label, exp_table, alpha);
          for (int t = 0; t < dim; t++) {
            neu1e[t] = fmaf(g, y[t], neu1e[t]);
            y[t] += g * x[t];
          }
        }
        for (int t = 0; t < dim; t++) x[t] += neu1e[t];
      }
    }
  }
}

void orc_cbow_batch(float *syn0, float *syn1, const float *exp_table, const int32_t *table,
                    int64_t table_size, long long vocab_size, const int32_t *sen,
                    const uint64_t *sent_start, uint64_t first_sentence, uint64_t n_sentences,
                    int window, int dim, int negative, float alpha) {
  float neu1[512], neu1e[512];
  for (uint64_t blk = 0; blk < n_sentences; blk++) {
    uint64_t s = first_sentence + blk;
    long long ss = (long long)sent_start[s], se = (long long)sent_start[s + 1];
    unsigned long next_random = (unsigned long)blk;
    for (long long pos = ss; pos < se; pos++) {
      int word = sen[pos];
      if (word == -1) continue;
      for (int t = 0; t < dim; t++) neu1[t] = neu1e[t] = 0;
      next_random = next_random * (unsigned long)2514903917 + 11;
      int b = (int)(next_random % (unsigned long)window);
      int cw = 0;
      for (int a = b; a < window * 2 + 1 - b; a++) {
        if (a == window) continue;
        long long c = pos - window + a;
        if (c < ss || c >= se || sen[c] == -1) continue;
        const float *x = syn0 + (long long)sen[c] * dim;
        for (int t = 0; t < dim; t++) neu1[t] += x[t];
        cw++;
      }
      if (!cw) continue;
      for (int t = 0; t < dim; t++) neu1[t] /= cw;
      for (int d = 0; d < negative + 1; d++) {
        int target, label;
        if (d == 0) {
          target = word;
          label = 1;
        } else {
          next_random = next_random * (unsigned long)25214903917 + 11;
          target = table[(next_random >> 16) % (unsigned long)table_size];
          if (target == 0) target = (int)(next_random % (unsigned long)(vocab_size - 1) + 1);
          if (target == word) continue;
          label = 0;
        }
        float *y = syn1 + (long long)target * dim;
        float f = sg_dot(neu1, y, dim);
        float g = sg_gradient(f, label, exp_table, alpha);
        for (int t = 0; t < dim; t++) {
          neu1e[t] = fmaf(g, y[t], neu1e[t]);
          y[t] += g * neu1[t];
        }
      }
      for (int a = b; a < window * 2 + 1 - b; a++) {
        if (a == window) continue;
        long long c = pos - window + a;
        if (c < ss || c >= se || sen[c] == -1) continue;
        float *x = syn0 + (long long)sen[c] * dim;
        for (int t = 0; t < dim; t++) x[t] += neu1e[t];
      }
    }
  }
}

/* ---- BF16 storage form (this project's precision form; no reference
 * counterpart).  Rows 0..n_hot-1 are FP32 master rows updated by addition;
 * rows n_hot.. are BF16 bit patterns, read as FP32 and written back as
 * SR(value + update): 16 random bits added below the BF16 mantissa, then
 * truncation.  The bits of one (pair, slot, lane) come from the pair's key:
 *   kp     = H(seed ^ ((u32)s * 0x9E3779B1 + pair * 0x85EBCA77))
 *   x      = kp ^ (lane * 0xC2B2AE3D)
 *   word k = (x + slot * 0x27D4EB2F + k * 0x165667B1) * 0x9E3779B1 (mod 2^32),
 *            one per two values: its low 16 bits round the lane's value 2k,
 *            its high 16 bits value 2k + 1
 * (s: sentence index in the plan; pair: index of the (center, context) pair in
 * the sentence, or of the center for CBOW)  * where H is a multiply / xor-shift mixer, slot = d (target index, 0 is the
 * positive) for syn1 rows and 256 (+ window position a for CBOW) for syn0
 * rows, and the lane's values j = 0, 1, 2, ... are the logical dimensions
 * l, l + 32, l + 64, ... of lane l.  Everything else is skip_gram_kernel / cbow_kernel
 * (word2vec.cu:442-646) exactly as in orc_skipgram_batch / orc_cbow_batch. */
static uint32_t sr_h(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}
uint32_t orc_lane_key(uint32_t seed, uint64_t s, uint32_t pair, uint32_t lane) {
  return sr_h(seed ^ ((uint32_t)s * 0x9E3779B1u + pair * 0x85EBCA77u)) ^ (lane * 0xC2B2AE3Du);
}
static float bf_to_f(uint16_t h) {
  uint32_t b = (uint32_t)h << 16;
  float f;
  memcpy(&f, &b, 4);
  return f;
}
static uint16_t f_to_bf_sr(float v, uint32_t r16) {
  uint32_t b;
  memcpy(&b, &v, 4);
  return (uint16_t)((b + r16) >> 16);
}
typedef struct {
  float *f32;
  uint16_t *bf;
  long long n_hot;
  int dim;
} mixed_rows;
static void mr_get(const mixed_rows *m, long long row, float *out) {
  if (row < m->n_hot) {
    memcpy(out, m->f32 + row * m->dim, sizeof(float) * m->dim);
  } else {
    const uint16_t *b = m->bf + (row - m->n_hot) * m->dim;
    for (int t = 0; t < m->dim; t++) out[t] = bf_to_f(b[t]);
  }
}
/* row += u (FP32 rows) or row = SR(cur + u) (BF16 rows; cur = the row as read) */
static void mr_add(const mixed_rows *m, long long row, const float *cur, const float *u, uint32_t seed, uint64_t s,
                   uint32_t pair, uint32_t slot) {
  if (row < m->n_hot) {
    float *r = m->f32 + row * m->dim;
    for (int t = 0; t < m->dim; t++) r[t] += u[t];
    return;
  }
  uint16_t *b = m->bf + (row - m->n_hot) * m->dim;
  for (int lane = 0; lane < 32; lane++) {
    const uint32_t x = orc_lane_key(seed, s, pair, (uint32_t)lane);
    uint32_t w = 0;
    for (int j = 0; lane + 32 * j < m->dim; j++) {
      int t = lane + 32 * j;
      if ((j & 1) == 0) w = (x + slot * 0x27D4EB2Fu + (uint32_t)(j / 2) * 0x165667B1u) * 0x9E3779B1u;
      b[t] = f_to_bf_sr(cur[t] + u[t], (j & 1) ? (w >> 16) : (w & 0xFFFFu));
    }
  }
}

/* rounding seed of one training round, from the context seed */
uint32_t orc_round_sr_seed(uint64_t seed, uint32_t round) {
  return sr_h((uint32_t)seed ^ sr_h((uint32_t)(seed >> 32) + round * 0x9E3779B9u));
}

/* negs == NULL: skip_gram_kernel draws; else __sgNegReuse (full window, the
 * sentence's plan negatives) as in orc_negreuse_batch */
static void sg_bf16_impl(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                         uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                         long long vocab_size, const int32_t *sen, const uint64_t *sent_start,
                         uint64_t first_sentence, uint64_t n_sentences, int window, int dim, int negative,
                         float alpha, const int32_t *negs) {
  mixed_rows m0 = {syn0, syn0_bf, n_hot, dim}, m1 = {syn1, syn1_bf, n_hot, dim};
  float x[512], y[512], neu1e[512], upd[512];
  for (uint64_t blk = 0; blk < n_sentences; blk++) {
    uint64_t s = first_sentence + blk;
    long long ss = (long long)sent_start[s], se = (long long)sent_start[s + 1];
    unsigned long next_random = (unsigned long)blk;
    uint32_t pair = 0;
    for (long long pos = ss; pos < se; pos++) {
      int word = sen[pos];
      if (word == -1) continue;
      int b = 0;
      if (!negs) {
        next_random = next_random * (unsigned long)2514903917 + 11;
        b = (int)(next_random % (unsigned long)window);
      }
      for (int a = b; a < window * 2 + 1 - b; a++) {
        if (a == window) continue;
        long long c = pos - window + a;
        if (c < ss || c >= se) continue;
        int last_word = sen[c];
        if (last_word == -1) continue;
        uint32_t pk = pair++;
        mr_get(&m0, last_word, x);
        for (int t = 0; t < dim; t++) neu1e[t] = 0;
        for (int d = 0; d < negative + 1; d++) {
          int target, label;
          if (d == 0) {
            target = word;
            label = 1;
          } else if (negs) {
            target = negs[s * (uint64_t)negative + d - 1];
            if (target == word) continue;
            label = 0;
          } else {
            next_random = next_random * (unsigned long)25214903917 + 11;
            target = table[(next_random >> 16) % (unsigned long)table_size];
            if (target == 0) target = (int)(next_random % (unsigned long)(vocab_size - 1) + 1);
            if (target == word) continue;
            label = 0;
          }
          mr_get(&m1, target, y);
          float f = sg_dot(x, y, dim);
          float g = sg_gradient(f, label, exp_table, alpha);
          for (int t = 0; t < dim; t++) {
            neu1e[t] = fmaf(g, y[t], neu1e[t]);
            upd[t] = g * x[t];
          }
          mr_add(&m1, target, y, upd, sr_seed, s, pk, (uint32_t)d);
        }
        mr_add(&m0, last_word, x, neu1e, sr_seed, s, pk, 256u);
      }
    }
  }
}

void orc_skipgram_bf16(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                       uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                       long long vocab_size, const int32_t *sen, const uint64_t *sent_start,
                       uint64_t first_sentence, uint64_t n_sentences, int window, int dim, int negative,
                       float alpha) {
  sg_bf16_impl(syn0, syn0_bf, syn1, syn1_bf, n_hot, sr_seed, exp_table, table, table_size, vocab_size, sen,
               sent_start, first_sentence, n_sentences, window, dim, negative, alpha, NULL);
}

void orc_negreuse_bf16(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                       uint32_t sr_seed, const float *exp_table, const int32_t *sen, const uint64_t *sent_start,
                       uint64_t first_sentence, uint64_t n_sentences, const int32_t *negs, int window, int dim,
                       int negative, float alpha) {
  sg_bf16_impl(syn0, syn0_bf, syn1, syn1_bf, n_hot, sr_seed, exp_table, NULL, 0, 0, sen, sent_start, first_sentence,
               n_sentences, window, dim, negative, alpha, negs);
}

/* -reuse-neg 2 (this project's option): __sgNegReuse's work (full window, the
 * sentence's K plan negatives) as one tile per center.  Per center: the K + 1
 * target rows (center word as positive, negatives not equal to it) are read
 * once; every context in window order is read fresh, scored against them with
 * the tree dot, and updated at once (x += sum_j g_j y_j, j in order); the
 * targets' updates dy_j = sum over contexts of g_j x (context order) are
 * applied at the end of the center, a negative that occurs twice adding its
 * dy into its first occurrence.  Rows in the mixed storage form (n_hot =
 * vocab_size: all FP32); rounding streams as orc_skipgram_bf16 with the
 * center's index in the sentence as the pair index, slot j for targets and
 * 256 + window position for contexts. */
static void tile_impl(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                      uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                      long long vocab_size, const int32_t *sen, const uint64_t *sent_start, uint64_t first_sentence,
                      uint64_t n_sentences, const int32_t *negs, int window, int dim, int negative, float alpha) {
  mixed_rows m0 = {syn0, syn0_bf, n_hot, dim}, m1 = {syn1, syn1_bf, n_hot, dim};
  float x[512], neu1e[512];
  float y[16][512], dy[16][512];
  int tg[16], wneg[16];
  for (uint64_t blk = 0; blk < n_sentences; blk++) {
    uint64_t s = first_sentence + blk;
    long long ss = (long long)sent_start[s], se = (long long)sent_start[s + 1];
    const int32_t *neg = negs ? negs + s * (uint64_t)negative : wneg;
    unsigned long next_random = (unsigned long)blk;
    for (long long pos = ss; pos < se; pos++) {
      int word = sen[pos];
      int b = 0;
      if (!negs) {
        next_random = next_random * (unsigned long)2514903917 + 11;
        b = (int)(next_random % (unsigned long)window);
      }
      long long c0 = pos - window + b < ss ? ss : pos - window + b;
      long long c1 = pos + window - b > se - 1 ? se - 1 : pos + window - b;
      if (c1 - c0 < 1) continue;
      if (!negs) {
        /* skip_gram_kernel draws K negatives per context (word2vec.cu:496-507);
         * the center keeps the draws of its first context and the stream moves
         * on past all of its contexts' draws */
        for (long long c = c0; c <= c1; c++) {
          if (c == pos) continue;
          for (int q = 0; q < negative; q++) {
            next_random = next_random * (unsigned long)25214903917 + 11;
            int t = table[(next_random >> 16) % (unsigned long)table_size];
            if (t == 0) t = (int)(next_random % (unsigned long)(vocab_size - 1) + 1);
            if (c == (c0 == pos ? c0 + 1 : c0)) wneg[q] = t;
          }
        }
      }
      int nt = negative + 1;
      tg[0] = word;
      for (int q = 0; q < negative; q++) tg[q + 1] = neg[q] == word ? -1 : neg[q];
      for (int q = 0; q < nt; q++) {
        for (int t = 0; t < dim; t++) dy[q][t] = 0;
        if (tg[q] >= 0) mr_get(&m1, tg[q], y[q]);
      }
      uint32_t center = (uint32_t)(pos - ss);
      for (long long c = c0; c <= c1; c++) {
        if (c == pos) continue;
        int l1 = sen[c];
        mr_get(&m0, l1, x);
        for (int t = 0; t < dim; t++) neu1e[t] = 0;
        for (int q = 0; q < nt; q++) {
          if (tg[q] < 0) continue;
          float f = sg_dot(x, y[q], dim);
          float g = sg_gradient(f, q == 0 ? 1 : 0, exp_table, alpha);
          for (int t = 0; t < dim; t++) {
            neu1e[t] = fmaf(g, y[q][t], neu1e[t]);
            dy[q][t] = fmaf(g, x[t], dy[q][t]);
          }
        }
        mr_add(&m0, l1, x, neu1e, sr_seed, s, center, 256u + (uint32_t)(c - pos + window));
      }
      for (int q = 2; q < nt; q++) {
        if (tg[q] < 0) continue;
        for (int r = 1; r < q; r++)
          if (tg[r] == tg[q]) {
            for (int t = 0; t < dim; t++) dy[r][t] = dy[r][t] + dy[q][t];
            tg[q] = -2;
            break;
          }
      }
      for (int q = 0; q < nt; q++)
        if (tg[q] >= 0) mr_add(&m1, tg[q], y[q], dy[q], sr_seed, s, center, (uint32_t)q);
    }
  }
}

void orc_negreuse_tile(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                       uint32_t sr_seed, const float *exp_table, const int32_t *sen, const uint64_t *sent_start,
                       uint64_t first_sentence, uint64_t n_sentences, const int32_t *negs, int window, int dim,
                       int negative, float alpha) {
  tile_impl(syn0, syn0_bf, syn1, syn1_bf, n_hot, sr_seed, exp_table, NULL, 0, 0, sen, sent_start, first_sentence,
            n_sentences, negs, window, dim, negative, alpha);
}

/* -reuse-neg 4 (this project's option): window tiles.  The center tile of
 * orc_negreuse_tile over skip_gram_kernel's own window and draws
 * (word2vec.cu:442-536): the window shrink b from the sentence's LCG
 * (:458-459), contexts pos - window + b .. pos + window - b, and as the
 * center's shared negatives the K draws the reference makes for the center's
 * first context (:496-507, 0 -> next % (vocab - 1) + 1, skipped when equal to
 * the word); the LCG then advances past the K draws of every context, so each
 * center's window is the reference's. */
void orc_window_tile(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                     uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                     long long vocab_size, const int32_t *sen, const uint64_t *sent_start, uint64_t first_sentence,
                     uint64_t n_sentences, int window, int dim, int negative, float alpha) {
  tile_impl(syn0, syn0_bf, syn1, syn1_bf, n_hot, sr_seed, exp_table, table, table_size, vocab_size, sen, sent_start,
            first_sentence, n_sentences, NULL, window, dim, negative, alpha);
}

/* -reuse-neg 3 (this project's option, BF16 form): the center tile scored on
 * tensor cores.  Per center all contexts (window order) and targets are read at
 * the start of the center; scores are dots of their round-to-nearest BF16
 * copies (the tensor core accumulates in FP32 in an unspecified order; here the
 * sum is FP64, rounded to FP32, so a test compares within a tolerance).
 * Rows of G belonging to a repeated context word are added into its first
 * occurrence (column by column, in window order); then, per context in order,
 * neu = sum_j G_cj y_j (y exact) and dy_j += G_cj xb_c (xb the BF16 copy); the
 * first occurrence of each context word is updated once; targets as in
 * orc_negreuse_tile. */
static float bf16_round_rn(float v) {
  uint32_t b;
  memcpy(&b, &v, 4);
  b = (b + 0x7FFFu + ((b >> 16) & 1u)) & 0xFFFF0000u;
  memcpy(&v, &b, 4);
  return v;
}

void orc_negreuse_tile_tc(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                          uint32_t sr_seed, const float *exp_table, const int32_t *sen, const uint64_t *sent_start,
                          uint64_t first_sentence, uint64_t n_sentences, const int32_t *negs, int window, int dim,
                          int negative, float alpha) {
  mixed_rows m0 = {syn0, syn0_bf, n_hot, dim}, m1 = {syn1, syn1_bf, n_hot, dim};
  static float xb[64][512], y[16][512], yb[16][512], dy[16][512];
  float neu1e[512], G[64][16];
  int tg[16], cw[64], first[64];
  long long cpos[64];
  for (uint64_t blk = 0; blk < n_sentences; blk++) {
    uint64_t s = first_sentence + blk;
    long long ss = (long long)sent_start[s], se = (long long)sent_start[s + 1];
    const int32_t *neg = negs + s * (uint64_t)negative;
    for (long long pos = ss; pos < se; pos++) {
      int word = sen[pos];
      long long c0 = pos - window < ss ? ss : pos - window;
      long long c1 = pos + window > se - 1 ? se - 1 : pos + window;
      int n = (int)(c1 - c0);
      if (n < 1) continue;
      int nt = negative + 1;
      tg[0] = word;
      for (int q = 0; q < negative; q++) tg[q + 1] = neg[q] == word ? -1 : neg[q];
      for (int q = 0; q < nt; q++) {
        for (int t = 0; t < dim; t++) y[q][t] = 0, dy[q][t] = 0;
        if (tg[q] >= 0) mr_get(&m1, tg[q], y[q]);
        for (int t = 0; t < dim; t++) yb[q][t] = bf16_round_rn(y[q][t]);
      }
      for (int i = 0; i < n; i++) {
        long long c = c0 + i;
        if (c >= pos) c++;
        cpos[i] = c;
        cw[i] = sen[c];
        mr_get(&m0, cw[i], xb[i]);
        for (int t = 0; t < dim; t++) xb[i][t] = bf16_round_rn(xb[i][t]);
        first[i] = i;
        for (int j = 0; j < i; j++)
          if (cw[j] == cw[i]) {
            first[i] = j;
            break;
          }
      }
      for (int i = 0; i < n; i++)
        for (int q = 0; q < nt; q++) {
          G[i][q] = 0;
          if (tg[q] < 0) continue;
          double f = 0;
          for (int t = 0; t < dim; t++) f += (double)xb[i][t] * (double)yb[q][t];
          G[i][q] = sg_gradient((float)f, q == 0 ? 1 : 0, exp_table, alpha);
        }
      for (int q = 0; q < nt; q++)
        for (int i = 1; i < n; i++)
          if (first[i] != i) {
            G[first[i]][q] = G[first[i]][q] + G[i][q];
            G[i][q] = 0;
          }
      uint32_t center = (uint32_t)(pos - ss);
      for (int i = 0; i < n; i++) {
        for (int t = 0; t < dim; t++) neu1e[t] = 0;
        for (int q = 0; q < nt; q++) {
          float g = G[i][q];
          for (int t = 0; t < dim; t++) {
            neu1e[t] = fmaf(g, y[q][t], neu1e[t]);
            dy[q][t] = fmaf(g, xb[i][t], dy[q][t]);
          }
        }
        if (first[i] == i) mr_add(&m0, cw[i], xb[i], neu1e, sr_seed, s, center, 256u + (uint32_t)(cpos[i] - pos + window));
      }
      for (int q = 2; q < nt; q++) {
        if (tg[q] < 0) continue;
        for (int r = 1; r < q; r++)
          if (tg[r] == tg[q]) {
            for (int t = 0; t < dim; t++) dy[r][t] = dy[r][t] + dy[q][t];
            tg[q] = -2;
            break;
          }
      }
      for (int q = 0; q < nt; q++)
        if (tg[q] >= 0) mr_add(&m1, tg[q], y[q], dy[q], sr_seed, s, center, (uint32_t)q);
    }
  }
}

void orc_cbow_bf16(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                   uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                   long long vocab_size, const int32_t *sen, const uint64_t *sent_start, uint64_t first_sentence,
                   uint64_t n_sentences, int window, int dim, int negative, float alpha) {
  mixed_rows m0 = {syn0, syn0_bf, n_hot, dim}, m1 = {syn1, syn1_bf, n_hot, dim};
  float x[512], y[512], neu1[512], neu1e[512], upd[512];
  for (uint64_t blk = 0; blk < n_sentences; blk++) {
    uint64_t s = first_sentence + blk;
    long long ss = (long long)sent_start[s], se = (long long)sent_start[s + 1];
    unsigned long next_random = (unsigned long)blk;
    for (long long pos = ss; pos < se; pos++) {
      int word = sen[pos];
      if (word == -1) continue;
      uint32_t pk = (uint32_t)(pos - ss);
      for (int t = 0; t < dim; t++) neu1[t] = neu1e[t] = 0;
      next_random = next_random * (unsigned long)2514903917 + 11;
      int b = (int)(next_random % (unsigned long)window);
      int cw = 0;
      for (int a = b; a < window * 2 + 1 - b; a++) {
        if (a == window) continue;
        long long c = pos - window + a;
        if (c < ss || c >= se || sen[c] == -1) continue;
        mr_get(&m0, sen[c], x);
        for (int t = 0; t < dim; t++) neu1[t] += x[t];
        cw++;
      }
      if (!cw) continue;
      for (int t = 0; t < dim; t++) neu1[t] /= cw;
      for (int d = 0; d < negative + 1; d++) {
        int target, label;
        if (d == 0) {
          target = word;
          label = 1;
        } else {
          next_random = next_random * (unsigned long)25214903917 + 11;
          target = table[(next_random >> 16) % (unsigned long)table_size];
          if (target == 0) target = (int)(next_random % (unsigned long)(vocab_size - 1) + 1);
          if (target == word) continue;
          label = 0;
        }
        mr_get(&m1, target, y);
        float f = sg_dot(neu1, y, dim);
        float g = sg_gradient(f, label, exp_table, alpha);
        for (int t = 0; t < dim; t++) {
          neu1e[t] = fmaf(g, y[t], neu1e[t]);
          upd[t] = g * neu1[t];
        }
        mr_add(&m1, target, y, upd, sr_seed, s, pk, (uint32_t)d);
      }
      for (int a = b; a < window * 2 + 1 - b; a++) {
        if (a == window) continue;
        long long c = pos - window + a;
        if (c < ss || c >= se || sen[c] == -1) continue;
        mr_get(&m0, sen[c], x);
        mr_add(&m0, sen[c], x, neu1e, sr_seed, s, pk, 256u + (uint32_t)a);
      }
    }
  }
}

void orc_init_net(float *syn0, float *syn1, long long vocab_size, int dim) {
  unsigned long long next_random = 1;
  for (long long a = 0; a < vocab_size; a++)
    for (int b = 0; b < dim; b++) {
      next_random = next_random * (unsigned long long)25214903917 + 11;
      syn0[a * dim + b] = (((next_random & 0xFFFF) / (float)65536) - 0.5) / dim;
    }
  if (syn1) memset(syn1, 0, sizeof(float) * (size_t)vocab_size * (size_t)dim);
}

/* batch_similarity_direct_index_optimized_kernel order with blockDim = 128 (dim <= 128) */
float orc_cosine(const float *a, const float *b, int dim) {
  float sd[256], sa[256], sb[256];
  int bd = dim > 200 ? 256 : 128;
  for (int t = 0; t < bd; t++) {
    float x = t < dim ? a[t] : 0.0f, y = t < dim ? b[t] : 0.0f;
    sd[t] = x * y;
    sa[t] = x * x;
    sb[t] = y * y;
  }
  for (int s = bd / 2; s > 0; s >>= 1)
    for (int t = 0; t < s; t++) {
      sd[t] += sd[t + s];
      sa[t] += sa[t + s];
      sb[t] += sb[t + s];
    }
  float na = sqrtf(sa[0]), nb = sqrtf(sb[0]);
  if (na == 0.0f || nb == 0.0f) return 0.0f;
  return sd[0] / (na * nb);
}

void orc_eval_choose(uint64_t seed, uint32_t round, uint32_t v, uint32_t deg, uint32_t *chosen) {
  /* partial Fisher-Yates over positions 0..deg-1, first 30 positions */
  uint32_t pos[30], val[30];
  int nsw = 0;
  for (uint32_t i = 0; i < 30; i++) {
    uint32_t ctr[4] = {v, round, i, 0x45564C31u};
    uint32_t key[2] = {(uint32_t)seed ^ 0x2545F491u, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    uint32_t j = i + mulhi64_u32(((uint64_t)o[1] << 32) | o[0], deg - i);
    /* current values at positions i and j */
    uint32_t vi = i, vj = j;
    int hi = -1, hj = -1;
    for (int k = 0; k < nsw; k++) {
      if (pos[k] == i) hi = k;
      if (pos[k] == j) hj = k;
    }
    if (hi >= 0) vi = val[hi];
    if (hj >= 0) vj = val[hj];
    chosen[i] = vj;
    /* position j now holds vi (position i is never read again) */
    if (hj >= 0) val[hj] = vi;
    else { pos[nsw] = j; val[nsw] = vi; nsw++; }
  }
}

uint64_t orc_convergence(const float *syn0, const uint32_t *id2offset, int dim, const orc_csr *g,
                         uint8_t *stop_flags, uint64_t seed, uint32_t round, float *sim) {
  uint64_t eva = 0;
  uint32_t chosen[30];
  for (uint32_t v = 0; v < g->v_num; v++) {
    if (stop_flags[v]) continue; /* word2vec.cu:2023-2027 */
    if (id2offset[v] == 0xFFFFFFFFu) continue; /* no row (out of vocabulary) */
    uint64_t b = g->row_ptr[v];
    uint32_t deg = (uint32_t)(g->row_ptr[v + 1] - b);
    int n = deg;
    if (deg > 30) {
      n = 30;
      orc_eval_choose(seed, round, v, deg, chosen);
    } else {
      for (uint32_t i = 0; i < deg; i++) chosen[i] = i;
    }
    float s = 0.0f;
    if (n > 0) {
      float sum = 0.0f;
      int used = 0;
      const float *a = syn0 + (uint64_t)id2offset[v] * dim;
      for (int j = 0; j < n; j++) {
        uint32_t u = g->nbr[b + chosen[j]];
        if (id2offset[u] == 0xFFFFFFFFu) continue;
        sum += orc_cosine(a, syn0 + (uint64_t)id2offset[u] * dim, dim);
        used++;
      }
      s = used > 0 ? sum / used : 0.0f;
    }
    if (sim) sim[v] = s;
    if (s > 0.65) stop_flags[v] = 1; /* word2vec.cu:2056-2061 */
    else eva++;
  }
  return eva;
}

/* ---- learned walk budget (this project's; no reference counterpart) ----
 * Features of vertex v, FP64: log1p(deg), log1p(sum of weights), entropy of
 * the normalized weights (natural log), log1p(sum of the neighbours'
 * degrees), log1p(visits), log1p(first walk length). */
void orc_budget_features(const orc_csr *g, const uint64_t *visits, const uint32_t *first_len, double *feat) {
  for (uint32_t v = 0; v < g->v_num; v++) {
    uint64_t b = g->row_ptr[v], e = g->row_ptr[v + 1];
    double ws = 0, hop2 = 0, h = 0;
    for (uint64_t i = b; i < e; i++) {
      ws += (double)g->data[i];
      uint32_t u = g->nbr[i];
      hop2 += (double)(g->row_ptr[u + 1] - g->row_ptr[u]);
    }
    if (ws > 0)
      for (uint64_t i = b; i < e; i++) {
        double p = (double)g->data[i] / ws;
        if (p > 0) h -= p * log(p);
      }
    double *f = feat + (uint64_t)v * 6;
    f[0] = log1p((double)(e - b));
    f[1] = log1p(ws);
    f[2] = h;
    f[3] = log1p(hop2);
    f[4] = log1p((double)visits[v]);
    f[5] = log1p((double)first_len[v]);
  }
}

/* MLP 6 -> 64 -> 64 -> (9 + 1), ReLU, parameters W1[64][6] b1 W2[64][64] b2
 * W3[10][64] b3; loss per sample = softmax cross-entropy of the 9 count logits
 * against count - 2 plus (out[9] - (length - 50) / 30)^2 / 2.  Mean loss and
 * mean gradient over n samples, all in FP64. */
#define MLP_IN 6
#define MLP_H 64
#define MLP_C 9
#define MLP_O 10
#define MLP_W1 0
#define MLP_B1 (MLP_W1 + MLP_H * MLP_IN)
#define MLP_W2 (MLP_B1 + MLP_H)
#define MLP_B2 (MLP_W2 + MLP_H * MLP_H)
#define MLP_W3 (MLP_B2 + MLP_H)
#define MLP_B3 (MLP_W3 + MLP_O * MLP_H)
#define MLP_P (MLP_B3 + MLP_O)

double orc_mlp_loss_grad(const float *params, const float *X, const uint8_t *count, const float *length, uint64_t n,
                         double *grad) {
  double P[MLP_P];
  for (int i = 0; i < MLP_P; i++) {
    P[i] = params[i];
    grad[i] = 0;
  }
  double loss = 0;
  for (uint64_t sidx = 0; sidx < n; sidx++) {
    double x[MLP_IN], h1[MLP_H], h2[MLP_H], out[MLP_O], d3[MLP_O], d2[MLP_H], d1[MLP_H];
    for (int i = 0; i < MLP_IN; i++) x[i] = X[sidx * MLP_IN + i];
    for (int u = 0; u < MLP_H; u++) {
      double a = P[MLP_B1 + u];
      for (int i = 0; i < MLP_IN; i++) a += P[MLP_W1 + u * MLP_IN + i] * x[i];
      h1[u] = a > 0 ? a : 0;
    }
    for (int u = 0; u < MLP_H; u++) {
      double a = P[MLP_B2 + u];
      for (int k = 0; k < MLP_H; k++) a += P[MLP_W2 + u * MLP_H + k] * h1[k];
      h2[u] = a > 0 ? a : 0;
    }
    for (int c = 0; c < MLP_O; c++) {
      double a = P[MLP_B3 + c];
      for (int u = 0; u < MLP_H; u++) a += P[MLP_W3 + c * MLP_H + u] * h2[u];
      out[c] = a;
    }
    double m = out[0], se = 0;
    for (int c = 1; c < MLP_C; c++) m = out[c] > m ? out[c] : m;
    for (int c = 0; c < MLP_C; c++) se += exp(out[c] - m);
    int yc = (int)count[sidx] - 2;
    double yl = ((double)length[sidx] - 50.0) / 30.0;
    double dl = out[MLP_C] - yl;
    loss += log(se) + m - out[yc] + 0.5 * dl * dl;
    for (int c = 0; c < MLP_C; c++) d3[c] = exp(out[c] - m) / se - (c == yc ? 1.0 : 0.0);
    d3[MLP_C] = dl;
    for (int c = 0; c < MLP_O; c++) {
      for (int u = 0; u < MLP_H; u++) grad[MLP_W3 + c * MLP_H + u] += d3[c] * h2[u];
      grad[MLP_B3 + c] += d3[c];
    }
    for (int u = 0; u < MLP_H; u++) {
      double d = 0;
      for (int c = 0; c < MLP_O; c++) d += P[MLP_W3 + c * MLP_H + u] * d3[c];
      d2[u] = h2[u] > 0 ? d : 0;
    }
    for (int u = 0; u < MLP_H; u++) {
      for (int k = 0; k < MLP_H; k++) grad[MLP_W2 + u * MLP_H + k] += d2[u] * h1[k];
      grad[MLP_B2 + u] += d2[u];
    }
    for (int k = 0; k < MLP_H; k++) {
      double d = 0;
      for (int u = 0; u < MLP_H; u++) d += P[MLP_W2 + u * MLP_H + k] * d2[u];
      d1[k] = h1[k] > 0 ? d : 0;
    }
    for (int k = 0; k < MLP_H; k++) {
      for (int i = 0; i < MLP_IN; i++) grad[MLP_W1 + k * MLP_IN + i] += d1[k] * x[i];
      grad[MLP_B1 + k] += d1[k];
    }
  }
  for (int i = 0; i < MLP_P; i++) grad[i] /= (double)n;
  return loss / (double)n;
}

/* ------------------------------------------------------------------------
 * Common neighbours (src/tools/gcn.cpp) */

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : x > y;
}

/* first index of [lo, hi) with v[i] >= key (std::lower_bound) */
static uint64_t lower_u32(const uint32_t *v, uint64_t lo, uint64_t hi, uint32_t key) {
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (v[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

/* myIntersectition (gcn.cpp:146-196): galloping search of each element of the
 * shorter list (the second list on a size tie) in the longer one; a match
 * appends the short element and keeps the long position, so repeated short
 * elements match again.  Appends to out (capacity >= |short|), returns the
 * count. */
static uint32_t gcn_intersect(const uint32_t *v1, int n1, const uint32_t *v2, int n2, uint32_t *out) {
  if (n1 == 0 || n2 == 0) return 0;
  const uint32_t *lv = n1 > n2 ? v1 : v2, *sv = n1 > n2 ? v2 : v1;
  const int nl = n1 > n2 ? n1 : n2, ns = n1 > n2 ? n2 : n1;
  if (lv[nl - 1] < sv[0] || lv[0] > sv[ns - 1]) return 0;
  uint32_t cnt = 0;
  int p1 = 0, p2 = 0;
  while (p1 < nl && p2 < ns) {
    int step = 1, last = step;
    if (sv[p2] < lv[p1]) {
      p2++;
      continue;
    }
    while (lv[p1 + step - 1] < sv[p2]) {
      step *= 2;
      last = p1 + step < nl ? step : nl - p1;
      if (p1 + step >= nl) break;
    }
    if (lv[nl - 1] < sv[p2]) {
      p2++;
      break;
    }
    const int t = (int)lower_u32(lv, (uint64_t)(p1 + step / 2), (uint64_t)(p1 + last), sv[p2]);
    if (lv[t] == sv[p2]) {
      out[cnt++] = sv[p2];
      p2++;
      p1 = t;
    } else {
      p2++;
      p1 = p1 + step / 2;
    }
  }
  return cnt;
}

int orc_common_neighbours(const uint32_t *src, const uint32_t *dst, uint64_t n, uint32_t v_num, int undirected,
                          int32_t *cn) {
  for (uint64_t e = 0; e < n; e++)
    if (src[e] >= v_num || dst[e] >= v_num) return -1;
  const uint64_t m = undirected ? 2 * n : n;
  uint64_t *rp = (uint64_t *)calloc((size_t)v_num + 1, sizeof(uint64_t));
  uint32_t *nbr = (uint32_t *)malloc((size_t)(m ? m : 1) * sizeof(uint32_t));
  int32_t *data = (int32_t *)malloc((size_t)(m ? m : 1) * sizeof(int32_t));
  uint64_t *fill = (uint64_t *)malloc(((size_t)v_num + 1) * sizeof(uint64_t));
  uint32_t *inter = NULL;
  if (!rp || !nbr || !data || !fill) goto fail;
  /* rows in input order, the doubled edge list interleaved (e, e^T) */
  for (uint64_t e = 0; e < n; e++) {
    rp[src[e] + 1]++;
    if (undirected) rp[dst[e] + 1]++;
  }
  for (uint32_t v = 0; v < v_num; v++) rp[v + 1] += rp[v];
  memcpy(fill, rp, ((size_t)v_num + 1) * sizeof(uint64_t));
  for (uint64_t e = 0; e < n; e++) {
    nbr[fill[src[e]]++] = dst[e];
    if (undirected) nbr[fill[dst[e]]++] = src[e];
  }
  uint64_t maxdeg = 0;
  for (uint32_t v = 0; v < v_num; v++) {
    const uint64_t d = rp[v + 1] - rp[v];
    if (d > 1) qsort(nbr + rp[v], (size_t)d, sizeof(uint32_t), cmp_u32);
    if (d > maxdeg) maxdeg = d;
  }
  for (uint64_t i = 0; i < m; i++) data[i] = -1;
  inter = (uint32_t *)malloc((size_t)(maxdeg ? maxdeg : 1) * sizeof(uint32_t));
  if (!inter) goto fail;
  for (uint64_t e = 0; e < n; e++) {
    const uint32_t s = src[e], d = dst[e];
    const uint64_t pos = lower_u32(nbr, rp[s], rp[s + 1], d);
    if (data[pos] != -1) continue;
    const uint32_t k = gcn_intersect(nbr + rp[s], (int)(rp[s + 1] - rp[s]), nbr + rp[d], (int)(rp[d + 1] - rp[d]), inter);
    uint32_t c = k;
    if (c > 0) {
      if (inter[0] == s || inter[0] == d) c--;
      if (c > 1)
        for (uint32_t i = 1; i < k; i++) {
          if (inter[i] == inter[i - 1]) c--;
          else if (inter[i] == s || inter[i] == d) c--;
        }
    }
    data[pos] = (int32_t)c;
    const uint64_t mp = lower_u32(nbr, rp[d], rp[d + 1], s);
    if (mp < rp[d + 1] && nbr[mp] == s) data[mp] = (int32_t)c;
  }
  for (uint64_t e = 0; e < n; e++) cn[e] = data[lower_u32(nbr, rp[src[e]], rp[src[e] + 1], dst[e])];
  free(rp); free(nbr); free(data); free(fill); free(inter);
  return 0;
fail:
  free(rp); free(nbr); free(data); free(fill); free(inter);
  return -1;
}
