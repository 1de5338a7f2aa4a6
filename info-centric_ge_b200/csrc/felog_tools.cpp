// Host-side data tools: seeded R-MAT graphs, the link-prediction split,
// the 12-byte binary edge format and an exact AUC.  Declarations and the
// reference files each function stands in for are in include/felog_tools.h.
#include "felog_tools.h"

#include <parallel/algorithm>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <unordered_set>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// Counter-based stream: value k of stream (seed, id).
inline uint64_t draw(uint64_t seed, uint64_t id, uint64_t k) {
  return mix64(mix64(seed ^ 0x5DEECE66DULL) + mix64(id * 0xD1B54A32D192ED03ULL + k));
}

inline double unit01(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

struct Cand {
  uint64_t key;  // (min << 32) | max
  uint64_t idx;  // candidate index (generation order)
  uint32_t src, dst;
};

}  // namespace

// 31-bit values of the split's random stream: value k of stream (seed ^ 0x5117, 1),
// in [0, 2^31 - 1], as rand() gives them to gtrain.cpp's get_big_rand.
inline uint64_t split_rand(uint64_t seed, uint64_t k) { return draw(seed ^ 0x5117ULL, 1, k) >> 33; }

// get_big_rand (gtrain.cpp:214-223) on the split stream; RAND_MAX = 2^31 - 1
inline uint64_t split_big_rand(uint64_t seed, uint64_t &k, uint64_t range) {
  const uint64_t rmax = 2147483647ULL;
  if (range < rmax) return split_rand(seed, k++) % range;
  const uint64_t round = range / rmax, mod = range % rmax;
  const uint64_t t = split_rand(seed, k++) % round + 1;
  if (t == round) return t * rmax + split_rand(seed, k++) % mod;
  return t * rmax + split_rand(seed, k++) % rmax;
}

// The held-out split of gtrain.cpp:293-343 over edges (in place): npos =
// holdout * E (float arithmetic, as the tool's float sample); positives by
// swap-to-tail, each drawn until both endpoints still have degree > 1, which
// then drops by one; negatives as (src, dst) draws until the pair is no
// edge and src -> dst is not yet a negative (a pair and its reverse are two
// candidates, a vertex paired with itself is allowed, as in the tool).  One
// random stream feeds every draw in the tool's order.  The train edges are
// edges[0 .. E - npos).  Returns npos, or ~0 when a draw loop runs away.
static uint64_t heldout_split(std::vector<felog_edge12> &edges, uint32_t nv, double holdout, uint64_t seed,
                       std::vector<uint32_t> &tsrc, std::vector<uint32_t> &tdst, std::vector<uint8_t> &tlab) {
  const uint64_t E = edges.size();
  const uint64_t npos = (uint64_t)((float)holdout * (float)E);
  std::vector<uint64_t> deg(nv, 0);
  for (auto &e : edges) {
    deg[e.src]++;
    deg[e.dst]++;
  }
  tsrc.clear();
  tdst.clear();
  tlab.clear();
  tsrc.reserve(2 * npos);
  tdst.reserve(2 * npos);
  tlab.reserve(2 * npos);
  if (npos > E) return ~0ULL;
  uint64_t k = 0, tail = E - 1;
  std::vector<uint64_t> pos_src, pos_dst;
  for (uint64_t i = 0; i < npos; i++) {
    uint64_t ep, guard = 0;
    do {
      ep = split_big_rand(seed, k, tail + 1);
      if (++guard > 1000000000ULL) return ~0ULL;
    } while (deg[edges[ep].src] <= 1 || deg[edges[ep].dst] <= 1);
    tsrc.push_back(edges[ep].src);
    tdst.push_back(edges[ep].dst);
    tlab.push_back(1);
    deg[edges[ep].src]--;
    deg[edges[ep].dst]--;
    std::swap(edges[ep], edges[tail]);
    tail--;
  }
  std::unordered_set<uint64_t> edge_set;
  edge_set.reserve(E * 2);
  for (auto &e : edges) {
    uint64_t lo = std::min(e.src, e.dst), hi = std::max(e.src, e.dst);
    edge_set.insert((lo << 32) | hi);
  }
  std::unordered_set<uint64_t> neg_set;  // directed: src << 32 | dst
  neg_set.reserve(npos * 2 + 1);
  for (uint64_t i = 0; i < npos; i++) {
    uint64_t guard = 0;
    for (;;) {
      const uint32_t a = (uint32_t)split_big_rand(seed, k, nv);
      const uint32_t b = (uint32_t)split_big_rand(seed, k, nv);
      if (++guard > 1000000000ULL) return ~0ULL;
      const uint64_t lo = std::min(a, b), hi = std::max(a, b);
      if (a != b && edge_set.count((lo << 32) | hi)) continue;
      if (!neg_set.insert(((uint64_t)a << 32) | b).second) continue;
      tsrc.push_back(a);
      tdst.push_back(b);
      tlab.push_back(0);
      break;
    }
  }
  return npos;
}

struct felog_synth {
  felog_synth_info info;
  std::vector<felog_edge12> train;
  std::vector<uint32_t> test_src, test_dst;
  std::vector<uint8_t> test_label;
};

extern "C" int felog_synth_generate(const felog_synth_params *p, felog_synth **out) {
  if (!p || !out || p->v_target < 2 || p->e_target == 0) return -1;
  if (p->v_target > 0xFFFFFFFFULL) return -1;
  double sum = p->a + p->b + p->c + p->d;
  if (!(sum > 0.999 && sum < 1.001)) return -1;
  if (p->holdout < 0.0 || p->holdout >= 1.0) return -1;
  felog_synth *s = new (std::nothrow) felog_synth();
  if (!s) return -2;
  const uint64_t V = p->v_target;
  int scale = 0;
  while ((1ULL << scale) < V) scale++;
  const double ta = p->a, tab = p->a + p->b, tabc = p->a + p->b + p->c;

  // ---- candidates, in rounds, until e_target unique undirected edges ----
  std::vector<Cand> uniq;
  uint64_t next_idx = 0;
  while (uniq.size() < p->e_target) {
    uint64_t need = p->e_target - uniq.size();
    uint64_t n = need + need / 2 + 1024;
    std::vector<Cand> c(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++) {
      uint64_t id = next_idx + (uint64_t)i;
      uint64_t u = 0, v = 0;
      for (int l = 0; l < scale; l++) {
        double r = unit01(draw(p->seed, id, (uint64_t)l));
        uint64_t bu, bv;
        if (r < ta) { bu = 0; bv = 0; }
        else if (r < tab) { bu = 0; bv = 1; }
        else if (r < tabc) { bu = 1; bv = 0; }
        else { bu = 1; bv = 1; }
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      Cand &x = c[(size_t)i];
      x.idx = id;
      if (u >= V || v >= V || u == v) {
        x.key = ~0ULL;
        x.src = x.dst = 0;
      } else {
        x.src = (uint32_t)u;
        x.dst = (uint32_t)v;
        uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
        x.key = (lo << 32) | hi;
      }
    }
    next_idx += n;
    // merge with what we have, keep the first occurrence of every key
    c.insert(c.end(), uniq.begin(), uniq.end());
    __gnu_parallel::sort(c.begin(), c.end(), [](const Cand &x, const Cand &y) {
      return x.key != y.key ? x.key < y.key : x.idx < y.idx;
    });
    std::vector<Cand> keep;
    keep.reserve(c.size());
    for (size_t i = 0; i < c.size(); i++) {
      if (c[i].key == ~0ULL) break;
      if (i > 0 && c[i].key == c[i - 1].key) continue;
      keep.push_back(c[i]);
    }
    __gnu_parallel::sort(keep.begin(), keep.end(), [](const Cand &x, const Cand &y) { return x.idx < y.idx; });
    if (keep.size() > p->e_target) keep.resize(p->e_target);
    uniq.swap(keep);
  }
  const uint64_t E = uniq.size();

  // ---- optional relabelling, then drop isolated vertices and compact ----
  std::vector<uint32_t> perm;
  if (p->permute_ids) {
    perm.resize(V);
    for (uint64_t i = 0; i < V; i++) perm[i] = (uint32_t)i;
    for (uint64_t i = V - 1; i > 0; i--) {  // Fisher-Yates
      uint64_t j = draw(p->seed ^ 0xA5A5A5A5ULL, 0xFFFFFFFFULL, i) % (i + 1);
      std::swap(perm[i], perm[j]);
    }
  }
  std::vector<uint8_t> touched(V, 0);
  for (auto &e : uniq) {
    if (p->permute_ids) {
      e.src = perm[e.src];
      e.dst = perm[e.dst];
    }
    touched[e.src] = touched[e.dst] = 1;
  }
  std::vector<uint32_t> newid(V, 0xFFFFFFFFu);
  uint32_t nv = 0;
  for (uint64_t v = 0; v < V; v++)
    if (touched[v]) newid[v] = nv++;

  std::vector<felog_edge12> edges(E);
  std::vector<uint64_t> deg(nv, 0);
  for (uint64_t i = 0; i < E; i++) {
    felog_edge12 &e = edges[i];
    e.src = newid[uniq[i].src];
    e.dst = newid[uniq[i].dst];
    uint64_t k = uniq[i].idx;
    if (p->weight_dist == FELOG_WEIGHT_LOGNORMAL) {
      // Box-Muller on two stream values
      double u1 = unit01(draw(p->seed ^ 0x77ULL, k, 1));
      double u2 = unit01(draw(p->seed ^ 0x77ULL, k, 2));
      if (u1 < 1e-300) u1 = 1e-300;
      double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
      e.data = (float)std::exp(p->lognormal_mu + p->lognormal_sigma * z);
    } else {
      uint32_t r24 = (uint32_t)(draw(p->seed ^ 0x77ULL, k, 0) >> 40);  // 24 bits
      e.data = (float)(r24 + 1) * (1.0f / 16777216.0f);                 // (0, 1]
    }
    deg[e.src]++;
    deg[e.dst]++;
  }

  // ---- the held-out split (gtrain.cpp:293-343), see felog_heldout_split ----
  std::vector<uint32_t> tsrc, tdst;
  std::vector<uint8_t> tlab;
  uint64_t npos = heldout_split(edges, nv, p->holdout, p->seed, tsrc, tdst, tlab);
  if (npos == ~0ULL) { delete s; return -3; }
  {
    std::vector<uint64_t> d2(nv, 0);
    for (uint64_t i = 0; i < E - npos; i++) { d2[edges[i].src]++; d2[edges[i].dst]++; }
    deg.swap(d2);
  }
  edges.resize(E - npos);
  uint64_t maxd = 0;
  for (uint32_t v = 0; v < nv; v++) maxd = std::max(maxd, deg[v]);
  s->train.swap(edges);
  s->test_src.swap(tsrc);
  s->test_dst.swap(tdst);
  s->test_label.swap(tlab);
  s->info.v_num = nv;
  s->info.n_full_edges = E;
  s->info.n_train_edges = s->train.size();
  s->info.n_test = s->test_src.size();
  s->info.n_test_pos = npos;
  s->info.max_degree = maxd;
  *out = s;
  return 0;
}

extern "C" int felog_synth_get_info(const felog_synth *s, felog_synth_info *info) {
  if (!s || !info) return -1;
  *info = s->info;
  return 0;
}

extern "C" int felog_synth_copy(const felog_synth *s, felog_edge12 *train, uint32_t *test_src,
                                uint32_t *test_dst, uint8_t *test_label) {
  if (!s) return -1;
  if (train) memcpy(train, s->train.data(), s->train.size() * sizeof(felog_edge12));
  if (test_src) memcpy(test_src, s->test_src.data(), s->test_src.size() * 4);
  if (test_dst) memcpy(test_dst, s->test_dst.data(), s->test_dst.size() * 4);
  if (test_label) memcpy(test_label, s->test_label.data(), s->test_label.size());
  return 0;
}

extern "C" int felog_write_edge_file(const char *path, const felog_edge12 *edges, size_t n) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  size_t w = n ? fwrite(edges, sizeof(felog_edge12), n, f) : 0;
  int rc = fclose(f);
  return (w == n && rc == 0) ? 0 : -1;
}

extern "C" int felog_synth_write_graph(const felog_synth *s, const char *path) {
  if (!s || !path) return -1;
  return felog_write_edge_file(path, s->train.data(), s->train.size());
}

extern "C" void felog_synth_free(felog_synth *s) { delete s; }

extern "C" int felog_read_edge_file(const char *path, felog_edge12 *edges, size_t cap, size_t *n) {
  if (!path || !n) return -1;
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  if (fseek(f, 0, SEEK_END) != 0) { fclose(f); return -1; }
  long sz = ftell(f);
  if (sz < 0) { fclose(f); return -1; }
  size_t total = (size_t)sz / sizeof(felog_edge12);
  *n = total;
  if (!edges) { fclose(f); return 0; }
  if (cap < total) { fclose(f); return -2; }
  fseek(f, 0, SEEK_SET);
  size_t got = fread(edges, sizeof(felog_edge12), total, f);
  fclose(f);
  return got == total ? 0 : -1;
}

extern "C" double felog_auc(const float *scores, const uint8_t *labels, size_t n) {
  std::vector<std::pair<float, uint8_t>> v(n);
  uint64_t npos = 0;
  for (size_t i = 0; i < n; i++) {
    v[i] = {scores[i], labels[i] ? (uint8_t)1 : (uint8_t)0};
    npos += v[i].second;
  }
  uint64_t nneg = n - npos;
  if (npos == 0 || nneg == 0) return std::nan("");
  std::sort(v.begin(), v.end(), [](const std::pair<float, uint8_t> &a, const std::pair<float, uint8_t> &b) {
    return a.first < b.first;
  });
  // rank sum of positives with average ranks for ties (ranks start at 1)
  double rank_sum = 0.0;
  size_t i = 0;
  while (i < n) {
    size_t j = i;
    while (j + 1 < n && v[j + 1].first == v[i].first) j++;
    double avg = 0.5 * ((double)(i + 1) + (double)(j + 1));
    for (size_t k = i; k <= j; k++)
      if (v[k].second) rank_sum += avg;
    i = j + 1;
  }
  double u = rank_sum - (double)npos * (double)(npos + 1) / 2.0;
  return u / ((double)npos * (double)nneg);
}

extern "C" int felog_heldout_split(const felog_edge12 *edges, uint64_t n, uint32_t v_num, double holdout,
                                   uint64_t seed, felog_edge12 *train, uint64_t *n_train, uint32_t *test_src,
                                   uint32_t *test_dst, uint8_t *test_label, uint64_t *n_test) {
  if ((n && (!edges || !train)) || !n_train || !n_test || holdout < 0.0 || holdout >= 1.0) return -1;
  for (uint64_t i = 0; i < n; i++)
    if (edges[i].src >= v_num || edges[i].dst >= v_num) return -1;
  std::vector<felog_edge12> e(edges, edges + n);
  std::vector<uint32_t> ts, td;
  std::vector<uint8_t> tl;
  const uint64_t npos = heldout_split(e, v_num, holdout, seed, ts, td, tl);
  if (npos == ~0ULL) return -3;
  if (ts.size() && (!test_src || !test_dst || !test_label)) return -1;
  *n_train = n - npos;
  *n_test = ts.size();
  if (*n_train) memcpy(train, e.data(), sizeof(felog_edge12) * *n_train);
  if (*n_test) {
    memcpy(test_src, ts.data(), 4 * ts.size());
    memcpy(test_dst, td.data(), 4 * td.size());
    memcpy(test_label, tl.data(), tl.size());
  }
  return 0;
}
