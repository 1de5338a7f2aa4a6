/*
 * felog_tools.h - host-side data tools for the FeLoG graph-embedding path.
 *
 * The reference ships these steps as separate offline executables; this
 * library replaces the ones the hot path's inputs and quality check need:
 *
 *   - the 12-byte binary edge format written by src/tools/gconverter.cpp:69-76
 *     and read by include/storage.hpp:14-61 ({u32 src, u32 dst, f32 data},
 *     include/type.hpp:66-72);
 *   - the link-prediction split of src/tools/gtrain.cpp:293-343 (held-out
 *     positives drawn among edges whose endpoints keep degree >= 1, plus an
 *     equal number of random non-edges);
 *   - a seeded R-MAT generator standing in for the reference's real datasets
 *     (LiveJournal / YouTube, absent from the reference checkout);
 *   - an exact FP64 link-prediction AUC (the reference has none: gtrain.cpp
 *     only writes test edges and labels, gtrain.cpp:345-384).
 *
 * All functions return 0 on success and a negative value on error; the
 * caller owns every buffer it passes in.
 */
#ifndef FELOG_TOOLS_H
#define FELOG_TOOLS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef FELOG_EDGE12_DEFINED
#define FELOG_EDGE12_DEFINED
/* One binary edge record, include/type.hpp:66-72 (Edge<real_t>). */
typedef struct felog_edge12 {
  uint32_t src;
  uint32_t dst;
  float data;
} felog_edge12;
#endif

typedef enum felog_weight_dist {
  FELOG_WEIGHT_UNIFORM01 = 0, /* f32 uniform in (0, 1] */
  FELOG_WEIGHT_LOGNORMAL = 1  /* exp(N(mu, sigma)) */
} felog_weight_dist;

typedef struct felog_synth_params {
  uint64_t seed;
  uint64_t v_target;       /* vertex id space before isolated vertices are dropped */
  uint64_t e_target;       /* unique undirected edges, no self-loops */
  double a, b, c, d;       /* R-MAT quadrant probabilities */
  int weight_dist;         /* felog_weight_dist */
  double lognormal_mu;
  double lognormal_sigma;
  double holdout;          /* fraction of edges held out as test positives */
  int permute_ids;         /* 1: seeded random relabelling before compaction */
} felog_synth_params;

typedef struct felog_synth_info {
  uint64_t v_num;          /* vertices after isolated ones are removed */
  uint64_t n_full_edges;   /* unique undirected edges generated */
  uint64_t n_train_edges;  /* edges left in the training graph */
  uint64_t n_test;         /* test pairs: positives first, then negatives */
  uint64_t n_test_pos;
  uint64_t max_degree;     /* in the training graph, undirected */
} felog_synth_info;

typedef struct felog_synth felog_synth;

int felog_synth_generate(const felog_synth_params *params, felog_synth **out);
int felog_synth_get_info(const felog_synth *s, felog_synth_info *info);
/* train: n_train_edges records; test_src/test_dst/test_label: n_test each (any may be NULL) */
int felog_synth_copy(const felog_synth *s, felog_edge12 *train, uint32_t *test_src,
                     uint32_t *test_dst, uint8_t *test_label);
/* writes the training edges in the 12-byte binary format */
int felog_synth_write_graph(const felog_synth *s, const char *path);
void felog_synth_free(felog_synth *s);

/* Exact Mann-Whitney AUC in FP64 (ties count 1/2). Returns NaN when a class is empty. */
/* The held-out split of the reference's gtrain tool (src/tools/gtrain.cpp:293-343)
 * over n undirected edges: floor(holdout * n) positives (float arithmetic,
 * like the tool's float -s), each drawn by swap-to-tail until both endpoints
 * keep degree >= 1, and as many negatives (pairs that are no edge, distinct as
 * ordered pairs, self pairs allowed, as in the tool), every draw from one
 * 31-bit stream keyed by seed in the tool's order (its rand() calls through
 * get_big_rand).  train: n entries (the kept edges in the tool's swapped
 * order, *n_train of them); test_*: 2 * floor(holdout * n) entries, positives
 * first.  Returns 0, -1 on bad arguments, -3 when a draw loop runs away. */
int felog_heldout_split(const felog_edge12 *edges, uint64_t n, uint32_t v_num, double holdout, uint64_t seed,
                        felog_edge12 *train, uint64_t *n_train, uint32_t *test_src, uint32_t *test_dst,
                        uint8_t *test_label, uint64_t *n_test);
double felog_auc(const float *scores, const uint8_t *labels, size_t n);

/* Reads a 12-byte binary edge file (storage.hpp:40-61 semantics: whole records only).
 * Call with edges == NULL to get the count in *n. */
int felog_read_edge_file(const char *path, felog_edge12 *edges, size_t cap, size_t *n);
int felog_write_edge_file(const char *path, const felog_edge12 *edges, size_t n);

#ifdef __cplusplus
}
#endif
#endif
