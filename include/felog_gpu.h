/*
 * felog_gpu.h - C ABI of the B200 implementation of FeLoG's graph-embedding
 * hot path: biased random walk with the information-centric stop rule,
 * per-vertex convergence (walk-budget) check, and skip-gram negative-sampling
 * training.  One context owns one GPU's state: the CSR, alias tables, walk
 * corpus, vocabulary, unigram table and embedding tables all stay resident in
 * device memory.  Plain pointers and sizes only; the library allocates device
 * memory, the caller owns every host buffer.  Every call returns a
 * felog_status; felog_last_error() gives the message of the last failure.
 * One context per host thread; all work of a context runs on its own stream.
 *
 * Reference seams each entry point replaces (RocmFang/Info-centric_GE paths):
 *   felog_load_graph        GraphEngine::load_graph, include/graph.hpp:712-919
 *   felog_build_alias       AliasTableContainer (declared, never built),
 *                           include/walk.hpp:87-103
 *   felog_walk_round        one round of WalkEngine::random_walk,
 *                           include/walk.hpp:547-610, :629-752, :847-1122
 *   felog_get_corpus        PathSet::dump -> corpus_t, include/path.hpp:70-109
 *   felog_init_model        ReadVocabFromDegree + InitNet + InitUnigramTable,
 *                           src/word2vec.cu:834-862, :864-902, :674-694
 *   felog_train_round       TrainModelThreadMemory + skip_gram_kernel /
 *                           __sgNegReuse / cbow_kernel, src/word2vec.cu:1133-1273,
 *                           :368-646
 *   felog_budget_check      the evaluation step of TrainModel,
 *                           src/word2vec.cu:2016-2080, :1748-1889, :1448-1506
 *   felog_run               the walk/train round loop of felog main +
 *                           train_corpus_cuda, src/examples/felog.cpp:33-172,
 *                           src/word2vec.cu:1922-2180
 *   felog_write_embeddings  the -emb_output writer, src/word2vec.cu:2112-2127
 *   felog_load_rmat         the synthetic stand-ins of the reference's datasets
 *                           (no reference counterpart), generated on the device
 */
#ifndef FELOG_GPU_H
#define FELOG_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FELOG_ABI_VERSION 3

typedef enum felog_status {
  FELOG_OK = 0,
  FELOG_INVALID_ARG = 1,
  FELOG_OOM = 2,
  FELOG_CUDA_ERROR = 3,
  FELOG_DEVICE_TIMEOUT = 4,
  FELOG_INTERNAL = 5,
  FELOG_IO_ERROR = 6,
  FELOG_NOT_READY = 7
} felog_status;

#ifndef FELOG_EDGE12_DEFINED
#define FELOG_EDGE12_DEFINED
/* One binary edge record, include/type.hpp:66-72 (Edge<real_t>, 12 bytes). */
typedef struct felog_edge12 {
  uint32_t src;
  uint32_t dst;
  float data;
} felog_edge12;
#endif

enum { FELOG_FP32 = 0, FELOG_BF16 = 1 };
enum { FELOG_BUDGET_PLAIN = 0, FELOG_BUDGET_LEARNED = 1 };

typedef struct felog_opts {
  /* graph and walk flags, include/option_helper.hpp:113-121, :161-165 */
  uint32_t v_num;           /* -v */
  uint32_t walker_num;      /* -w; 0 means v_num */
  uint32_t min_length;      /* --min_L (reference default 20, walk.hpp:416) */
  uint32_t min_rounds;      /* --min_R (init_round) */
  uint32_t eval_batch_size; /* --batch_size (accepted, evaluation is one device pass) */
  int32_t make_undirected;  /* --make-undirected */
  /* trainer flags, src/word2vec.cu:2269-2286 (defaults word2vec.cu:163-170) */
  int32_t size;             /* -size (power of two, 32..256) */
  int32_t window;           /* -window */
  int32_t negative;         /* -negative (1..15) */
  int32_t hs;               /* -hs (must be 0) */
  int32_t cbow;             /* -cbow */
  int32_t reuse_neg;        /* -reuse-neg: 1 the reference's pair order; B200 options: 2 one tile per center,
                               3 center tiles scored on the tensor cores (BF16 form), 4 window tiles (the
                               skip-gram windows and draws, each center sharing its first context's K
                               negatives across its contexts) */
  int32_t iter;             /* -iter (parsed, unused like the reference) */
  int32_t min_count;        /* -min-count */
  int32_t classes;          /* -classes (K-means output) */
  int32_t binary;           /* -binary */
  int32_t debug;            /* -debug */
  float sample;             /* -sample */
  float alpha;              /* -alpha (overridden by the LR schedule unless use_cli_alpha) */
  /* B200 options */
  int32_t use_cli_alpha;    /* 0: alpha_r = 0.025 e^(-0.1 r) like the reference */
  int32_t precision;        /* FELOG_FP32 or FELOG_BF16 embedding storage */
  int32_t deterministic;    /* 1: training runs as one warp in sentence order */
  int32_t weighted;         /* 1: candidates drawn from the alias table over edge data */
  int32_t budget_mode;      /* FELOG_BUDGET_PLAIN or FELOG_BUDGET_LEARNED */
  int32_t max_rounds;       /* felog_run stops after this many rounds (0: no cap) */
  int32_t device;           /* CUDA device ordinal */
  int32_t slot_len;         /* tokens reserved per walker before spilling (0: 64) */
  uint64_t seed;            /* Philox key for walks, neighbour choice, rounding */
  uint64_t long_arena_tokens; /* spill arena for long walks (0: automatic) */
  uint64_t wait_limit;      /* spin limit of device-side waits (0: default) */
  int64_t hot_rows;         /* BF16 mode: FP32 master rows (0: the top 1% of the vocabulary, at least 1) */
  float budget_confidence;  /* learned budget: predictions below this softmax confidence fall back (0: 0.9) */
  float budget_audit;       /* learned budget: fraction of confident vertices re-checked (0: 0.05; <0: none) */
  int32_t autotune;         /* 1 (default): the first round picks the pair trainer's launch shape by timing */
  uint32_t stream_walkers;  /* felog_run: walk and train each round in pieces of this many walkers, so the
                               corpus of a whole round is never resident (0: whole rounds) */
  int32_t bf16_reread;      /* BF16 form: read a row again right before its store, so concurrent updates of
                               it are kept (0: for vocabularies below 2^17 rows, 1 always, -1 never) */
} felog_opts;

typedef struct felog_ctx felog_ctx;

/* Injected draws for parity runs: per active walker k (k-th walker in id order
 * whose start vertex is not stopped), the candidate index draws
 * idx[idx_off[k] .. idx_off[k+1]) and the trace draws p[p_off[k] .. p_off[k+1])
 * in the order the walker consumes them (walk.hpp:976, :1005). */
typedef struct felog_draws {
  const uint64_t *idx_off;
  const uint32_t *idx;
  uint64_t n_idx;
  const uint64_t *p_off;
  const double *p;
  uint64_t n_p;
  uint64_t n_walkers;
} felog_draws;

typedef struct felog_walk_stats {
  uint64_t n_sentences;   /* walkers walked (= corpus sentences) */
  uint64_t n_tokens;      /* corpus tokens = walk steps incl. step 0 */
  uint64_t n_traces;      /* go-and-return steps */
  uint64_t n_iterations;  /* candidate draws */
  uint64_t n_long;        /* walks that spilled past slot_len */
  double kl;              /* round relative entropy, walk.hpp:754-787 */
  float ms;               /* device time of the round's walk kernels */
} felog_walk_stats;

typedef struct felog_train_stats {
  uint64_t words;         /* tokens considered by the trainer (before subsampling) */
  uint64_t kept_words;    /* tokens trained on */
  uint64_t pairs;         /* (center, context) updates performed */
  uint64_t sentences;
  uint64_t batches;
  float alpha;
  float ms_plan;
  float ms_train;
} felog_train_stats;

typedef struct felog_budget_stats {
  uint64_t evaluated;     /* vertices checked this round */
  uint64_t unconverged;   /* evaluated vertices still below the threshold (eva_num) */
  uint64_t stopped_total; /* vertices whose walkers are stopped */
  uint64_t predicted;     /* learned mode: vertices decided by the MLP */
  uint64_t audited;       /* learned mode: vertices re-checked by the plain criterion */
  uint64_t overruled;     /* learned mode: predictions the plain criterion reversed */
  int32_t stop_all;       /* 1 when unconverged / previous > 0.7 (word2vec.cu:2073-2078) */
  float ms;
} felog_budget_stats;

typedef struct felog_run_stats {
  uint32_t rounds;
  uint64_t walk_tokens;
  uint64_t train_words;
  double walk_ms;
  double train_ms;
  double budget_ms;
  double total_ms;
  uint64_t final_unconverged;
  uint64_t evaluated;     /* budget checks: vertices the plain criterion evaluated */
  uint64_t predicted;     /* learned mode: vertices decided by the MLP */
  uint64_t audited;       /* learned mode: confident predictions re-checked */
  uint64_t overruled;     /* learned mode: audited predictions the plain criterion reversed */
  uint64_t pairs;         /* (center, context) updates trained */
  double plan_ms;         /* the batch plans' share of train_ms */
} felog_run_stats;

/* ---- lifecycle ---- */
void felog_default_opts(felog_opts *opts);
felog_status felog_create(const felog_opts *opts, felog_ctx **out);
void felog_destroy(felog_ctx *ctx);
const char *felog_last_error(const felog_ctx *ctx);
int felog_abi_version(void);

/* ---- graph ---- */
/* n records of the 12-byte binary format; doubled (e, e^T interleaved) when
 * undirected; CSR bucketed by source in record order (graph.hpp:531-575).
 * Limits: at most 2^32-1 CSR entries (32-bit entry indices; the sorts and
 * scans count in 64 bits) and 2^31-2 vertices (FELOG_INVALID_ARG beyond).
 * Building the CSR of m entries holds 12 n + 24 m bytes of device scratch. */
felog_status felog_load_graph(felog_ctx *ctx, const felog_edge12 *edges, uint64_t n, uint32_t v_num,
                              int undirected);
felog_status felog_load_graph_file(felog_ctx *ctx, const char *path, uint32_t v_num, int undirected);

/* No counterpart in the reference (its datasets are files; this builds the
 * seeded R-MAT stand-ins on the device, at sizes a host edge list cannot
 * carry).  The graph equals felog_synth_generate (include/felog_tools.h) with
 * holdout 0 followed by felog_load_graph of its edges: the first e_target
 * distinct unordered pairs of the counter-based R-MAT candidate stream,
 * optionally permuted, untouched vertices dropped and the rest renumbered,
 * weights uniform in (0, 1] or lognormal (lognormal weights use the device's
 * FP64 log/cos/exp, so a weight may differ from the host's in its last bit).
 * Candidates are drawn (2 e_target at first, up to 2^32) until e_target
 * distinct pairs exist, else the graph keeps the pairs found.  Peak device
 * memory about 24 bytes per candidate, then the CSR build of felog_load_graph.
 * Needs v_target <= 2^31-2 and at most 2^32-1 CSR entries. */
typedef struct felog_rmat_params {
  uint64_t seed;
  uint64_t v_target;       /* vertex ids drawn from [0, v_target) */
  uint64_t e_target;       /* distinct undirected edges wanted */
  double a, b, c, d;       /* quadrant probabilities */
  int32_t lognormal;       /* 0: weights uniform in (0, 1]; 1: lognormal(mu, sigma) */
  double lognormal_mu, lognormal_sigma;
  int32_t permute_ids;     /* 1: relabel vertex ids by the seeded permutation */
} felog_rmat_params;
typedef struct felog_rmat_info {
  uint32_t v_num;          /* vertices kept (ids 0 .. v_num - 1) */
  uint64_t n_edges;        /* undirected edges (records) */
  uint32_t max_degree;
} felog_rmat_info;
felog_status felog_load_rmat(felog_ctx *ctx, const felog_rmat_params *params, int undirected,
                             felog_rmat_info *info);
felog_status felog_graph_info(felog_ctx *ctx, uint32_t *v_num, uint64_t *e_num);
felog_status felog_get_csr(felog_ctx *ctx, uint64_t *row_ptr, uint32_t *nbr, float *data);
felog_status felog_get_degrees(felog_ctx *ctx, uint32_t *deg);
/* Per-vertex alias tables over the edge data (Vose); FELOG_INVALID_ARG for a
 * negative or non-finite weight. prob/alias: e_num entries, optional. */
felog_status felog_build_alias(felog_ctx *ctx);
felog_status felog_get_alias(felog_ctx *ctx, float *prob, uint32_t *alias);

/* No counterpart in the reference.  The same alias tables as
 * felog_build_alias, for callers that cannot allocate device memory (their
 * device memory belongs to their own allocator, or they must not grow their
 * footprint after start-up).  It allocates nothing: inputs and outputs are the
 * caller's device buffers (row_ptr: v_num + 1 u64 CSR offsets; weight, prob,
 * alias: e_num entries) and its worklists live in a fixed device array of
 * FELOG_NOALLOC_MAX_ENTRIES entries (16 MiB) that a GPU holds, once mapped,
 * until exit; larger graphs get FELOG_INVALID_ARG.  CUDA maps that array on a
 * device lazily, at the first call there (with that device current): make
 * one call at start-up, before the caller's own pool reserves the free memory
 * and before any stream capture; a first call that finds no room returns
 * FELOG_OOM.  Every call looks the array's address up again.  Calls share the
 * array, so calls that overlap on the GPU race.
 * stream: a cudaStream_t, or NULL for the default stream; the call
 * synchronizes it.  Returns FELOG_INVALID_ARG for a null buffer, for more than
 * FELOG_NOALLOC_MAX_ENTRIES entries (before touching the device), for edges
 * without vertices, for a vertex whose row_ptr range is out of order or ends
 * past e_num (checked on the device before any worklist access) and for a
 * negative or non-finite weight; FELOG_CUDA_ERROR when a CUDA call fails. */
#define FELOG_NOALLOC_MAX_ENTRIES (1ull << 22)
felog_status felog_build_alias_noalloc(const uint64_t *row_ptr, const float *weight, uint32_t v_num,
                                       uint64_t e_num, float *prob, uint32_t *alias, void *stream);

/* ---- walk ---- */
felog_status felog_set_stop_flags(felog_ctx *ctx, const uint8_t *flags);
felog_status felog_get_stop_flags(felog_ctx *ctx, uint8_t *flags);
/* round: 0-based round index (part of the Philox counter). draws: NULL for the
 * native Philox stream. */
felog_status felog_walk_round(felog_ctx *ctx, uint32_t round, const felog_draws *draws,
                              felog_walk_stats *stats);
/* One piece of a round (no reference counterpart; the reference holds a whole
 * round's corpus): the active walkers first .. first + count - 1 of round
 * `round` walk, and their walks become the corpus, so a caller can train
 * piece by piece and never hold a round's corpus (a 111M-vertex round is
 * about 2.4 G tokens).  first == 0 rebuilds the round's active walker list
 * from the stop flags; *n_active (optional) returns its length.  The walks
 * are those felog_walk_round makes (Philox draws keyed by walker); the
 * round KL is computed with the last piece.  The next felog_train_round
 * trains on the piece with its own rounding seed. */
felog_status felog_walk_piece(felog_ctx *ctx, uint32_t round, uint64_t first, uint64_t count, uint64_t *n_active,
                              felog_walk_stats *stats);
felog_status felog_corpus_size(felog_ctx *ctx, uint64_t *n_sentences, uint64_t *n_tokens);
/* sentences in walker-id order; sent_off: n_sentences + 1 entries */
felog_status felog_get_corpus(felog_ctx *ctx, uint32_t *tokens, uint64_t tok_cap, uint64_t *sent_off,
                              uint64_t off_cap);
/* replace the corpus (training from a given walk file or a test corpus) */
felog_status felog_set_corpus(felog_ctx *ctx, const uint32_t *tokens, const uint64_t *sent_off,
                              uint64_t n_sentences);
felog_status felog_get_visit_freq(felog_ctx *ctx, uint64_t *freq);
/* Attainable-rate ceiling of the last walk round (no reference counterpart):
 * a memory skeleton of that round on the loaded CSR - the same walkers and
 * tokens per walker, the same launch shape, dependent uniform-neighbour
 * gathers at the round's forward-step rate, no arithmetic - timed on the
 * device (best of 3).  ms: its duration; tokens: the tokens it emits.  The
 * corpus is left unchanged. */
felog_status felog_walk_ceiling(felog_ctx *ctx, float *ms, uint64_t *tokens);
/* Walker entries (no counterpart in the reference, whose walker reads its CSR,
 * graph.hpp:531-575): next to the CSR, the library keeps every entry as 16
 * bytes {neighbour, data, the neighbour's first entry, its degree}, so a walk
 * step makes one dependent random read instead of two.  They are built by
 * load_graph / load_rmat when the device has room for them (16 bytes per CSR
 * entry), and the walker and felog_walk_ceiling use them then.
 * keep = 0 frees them (the walker reads the plain CSR from then on, until the
 * next graph load); bytes (may be NULL): their device size afterwards, 0 when
 * the walker reads the plain CSR. */
felog_status felog_walk_entries(felog_ctx *ctx, int keep, uint64_t *bytes);

/* ---- offline edge data ---- */
/* Common neighbours per input edge: the reference's offline tool
 * (src/tools/gcn.cpp:248-357; its CLI is gcn -i -o -v -t -s --make-undirected).
 * src/dst: n input edges (host memory); undirected != 0 doubles them as the
 * tool's --make-undirected does.  cn[e] (host, n entries): the number of
 * common neighbours of src[e] and dst[e] as the tool counts them (repeats and
 * src/dst themselves taken out by its rule; every edge of an unordered pair
 * reports the count of the pair's first edge).  ms (may be NULL): device time
 * of the computation, host copies excluded.  Needs no loaded graph.
 * FELOG_INVALID_ARG on a vertex id >= v_num or more than 2^31 - 1 adjacency
 * entries. */
felog_status felog_common_neighbours(felog_ctx *ctx, const uint32_t *src, const uint32_t *dst, uint64_t n,
                                     uint32_t v_num, int undirected, int32_t *cn, float *ms);

/* ---- trainer ---- */
/* Vocabulary, unigram table and InitNet rows (word2vec.cu:834-902); also starts a new
 * training run: stop flags, visit counts and the budget records are cleared. */
felog_status felog_init_model(felog_ctx *ctx);
/* First slot of every word in the reference's unigram table (replaces the
 * slot-by-slot loop of InitUnigramTable, word2vec.cu:674-694, with the same
 * FP64 sums): counts[0..n) are the vocabulary's counts in vocabulary order
 * (n <= 12.5 M words, the range where the table has the reference's 1e8
 * slots); start[k] receives the first slot holding word k, so slot a holds
 * the last word whose start is <= a (start values past the table's end mean
 * the word gets no slot).  Host only: no device or context needed; init_model
 * builds its table from these starts on the device. */
felog_status felog_unigram_starts(const uint64_t *counts, uint64_t n, uint64_t *start);
felog_status felog_vocab_info(felog_ctx *ctx, uint64_t *vocab_size, uint64_t *train_words);
felog_status felog_get_vocab(felog_ctx *ctx, uint32_t *vocab_vertex, uint32_t *id2offset);
/* alpha < 0: take the schedule value of round `round` */
felog_status felog_train_round(felog_ctx *ctx, uint32_t round, float alpha, felog_train_stats *stats);
/* Row references of the last trained pair-stream chunk (no reference
 * counterpart; for roofline accounting): pairs in the chunk, row references
 * (each pair's context row and its trained target rows) and how many of them
 * hit FP32 master rows (all of them in the FP32 form).  FELOG_NOT_READY before
 * a skip-gram round over the pair stream. */
felog_status felog_pair_row_mix(felog_ctx *ctx, uint64_t *pairs, uint64_t *row_refs, uint64_t *hot_refs);
/* rows in vocabulary order, logical dimension order, FP32 */
felog_status felog_get_embeddings(felog_ctx *ctx, float *syn0, float *syn1, uint64_t cap_floats);
felog_status felog_set_embeddings(felog_ctx *ctx, const float *syn0, const float *syn1);
/* syn0 as felog_get_embeddings returns it, copied to host memory behind the
 * caller's back: the call enqueues a device snapshot and a device-to-host copy
 * on a second stream and returns, so the copy overlaps the next round (the
 * reference copies syn0 back after every round, word2vec.cu:1264, while its
 * trainer waits).  The buffer must stay valid, and should be pinned for the
 * copy to be asynchronous, until felog_wait_embeddings returns.  A later call
 * is ordered after the previous copy. */
felog_status felog_copy_embeddings_async(felog_ctx *ctx, float *syn0, uint64_t cap_floats);
felog_status felog_wait_embeddings(felog_ctx *ctx);
/* No counterpart in the reference (precision study).  For n (context row,
 * target row, label) triples in vocabulary-row indices: dots[i] = the FP32
 * dot of syn0[ctx] and syn1[target] formed exactly as the trainer forms it
 * from the stored rows (FP32 or BF16 storage), and batch_loss[b] = the FP64
 * sum over triples i with batch_of[i] == b of -log sigma(label ? f : -f).
 * Host buffers. */
felog_status felog_score_pairs(felog_ctx *ctx, const int32_t *ctx_rows, const int32_t *tgt_rows,
                               const int8_t *labels, const uint64_t *batch_of, uint64_t n, uint64_t n_batches,
                               float *dots, double *batch_loss);
/* No counterpart in the reference (diagnostic of the BF16 form).  BF16 rows are
 * written back with plain stores (Hogwild), so two warps that update one row
 * at the same time can overwrite each other.  With counting on, the pair
 * trainer keeps a store version per row: a store finding its row's version
 * moved since its warp read the row has overwritten another warp's update.
 * felog_lost_updates: BF16-row updates and overwritten ones since counting
 * was turned on (FP32 master rows add atomically and lose nothing).  Same
 * training otherwise; counting costs an atomic per BF16-row store. */
felog_status felog_count_lost_updates(felog_ctx *ctx, int on);
felog_status felog_lost_updates(felog_ctx *ctx, uint64_t *bf16_updates, uint64_t *lost);
/* the batch plan of the last felog_train_round (parity checks) */
felog_status felog_plan_size(felog_ctx *ctx, uint64_t *n_sentences, uint64_t *n_sen, uint64_t *n_batches);
felog_status felog_get_plan(felog_ctx *ctx, int32_t *sen, uint64_t *sent_start, uint64_t *batch_first,
                            int32_t *negs);

/* ---- budget ---- */
felog_status felog_budget_check(felog_ctx *ctx, uint32_t round, felog_budget_stats *stats);
felog_status felog_get_similarity(felog_ctx *ctx, float *sim);

/* ---- classes ----
 * -classes k output (src/word2vec.cu:2128-2175 writes one class id per
 * vocabulary row): spherical K-means over the resident syn0 rows on the GPU.
 * Objective: the sum over rows of row . centroid(label) for unit centroids;
 * each iteration assigns every row to its largest-dot centroid (ties to the
 * lower index) and then replaces every centroid by the normalised sum of its
 * rows (an empty one keeps its value), so the objective never decreases.
 * Seeds: the normalised rows at vocabulary positions floor((j + 0.5) V / k).
 * Stops after max_iter assignment passes (0: 10) or at the first pass that
 * changes no label.  labels (host, vocab_size entries, vocabulary order),
 * objective (host, max_iter entries: the objective after each assignment
 * pass) and iterations (passes run) are optional.  Deterministic. */
felog_status felog_cluster_embeddings(felog_ctx *ctx, int32_t classes, int32_t max_iter, int32_t *labels,
                                      double *objective, int32_t *iterations);

/* ---- learned walk budget (no reference counterpart) ----
 * A 6 -> 64 -> 64 -> (9 + 1) MLP predicts each vertex's walk count (2..10)
 * and walk length (20..80) from per-vertex features; in FELOG_BUDGET_LEARNED
 * mode felog_budget_check lets confident predictions decide a vertex's stop
 * flag without the convergence check, and runs the plain check (which
 * decides) for the others and for an audited random sample. */
#define FELOG_MLP_PARAMS 5258 /* W1[64][6] b1[64] W2[64][64] b2[64] W3[10][64] b3[10] */
#define FELOG_MLP_STATE (FELOG_MLP_PARAMS + 12) /* + feature mean[6], 1/std[6] */
#define FELOG_MLP_FEATURES 6

typedef struct felog_mlp_opts {
  int32_t epochs;     /* passes over the labelled vertices (0: 8) */
  int32_t batch;      /* samples per Adam step, a multiple of 256 (0: 4096) */
  float lr;           /* Adam step size (0: 3e-3) */
  uint64_t seed;      /* initialisation and shuffling */
} felog_mlp_opts;

typedef struct felog_mlp_stats {
  uint64_t samples;
  uint64_t steps;
  double loss_first;   /* mean loss of the first epoch */
  double loss_last;    /* mean loss of the last epoch */
  double count_accuracy; /* argmax count == label, over all samples */
  double length_mae;   /* mean |predicted length - label| */
  float ms;
} felog_mlp_stats;

/* Raw features of every vertex (V x 6 floats, host, optional):
 * log1p(degree), log1p(weighted degree), entropy of the transition weights,
 * log1p(2-hop degree sum), log1p(visits so far), log1p(first walk length).
 * Needs at least one walk round. */
felog_status felog_budget_features(felog_ctx *ctx, float *features);
/* Labels recorded from the rounds run so far (plain criterion): count = the
 * number of walks a vertex made until a convergence check stopped it (10 when
 * none did), clipped to 2..10; length = its mean walk length, clipped to
 * 20..80.  Host buffers of V entries, optional. */
felog_status felog_budget_labels(felog_ctx *ctx, uint8_t *count, float *length);
/* Trains the MLP on the GPU (own forward/backward/Adam kernels) on this
 * context's features and recorded labels. */
felog_status felog_mlp_train(felog_ctx *ctx, const felog_mlp_opts *opts, felog_mlp_stats *stats);
/* Model state (FELOG_MLP_STATE floats: parameters, then the training graph's
 * feature mean and 1/std, for information) to move a trained model between
 * contexts.  Features are standardized with each graph's own moments, in
 * training and in prediction. */
felog_status felog_mlp_get_params(felog_ctx *ctx, float *state);
felog_status felog_mlp_set_params(felog_ctx *ctx, const float *state);
/* Mean loss gradient over n samples (host buffers; X standardized, n x 6),
 * for checking the backward kernel: grad has FELOG_MLP_PARAMS floats. */
felog_status felog_mlp_gradient(felog_ctx *ctx, const float *params, const float *X, const uint8_t *count,
                                const float *length, uint64_t n, float *grad, double *loss);
/* Inference for every vertex from its current features, standardized over
 * this graph's walked vertices (needs a walk round and a model); outputs (V
 * entries, host, optional) are also kept on the device for the learned budget
 * check. */
felog_status felog_mlp_predict(felog_ctx *ctx, uint8_t *count, float *confidence, float *length);

/* ---- whole loop ---- */
felog_status felog_run(felog_ctx *ctx, felog_run_stats *stats);
/* -emb_output (word2vec.cu:2112-2127): "<V> <dim>\n", then per vocabulary row
 * "<vertex> " + dim x "%lf " + "\n" (-binary 1: the dim floats raw).  Text rows
 * are formatted by all host threads with felog_format_lf's formatter and
 * written in order; the bytes equal the reference's serial fprintf. */
felog_status felog_write_embeddings(felog_ctx *ctx, const char *path);
/* The text writer's number formatter (no reference counterpart): each of the
 * n floats as printf("%lf ") prints it (exact value rounded to six decimals,
 * ties to even).  out: cap bytes; *len: bytes written.  FELOG_INVALID_ARG when
 * cap is too small. */
felog_status felog_format_lf(const float *x, uint64_t n, char *out, uint64_t cap, uint64_t *len);

/* Kernels this library has launched on the context (diagnostics). */
uint64_t felog_kernel_launches(const felog_ctx *ctx);
/* No reference counterpart: what the launch-shape autotuner measured (per-pair time of each candidate
 * register budget of the pair trainer) and chose, or "not tuned". */
const char *felog_tuning_report(const felog_ctx *ctx);
/* Device timer on the context's stream: mark(0) records the start event,
 * mark(1) the stop event; elapsed() synchronizes and returns milliseconds. */
felog_status felog_timer_mark(felog_ctx *ctx, int which);
felog_status felog_timer_elapsed(felog_ctx *ctx, float *ms);

#ifdef __cplusplus
}
#endif
#endif
