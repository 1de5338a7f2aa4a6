/*
 * felog_oracle.h - CPU restatement of FeLoG's graph-embedding hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against; nothing in the shipped library links or calls it.  It is pinned
 * against the reference's own code compiled with the loopback MPI shim
 * (oracle/ref/*): the walk against include/walk.hpp run with injected draws,
 * the trainer's batch plan against src/word2vec.cu's TrainModelThreadMemory,
 * and the skip-gram step against skip_gram_kernel run one sentence at a time.
 * Every function cites the reference lines it restates.
 */
#ifndef FELOG_ORACLE_H
#define FELOG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_edge12 {
  uint32_t src, dst;
  float data;
} orc_edge12;

/* CSR in the reference's adjacency order (graph.hpp:531-575). */
typedef struct orc_csr {
  uint32_t v_num;
  uint64_t e_num;
  uint64_t *row_ptr; /* v_num + 1 */
  uint32_t *nbr;     /* e_num */
  float *data;       /* e_num */
} orc_csr;

int orc_build_csr(const orc_edge12 *edges, uint64_t n, uint32_t v_num, int undirected, orc_csr *out);
void orc_free_csr(orc_csr *c);

/* Correlation state, walk.hpp:272-399 (field order of SetProperty). */
typedef struct orc_corr {
  double Hn, Sn, EnH, EnS, EnHS, EnHH, EnSS, N, R;
} orc_corr;
void orc_corr_init(orc_corr *c);
void orc_corr_iterate(orc_corr *c, double fi);
int orc_corr_stop(const orc_corr *c, uint32_t step, uint32_t min_len);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Native walk draws: counter (start vertex, round, iteration, replica). */
void orc_walk_draw(uint64_t seed, uint32_t start, uint32_t round, uint32_t iter, uint32_t replica,
                   uint32_t deg, uint32_t *index, double *p);

/* Injected draws: streams of walker k (k-th active walker in id order). */
typedef struct orc_draws {
  const uint64_t *idx_off; /* n_active + 1 */
  const uint32_t *idx;
  const uint64_t *p_off; /* n_active + 1 */
  const double *p;
} orc_draws;

typedef struct orc_walk_stats {
  uint64_t n_sentences;
  uint64_t n_tokens;
  uint64_t n_traces;
  uint64_t n_iterations;
  uint64_t n_long; /* walks longer than 64 tokens */
} orc_walk_stats;

/* One walk round, walk.hpp:547-610 + :847-1122 at np = 1, corpus order =
 * ascending walker id (path.hpp:70-109 with one worker).  Returns 0, or -1 if
 * the token buffer is too small, -2 if injected draws run out. */
int orc_walk_round(const orc_csr *g, uint32_t walker_num, const uint8_t *stop_flags, uint32_t min_len,
                   uint64_t seed, uint32_t round, const orc_draws *inj, uint32_t *tokens,
                   uint64_t tok_cap, uint64_t *sent_off, uint32_t *sent_walker, orc_walk_stats *st);

/* Round relative entropy KL(p_degree || q_visits), walk.hpp:754-796. */
double orc_round_kl(const uint32_t *deg, const uint64_t *freq, uint32_t v_num);

/* Learning rate of round r (r = 0, 1, ...), lr_scheduler.hpp:23-31, word2vec.cu:1958. */
float orc_lr(float initial, float decay, int r);

/* ---------------- trainer ---------------- */

/* Vocabulary from degrees, word2vec.cu:834-862 + SortVocab :734-755 (stable). */
int orc_vocab(const uint32_t *deg, uint32_t v_num, long long min_count, uint32_t *vocab_vertex,
              long long *vocab_cn, uint32_t *id2offset, long long *vocab_size, long long *train_words);

/* Unigram table, word2vec.cu:674-694. */
void orc_unigram_table(const long long *vocab_cn, long long vocab_size, int32_t *table, int64_t table_size);

/* Subsampling keep thresholds, word2vec.cu:180-212.  Returns 0 when the
 * reference would build an empty table (no subsampling), 1 otherwise. */
int orc_subsample_thresholds(const long long *vocab_cn, long long vocab_size, double sample,
                             long long train_words, uint16_t *thr);

/* exp table, word2vec.cu:2292-2297 (EXP_TABLE_SIZE 1000, MAX_EXP 6). */
void orc_exp_table(float *table /* 1000 */);

/* Batch plan, word2vec.cu:1133-1248: sentence packing, subsampling, per-batch
 * negatives.  Outputs (caller-sized):
 *   sen[]            kept vocab indices, all batches concatenated
 *   sent_start[]     n_out_sentences + 1 offsets into sen
 *   batch_first[]    n_batches + 1 first-sentence index of each batch
 *   negs[]           n_out_sentences * negative host negatives (batch order)
 * Returns the number of planned sentences, or -1 on overflow. */
typedef struct orc_plan_out {
  int32_t *sen;
  uint64_t sen_cap;
  uint64_t *sent_start;
  uint64_t *batch_first;
  int32_t *negs;
  uint64_t n_sentences;
  uint64_t n_batches;
  uint64_t n_sen;
  uint64_t words_considered;
} orc_plan_out;
int orc_plan_batches(const uint32_t *tokens, const uint64_t *sent_off, uint64_t n_corpus_sent,
                     const uint32_t *id2offset, const uint16_t *thr, int use_thr, const int32_t *table,
                     int64_t table_size, long long vocab_size, int negative, int rank, orc_plan_out *out);

/* skip_gram_kernel, word2vec.cu:442-536 (negative sampling, hs = 0), blocks
 * executed one after another in block order; dim must be a power of two >= 32. */
void orc_skipgram_batch(float *syn0, float *syn1, const float *exp_table, const int32_t *table,
                        int64_t table_size, long long vocab_size, const int32_t *sen,
                        const uint64_t *sent_start, uint64_t first_sentence, uint64_t n_sentences,
                        int window, int dim, int negative, float alpha);

/* Reuse-neg skip-gram, the algorithm of word2vec.cu:368-440 with a true dot
 * product: per context, all K+1 scores from the current rows, then updates. */
void orc_negreuse_batch(float *syn0, float *syn1, const float *exp_table, const int32_t *sen,
                        const uint64_t *sent_start, uint64_t first_sentence, uint64_t n_sentences,
                        const int32_t *negs, int window, int dim, int negative, float alpha);

/* cbow_kernel, word2vec.cu:538-646 (negative sampling, hs = 0). */
/* BF16 storage form of orc_skipgram_batch / orc_cbow_batch (FP32 master rows
 * 0..n_hot-1, stochastically rounded BF16 rows after them; rule in
 * felog_oracle.c).  syn*_bf hold (vocab_size - n_hot) * dim BF16 bit patterns,
 * logical dimension order. */
/* the lane's mixed rounding key of (seed, sentence, pair) */
uint32_t orc_lane_key(uint32_t seed, uint64_t s, uint32_t pair, uint32_t lane);
uint32_t orc_round_sr_seed(uint64_t seed, uint32_t round);
void orc_skipgram_bf16(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                       uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                       long long vocab_size, const int32_t *sen, const uint64_t *sent_start,
                       uint64_t first_sentence, uint64_t n_sentences, int window, int dim, int negative,
                       float alpha);
void orc_negreuse_bf16(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                       uint32_t sr_seed, const float *exp_table, const int32_t *sen, const uint64_t *sent_start,
                       uint64_t first_sentence, uint64_t n_sentences, const int32_t *negs, int window, int dim,
                       int negative, float alpha);
void orc_negreuse_tile(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                       uint32_t sr_seed, const float *exp_table, const int32_t *sen, const uint64_t *sent_start,
                       uint64_t first_sentence, uint64_t n_sentences, const int32_t *negs, int window, int dim,
                       int negative, float alpha);
void orc_window_tile(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                     uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                     long long vocab_size, const int32_t *sen, const uint64_t *sent_start, uint64_t first_sentence,
                     uint64_t n_sentences, int window, int dim, int negative, float alpha);
void orc_negreuse_tile_tc(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                          uint32_t sr_seed, const float *exp_table, const int32_t *sen, const uint64_t *sent_start,
                          uint64_t first_sentence, uint64_t n_sentences, const int32_t *negs, int window, int dim,
                          int negative, float alpha);
void orc_cbow_bf16(float *syn0, uint16_t *syn0_bf, float *syn1, uint16_t *syn1_bf, long long n_hot,
                   uint32_t sr_seed, const float *exp_table, const int32_t *table, int64_t table_size,
                   long long vocab_size, const int32_t *sen, const uint64_t *sent_start, uint64_t first_sentence,
                   uint64_t n_sentences, int window, int dim, int negative, float alpha);
/* Learned walk budget (this project's): per-vertex features (V x 6, FP64)
 * and the MLP's mean loss / gradient over n samples in FP64 (rules in
 * felog_oracle.c). */
void orc_budget_features(const orc_csr *g, const uint64_t *visits, const uint32_t *first_len, double *feat);
double orc_mlp_loss_grad(const float *params, const float *X, const uint8_t *count, const float *length, uint64_t n,
                         double *grad);
void orc_cbow_batch(float *syn0, float *syn1, const float *exp_table, const int32_t *table,
                    int64_t table_size, long long vocab_size, const int32_t *sen,
                    const uint64_t *sent_start, uint64_t first_sentence, uint64_t n_sentences,
                    int window, int dim, int negative, float alpha);

/* InitNet, word2vec.cu:864-902: syn0 from the LCG seeded 1, syn1 = 0. */
void orc_init_net(float *syn0, float *syn1, long long vocab_size, int dim);

/* Per-vertex convergence, word2vec.cu:1448-1506 + :1748-1889 + :2016-2080.
 * Neighbour choice for degree > 30 is a Philox partial Fisher-Yates keyed
 * (seed, round, v) instead of std::shuffle seeded by std::random_device.
 * Updates stop_flags; returns the number of evaluated vertices that stayed
 * unconverged (eva_num); sim[v] gets the mean cosine of evaluated vertices. */
uint64_t orc_convergence(const float *syn0, const uint32_t *id2offset, int dim, const orc_csr *g,
                         uint8_t *stop_flags, uint64_t seed, uint32_t round, float *sim);
void orc_eval_choose(uint64_t seed, uint32_t round, uint32_t v, uint32_t deg, uint32_t *chosen /* 30 */);
float orc_cosine(const float *a, const float *b, int dim);

/* Common neighbours per input edge: the reference's offline tool
 * (src/tools/gcn.cpp:248-357) with one thread.  The CSR holds the input
 * edges (doubled in input order when undirected), each row sorted by
 * neighbour; every input edge, in order, takes the first sorted entry of
 * (src, dst) and, unless that entry already holds a count, intersects the
 * two neighbour lists with the tool's galloping search and corrects the size
 * for src/dst and repeats; the count goes to that entry and to the first entry
 * of (dst, src).  cn[e] is the count held by the first (src, dst) entry.
 * Returns 0, or -1 on a vertex id >= v_num or an allocation failure. */
int orc_common_neighbours(const uint32_t *src, const uint32_t *dst, uint64_t n, uint32_t v_num, int undirected,
                          int32_t *cn);

#ifdef __cplusplus
}
#endif
#endif
