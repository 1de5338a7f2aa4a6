// C ABI of the B200 FeLoG hot path (declarations and reference seams in
// include/felog_gpu.h).  One felog_ctx owns one device's resident state and a
// stream; kernels live in the .cuh files next to this one.
#include "felog_gpu.h"

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "budget.cuh"
#include "cluster.cuh"
#include "common.cuh"
#include "gcn.cuh"
#include "graph.cuh"
#include "mlp.cuh"
#include "pairs.cuh"
#include "plan.cuh"
#include "rmat.cuh"
#include "sgns.cuh"
#include "umma.cuh"
#include "walk.cuh"

using namespace felog;

namespace {

constexpr int64_t kTableSize = 100000000;  // table_size, word2vec.cu:171
// Vocabularies up to this size use the reference's table; larger ones a
// table of 8 slots per word (the reference's 1e8 slots would leave most of a
// 111M-word vocabulary without one).
constexpr long long kRefTableMaxVocab = kTableSize / 8;
constexpr uint64_t kPairChunk = 1ull << 27;  // pair records generated and trained per chunk

template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }  // temporaries are freed on every return path
  cudaError_t ensure(size_t want) {
    if (want <= n && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    size_t bytes = std::max<size_t>(want, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = std::max<size_t>(want, 1);
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct Status {
  felog_status s = FELOG_OK;
};

}  // namespace

struct felog_ctx {
  felog_opts o;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t tm0 = nullptr, tm1 = nullptr;  // user timer (felog_timer_mark)
  // asynchronous embedding copies (felog_copy_embeddings_async)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ready = nullptr, copy_done = nullptr;
  bool copy_pending = false;
  std::string err;
  int sm_count = 148;

  // graph
  uint32_t V = 0;
  uint64_t M = 0;
  DevBuf<uint64_t> row_ptr;
  DevBuf<uint2> adj;
  DevBuf<uint4> wadj;  // walker entries (k_fuse_adj); empty without room for them or once the caller frees them
  DevBuf<uint32_t> deg;
  std::vector<uint32_t> h_deg;
  DevBuf<float> alias_prob;
  DevBuf<uint32_t> alias_idx;
  bool has_alias = false;

  // walk
  DevBuf<uint8_t> stop;
  DevBuf<uint32_t> active;
  uint32_t n_active = 0;
  uint32_t chunk_base = 0;  // first active walker of the corpus (streamed rounds; 0 otherwise)
  DevBuf<uint32_t> arena;
  uint64_t arena_cap = 0;
  uint64_t spill_base = 0;
  DevBuf<uint64_t> sent_ptr;
  DevBuf<uint32_t> sent_len;
  uint64_t n_sent = 0, n_tok = 0;
  uint64_t last_walk_tokens = 0, last_walk_traces = 0;  // totals of the last walk round
  uint64_t last_chunk_pairs = 0;  // pair records of the last trained chunk (still in pr_rec)
  uint64_t round_stream_pairs = 0;  // pairs of the round's pair stream (the pair trainer counts none itself)
  bool round_used_stream = false;
  int last_chunk_stride = 0;
  bool corpus_ready = false;
  DevBuf<unsigned int> visit_freq;
  uint64_t words_sum_cum = 0;
  DevBuf<unsigned long long> counters;  // scratch counters
  DevBuf<unsigned int> walk_claim;     // walker claim counter
  DevBuf<int> derr;
  DevBuf<uint64_t> inj_idx_off, inj_p_off;
  DevBuf<uint32_t> inj_idx;
  DevBuf<double> inj_p;
  DevBuf<uint32_t> flags_tmp;
  DevBuf<double> kl_partial;
  DevBuf<double> corr_tab;
  DevBuf<double4> corr_series;
  bool corr_tab_ready = false;

  // vocabulary / model
  long long vocab_size = 0, train_words = 0;
  std::vector<uint32_t> h_vocab_vertex, h_id2offset;
  DevBuf<uint32_t> id2offset;
  DevBuf<uint16_t> thr;
  bool use_thr = false;
  DevBuf<int32_t> table;
  uint64_t table_size = kTableSize;  // unigram slots (more for vocabularies beyond kRefTableMaxVocab)
  DevBuf<uint32_t> table_coarse;  // per 64-slot bucket: first word, top bit when uniform
  DevBuf<float> exp_table;
  DevBuf<float> syn0, syn1;        // FP32 rows 0..n_f32-1 (all rows in FP32 mode)
  DevBuf<uint16_t> syn0_bf, syn1_bf;  // BF16 mode: rows n_f32.. as BF16 bits
  long long n_f32 = 0;
  bool model_ready = false;
  DevBuf<LcgJump> jump;

  // plan
  DevBuf<uint32_t> p_cand, p_draws, p_cons, p_kept, p_blk;
  DevBuf<unsigned long long> p_state, p_neg_state;
  DevBuf<uint64_t> p_out_off, p_batch_first;
  DevBuf<int32_t> p_sen, p_negs;
  DevBuf<uint64_t> pr_count, pr_off;  // pair stream: pairs per sentence, offsets
  DevBuf<int32_t> pr_rec;             // pair stream records
  int pair_minb = 0;                  // autotuned blocks per SM of the pair trainer (0: not tuned yet)
  int tile_minb = 0;                  // autotuned blocks per SM of the tile kernels at -size 128 (0: not tuned yet)
  bool count_lost = false;            // BF16 pair trainer counts overwritten row updates (diagnostic)
  DevBuf<uint32_t> lost_ver0, lost_ver1;
  DevBuf<unsigned long long> lost_tot;
  std::string tuning;                 // what the autotuner measured and chose
  DevBuf<unsigned long long> pr_cstate, pr_jump;
  DevBuf<uint32_t> pr_cfirst;
  int pr_jump_window = -1, pr_jump_k = -1;
  std::vector<uint64_t> h_pr_off;
  uint64_t plan_sent = 0, plan_sen = 0, plan_batches = 0;

  // budget
  DevBuf<float> sim;
  // learned budget: per-vertex records of the rounds run (labels, features)
  DevBuf<uint32_t> bud_walks, bud_len_sum, bud_first_len;
  DevBuf<uint8_t> bud_stop_round;
  DevBuf<float> feat, mlp_params, mlp_m1, mlp_m2, mlp_partial, mlp_norm, mlp_grad, pred_conf, pred_len;
  DevBuf<double> mlp_loss;
  DevBuf<float2> mlp_bc;       // Adam bias corrections per step
  DevBuf<uint32_t> mlp_step;   // first step of the epoch being replayed
  DevBuf<uint32_t> mlp_idx;
  DevBuf<uint8_t> mlp_ycount, pred_count;
  DevBuf<float> mlp_ylen;
  bool mlp_ready = false, pred_ready = false;
  uint64_t last_eva = 0;
  bool have_last_eva = false;

  // cub scratch, output staging, launch count of this library's kernels
  DevBuf<unsigned char> cub_tmp;
  DevBuf<float> out_tmp;
  DevBuf<float> copy_stage;  // syn0 snapshot being copied to the host
  // pinned, device-mapped host buffer for the small readbacks of a round (counts,
  // offsets, flags): a kernel writes it, so a readback never waits behind a bulk
  // copy that occupies the device-to-host copy engine
  uint8_t *mbox = nullptr;
  size_t mbox_cap = 0;
  uint64_t launches = 0;
};

namespace {

felog_status fail(felog_ctx *c, felog_status s, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return s;
}

felog_status cuda_fail(felog_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return fail(c, FELOG_OOM, "%s: out of device memory", what);
  }
  return fail(c, FELOG_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(expr, what)                                   \
  do {                                                   \
    cudaError_t _e = (expr);                             \
    if (_e != cudaSuccess) return cuda_fail(c, _e, what); \
  } while (0)

int grid_for(felog_ctx *c, uint64_t n, int threads, int per_sm = 8) {
  uint64_t g = (n + threads - 1) / threads;
  uint64_t cap = (uint64_t)c->sm_count * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Copies device bytes into the mapped host buffer with plain stores: 16- or
// 4-byte words as far as the source alignment allows, the rest byte by byte.
__global__ void k_to_host(const void *src, void *dst, uint64_t bytes) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t a = (uint64_t)(uintptr_t)src;
  uint64_t body = 0;
  if ((a & 15) == 0) {
    body = bytes & ~(uint64_t)15;
    const uint4 *s = static_cast<const uint4 *>(src);
    uint4 *d = static_cast<uint4 *>(dst);
    for (uint64_t i = t0; i < body / 16; i += stride) d[i] = s[i];
  } else if ((a & 3) == 0) {
    body = bytes & ~(uint64_t)3;
    const uint32_t *s = static_cast<const uint32_t *>(src);
    uint32_t *d = static_cast<uint32_t *>(dst);
    for (uint64_t i = t0; i < body / 4; i += stride) d[i] = s[i];
  }
  const uint8_t *s = static_cast<const uint8_t *>(src);
  uint8_t *d = static_cast<uint8_t *>(dst);
  for (uint64_t i = body + t0; i < bytes; i += stride) d[i] = s[i];
}

// out += sum of x[0..n) (per-warp sums, one atomic per warp)
__global__ void k_sum_u32(const uint32_t *__restrict__ x, uint64_t n, unsigned long long *out) {
  unsigned long long t = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    t += x[i];
  for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0 && t) atomicAdd(out, t);
}

// Synchronous readback of `bytes` device bytes on the context's stream, through
// the mapped host buffer (grown on demand, in 64 KiB steps).
felog_status readback(felog_ctx *c, void *dst, const void *dsrc, size_t bytes, const char *what) {
  if (!bytes) return FELOG_OK;
  if (bytes > c->mbox_cap) {
    CK(cudaStreamSynchronize(c->stream), what);
    if (c->mbox) CK(cudaFreeHost(c->mbox), what);
    c->mbox = nullptr;
    c->mbox_cap = 0;
    const size_t cap = (bytes + 65535) & ~(size_t)65535;
    CK(cudaHostAlloc((void **)&c->mbox, cap, cudaHostAllocMapped), what);
    c->mbox_cap = cap;
  }
  void *dmb = nullptr;
  CK(cudaHostGetDevicePointer(&dmb, c->mbox, 0), what);
  k_to_host<<<grid_for(c, (bytes + 15) / 16, 256), 256, 0, c->stream>>>(dsrc, dmb, bytes);
  c->launches++;
  CK(cudaGetLastError(), what);
  CK(cudaStreamSynchronize(c->stream), what);
  memcpy(dst, c->mbox, bytes);
  return FELOG_OK;
}

#define RB(dst, src, bytes, what)                              \
  do {                                                         \
    felog_status _s = readback(c, (dst), (src), (bytes), what); \
    if (_s != FELOG_OK) return _s;                             \
  } while (0)

felog_status check_dev_err(felog_ctx *c, const char *what) {
  int h = 0;
  RB(&h, c->derr.p, sizeof(int), what);
  if (h == kErrNone) return FELOG_OK;
  CK(cudaMemsetAsync(c->derr.p, 0, sizeof(int), c->stream), what);
  switch (h) {
    case kErrDrawsExhausted: return fail(c, FELOG_INVALID_ARG, "%s: injected draws exhausted or out of range", what);
    case kErrArenaFull: return fail(c, FELOG_OOM, "%s: spill arena for long walks exhausted", what);
    case kErrBadVertex: return fail(c, FELOG_INVALID_ARG, "%s: edge endpoint >= v_num", what);
    case kErrWaitTimeout: return fail(c, FELOG_DEVICE_TIMEOUT, "%s: device wait timed out", what);
    case kErrBadWeight: return fail(c, FELOG_INVALID_ARG, "%s: negative or non-finite edge weight", what);
    case kErrPlanOverflow: return fail(c, FELOG_INTERNAL, "%s: batch plan overflow", what);
    case kErrWalkLimit:
      return fail(c, FELOG_INVALID_ARG, "%s: a walker exceeded %u draws (start vertex whose only neighbour is itself)",
                  what, kWalkIterLimit);
    default: return fail(c, FELOG_INTERNAL, "%s: device error %d", what, h);
  }
}

bool dim_ok(int d) { return d == 32 || d == 64 || d == 128 || d == 256; }

// logical <-> interleaved row layout (see sgns.cuh)
inline size_t phys_index(int dim, int logical) {
  int J = dim / 32;
  int lane = logical % 32, j = logical / 32;
  return (size_t)lane * J + j;
}

}  // namespace

// =================================================================== ABI

extern "C" int felog_abi_version(void) { return FELOG_ABI_VERSION; }

extern "C" void felog_default_opts(felog_opts *o) {
  memset(o, 0, sizeof(*o));
  o->min_length = 20;  // walk.hpp:416
  o->min_rounds = 5;   // walk.hpp:417
  o->eval_batch_size = 16384;
  o->make_undirected = 0;
  o->size = 100;       // word2vec.cu:164
  o->window = 5;
  o->negative = 5;
  o->hs = 0;
  o->cbow = 1;         // word2vec.cu:163
  o->reuse_neg = 1;
  o->iter = 5;
  o->min_count = 5;
  o->classes = 0;
  o->binary = 0;
  o->debug = 2;
  o->sample = 1e-3f;
  o->alpha = 0.025f;
  o->precision = FELOG_FP32;
  o->seed = 0x5EED0001ULL;
  o->slot_len = 64;
  o->autotune = 1;
}

extern "C" felog_status felog_create(const felog_opts *opts, felog_ctx **out) {
  if (!opts || !out) return FELOG_INVALID_ARG;
  *out = nullptr;
  felog_ctx *c = new (std::nothrow) felog_ctx();
  if (!c) return FELOG_OOM;
  c->o = *opts;
  if (c->o.slot_len <= 0) c->o.slot_len = 64;
  c->o.slot_len = (c->o.slot_len + 3) & ~3;
  c->device = opts->device;
  cudaError_t e = cudaSetDevice(c->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e == cudaSuccess) e = cudaEventCreate(&c->tm0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->tm1);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
  if (e == cudaSuccess) e = c->counters.ensure(16);
  if (e == cudaSuccess) e = c->derr.ensure(1);
  if (e == cudaSuccess) e = cudaMemset(c->derr.p, 0, sizeof(int));
  if (e == cudaSuccess) {
    LcgJump j;
    lcg_jump_table(j);
    e = c->jump.ensure(1);
    if (e == cudaSuccess) e = cudaMemcpy(c->jump.p, &j, sizeof j, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    felog_status s = e == cudaErrorMemoryAllocation ? FELOG_OOM : FELOG_CUDA_ERROR;
    felog_destroy(c);
    return s;
  }
  *out = c;
  return FELOG_OK;
}

extern "C" void felog_destroy(felog_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->copy_pending && c->copy_done) cudaEventSynchronize(c->copy_done);
  if (c->copy_ready) cudaEventDestroy(c->copy_ready);
  if (c->copy_done) cudaEventDestroy(c->copy_done);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  c->copy_stage.release();
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->mbox) cudaFreeHost(c->mbox);
  c->row_ptr.release(); c->adj.release(); c->wadj.release(); c->deg.release(); c->alias_prob.release(); c->alias_idx.release();
  c->stop.release(); c->active.release(); c->arena.release(); c->sent_ptr.release(); c->sent_len.release();
  c->visit_freq.release(); c->counters.release(); c->derr.release(); c->inj_idx_off.release();
  c->inj_p_off.release(); c->inj_idx.release(); c->inj_p.release(); c->flags_tmp.release();
  c->kl_partial.release(); c->corr_tab.release(); c->corr_series.release(); c->id2offset.release(); c->thr.release(); c->table.release();
  c->exp_table.release(); c->syn0.release(); c->syn1.release(); c->syn0_bf.release(); c->syn1_bf.release(); c->jump.release();
  c->p_cand.release(); c->p_draws.release(); c->p_cons.release(); c->p_kept.release(); c->p_blk.release();
  c->p_state.release(); c->p_neg_state.release(); c->p_out_off.release(); c->p_batch_first.release();
  c->p_sen.release(); c->table_coarse.release(); c->walk_claim.release(); c->pr_count.release(); c->pr_off.release(); c->pr_rec.release(); c->pr_cstate.release(); c->pr_jump.release(); c->pr_cfirst.release(); c->p_negs.release(); c->sim.release(); c->bud_walks.release(); c->bud_len_sum.release(); c->bud_first_len.release(); c->bud_stop_round.release(); c->feat.release(); c->mlp_params.release(); c->mlp_m1.release(); c->mlp_m2.release(); c->mlp_partial.release(); c->mlp_norm.release(); c->mlp_grad.release(); c->pred_conf.release(); c->pred_len.release(); c->mlp_loss.release(); c->mlp_bc.release(); c->mlp_step.release(); c->mlp_idx.release(); c->mlp_ycount.release(); c->pred_count.release(); c->mlp_ylen.release(); c->cub_tmp.release(); c->out_tmp.release();
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->tm0) cudaEventDestroy(c->tm0);
  if (c->tm1) cudaEventDestroy(c->tm1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" const char *felog_last_error(const felog_ctx *c) { return c ? c->err.c_str() : "null context"; }

// ----------------------------------------------------------------- graph

namespace {

// host threads for init_model's per-word loops: a few, so that a busy shared
// host does not hold a parallel region up on a descheduled thread
#define FELOG_INIT_THREADS 8

// CSR of n device records (3 words each: src, dst, data bits), doubled when
// undirected; the records stay the caller's.  Entry indices are 32-bit, so at
// most 2^32 - 1 directed entries; the sorts and scans count items in 64 bits.
felog_status build_csr(felog_ctx *c, const uint32_t *rec, uint64_t n, uint32_t v_num, int undirected) {
  const uint64_t m = undirected ? 2 * n : n;
  DevBuf<uint32_t> keys, vals, keys2, vals2;
  CK(keys.ensure(m), "load_graph");
  CK(vals.ensure(m), "load_graph");
  CK(keys2.ensure(m), "load_graph");
  CK(vals2.ensure(m), "load_graph");
  CK(c->deg.ensure(v_num), "load_graph");
  CK(c->row_ptr.ensure((size_t)v_num + 1), "load_graph");
  CK(c->adj.ensure(m), "load_graph");
  CK(cudaMemsetAsync(c->deg.p, 0, sizeof(uint32_t) * v_num, c->stream), "load_graph");
  CK(cudaMemsetAsync(c->derr.p, 0, sizeof(int), c->stream), "load_graph");
  if (m) {
    k_expand_edges<<<grid_for(c, m, 256), 256, 0, c->stream>>>(rec, n, undirected, v_num, keys.p, vals.p, c->deg.p,
                                                                  c->derr.p);
    c->launches++;
    CK(cudaGetLastError(), "load_graph: expand");
    int end_bit = 1;
    while (end_bit < 32 && (1ULL << end_bit) < v_num) end_bit++;
    cub::DoubleBuffer<uint32_t> dk(keys.p, keys2.p), dv(vals.p, vals2.p);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int64_t)m, 0, end_bit, c->stream), "load_graph: sort");
    CK(c->cub_tmp.ensure(tmp), "load_graph: sort scratch");
    CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tmp, dk, dv, (int64_t)m, 0, end_bit, c->stream),
       "load_graph: sort");
    k_gather_adj<<<grid_for(c, m, 256), 256, 0, c->stream>>>(rec, dv.Current(), m, undirected, c->adj.p);
    c->launches++;
    CK(cudaGetLastError(), "load_graph: gather");
  }
  // row_ptr = exclusive scan of degrees (u32 -> u64)
  {
    CK(cudaMemsetAsync(c->row_ptr.p, 0, sizeof(uint64_t), c->stream), "load_graph");
    size_t tmp = 0;
    CK(cub::DeviceScan::InclusiveSum(nullptr, tmp, c->deg.p, c->row_ptr.p + 1, (int64_t)v_num, c->stream),
       "load_graph: scan");
    CK(c->cub_tmp.ensure(tmp), "load_graph: scan scratch");
    CK(cub::DeviceScan::InclusiveSum(c->cub_tmp.p, tmp, c->deg.p, c->row_ptr.p + 1, (int64_t)v_num, c->stream),
       "load_graph: scan");
  }
  felog_status s = check_dev_err(c, "load_graph");
  if (s != FELOG_OK) return s;
  c->h_deg.resize(v_num);
  CK(cudaMemcpyAsync(c->h_deg.data(), c->deg.p, sizeof(uint32_t) * v_num, cudaMemcpyDeviceToHost, c->stream),
     "load_graph");
  CK(cudaStreamSynchronize(c->stream), "load_graph");
  keys.release(); vals.release(); keys2.release(); vals2.release();
  c->cub_tmp.release();
  // walker entries (16 B per entry, next to the 8-B CSR entry); without room
  // for them the walk reads the plain CSR
  c->wadj.release();
  if (m) {
    if (c->wadj.ensure(m) == cudaSuccess) {
      k_fuse_adj<<<grid_for(c, m, 256), 256, 0, c->stream>>>(c->row_ptr.p, c->adj.p, m, c->wadj.p);
      c->launches++;
      CK(cudaGetLastError(), "load_graph: walker entries");
    } else {
      cudaGetLastError();
      c->wadj.release();
    }
  }
  c->V = v_num;
  c->M = m;
  c->has_alias = false;
  c->model_ready = false;
  c->corpus_ready = false;
  c->have_last_eva = false;
  c->words_sum_cum = 0;
  CK(c->stop.ensure(v_num), "load_graph");
  CK(cudaMemsetAsync(c->stop.p, 0, v_num, c->stream), "load_graph");
  CK(c->visit_freq.ensure(v_num), "load_graph");
  CK(cudaMemsetAsync(c->visit_freq.p, 0, sizeof(unsigned int) * v_num, c->stream), "load_graph");
  CK(cudaStreamSynchronize(c->stream), "load_graph");
  return FELOG_OK;
}

// the previous graph is gone as soon as its buffers are reused
void forget_graph(felog_ctx *c) {
  c->V = 0;
  c->M = 0;
  c->model_ready = false;
  c->corpus_ready = false;
  c->has_alias = false;
}

}  // namespace

extern "C" felog_status felog_load_graph(felog_ctx *c, const felog_edge12 *edges, uint64_t n, uint32_t v_num,
                                         int undirected) {
  if (!c) return FELOG_INVALID_ARG;
  if (v_num == 0) return fail(c, FELOG_INVALID_ARG, "load_graph: v_num must be > 0");
  if (n && !edges) return fail(c, FELOG_INVALID_ARG, "load_graph: edges is NULL");
  const uint64_t m = undirected ? 2 * n : n;
  // 32-bit entry indices (the sorts count items in 64 bits)
  if (m > 0xFFFFFFFFULL) return fail(c, FELOG_INVALID_ARG, "load_graph: more than 2^32-1 CSR entries");
  if (v_num > 0x7FFFFFFEu) return fail(c, FELOG_INVALID_ARG, "load_graph: more than 2^31-2 vertices");
  forget_graph(c);
  CK(cudaSetDevice(c->device), "load_graph");
  DevBuf<uint32_t> rec;
  CK(rec.ensure(3 * std::max<uint64_t>(n, 1)), "load_graph: records");
  if (n) CK(cudaMemcpyAsync(rec.p, edges, n * 12, cudaMemcpyHostToDevice, c->stream), "load_graph: upload");
  return build_csr(c, rec.p, n, v_num, undirected);
}

extern "C" felog_status felog_load_rmat(felog_ctx *c, const felog_rmat_params *p, int undirected,
                                        felog_rmat_info *info) {
  if (!c || !p) return FELOG_INVALID_ARG;
  const double sum = p->a + p->b + p->c + p->d;
  if (p->v_target < 2 || p->v_target > 0x7FFFFFFEull || p->e_target == 0 || !(sum > 0.999 && sum < 1.001))
    return fail(c, FELOG_INVALID_ARG, "load_rmat: need 2 <= v_target <= 2^31-2, e_target > 0, a+b+c+d = 1");
  if ((undirected ? 2 : 1) * p->e_target > 0xFFFFFFFFull)
    return fail(c, FELOG_INVALID_ARG, "load_rmat: more than 2^32-1 CSR entries");
  forget_graph(c);
  CK(cudaSetDevice(c->device), "load_rmat");
  RmatArgs a{};
  a.hs = rmat_mix64(p->seed ^ 0x5DEECE66DULL);
  a.hw = rmat_mix64((p->seed ^ 0x77ULL) ^ 0x5DEECE66DULL);
  a.V = p->v_target;
  while ((1ULL << a.scale) < a.V) a.scale++;
  a.ta = p->a;
  a.tab = p->a + p->b;
  a.tabc = p->a + p->b + p->c;
  a.lognormal = p->lognormal;
  a.mu = p->lognormal_mu;
  a.sigma = p->lognormal_sigma;
  // candidates until e_target distinct pairs are among them (each try starts
  // over with more; the first e_target pairs in candidate order do not depend
  // on how many candidates were drawn beyond them)
  DevBuf<uint32_t> kept;
  uint64_t E = 0;
  for (uint64_t n = std::min<uint64_t>(2 * p->e_target + 1024, 0xFFFFFFFFull);;) {
    DevBuf<uint64_t> key, key2;
    DevBuf<uint32_t> idx, idx2;
    DevBuf<uint8_t> flag;
    DevBuf<unsigned long long> cnt;
    CK(key.ensure(n), "load_rmat: candidates");
    CK(key2.ensure(n), "load_rmat: candidates");
    CK(idx.ensure(n), "load_rmat: candidates");
    CK(idx2.ensure(n), "load_rmat: candidates");
    CK(cnt.ensure(1), "load_rmat");
    k_rmat_candidates<<<grid_for(c, n, 256), 256, 0, c->stream>>>(a, 0, n, key.p, idx.p);
    c->launches++;
    CK(cudaGetLastError(), "load_rmat: candidates");
    cub::DoubleBuffer<uint64_t> dk(key.p, key2.p);
    cub::DoubleBuffer<uint32_t> dv(idx.p, idx2.p);
    size_t tmp = 0;
    const int end_bit = std::min(64, 32 + a.scale);
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int64_t)n, 0, end_bit, c->stream), "load_rmat: sort");
    CK(c->cub_tmp.ensure(tmp), "load_rmat: sort scratch");
    CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tmp, dk, dv, (int64_t)n, 0, end_bit, c->stream),
       "load_rmat: sort");
    CK(flag.ensure(n), "load_rmat: flags");
    k_rmat_first<<<grid_for(c, n, 256), 256, 0, c->stream>>>(dk.Current(), n, flag.p);
    c->launches++;
    uint32_t *firsts = dk.Current() == key.p ? reinterpret_cast<uint32_t *>(key2.p) : reinterpret_cast<uint32_t *>(key.p);
    tmp = 0;
    CK(cub::DeviceSelect::Flagged(nullptr, tmp, dv.Current(), flag.p, firsts, cnt.p, (int64_t)n, c->stream),
       "load_rmat: select");
    CK(c->cub_tmp.ensure(tmp), "load_rmat: select scratch");
    CK(cub::DeviceSelect::Flagged(c->cub_tmp.p, tmp, dv.Current(), flag.p, firsts, cnt.p, (int64_t)n, c->stream),
       "load_rmat: select");
    unsigned long long U = 0;
    RB(&U, cnt.p, sizeof U, "load_rmat");
    if (U < p->e_target && n < 0xFFFFFFFFull) {
      n = std::min<uint64_t>(n + n / 2, 0xFFFFFFFFull);
      continue;
    }
    // the distinct pairs' first candidates in candidate order, cut at e_target
    uint32_t *sorted = dv.Current() == idx.p ? idx2.p : idx.p;
    cub::DoubleBuffer<uint32_t> dd(firsts, sorted);
    int ib = 1;
    while (ib < 32 && (1ULL << ib) < n) ib++;
    tmp = 0;
    CK(cub::DeviceRadixSort::SortKeys(nullptr, tmp, dd, (int64_t)U, 0, ib, c->stream), "load_rmat: order");
    CK(c->cub_tmp.ensure(tmp), "load_rmat: order scratch");
    CK(cub::DeviceRadixSort::SortKeys(c->cub_tmp.p, tmp, dd, (int64_t)U, 0, ib, c->stream), "load_rmat: order");
    E = std::min<uint64_t>(U, p->e_target);
    CK(kept.ensure(std::max<uint64_t>(E, 1)), "load_rmat");
    CK(cudaMemcpyAsync(kept.p, dd.Current(), 4 * E, cudaMemcpyDeviceToDevice, c->stream), "load_rmat");
    CK(cudaStreamSynchronize(c->stream), "load_rmat");
    break;
  }
  c->cub_tmp.release();
  const uint64_t V = p->v_target;
  // optional relabelling: the host generator's Fisher-Yates (sequential, on the host)
  DevBuf<uint32_t> perm;
  if (p->permute_ids) {
    std::vector<uint32_t> hp(V);
    for (uint64_t i = 0; i < V; i++) hp[i] = (uint32_t)i;
    const uint64_t hf = rmat_mix64((p->seed ^ 0xA5A5A5A5ULL) ^ 0x5DEECE66DULL);
    for (uint64_t i = V - 1; i > 0; i--) std::swap(hp[i], hp[rmat_draw(hf, 0xFFFFFFFFULL, i) % (i + 1)]);
    CK(perm.ensure(V), "load_rmat");
    CK(cudaMemcpy(perm.p, hp.data(), 4 * V, cudaMemcpyHostToDevice), "load_rmat");
  }
  // drop untouched vertices, renumber the rest in increasing order
  DevBuf<uint8_t> touched;
  DevBuf<uint32_t> t32, newid;
  CK(touched.ensure(V), "load_rmat");
  CK(cudaMemsetAsync(touched.p, 0, V, c->stream), "load_rmat");
  if (E) {
    k_rmat_touch<<<grid_for(c, E, 256), 256, 0, c->stream>>>(a, kept.p, E, perm.p, touched.p);
    c->launches++;
  }
  CK(t32.ensure(V + 1), "load_rmat");
  CK(newid.ensure(V + 1), "load_rmat");
  CK(cudaMemsetAsync(t32.p + V, 0, 4, c->stream), "load_rmat");
  k_u8_to_u32<<<grid_for(c, V, 256), 256, 0, c->stream>>>(touched.p, V, t32.p);
  c->launches++;
  size_t tmp = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, t32.p, newid.p, (int64_t)(V + 1), c->stream), "load_rmat: scan");
  CK(c->cub_tmp.ensure(tmp), "load_rmat: scan scratch");
  CK(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tmp, t32.p, newid.p, (int64_t)(V + 1), c->stream),
     "load_rmat: scan");
  uint32_t nv = 0;
  RB(&nv, newid.p + V, 4, "load_rmat");
  touched.release();
  t32.release();
  if (nv == 0) return fail(c, FELOG_INVALID_ARG, "load_rmat: no edges drawn");
  DevBuf<uint32_t> rec;
  CK(rec.ensure(3 * std::max<uint64_t>(E, 1)), "load_rmat: records");
  if (E) {
    k_rmat_records<<<grid_for(c, E, 256), 256, 0, c->stream>>>(a, kept.p, E, perm.p, newid.p, rec.p);
    c->launches++;
    CK(cudaGetLastError(), "load_rmat: records");
  }
  kept.release();
  perm.release();
  newid.release();
  felog_status s = build_csr(c, rec.p, E, nv, undirected);
  if (s != FELOG_OK) return s;
  if (info) {
    memset(info, 0, sizeof(*info));
    info->v_num = nv;
    info->n_edges = E;
    CK(cudaMemsetAsync(c->counters.p, 0, 8, c->stream), "load_rmat");
    k_max_u32<<<grid_for(c, nv, 256), 256, 0, c->stream>>>(c->deg.p, nv, (unsigned int *)c->counters.p);
    c->launches++;
    unsigned int md = 0;
    RB(&md, c->counters.p, 4, "load_rmat");
    info->max_degree = md;
  }
  return FELOG_OK;
}

extern "C" felog_status felog_load_graph_file(felog_ctx *c, const char *path, uint32_t v_num, int undirected) {
  if (!c || !path) return FELOG_INVALID_ARG;
  FILE *f = fopen(path, "rb");
  if (!f) return fail(c, FELOG_IO_ERROR, "cannot open graph file %s", path);
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    fclose(f);
    return fail(c, FELOG_IO_ERROR, "cannot size graph file %s", path);
  }
  size_t n = (size_t)sz / sizeof(felog_edge12);  // whole records only, storage.hpp:49-52
  std::vector<felog_edge12> e(n);
  size_t got = n ? fread(e.data(), sizeof(felog_edge12), n, f) : 0;
  fclose(f);
  if (got != n) return fail(c, FELOG_IO_ERROR, "short read on %s", path);
  return felog_load_graph(c, e.data(), n, v_num, undirected);
}

extern "C" felog_status felog_graph_info(felog_ctx *c, uint32_t *v_num, uint64_t *e_num) {
  if (!c) return FELOG_INVALID_ARG;
  if (v_num) *v_num = c->V;
  if (e_num) *e_num = c->M;
  return FELOG_OK;
}

extern "C" felog_status felog_get_csr(felog_ctx *c, uint64_t *row_ptr, uint32_t *nbr, float *data) {
  if (!c || !c->V) return c ? fail(c, FELOG_NOT_READY, "no graph loaded") : FELOG_INVALID_ARG;
  if (row_ptr)
    CK(cudaMemcpy(row_ptr, c->row_ptr.p, sizeof(uint64_t) * (c->V + 1ULL), cudaMemcpyDeviceToHost), "get_csr");
  if ((nbr || data) && c->M) {
    // in pieces of 2^26 entries (512 MiB), so a 3.2 G-entry CSR needs no host copy of its own
    const uint64_t piece = std::min<uint64_t>(c->M, 1ull << 26);
    std::vector<uint2> a(piece);
    for (uint64_t b = 0; b < c->M; b += piece) {
      const uint64_t n = std::min(piece, c->M - b);
      CK(cudaMemcpy(a.data(), c->adj.p + b, sizeof(uint2) * n, cudaMemcpyDeviceToHost), "get_csr");
      for (uint64_t i = 0; i < n; i++) {
        if (nbr) nbr[b + i] = a[i].x;
        if (data) memcpy(&data[b + i], &a[i].y, 4);
      }
    }
  }
  return FELOG_OK;
}

extern "C" felog_status felog_get_degrees(felog_ctx *c, uint32_t *deg) {
  if (!c || !deg) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  memcpy(deg, c->h_deg.data(), sizeof(uint32_t) * c->V);
  return FELOG_OK;
}

extern "C" felog_status felog_build_alias(felog_ctx *c) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  CK(cudaSetDevice(c->device), "build_alias");
  CK(c->alias_prob.ensure(c->M), "build_alias");
  CK(c->alias_idx.ensure(c->M), "build_alias");
  DevBuf<uint32_t> scratch;
  CK(scratch.ensure(c->M), "build_alias");
  CK(cudaMemsetAsync(c->derr.p, 0, sizeof(int), c->stream), "build_alias");
  k_build_alias<<<grid_for(c, (uint64_t)c->V * 32, 256), 256, 0, c->stream>>>(c->row_ptr.p, c->adj.p, c->V,
                                                                              c->alias_prob.p, c->alias_idx.p,
                                                                              scratch.p, c->derr.p);
  c->launches++;
  CK(cudaGetLastError(), "build_alias");
  felog_status s = check_dev_err(c, "build_alias");
  scratch.release();
  if (s != FELOG_OK) return s;
  c->has_alias = true;
  return FELOG_OK;
}

extern "C" felog_status felog_get_alias(felog_ctx *c, float *prob, uint32_t *alias) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->has_alias) return fail(c, FELOG_NOT_READY, "alias tables not built");
  if (prob) CK(cudaMemcpy(prob, c->alias_prob.p, 4 * c->M, cudaMemcpyDeviceToHost), "get_alias");
  if (alias) CK(cudaMemcpy(alias, c->alias_idx.p, 4 * c->M, cudaMemcpyDeviceToHost), "get_alias");
  return FELOG_OK;
}

// ------------------------------------------------------------------ walk

extern "C" felog_status felog_set_stop_flags(felog_ctx *c, const uint8_t *flags) {
  if (!c || !flags) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  CK(cudaSetDevice(c->device), "set_stop_flags");
  // work still queued on the context's stream (a snapshot for an asynchronous
  // copy) finishes before the flags change
  CK(cudaMemcpyAsync(c->stop.p, flags, c->V, cudaMemcpyHostToDevice, c->stream), "set_stop_flags");
  CK(cudaStreamSynchronize(c->stream), "set_stop_flags");
  return FELOG_OK;
}

extern "C" felog_status felog_get_stop_flags(felog_ctx *c, uint8_t *flags) {
  if (!c || !flags) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  CK(cudaSetDevice(c->device), "get_stop_flags");
  RB(flags, c->stop.p, c->V, "get_stop_flags");
  return FELOG_OK;
}

namespace {

__global__ void k_active_flags(const uint8_t *stop, uint32_t v_num, uint32_t walker_num, uint32_t *flag) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < walker_num; w += gridDim.x * blockDim.x)
    flag[w] = stop[w % v_num] ? 0u : 1u;
}

__global__ void k_active_scatter(const uint32_t *flag, const uint32_t *pos, uint32_t walker_num, uint32_t *active) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < walker_num; w += gridDim.x * blockDim.x)
    if (flag[w]) active[pos[w]] = w;
}

// walkers whose start vertex is not stopped, ascending (walk.hpp:563-572)
felog_status build_active(felog_ctx *c, uint32_t walker_num) {
  CK(c->flags_tmp.ensure(2 * (size_t)walker_num + 2), "walk_round: active");
  CK(c->active.ensure(walker_num), "walk_round: active");
  uint32_t *flag = c->flags_tmp.p, *pos = c->flags_tmp.p + walker_num + 1;
  k_active_flags<<<grid_for(c, walker_num, 256), 256, 0, c->stream>>>(c->stop.p, c->V, walker_num, flag);
  c->launches++;
  size_t tmp = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, flag, pos, (int)walker_num + 1, c->stream), "walk_round: scan");
  CK(c->cub_tmp.ensure(tmp), "walk_round: scan");
  CK(cudaMemsetAsync(flag + walker_num, 0, sizeof(uint32_t), c->stream), "walk_round");
  CK(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tmp, flag, pos, (int)walker_num + 1, c->stream),
     "walk_round: scan");
  k_active_scatter<<<grid_for(c, walker_num, 256), 256, 0, c->stream>>>(flag, pos, walker_num, c->active.p);
  c->launches++;
  uint32_t na = 0;
  RB(&na, pos + walker_num, sizeof(uint32_t), "walk_round");
  c->n_active = na;
  return FELOG_OK;
}

// per start vertex: walks, their total length, the first walk's length
__global__ void k_budget_record_walk(const uint32_t *active, uint32_t n_active, uint32_t v_num,
                                     const uint32_t *sent_len, uint32_t *walks, uint32_t *len_sum,
                                     uint32_t *first_len) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_active; k += gridDim.x * blockDim.x) {
    const uint32_t v = active[k] % v_num;
    const uint32_t old = atomicAdd(&walks[v], 1u);
    atomicAdd(&len_sum[v], sent_len[k]);
    if (old == 0) first_len[v] = sent_len[k];
  }
}

felog_status budget_records(felog_ctx *c) {
  if (c->bud_walks.p && c->bud_walks.n >= c->V) return FELOG_OK;
  CK(c->bud_walks.ensure(c->V), "budget records");
  CK(c->bud_len_sum.ensure(c->V), "budget records");
  CK(c->bud_first_len.ensure(c->V), "budget records");
  CK(c->bud_stop_round.ensure(c->V), "budget records");
  CK(cudaMemsetAsync(c->bud_walks.p, 0, 4 * (size_t)c->V, c->stream), "budget records");
  CK(cudaMemsetAsync(c->bud_len_sum.p, 0, 4 * (size_t)c->V, c->stream), "budget records");
  CK(cudaMemsetAsync(c->bud_first_len.p, 0, 4 * (size_t)c->V, c->stream), "budget records");
  CK(cudaMemsetAsync(c->bud_stop_round.p, 0xFF, (size_t)c->V, c->stream), "budget records");
  return FELOG_OK;
}

felog_status round_kl(felog_ctx *c, double *out) {
  const int nb = 256;
  CK(c->kl_partial.ensure(nb + 1), "kl");
  double deg_sum = (double)c->M;
  double words = (double)c->words_sum_cum;
  if (words <= 0) {
    *out = NAN;
    return FELOG_OK;
  }
  k_kl_partial<<<nb, 256, 0, c->stream>>>(c->deg.p, c->visit_freq.p, c->V, deg_sum, words, c->kl_partial.p);
  c->launches++;
  k_kl_final<<<1, 32, 0, c->stream>>>(c->kl_partial.p, nb, c->kl_partial.p + nb);
  c->launches++;
  RB(out, c->kl_partial.p + nb, sizeof(double), "kl");
  return FELOG_OK;
}

}  // namespace

namespace {

// Walks the active walkers k0 .. k1 - 1 of the round (after build_active);
// their walks become the corpus.  with_kl: also the round relative entropy
// (after the last range of a round).
felog_status walk_range(felog_ctx *c, uint32_t round, const felog_draws *draws, uint32_t k0, uint32_t k1,
                        felog_walk_stats *stats, bool with_kl) {
  felog_status s;
  const uint32_t na = k1 - k0;
  if (draws && draws->n_walkers != na)
    return fail(c, FELOG_INVALID_ARG, "walk_round: draws cover %llu walkers, %u are active",
                (unsigned long long)draws->n_walkers, na);
  const uint64_t slot = (uint64_t)c->o.slot_len;
  uint64_t spill = c->o.long_arena_tokens ? c->o.long_arena_tokens
                                          : std::max<uint64_t>(1u << 20, (uint64_t)na * slot / 8);
  spill = (spill + 3) & ~3ULL;
  c->spill_base = (uint64_t)na * slot;
  c->arena_cap = c->spill_base + spill;
  CK(c->arena.ensure(c->arena_cap), "walk_round: arena");
  CK(c->sent_ptr.ensure((size_t)na + 1), "walk_round");
  CK(c->sent_len.ensure((size_t)na + 1), "walk_round");
  if (draws) {
    CK(c->inj_idx_off.ensure((size_t)na + 1), "walk_round: draws");
    CK(c->inj_p_off.ensure((size_t)na + 1), "walk_round: draws");
    CK(c->inj_idx.ensure(draws->n_idx), "walk_round: draws");
    CK(c->inj_p.ensure(draws->n_p), "walk_round: draws");
    CK(cudaMemcpyAsync(c->inj_idx_off.p, draws->idx_off, 8 * ((size_t)na + 1), cudaMemcpyHostToDevice, c->stream),
       "walk_round: draws");
    CK(cudaMemcpyAsync(c->inj_p_off.p, draws->p_off, 8 * ((size_t)na + 1), cudaMemcpyHostToDevice, c->stream),
       "walk_round: draws");
    if (draws->n_idx)
      CK(cudaMemcpyAsync(c->inj_idx.p, draws->idx, 4 * draws->n_idx, cudaMemcpyHostToDevice, c->stream),
         "walk_round: draws");
    if (draws->n_p)
      CK(cudaMemcpyAsync(c->inj_p.p, draws->p, 8 * draws->n_p, cudaMemcpyHostToDevice, c->stream),
         "walk_round: draws");
  }
  if (!c->corr_tab_ready) {
    CK(c->corr_tab.ensure((kCorrTableS + 1) * (kCorrTableS + 1)), "walk_round: correlation table");
    k_corr_table<<<64, 256, 0, c->stream>>>(c->corr_tab.p);
    c->launches++;
    CK(c->corr_series.ensure(kCorrSeries), "walk_round: correlation series");
    k_corr_series<<<1, 32, 0, c->stream>>>(c->corr_series.p);
    c->launches++;
    CK(cudaGetLastError(), "walk_round: correlation table");
    c->corr_tab_ready = true;
  }
  CK(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * 16, c->stream), "walk_round");
  CK(cudaMemsetAsync(c->derr.p, 0, sizeof(int), c->stream), "walk_round");
  WalkArgs a{};
  a.row_ptr = c->row_ptr.p;
  a.adj = c->adj.p;
  a.wadj = c->wadj.p;
  a.alias_prob = c->alias_prob.p;
  a.alias_idx = c->alias_idx.p;
  a.v_num = c->V;
  a.n_active = na;
  a.active = c->active.p + k0;
  a.min_len = c->o.min_length;
  a.round = round;
  a.seed = c->o.seed;
  a.weighted = c->o.weighted && !draws;
  a.injected = draws != nullptr;
  a.inj_idx_off = c->inj_idx_off.p;
  a.inj_idx = c->inj_idx.p;
  a.inj_p_off = c->inj_p_off.p;
  a.inj_p = c->inj_p.p;
  a.arena = c->arena.p;
  a.slot_len = (uint32_t)slot;
  a.spill_cursor = c->counters.p + 8;
  a.spill_base = c->spill_base;
  a.arena_cap = c->arena_cap;
  a.sent_ptr = c->sent_ptr.p;
  a.sent_len = c->sent_len.p;
  a.visit_freq = c->visit_freq.p;
  a.corr_tab = c->corr_tab.p;
  a.corr_series = c->corr_series.p;
  CK(c->walk_claim.ensure(1), "walk_round");
  CK(cudaMemsetAsync(c->walk_claim.p, 0, 4, c->stream), "walk_round");
  a.next_walker = c->walk_claim.p;
  a.stats = c->counters.p;
  a.err = c->derr.p;
  CK(cudaEventRecord(c->ev0, c->stream), "walk_round");
  if (na) {
    // persistent grid: exactly the blocks that are resident at once, so no
    // block waits for a slot only to find every walker claimed
    void (*kern)(WalkArgs);
    if (a.wadj) kern = a.injected ? k_walk<true, false, true> : a.weighted ? k_walk<false, true, true> : k_walk<false, false, true>;
    else kern = a.injected ? k_walk<true, false, false> : a.weighted ? k_walk<false, true, false> : k_walk<false, false, false>;
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWalkThreads, 0), "walk_round: occupancy");
    const int blocks = c->sm_count * std::max(per_sm, 1);
    kern<<<blocks, kWalkThreads, 0, c->stream>>>(a);
    c->launches++;
    CK(cudaGetLastError(), "walk_round: launch");
  }
  CK(cudaEventRecord(c->ev1, c->stream), "walk_round");
  unsigned long long h[16];
  RB(h, c->counters.p, sizeof h, "walk_round");
  s = check_dev_err(c, "walk_round");
  if (s != FELOG_OK) return s;
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1), "walk_round");
  c->n_sent = na;
  c->n_tok = h[0];
  c->last_walk_tokens = h[0];
  c->last_walk_traces = h[1];
  c->corpus_ready = true;
  s = budget_records(c);
  if (s != FELOG_OK) return s;
  if (na) {
    k_budget_record_walk<<<grid_for(c, na, 256), 256, 0, c->stream>>>(c->active.p + k0, na, c->V, c->sent_len.p,
                                                                     c->bud_walks.p, c->bud_len_sum.p,
                                                                     c->bud_first_len.p);
    c->launches++;
    CK(cudaGetLastError(), "walk_round: budget records");
  }
  c->words_sum_cum += h[0];
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->n_sentences = na;
    stats->n_tokens = h[0];
    stats->n_traces = h[1];
    stats->n_iterations = h[2];
    stats->n_long = h[3];
    stats->ms = ms;
    stats->kl = NAN;
    if (with_kl) {
      s = round_kl(c, &stats->kl);
      if (s != FELOG_OK) return s;
    }
  }
  return FELOG_OK;
}

felog_status walk_prepare(felog_ctx *c) {
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  if (c->o.weighted && !c->has_alias) return fail(c, FELOG_NOT_READY, "weighted walk needs felog_build_alias");
  CK(cudaSetDevice(c->device), "walk_round");
  const uint32_t walker_num = c->o.walker_num ? c->o.walker_num : c->V;
  if (walker_num > 0x7FFFFFFEu) return fail(c, FELOG_INVALID_ARG, "walk_round: more than 2^31-2 walkers");
  return build_active(c, walker_num);
}

}  // namespace

extern "C" felog_status felog_walk_piece(felog_ctx *c, uint32_t round, uint64_t first, uint64_t count,
                                         uint64_t *n_active, felog_walk_stats *stats) {
  if (!c) return FELOG_INVALID_ARG;
  felog_status s;
  if (first == 0) {
    s = walk_prepare(c);
    if (s != FELOG_OK) return s;
  } else if (!c->V) {
    return fail(c, FELOG_NOT_READY, "no graph loaded");
  }
  const uint64_t na = c->n_active;
  if (n_active) *n_active = na;
  if (first > na) return fail(c, FELOG_INVALID_ARG, "walk_piece: first walker %llu past the %llu active ones",
                              (unsigned long long)first, (unsigned long long)na);
  const uint64_t last = std::min<uint64_t>(na, first + count);
  c->chunk_base = (uint32_t)first;
  return walk_range(c, round, nullptr, (uint32_t)first, (uint32_t)last, stats, last == na);
}

extern "C" felog_status felog_walk_round(felog_ctx *c, uint32_t round, const felog_draws *draws,
                                         felog_walk_stats *stats) {
  if (!c) return FELOG_INVALID_ARG;
  felog_status s = walk_prepare(c);
  if (s != FELOG_OK) return s;
  c->chunk_base = 0;
  return walk_range(c, round, draws, 0, c->n_active, stats, true);
}

namespace {
felog_status walk_ceiling_run(felog_ctx *c, DevBuf<uint32_t> &scratch, float *ms) {
  // forward steps per token of the last round: every token but the start and
  // the return tokens of traces came from a gather
  const double fwd = (double)(c->last_walk_tokens - c->n_sent - c->last_walk_traces) / (double)c->last_walk_tokens;
  const uint32_t frac = (uint32_t)std::min(4294967295.0, std::max(0.0, fwd) * 4294967296.0);
  CK(scratch.ensure(c->arena_cap), "walk_ceiling: scratch");
  CK(c->walk_claim.ensure(1), "walk_ceiling");
  int per_sm = 0;
  const bool fused = c->wadj.p != nullptr;
  void (*skel)(const uint64_t *, const uint2 *, const uint4 *, uint32_t, uint32_t, const uint32_t *, const uint64_t *,
               const uint32_t *, uint32_t, uint32_t *, unsigned int *) =
      fused ? k_walk_skeleton<true> : k_walk_skeleton<false>;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, skel, kWalkThreads, 0), "walk_ceiling");
  const int blocks = c->sm_count * std::max(per_sm, 1);
  float best = 0;
  for (int rep = 0; rep < 3; rep++) {
    CK(cudaMemsetAsync(c->walk_claim.p, 0, 4, c->stream), "walk_ceiling");
    CK(cudaEventRecord(c->ev0, c->stream), "walk_ceiling");
    skel<<<blocks, kWalkThreads, 0, c->stream>>>(c->row_ptr.p, c->adj.p, c->wadj.p, c->V, (uint32_t)c->n_sent,
                                                             c->active.p + c->chunk_base, c->sent_ptr.p, c->sent_len.p,
                                                             frac, scratch.p, c->walk_claim.p);
    c->launches++;
    CK(cudaGetLastError(), "walk_ceiling");
    CK(cudaEventRecord(c->ev1, c->stream), "walk_ceiling");
    CK(cudaEventSynchronize(c->ev1), "walk_ceiling");
    float t = 0;
    CK(cudaEventElapsedTime(&t, c->ev0, c->ev1), "walk_ceiling");
    if (rep == 0 || t < best) best = t;
  }
  *ms = best;
  return FELOG_OK;
}
}  // namespace

extern "C" felog_status felog_walk_entries(felog_ctx *c, int keep, uint64_t *bytes) {
  if (!c) return FELOG_INVALID_ARG;
  if (!keep && c->wadj.p) {
    CK(cudaSetDevice(c->device), "walk_entries");
    CK(cudaStreamSynchronize(c->stream), "walk_entries");
    c->wadj.release();
  }
  if (bytes) *bytes = c->wadj.p ? (uint64_t)c->M * sizeof(uint4) : 0;
  return FELOG_OK;
}

extern "C" felog_status felog_walk_ceiling(felog_ctx *c, float *ms, uint64_t *tokens) {
  if (!c || !ms) return FELOG_INVALID_ARG;
  if (!c->corpus_ready || !c->n_sent || !c->last_walk_tokens)
    return fail(c, FELOG_NOT_READY, "walk_ceiling: run a walk round first");
  CK(cudaSetDevice(c->device), "walk_ceiling");
  DevBuf<uint32_t> scratch;
  const felog_status s = walk_ceiling_run(c, scratch, ms);
  scratch.release();
  if (s == FELOG_OK && tokens) *tokens = c->last_walk_tokens;
  return s;
}

namespace {
struct GcnBufs {
  DevBuf<uint32_t> src, dst, nbr, heavy, idx, idx_alt;
  DevBuf<unsigned long long> keys, keys_alt, pkeys, pkeys_alt, n_heavy;
  DevBuf<uint64_t> row_ptr, head, head_scan;
  DevBuf<int32_t> cn_own, cn_out;
  DevBuf<unsigned char> tmp;
  void release() {
    src.release(); dst.release(); nbr.release(); heavy.release(); idx.release(); idx_alt.release();
    keys.release(); keys_alt.release(); pkeys.release(); pkeys_alt.release(); n_heavy.release();
    row_ptr.release(); head.release(); head_scan.release(); cn_own.release(); cn_out.release(); tmp.release();
  }
};

int key_bits(uint32_t v_num) {
  int b = 1;
  while (b < 32 && (1ULL << b) < (uint64_t)v_num) b++;
  return 32 + b;
}

felog_status gcn_run(felog_ctx *c, GcnBufs &B, const uint32_t *src, const uint32_t *dst, uint64_t n, uint32_t v_num,
                     int undirected, int32_t *cn, float *ms) {
  const uint64_t m = undirected ? 2 * n : n;
  CK(B.src.ensure(n), "common_neighbours");
  CK(B.dst.ensure(n), "common_neighbours");
  CK(B.keys.ensure(m), "common_neighbours");
  CK(B.keys_alt.ensure(m), "common_neighbours");
  CK(B.nbr.ensure(m), "common_neighbours");
  CK(B.row_ptr.ensure((size_t)v_num + 1), "common_neighbours");
  CK(B.cn_own.ensure(n), "common_neighbours");
  CK(B.cn_out.ensure(n), "common_neighbours");
  CK(B.heavy.ensure(n), "common_neighbours");
  CK(B.n_heavy.ensure(1), "common_neighbours");
  CK(B.pkeys.ensure(n), "common_neighbours");
  CK(B.pkeys_alt.ensure(n), "common_neighbours");
  CK(B.idx.ensure(n), "common_neighbours");
  CK(B.idx_alt.ensure(n), "common_neighbours");
  CK(B.head.ensure(n), "common_neighbours");
  CK(B.head_scan.ensure(n), "common_neighbours");
  CK(cudaMemcpyAsync(B.src.p, src, 4 * n, cudaMemcpyHostToDevice, c->stream), "common_neighbours");
  CK(cudaMemcpyAsync(B.dst.p, dst, 4 * n, cudaMemcpyHostToDevice, c->stream), "common_neighbours");
  CK(cudaMemsetAsync(c->derr.p, 0, sizeof(int), c->stream), "common_neighbours");
  CK(cudaMemsetAsync(B.n_heavy.p, 0, 8, c->stream), "common_neighbours");
  CK(cudaEventRecord(c->ev0, c->stream), "common_neighbours");
  const int kb = key_bits(v_num);
  k_gcn_keys<<<grid_for(c, n, 256), 256, 0, c->stream>>>(B.src.p, B.dst.p, n, v_num, undirected, B.keys.p, c->derr.p);
  c->launches++;
  // rows sorted by neighbour: one radix sort of (src << 32 | dst)
  cub::DoubleBuffer<unsigned long long> kd(B.keys.p, B.keys_alt.p);
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, kd, (int)m, 0, kb, c->stream), "common_neighbours: sort");
  CK(B.tmp.ensure(tb), "common_neighbours");
  CK(cub::DeviceRadixSort::SortKeys(B.tmp.p, tb, kd, (int)m, 0, kb, c->stream), "common_neighbours: sort");
  k_gcn_rows<<<grid_for(c, std::max<uint64_t>(m, 1), 256), 256, 0, c->stream>>>(kd.Current(), m, v_num, B.row_ptr.p,
                                                                                B.nbr.p);
  c->launches++;
  k_gcn_edges<<<grid_for(c, n, 256), 256, 0, c->stream>>>(B.src.p, B.dst.p, n, B.row_ptr.p, B.nbr.p, B.cn_own.p,
                                                          B.heavy.p, B.n_heavy.p);
  c->launches++;
  k_gcn_heavy<<<c->sm_count * 8, 256, 0, c->stream>>>(B.src.p, B.dst.p, B.heavy.p, B.n_heavy.p, B.row_ptr.p, B.nbr.p,
                                                      B.cn_own.p);
  c->launches++;
  // every edge of an unordered pair takes the count of the pair's first edge
  k_gcn_pair_keys<<<grid_for(c, n, 256), 256, 0, c->stream>>>(B.src.p, B.dst.p, n, B.pkeys.p, B.idx.p);
  c->launches++;
  cub::DoubleBuffer<unsigned long long> pk(B.pkeys.p, B.pkeys_alt.p);
  cub::DoubleBuffer<uint32_t> pv(B.idx.p, B.idx_alt.p);
  tb = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, pk, pv, (int)n, 0, kb, c->stream), "common_neighbours: sort");
  CK(B.tmp.ensure(tb), "common_neighbours");
  CK(cub::DeviceRadixSort::SortPairs(B.tmp.p, tb, pk, pv, (int)n, 0, kb, c->stream), "common_neighbours: sort");
  k_gcn_heads<<<grid_for(c, n, 256), 256, 0, c->stream>>>(pk.Current(), n, B.head.p);
  c->launches++;
  tb = 0;
  CK(cub::DeviceScan::InclusiveScan(nullptr, tb, B.head.p, B.head_scan.p, GcnMax(), (int)n, c->stream),
     "common_neighbours: scan");
  CK(B.tmp.ensure(tb), "common_neighbours");
  CK(cub::DeviceScan::InclusiveScan(B.tmp.p, tb, B.head.p, B.head_scan.p, GcnMax(), (int)n, c->stream),
     "common_neighbours: scan");
  k_gcn_scatter<<<grid_for(c, n, 256), 256, 0, c->stream>>>(pv.Current(), B.head_scan.p, n, B.cn_own.p, B.cn_out.p);
  c->launches++;
  CK(cudaGetLastError(), "common_neighbours");
  CK(cudaEventRecord(c->ev1, c->stream), "common_neighbours");
  felog_status s = check_dev_err(c, "common_neighbours");
  if (s != FELOG_OK) return s;
  CK(cudaMemcpyAsync(cn, B.cn_out.p, 4 * n, cudaMemcpyDeviceToHost, c->stream), "common_neighbours");
  CK(cudaStreamSynchronize(c->stream), "common_neighbours");
  if (ms) CK(cudaEventElapsedTime(ms, c->ev0, c->ev1), "common_neighbours");
  return FELOG_OK;
}
}  // namespace

extern "C" felog_status felog_common_neighbours(felog_ctx *c, const uint32_t *src, const uint32_t *dst, uint64_t n,
                                                uint32_t v_num, int undirected, int32_t *cn, float *ms) {
  if (!c || (n && (!src || !dst || !cn))) return FELOG_INVALID_ARG;
  if ((undirected ? 2 * n : n) >= (1ULL << 31))
    return fail(c, FELOG_INVALID_ARG, "common_neighbours: at most 2^31 - 1 adjacency entries");
  if (ms) *ms = 0;
  if (n == 0) return FELOG_OK;
  // ids are checked here: the device passes index rows with them
  for (uint64_t e = 0; e < n; e++)
    if (src[e] >= v_num || dst[e] >= v_num)
      return fail(c, FELOG_INVALID_ARG, "common_neighbours: edge %llu has an endpoint >= v_num",
                  (unsigned long long)e);
  CK(cudaSetDevice(c->device), "common_neighbours");
  GcnBufs B;
  const felog_status s = gcn_run(c, B, src, dst, n, v_num, undirected, cn, ms);
  B.release();
  return s;
}

extern "C" felog_status felog_pair_row_mix(felog_ctx *c, uint64_t *pairs, uint64_t *row_refs, uint64_t *hot_refs) {
  if (!c || !pairs || !row_refs || !hot_refs) return FELOG_INVALID_ARG;
  if (!c->last_chunk_pairs) return fail(c, FELOG_NOT_READY, "pair_row_mix: no pair-stream chunk trained yet");
  CK(cudaSetDevice(c->device), "pair_row_mix");
  CK(cudaMemsetAsync(c->counters.p + 12, 0, 16, c->stream), "pair_row_mix");
  const uint64_t n = c->last_chunk_pairs;
  k_pair_row_mix<<<grid_for(c, n, 256), 256, 0, c->stream>>>(c->pr_rec.p, n, c->last_chunk_stride,
                                                             c->o.negative + 1, (uint32_t)c->n_f32,
                                                             c->counters.p + 12);
  c->launches++;
  CK(cudaGetLastError(), "pair_row_mix");
  unsigned long long h[2];
  RB(h, c->counters.p + 12, sizeof h, "pair_row_mix");
  *pairs = n;
  *row_refs = h[0];
  *hot_refs = h[1];
  return FELOG_OK;
}

extern "C" felog_status felog_corpus_size(felog_ctx *c, uint64_t *n_sentences, uint64_t *n_tokens) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->corpus_ready) return fail(c, FELOG_NOT_READY, "no corpus");
  if (n_sentences) *n_sentences = c->n_sent;
  if (n_tokens) *n_tokens = c->n_tok;
  return FELOG_OK;
}

extern "C" felog_status felog_get_corpus(felog_ctx *c, uint32_t *tokens, uint64_t tok_cap, uint64_t *sent_off,
                                         uint64_t off_cap) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->corpus_ready) return fail(c, FELOG_NOT_READY, "no corpus");
  if (tok_cap < c->n_tok || off_cap < c->n_sent + 1)
    return fail(c, FELOG_INVALID_ARG, "get_corpus: buffers too small (%llu tokens, %llu sentences)",
                (unsigned long long)c->n_tok, (unsigned long long)c->n_sent);
  std::vector<uint64_t> ptr(c->n_sent);
  std::vector<uint32_t> len(c->n_sent);
  if (c->n_sent) {
    CK(cudaMemcpy(ptr.data(), c->sent_ptr.p, 8 * c->n_sent, cudaMemcpyDeviceToHost), "get_corpus");
    CK(cudaMemcpy(len.data(), c->sent_len.p, 4 * c->n_sent, cudaMemcpyDeviceToHost), "get_corpus");
  }
  std::vector<uint32_t> ar(c->arena_cap);
  if (c->arena_cap) CK(cudaMemcpy(ar.data(), c->arena.p, 4 * c->arena_cap, cudaMemcpyDeviceToHost), "get_corpus");
  uint64_t o = 0;
  sent_off[0] = 0;
  for (uint64_t k = 0; k < c->n_sent; k++) {
    memcpy(tokens + o, ar.data() + ptr[k], 4 * (size_t)len[k]);
    o += len[k];
    sent_off[k + 1] = o;
  }
  return FELOG_OK;
}

extern "C" felog_status felog_set_corpus(felog_ctx *c, const uint32_t *tokens, const uint64_t *sent_off,
                                         uint64_t n_sentences) {
  if (c) c->chunk_base = 0;
  if (!c || !sent_off || (n_sentences && !tokens)) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  uint64_t ntok = sent_off[n_sentences];
  for (uint64_t k = 0; k < n_sentences; k++)
    if (sent_off[k + 1] < sent_off[k]) return fail(c, FELOG_INVALID_ARG, "set_corpus: offsets not ascending");
  for (uint64_t t = 0; t < ntok; t++)
    if (tokens[t] >= c->V) return fail(c, FELOG_INVALID_ARG, "set_corpus: token %llu out of range",
                                       (unsigned long long)t);
  CK(c->arena.ensure(std::max<uint64_t>(ntok, 4)), "set_corpus");
  CK(c->sent_ptr.ensure(n_sentences + 1), "set_corpus");
  CK(c->sent_len.ensure(n_sentences + 1), "set_corpus");
  std::vector<uint64_t> ptr(n_sentences);
  std::vector<uint32_t> len(n_sentences);
  for (uint64_t k = 0; k < n_sentences; k++) {
    ptr[k] = sent_off[k];
    len[k] = (uint32_t)(sent_off[k + 1] - sent_off[k]);
  }
  if (ntok) CK(cudaMemcpy(c->arena.p, tokens, 4 * ntok, cudaMemcpyHostToDevice), "set_corpus");
  if (n_sentences) {
    CK(cudaMemcpy(c->sent_ptr.p, ptr.data(), 8 * n_sentences, cudaMemcpyHostToDevice), "set_corpus");
    CK(cudaMemcpy(c->sent_len.p, len.data(), 4 * n_sentences, cudaMemcpyHostToDevice), "set_corpus");
  }
  c->arena_cap = std::max<uint64_t>(ntok, 4);
  c->n_sent = n_sentences;
  c->last_walk_tokens = 0;  // no walk round behind this corpus
  c->n_tok = ntok;
  c->corpus_ready = true;
  return FELOG_OK;
}

extern "C" felog_status felog_get_visit_freq(felog_ctx *c, uint64_t *freq) {
  if (!c || !freq) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  std::vector<unsigned int> f(c->V);
  CK(cudaMemcpy(f.data(), c->visit_freq.p, 4 * (size_t)c->V, cudaMemcpyDeviceToHost), "get_visit_freq");
  for (uint32_t v = 0; v < c->V; v++) freq[v] = f[v];
  return FELOG_OK;
}

// --------------------------------------------------------------- trainer

namespace {

// FP32 -> BF16 bits, round to nearest even (finite inputs)
__host__ __device__ inline uint32_t bf16_rne(float v) {
#ifdef __CUDA_ARCH__
  const uint32_t b = __float_as_uint(v);
#else
  uint32_t b;
  memcpy(&b, &v, 4);
#endif
  return (b + 0x7FFFu + ((b >> 16) & 1u)) >> 16;
}

// InitNet rows (word2vec.cu:893-896) in the interleaved layout; in BF16 mode
// rows n_f32.. are stored rounded to nearest.
__global__ void k_init_syn0(float *syn0, uint16_t *syn0_bf, uint64_t n_f32, uint64_t vocab_size, int dim,
                            const LcgJump *J) {
  const uint64_t n = vocab_size * (uint64_t)dim;
  const int Jn = dim / 32;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    // element e of the row-major LCG fill: state after e + 1 steps from 1
    unsigned long long s = lcg_jump(*J, 1ULL, e + 1);
    float q = __fdiv_rn((float)(s & 0xFFFF), 65536.0f);
    float v = (float)__ddiv_rn(__dsub_rn((double)q, 0.5), (double)dim);
    uint64_t row = e / dim;
    int logical = (int)(e % dim);
    const uint64_t col = (uint64_t)(logical % 32) * Jn + logical / 32;
    if (row < n_f32) syn0[row * dim + col] = v;
    else syn0_bf[(row - n_f32) * dim + col] = (uint16_t)bf16_rne(v);
  }
}

}  // namespace

namespace {
// vocabulary sort keys: ~degree (a stable ascending sort gives degree descending), vertex id
__global__ void k_vocab_keys(const uint32_t *__restrict__ deg, uint32_t V, uint32_t *__restrict__ key,
                             uint32_t *__restrict__ val) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    key[v] = ~deg[v];
    val[v] = (uint32_t)v;
  }
}
// degree^0.75 per vocabulary row (rows by id2offset; words outside the vocabulary skipped)
__global__ void k_unigram_weights(const uint32_t *__restrict__ deg, const uint32_t *__restrict__ id2offset,
                                  uint32_t V, double *__restrict__ w) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = id2offset[v];
    if (r != 0xFFFFFFFFu) w[r] = pow((double)deg[v], 0.75);
  }
}
// slot a -> first row whose cumulative weight exceeds (a + 1/2) / T of the total
__global__ void k_unigram_fill(const double *__restrict__ cum, uint64_t n, uint64_t T, int32_t *__restrict__ table) {
  const double total = cum[n - 1];
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < T; a += (uint64_t)gridDim.x * blockDim.x) {
    const double x = ((double)a + 0.5) / (double)T * total;
    uint64_t lo = 0, hi = n - 1;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (cum[mid] > x) hi = mid;
      else lo = mid + 1;
    }
    table[a] = (int32_t)lo;
  }
}
// The reference's table (word2vec.cu:674-694) walks the slots in order and
// moves to the next word at most once per slot, when a / T > d1, d1 being the
// running FP64 sum of the words' shares.  With D(k) that sum through word k
// (the same sequential FP64 sum) and firstA(k) the first slot with
// a / T > D(k), the first slot of word k + 1 is max(start(k), firstA(k)) + 1,
// so start(k) = k + max(0, max_{j<k} (firstA(j) - j)): a prefix maximum the
// host takes in one pass.  Slot a then holds the last word whose start is
// <= a (the last word once the walk passes it, as the reference clamps).
__global__ void k_unigram_fill_starts(const uint64_t *__restrict__ start, uint64_t n, uint64_t T,
                                      int32_t *__restrict__ table) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < T; a += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = n - 1;  // last k with start[k] <= a (start[0] = 0)
    while (lo < hi) {
      const uint64_t mid = (lo + hi + 1) >> 1;
      if (start[mid] <= a) lo = mid;
      else hi = mid - 1;
    }
    table[a] = (int32_t)lo;
  }
}
// First slot of every word in the reference's 1e8-slot unigram table (see
// k_unigram_fill_starts): the words' shares cn^0.75 / total, their running
// FP64 sums in the reference's order, the first slot past each sum, and the
// prefix maximum that turns those into first slots.
void unigram_starts(const long long *cn, long long size, uint64_t *start) {
  const double power = 0.75, T = (double)kTableSize;
  std::vector<double> w(size);
  for (long long a = 0; a < size; a++) w[a] = (a > 0 && cn[a] == cn[a - 1]) ? w[a - 1] : pow((double)cn[a], power);
  double twp = 0;
  for (long long a = 0; a < size; a++) twp += w[a];
  // D(k) in the reference's order, then firstA(k) per word (independent,
  // on all host threads), then the prefix maximum
  std::vector<double> dsum(size);
  double d1 = w[0] / twp;
  dsum[0] = d1;
  for (long long k = 1; k < size; k++) dsum[k] = d1 += w[k] / twp;
  std::vector<long long> fa(size);
#pragma omp parallel for schedule(static) num_threads(FELOG_INIT_THREADS) if (size > 65536)
  for (long long k = 0; k < size; k++) {
    // firstA(k): the first slot a with a / T > D(k)
    long long x = (long long)std::floor(dsum[k] * T);
    if (x < 0) x = 0;
    while (x > 0 && (double)(x - 1) / T > dsum[k]) x--;
    while (!((double)x / T > dsum[k])) x++;
    fa[k] = x;
  }
  long long run = 0;  // max_{j<k} (firstA(j) - j), or 0
  for (long long k = 0; k < size; k++) {
    start[k] = (uint64_t)(k + run);
    run = std::max(run, fa[k] - k);
  }
}
}  // namespace

extern "C" felog_status felog_unigram_starts(const uint64_t *counts, uint64_t n, uint64_t *start) {
  if (!counts || !start || n == 0 || n > (uint64_t)kRefTableMaxVocab) return FELOG_INVALID_ARG;
  std::vector<long long> cn(n);
  for (uint64_t i = 0; i < n; i++) cn[i] = (long long)counts[i];
  unigram_starts(cn.data(), (long long)n, start);
  return FELOG_OK;
}

extern "C" felog_status felog_init_model(felog_ctx *c) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  const int dim = c->o.size;
  if (!dim_ok(dim)) return fail(c, FELOG_INVALID_ARG, "-size %d: supported sizes are 32, 64, 128, 256", dim);
  if (c->o.hs) return fail(c, FELOG_INVALID_ARG, "-hs 1 is not supported; use negative sampling");
  if (c->o.negative < 1 || c->o.negative > kMaxNeg)
    return fail(c, FELOG_INVALID_ARG, "-negative %d: supported range is 1..%d", c->o.negative, kMaxNeg);
  if (c->o.window < 1) return fail(c, FELOG_INVALID_ARG, "-window must be >= 1");
  if (c->o.precision != FELOG_FP32 && c->o.precision != FELOG_BF16)
    return fail(c, FELOG_INVALID_ARG, "precision %d: use FELOG_FP32 or FELOG_BF16", c->o.precision);
  CK(cudaSetDevice(c->device), "init_model");
  // vocabulary from degrees: stable sort, degree descending (word2vec.cu:834-862, :734-755),
  // as a stable radix sort of (~degree, vertex) on the device
  const uint32_t V = c->V;
  std::vector<uint32_t> order(V);
  {
    DevBuf<uint32_t> k0, k1, v0, v1;
    CK(k0.ensure(V), "init_model: vocabulary");
    CK(k1.ensure(V), "init_model: vocabulary");
    CK(v0.ensure(V), "init_model: vocabulary");
    CK(v1.ensure(V), "init_model: vocabulary");
    k_vocab_keys<<<grid_for(c, V, 256), 256, 0, c->stream>>>(c->deg.p, V, k0.p, v0.p);
    c->launches++;
    cub::DoubleBuffer<uint32_t> dk(k0.p, k1.p), dv(v0.p, v1.p);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int64_t)V, 0, 32, c->stream), "init_model: sort");
    CK(c->cub_tmp.ensure(tmp), "init_model: sort scratch");
    CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tmp, dk, dv, (int64_t)V, 0, 32, c->stream), "init_model: sort");
    CK(cudaMemcpyAsync(order.data(), dv.Current(), 4 * (size_t)V, cudaMemcpyDeviceToHost, c->stream), "init_model");
    CK(cudaStreamSynchronize(c->stream), "init_model");
  }
  long long size = V, tw = 0;
  for (uint32_t i = 0; i < V; i++) {
    if ((long long)c->h_deg[order[i]] < c->o.min_count && i != 0) size--;
    else tw += c->h_deg[order[i]];
  }
  if (size < 2) return fail(c, FELOG_INVALID_ARG, "vocabulary has fewer than 2 words");
  c->h_vocab_vertex.assign(order.begin(), order.begin() + size);
  c->h_id2offset.assign(V, 0xFFFFFFFFu);
  for (long long i = 0; i < size; i++) c->h_id2offset[order[i]] = (uint32_t)i;
  c->vocab_size = size;
  c->train_words = tw;
  std::vector<long long> cn(size);
  for (long long i = 0; i < size; i++) cn[i] = c->h_deg[order[i]];
  CK(c->id2offset.ensure(V), "init_model");
  CK(cudaMemcpy(c->id2offset.p, c->h_id2offset.data(), 4 * (size_t)V, cudaMemcpyHostToDevice), "init_model");
  if (size <= kRefTableMaxVocab) {
    // unigram table (word2vec.cu:674-694): the reference's 1e8 slots and FP64
    // sums; the first slot of every word on the host (k_unigram_fill_starts
    // has the argument), the slots on the device
    std::vector<uint64_t> start(size);
    unigram_starts(cn.data(), size, start.data());
    c->table_size = kTableSize;
    CK(c->table.ensure(kTableSize), "init_model: unigram table");
    DevBuf<uint64_t> dstart;
    CK(dstart.ensure(size), "init_model: unigram table");
    CK(cudaMemcpyAsync(dstart.p, start.data(), 8 * (size_t)size, cudaMemcpyHostToDevice, c->stream), "init_model");
    k_unigram_fill_starts<<<grid_for(c, kTableSize, 256), 256, 0, c->stream>>>(dstart.p, (uint64_t)size, kTableSize,
                                                                              c->table.p);
    c->launches++;
    CK(cudaGetLastError(), "init_model: unigram table");
    CK(cudaStreamSynchronize(c->stream), "init_model");
  } else {
    // larger vocabularies: 1e8 slots would leave most words without a slot, so
    // the table has the power of two >= 8 x vocabulary slots, slot a holding
    // the first word whose cumulative degree^0.75 exceeds (a + 1/2) / slots of
    // the total (built on the device; a deviation from word2vec.cu:171)
    uint64_t T = 1;
    while (T < 8ull * (uint64_t)size) T <<= 1;
    if (T > 0x80000000ull) return fail(c, FELOG_INVALID_ARG, "init_model: vocabulary too large for the unigram table");
    DevBuf<double> wcum;
    CK(wcum.ensure(size), "init_model: unigram weights");
    k_unigram_weights<<<grid_for(c, size, 256), 256, 0, c->stream>>>(c->deg.p, c->id2offset.p, V, wcum.p);
    c->launches++;
    size_t tmp = 0;
    CK(cub::DeviceScan::InclusiveSum(nullptr, tmp, wcum.p, wcum.p, (int64_t)size, c->stream), "init_model: scan");
    CK(c->cub_tmp.ensure(tmp), "init_model: scan scratch");
    CK(cub::DeviceScan::InclusiveSum(c->cub_tmp.p, tmp, wcum.p, wcum.p, (int64_t)size, c->stream),
       "init_model: scan");
    c->table_size = T;
    CK(c->table.ensure(T), "init_model: unigram table");
    k_unigram_fill<<<grid_for(c, T, 256), 256, 0, c->stream>>>(wcum.p, (uint64_t)size, T, c->table.p);
    c->launches++;
    CK(cudaGetLastError(), "init_model: unigram table");
    CK(cudaStreamSynchronize(c->stream), "init_model");
  }
  c->cub_tmp.release();
  // subsampling thresholds (word2vec.cu:180-212)
  std::vector<uint16_t> thr;
  {
    double sample = c->o.sample;
    if (sample > 0.0 && tw > 0) {
      double stw = sample * (double)tw;
      if (stw > 0.0) {
        thr.assign(size, 65535);
#pragma omp parallel for schedule(static) num_threads(FELOG_INIT_THREADS) if (size > 65536)
        for (long long i = 0; i < size; i++) {
          long long count = cn[i];
          if (count <= 0) continue;
          double prob = (sqrt(count / stw) + 1.0) * (stw / (double)count);
          if (prob > 1.0) prob = 1.0;
          else if (prob < 0.0) prob = 0.0;
          thr[i] = prob >= 1.0 ? 65535 : (uint16_t)(prob * 65535.0 + 0.5);
        }
      }
    }
  }
  // exp table (word2vec.cu:2292-2297), host libm
  float et[1000];
  for (int i = 0; i < 1000; i++) {
    et[i] = expf((i / (float)1000 * 2 - 1) * 6);
    et[i] = et[i] / (et[i] + 1);
  }
  {
    const uint64_t nb = (c->table_size + 63) >> kCoarseShift;
    CK(c->table_coarse.ensure(nb), "init_model: unigram buckets");
    k_unigram_coarse<<<grid_for(c, nb, 256), 256, 0, c->stream>>>(c->table.p, c->table_size, c->table_coarse.p);
    c->launches++;
    CK(cudaGetLastError(), "init_model: unigram buckets");
  }
  c->use_thr = !thr.empty();
  CK(c->thr.ensure(std::max<size_t>(thr.size(), 1)), "init_model");
  if (c->use_thr) CK(cudaMemcpy(c->thr.p, thr.data(), 2 * thr.size(), cudaMemcpyHostToDevice), "init_model");
  CK(c->exp_table.ensure(1000), "init_model");
  CK(cudaMemcpy(c->exp_table.p, et, sizeof et, cudaMemcpyHostToDevice), "init_model");
  // BF16 mode: FP32 master rows for the top 1% of the vocabulary (at least one row)
  c->n_f32 = size;
  if (c->o.precision == FELOG_BF16)
    c->n_f32 = std::min<long long>(size, c->o.hot_rows > 0 ? c->o.hot_rows : std::max<long long>(1, (size + 99) / 100));
  const uint64_t nel = (uint64_t)size * dim;
  const uint64_t nf = (uint64_t)c->n_f32 * dim, nb = nel - nf;
  CK(c->syn0.ensure(nf), "init_model: syn0");
  CK(c->syn1.ensure(nf), "init_model: syn1");
  CK(cudaMemsetAsync(c->syn1.p, 0, 4 * nf, c->stream), "init_model");
  if (nb) {
    CK(c->syn0_bf.ensure(nb), "init_model: syn0 (BF16)");
    CK(c->syn1_bf.ensure(nb), "init_model: syn1 (BF16)");
    CK(cudaMemsetAsync(c->syn1_bf.p, 0, 2 * nb, c->stream), "init_model");
  }
  k_init_syn0<<<grid_for(c, nel, 256), 256, 0, c->stream>>>(c->syn0.p, c->syn0_bf.p, (uint64_t)c->n_f32,
                                                             (uint64_t)size, dim, c->jump.p);
  c->launches++;
  CK(cudaGetLastError(), "init_model");
  CK(c->sim.ensure(V), "init_model");
  CK(cudaMemsetAsync(c->sim.p, 0, 4 * (size_t)V, c->stream), "init_model");
  // a new training run: no stopped walkers, no visits, no budget history
  CK(cudaMemsetAsync(c->stop.p, 0, V, c->stream), "init_model");
  CK(cudaMemsetAsync(c->visit_freq.p, 0, sizeof(unsigned int) * (size_t)V, c->stream), "init_model");
  c->words_sum_cum = 0;
  c->have_last_eva = false;
  c->pred_ready = false;
  if (c->bud_walks.p) {
    CK(cudaMemsetAsync(c->bud_walks.p, 0, 4 * (size_t)V, c->stream), "init_model");
    CK(cudaMemsetAsync(c->bud_len_sum.p, 0, 4 * (size_t)V, c->stream), "init_model");
    CK(cudaMemsetAsync(c->bud_first_len.p, 0, 4 * (size_t)V, c->stream), "init_model");
    CK(cudaMemsetAsync(c->bud_stop_round.p, 0xFF, (size_t)V, c->stream), "init_model");
  }
  CK(cudaStreamSynchronize(c->stream), "init_model");
  c->model_ready = true;
  return FELOG_OK;
}

extern "C" felog_status felog_vocab_info(felog_ctx *c, uint64_t *vocab_size, uint64_t *train_words) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  if (vocab_size) *vocab_size = (uint64_t)c->vocab_size;
  if (train_words) *train_words = (uint64_t)c->train_words;
  return FELOG_OK;
}

extern "C" felog_status felog_get_vocab(felog_ctx *c, uint32_t *vocab_vertex, uint32_t *id2offset) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  if (vocab_vertex) memcpy(vocab_vertex, c->h_vocab_vertex.data(), 4 * c->h_vocab_vertex.size());
  if (id2offset) memcpy(id2offset, c->h_id2offset.data(), 4 * c->h_id2offset.size());
  return FELOG_OK;
}

namespace {

float schedule_alpha(const felog_ctx *c, uint32_t round) {
  // ExponentialDecayLR(0.025, 0.1), lr_scheduler.hpp:23-31: step counts rounds from 0
  float initial = c->o.use_cli_alpha ? c->o.alpha : 0.025f;
  float decay = 0.1f;
  return initial * expf(-decay * (int)round);
}

felog_status plan_round(felog_ctx *c, float *ms) {
  const uint64_t n = c->n_sent;
  CK(c->p_cand.ensure(n + 1), "plan");
  CK(c->p_draws.ensure(n + 1), "plan");
  CK(c->p_cons.ensure(n + 1), "plan");
  CK(c->p_kept.ensure(n + 1), "plan");
  CK(c->p_blk.ensure(n + 1), "plan");
  CK(c->p_state.ensure(n + 1), "plan");
  CK(c->p_out_off.ensure(n + 1), "plan");
  CK(c->p_batch_first.ensure(n + 2), "plan");
  CK(c->p_neg_state.ensure(n + 1), "plan");
  CK(c->p_negs.ensure(n * (uint64_t)c->o.negative + 1), "plan");
  PlanArgs a{};
  a.arena = c->arena.p;
  a.sent_ptr = c->sent_ptr.p;
  a.sent_len = c->sent_len.p;
  a.n_sent = n;
  a.id2offset = c->id2offset.p;
  a.thr = c->use_thr ? c->thr.p : nullptr;
  a.table = c->table.p;
  a.table_size = c->table_size;
  a.vocab_size = c->vocab_size;
  a.negative = c->o.negative;
  a.seed = 0x9E3779B97F4A7C15ULL ^ ((0ULL + 1ULL) << 1) ^ 0x2ULL;  // InitSeedForRank(0, 2), word2vec.cu:146-152
  a.cand = c->p_cand.p;
  a.draws = c->p_draws.p;
  a.considered = c->p_cons.p;
  a.kept = c->p_kept.p;
  a.state = c->p_state.p;
  a.blk = c->p_blk.p;
  a.out_off = c->p_out_off.p;
  a.batch_first = c->p_batch_first.p;
  a.neg_state = c->p_neg_state.p;
  a.max_batches = n + 1;
  a.counters = c->counters.p + 4;
  a.jump = c->jump.p;
  a.err = c->derr.p;
  CK(cudaEventRecord(c->ev0, c->stream), "plan");
  k_plan_scan<<<grid_for(c, n, 256), 256, 0, c->stream>>>(a);
  c->launches++;
  k_plan_batches<1024><<<1, 1024, 0, c->stream>>>(a);
  c->launches++;
  // out_off = exclusive scan of kept
  size_t tmp = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, c->p_kept.p, c->p_out_off.p, (int)(n + 1), c->stream), "plan");
  CK(c->cub_tmp.ensure(tmp), "plan");
  CK(cudaMemsetAsync(c->p_kept.p + n, 0, 4, c->stream), "plan");
  CK(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tmp, c->p_kept.p, c->p_out_off.p, (int)(n + 1), c->stream),
     "plan");
  uint64_t total = 0, nb = 0;
  RB(&total, c->p_out_off.p + n, 8, "plan");
  unsigned long long hc[2];
  RB(hc, c->counters.p + 4, sizeof hc, "plan");
  nb = hc[0];
  CK(c->p_sen.ensure(total + 1), "plan");
  a.sen = c->p_sen.p;
  a.negs = c->p_negs.p;
  k_plan_emit<<<grid_for(c, n, 256), 256, 0, c->stream>>>(a);
  c->launches++;
  if (n) k_plan_negs<<<grid_for(c, n * (uint64_t)c->o.negative, 256), 256, 0, c->stream>>>(a, nb);
  c->launches++;
  CK(cudaGetLastError(), "plan");
  CK(cudaEventRecord(c->ev1, c->stream), "plan");
  felog_status s = check_dev_err(c, "plan");
  if (s != FELOG_OK) return s;
  CK(cudaEventElapsedTime(ms, c->ev0, c->ev1), "plan");
  c->plan_sent = n;
  c->plan_sen = total;
  c->plan_batches = nb;
  return FELOG_OK;
}

template <int D, class P>
void launch_dim(felog_ctx *c, const SgArgs &g, int blocks, int threads) {
  if (c->o.cbow) k_sgns_cbow<D, P><<<blocks, threads, 0, c->stream>>>(g);
  else k_sgns_skipgram_any<D, P><<<blocks, threads, 0, c->stream>>>(g);
}

template <class P>
void launch_trainer(felog_ctx *c, const SgArgs &g, int blocks, int threads) {
  switch (c->o.size) {
    case 32: launch_dim<32, P>(c, g, blocks, threads); break;
    case 64: launch_dim<64, P>(c, g, blocks, threads); break;
    case 128: launch_dim<128, P>(c, g, blocks, threads); break;
    case 256: launch_dim<256, P>(c, g, blocks, threads); break;
  }
}

template <int D, int K, class P, bool RR>
void launch_pairs_minb(felog_ctx *c, const SgArgs &g, int blocks, int threads, uint64_t base, uint64_t s0) {
  // untuned: 5 blocks per SM for BF16 rows (48 registers), 4 for FP32 rows (5 spills)
  const int minb = D >= 256 ? 2 : (c->pair_minb ? c->pair_minb : (P::kBF16 ? 5 : 4));
  constexpr int M2 = 2, M3 = D >= 256 ? 2 : 3, M4 = D >= 256 ? 2 : 4, M5 = D >= 256 ? 2 : 5;
  if (minb == 2)
    k_sgns_train_pairs<D, K, P, M2, RR><<<blocks, threads, 0, c->stream>>>(g, c->pr_rec.p, c->pr_off.p, base, s0);
  else if (minb == 3)
    k_sgns_train_pairs<D, K, P, M3, RR><<<blocks, threads, 0, c->stream>>>(g, c->pr_rec.p, c->pr_off.p, base, s0);
  else if (minb == 5)
    k_sgns_train_pairs<D, K, P, M5, RR><<<blocks, threads, 0, c->stream>>>(g, c->pr_rec.p, c->pr_off.p, base, s0);
  else
    k_sgns_train_pairs<D, K, P, M4, RR><<<blocks, threads, 0, c->stream>>>(g, c->pr_rec.p, c->pr_off.p, base, s0);
}

template <int D, int K, class P>
void launch_pairs_dkp(felog_ctx *c, const SgArgs &g, int blocks, int threads, uint64_t base, uint64_t s0) {
  if constexpr (P::kBF16) {
    if constexpr (D <= 128) {
      if (c->count_lost) {  // diagnostic variant: same training, plus the lost-update count
        SgArgs gc = g;
        gc.ver0 = c->lost_ver0.p;
        gc.ver1 = c->lost_ver1.p;
        gc.lost = c->lost_tot.p;
        if (g.reread)
          k_sgns_train_pairs<D, K, P, 5, true, true><<<blocks, threads, 0, c->stream>>>(gc, c->pr_rec.p, c->pr_off.p,
                                                                                       base, s0);
        else
          k_sgns_train_pairs<D, K, P, 5, false, true><<<blocks, threads, 0, c->stream>>>(gc, c->pr_rec.p, c->pr_off.p,
                                                                                        base, s0);
        return;
      }
    }
    if (g.reread) {
      launch_pairs_minb<D, K, P, true>(c, g, blocks, threads, base, s0);
      return;
    }
  }
  launch_pairs_minb<D, K, P, false>(c, g, blocks, threads, base, s0);
}

template <int K, class P>
void launch_pairs_kp(felog_ctx *c, const SgArgs &g, int blocks, int threads, uint64_t base, uint64_t s0) {
  switch (c->o.size) {
    case 64: launch_pairs_dkp<64, K, P>(c, g, blocks, threads, base, s0); break;
    case 128: launch_pairs_dkp<128, K, P>(c, g, blocks, threads, base, s0); break;
    case 256: launch_pairs_dkp<256, K, P>(c, g, blocks, threads, base, s0); break;
  }
}

// The negative LCG advanced by K j steps, j = 0 .. 2 window (a center with j
// contexts draws K j times): x -> pr_jump[j] x + pr_jump[2 window + 1 + j]
felog_status ensure_jump(felog_ctx *c, const SgArgs &g) {
  const int K = c->o.negative;
  const int nj = 2 * c->o.window + 1;
  if (c->pr_jump_window != c->o.window || c->pr_jump_k != K) {
    std::vector<unsigned long long> jt(2 * (size_t)nj);
    unsigned long long A = 1, C = 0;
    for (int j = 0; j < nj; j++) {
      jt[j] = A;
      jt[nj + j] = C;
      A = A * g.lcg_a[K - 1];
      C = C * g.lcg_a[K - 1] + g.lcg_c[K - 1];
    }
    CK(c->pr_jump.ensure(2 * (size_t)nj), "train: jump table");
    CK(cudaMemcpy(c->pr_jump.p, jt.data(), 8 * jt.size(), cudaMemcpyHostToDevice), "train: jump table");
    c->pr_jump_window = c->o.window;
    c->pr_jump_k = K;
  }
  return FELOG_OK;
}

// Skip-gram with K = 5 or 7 over the pair stream: count the pairs of every
// sentence, scan, then per chunk of at most kPairChunk pairs emit the records
// and train them.
felog_status train_pairs(felog_ctx *c, SgArgs g, int blocks, int threads) {
  const uint64_t n = c->plan_sent;
  const int K = c->o.negative;
  const int stride = pair_stride(K);
  CK(c->pr_count.ensure(n + 1), "train: pair counts");
  CK(c->pr_off.ensure(n + 1), "train: pair offsets");
  PairArgs pa{};
  pa.sen = c->p_sen.p;
  pa.sent_start = c->p_out_off.p;
  pa.blk = c->p_blk.p;
  pa.s0 = 0;
  pa.s1 = n;
  pa.table = c->table.p;
  pa.fm_window = g.fm_window;
  pa.fm_vocab1 = g.fm_vocab1;
  pa.fm_table = make_fastmod((uint32_t)c->table_size);
  pa.window = c->o.window;
  pa.negative = K;
  pa.stride = stride;
  felog_status js = ensure_jump(c, g);
  if (js != FELOG_OK) return js;
  pa.jump_a = c->pr_jump.p;
  pa.jump_c = c->pr_jump.p + 2 * c->o.window + 1;
  CK(c->pr_cstate.ensure(c->plan_sen + 1), "train: center states");
  CK(c->pr_cfirst.ensure(c->plan_sen + 1), "train: center offsets");
  pa.cstate = c->pr_cstate.p;
  pa.cfirst = c->pr_cfirst.p;
  pa.reuse = c->o.reuse_neg ? 1 : 0;
  pa.coarse = c->table_coarse.p;
  pa.sr_seed = g.sr_seed;
  pa.negs = c->p_negs.p;
  pa.count = c->pr_count.p;
  pa.off = c->pr_off.p;
  CK(cudaMemsetAsync(c->pr_count.p + n, 0, 8, c->stream), "train");
  if (n) {
    k_pair_count<<<grid_for(c, n, 256), 256, 0, c->stream>>>(pa);
    c->launches++;
  }
  size_t tmp = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, c->pr_count.p, c->pr_off.p, (int)(n + 1), c->stream), "train");
  CK(c->cub_tmp.ensure(tmp), "train");
  CK(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tmp, c->pr_count.p, c->pr_off.p, (int)(n + 1), c->stream),
     "train");
  uint64_t total = 0;
  RB(&total, c->pr_off.p + n, 8, "train");
  c->round_stream_pairs = total;
  c->round_used_stream = true;
  // chunks of whole sentences
  std::vector<std::pair<uint64_t, uint64_t>> chunks;
  if (total <= kPairChunk) {
    chunks.push_back({0, n});
  } else {
    c->h_pr_off.resize(n + 1);
    RB(c->h_pr_off.data(), c->pr_off.p, 8 * (n + 1), "train");
    uint64_t s0 = 0;
    while (s0 < n) {
      uint64_t s1 = s0 + 1;
      while (s1 < n && c->h_pr_off[s1 + 1] - c->h_pr_off[s0] <= kPairChunk) s1++;
      chunks.push_back({s0, s1});
      s0 = s1;
    }
  }
  const uint64_t cap = std::min<uint64_t>(total, kPairChunk) + 1;
  uint64_t need = cap;
  for (auto &ch : chunks)
    if (total > kPairChunk) need = std::max<uint64_t>(need, c->h_pr_off[ch.second] - c->h_pr_off[ch.first] + 1);
  CK(c->pr_rec.ensure(need * stride), "train: pair records");
  pa.rec = c->pr_rec.p;
  const bool bf = c->o.precision == FELOG_BF16;
  for (auto &ch : chunks) {
    pa.s0 = ch.first;
    pa.s1 = ch.second;
    pa.base = total > kPairChunk ? c->h_pr_off[ch.first] : 0;
    c->last_chunk_pairs = total > kPairChunk ? c->h_pr_off[ch.second] - c->h_pr_off[ch.first] : total;
    c->last_chunk_stride = stride;
    const int eb = grid_for(c, (ch.second - ch.first) * 32, 256);
    if (K == 5) k_pair_emit<5><<<eb, 256, 0, c->stream>>>(pa);
    else k_pair_emit<7><<<eb, 256, 0, c->stream>>>(pa);
    c->launches++;
    // launch-shape autotuner: the first chunk of the first tuned round is
    // trained in four slices of sentences, one per candidate register budget
    // (5, 4, 3 or 2 resident blocks per SM; real work, nothing repeated); the
    // fastest per pair is kept
    const uint64_t nch = ch.second - ch.first;
    constexpr int kCand = 4;
    if (c->o.autotune && !c->o.deterministic && c->o.size <= 128 && c->pair_minb == 0 &&
        nch >= kCand * (uint64_t)blocks * (threads / 32)) {
      const int cand[kCand] = {5, 4, 3, 2};
      cudaEvent_t ev[kCand + 1];
      for (int i = 0; i <= kCand; i++) CK(cudaEventCreate(&ev[i]), "autotune");
      uint64_t bound[kCand + 1];
      for (int i = 0; i <= kCand; i++) bound[i] = ch.first + nch * i / kCand;
      for (int i = 0; i < kCand; i++) {
        CK(cudaMemsetAsync(c->counters.p + 0, 0, 8, c->stream), "train");
        SgArgs gi = g;
        gi.n_sent = bound[i + 1] - bound[i];
        c->pair_minb = cand[i];
        CK(cudaEventRecord(ev[i], c->stream), "autotune");
        if (K == 5) {
          if (bf) launch_pairs_kp<5, RowsBF16>(c, gi, blocks, threads, pa.base, bound[i]);
          else launch_pairs_kp<5, RowsF32>(c, gi, blocks, threads, pa.base, bound[i]);
        } else {
          if (bf) launch_pairs_kp<7, RowsBF16>(c, gi, blocks, threads, pa.base, bound[i]);
          else launch_pairs_kp<7, RowsF32>(c, gi, blocks, threads, pa.base, bound[i]);
        }
        c->launches++;
        CK(cudaGetLastError(), "train_round: launch");
      }
      CK(cudaEventRecord(ev[kCand], c->stream), "autotune");
      uint64_t offs[kCand + 1];
      for (int i = 0; i <= kCand; i++) RB(&offs[i], c->pr_off.p + bound[i], 8, "autotune");
      double best = 1e300;
      int pick = 4;
      char buf[256];
      std::string rep = "pair trainer blocks/SM:";
      for (int i = 0; i < kCand; i++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]), "autotune");
        const double per = ms / (double)std::max<uint64_t>(1, offs[i + 1] - offs[i]);
        snprintf(buf, sizeof buf, " %d -> %.3f ns/pair", cand[i], per * 1e6);
        rep += buf;
        if (per < best) {
          best = per;
          pick = cand[i];
        }
      }
      snprintf(buf, sizeof buf, "; chose %d", pick);
      c->tuning = rep + buf;
      c->pair_minb = pick;
      for (int i = 0; i <= kCand; i++) cudaEventDestroy(ev[i]);
      continue;
    }
    CK(cudaMemsetAsync(c->counters.p + 0, 0, 8, c->stream), "train");  // sentence claim counter
    g.n_sent = ch.second - ch.first;
    if (K == 5) {
      if (bf) launch_pairs_kp<5, RowsBF16>(c, g, blocks, threads, pa.base, pa.s0);
      else launch_pairs_kp<5, RowsF32>(c, g, blocks, threads, pa.base, pa.s0);
    } else {
      if (bf) launch_pairs_kp<7, RowsBF16>(c, g, blocks, threads, pa.base, pa.s0);
      else launch_pairs_kp<7, RowsF32>(c, g, blocks, threads, pa.base, pa.s0);
    }
    c->launches++;
    CK(cudaGetLastError(), "train_round: launch");
  }
  return FELOG_OK;
}

}  // namespace

extern "C" felog_status felog_train_round(felog_ctx *c, uint32_t round, float alpha, felog_train_stats *stats) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  if (!c->corpus_ready) return fail(c, FELOG_NOT_READY, "no corpus");
  // -reuse-neg applies to skip-gram only; with -cbow 1 the CBOW kernel runs (word2vec.cu:1255-1258)
  if (c->o.reuse_neg && !c->o.cbow && (c->o.size < 64 || (c->o.negative != 5 && c->o.negative != 7)))
    return fail(c, FELOG_INVALID_ARG, "-reuse-neg runs skip-gram with -negative 5 or 7 and -size >= 64");
  if (c->o.reuse_neg < 0 || c->o.reuse_neg > 4)
    return fail(c, FELOG_INVALID_ARG,
                "-reuse-neg %d: 0, 1 (pair order), 2 (center tiles), 3 (tensor-core tiles) or 4 (window tiles)",
                c->o.reuse_neg);
  if (c->o.reuse_neg == 3 && !c->o.cbow &&
      (c->o.precision != FELOG_BF16 || (c->o.size != 64 && c->o.size != 128) || 2 * c->o.window > kTileRows))
    return fail(c, FELOG_INVALID_ARG, "-reuse-neg 3 needs the BF16 form, -size 64 or 128 and -window <= %d",
                kTileRows / 2);
  CK(cudaSetDevice(c->device), "train_round");
  if (alpha < 0) alpha = schedule_alpha(c, round);
  float ms_plan = 0, ms_train = 0;
  CK(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * 16, c->stream), "train_round");
  CK(cudaMemsetAsync(c->derr.p, 0, sizeof(int), c->stream), "train_round");
  c->last_chunk_pairs = 0;  // set again if this round trains over the pair stream
  c->round_used_stream = false;
  felog_status s = plan_round(c, &ms_plan);
  if (s != FELOG_OK) return s;
  CK(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * 4, c->stream), "train_round");
  SgArgs g{};
  g.syn0 = c->syn0.p;
  g.syn1 = c->syn1.p;
  g.sen = c->p_sen.p;
  g.sent_start = c->p_out_off.p;
  g.blk = c->p_blk.p;
  g.negs = c->p_negs.p;
  g.n_sent = c->plan_sent;
  g.table = c->table.p;
  g.table_size = c->table_size;
  g.vocab_size = c->vocab_size;
  g.exp_table = c->exp_table.p;
  g.window = c->o.window;
  g.negative = c->o.negative;
  g.alpha = alpha;
  g.next_sent = c->counters.p + 0;
  g.pairs = c->counters.p + 1;
  g.fm_window = make_fastmod((uint32_t)c->o.window);
  g.fm_vocab1 = make_fastmod((uint32_t)(c->vocab_size - 1));
  g.syn0_bf = c->syn0_bf.p;
  g.syn1_bf = c->syn1_bf.p;
  g.n_hot = c->n_f32;
  g.err = c->derr.p;
  // re-read before store: asked for, or automatic below 2^17 vocabulary rows, where
  // thousands of warps share few rows and plain stores would overwrite most concurrent updates
  g.reread = c->o.precision == FELOG_BF16 &&
             (c->o.bf16_reread > 0 || (c->o.bf16_reread == 0 && c->vocab_size < (1ll << 17)));
  g.sr_seed = sr_hash((uint32_t)c->o.seed ^ sr_hash((uint32_t)(c->o.seed >> 32) + round * 0x9E3779B9u));
  // a streamed round trains its pieces one by one; each piece gets its own rounding seed
  if (c->chunk_base) g.sr_seed = sr_hash(g.sr_seed ^ sr_hash(c->chunk_base));
  {
    // negative-draw LCG x -> 25214903917 x + 11 (word2vec.cu:502) composed q + 1 times
    unsigned long long A = 1, C = 0;
    for (int q = 0; q < kMaxNeg; q++) {
      A = A * 25214903917ULL;
      C = C * 25214903917ULL + 11ULL;
      g.lcg_a[q] = A;
      g.lcg_c[q] = C;
    }
  }
  const int blocks = c->o.deterministic ? 1 : c->sm_count * 8;
  const int threads = c->o.deterministic ? 32 : 256;
  CK(cudaEventRecord(c->ev0, c->stream), "train_round");
  if (!c->o.cbow && c->o.reuse_neg == 3) {
    // center tiles scored by tcgen05.mma, four centers (one per warp) per CTA
    // (k_sgns_tile_umma); one working warp in the deterministic mode
    const int tb = c->o.deterministic ? 1 : c->sm_count * 4;
    const int workers = c->o.deterministic ? 1 : kUmmaWarps;
    const int K = c->o.negative, D = c->o.size;
#define FELOG_UMMA(DD, KK)                                                                                      \
  do {                                                                                                         \
    CK(cudaFuncSetAttribute(k_sgns_tile_umma<DD, KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,             \
                            (int)UmmaSmem<DD>::kDynamic),                                                      \
       "train_round: tile shared memory");                                                                     \
    k_sgns_tile_umma<DD, KK><<<tb, 32 * kUmmaWarps, UmmaSmem<DD>::kDynamic, c->stream>>>(g, workers);         \
  } while (0)
    if (K == 5 && D == 64) FELOG_UMMA(64, 5);
    else if (K == 5 && D == 128) FELOG_UMMA(128, 5);
    else if (K == 7 && D == 64) FELOG_UMMA(64, 7);
    else FELOG_UMMA(128, 7);
#undef FELOG_UMMA
    c->launches++;
    CK(cudaGetLastError(), "train_round: launch");
  } else if (!c->o.cbow && (c->o.reuse_neg == 2 || c->o.reuse_neg == 4)) {
    // center tiles over the plan negatives (2) or over the skip-gram windows and
    // each center's first draws (4, window tiles) (k_sgns_reuse_tile)
    const bool bf = c->o.precision == FELOG_BF16;
    const bool win = c->o.reuse_neg == 4;
    if (win) {
      s = ensure_jump(c, g);
      if (s != FELOG_OK) return s;
      g.jump_a = c->pr_jump.p;
      g.jump_c = c->pr_jump.p + 2 * c->o.window + 1;
      g.coarse = c->table_coarse.p;
      g.fm_table = make_fastmod((uint32_t)c->table_size);
    }
    // launch-shape autotuner: the first tiled round at -size 128 trains three
    // slices of its sentences with register budgets for 4, 3 and 2 resident
    // blocks per SM (real work, nothing repeated) and keeps the fastest per
    // kept token
    auto launch_tile = [&](const SgArgs &ga, int minb) {
      const int K = c->o.negative, D = c->o.size;
#define FELOG_RT(D_, K_, MB)                                                                              \
  do {                                                                                                    \
    if (win) {                                                                                            \
      if (bf) k_sgns_reuse_tile<D_, K_, RowsBF16, true, MB><<<blocks, threads, 0, c->stream>>>(ga);      \
      else k_sgns_reuse_tile<D_, K_, RowsF32, true, MB><<<blocks, threads, 0, c->stream>>>(ga);          \
    } else {                                                                                              \
      if (bf) k_sgns_reuse_tile<D_, K_, RowsBF16, false, MB><<<blocks, threads, 0, c->stream>>>(ga);     \
      else k_sgns_reuse_tile<D_, K_, RowsF32, false, MB><<<blocks, threads, 0, c->stream>>>(ga);         \
    }                                                                                                     \
  } while (0)
      if (D == 128) {
        if (K == 5) {
          if (minb == 3) FELOG_RT(128, 5, 3);
          else if (minb == 2) FELOG_RT(128, 5, 2);
          else FELOG_RT(128, 5, 4);
        } else {
          if (minb == 3) FELOG_RT(128, 7, 3);
          else if (minb == 2) FELOG_RT(128, 7, 2);
          else FELOG_RT(128, 7, 4);
        }
      } else if (K == 5 && D == 64) FELOG_RT(64, 5, 4);
      else if (K == 5 && D == 256) FELOG_RT(256, 5, 4);
      else if (K == 7 && D == 64) FELOG_RT(64, 7, 4);
      else FELOG_RT(256, 7, 4);
#undef FELOG_RT
      c->launches++;
    };
    const uint64_t ns = g.n_sent;
    constexpr int kTileCand = 3;
    if (c->o.autotune && !c->o.deterministic && c->o.size == 128 && c->tile_minb == 0 &&
        ns >= (uint64_t)kTileCand * blocks * (threads / 32)) {
      const int cand[kTileCand] = {4, 3, 2};
      cudaEvent_t ev[kTileCand + 1];
      for (int i = 0; i <= kTileCand; i++) CK(cudaEventCreate(&ev[i]), "autotune");
      uint64_t bound[kTileCand + 1];
      for (int i = 0; i <= kTileCand; i++) bound[i] = ns * i / kTileCand;
      for (int i = 0; i < kTileCand; i++) {
        CK(cudaMemsetAsync(c->counters.p + 0, 0, 8, c->stream), "train");  // sentence claim counter
        SgArgs gi = g;
        gi.s_first = bound[i];
        gi.n_sent = bound[i + 1] - bound[i];
        CK(cudaEventRecord(ev[i], c->stream), "autotune");
        launch_tile(gi, cand[i]);
        CK(cudaGetLastError(), "train_round: launch");
      }
      CK(cudaEventRecord(ev[kTileCand], c->stream), "autotune");
      uint64_t kept[kTileCand + 1];
      for (int i = 0; i <= kTileCand; i++) RB(&kept[i], c->p_out_off.p + bound[i], 8, "autotune");
      double best = 1e300;
      int pick = 4;
      char buf[256];
      std::string rep = "tile blocks/SM:";
      for (int i = 0; i < kTileCand; i++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]), "autotune");
        const double per = ms / (double)std::max<uint64_t>(1, kept[i + 1] - kept[i]);
        snprintf(buf, sizeof buf, " %d -> %.3f ns/token", cand[i], per * 1e6);
        rep += buf;
        if (per < best) {
          best = per;
          pick = cand[i];
        }
      }
      snprintf(buf, sizeof buf, "; chose %d", pick);
      c->tuning = rep + buf;
      c->tile_minb = pick;
      for (int i = 0; i <= kTileCand; i++) cudaEventDestroy(ev[i]);
    } else {
      launch_tile(g, c->tile_minb ? c->tile_minb : 4);
    }
    CK(cudaGetLastError(), "train_round: launch");
  } else if (!c->o.cbow && c->o.size >= 64 && (c->o.negative == 5 || c->o.negative == 7)) {
    s = train_pairs(c, g, blocks, threads);
    if (s != FELOG_OK) return s;
  } else {
    if (c->o.precision == FELOG_BF16) launch_trainer<RowsBF16>(c, g, blocks, threads);
    else launch_trainer<RowsF32>(c, g, blocks, threads);
    c->launches++;
    CK(cudaGetLastError(), "train_round: launch");
  }
  CK(cudaEventRecord(c->ev1, c->stream), "train_round");
  // words considered = sum of the plan's considered tokens per sentence (counter 2)
  CK(cudaMemsetAsync(c->counters.p + 2, 0, 8, c->stream), "train_round");
  if (c->plan_sent) {
    k_sum_u32<<<grid_for(c, c->plan_sent, 256), 256, 0, c->stream>>>(c->p_cons.p, c->plan_sent, c->counters.p + 2);
    c->launches++;
  }
  unsigned long long h[4];
  RB(h, c->counters.p, sizeof h, "train_round");
  s = check_dev_err(c, "train_round");
  if (s != FELOG_OK) return s;
  CK(cudaEventElapsedTime(&ms_train, c->ev0, c->ev1), "train_round");
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->words = h[2];
    stats->kept_words = c->plan_sen;
    stats->pairs = c->round_used_stream ? c->round_stream_pairs : h[1];
    stats->sentences = c->plan_sent;
    stats->batches = c->plan_batches;
    stats->alpha = alpha;
    stats->ms_plan = ms_plan;
    stats->ms_train = ms_train;
  }
  return FELOG_OK;
}

extern "C" felog_status felog_count_lost_updates(felog_ctx *c, int on) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  CK(cudaSetDevice(c->device), "count_lost_updates");
  c->count_lost = false;
  c->lost_ver0.release();
  c->lost_ver1.release();
  c->lost_tot.release();
  if (!on) return FELOG_OK;
  if (c->o.precision != FELOG_BF16 || c->o.size > 128)
    return fail(c, FELOG_INVALID_ARG, "count_lost_updates: the BF16 form of the pair trainer (-size <= 128) only");
  const size_t n = (size_t)c->vocab_size;
  CK(c->lost_ver0.ensure(n), "count_lost_updates");
  CK(c->lost_ver1.ensure(n), "count_lost_updates");
  CK(c->lost_tot.ensure(2), "count_lost_updates");
  CK(cudaMemsetAsync(c->lost_ver0.p, 0, 4 * n, c->stream), "count_lost_updates");
  CK(cudaMemsetAsync(c->lost_ver1.p, 0, 4 * n, c->stream), "count_lost_updates");
  CK(cudaMemsetAsync(c->lost_tot.p, 0, 16, c->stream), "count_lost_updates");
  CK(cudaStreamSynchronize(c->stream), "count_lost_updates");
  c->count_lost = true;
  return FELOG_OK;
}

extern "C" felog_status felog_lost_updates(felog_ctx *c, uint64_t *bf16_updates, uint64_t *lost) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->count_lost) return fail(c, FELOG_NOT_READY, "lost_updates: counting is off (felog_count_lost_updates)");
  unsigned long long h[2];
  RB(h, c->lost_tot.p, sizeof h, "lost_updates");
  if (bf16_updates) *bf16_updates = h[0];
  if (lost) *lost = h[1];
  return FELOG_OK;
}

extern "C" felog_status felog_plan_size(felog_ctx *c, uint64_t *n_sentences, uint64_t *n_sen, uint64_t *n_batches) {
  if (!c) return FELOG_INVALID_ARG;
  if (n_sentences) *n_sentences = c->plan_sent;
  if (n_sen) *n_sen = c->plan_sen;
  if (n_batches) *n_batches = c->plan_batches;
  return FELOG_OK;
}

extern "C" felog_status felog_get_plan(felog_ctx *c, int32_t *sen, uint64_t *sent_start, uint64_t *batch_first,
                                       int32_t *negs) {
  if (!c) return FELOG_INVALID_ARG;
  if (sen && c->plan_sen) CK(cudaMemcpy(sen, c->p_sen.p, 4 * c->plan_sen, cudaMemcpyDeviceToHost), "get_plan");
  if (sent_start)
    CK(cudaMemcpy(sent_start, c->p_out_off.p, 8 * (c->plan_sent + 1), cudaMemcpyDeviceToHost), "get_plan");
  if (batch_first)
    CK(cudaMemcpy(batch_first, c->p_batch_first.p, 8 * (c->plan_batches + 1), cudaMemcpyDeviceToHost), "get_plan");
  if (negs && c->plan_sent)
    CK(cudaMemcpy(negs, c->p_negs.p, 4 * c->plan_sent * (uint64_t)c->o.negative, cudaMemcpyDeviceToHost),
       "get_plan");
  return FELOG_OK;
}

namespace {

// interleaved rows -> logical order (see sgns.cuh); rows n_f32.. from BF16
// rows r0 .. r0 + rows - 1 into dst (row r0 first)
__global__ void k_unpermute(const float *src, const uint16_t *src_bf, uint64_t n_f32, float *dst, uint64_t rows,
                            int dim, uint64_t r0 = 0) {
  const int Jn = dim / 32;
  const uint64_t n = rows * (uint64_t)dim;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = r0 + e / dim;
    int l = (int)(e % dim);
    const uint64_t col = (uint64_t)(l % 32) * Jn + l / 32;
    dst[e] = r < n_f32 ? src[r * dim + col] : __uint_as_float((uint32_t)src_bf[(r - n_f32) * dim + col] << 16);
  }
}

}  // namespace

extern "C" felog_status felog_get_embeddings(felog_ctx *c, float *syn0, float *syn1, uint64_t cap_floats) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  const int dim = c->o.size;
  const uint64_t nel = (uint64_t)c->vocab_size * dim;
  if (cap_floats < nel) return fail(c, FELOG_INVALID_ARG, "get_embeddings: need %llu floats", (unsigned long long)nel);
  CK(cudaSetDevice(c->device), "get_embeddings");
  // staged through at most 1 GiB of device memory at a time
  const uint64_t step = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)c->vocab_size, (1ull << 28) / dim));
  CK(c->out_tmp.ensure(std::min<uint64_t>(nel, step * dim)), "get_embeddings");
  for (int which = 0; which < 2; which++) {
    float *dst = which ? syn1 : syn0;
    if (!dst) continue;
    for (uint64_t r0 = 0; r0 < (uint64_t)c->vocab_size; r0 += step) {
      const uint64_t nr = std::min<uint64_t>(step, (uint64_t)c->vocab_size - r0);
      k_unpermute<<<grid_for(c, nr * dim, 256), 256, 0, c->stream>>>(which ? c->syn1.p : c->syn0.p,
                                                                    which ? c->syn1_bf.p : c->syn0_bf.p,
                                                                    (uint64_t)c->n_f32, c->out_tmp.p, nr, dim, r0);
      c->launches++;
      CK(cudaGetLastError(), "get_embeddings");
      CK(cudaMemcpyAsync(dst + r0 * dim, c->out_tmp.p, 4 * nr * dim, cudaMemcpyDeviceToHost, c->stream),
         "get_embeddings");
      CK(cudaStreamSynchronize(c->stream), "get_embeddings");
    }
  }
  return FELOG_OK;
}

extern "C" felog_status felog_copy_embeddings_async(felog_ctx *c, float *syn0, uint64_t cap_floats) {
  if (!c || !syn0) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  const int dim = c->o.size;
  const uint64_t nel = (uint64_t)c->vocab_size * dim;
  if (cap_floats < nel)
    return fail(c, FELOG_INVALID_ARG, "copy_embeddings_async: need %llu floats", (unsigned long long)nel);
  CK(cudaSetDevice(c->device), "copy_embeddings_async");
  if (!c->copy_stream) {
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "copy_embeddings_async");
    CK(cudaEventCreateWithFlags(&c->copy_ready, cudaEventDisableTiming), "copy_embeddings_async");
    CK(cudaEventCreateWithFlags(&c->copy_done, cudaEventDisableTiming), "copy_embeddings_async");
  }
  CK(c->copy_stage.ensure(nel), "copy_embeddings_async");
  // the staging buffer is rewritten only after the previous copy has left it
  if (c->copy_pending) CK(cudaStreamWaitEvent(c->stream, c->copy_done, 0), "copy_embeddings_async");
  k_unpermute<<<grid_for(c, nel, 256), 256, 0, c->stream>>>(c->syn0.p, c->syn0_bf.p, (uint64_t)c->n_f32,
                                                             c->copy_stage.p, (uint64_t)c->vocab_size, dim);
  c->launches++;
  CK(cudaGetLastError(), "copy_embeddings_async");
  CK(cudaEventRecord(c->copy_ready, c->stream), "copy_embeddings_async");
  CK(cudaStreamWaitEvent(c->copy_stream, c->copy_ready, 0), "copy_embeddings_async");
  CK(cudaMemcpyAsync(syn0, c->copy_stage.p, 4 * nel, cudaMemcpyDeviceToHost, c->copy_stream),
     "copy_embeddings_async");
  CK(cudaEventRecord(c->copy_done, c->copy_stream), "copy_embeddings_async");
  c->copy_pending = true;
  return FELOG_OK;
}

extern "C" felog_status felog_wait_embeddings(felog_ctx *c) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->copy_pending) return FELOG_OK;
  CK(cudaEventSynchronize(c->copy_done), "wait_embeddings");
  // later work on the context's stream (and its timer events) comes after the copy
  CK(cudaStreamWaitEvent(c->stream, c->copy_done, 0), "wait_embeddings");
  c->copy_pending = false;
  return FELOG_OK;
}

extern "C" uint64_t felog_kernel_launches(const felog_ctx *c) { return c ? c->launches : 0; }

extern "C" const char *felog_tuning_report(const felog_ctx *c) {
  return !c ? "null context" : c->tuning.empty() ? "not tuned" : c->tuning.c_str();
}

extern "C" felog_status felog_timer_mark(felog_ctx *c, int which) {
  if (!c || (which != 0 && which != 1)) return FELOG_INVALID_ARG;
  CK(cudaEventRecord(which ? c->tm1 : c->tm0, c->stream), "timer_mark");
  return FELOG_OK;
}

extern "C" felog_status felog_timer_elapsed(felog_ctx *c, float *ms) {
  if (!c || !ms) return FELOG_INVALID_ARG;
  CK(cudaEventSynchronize(c->tm1), "timer_elapsed");
  CK(cudaEventElapsedTime(ms, c->tm0, c->tm1), "timer_elapsed");
  return FELOG_OK;
}

extern "C" felog_status felog_set_embeddings(felog_ctx *c, const float *syn0, const float *syn1) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  const int dim = c->o.size;
  const uint64_t nf = (uint64_t)c->n_f32 * dim, nel = (uint64_t)c->vocab_size * dim;
  CK(cudaSetDevice(c->device), "set_embeddings");
  // a snapshot still queued for an asynchronous copy reads the rows first
  CK(cudaStreamSynchronize(c->stream), "set_embeddings");
  std::vector<float> buf(nf);
  std::vector<uint16_t> bbuf(nel - nf);
  for (int which = 0; which < 2; which++) {
    const float *src = which ? syn1 : syn0;
    if (!src) continue;
    for (uint64_t r = 0; r < (uint64_t)c->vocab_size; r++)
      for (int l = 0; l < dim; l++) {
        const float v = src[r * dim + l];
        if (r < (uint64_t)c->n_f32) buf[r * dim + phys_index(dim, l)] = v;
        else bbuf[(r - c->n_f32) * dim + phys_index(dim, l)] = (uint16_t)bf16_rne(v);  // BF16 rows: nearest
      }
    CK(cudaMemcpy(which ? c->syn1.p : c->syn0.p, buf.data(), 4 * nf, cudaMemcpyHostToDevice), "set_embeddings");
    if (nel > nf)
      CK(cudaMemcpy(which ? c->syn1_bf.p : c->syn0_bf.p, bbuf.data(), 2 * (nel - nf), cudaMemcpyHostToDevice),
         "set_embeddings");
  }
  return FELOG_OK;
}

extern "C" felog_status felog_score_pairs(felog_ctx *c, const int32_t *ctx_rows, const int32_t *tgt_rows,
                                          const int8_t *labels, const uint64_t *batch_of, uint64_t n,
                                          uint64_t n_batches, float *dots, double *batch_loss) {
  if (!c || (n && (!ctx_rows || !tgt_rows || !labels || !batch_of || !dots)) || (n_batches && !batch_loss))
    return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  for (uint64_t i = 0; i < n; i++) {
    if (ctx_rows[i] < 0 || ctx_rows[i] >= c->vocab_size || tgt_rows[i] < 0 || tgt_rows[i] >= c->vocab_size)
      return fail(c, FELOG_INVALID_ARG, "score_pairs: row index out of range at %llu", (unsigned long long)i);
    if (batch_of[i] >= n_batches) return fail(c, FELOG_INVALID_ARG, "score_pairs: batch index out of range");
  }
  if (!n) {
    for (uint64_t b = 0; b < n_batches; b++) batch_loss[b] = 0.0;
    return FELOG_OK;
  }
  CK(cudaSetDevice(c->device), "score_pairs");
  int32_t *d_ctx = nullptr, *d_tgt = nullptr;
  int8_t *d_lab = nullptr;
  uint64_t *d_b = nullptr;
  float *d_dots = nullptr;
  double *d_loss = nullptr;
  cudaError_t e = cudaMalloc(&d_ctx, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_tgt, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_lab, n);
  if (e == cudaSuccess) e = cudaMalloc(&d_b, 8 * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_dots, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_loss, 8 * std::max<uint64_t>(n_batches, 1));
  if (e == cudaSuccess) e = cudaMemcpy(d_ctx, ctx_rows, 4 * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_tgt, tgt_rows, 4 * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_lab, labels, n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_b, batch_of, 8 * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d_loss, 0, 8 * std::max<uint64_t>(n_batches, 1));
  if (e == cudaSuccess) {
    SgArgs g{};
    g.syn0 = c->syn0.p;
    g.syn1 = c->syn1.p;
    g.syn0_bf = c->syn0_bf.p;
    g.syn1_bf = c->syn1_bf.p;
    g.n_hot = c->n_f32;
    const int blocks = grid_for(c, n * 32, 256);
    const bool bf = c->o.precision == FELOG_BF16;
    switch (c->o.size) {
#define FELOG_SP(D)                                                                                     \
  case D:                                                                                               \
    if (bf) k_score_pairs<D, RowsBF16><<<blocks, 256, 0, c->stream>>>(g, d_ctx, d_tgt, d_lab, d_b, n, d_dots, d_loss); \
    else k_score_pairs<D, RowsF32><<<blocks, 256, 0, c->stream>>>(g, d_ctx, d_tgt, d_lab, d_b, n, d_dots, d_loss);    \
    break;
      FELOG_SP(32)
      FELOG_SP(64)
      FELOG_SP(128)
      FELOG_SP(256)
#undef FELOG_SP
    }
    c->launches++;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(dots, d_dots, 4 * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && n_batches) e = cudaMemcpy(batch_loss, d_loss, 8 * n_batches, cudaMemcpyDeviceToHost);
  }
  cudaFree(d_ctx);
  cudaFree(d_tgt);
  cudaFree(d_lab);
  cudaFree(d_b);
  cudaFree(d_dots);
  cudaFree(d_loss);
  if (e != cudaSuccess) return cuda_fail(c, e, "score_pairs");
  return FELOG_OK;
}

// ---------------------------------------------------------------- budget

extern "C" felog_status felog_budget_check(felog_ctx *c, uint32_t round, felog_budget_stats *stats) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  CK(cudaSetDevice(c->device), "budget_check");
  CK(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * 8, c->stream), "budget_check");
  const bool learned = c->o.budget_mode == FELOG_BUDGET_LEARNED;
  if (learned && !c->pred_ready)
    return fail(c, FELOG_NOT_READY, "learned budget: no predictions (felog_mlp_predict after a walk round)");
  felog_status bs0 = budget_records(c);
  if (bs0 != FELOG_OK) return bs0;
  ConvArgs a{};
  a.stop_round = c->bud_stop_round.p;
  if (learned) {
    a.pred_count = c->pred_count.p;
    a.pred_conf = c->pred_conf.p;
    a.conf_min = c->o.budget_confidence > 0.0f ? c->o.budget_confidence : 0.9f;
    const double audit = c->o.budget_audit == 0.0f ? 0.05 : std::max(0.0, (double)c->o.budget_audit);
    a.audit_threshold = (uint32_t)std::min(4294967295.0, audit * 4294967296.0);
  }
  a.rows.syn0 = c->syn0.p;
  a.rows.syn0_bf = c->syn0_bf.p;
  a.rows.n_hot = c->n_f32;
  a.id2offset = c->id2offset.p;
  a.row_ptr = c->row_ptr.p;
  a.adj = c->adj.p;
  a.v_num = c->V;
  a.stop = c->stop.p;
  a.sim = c->sim.p;
  a.seed = c->o.seed;
  a.round = round;
  a.counters = c->counters.p;
  CK(cudaEventRecord(c->ev0, c->stream), "budget_check");
  const int blocks = grid_for(c, (uint64_t)c->V * 32, 256, 8);
  const bool bf = c->o.precision == FELOG_BF16;
  switch (c->o.size) {
#define FELOG_CV(D)                                                            \
  case D:                                                                      \
    if (bf) k_converge<D, RowsBF16><<<blocks, 256, 0, c->stream>>>(a);         \
    else k_converge<D, RowsF32><<<blocks, 256, 0, c->stream>>>(a);             \
    break;
    FELOG_CV(32)
    FELOG_CV(64)
    FELOG_CV(128)
    FELOG_CV(256)
#undef FELOG_CV
  }
  c->launches++;
  k_count_stopped<<<grid_for(c, c->V, 256), 256, 0, c->stream>>>(c->stop.p, c->V, c->counters.p + 2);
  c->launches++;
  CK(cudaGetLastError(), "budget_check");
  CK(cudaEventRecord(c->ev1, c->stream), "budget_check");
  unsigned long long h[8];
  RB(h, c->counters.p, sizeof h, "budget_check");
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1), "budget_check");
  // eva_num ratio test (word2vec.cu:2073-2080); the first comparison is against
  // vocab_size.  Learned mode: the plain criterion's count among the confident
  // (predicted or audited) vertices is estimated from the audited random
  // sample, so that the test follows what the plain criterion would decide.
  uint64_t eva = h[1];
  if (learned && h[4] > 0) {
    const double conf_unconv = (double)h[6] / (double)h[4] * (double)(h[3] + h[4]);
    eva = (uint64_t)std::llround((double)(h[7] - h[6]) + conf_unconv);
  }
  uint64_t last = c->have_last_eva ? c->last_eva : (uint64_t)c->vocab_size;
  float ratio = last ? (float)eva / (float)last : 0.0f;
  int stop_all = (last != 0 && ratio > 0.7f) ? 1 : 0;
  c->last_eva = eva;
  c->have_last_eva = true;
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->evaluated = h[0];
    stats->unconverged = h[1];
    stats->stopped_total = h[2];
    stats->stop_all = stop_all;
    stats->predicted = h[3];
    stats->audited = h[4];
    stats->overruled = h[5];
    stats->ms = ms;
  }
  return FELOG_OK;
}

extern "C" felog_status felog_get_similarity(felog_ctx *c, float *sim) {
  if (!c || !sim) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  CK(cudaMemcpy(sim, c->sim.p, 4 * (size_t)c->V, cudaMemcpyDeviceToHost), "get_similarity");
  return FELOG_OK;
}

// ---------------------------------------------------------------- classes

namespace {
template <int D, class P>
void km_launch(felog_ctx *c, KmArgs &a, int which, int blocks, const uint32_t *sorted, const uint64_t *seg) {
  if (which == 0) k_km_seed<D, P><<<std::min(a.k, 4096), 32, 0, c->stream>>>(a);
  else if (which == 1) k_km_assign<D, P><<<blocks, 256, 0, c->stream>>>(a);
  else k_km_update<D, P><<<std::min(a.k, 65535), 256, 0, c->stream>>>(a, sorted, seg);
  c->launches++;
}
template <class P>
void km_dispatch(felog_ctx *c, KmArgs &a, int which, int blocks, const uint32_t *sorted, const uint64_t *seg) {
  switch (c->o.size) {
    case 32: km_launch<32, P>(c, a, which, blocks, sorted, seg); break;
    case 64: km_launch<64, P>(c, a, which, blocks, sorted, seg); break;
    case 128: km_launch<128, P>(c, a, which, blocks, sorted, seg); break;
    case 256: km_launch<256, P>(c, a, which, blocks, sorted, seg); break;
  }
}
}  // namespace

extern "C" felog_status felog_cluster_embeddings(felog_ctx *c, int32_t classes, int32_t max_iter, int32_t *labels,
                                                 double *objective, int32_t *iterations) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  const uint64_t n = (uint64_t)c->vocab_size;
  if (classes < 1 || (uint64_t)classes > n || classes > (1 << 24))
    return fail(c, FELOG_INVALID_ARG, "cluster_embeddings: classes must be in [1, min(vocab, 2^24)]");
  if (max_iter < 0) return fail(c, FELOG_INVALID_ARG, "cluster_embeddings: max_iter must be >= 0");
  if (max_iter == 0) max_iter = 10;
  if (n > 0xFFFFFFFFull) return fail(c, FELOG_INVALID_ARG, "cluster_embeddings: more than 2^32 rows");
  CK(cudaSetDevice(c->device), "cluster_embeddings");
  const int dim = c->o.size;
  DevBuf<float> cent;
  DevBuf<int32_t> lab;
  DevBuf<double> part;
  DevBuf<uint32_t> keys, vals, keys2, vals2;
  DevBuf<unsigned long long> cnt;
  DevBuf<uint64_t> seg;
  const int blocks = grid_for(c, n * 32, 256, 8);
  CK(cent.ensure((size_t)classes * dim), "cluster_embeddings");
  CK(lab.ensure(n), "cluster_embeddings");
  CK(part.ensure(blocks), "cluster_embeddings");
  CK(keys.ensure(n), "cluster_embeddings");
  CK(vals.ensure(n), "cluster_embeddings");
  CK(keys2.ensure(n), "cluster_embeddings");
  CK(vals2.ensure(n), "cluster_embeddings");
  CK(cnt.ensure((size_t)classes + 1), "cluster_embeddings");
  CK(seg.ensure((size_t)classes + 1), "cluster_embeddings");
  KmArgs a{};
  a.rows.syn0 = c->syn0.p;
  a.rows.syn0_bf = c->syn0_bf.p;
  a.rows.n_hot = c->n_f32;
  a.n_rows = n;
  a.k = classes;
  a.cent = cent.p;
  a.labels = lab.p;
  a.obj_partial = part.p;
  a.changed = c->counters.p;
  const bool bf = c->o.precision == FELOG_BF16;
  auto launch = [&](int which, const uint32_t *sorted, const uint64_t *sg) {
    if (bf) km_dispatch<RowsBF16>(c, a, which, blocks, sorted, sg);
    else km_dispatch<RowsF32>(c, a, which, blocks, sorted, sg);
  };
  launch(0, nullptr, nullptr);
  CK(cudaGetLastError(), "cluster_embeddings: seed");
  int end_bit = 1;
  while (end_bit < 32 && (1ULL << end_bit) < (uint64_t)classes) end_bit++;
  std::vector<double> hp(blocks);
  int it = 0;
  for (; it < max_iter; it++) {
    a.first = it == 0;
    CK(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long), c->stream), "cluster_embeddings");
    launch(1, nullptr, nullptr);
    CK(cudaGetLastError(), "cluster_embeddings: assign");
    unsigned long long changed = 0;
    RB(&changed, c->counters.p, sizeof changed, "cluster_embeddings");
    RB(hp.data(), part.p, sizeof(double) * blocks, "cluster_embeddings");
    double obj = 0.0;
    for (int b = 0; b < blocks; b++) obj += hp[b];
    if (objective) objective[it] = obj;
    if (changed == 0) {
      it++;
      break;
    }
    // rows grouped by label (stable: ascending row index inside a label)
    CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long) * (classes + 1), c->stream), "cluster_embeddings");
    k_km_count<<<grid_for(c, n, 256), 256, 0, c->stream>>>(lab.p, n, keys.p, vals.p, cnt.p);
    c->launches++;
    cub::DoubleBuffer<uint32_t> dk(keys.p, keys2.p), dv(vals.p, vals2.p);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, dk, dv, (int)n, 0, end_bit, c->stream), "cluster_embeddings");
    CK(c->cub_tmp.ensure(tmp), "cluster_embeddings");
    CK(cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, tmp, dk, dv, (int)n, 0, end_bit, c->stream),
       "cluster_embeddings");
    tmp = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt.p, (unsigned long long *)seg.p, classes + 1, c->stream),
       "cluster_embeddings");
    CK(c->cub_tmp.ensure(tmp), "cluster_embeddings");
    CK(cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, tmp, cnt.p, (unsigned long long *)seg.p, classes + 1, c->stream),
       "cluster_embeddings");
    launch(2, dv.Current(), seg.p);
    CK(cudaGetLastError(), "cluster_embeddings: update");
  }
  if (iterations) *iterations = it;
  if (labels) CK(cudaMemcpy(labels, lab.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "cluster_embeddings");
  return FELOG_OK;
}

// -------------------------------------------------------- learned budget

namespace {

felog_status compute_features(felog_ctx *c) {
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  if (!c->bud_walks.p || !c->visit_freq.p) return fail(c, FELOG_NOT_READY, "budget features need a walk round");
  CK(c->feat.ensure((size_t)c->V * kMlpIn), "budget features");
  k_budget_features<<<grid_for(c, (uint64_t)c->V * 32, 256), 256, 0, c->stream>>>(
      c->row_ptr.p, c->adj.p, c->V, c->visit_freq.p, c->bud_first_len.p, c->feat.p);
  c->launches++;
  CK(cudaGetLastError(), "budget features");
  return FELOG_OK;
}

felog_status host_labels(felog_ctx *c, std::vector<uint8_t> &cnt, std::vector<float> &len,
                         std::vector<uint32_t> &walks) {
  if (!c->bud_walks.p) return fail(c, FELOG_NOT_READY, "no rounds recorded");
  const uint32_t V = c->V;
  std::vector<uint8_t> sr(V);
  std::vector<uint32_t> ls(V);
  walks.resize(V);
  CK(cudaStreamSynchronize(c->stream), "budget labels");
  CK(cudaMemcpy(sr.data(), c->bud_stop_round.p, V, cudaMemcpyDeviceToHost), "budget labels");
  CK(cudaMemcpy(ls.data(), c->bud_len_sum.p, 4 * (size_t)V, cudaMemcpyDeviceToHost), "budget labels");
  CK(cudaMemcpy(walks.data(), c->bud_walks.p, 4 * (size_t)V, cudaMemcpyDeviceToHost), "budget labels");
  cnt.resize(V);
  len.resize(V);
  for (uint32_t v = 0; v < V; v++) {
    const int k = sr[v] == 0xFF ? 10 : (int)sr[v] + 1;
    cnt[v] = (uint8_t)std::min(10, std::max(2, k));
    const float l = walks[v] ? (float)ls[v] / (float)walks[v] : 20.0f;
    len[v] = std::min(80.0f, std::max(20.0f, l));
  }
  return FELOG_OK;
}

// mean and 1/std of each raw feature over the vertices that have walked (FP64)
felog_status graph_feature_norm(felog_ctx *c, float *norm, std::vector<uint32_t> *walked) {
  const uint32_t V = c->V;
  std::vector<float> fh((size_t)V * kMlpIn);
  std::vector<uint32_t> walks(V);
  CK(cudaStreamSynchronize(c->stream), "feature norm");
  CK(cudaMemcpy(fh.data(), c->feat.p, 4 * fh.size(), cudaMemcpyDeviceToHost), "feature norm");
  CK(cudaMemcpy(walks.data(), c->bud_walks.p, 4 * (size_t)V, cudaMemcpyDeviceToHost), "feature norm");
  std::vector<uint32_t> idx;
  for (uint32_t v = 0; v < V; v++)
    if (walks[v]) idx.push_back(v);
  if (idx.empty()) return fail(c, FELOG_NOT_READY, "no vertex has walked");
  for (int k = 0; k < kMlpIn; k++) {
    double m = 0, q = 0;
    for (uint32_t v : idx) m += fh[(size_t)v * kMlpIn + k];
    m /= idx.size();
    for (uint32_t v : idx) q += (fh[(size_t)v * kMlpIn + k] - m) * (fh[(size_t)v * kMlpIn + k] - m);
    const double sd = std::sqrt(q / idx.size());
    norm[k] = (float)m;
    norm[kMlpIn + k] = sd > 1e-12 ? (float)(1.0 / sd) : 1.0f;
  }
  if (walked) *walked = std::move(idx);
  return FELOG_OK;
}

felog_status mlp_buffers(felog_ctx *c) {
  CK(c->mlp_params.ensure(kMlpParams), "mlp");
  CK(c->mlp_norm.ensure(2 * kMlpIn), "mlp");
  CK(c->mlp_m1.ensure(kMlpParams), "mlp");
  CK(c->mlp_m2.ensure(kMlpParams), "mlp");
  CK(c->mlp_grad.ensure(kMlpParams), "mlp");
  static bool attr_set[64] = {false};
  if (c->device < 64 && !attr_set[c->device]) {
    CK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(sizeof(float) * (kMlpParams + kMlpBatch * (2 * kMlpPad + kMlpOut + kMlpIn)))),
       "mlp");
    attr_set[c->device] = true;
  }
  return FELOG_OK;
}

constexpr size_t kMlpSmem = sizeof(float) * (kMlpParams + kMlpBatch * (2 * kMlpPad + kMlpOut + kMlpIn));

}  // namespace

extern "C" felog_status felog_budget_features(felog_ctx *c, float *features) {
  if (!c) return FELOG_INVALID_ARG;
  CK(cudaSetDevice(c->device), "budget features");
  felog_status s = compute_features(c);
  if (s != FELOG_OK) return s;
  if (features)
    CK(cudaMemcpyAsync(features, c->feat.p, 4 * (size_t)c->V * kMlpIn, cudaMemcpyDeviceToHost, c->stream),
       "budget features");
  CK(cudaStreamSynchronize(c->stream), "budget features");
  return FELOG_OK;
}

extern "C" felog_status felog_budget_labels(felog_ctx *c, uint8_t *count, float *length) {
  if (!c) return FELOG_INVALID_ARG;
  std::vector<uint8_t> cnt;
  std::vector<float> len;
  std::vector<uint32_t> walks;
  felog_status s = host_labels(c, cnt, len, walks);
  if (s != FELOG_OK) return s;
  if (count) memcpy(count, cnt.data(), cnt.size());
  if (length) memcpy(length, len.data(), 4 * len.size());
  return FELOG_OK;
}

extern "C" felog_status felog_mlp_train(felog_ctx *c, const felog_mlp_opts *opts, felog_mlp_stats *stats) {
  if (!c) return FELOG_INVALID_ARG;
  felog_mlp_opts o{};
  if (opts) o = *opts;
  if (o.epochs <= 0) o.epochs = 8;
  if (o.batch <= 0) o.batch = 4096;
  if (o.batch % kMlpBatch) return fail(c, FELOG_INVALID_ARG, "mlp batch must be a multiple of %d", kMlpBatch);
  if (o.lr <= 0.0f) o.lr = 3e-3f;
  CK(cudaSetDevice(c->device), "mlp_train");
  CK(cudaEventRecord(c->ev0, c->stream), "mlp_train");
  felog_status s = compute_features(c);
  if (s != FELOG_OK) return s;
  s = mlp_buffers(c);
  if (s != FELOG_OK) return s;
  std::vector<uint8_t> cnt;
  std::vector<float> len;
  std::vector<uint32_t> walks;
  s = host_labels(c, cnt, len, walks);
  if (s != FELOG_OK) return s;
  const uint32_t V = c->V;
  // features standardized over this graph's walked vertices (FP64 moments)
  std::vector<uint32_t> idx;
  float norm[2 * kMlpIn];
  s = graph_feature_norm(c, norm, &idx);
  if (s != FELOG_OK) return s;
  CK(cudaMemcpy(c->mlp_norm.p, norm, sizeof norm, cudaMemcpyHostToDevice), "mlp_train");
  k_budget_standardize<<<grid_for(c, (uint64_t)V * kMlpIn, 256), 256, 0, c->stream>>>(c->feat.p, V, c->mlp_norm.p,
                                                                                      c->mlp_norm.p + kMlpIn);
  c->launches++;
  CK(c->mlp_ycount.ensure(V), "mlp_train");
  CK(c->mlp_ylen.ensure(V), "mlp_train");
  CK(cudaMemcpy(c->mlp_ycount.p, cnt.data(), V, cudaMemcpyHostToDevice), "mlp_train");
  CK(cudaMemcpy(c->mlp_ylen.p, len.data(), 4 * (size_t)V, cudaMemcpyHostToDevice), "mlp_train");
  // He-uniform initialisation, zero biases
  std::mt19937_64 rng(o.seed ^ 0x4D4C5031ULL);
  std::vector<float> P(kMlpParams, 0.0f);
  auto fill = [&](int off, int n, int fan_in) {
    const float r = std::sqrt(6.0f / (float)fan_in);
    std::uniform_real_distribution<float> U(-r, r);
    for (int i = 0; i < n; i++) P[off + i] = U(rng);
  };
  fill(kMlpW1, kMlpH * kMlpIn, kMlpIn);
  fill(kMlpW2, kMlpH * kMlpH, kMlpH);
  fill(kMlpW3, kMlpOut * kMlpH, kMlpH);
  CK(cudaMemcpy(c->mlp_params.p, P.data(), 4 * P.size(), cudaMemcpyHostToDevice), "mlp_train");
  CK(cudaMemset(c->mlp_m1.p, 0, 4 * kMlpParams), "mlp_train");
  CK(cudaMemset(c->mlp_m2.p, 0, 4 * kMlpParams), "mlp_train");
  const uint64_t n = idx.size();
  const int max_blocks = o.batch / kMlpBatch;
  CK(c->mlp_partial.ensure((size_t)max_blocks * kMlpParams), "mlp_train");
  CK(c->mlp_idx.ensure(n), "mlp_train");
  CK(c->mlp_loss.ensure(n / kMlpBatch + 2), "mlp_train");
  std::vector<double> lp(n / kMlpBatch + 2);
  double loss_first = 0, loss_last = 0;
  const float b1 = 0.9f, b2 = 0.999f;
  // One epoch (a gradient and an Adam launch per batch, the same batches every
  // epoch) is captured once as a CUDA graph and replayed; the Adam bias
  // corrections come from a per-step table and the epoch's first step from
  // device memory, so the captured launches stay the same.
  const uint64_t n_batches = (n + o.batch - 1) / o.batch;
  const uint64_t steps = n_batches * (uint64_t)o.epochs;
  std::vector<float2> bct(steps);
  for (uint64_t s1 = 1; s1 <= steps; s1++)
    bct[s1 - 1] = make_float2(1.0f - std::pow(b1, (float)s1), 1.0f - std::pow(b2, (float)s1));
  CK(c->mlp_bc.ensure(std::max<uint64_t>(steps, 1)), "mlp_train");
  CK(c->mlp_step.ensure(1), "mlp_train");
  CK(cudaMemcpyAsync(c->mlp_bc.p, bct.data(), sizeof(float2) * steps, cudaMemcpyHostToDevice, c->stream), "mlp_train");
  uint64_t nblk_total = 0;
  for (uint64_t b0 = 0; b0 < n; b0 += o.batch) nblk_total += (std::min<uint64_t>(o.batch, n - b0) + kMlpBatch - 1) / kMlpBatch;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto capture_epoch = [&]() -> cudaError_t {
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    uint64_t blk = 0, j = 0;
    for (uint64_t b0 = 0; b0 < n; b0 += o.batch, j++) {
      const uint64_t nb = std::min<uint64_t>(o.batch, n - b0);
      const int blocks = (int)((nb + kMlpBatch - 1) / kMlpBatch);
      MlpGradArgs ga{};
      ga.params = c->mlp_params.p;
      ga.X = c->feat.p;
      ga.y_count = c->mlp_ycount.p;
      ga.y_len = c->mlp_ylen.p;
      ga.idx = c->mlp_idx.p + b0;
      ga.n = nb;
      ga.partial = c->mlp_partial.p;
      ga.loss_partial = c->mlp_loss.p + blk;
      k_mlp_grad<<<blocks, kMlpBatch, kMlpSmem, c->stream>>>(ga);
      k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, c->stream>>>(c->mlp_params.p, c->mlp_m1.p, c->mlp_m2.p,
                                                                  c->mlp_partial.p, blocks, 1.0f / (float)nb, o.lr,
                                                                  b1, b2, 1e-8f, 1.0f, 1.0f, nullptr, c->mlp_bc.p,
                                                                  c->mlp_step.p, (uint32_t)j);
      blk += blocks;
    }
    const cudaError_t le = cudaGetLastError();
    e = cudaStreamEndCapture(c->stream, &graph);
    if (le != cudaSuccess) return le;
    if (e != cudaSuccess) return e;
    return cudaGraphInstantiate(&exec, graph, 0);
  };
  felog_status st = FELOG_OK;
  std::vector<uint32_t> base(1);
  for (int ep = 0; ep < o.epochs && st == FELOG_OK; ep++) {
    std::shuffle(idx.begin(), idx.end(), rng);
    cudaError_t e = cudaMemcpyAsync(c->mlp_idx.p, idx.data(), 4 * n, cudaMemcpyHostToDevice, c->stream);
    base[0] = (uint32_t)(n_batches * (uint64_t)ep);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->mlp_step.p, base.data(), 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && !exec) e = capture_epoch();
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, c->stream);
    c->launches += 2 * n_batches;
    if (e == cudaSuccess) e = cudaMemcpyAsync(lp.data(), c->mlp_loss.p, 8 * nblk_total, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
      st = cuda_fail(c, e, "mlp_train");
      break;
    }
    double l = 0;
    for (uint64_t i = 0; i < nblk_total; i++) l += lp[i];
    l /= (double)n;
    if (ep == 0) loss_first = l;
    loss_last = l;
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (st != FELOG_OK) return st;
  c->mlp_ready = true;
  // fit on the training vertices
  CK(c->pred_count.ensure(V), "mlp_train");
  CK(c->pred_conf.ensure(V), "mlp_train");
  CK(c->pred_len.ensure(V), "mlp_train");
  k_mlp_infer<<<grid_for(c, V, 128), 128, 0, c->stream>>>(c->mlp_params.p, c->feat.p, V, c->pred_count.p,
                                                          c->pred_conf.p, c->pred_len.p);
  c->launches++;
  CK(cudaGetLastError(), "mlp_train");
  CK(cudaEventRecord(c->ev1, c->stream), "mlp_train");
  std::vector<uint8_t> pc(V);
  std::vector<float> pl(V);
  CK(cudaMemcpyAsync(pc.data(), c->pred_count.p, V, cudaMemcpyDeviceToHost, c->stream), "mlp_train");
  CK(cudaMemcpyAsync(pl.data(), c->pred_len.p, 4 * (size_t)V, cudaMemcpyDeviceToHost, c->stream), "mlp_train");
  CK(cudaStreamSynchronize(c->stream), "mlp_train");
  c->pred_ready = false;  // predictions for the budget check come from felog_mlp_predict
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    uint64_t ok = 0;
    double mae = 0;
    for (uint32_t v : idx) {
      ok += pc[v] == cnt[v];
      mae += std::fabs((double)pl[v] - (double)len[v]);
    }
    stats->samples = n;
    stats->steps = steps;
    stats->loss_first = loss_first;
    stats->loss_last = loss_last;
    stats->count_accuracy = (double)ok / (double)n;
    stats->length_mae = mae / (double)n;
    CK(cudaEventElapsedTime(&stats->ms, c->ev0, c->ev1), "mlp_train");
  }
  return FELOG_OK;
}

extern "C" felog_status felog_mlp_get_params(felog_ctx *c, float *state) {
  if (!c || !state) return FELOG_INVALID_ARG;
  if (!c->mlp_ready) return fail(c, FELOG_NOT_READY, "no trained model");
  CK(cudaMemcpy(state, c->mlp_params.p, 4 * kMlpParams, cudaMemcpyDeviceToHost), "mlp_get_params");
  CK(cudaMemcpy(state + kMlpParams, c->mlp_norm.p, 4 * 2 * kMlpIn, cudaMemcpyDeviceToHost), "mlp_get_params");
  return FELOG_OK;
}

extern "C" felog_status felog_mlp_set_params(felog_ctx *c, const float *state) {
  if (!c || !state) return FELOG_INVALID_ARG;
  CK(cudaSetDevice(c->device), "mlp_set_params");
  felog_status s = mlp_buffers(c);
  if (s != FELOG_OK) return s;
  CK(cudaMemcpy(c->mlp_params.p, state, 4 * kMlpParams, cudaMemcpyHostToDevice), "mlp_set_params");
  CK(cudaMemcpy(c->mlp_norm.p, state + kMlpParams, 4 * 2 * kMlpIn, cudaMemcpyHostToDevice), "mlp_set_params");
  c->mlp_ready = true;
  c->pred_ready = false;
  return FELOG_OK;
}

extern "C" felog_status felog_mlp_gradient(felog_ctx *c, const float *params, const float *X, const uint8_t *count,
                                          const float *length, uint64_t n, float *grad, double *loss) {
  if (!c || !params || !X || !count || !length || !grad || n == 0) return FELOG_INVALID_ARG;
  for (uint64_t i = 0; i < n; i++)
    if (count[i] < 2 || count[i] > 10) return fail(c, FELOG_INVALID_ARG, "mlp_gradient: count label outside 2..10");
  CK(cudaSetDevice(c->device), "mlp_gradient");
  felog_status s = mlp_buffers(c);
  if (s != FELOG_OK) return s;
  const int blocks = (int)((n + kMlpBatch - 1) / kMlpBatch);
  float *dP = nullptr, *dX = nullptr, *dL = nullptr, *dPart = nullptr, *dG = nullptr;
  uint8_t *dC = nullptr;
  uint32_t *dI = nullptr;
  double *dLoss = nullptr;
  cudaError_t e = cudaMalloc(&dP, 4 * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc(&dX, 4 * n * kMlpIn);
  if (e == cudaSuccess) e = cudaMalloc(&dL, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&dC, n);
  if (e == cudaSuccess) e = cudaMalloc(&dI, 4 * n);
  if (e == cudaSuccess) e = cudaMalloc(&dPart, 4 * (size_t)blocks * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc(&dG, 4 * kMlpParams);
  if (e == cudaSuccess) e = cudaMalloc(&dLoss, 8 * (size_t)blocks);
  std::vector<uint32_t> id(n);
  std::iota(id.begin(), id.end(), 0u);
  if (e == cudaSuccess) e = cudaMemcpy(dP, params, 4 * kMlpParams, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dX, X, 4 * n * kMlpIn, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dL, length, 4 * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dC, count, n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dI, id.data(), 4 * n, cudaMemcpyHostToDevice);
  std::vector<double> lp(blocks);
  if (e == cudaSuccess) {
    MlpGradArgs ga{};
    ga.params = dP;
    ga.X = dX;
    ga.y_count = dC;
    ga.y_len = dL;
    ga.idx = dI;
    ga.n = n;
    ga.partial = dPart;
    ga.loss_partial = dLoss;
    k_mlp_grad<<<blocks, kMlpBatch, kMlpSmem, c->stream>>>(ga);
    c->launches++;
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, c->stream>>>(dP, nullptr, nullptr, dPart, blocks, 1.0f / (float)n,
                                                                0.0f, 0.f, 0.f, 0.f, 1.f, 1.f, dG);
    c->launches++;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(grad, dG, 4 * kMlpParams, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(lp.data(), dLoss, 8 * (size_t)blocks, cudaMemcpyDeviceToHost);
  }
  cudaFree(dP);
  cudaFree(dX);
  cudaFree(dL);
  cudaFree(dC);
  cudaFree(dI);
  cudaFree(dPart);
  cudaFree(dG);
  cudaFree(dLoss);
  if (e != cudaSuccess) return cuda_fail(c, e, "mlp_gradient");
  if (loss) {
    double l = 0;
    for (double x : lp) l += x;
    *loss = l / (double)n;
  }
  return FELOG_OK;
}

extern "C" felog_status felog_mlp_predict(felog_ctx *c, uint8_t *count, float *confidence, float *length) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->mlp_ready) return fail(c, FELOG_NOT_READY, "no trained model (felog_mlp_train or felog_mlp_set_params)");
  CK(cudaSetDevice(c->device), "mlp_predict");
  felog_status s = compute_features(c);
  if (s != FELOG_OK) return s;
  const uint32_t V = c->V;
  // standardize with this graph's own feature moments, as in training
  float norm[2 * kMlpIn];
  s = graph_feature_norm(c, norm, nullptr);
  if (s != FELOG_OK) return s;
  CK(c->mlp_grad.ensure(kMlpParams), "mlp_predict");
  CK(cudaMemcpyAsync(c->mlp_grad.p, norm, sizeof norm, cudaMemcpyHostToDevice, c->stream), "mlp_predict");
  k_budget_standardize<<<grid_for(c, (uint64_t)V * kMlpIn, 256), 256, 0, c->stream>>>(c->feat.p, V, c->mlp_grad.p,
                                                                                      c->mlp_grad.p + kMlpIn);
  c->launches++;
  CK(c->pred_count.ensure(V), "mlp_predict");
  CK(c->pred_conf.ensure(V), "mlp_predict");
  CK(c->pred_len.ensure(V), "mlp_predict");
  k_mlp_infer<<<grid_for(c, V, 128), 128, 0, c->stream>>>(c->mlp_params.p, c->feat.p, V, c->pred_count.p,
                                                          c->pred_conf.p, c->pred_len.p);
  c->launches++;
  CK(cudaGetLastError(), "mlp_predict");
  if (count) CK(cudaMemcpyAsync(count, c->pred_count.p, V, cudaMemcpyDeviceToHost, c->stream), "mlp_predict");
  if (confidence)
    CK(cudaMemcpyAsync(confidence, c->pred_conf.p, 4 * (size_t)V, cudaMemcpyDeviceToHost, c->stream), "mlp_predict");
  if (length) CK(cudaMemcpyAsync(length, c->pred_len.p, 4 * (size_t)V, cudaMemcpyDeviceToHost, c->stream), "mlp_predict");
  CK(cudaStreamSynchronize(c->stream), "mlp_predict");
  c->pred_ready = true;
  return FELOG_OK;
}

// ------------------------------------------------------------ whole loop

extern "C" felog_status felog_run(felog_ctx *c, felog_run_stats *st) {
  if (!c) return FELOG_INVALID_ARG;
  if (!c->V) return fail(c, FELOG_NOT_READY, "no graph loaded");
  felog_run_stats rs{};
  felog_status s;
  if (!c->model_ready) {
    s = felog_init_model(c);
    if (s != FELOG_OK) return s;
  }
  const uint32_t min_r = c->o.min_rounds ? c->o.min_rounds : 1;
  for (uint32_t r = 0;; r++) {
    if (c->o.max_rounds > 0 && (int)r >= c->o.max_rounds) break;
    // the round's walkers, whole or in pieces of stream_walkers: walk a piece,
    // train on its corpus, go on (walks depend on the graph and the stop flags
    // only, so the pieces walk exactly what the whole round would)
    s = walk_prepare(c);
    if (s != FELOG_OK) return s;
    const uint32_t na = c->n_active;
    const uint32_t piece = c->o.stream_walkers ? c->o.stream_walkers : std::max<uint32_t>(na, 1);
    for (uint32_t k0 = 0; k0 < na || k0 == 0; k0 += piece) {
      const uint32_t k1 = std::min<uint64_t>((uint64_t)k0 + piece, na);
      c->chunk_base = k0;
      felog_walk_stats ws;
      s = walk_range(c, r, nullptr, k0, k1, &ws, k1 == na);
      if (s != FELOG_OK) return s;
      rs.walk_tokens += ws.n_tokens;
      rs.walk_ms += ws.ms;
      if (c->o.budget_mode == FELOG_BUDGET_LEARNED && !c->pred_ready && k1 == na) {
        s = felog_mlp_predict(c, nullptr, nullptr, nullptr);  // features from the first round's walks
        if (s != FELOG_OK) return s;
      }
      felog_train_stats ts;
      s = felog_train_round(c, r, -1.0f, &ts);
      if (s != FELOG_OK) return s;
      rs.train_words += ts.words;
      rs.train_ms += ts.ms_plan + ts.ms_train;
      rs.plan_ms += ts.ms_plan;
      rs.pairs += ts.pairs;
      if (k1 >= na) break;
    }
    c->chunk_base = 0;
    rs.rounds = r + 1;
    if (r + 1 >= min_r) {  // train_iter >= init_round, word2vec.cu:2011-2017
      felog_budget_stats bs;
      s = felog_budget_check(c, r, &bs);
      if (s != FELOG_OK) return s;
      rs.budget_ms += bs.ms;
      rs.final_unconverged = bs.unconverged;
      rs.evaluated += bs.evaluated;
      rs.predicted += bs.predicted;
      rs.audited += bs.audited;
      rs.overruled += bs.overruled;
      if (bs.stop_all) break;
    }
  }
  rs.total_ms = rs.walk_ms + rs.train_ms + rs.budget_ms;
  if (st) *st = rs;
  return FELOG_OK;
}

namespace {
// "%lf" of a float, as glibc prints it: the exact binary value rounded to six
// decimals, ties to even.  A finite float is M * 2^E with M < 2^24; M * 10^6
// fits in 64 bits, so shifting it by -E with round-half-even gives the six-
// decimal integer exactly.  Values of 2^40 and above and non-finite values go
// to snprintf.  Returns the number of characters written to out (>= 48 bytes).
int format_lf(float x, char *out) {
  uint32_t bits;
  memcpy(&bits, &x, 4);
  const int exp_field = (int)((bits >> 23) & 0xFF);
  if (exp_field == 0xFF || (exp_field - 127) >= 40) return snprintf(out, 48, "%lf", (double)x);
  const bool neg = bits >> 31;
  uint64_t mant = bits & 0x7FFFFFu;
  int e2;
  if (exp_field == 0) {
    e2 = -149;  // subnormal: M * 2^-149
  } else {
    mant |= 0x800000u;
    e2 = exp_field - 150;
  }
  unsigned __int128 p = (unsigned __int128)mant * 1000000u;
  uint64_t q;
  if (e2 >= 0) {
    q = (uint64_t)(p << e2);
  } else {
    const int sh = -e2;
    if (sh >= 100) {
      q = 0;  // p < 2^44 < half of 2^sh
    } else {
      const unsigned __int128 one = 1;
      const unsigned __int128 rem = p & ((one << sh) - 1), half = one << (sh - 1);
      q = (uint64_t)(p >> sh);
      if (rem > half || (rem == half && (q & 1))) q++;
    }
  }
  char tmp[32];
  int n = 0;
  const uint64_t ip = q / 1000000u;
  uint32_t fr = (uint32_t)(q % 1000000u);
  for (int i = 0; i < 6; i++) {
    tmp[n++] = (char)('0' + fr % 10);
    fr /= 10;
  }
  tmp[n++] = '.';
  uint64_t v = ip;
  do {
    tmp[n++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  int k = 0;
  if (neg) out[k++] = '-';
  while (n) out[k++] = tmp[--n];
  return k;
}

// Rows [a0, a1) of the word2vec text format: "<vertex> " + dim x "%lf " + "\n".
void format_rows(const float *s0, const uint32_t *vertex, long long a0, long long a1, int dim, std::string &buf) {
  buf.clear();
  char tmp[64];
  for (long long a = a0; a < a1; a++) {
    int k = snprintf(tmp, sizeof tmp, "%u ", vertex[a]);
    buf.append(tmp, (size_t)k);
    for (int b = 0; b < dim; b++) {
      k = format_lf(s0[(uint64_t)a * dim + b], tmp);
      tmp[k++] = ' ';
      buf.append(tmp, (size_t)k);
    }
    buf.push_back('\n');
  }
}
}  // namespace

extern "C" felog_status felog_format_lf(const float *x, uint64_t n, char *out, uint64_t cap, uint64_t *len) {
  if ((n && !x) || (cap && !out)) return FELOG_INVALID_ARG;
  uint64_t k = 0;
  char tmp[64];
  for (uint64_t i = 0; i < n; i++) {
    const int m = format_lf(x[i], tmp);
    if (k + (uint64_t)m + 1 > cap) return FELOG_INVALID_ARG;
    memcpy(out + k, tmp, (size_t)m);
    k += (uint64_t)m;
    out[k++] = ' ';
  }
  if (len) *len = k;
  return FELOG_OK;
}

extern "C" felog_status felog_write_embeddings(felog_ctx *c, const char *path) {
  if (!c || !path) return FELOG_INVALID_ARG;
  if (!c->model_ready) return fail(c, FELOG_NOT_READY, "model not initialised");
  const int dim = c->o.size;
  std::vector<float> s0((uint64_t)c->vocab_size * dim);
  felog_status s = felog_get_embeddings(c, s0.data(), nullptr, s0.size());
  if (s != FELOG_OK) return s;
  FILE *fo = fopen(path, "wb");
  if (!fo) return fail(c, FELOG_IO_ERROR, "cannot open %s", path);
  // word2vec.cu:2121-2127
  bool ok = fprintf(fo, "%lld %lld\n", (long long)c->vocab_size, (long long)dim) > 0;
  if (c->o.binary) {
    for (long long a = 0; ok && a < c->vocab_size; a++) {
      ok = fprintf(fo, "%u ", c->h_vocab_vertex[a]) > 0 &&
           fwrite(&s0[(uint64_t)a * dim], sizeof(float), dim, fo) == (size_t)dim && fputc('\n', fo) != EOF;
    }
  } else {
    // text: blocks of rows formatted by all host threads, written in order
    const int nt = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const long long rows_per_block = 4096LL * nt;
    std::vector<std::string> bufs((size_t)nt);
    for (long long b0 = 0; ok && b0 < c->vocab_size; b0 += rows_per_block) {
      const long long b1 = std::min<long long>(c->vocab_size, b0 + rows_per_block);
      const long long per = (b1 - b0 + nt - 1) / nt;
      std::vector<std::thread> th;
      for (int t = 0; t < nt; t++) {
        const long long r0 = std::min(b1, b0 + t * per), r1 = std::min(b1, r0 + per);
        th.emplace_back(format_rows, s0.data(), c->h_vocab_vertex.data(), r0, r1, dim, std::ref(bufs[(size_t)t]));
      }
      for (auto &t : th) t.join();
      for (int t = 0; ok && t < nt; t++)
        ok = fwrite(bufs[(size_t)t].data(), 1, bufs[(size_t)t].size(), fo) == bufs[(size_t)t].size();
    }
  }
  if (fclose(fo) != 0 || !ok) return fail(c, FELOG_IO_ERROR, "write failed on %s", path);
  return FELOG_OK;
}
