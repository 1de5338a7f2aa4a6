/*
 * Reference trainer-plan harness (test infrastructure, never shipped).
 *
 * Compiles the reference's src/word2vec.cu unmodified, with the CUDA runtime
 * calls that move data redirected to host memory, and runs its own
 * ReadVocabFromDegree (word2vec.cu:834-862), InitNet (:864-902),
 * InitUnigramTable (:674-694) and TrainModelThreadMemory (:1133-1273) on a
 * given corpus.  Every host-to-device copy TrainModelThreadMemory makes is
 * logged; its three copies per batch (sen, sentence_length, negSample,
 * word2vec.cu:1251-1253) are the batch plan.  Kernel launches fail harmlessly
 * without a GPU; their return codes are not checked by the reference.
 *
 * Input files: degrees (u32 x V), corpus (u32 n_sent, then per sentence u32
 * len + u32 tokens).  Output (binary): i64 vocab_size, i64 train_words,
 * u32 vocab_vertex[vocab_size], u32 n_thr, u16 thr[n_thr],
 * u64 table_fnv1a (FNV-1a 64 of the 1e8-int unigram table),
 * i32 table_head[4096], f32 syn0_head[min(vocab,64) * dim],
 * u32 n_batches, then per batch: u32 cnt, u32 total,
 *   i32 sentence_length[cnt + 1], i32 sen[total], i32 negSample[cnt * negative]
 *
 * Usage: ref_sgns_plan deg.bin corpus.bin out.bin dim window negative sample min_count [table.bin]
 * (the optional last argument receives the whole unigram table)
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace harness {
struct Copy {
  size_t bytes;
  std::vector<char> data;
};
static std::vector<Copy> h2d;
static bool logging = false;
}  // namespace harness

static cudaError_t h_cudaMalloc(void **p, size_t n) {
  *p = calloc(n ? n : 1, 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
template <class T>
static cudaError_t h_cudaMalloc(T **p, size_t n) {
  return h_cudaMalloc((void **)p, n);
}
static cudaError_t h_cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind kind) {
  if (n) memcpy(dst, src, n);
  if (harness::logging && kind == cudaMemcpyHostToDevice) {
    harness::Copy c;
    c.bytes = n;
    c.data.assign((const char *)src, (const char *)src + n);
    harness::h2d.push_back(std::move(c));
  }
  return cudaSuccess;
}
static cudaError_t h_cudaFree(void *p) {
  free(p);
  return cudaSuccess;
}
static cudaError_t h_cudaDeviceSynchronize() { return cudaSuccess; }

#define cudaMalloc h_cudaMalloc
#define cudaMemcpy h_cudaMemcpy
#define cudaFree h_cudaFree
#define cudaDeviceSynchronize h_cudaDeviceSynchronize
#include "word2vec.cu"
#undef cudaMalloc
#undef cudaMemcpy
#undef cudaFree
#undef cudaDeviceSynchronize

volatile bool stop_sampling_flag = false;

static std::vector<uint32_t> read_u32(const char *path) {
  FILE *f = fopen(path, "rb");
  if (!f) { perror(path); exit(2); }
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<uint32_t> v((size_t)sz / 4);
  if (fread(v.data(), 4, v.size(), f) != v.size()) exit(2);
  fclose(f);
  return v;
}

int main(int argc, char **argv) {
  if (argc < 9) {
    fprintf(stderr, "usage: %s deg.bin corpus.bin out.bin dim window negative sample min_count\n", argv[0]);
    return 2;
  }
  std::vector<uint32_t> deg = read_u32(argv[1]);
  std::vector<uint32_t> cbuf = read_u32(argv[2]);
  layer1_size = atoi(argv[4]);
  window = atoi(argv[5]);
  negative = atoi(argv[6]);
  sample = (float)atof(argv[7]);
  min_count = atoi(argv[8]);
  cbow = 0;
  reuseNeg = 0;
  hs = 0;
  my_rank = 0;
  num_procs = 1;

  corpus_t corpus;
  size_t i = 0;
  uint32_t ns = cbuf[i++];
  for (uint32_t s = 0; s < ns; s++) {
    uint32_t len = cbuf[i++];
    corpus.emplace_back(cbuf.begin() + i, cbuf.begin() + i + len);
    i += len;
  }

  vocab_max_size = (long long)deg.size() + 1000;
  vocab = (struct vocab_word *)calloc(vocab_max_size, sizeof(struct vocab_word));
  expTable = (float *)malloc((EXP_TABLE_SIZE + 1) * sizeof(float));
  for (int k = 0; k < EXP_TABLE_SIZE; k++) {
    expTable[k] = exp((k / (float)EXP_TABLE_SIZE * 2 - 1) * MAX_EXP);
    expTable[k] = expTable[k] / (expTable[k] + 1);
  }
  std::vector<vertex_id_t> degrees(deg.begin(), deg.end());
  ReadVocabFromDegree(degrees);
  InitNet();
  InitUnigramTable();

  harness::logging = true;
  TrainModelThreadMemory(corpus);
  harness::logging = false;

  FILE *fo = fopen(argv[3], "wb");
  long long vs = vocab_size, tw = train_words;
  fwrite(&vs, 8, 1, fo);
  fwrite(&tw, 8, 1, fo);
  for (long long a = 0; a < vocab_size; a++) {
    uint32_t v = (uint32_t)strtoul(vocab[a].word, nullptr, 10);
    fwrite(&v, 4, 1, fo);
  }
  std::vector<uint16_t> thr = BuildSubsamplingThresholds(sample, train_words);
  uint32_t nthr = (uint32_t)thr.size();
  fwrite(&nthr, 4, 1, fo);
  fwrite(thr.data(), 2, nthr, fo);
  if (argc > 9) {
    FILE *ft = fopen(argv[9], "wb");
    fwrite(table, 4, (size_t)table_size, ft);
    fclose(ft);
  }
  uint64_t h = 1469598103934665603ULL;
  const unsigned char *tb = (const unsigned char *)table;
  for (size_t k = 0; k < (size_t)table_size * 4; k++) h = (h ^ tb[k]) * 1099511628211ULL;
  fwrite(&h, 8, 1, fo);
  fwrite(table, 4, 4096, fo);
  long long nrow = vocab_size < 64 ? vocab_size : 64;
  fwrite(syn0, 4, (size_t)nrow * layer1_size, fo);
  /* batches: triples of copies (sen, sentence_length, negSample) */
  uint32_t nb = (uint32_t)(harness::h2d.size() / 3);
  fwrite(&nb, 4, 1, fo);
  for (uint32_t b = 0; b < nb; b++) {
    const harness::Copy &cs = harness::h2d[3 * b], &cl = harness::h2d[3 * b + 1], &cn = harness::h2d[3 * b + 2];
    uint32_t cnt = (uint32_t)(cl.bytes / 4) - 1, total = (uint32_t)(cs.bytes / 4);
    fwrite(&cnt, 4, 1, fo);
    fwrite(&total, 4, 1, fo);
    fwrite(cl.data.data(), 1, cl.bytes, fo);
    fwrite(cs.data.data(), 1, cs.bytes, fo);
    fwrite(cn.data.data(), 1, cn.bytes, fo);
  }
  fclose(fo);
  fprintf(stderr, "ref_sgns_plan: vocab %lld, %u batches\n", vocab_size, nb);
  return 0;
}
