/*
 * Reference pipeline harness (the reference arm of bench.py; never shipped).
 *
 * Runs the reference's own graph-embedding path, compiled unmodified from
 * include/walk.hpp (+ graph.hpp, path.hpp) and src/word2vec.cu against the
 * loopback MPI shim, the way src/examples/felog.cpp drives it: the walk engine
 * in one thread with its OpenMP team (hardware_concurrency - 1 workers,
 * graph.hpp:322), the trainer in another, corpora handed over per round
 * through out_queue (walk.hpp:720-752, word2vec.cu:1990-1998), and per round
 * TrainModelThreadMemory (word2vec.cu:1133-1273) with skip_gram_kernel on the
 * GPU and the per-vertex evaluation (batch_node_neighbor_direct_index,
 * word2vec.cu:1748-1889; threshold word2vec.cu:2048-2062) from round min_R on.
 * Rounds are not cut short (pauseWalk is never raised), so every round walks
 * all walkers - the same work the B200 path does per round.
 *
 * Usage: ref_pipeline graph.bin V warmup_rounds timed_rounds walkers [emb_out]
 * Prints one JSON line: tokens, seconds (timed rounds, walk overlapped with
 * training as in the reference), walk_tokens, walk_seconds, train_words,
 * train_seconds, threads, walkers.
 *
 * emb_out (optional): after the last round, the trained tables in the
 * reference's own -binary 1 layout (the writer of TrainModel,
 * word2vec.cu:2119-2126: "<vocab_size> <layer1_size>\n", then per vocabulary
 * row its word, a space, layer1_size raw floats and "\n") - syn0 as the
 * trainer copied it back (word2vec.cu:1264), followed by the same rows of the
 * device syn1neg table (d_syn1) so that the syn0 . syn1 link score can be
 * formed too.
 */
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <thread>
#include <vector>

#include "walk.hpp"
#include "word2vec.cu"

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char **argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: %s graph.bin V warmup timed walkers\n", argv[0]);
    return 2;
  }
  const char *gpath = argv[1];
  uint32_t V = (uint32_t)strtoul(argv[2], nullptr, 10);
  int warm = atoi(argv[3]), timed = atoi(argv[4]);
  uint32_t walkers = (uint32_t)strtoul(argv[5], nullptr, 10);
  const char *emb_out = argc > 6 ? argv[6] : nullptr;
  if (walkers == 0 || walkers > V) walkers = V;
  int total_rounds = warm + timed;
  int margc = 1;
  MPI_Instance mpi_instance(&margc, &argv);

  WalkEngine<real_t, uint32_t> graph;
  graph.set_minLength(20);
  graph.set_init_round(2);
  graph.load_graph(V, gpath, "", true);
  graph.vertex_cn.resize(graph.get_vertex_num());
  int threads = graph.get_worker_num() + 1;

  // trainer globals as train_corpus_cuda sets them for the benchmark flags
  layer1_size = 128;
  window = 10;
  negative = 5;
  sample = 1e-3f;
  cbow = 0;
  reuseNeg = 0;
  hs = 0;
  min_count = 0;
  my_rank = 0;
  num_procs = 1;
  vertex_walker_stop_flag.assign(V, 0);
  g_v_degree.assign(V, 0);
  for (uint32_t v = 0; v < V; v++) g_v_degree[v] = graph.vertex_out_degree[v];
  vocab_max_size = (long long)V + 1000;
  vocab = (struct vocab_word *)calloc(vocab_max_size, sizeof(struct vocab_word));
  expTable = (float *)malloc((EXP_TABLE_SIZE + 1) * sizeof(float));
  for (int i = 0; i < EXP_TABLE_SIZE; i++) {
    expTable[i] = exp((i / (float)EXP_TABLE_SIZE * 2 - 1) * MAX_EXP);
    expTable[i] = expTable[i] / (expTable[i] + 1);
  }
  cudaMalloc((void **)&d_expTable, (EXP_TABLE_SIZE + 1) * sizeof(float));
  cudaMemcpy(d_expTable, expTable, (EXP_TABLE_SIZE + 1) * sizeof(float), cudaMemcpyHostToDevice);
  ReadVocabFromDegree(g_v_degree);
  InitNet();
  InitUnigramTable();
  ExponentialDecayLR lr(0.025, 0.1);

  // CSR copy for the evaluation step, as felog.cpp:72-85
  myEdgeContainer *myec = new myEdgeContainer();
  myec->adj_lists = new myAdjList[V];
  myec->adj_units = new myAdjUnit[graph.e_num];
  edge_id_t idx = 0;
  for (uint32_t v = 0; v < V; v++) {
    myec->adj_lists[v].begin = myec->adj_units + idx;
    idx += graph.csr->adj_lists[v].end - graph.csr->adj_lists[v].begin;
    myec->adj_lists[v].end = myec->adj_units + idx;
  }
  for (edge_id_t e = 0; e < graph.e_num; e++) {
    myec->adj_units[e].neighbour = graph.csr->adj_units[e].neighbour;
    myec->adj_units[e].data = graph.csr->adj_units[e].data;
  }

  if (total_rounds <= 1) stop_sampling_flag = true;
  // the timed window opens at the hand-off of round warm-1, so it covers the
  // walks and the trainings of the timed rounds
  double t_start = now_s(), walk_s = 0, train_s = 0;
  uint64_t tokens = 0, walk_tokens = 0, words = 0;
  double last_got = t_start;
  double t_end = 0;
  // trainer thread (felog.cpp runs train_corpus_cuda beside the walk, which
  // stays on the main thread)
  std::thread trainer([&]() {
  for (int r = 0; r < total_rounds; r++) {
    corpus_t corpus;
    {
      std::unique_lock<std::mutex> lock(mtx);
      cv.wait(lock, [] { return hasResource; });
      corpus = graph.out_queue.pop();
      if (r + 2 >= total_rounds) stop_sampling_flag = true;
      hasResource = false;
      cv.notify_one();
    }
    double got = now_s();
    if (r + 1 == warm) t_start = got;
    uint64_t ntok = 0;
    for (auto &s : corpus) ntok += s.size();
    alpha = lr.get_lr();
    double t0 = now_s();
    TrainModelThreadMemory(corpus);
    double t1 = now_s();
    if (r + 1 >= 2) {  // evaluation from round min_R on (word2vec.cu:2017-2062), over the walked vertices
      std::vector<vertex_id_t> nodes;
      for (uint32_t v = 0; v < walkers; v++)
        if (vertex_walker_stop_flag[v] == 0) nodes.push_back(v);
      std::vector<float> sim = batch_node_neighbor_direct_index(nodes, myec, 16384, true);
      for (size_t i = 0; i < nodes.size(); i++)
        if (sim[i] > NODE_TRAINING_CONVERGE_THRESHOLD) vertex_walker_stop_flag[nodes[i]] = 1;
    }
    double t2 = now_s();
    if (r >= warm) {
      // the walk runs ahead by one round; when it is the slower stage the
      // interval between hand-offs is the walk time of a round
      tokens += ntok;
      walk_tokens += ntok;
      words += ntok;
      walk_s += got - last_got;
      train_s += t2 - t0;
    }
    last_got = got;
    (void)t1;
  }
  t_end = now_s();
  });
  {
    WalkerConfig<real_t, uint32_t> walker_conf(walkers);
    auto ext = [&](Walker<uint32_t> &w, vertex_id_t) { return w.step >= 40 ? 0.0 : 1.0; };
    TransitionConfig<real_t, uint32_t> tr(ext);
    WalkConfig wc;
    wc.set_output_file("bench");
    graph.random_walk(&walker_conf, &tr, &wc);
  }
  trainer.join();
  graph.out_queue.closeQueue();
  if (emb_out) {
    std::vector<float> s1((size_t)vocab_size * layer1_size);
    cudaMemcpy(s1.data(), d_syn1, s1.size() * sizeof(float), cudaMemcpyDeviceToHost);
    FILE *fo = fopen(emb_out, "wb");
    if (!fo) {
      fprintf(stderr, "cannot open %s\n", emb_out);
      return 1;
    }
    for (int t = 0; t < 2; t++) {
      const float *tab = t == 0 ? syn0 : s1.data();
      fprintf(fo, "%lld %lld\n", vocab_size, layer1_size);
      for (long long a = 0; a < vocab_size; a++) {
        fprintf(fo, "%s ", vocab[a].word);
        fwrite(&tab[a * layer1_size], sizeof(float), layer1_size, fo);
        fprintf(fo, "\n");
      }
    }
    fclose(fo);
  }
  printf("{\"tokens\": %llu, \"seconds\": %.6f, \"walk_tokens\": %llu, \"walk_seconds\": %.6f, "
         "\"train_words\": %llu, \"train_seconds\": %.6f, \"threads\": %d, \"walkers\": %u}\n",
         (unsigned long long)tokens, t_end - t_start, (unsigned long long)walk_tokens, walk_s > 0 ? walk_s : 1e-9,
         (unsigned long long)words, train_s, threads, walkers);
  return 0;
}
