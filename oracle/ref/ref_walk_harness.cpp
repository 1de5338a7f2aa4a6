/*
 * Reference walk harness (test infrastructure, never shipped).
 *
 * Compiles the reference's own walk engine (include/walk.hpp, graph.hpp,
 * path.hpp, storage.hpp) unmodified against the loopback MPI shim and runs
 * `WalkEngine::random_walk` at np = 1 with ONE worker thread, exactly as
 * src/examples/felog.cpp:51-136 drives it, but with every random draw
 * injected so the result is reproducible:
 *
 *   - the candidate index draw `gen->gen(degree)` (walk.hpp:976) comes from a
 *     generator placed over the engine's per-thread StdRandNumGenerator
 *     (util.hpp:22-47; reachable through the public get_thread_local_rand_gen,
 *     walk.hpp:515-518);
 *   - the trace draw `rand()` (walk.hpp:1005) is redirected by macro to
 *     `felog_inj_rand`;
 *   - walker boundaries in the draw sequence are taken from the first access to
 *     each walker's visit map `walker_to_path[walker.id][current_v]++`
 *     (walk.hpp:874, :926): the map type is replaced by a subclass of
 *     std::unordered_map that reports that access.
 *
 * With one thread and np = 1 the engine walks each walker to completion in
 * ascending id order (walk.hpp:899-1104), so the global draw log splits into
 * per-walker streams.  A consumer thread plays the trainer's side of the
 * walk/train hand-off (walk.hpp:720-752; word2vec.cu:1990-1998) and sets
 * stop_sampling_flag before the last round is pushed so exactly `rounds`
 * complete rounds are walked.
 *
 * Output (binary, little endian), one block per round:
 *   u32 n_sentences, then per sentence: u32 len, u32 tokens[len]
 * followed by the draw log:
 *   u32 n_walkers_logged, then per logged walker (in processing order):
 *   u32 round, u32 start_vertex, u32 n_idx, u32 idx[n_idx], u32 n_p, i32 p[n_p]
 *
 * Usage: ref_walk <graph.bin> <V> <min_L> <rounds> <seed> <out.bin>
 *                 [stopflags.u8 (V bytes, applied from round 1)] [walker_num]
 */
#include <algorithm>
#include <atomic>
#include <cassert>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <queue>
#include <random>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>
#include <omp.h>

/* ---- draw injection state ------------------------------------------------ */
struct WalkerLog {
  uint32_t round;
  uint32_t start;
  std::vector<uint32_t> idx;
  std::vector<int32_t> p;
};
static std::vector<WalkerLog> g_log;
static uint64_t g_active_per_round = 1; /* walkers started per round */
static uint64_t g_seed = 1;
static uint64_t g_ctr = 0;

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
static inline uint64_t next_draw() { return splitmix64(g_seed * 0x100000001B3ULL + (g_ctr++)); }

/* called on the first visit-map access of a walker (its start vertex) */
static void felog_walker_begin(uint32_t start_vertex) {
  WalkerLog w;
  w.round = (uint32_t)(g_log.size() / g_active_per_round) + 1;
  w.start = start_vertex;
  g_log.push_back(std::move(w));
}

int felog_inj_rand() {
  assert(!g_log.empty());
  uint64_t r = next_draw();
  int32_t v;
  /* exercise both ends of the range now and then */
  switch (r & 63) {
    case 0: v = 0; break;
    case 1: v = RAND_MAX; break;
    default: v = (int32_t)((r >> 8) % ((uint64_t)RAND_MAX + 1)); break;
  }
  g_log.back().p.push_back(v);
  return v;
}

/* visit-map subclass: reports the first access of each walker */
namespace std {
template <class K, class V, class H = hash<K>, class E = equal_to<K>,
          class A = allocator<pair<const K, V>>>
struct felog_probe_map : public unordered_map<K, V, H, E, A> {
  using base = unordered_map<K, V, H, E, A>;
  using base::base;
  felog_probe_map() = default;
  V &operator[](const K &k) {
    if constexpr (is_same<K, unsigned int>::value && is_same<V, int>::value) {
      if (this->empty()) felog_walker_begin((uint32_t)k);
    }
    return base::operator[](k);
  }
};
}  // namespace std

#define unordered_map felog_probe_map
#define rand felog_inj_rand
#include "walk.hpp"
#undef rand
#undef unordered_map

/* globals the trainer translation unit normally defines (word2vec.cu:58-62) */
vector<int> vertex_walker_stop_flag;
std::mutex mtx;
std::condition_variable cv;
bool hasResource = false;
std::atomic<bool> pauseWalk{false};

class InjectedGen : public StdRandNumGenerator {
 public:
  vertex_id_t gen(vertex_id_t upper_bound) override {
    assert(!g_log.empty());
    uint64_t r = next_draw();
    vertex_id_t v = (vertex_id_t)(r % upper_bound);
    g_log.back().idx.push_back(v);
    return v;
  }
  float gen_float(float upper_bound) override { return 0.0f * upper_bound; }
};
static_assert(sizeof(InjectedGen) == sizeof(StdRandNumGenerator), "same object size");

int main(int argc, char **argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s graph.bin V min_L rounds seed out.bin [stopflags] [walker_num]\n", argv[0]);
    return 2;
  }
  const char *graph_path = argv[1];
  uint32_t V = (uint32_t)strtoul(argv[2], nullptr, 10);
  uint32_t min_L = (uint32_t)strtoul(argv[3], nullptr, 10);
  uint32_t rounds = (uint32_t)strtoul(argv[4], nullptr, 10);
  g_seed = strtoull(argv[5], nullptr, 10);
  const char *out_path = argv[6];
  const char *stop_path = argc > 7 ? argv[7] : "";
  uint32_t walker_num = argc > 8 ? (uint32_t)strtoul(argv[8], nullptr, 10) : V;

  int margc = 1;
  char **margv = argv;
  MPI_Instance mpi_instance(&margc, &margv);
  omp_set_num_threads(1);

  WalkEngine<real_t, uint32_t> graph;
  graph.set_concurrency(1);
  graph.set_minLength(min_L);
  graph.set_init_round(1);
  graph.load_graph(V, graph_path, "", true);
  graph.vertex_cn.resize(graph.get_vertex_num());

  vertex_walker_stop_flag.assign(V, 0);
  if (stop_path[0]) {
    FILE *f = fopen(stop_path, "rb");
    assert(f);
    std::vector<uint8_t> flags(V);
    size_t got = fread(flags.data(), 1, V, f);
    assert(got == V);
    fclose(f);
    for (uint32_t v = 0; v < V; v++) vertex_walker_stop_flag[v] = flags[v] ? 1 : 0;
  }

  g_active_per_round = 0;
  for (uint32_t w = 0; w < walker_num; w++) g_active_per_round += vertex_walker_stop_flag[w % V] ? 0 : 1;
  if (g_active_per_round == 0) g_active_per_round = 1;

  /* one worker thread: replace its generator in place */
  StdRandNumGenerator *slot = graph.get_thread_local_rand_gen();
  new (slot) InjectedGen();

  std::vector<corpus_t> rounds_out;
  if (rounds <= 1) stop_sampling_flag = true;
  std::thread consumer([&]() {
    for (uint32_t r = 1; r <= rounds; r++) {
      std::unique_lock<std::mutex> lock(mtx);
      cv.wait(lock, [] { return hasResource; });
      rounds_out.push_back(graph.out_queue.pop());
      if (r + 1 >= rounds) stop_sampling_flag = true;
      hasResource = false;
      cv.notify_one();
    }
  });

  WalkerConfig<real_t, uint32_t> walker_conf(walker_num);
  auto extension_comp = [&](Walker<uint32_t> &walker, vertex_id_t) { return walker.step >= 40 ? 0.0 : 1.0; };
  TransitionConfig<real_t, uint32_t> tr_conf(extension_comp);
  WalkConfig walk_conf;
  walk_conf.set_output_file("harness");
  graph.random_walk(&walker_conf, &tr_conf, &walk_conf);
  consumer.join();

  FILE *fo = fopen(out_path, "wb");
  assert(fo);
  for (auto &corpus : rounds_out) {
    uint32_t n = (uint32_t)corpus.size();
    fwrite(&n, 4, 1, fo);
    for (auto &s : corpus) {
      uint32_t len = (uint32_t)s.size();
      fwrite(&len, 4, 1, fo);
      fwrite(s.data(), 4, len, fo);
    }
  }
  uint32_t nw = (uint32_t)g_log.size();
  fwrite(&nw, 4, 1, fo);
  for (auto &w : g_log) {
    uint32_t ni = (uint32_t)w.idx.size(), np = (uint32_t)w.p.size();
    fwrite(&w.round, 4, 1, fo);
    fwrite(&w.start, 4, 1, fo);
    fwrite(&ni, 4, 1, fo);
    fwrite(w.idx.data(), 4, ni, fo);
    fwrite(&np, 4, 1, fo);
    fwrite(w.p.data(), 4, np, fo);
  }
  fclose(fo);
  fprintf(stderr, "ref_walk: %zu rounds, %u walkers logged\n", rounds_out.size(), nw);
  return 0;
}
