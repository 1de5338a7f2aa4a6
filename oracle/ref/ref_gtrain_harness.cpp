// Runs the reference's held-out split tool on a text edge file: the tool's own
// source file (src/tools/gtrain.cpp), compiled unmodified with its main()
// renamed, called through its gtrain<vertex_id_t>() template.  Its random
// draws are injected: rand() returns value k of the split stream (the 31-bit
// counter-based stream felog_heldout_split draws from, restated below for
// this binary) and srand() does nothing, so the tool and the library see the
// same draws.
//
//   ref_gtrain <edges.txt> <train.txt> <test_edges.txt> <test_labels.txt> <sample> <v_num> <seed>
//
// Test infrastructure only: it generates the golden split vectors.
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
#include <ctime>
#include <fstream>
#include <functional>
#include <iostream>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <queue>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>
#include <omp.h>

namespace {
uint64_t g_seed = 0, g_k = 0;
inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
inline uint64_t draw(uint64_t seed, uint64_t id, uint64_t k) {
  return mix64(mix64(seed ^ 0x5DEECE66DULL) + mix64(id * 0xD1B54A32D192ED03ULL + k));
}
}  // namespace

int felog_inj_rand() { return (int)(draw(g_seed ^ 0x5117ULL, 1, g_k++) >> 33); }
void felog_inj_srand(unsigned) {}

#define rand felog_inj_rand
#define srand felog_inj_srand
#define main gtrain_tool_main
#include "tools/gtrain.cpp"
#undef main
#undef srand
#undef rand

int main(int argc, char **argv) {
  if (argc != 8) {
    fprintf(stderr, "usage: %s edges.txt train.txt test_edges.txt test_labels.txt sample v_num seed\n", argv[0]);
    return 2;
  }
  thread_num = 1;
  g_seed = strtoull(argv[7], nullptr, 10);
  g_k = 0;
  gtrain<vertex_id_t>(argv[1], argv[2], argv[3], argv[4], (float)atof(argv[5]),
                      (vertex_id_t)strtoul(argv[6], nullptr, 10));
  return 0;
}
