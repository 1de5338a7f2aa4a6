// felog - drop-in command line for the graph-embedding path.
//
// Accepts the reference's flags (graph/walk flags of
// include/option_helper.hpp:113-121, :161-165 and trainer flags of
// src/word2vec.cu:2269-2288) in any order; the reference requires the graph
// and walk flags first because its parser stops at the first unknown flag.
// Flags the reference parses but ignores (-threads, -batch-size, -iter, -train,
// -read-vocab, -r) are accepted with a note.  Behaviour that differs from the
// reference is opt-in: --use-cli-alpha honours -alpha instead of the fixed
// 0.025 e^(-0.1 r) schedule (word2vec.cu:1958, :2001).  Errors exit non-zero
// (the reference exits 0 on CUDA errors, word2vec.cu:50-56).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>
#include <string>
#include <vector>

#include "felog_gpu.h"

namespace {

struct Cli {
  std::string graph, partition, out_prefix, emb_output, save_vocab, budget_model;
  bool have_v = false, have_minl = false, have_minr = false;
  bool have_alpha = false, have_cbow = false;
};

void usage() {
  fprintf(stderr,
          "usage: felog -g <graph.bin> -v <V> -w <walkers> --min_L <L> --min_R <R> -o <prefix>\n"
          "             [--make-undirected] [-p <partition>] [--batch_size <n>] [-r <rate>]\n"
          "             [-size n] [-window n] [-negative n] [-sample x] [-alpha x] [-cbow 0|1]\n"
          "             [-reuse-neg 0|1|2|3|4] [-hs 0] [-iter n] [-min-count n] [-classes k] [-binary 0|1]\n"
          "             [-debug n] [-save-vocab f] [-emb_output f]\n"
          "             [--use-cli-alpha] [--precision fp32|bf16] [--budget plain|learned] [--budget-model f]\n"
          "             [--seed n] [--deterministic] [--weighted] [--max-rounds n] [--device n]\n");
}

// Budget MLP state: FELOG_MLP_STATE float32 values, as a 1-D .npy array or a
// raw little-endian file.
bool read_budget_model(const std::string &path, std::vector<float> &state) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) return false;
  std::vector<unsigned char> buf;
  unsigned char tmp[65536];
  size_t got;
  while ((got = fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
  fclose(f);
  size_t off = 0;
  if (buf.size() >= 10 && buf[0] == 0x93 && memcmp(&buf[1], "NUMPY", 5) == 0) {
    const int major = buf[6];
    size_t hlen, hstart;
    if (major == 1) {
      hlen = buf[8] | (buf[9] << 8);
      hstart = 10;
    } else {
      if (buf.size() < 12) return false;
      hlen = buf[8] | (buf[9] << 8) | ((size_t)buf[10] << 16) | ((size_t)buf[11] << 24);
      hstart = 12;
    }
    const std::string header(buf.begin() + hstart, buf.begin() + std::min(buf.size(), hstart + hlen));
    if (header.find("<f4") == std::string::npos || header.find("'fortran_order': False") == std::string::npos)
      return false;
    off = hstart + hlen;
  }
  if (buf.size() - off != sizeof(float) * (size_t)FELOG_MLP_STATE) return false;
  state.resize(FELOG_MLP_STATE);
  memcpy(state.data(), buf.data() + off, sizeof(float) * (size_t)FELOG_MLP_STATE);
  return true;
}

bool validate_partition(const std::string &path, uint32_t v_num) {
  // graph.hpp:854-864: one "begin end" line per rank; with one process the
  // single range must cover [0, v_num)
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return false;
  unsigned b = 0, e = 0;
  int t = fscanf(f, "%u %u", &b, &e);
  fclose(f);
  return t == 2 && b == 0;
}

}  // namespace

int main(int argc, char **argv) {
  felog_opts o;
  felog_default_opts(&o);
  Cli cli;
  if (argc == 1) {
    usage();
    return 2;
  }
  auto need = [&](int &i) -> const char * {
    if (i + 1 >= argc) {
      fprintf(stderr, "felog: argument missing for %s\n", argv[i]);
      exit(2);
    }
    return argv[++i];
  };
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "-g") cli.graph = need(i);
    else if (a == "-p") cli.partition = need(i);
    else if (a == "-v") { o.v_num = (uint32_t)strtoul(need(i), nullptr, 10); cli.have_v = true; }
    else if (a == "-w") o.walker_num = (uint32_t)strtoul(need(i), nullptr, 10);
    else if (a == "-o") cli.out_prefix = need(i);
    else if (a == "--min_L") { o.min_length = (uint32_t)strtoul(need(i), nullptr, 10); cli.have_minl = true; }
    else if (a == "--min_R") { o.min_rounds = (uint32_t)strtoul(need(i), nullptr, 10); cli.have_minr = true; }
    else if (a == "--batch_size") o.eval_batch_size = (uint32_t)strtoul(need(i), nullptr, 10);
    else if (a == "--make-undirected") o.make_undirected = 1;
    else if (a == "-r") { need(i); fprintf(stderr, "felog: note: -r has no effect (walk.hpp:637-641)\n"); }
    else if (a == "-size") o.size = atoi(need(i));
    else if (a == "-window") o.window = atoi(need(i));
    else if (a == "-negative") o.negative = atoi(need(i));
    else if (a == "-sample") o.sample = (float)atof(need(i));
    else if (a == "-alpha") { o.alpha = (float)atof(need(i)); cli.have_alpha = true; }
    else if (a == "-cbow") { o.cbow = atoi(need(i)); cli.have_cbow = true; }
    else if (a == "-reuse-neg") o.reuse_neg = atoi(need(i));
    else if (a == "-hs") o.hs = atoi(need(i));
    else if (a == "-iter") o.iter = atoi(need(i));
    else if (a == "-min-count") o.min_count = atoi(need(i));
    else if (a == "-classes") o.classes = atoi(need(i));
    else if (a == "-binary") o.binary = atoi(need(i));
    else if (a == "-debug") o.debug = atoi(need(i));
    else if (a == "-save-vocab") cli.save_vocab = need(i);
    else if (a == "-read-vocab") { need(i); fprintf(stderr, "felog: note: -read-vocab is ignored (vocabulary comes from degrees)\n"); }
    else if (a == "-train") { need(i); fprintf(stderr, "[ Warning ] '-train' option is ignored; training data comes from in-memory corpus.\n"); }
    else if (a == "-emb_output") cli.emb_output = need(i);
    else if (a == "-threads" || a == "-batch-size") { need(i); fprintf(stderr, "felog: note: %s is ignored (the reference parses it nowhere)\n", a.c_str()); }
    else if (a == "--use-cli-alpha") o.use_cli_alpha = 1;
    else if (a == "--precision") {
      std::string p = need(i);
      if (p == "fp32") o.precision = FELOG_FP32;
      else if (p == "bf16") o.precision = FELOG_BF16;
      else { fprintf(stderr, "felog: --precision must be fp32 or bf16\n"); return 2; }
    }
    else if (a == "--budget") {
      std::string p = need(i);
      if (p == "plain") o.budget_mode = FELOG_BUDGET_PLAIN;
      else if (p == "learned") o.budget_mode = FELOG_BUDGET_LEARNED;
      else { fprintf(stderr, "felog: --budget must be plain or learned\n"); return 2; }
    }
    else if (a == "--budget-model") cli.budget_model = need(i);
    else if (a == "--seed") o.seed = strtoull(need(i), nullptr, 10);
    else if (a == "--deterministic") o.deterministic = 1;
    else if (a == "--weighted") o.weighted = 1;
    else if (a == "--max-rounds") o.max_rounds = atoi(need(i));
    else if (a == "--device") o.device = atoi(need(i));
    else if (a == "-h" || a == "--help") { usage(); return 0; }
    else { fprintf(stderr, "felog: unknown flag %s\n", a.c_str()); usage(); return 2; }
  }
  if (cli.graph.empty() || !cli.have_v || !cli.have_minl || !cli.have_minr) {
    fprintf(stderr, "felog: -g, -v, --min_L and --min_R are required (option_helper.hpp:126-142)\n");
    return 2;
  }
  if (!cli.have_alpha && o.cbow) o.alpha = 0.05f;  // word2vec.cu:2276
  if (!cli.partition.empty() && !validate_partition(cli.partition, o.v_num)) {
    fprintf(stderr, "felog: partition file %s is not a valid single-range partition\n", cli.partition.c_str());
    return 2;
  }
  if (cli.have_alpha && !o.use_cli_alpha)
    fprintf(stderr, "felog: note: -alpha is overridden by the schedule 0.025 e^(-0.1 r); pass --use-cli-alpha to use it\n");
  if (cli.emb_output.empty()) fprintf(stderr, "[ Warning ] output file missing\n");

  auto t0 = std::chrono::steady_clock::now();
  felog_ctx *ctx = nullptr;
  felog_status st = felog_create(&o, &ctx);
  if (st != FELOG_OK) {
    fprintf(stderr, "felog: cannot create context (status %d)\n", (int)st);
    return 1;
  }
  auto die = [&](const char *what) {
    fprintf(stderr, "felog: %s failed: %s\n", what, felog_last_error(ctx));
    felog_destroy(ctx);
    exit(1);
  };
  if (felog_load_graph_file(ctx, cli.graph.c_str(), o.v_num, o.make_undirected) != FELOG_OK) die("load_graph");
  auto t1 = std::chrono::steady_clock::now();
  if (o.weighted && felog_build_alias(ctx) != FELOG_OK) die("build_alias");
  if (o.budget_mode == FELOG_BUDGET_LEARNED) {
    // default: the model shipped beside this executable
    std::string path = cli.budget_model;
    if (path.empty()) {
      char exe[4096];
      const ssize_t n = readlink("/proc/self/exe", exe, sizeof exe - 1);
      std::string dir = n > 0 ? std::string(exe, (size_t)n) : std::string(".");
      dir = dir.substr(0, dir.find_last_of('/') == std::string::npos ? 0 : dir.find_last_of('/'));
      path = (dir.empty() ? std::string(".") : dir) + "/budget_mlp_c4.npy";
    }
    std::vector<float> state;
    if (!read_budget_model(path, state)) {
      fprintf(stderr, "felog: cannot read the budget model %s (%d float32 values)\n", path.c_str(), FELOG_MLP_STATE);
      felog_destroy(ctx);
      return 2;
    }
    if (felog_mlp_set_params(ctx, state.data()) != FELOG_OK) die("budget model");
  }
  felog_run_stats rs;
  if (felog_run(ctx, &rs) != FELOG_OK) die("run");
  auto t2 = std::chrono::steady_clock::now();
  printf("> rounds %u, walk tokens %llu, trained words %llu, unconverged %llu\n", rs.rounds,
         (unsigned long long)rs.walk_tokens, (unsigned long long)rs.train_words,
         (unsigned long long)rs.final_unconverged);
  printf("> walk %.3f ms (%.3g steps/s), train %.3f ms (%.3g words/s), budget %.3f ms\n", rs.walk_ms,
         rs.walk_tokens / (rs.walk_ms * 1e-3), rs.train_ms, rs.train_words / (rs.train_ms * 1e-3), rs.budget_ms);
  if (!cli.save_vocab.empty()) {
    uint64_t vs = 0;
    felog_vocab_info(ctx, &vs, nullptr);
    std::vector<uint32_t> vv(vs), deg(o.v_num);
    felog_get_vocab(ctx, vv.data(), nullptr);
    felog_get_degrees(ctx, deg.data());
    FILE *f = fopen(cli.save_vocab.c_str(), "wb");
    if (!f) die("save-vocab");
    for (uint64_t i = 0; i < vs; i++) fprintf(f, "%u %lld\n", vv[i], (long long)deg[vv[i]]);  // word2vec.cu:825-830
    fclose(f);
  }
  if (!cli.emb_output.empty()) {
    if (o.classes > 0) {
      // class ids from the GPU spherical K-means (10 passes at most)
      uint64_t vs = 0;
      felog_vocab_info(ctx, &vs, nullptr);
      std::vector<uint32_t> vv(vs);
      std::vector<int32_t> cl(vs);
      felog_get_vocab(ctx, vv.data(), nullptr);
      if (felog_cluster_embeddings(ctx, o.classes, 10, cl.data(), nullptr, nullptr) != FELOG_OK)
        die("cluster_embeddings");
      FILE *f = fopen(cli.emb_output.c_str(), "wb");
      if (!f) die("emb_output");
      for (uint64_t a = 0; a < vs; a++) fprintf(f, "%u %d\n", vv[a], cl[a]);
      fclose(f);
    } else if (felog_write_embeddings(ctx, cli.emb_output.c_str()) != FELOG_OK) {
      die("write_embeddings");
    }
  }
  auto t3 = std::chrono::steady_clock::now();
  auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
  printf("> load graph time: %lf\n> WHOLE TIME: %lf\n", sec(t0, t1), sec(t0, t3));
  (void)t2;
  felog_destroy(ctx);
  return 0;
}
