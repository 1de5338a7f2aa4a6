// Runs the reference's common-neighbour tool on a text edge file: the tool's
// own source file (src/tools/gcn.cpp), compiled unmodified with its main()
// renamed, called through its gcn<EmptyData>() template with one thread.
//
//   ref_gcn <edges.txt> <out.txt> <v_num> <make_undirected 0|1>
//
// Test infrastructure only: it generates the golden common-neighbour vectors.
#include <cstdlib>
#define main gcn_tool_main
#include "tools/gcn.cpp"
#undef main

int main(int argc, char **argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s edges.txt out.txt v_num make_undirected\n", argv[0]);
    return 2;
  }
  thread_num = 1;
  gcn<EmptyData>(argv[1], argv[2], atoi(argv[4]) != 0, (vertex_id_t)strtoul(argv[3], nullptr, 10));
  return 0;
}
