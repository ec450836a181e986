// preprocess_graph: the reference's preprocessing tool
// (src/preprocess/PreprocessGraph.cpp:5-37) over the C ABI.  Same flags
// (-f GRAPH_FILENAME -d DIRECTED -o OUTPUT_FORMAT) and the same output names:
// the input name plus ".snap.txt" (-o 0), ".bin" (-o 1, default) or
// ".adj.txt" with ".adj.txt.info" (-o 3).
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "../../include/sme.h"

namespace {
const char* Arg(int argc, char** argv, const char* opt, const char* def) {
  for (int i = 1; i + 1 < argc; ++i)
    if (std::strcmp(argv[i], opt) == 0) return argv[i + 1];
  return def;
}
int Die(const char* what, sme_status st) {
  std::cerr << what << " failed (status " << st << "): " << sme_last_error() << std::endl;
  return 1;
}
}  // namespace

int main(int argc, char** argv) {
  if (argc == 1) {
    std::cout << "./preprocess_graph -f GRAPH_FILENAME(SNAP format) -d DIRECTED -o OUTPUT_FORMAT" << std::endl;
    std::cout << "OUTPUT_FORMAT: 0  for .snap, 1 (Default) for .bin, 3 for .adj, " << std::endl;
    return 255;
  }
  const std::string filename = Arg(argc, argv, "-f", "../../data/com-dblp.ungraph.txt");
  const int directed = std::atoi(Arg(argc, argv, "-d", "0"));
  const int format = std::atoi(Arg(argc, argv, "-o", "1"));
  if (format != 0 && format != 1 && format != 3) {
    std::cerr << "-o must be 0 (SNAP), 1 (BIN) or 3 (ADJ)" << std::endl;
    return 1;
  }
  sme_graph* g = nullptr;
  sme_status st = sme_graph_load(filename.c_str(), directed, &g);
  if (st != SME_OK) return Die("graph load", st);
  if ((st = sme_graph_preprocess(g)) != SME_OK) return Die("preprocess", st);
  if ((st = sme_graph_validate(g)) != SME_OK) return Die("validate", st);
  if (format == 0)
    st = sme_graph_write_snap(g, (filename + ".snap.txt").c_str());
  else if (format == 1)
    st = sme_graph_write_bin(g, (filename + ".bin").c_str());
  else
    st = sme_graph_write_adj(g, (filename + ".adj.txt").c_str());
  if (st != SME_OK) return Die("write", st);
  uint64_t n = 0, m = 0;
  sme_graph_info(g, &n, &m, nullptr);
  std::cout << "vertex_count=" << n << ",edge_count=" << m << std::endl;
  sme_graph_free(g);
  return 0;
}
