// patternmatchgpu: command-line driver with the flags and the final output
// line of the reference GPU program (src/gpu/PatternMatchGPU.cu:11-83,
// help text src/gpu/PatternMatchGPUInstance.cuh:230-271, result line
// src/gpu/executor/PatternMatch.cuh:84-86).  Links only against libsme.so.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/sme.h"

namespace {
// "-flag value" lookup (CommandLine, src/utils/CommandLine.h:46-66).
struct Args {
  int argc;
  char** argv;
  const char* Get(const char* opt) const {
    for (int i = 1; i + 1 < argc; ++i)
      if (std::strcmp(argv[i], opt) == 0) return argv[i + 1];
    return nullptr;
  }
  std::string Str(const char* opt, const std::string& def) const {
    const char* v = Get(opt);
    return v ? v : def;
  }
  long Int(const char* opt, long def) const {
    const char* v = Get(opt);
    return v ? std::atol(v) : def;
  }
};

void Help() {
  std::cout << "./patternmatchgpu -f FILENAME -d IS_DIRECTED -a ALGORITHM -q QUERY "
               "-e PARTITION_FILENAME -p PARTITION_NUM -t THREAD_NUM -v DEVICE_NUM "
               "-m EXECUTE_MODE -o VARIANT [ -l MATERIALIZE -r ENABLE_ORDERING -c "
               "LAZY_TRAVERSAL_COMPRESS_LEVEL -x GPU_LIGHT_ITP_VARIANT -y GPU_LIGHT_EXT_VARIANT"
               " -g REUSE_AUTOGEN -b ROOT_BEGIN -n ROOT_END -M MEM_LIMIT_MB -O DEGREE_ORDER ]\n";
  std::cout << "ALGORITHM: ,GPU_GPSM=4,GPU_GPSM_REUSE=5,GPU_LIGHT=6\n";
  std::cout << "QUERY: Q0 (TRIANGLE) 0, Q1 (square) 1, Q2 (chordal square) 2, Q3 (4 clique) 3, "
               "Q4 (house) 4, Q5 (quad triangle) 5, Q6 (near5clique) 6, Q7 (5 clique) 7, "
               "Q8 (chordal roof) 8, Q9 (three triangle) 9, Q10 (solar square) 10, Q11 (6 clique) 11, "
               "Q12 (near near 5 clique) 12, Q13 (triangle in diamond) 13\n";
  std::cout << "MODE: HYBRID_CPU_GPU=0 (partition counts; -e PARTITION_FILENAME -p PARTITION_NUM), "
               "IN_MEMORY_GPU=1, EXTERNAL_GPU=2\n";
  std::cout << "LAZY_TRAVERSAL_COMPRESS_LEVEL: COMPRESS_LEVEL_MATERIALIZE=0, "
               "COMPRESS_LEVEL_NON_MATERIALIZE=1, COMPRESS_LEVEL_NON_MATERIALIZE_OPT=2, "
               "COMPRESS_LEVEL_SPECIAL(DEFAULT)=3\n";
  std::cout << "GPU_LIGHT_EXT_VARIANT: EXT_CACHE(DEFAULT)=0, EXT_UMA=1\n";
  std::cout << "DEGREE_ORDER: none(DEFAULT)=0, renumber by degree=1, renumber and orient (clique "
               "queries 0/3/7/11 only)=2\n";
}

int Die(const char* what, sme_status st) {
  std::cerr << what << " failed (status " << st << "): " << sme_last_error() << std::endl;
  return 1;
}
}  // namespace

int main(int argc, char** argv) {
  if (argc == 1) {
    Help();
    return 255;
  }
  Args a{argc, argv};
  std::string filename = a.Str("-f", "../../data/com-dblp.ungraph.txt");
  int directed = (int)a.Int("-d", 1);
  sme_opts o;
  sme_opts_default(&o);
  o.algo = (int32_t)a.Int("-a", 0);
  o.query_type = (int32_t)a.Int("-q", 0);
  int partition_num = (int)a.Int("-p", 1);
  int dev_num = (int)a.Int("-v", 1);
  o.execute_mode = (int32_t)a.Int("-m", SME_HYBRID_CPU_GPU);
  int materialize = (int)a.Int("-l", 0);
  o.compress_level = (int32_t)a.Int("-c", SME_COMPRESS_SPECIAL);
  o.enable_ordering = (int32_t)a.Int("-r", 1);
  o.ext_variant = (int32_t)a.Int("-y", SME_EXT_CACHE);
  o.reuse_autogen = (int32_t)a.Int("-g", -1);
  o.root_begin = (uint64_t)a.Int("-b", 0);
  o.root_end = (uint64_t)a.Int("-n", 0);
  o.mem_limit_bytes = (uint64_t)a.Int("-M", 0) << 20;
  const int degree_order = (int)a.Int("-O", 0);

  std::cout << "filename=" << filename << ",directed=" << directed << ",algo=" << o.algo
            << ",query_type=" << o.query_type << std::endl;
  std::cout << ",partition_filename=" << a.Str("-e", "") << ",partition_num=" << partition_num
            << ",thread_num=" << a.Int("-t", 1) << ",execute_mode=" << o.execute_mode
            << ",variant=" << a.Int("-o", 1) << ",materialize=" << materialize
            << ",lazy_traversal_compress_level=" << o.compress_level
            << ",enable_ordering=" << o.enable_ordering << ",gpu_light_ext_variant=" << o.ext_variant
            << std::endl;
  if (partition_num < 1) {
    std::cerr << "-p must be >= 1" << std::endl;
    return 1;
  }
  if (partition_num != 1 && o.execute_mode != SME_HYBRID_CPU_GPU) {
    std::cerr << "-p > 1 partitions the graph for -m 0 (HYBRID_CPU_GPU) only" << std::endl;
    return 1;
  }
  if (dev_num != 1) std::cout << "note: running on device 0 only (-v " << dev_num << " requested)" << std::endl;

  sme_graph* g = nullptr;
  sme_status st = sme_graph_load(filename.c_str(), directed, &g);
  if (st != SME_OK) return Die("graph load", st);
  if (degree_order == 1 || degree_order == 2) {
    sme_graph* d = nullptr;
    st = sme_graph_degree_order(g, degree_order - 1, &d, nullptr);
    if (st != SME_OK) return Die("degree order", st);
    sme_graph_free(g);
    g = d;
  } else if (degree_order != 0) {
    std::cerr << "-O must be 0, 1 or 2" << std::endl;
    return 1;
  }
  uint64_t n = 0, m = 0, dmax = 0;
  sme_graph_info(g, &n, &m, &dmax);
  std::cout << "vertex_count=" << n << ",edge_count=" << m << ",max_degree=" << dmax << std::endl;

  uint64_t count = 0;
  if (o.execute_mode == SME_HYBRID_CPU_GPU) {
    // -m 0: intra-partition counts per partition of the -e file, the rest is
    // inter-partition; the total is the answer
    if (materialize) {
      std::cerr << "-l 1 runs in -m 1 (IN_MEMORY_GPU)" << std::endl;
      return 1;
    }
    std::vector<uint32_t> part(n ? n : 1);
    st = sme_read_partition_file(a.Str("-e", "").c_str(), n, (uint32_t)partition_num, part.data());
    if (st != SME_OK) return Die("partition file", st);
    std::vector<uint64_t> intra(partition_num);
    st = sme_count_partitioned(g, &o, part.data(), (uint32_t)partition_num, &count, intra.data());
    if (st != SME_OK) return Die("count", st);
    uint64_t intra_sum = 0;
    for (int p = 0; p < partition_num; ++p) {
      std::cout << "partition_id=" << p << ",intra_partition_count=" << intra[p] << std::endl;
      intra_sum += intra[p];
    }
    std::cout << "inter_partition_count=" << count - intra_sum << std::endl;
  } else if (materialize) {
    // enumerate into a host buffer sized by a first counting pass
    st = sme_count(g, &o, &count);
    if (st != SME_OK) return Die("count", st);
    int k = sme_query_vertex_count(o.query_type);
    std::vector<uint32_t> out((size_t)count * k + 1);
    uint64_t got = 0;
    st = sme_enumerate(g, &o, out.data(), count, &got);
    if (st != SME_OK) return Die("enumerate", st);
    count = got;
  } else {
    st = sme_count(g, &o, &count);
    if (st != SME_OK) return Die("count", st);
  }
  sme_stats s;
  sme_last_stats(&s);
  static const char* kPhases[8] = {"compute_time",        "materialize_time",        "filter_compute_time",
                                   "compute_count_time",  "compute_path_count_time", "count_time",
                                   "organize_batch_time", "load_subgraph_time"};
  for (int i = 0; i < 8; ++i)
    if (s.phase_ms[i] > 0) std::cout << kPhases[i] << "=" << s.phase_ms[i] << "ms" << std::endl;
  std::cout << "kernel_time=" << s.kernel_ms << "ms,device_time=" << s.device_ms << "ms,batches=" << s.batches
            << ",kernel_launches=" << s.kernel_launches << ",peak_device_bytes=" << s.peak_device_bytes
            << std::endl;
  std::cout << "total_match_count=" << count << ", elapsed_time=" << s.elapsed_ms << "ms" << std::endl;
  sme_graph_free(g);
  return 0;
}
