// Test infrastructure: times the reference's own CPU_WCOJ on root tasks.
//
// The reference's CPU program (src/cpu/PatternMatchCPU.cpp:55-62) counts a
// query over every root of a graph: CPUWCOJoin::Execute
// (src/cpu/CPUWCOJ.h:21-77) runs, per root u, DFS(thread, 1, path=[u], ...)
// under `#pragma omp parallel for schedule(dynamic)`.  A whole-graph run of a
// 4-clique, 4-cycle or diamond on R-MAT scale 20 takes tens of minutes on a
// host, so this driver runs the same per-root DFS (the reference's code,
// compiled from its unmodified headers where they lie) over a root task
// instead: a strided root range or a slice of an explicit root list, each
// task in the same OpenMP loop shape as Execute.  It prints, per task, the
// reference's result line (total_match_count=..., elapsed_time=...ms).
//
//   ref_wcoj_task -f GRAPH.bin -q QUERY -t THREADS [-r ROOTS.u32] TASK...
//   TASK = S:STRIDE:OFFSET  roots OFFSET, OFFSET+STRIDE, ... < n
//        | L:START:COUNT    roots ROOTS[START .. START+COUNT) of the list file
//                           (raw little-endian uint32 vertex ids)
//
// Built by oracle/Makefile (`make -C oracle ref`) into oracle/_ref/ with the
// reference's own flags; used only by the bench's reference arm and CPU
// baseline and by tests.
#include <omp.h>
#include <pthread.h>

#include <algorithm>
#include <cassert>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "CPUGraph.h"
#include "Meta.h"
#include "TraversalPlan.h"

// CPUWCOJoin::DFS is private; Execute, its only caller, has no root-range
// form.  Opening the class's access lets this driver call the same DFS per
// root without editing the reference's header.
#define private public
#include "CPUWCOJ.h"
#undef private

namespace {

struct Task {
  bool list;                 // slice of the root list, else a strided range
  unsigned long long a, b;   // stride, offset | start, count
};

bool ParseTask(const char* s, Task* t) {
  if ((s[0] != 'S' && s[0] != 'L') || s[1] != ':') return false;
  t->list = s[0] == 'L';
  char* end = nullptr;
  t->a = std::strtoull(s + 2, &end, 10);
  if (!end || *end != ':' || (!t->list && t->a == 0)) return false;
  t->b = std::strtoull(end + 1, &end, 10);
  return end && *end == '\0';
}

}  // namespace

int main(int argc, char* argv[]) {
  std::string filename, roots_file;
  int query_type = -1, threads = 1;
  std::vector<Task> tasks;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "-f" && i + 1 < argc) {
      filename = argv[++i];
    } else if (a == "-q" && i + 1 < argc) {
      query_type = std::atoi(argv[++i]);
    } else if (a == "-r" && i + 1 < argc) {
      roots_file = argv[++i];
    } else if (a == "-t" && i + 1 < argc) {
      threads = std::max(1, std::atoi(argv[++i]));
    } else {
      Task t;
      if (!ParseTask(argv[i], &t)) {
        std::cerr << "bad argument: " << a << std::endl;
        return 2;
      }
      tasks.push_back(t);
    }
  }
  if (filename.empty() || query_type < 0 || tasks.empty()) {
    std::cerr << "usage: ref_wcoj_task -f GRAPH.bin -q QUERY -t THREADS [-r ROOTS.u32] "
                 "S:STRIDE:OFFSET | L:START:COUNT ..."
              << std::endl;
    return 2;
  }
  std::vector<uintV> root_list;
  if (!roots_file.empty()) {
    std::ifstream in(roots_file.c_str(), std::ios::binary | std::ios::ate);
    if (!in) {
      std::cerr << "cannot read " << roots_file << std::endl;
      return 2;
    }
    root_list.resize((size_t)in.tellg() / sizeof(uintV));
    in.seekg(0);
    in.read(reinterpret_cast<char*>(root_list.data()), root_list.size() * sizeof(uintV));
  }

  // As PatternMatchCPU.cpp:52-62 with -a 0 (one partition, one device).
  Query* query = new Query((QueryType)query_type);
  Graph* graph = new Graph(filename, false);
  TraversalPlan* plan = new TraversalPlan(query, 1, 1);
  CPUWCOJoin* wcoj = new CPUWCOJoin(plan, graph, threads);

  std::vector<std::vector<uintV> > intersect_levels;
  plan->GetOrderedConnectivity(intersect_levels);
  AllCondType conditions;
  plan->GetOrderedOrdering(conditions);
  omp_set_num_threads(threads);
  const size_t nv = graph->GetVertexCount();
  std::vector<std::vector<uintV> > paths(threads, std::vector<uintV>(plan->GetVertexCount()));

  for (const Task& t : tasks) {
    if (t.list && t.a + t.b > root_list.size()) {
      std::cerr << "list slice out of range" << std::endl;
      return 2;
    }
    const long long nroots =
        t.list ? (long long)t.b : (t.b < nv ? (long long)((nv - 1 - t.b) / t.a + 1) : 0);
    const uintV* slice = t.list ? root_list.data() + t.a : nullptr;
    if (slice)
      for (long long r = 0; r < nroots; ++r)
        if (slice[r] >= nv) {
          std::cerr << "root " << slice[r] << " out of range" << std::endl;
          return 2;
        }
    auto t0 = std::chrono::steady_clock::now();
    long long total_match_count = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total_match_count)
    for (long long r = 0; r < nroots; ++r) {
      long long ans = 0;
      const int tid = omp_get_thread_num();
      uintV* path = paths[tid].data();
      path[0] = slice ? slice[r] : (uintV)(t.b + (unsigned long long)r * t.a);
      wcoj->DFS(tid, 1, path, ans, intersect_levels, conditions);
      total_match_count += ans;
    }
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "task=" << (t.list ? "L:" : "S:") << t.a << ":" << t.b << ", roots=" << nroots
              << ", total_match_count=" << total_match_count << ", elapsed_time=" << ms << "ms" << std::endl;
  }
  return 0;
}
