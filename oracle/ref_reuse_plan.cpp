// Test infrastructure: prints the reference's hard-coded reuse plan.
//
// The reference's test_plan (src/query/TestPlan.cpp:38-48) prints the
// ReuseTraversalPlan with autogen on (-t 1); the GPU reuse-BFS path
// (patternmatchgpu -a 5) builds it with autogen off, which picks the plans of
// src/query/optimizer/ReuseTraversalPlanHardCode.h:9-72.  This driver builds
// that plan the way test_plan builds the others (one partition, one device,
// -m 1, -o 0) and prints it with the reference's own Print(), then each reuse
// meta's vertex mapping ("mapping level L: m0 m1 ...", n = none), which
// Print() leaves out.
//
//   ref_reuse_plan QUERY
//
// Queries without a hard-coded plan (Q1, Q4) end in the reference's assert.
// Built by oracle/Makefile (`make -C oracle ref`) into oracle/_ref/.
#include <cstdlib>
#include <iostream>

#include "ReuseTraversalPlan.h"

int main(int argc, char* argv[]) {
  if (argc != 2) {
    std::cerr << "usage: ref_reuse_plan QUERY" << std::endl;
    return 2;
  }
  Query* query = new Query((QueryType)std::atoi(argv[1]));
  ReuseTraversalPlan* plan = new ReuseTraversalPlan(query, 1, 1, (ExecuteMode)1, (Variant)0, false);
  plan->Print();
  LevelReuseIntersectPlan& levels = plan->GetLevelReuseIntersectPlan();
  for (size_t i = 0; i < levels.size(); ++i)
    for (auto& meta : levels[i].GetReuseConnectivityMeta()) {
      std::cout << "mapping level " << i << ":";
      for (auto x : meta.GetMapping()) std::cout << " " << x;
      std::cout << std::endl;
    }
  return 0;
}
