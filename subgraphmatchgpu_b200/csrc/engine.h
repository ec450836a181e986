// Device engine interface (engine.cu).
#pragma once

#include <cuda_runtime.h>

#include "sme_internal.h"

namespace sme {

// Resident device copy of a CSR graph.
struct DeviceGraph {
  int device = -1;
  uint64_t n = 0, m = 0;
  uintE* row_ptrs = nullptr;
  uintV* cols = nullptr;
  bool host_mapped = false;  // cols live in mapped pinned host memory (EXT_UMA)
  bool in_arena = false;     // arrays live in a context's arena (per-call upload)
  // dense adjacency bitmaps of the highest-degree vertices
  int32_t* hub_slot = nullptr;  // per vertex: bitmap slot or -1
  uint32_t* bitmaps = nullptr;  // nhubs x words
  uint32_t words = 0, nhubs = 0;
  // per hub, one bit per 32-vertex block of its bitmap (set: the block holds
  // a neighbour); nhubs x cwords, null when not built
  uint32_t* coarse = nullptr;
  uint32_t cwords = 0;
};

// Stack allocator over one device allocation.  Levels are processed depth
// first, so every allocation of a level batch is released (in LIFO order)
// before the next batch of the same level starts.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, top = 0, peak = 0;
  void* Alloc(size_t bytes);
  size_t Mark() const { return top; }
  void Release(size_t mark) { top = mark; }
  size_t Free() const { return cap - top; }
};

// Byte ranges a per-call packed upload is cut into (copy and expansion overlap).
constexpr int kUploadChunks = 8;

// Per-device execution context: stream, arena, pinned staging buffers.
struct DeviceContext {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;             // per-call uploads
  cudaEvent_t copy_ev[kUploadChunks + 1] = {};    // upload ranges landed
  Arena arena;
  uint64_t* h_pinned = nullptr;  // small pinned host buffer for batch bounds
  size_t pinned_words = 0;
  ~DeviceContext();
};

// Allocates a context with an arena of `bytes` (0 = most of free memory).
DeviceContext* CreateContext(int device, uint64_t bytes);
void DestroyContext(DeviceContext* c);

DeviceGraph* UploadGraph(const HostGraph& g, int device, cudaStream_t stream, uint64_t* h2d_bytes);
// Per-call upload into the context's arena: no device allocation; the caller
// takes an arena mark before and releases it after the run.
DeviceGraph* UploadGraphToArena(const HostGraph& g, DeviceContext& ctx, uint64_t* h2d_bytes);
void FreeDeviceGraph(DeviceGraph* d);

// The first-level vertices of one run (an IntraPartScheduler task,
// src/gpu/task/IntraPartScheduler.h:77-101, generalised): the roots
// begin, begin+stride, ... < end, or, when `list` is set, exactly
// list[0 .. list_len) in that order (host memory, ids below n).
struct RootTask {
  uint64_t begin = 0, end = 0;
  uint32_t stride = 1;
  const uint32_t* list = nullptr;
  uint64_t list_len = 0;
  uint64_t Count() const {
    if (list) return list_len;
    const uint64_t st = stride ? stride : 1;
    return end > begin ? (end - begin + st - 1) / st : 0;
  }
};
// The task of `o` on a graph of n vertices (validated: list ids below n).
RootTask TaskOf(const sme_opts& o, uint64_t n);

struct RunResult {
  uint64_t count = 0;
  uint64_t emitted = 0;
  sme_stats stats{};
};

// Runs `prog` over the roots of `task` on `g`.  When prog.enumerate,
// instances are written to out (device) up to cap.
RunResult RunProgram(const Program& prog, const DeviceGraph& g, DeviceContext& ctx, const RootTask& task,
                     uint32_t* d_out, uint64_t cap, int tuning);
// `tuning`: low byte = intersection launch (0 auto: warp per path,
// specialised; 1 warp per path generic; 2 flattened, specialised; 3 as 0 at
// six blocks per SM); bit 8 set = no hub bitmaps.
inline int Tuning(const sme_opts& o) { return (o.warp_granularity & 0xff) | (o.list_only ? 0x100 : 0); }
// The launch for a graph: the auto choice (granularity 0) takes the
// flattened kernel on an oriented graph, whose lists are short (the
// degree-oriented R-MAT s22 4-clique 2026 -> 1501 ms, 5-clique every 16th
// root 6772 -> 4391 ms), and the warp per path elsewhere (on R-MAT s20 as
// generated the flattened kernel is 40-60% slower on the 4-cycle, diamond and
// house).
inline int TuningFor(const sme_opts& o, const HostGraph& g) {
  int t = Tuning(o);
  if ((t & 0xff) == 0 && g.oriented) t |= 2;
  return t;
}

// External (chunked) execution over a graph that stays in host memory.
RunResult RunProgramExternal(const Program& prog, const HostGraph& g, DeviceContext& ctx, const RootTask& task,
                             int ext_variant, uint64_t graph_budget_bytes);

int DeviceCount();

}  // namespace sme
