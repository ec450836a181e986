// C-ABI of libsme (include/sme.h): handles, status codes, per-thread errors.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

#include "engine.h"
#include "sme_internal.h"

namespace sme {

static thread_local std::string t_last_error;
static thread_local sme_stats t_last_stats{};

void SetLastError(const std::string& msg) { t_last_error = msg; }

template <typename F>
static sme_status Guard(F&& f) {
  try {
    f();
    t_last_error.clear();
    return SME_OK;
  } catch (const Error& e) {
    t_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    t_last_error = "host allocation failed";
    return SME_ERR_OOM;
  } catch (const std::exception& e) {
    t_last_error = e.what();
    return SME_ERR_INVALID_ARG;
  }
}

// One execution context per device for the synchronous API; calls on the
// same device are serialised by its mutex.
struct CtxSlot {
  std::mutex mu;
  DeviceContext* ctx = nullptr;
  uint64_t bytes = 0;
};
static std::mutex g_ctx_mu;
static std::map<int, std::unique_ptr<CtxSlot>> g_ctx;

static CtxSlot& SlotFor(int device) {
  std::lock_guard<std::mutex> l(g_ctx_mu);
  auto& s = g_ctx[device];
  if (!s) s.reset(new CtxSlot());
  return *s;
}

static void CheckOpts(const sme_opts& o) {
  if (o.query_type < 0 || o.query_type >= SME_NUM_QUERIES)
    Fail(SME_ERR_UNSUPPORTED_QUERY, "query_type must be 0..13");
  if (o.execute_mode == SME_HYBRID_CPU_GPU)
    Fail(SME_ERR_INVALID_ARG, "execute_mode 0 (HYBRID_CPU_GPU) is not part of this engine; use 1 or 2");
  if (o.execute_mode != SME_IN_MEMORY_GPU && o.execute_mode != SME_EXTERNAL_GPU)
    Fail(SME_ERR_INVALID_ARG, "execute_mode must be 1 (IN_MEMORY_GPU) or 2 (EXTERNAL_GPU)");
  if (o.execute_mode == SME_EXTERNAL_GPU && o.algo != SME_GPU_LIGHT)
    Fail(SME_ERR_INVALID_ARG, "EXTERNAL_GPU runs the LIGHT plan only (algo 6)");
}

RootTask TaskOf(const sme_opts& o, uint64_t n) {
  RootTask t;
  if (o.num_roots > 0) {
    if (!o.roots) Fail(SME_ERR_INVALID_ARG, "num_roots > 0 with a null roots array");
    for (uint64_t i = 0; i < o.num_roots; ++i)
      if (o.roots[i] >= n)
        Fail(SME_ERR_INVALID_ARG, "roots[" + std::to_string(i) + "] = " + std::to_string(o.roots[i]) +
                                      " is not a vertex (n = " + std::to_string(n) + ")");
    t.list = o.roots;
    t.list_len = o.num_roots;
    return t;
  }
  t.begin = o.root_begin;
  t.end = o.root_end ? std::min<uint64_t>(o.root_end, n) : n;
  if (t.begin > t.end) t.begin = t.end;
  t.stride = o.root_stride ? o.root_stride : 1;
  return t;
}

struct RunOut {
  uint64_t count = 0;
  uint64_t emitted = 0;
};

// Shared by sme_count / sme_enumerate.
static RunOut Execute(sme_graph* g, const sme_opts& o, bool enumerate, uint32_t* host_out, uint64_t cap) {
  CheckOpts(o);
  auto t0 = std::chrono::steady_clock::now();
  Program prog = Compile(o, enumerate, g->g.LoopFree());
  if (g->g.oriented) RequireOrientable(prog, o.enable_ordering != 0);
  CtxSlot& slot = SlotFor(o.device);
  std::lock_guard<std::mutex> lock(slot.mu);
  // the arena follows each call's budget (0 = auto), so a call never runs in
  // the smaller arena a previous call asked for
  if (!slot.ctx || slot.bytes != o.mem_limit_bytes) {
    if (slot.ctx) DestroyContext(slot.ctx);
    slot.ctx = nullptr;
    slot.ctx = CreateContext(o.device, o.mem_limit_bytes);
    slot.bytes = o.mem_limit_bytes;
  }
  DeviceContext& ctx = *slot.ctx;
  const RootTask task = TaskOf(o, g->g.n);
  RunResult r;
  uint64_t h2d = 0, d2h = 8;
  if (o.execute_mode == SME_EXTERNAL_GPU) {
    if (enumerate) Fail(SME_ERR_INVALID_ARG, "enumeration runs in IN_MEMORY_GPU mode");
    r = RunProgramExternal(prog, g->g, ctx, task, o.ext_variant, 0);
    h2d = r.stats.h2d_bytes;
  } else {
    DeviceGraph* dg = g->g.dev;
    bool temp = false;
    const size_t graph_mark = ctx.arena.Mark();
    if (!dg || dg->device != o.device) {
      // not resident: the graph shares the call's arena (budget covers
      // frontiers + graph) and leaves with it
      try {
        dg = UploadGraphToArena(g->g, ctx, &h2d);
      } catch (...) {
        ctx.arena.Release(graph_mark);
        throw;
      }
      temp = true;
    }
    uint32_t* d_out = nullptr;
    try {
      if (enumerate && cap) {
        size_t bytes = (size_t)cap * prog.n * sizeof(uint32_t);
        if (cudaMalloc((void**)&d_out, bytes) != cudaSuccess) {
          cudaGetLastError();
          Fail(SME_ERR_OOM, "cannot allocate enumeration buffer");
        }
      }
      r = RunProgram(prog, *dg, ctx, task, d_out, cap, TuningFor(o, g->g));
      if (enumerate && cap && host_out) {
        uint64_t ncopy = std::min<uint64_t>(r.emitted, cap);
        if (ncopy) {
          if (cudaMemcpy(host_out, d_out, ncopy * prog.n * sizeof(uint32_t), cudaMemcpyDeviceToHost) !=
              cudaSuccess)
            Fail(SME_ERR_CUDA, "copy of enumerated instances failed");
          d2h += ncopy * prog.n * sizeof(uint32_t);
        }
      }
    } catch (...) {
      if (d_out) cudaFree(d_out);
      if (temp) FreeDeviceGraph(dg);
      ctx.arena.Release(graph_mark);
      throw;
    }
    if (d_out) cudaFree(d_out);
    if (temp) FreeDeviceGraph(dg);
    ctx.arena.Release(graph_mark);
  }
  if (o.execute_mode != SME_EXTERNAL_GPU) h2d += r.stats.h2d_bytes;  // the root list
  r.stats.h2d_bytes = h2d;
  r.stats.d2h_bytes = d2h;
  r.stats.elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  t_last_stats = r.stats;
  RunOut ro;
  ro.count = r.count;
  ro.emitted = r.emitted;
  return ro;
}

}  // namespace sme

using namespace sme;

extern "C" {

sme_status sme_opts_default(sme_opts* o) {
  if (!o) return SME_ERR_INVALID_ARG;
  std::memset(o, 0, sizeof(*o));
  o->query_type = 0;
  o->algo = SME_GPU_LIGHT;
  o->execute_mode = SME_IN_MEMORY_GPU;
  o->compress_level = SME_COMPRESS_SPECIAL;
  o->enable_ordering = 1;
  o->ext_variant = SME_EXT_CACHE;
  o->reuse_autogen = -1;
  o->device = 0;
  return SME_OK;
}

sme_status sme_graph_load_bin(const char* path, sme_graph** out) {
  if (!path || !out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> g(new sme_graph());
    ReadBinFile(path, g->g);
    *out = g.release();
  });
}

sme_status sme_graph_load_snap(const char* path, int directed, sme_graph** out) {
  if (!path || !out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> g(new sme_graph());
    ReadSnapFile(path, directed != 0, g->g);
    *out = g.release();
  });
}

sme_status sme_graph_load_snap_lvid(const char* path, int directed, sme_graph** out) {
  if (!path || !out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> g(new sme_graph());
    ReadSnapLvidFile(path, directed != 0, g->g);
    *out = g.release();
  });
}

sme_status sme_graph_load(const char* path, int directed, sme_graph** out) {
  if (!path || !out) return SME_ERR_INVALID_ARG;
  std::string p(path);
  std::string suf = p.substr(p.rfind('.') + 1);
  if (suf == "bin") return sme_graph_load_bin(path, out);
  if (suf == "txt") return sme_graph_load_snap(path, directed, out);
  if (suf == "lvid") return sme_graph_load_snap_lvid(path, directed, out);
  SetLastError("unknown graph file suffix ." + suf + " (expected .bin, .txt or .lvid)");
  return SME_ERR_BAD_FILE;
}

sme_status sme_graph_write_snap(const sme_graph* g, const char* path) {
  if (!g || !path) return SME_ERR_INVALID_ARG;
  return Guard([&] { WriteSnapFile(path, g->g); });
}

sme_status sme_graph_write_adj(const sme_graph* g, const char* path) {
  if (!g || !path) return SME_ERR_INVALID_ARG;
  return Guard([&] { WriteAdjFile(path, g->g); });
}

sme_status sme_graph_from_csr(const uint64_t* row_ptrs, const uint32_t* cols, uint64_t n, uint64_t m, int copy,
                              sme_graph** out) {
  if (!row_ptrs || (!cols && m) || !out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    if (row_ptrs[0] != 0 || row_ptrs[n] != m) Fail(SME_ERR_INVALID_ARG, "row_ptrs must span [0, m]");
    for (uint64_t u = 0; u < n; ++u)
      if (row_ptrs[u] > row_ptrs[u + 1]) Fail(SME_ERR_INVALID_ARG, "row_ptrs not monotone");
    for (uint64_t j = 0; j < m; ++j)
      if (cols[j] >= n) Fail(SME_ERR_INVALID_ARG, "column id out of range");
    std::unique_ptr<sme_graph> g(new sme_graph());
    if (copy) {
      g->g.Adopt(std::vector<uintE>(row_ptrs, row_ptrs + n + 1), std::vector<uintV>(cols, cols + m));
    } else {
      g->g.n = n;
      g->g.m = m;
      g->g.row_ptrs = const_cast<uintE*>(row_ptrs);
      g->g.cols = const_cast<uintV*>(cols);
      g->g.borrowed = true;
    }
    *out = g.release();
  });
}

sme_status sme_graph_info(const sme_graph* g, uint64_t* n, uint64_t* m, uint64_t* max_degree) {
  if (!g) return SME_ERR_INVALID_ARG;
  if (n) *n = g->g.n;
  if (m) *m = g->g.m;
  if (max_degree) *max_degree = g->g.MaxDegree();
  return SME_OK;
}

sme_status sme_graph_csr(const sme_graph* g, const uint64_t** row_ptrs, const uint32_t** cols) {
  if (!g) return SME_ERR_INVALID_ARG;
  if (row_ptrs) *row_ptrs = g->g.row_ptrs;
  if (cols) *cols = g->g.cols;
  return SME_OK;
}

sme_status sme_graph_write_bin(const sme_graph* g, const char* path) {
  if (!g || !path) return SME_ERR_INVALID_ARG;
  return Guard([&] { WriteBinFile(path, g->g); });
}

sme_status sme_graph_preprocess(sme_graph* g) {
  if (!g) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    if (g->g.oriented) Fail(SME_ERR_INVALID_ARG, "an oriented graph cannot be preprocessed");
    if (g->g.dev) {
      FreeDeviceGraph(g->g.dev);
      g->g.dev = nullptr;
    }
    Preprocess(g->g);
  });
}

sme_status sme_graph_degree_order(const sme_graph* g, int32_t orient, sme_graph** out, uint32_t* new_to_old) {
  if (!g || !out || (orient != 0 && orient != 1)) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    if (g->g.oriented) Fail(SME_ERR_INVALID_ARG, "the graph is oriented already");
    std::unique_ptr<sme_graph> r(new sme_graph());
    std::vector<uintV> map;
    DegreeOrder(g->g, orient != 0, r->g, new_to_old ? &map : nullptr);
    if (new_to_old) std::copy(map.begin(), map.end(), new_to_old);
    *out = r.release();
  });
}

int32_t sme_graph_is_oriented(const sme_graph* g) { return g && g->g.oriented ? 1 : 0; }

sme_status sme_graph_validate(const sme_graph* g) {
  if (!g) return SME_ERR_INVALID_ARG;
  return Guard([&] { Validate(g->g); });
}

sme_status sme_graph_to_device(sme_graph* g, int device) {
  if (!g) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    if (g->g.dev && g->g.dev->device == device) return;
    if (g->g.dev) {
      FreeDeviceGraph(g->g.dev);
      g->g.dev = nullptr;
    }
    if (DeviceCount() <= device) Fail(SME_ERR_NO_DEVICE, "no CUDA device " + std::to_string(device));
    cudaSetDevice(device);
    g->g.dev = UploadGraph(g->g, device, 0, nullptr);
  });
}

sme_status sme_graph_device_arrays(const sme_graph* g, int device, const uint64_t** row_ptrs,
                                   const uint32_t** cols) {
  if (!g) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    const DeviceGraph* d = g->g.dev;
    if (!d || d->device != device) Fail(SME_ERR_INVALID_ARG, "the graph is not resident on that device");
    if (row_ptrs) *row_ptrs = d->row_ptrs;
    if (cols) *cols = d->cols;
  });
}

sme_status sme_graph_pack(sme_graph* g, int enable, uint64_t* packed_bytes) {
  if (!g) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    if (enable)
      g->g.packed = PackLists(g->g);
    else
      g->g.packed.reset();
    if (packed_bytes) *packed_bytes = g->g.packed ? g->g.packed->total : 0;
  });
}

sme_status sme_graph_release_device(sme_graph* g) {
  if (!g) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    FreeDeviceGraph(g->g.dev);
    g->g.dev = nullptr;
  });
}

sme_status sme_graph_free(sme_graph* g) {
  if (!g) return SME_OK;
  return Guard([&] {
    FreeDeviceGraph(g->g.dev);
    g->g.dev = nullptr;
    delete g;
  });
}

sme_status sme_generate_rmat(int32_t scale, int32_t ef, double a, double b, double c, uint64_t seed,
                             sme_graph** out) {
  if (!out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> g(new sme_graph());
    GenerateRmat(scale, ef, a, b, c, seed, g->g);
    *out = g.release();
  });
}

sme_status sme_generate_er(uint64_t n, double d, uint64_t seed, sme_graph** out) {
  if (!out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> g(new sme_graph());
    GenerateER(n, d, seed, g->g);
    *out = g.release();
  });
}

sme_status sme_generate_ba(uint64_t n, uint32_t m, uint64_t seed, sme_graph** out) {
  if (!out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> g(new sme_graph());
    GenerateBA(n, m, seed, g->g);
    *out = g.release();
  });
}

sme_status sme_generate_clique(uint64_t n, sme_graph** out) {
  if (!out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> g(new sme_graph());
    GenerateClique(n, g->g);
    *out = g.release();
  });
}

sme_status sme_count(sme_graph* g, const sme_opts* opts, uint64_t* count) {
  if (!g || !opts || !count) return SME_ERR_INVALID_ARG;
  return Guard([&] { *count = Execute(g, *opts, false, nullptr, 0).count; });
}

sme_status sme_read_partition_file(const char* path, uint64_t n, uint32_t partition_num, uint32_t* vertex_partition) {
  if (!vertex_partition && n) return SME_ERR_INVALID_ARG;
  return Guard([&] { ReadPartitionFile(path ? path : "", n, partition_num, vertex_partition); });
}

sme_status sme_graph_partition(const sme_graph* g, const uint32_t* vertex_partition, uint32_t p, sme_graph** out) {
  if (!g || !vertex_partition || !out) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    std::unique_ptr<sme_graph> r(new sme_graph());
    InducedPartition(g->g, vertex_partition, p, r->g, nullptr);
    *out = r.release();
  });
}

// HYBRID_CPU_GPU (-m 0): the whole graph fits in one B200's memory, so the
// total is counted on it in one in-memory run, and each partition's
// intra-partition share on its induced subgraph; the inter-partition share
// is the difference.  Plans as InitGPUInstance allows for this mode
// (src/gpu/PatternMatchGPUInstance.cuh:43-63): reuse BFS or LIGHT.
sme_status sme_count_partitioned(sme_graph* g, const sme_opts* opts, const uint32_t* vertex_partition,
                                 uint32_t partition_num, uint64_t* total, uint64_t* intra) {
  if (!g || !opts || !vertex_partition || !total || partition_num == 0) return SME_ERR_INVALID_ARG;
  return Guard([&] {
    if (opts->algo != SME_GPU_GPSM_REUSE && opts->algo != SME_GPU_LIGHT)
      Fail(SME_ERR_INVALID_ARG, "HYBRID_CPU_GPU runs the reuse BFS (5) or LIGHT (6) plan");
    if (opts->execute_mode != SME_HYBRID_CPU_GPU && opts->execute_mode != SME_IN_MEMORY_GPU)
      Fail(SME_ERR_INVALID_ARG, "partitioned counting takes execute_mode 0 (HYBRID_CPU_GPU) or 1");
    for (uint64_t u = 0; u < g->g.n; ++u)
      if (vertex_partition[u] >= partition_num)
        Fail(SME_ERR_INVALID_ARG, "vertex " + std::to_string(u) + " has partition id " +
                                      std::to_string(vertex_partition[u]) + " >= partition_num");
    sme_opts o = *opts;
    o.execute_mode = SME_IN_MEMORY_GPU;
    o.root_begin = o.root_end = 0;
    o.root_stride = 1;
    double elapsed = 0;
    uint64_t launches = 0, h2d = 0;
    *total = Execute(g, o, false, nullptr, 0).count;
    elapsed += t_last_stats.elapsed_ms;
    launches += t_last_stats.kernel_launches;
    h2d += t_last_stats.h2d_bytes;
    uint64_t intra_sum = 0;
    for (uint32_t p = 0; p < partition_num; ++p) {
      sme_graph part;
      InducedPartition(g->g, vertex_partition, p, part.g, nullptr);
      const uint64_t c = part.g.n ? Execute(&part, o, false, nullptr, 0).count : 0;
      if (part.g.n) {
        elapsed += t_last_stats.elapsed_ms;
        launches += t_last_stats.kernel_launches;
        h2d += t_last_stats.h2d_bytes;
      }
      if (intra) intra[p] = c;
      intra_sum += c;
    }
    if (intra_sum > *total) Fail(SME_ERR_CUDA, "intra-partition counts exceed the total");
    t_last_stats.elapsed_ms = elapsed;
    t_last_stats.kernel_launches = launches;
    t_last_stats.h2d_bytes = h2d;
  });
}

sme_status sme_enumerate(sme_graph* g, const sme_opts* opts, uint32_t* out, uint64_t cap, uint64_t* n_out) {
  if (!g || !opts || !n_out || (cap && !out)) return SME_ERR_INVALID_ARG;
  sme_status st = Guard([&] {
    RunOut r = Execute(g, *opts, true, out, cap);
    *n_out = r.emitted;
  });
  if (st == SME_OK && *n_out > cap) {
    SetLastError("enumeration produced " + std::to_string(*n_out) + " instances, buffer holds " +
                 std::to_string(cap));
    return SME_ERR_CAPACITY;
  }
  return st;
}

sme_status sme_last_stats(sme_stats* s) {
  if (!s) return SME_ERR_INVALID_ARG;
  *s = t_last_stats;
  return SME_OK;
}

int32_t sme_query_vertex_count(int32_t q) {
  if (q < 0 || q >= SME_NUM_QUERIES) return -1;
  return Query(q).n;
}

sme_status sme_plan_describe(int32_t q, int32_t plan_type, char* buf, uint64_t cap, uint64_t* needed) {
  std::string text;
  sme_status st = Guard([&] {
    Query query(q);
    switch (plan_type) {
      case 0: text = TraversalPlan(query).Describe(); break;
      case 1: text = ReusePlan(query, true).Describe(); break;
      case 2: text = LazyPlan(query, SME_COMPRESS_NON_MATERIALIZE_OPT).Describe(); break;
      case 3: text = ReusePlan(query, false).Describe(); break;
      case 4: text = LazyPlan(query, SME_COMPRESS_SPECIAL).Describe(); break;
      case 5:
      case 6: {
        sme_opts o;
        sme_opts_default(&o);
        o.query_type = q;
        for (int a : {SME_GPU_GPSM, SME_GPU_GPSM_REUSE, SME_GPU_LIGHT}) {
          o.algo = a;
          text += Compile(o, false, plan_type == 6).Describe();
        }
        break;
      }
      default: Fail(SME_ERR_INVALID_ARG, "plan_type must be 0..6");
    }
  });
  if (st != SME_OK) return st;
  if (needed) *needed = text.size() + 1;
  if (!buf || cap < text.size() + 1) return SME_ERR_CAPACITY;
  std::memcpy(buf, text.c_str(), text.size() + 1);
  return SME_OK;
}

const char* sme_last_error(void) { return t_last_error.c_str(); }
const char* sme_version(void) { return "sme-b200 0.1 (sm_100a)"; }

}  // extern "C"
