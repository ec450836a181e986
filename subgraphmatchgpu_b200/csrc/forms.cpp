// Served form: a request loop over device-resident graphs with admission by
// estimated frontier memory and continuous batching across slots.
//
// Each slot owns a CUDA stream and a frontier arena, and a host worker that
// runs one request at a time through the level engine; requests of different
// patterns and graphs therefore run concurrently on the device.  A request is
// admitted when a slot is idle and the sum of the estimated frontier bytes of
// the requests in flight stays within the server budget.  Among the queued
// requests that fit, the one with the least estimated work goes first, so
// short requests are not stuck behind long ones; a request that has waited
// longer than kStarveMs goes first regardless (nothing starves).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"
#include "sme_internal.h"

namespace sme {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id;
  int32_t gid;
  sme_graph* attached;
  sme_opts opts;
  std::shared_ptr<std::vector<uint32_t>> roots;  // copy of an explicit root task
  uint64_t est_bytes;
  double est_work;
  Clock::time_point submitted;
};

constexpr double kStarveMs = 500.0;

// Work estimate used only to order admission: roots of the task times the
// average degree to the power of the pattern's later levels.
double EstimateWork(const HostGraph& g, const sme_opts& o) {
  const int k = Query(o.query_type).n;
  const double roots = (double)TaskOf(o, g.n).Count();
  const double davg = g.n ? (double)g.m / (double)g.n : 0.0;
  double w = roots;
  for (int i = 1; i < k; ++i) w *= std::max(1.0, davg);
  return w;
}

struct Result {
  sme_status status = SME_ERR_BUSY;
  uint64_t count = 0;
  double latency_ms = 0;
  std::string error;
};

// Frontier estimate of a request: the partial instances of the widest level
// are bounded by the edge count times the pattern's later levels; the engine
// batches to its slot arena, so the estimate only orders admission.
uint64_t EstimateBytes(const HostGraph& g, int query) {
  const int k = Query(query).n;
  uint64_t graph = (g.n + 1) * 8 + g.m * 4;
  uint64_t frontier = g.m * 4ULL * (uint64_t)std::max(1, k - 2) * 4ULL;
  return graph + frontier;
}

}  // namespace
}  // namespace sme

using namespace sme;

struct sme_server {
  sme_server_opts o{};
  std::vector<sme_graph*> resident;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request> queue;
  std::map<uint64_t, Result> results;
  std::vector<std::thread> workers;
  std::vector<DeviceContext*> ctxs;
  uint64_t next_id = 1;
  uint64_t inflight_bytes = 0;
  uint64_t inflight = 0, max_inflight = 0, completed = 0, rejected = 0;
  bool stop = false;
  uint64_t slot_arena = 0;

  // Index of the queued request to admit next, or -1 (caller holds mu).
  long Pick() const {
    if (queue.empty()) return -1;
    auto fits = [&](const Request& r) { return inflight == 0 || inflight_bytes + r.est_bytes <= o.mem_budget_bytes; };
    const double age =
        std::chrono::duration<double, std::milli>(Clock::now() - queue.front().submitted).count();
    if (age > kStarveMs) return fits(queue.front()) ? 0 : -1;
    long best = -1;
    const size_t scan = std::min<size_t>(queue.size(), 256);
    for (size_t i = 0; i < scan; ++i)
      if (fits(queue[i]) && (best < 0 || queue[i].est_work < queue[best].est_work)) best = (long)i;
    return best;
  }

  void Worker(int slot) {
    cudaSetDevice(o.device);
    DeviceContext* ctx = ctxs[slot];
    while (true) {
      Request r;
      {
        std::unique_lock<std::mutex> l(mu);
        long pick = -1;
        // wake at least every kStarveMs so ageing is noticed without new work
        while (!(stop && queue.empty())) {
          pick = Pick();
          if (pick >= 0) break;
          cv_work.wait_for(l, std::chrono::milliseconds((long)kStarveMs));
        }
        if (pick < 0) return;  // stopping and the queue is empty
        r = queue[pick];
        queue.erase(queue.begin() + pick);
        inflight_bytes += r.est_bytes;
        ++inflight;
        max_inflight = std::max(max_inflight, inflight);
      }
      Result res;
      try {
        const HostGraph& hg = r.attached ? r.attached->g : resident[r.gid]->g;
        Program prog = Compile(r.opts, false, hg.LoopFree());
        if (hg.oriented) RequireOrientable(prog, r.opts.enable_ordering != 0);
        DeviceGraph* dg = hg.dev;
        bool temp = false;
        // an attached graph is uploaded into the slot's arena and released
        // with it: no device allocation or free (a cudaFree would stall the
        // other slots' streams)
        const size_t graph_mark = ctx->arena.Mark();
        RunResult rr;
        try {
          if (!dg || dg->device != o.device) {
            dg = UploadGraphToArena(hg, *ctx, nullptr);
            temp = true;
          }
          rr = RunProgram(prog, *dg, *ctx, TaskOf(r.opts, hg.n), nullptr, 0, TuningFor(r.opts, hg));
        } catch (...) {
          if (temp) FreeDeviceGraph(dg);
          ctx->arena.Release(graph_mark);
          throw;
        }
        if (temp) FreeDeviceGraph(dg);
        ctx->arena.Release(graph_mark);
        res.status = SME_OK;
        res.count = rr.count;
      } catch (const Error& e) {
        res.status = e.status;
        res.error = e.what();
      } catch (const std::exception& e) {
        res.status = SME_ERR_INVALID_ARG;
        res.error = e.what();
      }
      res.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - r.submitted).count();
      {
        std::lock_guard<std::mutex> l(mu);
        results[r.id] = res;
        inflight_bytes -= r.est_bytes;
        --inflight;
        ++completed;
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

namespace {
template <typename F>
sme_status SGuard(F&& f) {
  try {
    f();
    return SME_OK;
  } catch (const Error& e) {
    SetLastError(e.what());
    return e.status;
  } catch (const std::exception& e) {
    SetLastError(e.what());
    return SME_ERR_INVALID_ARG;
  }
}
}  // namespace

extern "C" {

sme_status sme_server_opts_default(sme_server_opts* o) {
  if (!o) return SME_ERR_INVALID_ARG;
  *o = sme_server_opts{};
  o->device = 0;
  o->slots = 4;
  o->mem_budget_bytes = 0;  // 0: 60% of free device memory
  o->queue_capacity = 1 << 16;
  return SME_OK;
}

sme_status sme_server_create(const sme_server_opts* opts, sme_server** out) {
  if (!out) return SME_ERR_INVALID_ARG;
  return SGuard([&] {
    std::unique_ptr<sme_server> s(new sme_server());
    sme_server_opts_default(&s->o);
    if (opts) s->o = *opts;
    if (s->o.slots < 1 || s->o.slots > 64) Fail(SME_ERR_INVALID_ARG, "slots must be 1..64");
    if (DeviceCount() <= s->o.device) Fail(SME_ERR_NO_DEVICE, "no CUDA device " + std::to_string(s->o.device));
    cudaSetDevice(s->o.device);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    if (!s->o.mem_budget_bytes) s->o.mem_budget_bytes = (uint64_t)(fr * 0.6);
    s->slot_arena = std::max<uint64_t>(s->o.mem_budget_bytes / s->o.slots, 256ULL << 20);
    for (int i = 0; i < s->o.slots; ++i) s->ctxs.push_back(CreateContext(s->o.device, s->slot_arena));
    for (int i = 0; i < s->o.slots; ++i) s->workers.emplace_back(&sme_server::Worker, s.get(), i);
    *out = s.release();
  });
}

sme_status sme_server_add_graph(sme_server* s, sme_graph* g, int32_t* gid) {
  if (!s || !g || !gid) return SME_ERR_INVALID_ARG;
  return SGuard([&] {
    if (!g->g.dev || g->g.dev->device != s->o.device) {
      if (g->g.dev) FreeDeviceGraph(g->g.dev);
      g->g.dev = nullptr;
      cudaSetDevice(s->o.device);
      g->g.dev = UploadGraph(g->g, s->o.device, 0, nullptr);
    }
    std::lock_guard<std::mutex> l(s->mu);
    s->resident.push_back(g);
    *gid = (int32_t)s->resident.size() - 1;
  });
}

sme_status sme_server_submit(sme_server* s, int32_t gid, sme_graph* attached, const sme_opts* opts,
                             uint64_t* request_id) {
  if (!s || !opts || !request_id) return SME_ERR_INVALID_ARG;
  return SGuard([&] {
    if (opts->execute_mode != SME_IN_MEMORY_GPU) Fail(SME_ERR_INVALID_ARG, "served requests run IN_MEMORY_GPU");
    Request r;
    r.gid = gid;
    r.attached = attached;
    r.opts = *opts;
    r.opts.device = s->o.device;
    if (opts->num_roots > 0) {  // the caller's array may go away after submit
      if (!opts->roots) Fail(SME_ERR_INVALID_ARG, "num_roots > 0 with a null roots array");
      r.roots = std::make_shared<std::vector<uint32_t>>(opts->roots, opts->roots + opts->num_roots);
      r.opts.roots = r.roots->data();
    }
    r.submitted = Clock::now();
    {
      std::lock_guard<std::mutex> l(s->mu);
      if (!attached && (gid < 0 || gid >= (int32_t)s->resident.size()))
        Fail(SME_ERR_INVALID_ARG, "unknown graph id " + std::to_string(gid));
      if ((int64_t)s->queue.size() >= s->o.queue_capacity) {
        ++s->rejected;
        Fail(SME_ERR_BUSY, "server queue full");
      }
      const HostGraph& hg = attached ? attached->g : s->resident[gid]->g;
      Compile(r.opts, false);  // validate query / plan before queueing
      TaskOf(r.opts, hg.n);    // and an explicit root task
      r.est_bytes = EstimateBytes(hg, r.opts.query_type);
      r.est_work = EstimateWork(hg, r.opts);
      r.id = s->next_id++;
      s->results[r.id] = Result();
      s->queue.push_back(r);
      *request_id = r.id;
    }
    s->cv_work.notify_one();
  });
}

sme_status sme_server_poll(sme_server* s, uint64_t id, uint64_t* count, double* latency_ms) {
  if (!s) return SME_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> l(s->mu);
  auto it = s->results.find(id);
  if (it == s->results.end()) {
    SetLastError("unknown request id");
    return SME_ERR_INVALID_ARG;
  }
  if (it->second.status == SME_ERR_BUSY) return SME_ERR_BUSY;
  if (count) *count = it->second.count;
  if (latency_ms) *latency_ms = it->second.latency_ms;
  if (it->second.status != SME_OK) SetLastError(it->second.error);
  return it->second.status;
}

sme_status sme_server_wait(sme_server* s, uint64_t id, uint64_t* count, double* latency_ms) {
  if (!s) return SME_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> l(s->mu);
  auto it = s->results.find(id);
  if (it == s->results.end()) {
    SetLastError("unknown request id");
    return SME_ERR_INVALID_ARG;
  }
  s->cv_done.wait(l, [&] { return s->results[id].status != SME_ERR_BUSY; });
  const Result& r = s->results[id];
  if (count) *count = r.count;
  if (latency_ms) *latency_ms = r.latency_ms;
  if (r.status != SME_OK) SetLastError(r.error);
  return r.status;
}

sme_status sme_server_stats(sme_server* s, uint64_t* completed, uint64_t* max_inflight, uint64_t* rejected) {
  if (!s) return SME_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> l(s->mu);
  if (completed) *completed = s->completed;
  if (max_inflight) *max_inflight = s->max_inflight;
  if (rejected) *rejected = s->rejected;
  return SME_OK;
}

sme_status sme_server_destroy(sme_server* s) {
  if (!s) return SME_OK;
  {
    std::lock_guard<std::mutex> l(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto* c : s->ctxs) DestroyContext(c);
  delete s;
  return SME_OK;
}

}  // extern "C"
