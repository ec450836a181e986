// Batched form: thousands of small (graph, query) pairs in one persistent
// launch, captured in a CUDA graph.
//
// Every graph is packed into one CSR (local vertex ids); the work items are
// (graph, root vertex) pairs ordered heaviest first.  A persistent grid of
// thread groups (4..32 lanes) pulls items from an atomic counter and runs a
// depth-first enumeration of the item's root: each level's candidate set is
// computed cooperatively by the group (pivot list clipped by the order
// constraints, binary search in the other lists, ballot compaction), kept as a
// view of an adjacency list when it is one, else in the group's scratch
// buffer; the last level is only counted.  Counts accumulate per graph.
//
// An autotuner times every (group size, block size) candidate on the batch
// itself and keeps the fastest; the winner is captured in a CUDA graph that
// sme_batch_run replays.  Per-level semantics follow the plain traversal plan
// (ordered backward connectivity + whole-ordered conditions,
// src/gpu/plan/DevTraversalPlan.cuh:9-16); cliques reuse the previous level's
// set (their chain order implies every earlier condition) and the diamond
// uses the closed form of LIGHTDirectCount (c(c-1)/2 per edge,
// src/gpu/impl/light/op/LIGHTDirectCount.cuh:31-37).
#include <algorithm>
#include <chrono>
#include <memory>
#include <mutex>
#include <vector>

#include "engine.h"
#include "kernels.cuh"

namespace sme {
using namespace dev;

#define BCK(x)                                                                                 \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess) Fail(SME_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

constexpr int BMAXV = 6;

struct BLevel {
  uint8_t nconn;
  uint8_t conn[BMAXV];
  int8_t reuse;  // earlier level whose set joins the intersection
  uint8_t ncond;
  uint8_t op[BMAXV];
  uint8_t operand[BMAXV];
};
struct BProg {
  uint8_t n;         // pattern vertices; levels 1..n-1
  uint8_t pair;      // last level adds c*(c-1)/2 instead of c
  uint8_t buffered[BMAXV];  // level needs a scratch buffer (multi-list)
  uint8_t buf_slot[BMAXV];
  BLevel lv[BMAXV];
};

__constant__ BProg c_prog[SME_NUM_QUERIES];

struct BArgs {
  const uint32_t* rp;    // packed row pointers (uint32 offsets into cols)
  const uint32_t* cols;  // packed local ids
  const uint32_t* goff;  // graph -> first row pointer index
  const uint8_t* query;  // graph -> query id
  const uint64_t* items; // (graph << 32) | root
  uint64_t nitems;
  unsigned long long* counts;
  unsigned int* next;
  uint32_t* scratch;     // per group: nbuf * cap uint32
  uint32_t cap;          // max degree in the batch
  uint32_t nbuf;
  uint32_t chunk;        // work items a group takes per fetch
};

// A thread group of G lanes that runs one work item: a part of a warp
// (G = 4..32, warp intrinsics) or several warps of a CTA (G = 64, 128: the
// CTA granularity; named barrier 1 + group index, ballot counts exchanged in
// shared memory).  All lanes of a group follow the same control flow.
constexpr int kMaxGroupWarps = 4;  // G <= 128
template <int G>
struct Tile {
  int lane;            // lane within the group
  unsigned mask;       // lanes of this group within the warp (G <= 32)
  int base;            // first lane of the group in the warp (G <= 32)
  uint32_t* xs;        // G > 32: this group's exchange words in shared memory
  int bar;             // G > 32: named barrier of the group
  __device__ explicit Tile(uint32_t* shared = nullptr) {
    if constexpr (G <= 32) {
      int l = threadIdx.x & 31;
      lane = l % G;
      base = l - lane;
      mask = (G == 32) ? FULL : (((1u << G) - 1) << base);
      xs = nullptr;
      bar = 0;
    } else {
      lane = threadIdx.x % G;
      base = 0;
      mask = FULL;
      const int grp = threadIdx.x / G;
      xs = shared + grp * (kMaxGroupWarps + 1);
      bar = 1 + grp;
    }
  }
  __device__ void sync() const {
    if constexpr (G > 32) asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(G) : "memory");
  }
  // Writes of the group's lanes become visible to the whole group.
  __device__ void publish() const {
    if constexpr (G <= 32) __syncwarp(mask);
    else sync();
  }
  __device__ uint32_t bcast(uint32_t v) const {
    if constexpr (G <= 32) {
      return __shfl_sync(mask, v, base);
    } else {
      if (lane == 0) xs[kMaxGroupWarps] = v;
      sync();
      const uint32_t r = xs[kMaxGroupWarps];
      sync();
      return r;
    }
  }
  // Number of lanes before this one whose `ok` holds; *total = all of them.
  __device__ uint32_t rank(bool ok, uint32_t* total) const {
    if constexpr (G <= 32) {
      const unsigned m = (__ballot_sync(mask, ok) & mask) >> base;
      *total = __popc(m);
      return __popc(m & ((1u << lane) - 1));
    } else {
      const unsigned m = __ballot_sync(FULL, ok);
      const int w = lane >> 5, l = lane & 31;
      if (l == 0) xs[w] = __popc(m);
      sync();
      uint32_t before = 0, tot = 0;
#pragma unroll
      for (int k = 0; k < G / 32; ++k) {
        const uint32_t c = xs[k];
        before += k < w ? c : 0;
        tot += c;
      }
      sync();  // the words are rewritten by the next call
      *total = tot;
      return before + __popc(m & ((1u << l) - 1));
    }
  }
};

// Candidate set of level `l` for the current partial instance M: written to
// `out` (when non-null) or counted.  Returns the group-uniform size; when the
// set is a single clipped list without exclusions, *view points into it.
template <int G, typename RP>
__device__ uint32_t LevelSet(const Tile<G>& t, const BLevel& L, const uint32_t* M, const RP* rp,
                             const uint32_t* cols, const uint32_t* const* sptr, const uint32_t* slen,
                             uint32_t* out, const uint32_t** view, bool pair_count,
                             unsigned long long* cnt) {
  const uint32_t* A[BMAXV];
  uint32_t N[BMAXV];
  int nl = 0;
#pragma unroll
  for (int i = 0; i < BMAXV; ++i) {
    if (i < L.nconn) {
      uint32_t v = M[L.conn[i]];
      A[i] = cols + rp[v];
      N[i] = (uint32_t)(rp[v + 1] - rp[v]);
      nl = i + 1;
    }
  }
  if (L.reuse >= 0) {
#pragma unroll
    for (int i = 0; i < BMAXV; ++i)
      if (i == nl) {
        A[i] = sptr[L.reuse];
        N[i] = slen[L.reuse];
      }
    ++nl;
  }
#pragma unroll
  for (int i = 1; i < BMAXV; ++i) {
    if (i < nl && N[i] < N[0]) {
      const uint32_t* tp = A[0];
      A[0] = A[i];
      A[i] = tp;
      uint32_t tn = N[0];
      N[0] = N[i];
      N[i] = tn;
    }
  }
  uint64_t lo = 0, hi = 1ULL << 32;
  uint32_t ne[BMAXV];
  int nne = 0;
#pragma unroll
  for (int i = 0; i < BMAXV; ++i) {
    if (i < L.ncond) {
      uint32_t v = M[L.operand[i]];
      if (L.op[i] == 0) hi = min(hi, (uint64_t)v);
      else if (L.op[i] == 1) lo = max(lo, (uint64_t)v + 1);
      else ne[nne++] = v;
    }
  }
  if (lo >= hi || nl == 0) return 0;
  uint32_t r0 = lo == 0 ? 0 : (lo > 0xffffffffULL ? N[0] : LowerBound(A[0], N[0], (uint32_t)lo));
  uint32_t r1 = hi > 0xffffffffULL ? N[0] : LowerBound(A[0], N[0], (uint32_t)hi);
  if (r1 < r0) r1 = r0;
  if (nl == 1 && view) {
    bool hit = false;
    for (int k = 0; k < nne; ++k) {
      uint32_t pos = r0 + LowerBound(A[0] + r0, r1 - r0, ne[k]);
      if (pos < r1 && A[0][pos] == ne[k]) hit = true;
    }
    if (!hit) {
      *view = A[0] + r0;
      if (cnt) {
        unsigned long long c = r1 - r0;
        *cnt += pair_count ? (c > 0 ? c * (c - 1) / 2 : 0) : c;
      }
      return r1 - r0;
    }
  }
  uint32_t cur[BMAXV];
#pragma unroll
  for (int i = 0; i < BMAXV; ++i) cur[i] = 0;
  uint32_t written = 0;
  for (uint32_t b = r0; b < r1; b += G) {
    uint32_t i = b + t.lane;
    bool ok = i < r1;
    uint32_t x = ok ? __ldg(A[0] + i) : 0;
    for (int k = 0; k < nne; ++k)
      if (x == ne[k]) ok = false;
#pragma unroll
    for (int j = 1; j < BMAXV; ++j) {
      if (j < nl && ok) {
        uint32_t pos = cur[j] + LowerBound(A[j] + cur[j], N[j] - cur[j], x);
        cur[j] = pos;
        ok = pos < N[j] && __ldg(A[j] + pos) == x;
      }
    }
    uint32_t total;
    const uint32_t r = t.rank(ok, &total);
    if (out && ok) out[written + r] = x;
    written += total;
  }
  if (cnt) {
    unsigned long long c = written;
    *cnt += pair_count ? (c > 0 ? c * (c - 1) / 2 : 0) : c;
  }
  if (out) t.publish();  // the set is read by every lane of the group next
  if (view) *view = out;
  return written;
}

// Groups take `a.chunk` consecutive items per fetch (heaviest first): fewer
// atomics on the shared counter against a coarser balance at the tail.
// Registers are held to 64 (two 512-thread blocks per SM): the level state
// spills to L1, but twice the resident warps hide more probe latency
// (4 096-graph batch: 1.17e9 unbounded at ~114 registers, 1.43e9 at 64,
// 1.20e9 at 40, 1.00e9 at 32 instances/s).
template <int G>
__global__ void __launch_bounds__(512, 2) k_batch(BArgs a) {
  __shared__ uint32_t xs_sh[16 * (kMaxGroupWarps + 1)];
  Tile<G> t(xs_sh);
  const uint32_t groups_per_block = blockDim.x / G;
  const uint32_t gid = blockIdx.x * groups_per_block + threadIdx.x / G;
  uint32_t* scratch = a.scratch + (size_t)gid * a.nbuf * a.cap;
  uint32_t it = 0, it_end = 0;
  while (true) {
    if (it == it_end) {
      uint32_t first = 0;
      if (t.lane == 0) first = atomicAdd(a.next, a.chunk);
      it = t.bcast(first);
      if (it >= a.nitems) break;
      it_end = (uint32_t)min((uint64_t)it + a.chunk, a.nitems);
    }
    const uint64_t item = a.items[it++];
    const uint32_t g = (uint32_t)(item >> 32);
    const uint32_t root = (uint32_t)item;
    const BProg& P = c_prog[a.query[g]];
    const uint32_t* rp = a.rp + a.goff[g];
    uint32_t M[BMAXV];
    const uint32_t* sptr[BMAXV];
    uint32_t slen[BMAXV], idx[BMAXV];
    M[0] = root;
    unsigned long long local = 0;
    const int last = P.n - 1;
    // level 1
    int level = 1;
    if (level == last) {
      LevelSet<G>(t, P.lv[1], M, rp, a.cols, sptr, slen, nullptr, nullptr, P.pair, &local);
    } else {
      uint32_t* out = P.buffered[1] ? scratch + P.buf_slot[1] * a.cap : nullptr;
      slen[1] = LevelSet<G>(t, P.lv[1], M, rp, a.cols, sptr, slen, out, &sptr[1], false, nullptr);
      idx[1] = 0;
      while (level >= 1) {
        if (idx[level] < slen[level]) {
          M[level] = sptr[level][idx[level]];
          ++idx[level];
          const int nx = level + 1;
          if (nx == last) {
            LevelSet<G>(t, P.lv[nx], M, rp, a.cols, sptr, slen, nullptr, nullptr, P.pair, &local);
          } else {
            uint32_t* out = P.buffered[nx] ? scratch + P.buf_slot[nx] * a.cap : nullptr;
            slen[nx] = LevelSet<G>(t, P.lv[nx], M, rp, a.cols, sptr, slen, out, &sptr[nx], false, nullptr);
            idx[nx] = 0;
            level = nx;
          }
        } else {
          --level;
        }
      }
    }
    // set sizes are group-uniform (ballot popcounts), so every lane holds the
    // same count; the leader adds it
    if (t.lane == 0 && local) atomicAdd(a.counts + g, local);
  }
}

BProg CompileBatchProgram(int q) {
  BProg p{};
  Query query(q);
  TraversalPlan tp(query);
  p.n = (uint8_t)query.n;
  if (q == 2) {
    // diamond: edges (u0 < u2), c = |N(u0) ∩ N(u2)|, count c(c-1)/2
    p.n = 3;
    p.pair = 1;
    p.lv[1].nconn = 1;
    p.lv[1].conn[0] = 0;
    p.lv[1].reuse = -1;
    p.lv[1].ncond = 1;
    p.lv[1].op[0] = LARGER_THAN;
    p.lv[1].operand[0] = 0;
    p.lv[2].nconn = 2;
    p.lv[2].conn[0] = 0;
    p.lv[2].conn[1] = 1;
    p.lv[2].reuse = -1;
    p.lv[2].ncond = 0;
  } else {
    const bool clique = q == 3 || q == 7 || q == 11 || q == 0;
    for (int u = 1; u < query.n; ++u) {
      BLevel& L = p.lv[u];
      L.reuse = -1;
      if (clique && u >= 2) {
        // chain order u0 < u1 < ... : previous level's set ∩ N(M[u-1]) ∩ (> M[u-1])
        L.nconn = 1;
        L.conn[0] = (uint8_t)(u - 1);
        L.reuse = (int8_t)(u - 1);
        L.ncond = 1;
        L.op[0] = LARGER_THAN;
        L.operand[0] = (uint8_t)(u - 1);
      } else {
        L.nconn = (uint8_t)tp.ordered_conn[u].size();
        for (size_t i = 0; i < tp.ordered_conn[u].size(); ++i) L.conn[i] = (uint8_t)tp.ordered_conn[u][i];
        L.ncond = (uint8_t)tp.whole_order[u].size();
        for (size_t i = 0; i < tp.whole_order[u].size(); ++i) {
          L.op[i] = (uint8_t)tp.whole_order[u][i].first;
          L.operand[i] = (uint8_t)tp.whole_order[u][i].second;
        }
      }
    }
  }
  int slot = 0;
  for (int u = 1; u + 1 < p.n; ++u) {
    // a set needs storage unless it is always a clipped single list (a view):
    // several lists, or an excluded value that may fall inside the range
    int lists = p.lv[u].nconn + (p.lv[u].reuse >= 0 ? 1 : 0);
    bool ne = false;
    for (int i = 0; i < p.lv[u].ncond; ++i) ne = ne || p.lv[u].op[i] == NON_EQUAL;
    if (lists > 1 || ne) {
      p.buffered[u] = 1;
      p.buf_slot[u] = (uint8_t)slot++;
    }
  }
  return p;
}

// Uploads the 14 level programs to the current device once per device; host
// threads preparing batches or allocation-free counts on the same device at
// the same time serialise here.
void UploadPrograms(int device) {
  static std::mutex mu;
  static bool done[64] = {false};
  std::lock_guard<std::mutex> l(mu);
  if (device >= 0 && device < 64 && done[device]) return;
  BProg all[SME_NUM_QUERIES];
  for (int q = 0; q < SME_NUM_QUERIES; ++q) all[q] = CompileBatchProgram(q);
  BCK(cudaMemcpyToSymbol(c_prog, all, sizeof(all)));
  if (device >= 0 && device < 64) done[device] = true;
}

int MaxBuffers(const std::vector<int32_t>& queries) {
  int nb = 0;
  for (int q : queries) {
    BProg p = CompileBatchProgram(q);
    int c = 0;
    for (int u = 0; u < BMAXV; ++u) c += p.buffered[u];
    nb = std::max(nb, c);
  }
  return std::max(nb, 1);
}

// ---- allocation-free single-graph count (sme_count_noalloc) ---------------
// Library-owned device memory, reserved when the library is loaded and kept
// by every GPU that loads it until the process exits: 16 MiB.  Words [0,64)
// hold one call's control values (word 0: next work item, words 2-3: the
// uint64 count, word 4: the graph's maximum degree, word 5: set when a list
// is unsorted, holds a duplicate, a self loop or an id >= n); the rest holds
// the thread groups' level buffers.  Every call reuses (and first clears) it.
constexpr size_t kNoAllocWords = size_t(4) << 20;
constexpr size_t kNoAllocHeader = 64;
constexpr uint32_t kNoAllocMaxDegree = 32768;
constexpr int kNoAllocGroup = 8;
constexpr int kNoAllocBlock = 128;
// At the maximum degree, the level buffers of the deepest program (at most
// BMAXV - 2 buffered levels) must still fit one block of thread groups.
static_assert((kNoAllocWords - kNoAllocHeader) / ((size_t)(BMAXV - 2) * kNoAllocMaxDegree) >=
                  (size_t)(kNoAllocBlock / kNoAllocGroup),
              "allocation-free scratch must hold at least one block of level buffers");
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

// One pass over the caller's CSR: the maximum degree (word 4 of `hdr`) and
// the input contract of the sorted-list searches (word 5: 1 when a list is
// not strictly increasing, holds its own vertex or an id >= n).
__global__ void k_noalloc_inspect(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ cols, uint32_t n,
                                  unsigned int* hdr) {
  unsigned int m = 0;
  bool bad = false;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint64_t b = rp[v], e = rp[v + 1];
    const uint64_t d = e - b;  // wraps to a huge degree when e < b
    m = max(m, (unsigned int)min(d, (uint64_t)0xffffffffu));
    if (e < b || d > kNoAllocMaxDegree) continue;  // refused on the degree alone
    uint32_t prev = 0;
    for (uint64_t i = b; i < e; ++i) {
      const uint32_t x = __ldg(cols + i);
      bad = bad || x >= n || x == v || (i > b && x <= prev);
      prev = x;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    // every lane takes part in both shuffles (no short-circuit around one)
    const unsigned int om = __shfl_down_sync(FULL, m, o);
    const int ob = __shfl_down_sync(FULL, (int)bad, o);
    m = max(m, om);
    bad = bad || ob != 0;
  }
  if ((threadIdx.x & 31) == 0) {
    if (m) atomicMax(hdr + 4, m);
    if (bad) atomicOr(hdr + 5, 1u);
  }
}

// The batched form's depth-first enumeration for one graph with 64-bit row
// pointers: work item i is root vertex i; level buffers in `base`.
template <int G>
__global__ void k_noalloc_dfs(const uint64_t* __restrict__ rp, const uint32_t* __restrict__ cols, uint32_t n,
                              int32_t query, uint32_t cap, uint32_t nbuf, uint32_t* base) {
  Tile<G> t;
  const uint32_t gid = blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
  uint32_t* scratch = base + kNoAllocHeader + (size_t)gid * nbuf * cap;
  unsigned int* next = base;
  unsigned long long* total = reinterpret_cast<unsigned long long*>(base + 2);
  const BProg& P = c_prog[query];
  const int last = P.n - 1;
  while (true) {
    uint32_t it = 0;
    if (t.lane == 0) it = atomicAdd(next, 1u);
    it = t.bcast(it);
    if (it >= n) break;
    uint32_t M[BMAXV];
    const uint32_t* sptr[BMAXV];
    uint32_t slen[BMAXV], idx[BMAXV];
    M[0] = it;
    unsigned long long local = 0;
    int level = 1;
    if (level == last) {
      LevelSet<G>(t, P.lv[1], M, rp, cols, sptr, slen, nullptr, nullptr, P.pair, &local);
    } else {
      uint32_t* out = P.buffered[1] ? scratch + P.buf_slot[1] * cap : nullptr;
      slen[1] = LevelSet<G>(t, P.lv[1], M, rp, cols, sptr, slen, out, &sptr[1], false, nullptr);
      idx[1] = 0;
      while (level >= 1) {
        if (idx[level] < slen[level]) {
          M[level] = sptr[level][idx[level]];
          ++idx[level];
          const int nx = level + 1;
          if (nx == last) {
            LevelSet<G>(t, P.lv[nx], M, rp, cols, sptr, slen, nullptr, nullptr, P.pair, &local);
          } else {
            uint32_t* o2 = P.buffered[nx] ? scratch + P.buf_slot[nx] * cap : nullptr;
            slen[nx] = LevelSet<G>(t, P.lv[nx], M, rp, cols, sptr, slen, o2, &sptr[nx], false, nullptr);
            idx[nx] = 0;
            level = nx;
          }
        } else {
          --level;
        }
      }
    }
    if (t.lane == 0 && local) atomicAdd(total, local);
  }
}

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the symbol's host-side name is not a device address).
uint32_t* NoAllocScratch(int device) {
  static std::mutex mu;
  static uint32_t* base[64] = {nullptr};
  if (device < 0 || device >= 64) Fail(SME_ERR_NO_DEVICE, "device ordinal out of range");
  std::lock_guard<std::mutex> l(mu);
  if (!base[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      Fail(SME_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
    base[device] = static_cast<uint32_t*>(p);
  }
  return base[device];
}

uint64_t CountNoAlloc(const uint64_t* d_rp, const uint32_t* d_cols, uint64_t n, int32_t q) {
  if (q < 0 || q >= SME_NUM_QUERIES) Fail(SME_ERR_UNSUPPORTED_QUERY, "query_type must be 0..13");
  if (n >= (1ULL << 31)) Fail(SME_ERR_INVALID_ARG, "sme_count_noalloc: n must be below 2^31");
  if (n > 0 && (!d_rp || !d_cols)) Fail(SME_ERR_INVALID_ARG, "sme_count_noalloc: null device CSR");
  int device = 0;
  BCK(cudaGetDevice(&device));
  uint32_t* base = NoAllocScratch(device);
  UploadPrograms(device);
  BCK(cudaMemsetAsync(base, 0, kNoAllocHeader * sizeof(uint32_t), 0));
  if (n == 0) {
    BCK(cudaStreamSynchronize(0));
    return 0;
  }
  const uint32_t nv = (uint32_t)n;
  int sms = 148;
  BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  k_noalloc_inspect<<<sms * 4, 256, 0, 0>>>(d_rp, d_cols, nv, base);
  uint32_t hdr[8] = {0};
  BCK(cudaMemcpy(hdr, base, sizeof(hdr), cudaMemcpyDeviceToHost));
  const uint32_t maxdeg = hdr[4];
  if (maxdeg > kNoAllocMaxDegree)
    Fail(SME_ERR_CAPACITY, "sme_count_noalloc: maximum degree " + std::to_string(maxdeg) +
                               " exceeds the allocation-free limit " + std::to_string(kNoAllocMaxDegree));
  if (hdr[5])
    Fail(SME_ERR_INVALID_ARG, "sme_count_noalloc: every adjacency list must be strictly increasing, hold ids "
                              "below n and not its own vertex (sorted, no duplicates, no self loops)");
  const uint32_t nbuf = (uint32_t)MaxBuffers({q});
  const uint32_t cap = std::max<uint32_t>(maxdeg, 1);
  const size_t groups_fit = (kNoAllocWords - kNoAllocHeader) / ((size_t)nbuf * cap);
  if (nbuf > BMAXV - 2 || groups_fit < (size_t)(kNoAllocBlock / kNoAllocGroup))
    Fail(SME_ERR_CAPACITY, "sme_count_noalloc: level buffers exceed the allocation-free scratch");
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_noalloc_dfs<kNoAllocGroup>, kNoAllocBlock, 0);
  const size_t gpb = kNoAllocBlock / kNoAllocGroup;
  const size_t grid = std::max<size_t>(1, std::min<size_t>((size_t)std::max(1, per_sm) * sms, groups_fit / gpb));
  k_noalloc_dfs<kNoAllocGroup><<<(unsigned)grid, kNoAllocBlock, 0, 0>>>(d_rp, d_cols, nv, q, cap, nbuf, base);
  uint64_t total = 0;
  BCK(cudaMemcpy(&total, base + 2, sizeof(total), cudaMemcpyDeviceToHost));
  BCK(cudaGetLastError());
  return total;
}

}  // namespace
}  // namespace sme

using namespace sme;

struct sme_batch_plan {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint64_t num = 0, nitems = 0;
  uint32_t cap = 1, nbuf = 1;
  uint32_t *d_rp = nullptr, *d_cols = nullptr, *d_goff = nullptr, *d_scratch = nullptr;
  uint8_t* d_query = nullptr;
  uint64_t* d_items = nullptr;
  unsigned long long* d_counts = nullptr;
  unsigned int* d_next = nullptr;
  int G = 8, block = 256, grid = 0, chunk = 1;
  float tuned_ms = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool use_graph = true;
  ~sme_batch_plan() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void* p : {(void*)d_rp, (void*)d_cols, (void*)d_goff, (void*)d_scratch, (void*)d_query, (void*)d_items,
                    (void*)d_counts, (void*)d_next})
      if (p) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

BArgs Args(sme_batch_plan* p) {
  BArgs a;
  a.rp = p->d_rp;
  a.cols = p->d_cols;
  a.goff = p->d_goff;
  a.query = p->d_query;
  a.items = p->d_items;
  a.nitems = p->nitems;
  a.counts = p->d_counts;
  a.next = p->d_next;
  a.scratch = p->d_scratch;
  a.cap = p->cap;
  a.nbuf = p->nbuf;
  a.chunk = (uint32_t)std::max(1, p->chunk);
  return a;
}

int SmCountB(int device) {
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  return v;
}

// Launches the persistent kernel with group size G and `block` threads on a
// grid of resident blocks; the scratch holds a buffer set per group.
void Launch(sme_batch_plan* p, int G, int block, int grid) {
  BArgs a = Args(p);
  switch (G) {
    case 4: k_batch<4><<<grid, block, 0, p->stream>>>(a); break;
    case 8: k_batch<8><<<grid, block, 0, p->stream>>>(a); break;
    case 16: k_batch<16><<<grid, block, 0, p->stream>>>(a); break;
    case 64: k_batch<64><<<grid, block, 0, p->stream>>>(a); break;
    case 128: k_batch<128><<<grid, block, 0, p->stream>>>(a); break;
    default: k_batch<32><<<grid, block, 0, p->stream>>>(a); break;
  }
}

int GridFor(sme_batch_plan* p, int G, int block) {
  int blocks_per_sm = 0;
  switch (G) {
    case 4: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_batch<4>, block, 0); break;
    case 8: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_batch<8>, block, 0); break;
    case 16: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_batch<16>, block, 0); break;
    case 64: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_batch<64>, block, 0); break;
    case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_batch<128>, block, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_batch<32>, block, 0); break;
  }
  return std::max(1, blocks_per_sm) * SmCountB(p->device);
}

void Reset(sme_batch_plan* p) {
  BCK(cudaMemsetAsync(p->d_counts, 0, p->num * sizeof(unsigned long long), p->stream));
  BCK(cudaMemsetAsync(p->d_next, 0, sizeof(unsigned int), p->stream));
}

float TimeConfig(sme_batch_plan* p, int G, int block) {
  int grid = GridFor(p, G, block);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  Reset(p);
  Launch(p, G, block, grid);  // warm
  Reset(p);
  cudaEventRecord(e0, p->stream);
  Launch(p, G, block, grid);
  cudaEventRecord(e1, p->stream);
  BCK(cudaStreamSynchronize(p->stream));
  BCK(cudaGetLastError());
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

void Prepare(sme_graph* const* graphs, const int32_t* queries, uint64_t num, const sme_batch_opts& o,
             sme_batch_plan* p) {
  if (num == 0) Fail(SME_ERR_INVALID_ARG, "empty batch");
  if (DeviceCount() <= o.device) Fail(SME_ERR_NO_DEVICE, "no CUDA device " + std::to_string(o.device));
  BCK(cudaSetDevice(o.device));
  p->device = o.device;
  p->num = num;
  p->use_graph = o.use_graph != 0;
  BCK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  UploadPrograms(o.device);
  std::vector<int32_t> qs(queries, queries + num);
  for (int32_t q : qs)
    if (q < 0 || q >= SME_NUM_QUERIES) Fail(SME_ERR_UNSUPPORTED_QUERY, "query out of range in batch");
  // pack CSRs (uint32 offsets; graphs are small)
  std::vector<uint32_t> rp, cols, goff(num);
  std::vector<uint8_t> qv(num);
  std::vector<std::pair<uint64_t, uint64_t>> work;  // (cost, item)
  uint64_t maxdeg = 1;
  for (uint64_t i = 0; i < num; ++i) {
    const HostGraph& g = graphs[i]->g;
    if (g.n >= (1ULL << 31)) Fail(SME_ERR_INVALID_ARG, "batched graphs must be small");
    goff[i] = (uint32_t)rp.size();
    qv[i] = (uint8_t)qs[i];
    uint64_t base = cols.size();
    if (base + g.m >= (1ULL << 32)) Fail(SME_ERR_INVALID_ARG, "batch too large for 32-bit packing");
    for (uint64_t u = 0; u <= g.n; ++u) rp.push_back((uint32_t)(base + g.row_ptrs[u]));
    cols.insert(cols.end(), g.cols, g.cols + g.m);
    for (uint64_t u = 0; u < g.n; ++u) {
      uint64_t d = g.row_ptrs[u + 1] - g.row_ptrs[u];
      maxdeg = std::max(maxdeg, d);
      // cost estimate: sum of neighbour degrees (two-level fan-out)
      uint64_t c = 1;
      for (uint64_t j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j) {
        uintV v = g.cols[j];
        c += g.row_ptrs[v + 1] - g.row_ptrs[v];
      }
      work.emplace_back(c, (i << 32) | u);
    }
  }
  std::stable_sort(work.begin(), work.end(), [](const std::pair<uint64_t, uint64_t>& a,
                                                const std::pair<uint64_t, uint64_t>& b) { return a.first > b.first; });
  std::vector<uint64_t> items(work.size());
  for (size_t i = 0; i < work.size(); ++i) items[i] = work[i].second;
  p->nitems = items.size();
  p->cap = (uint32_t)maxdeg;
  p->nbuf = (uint32_t)MaxBuffers(qs);
  auto up = [&](void** dst, const void* src, size_t bytes) {
    BCK(cudaMalloc(dst, std::max<size_t>(bytes, 4)));
    if (bytes) BCK(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, p->stream));
  };
  up((void**)&p->d_rp, rp.data(), rp.size() * 4);
  up((void**)&p->d_cols, cols.data(), cols.size() * 4);
  up((void**)&p->d_goff, goff.data(), goff.size() * 4);
  up((void**)&p->d_query, qv.data(), qv.size());
  up((void**)&p->d_items, items.data(), items.size() * 8);
  BCK(cudaMalloc((void**)&p->d_counts, num * sizeof(unsigned long long)));
  BCK(cudaMalloc((void**)&p->d_next, sizeof(unsigned int)));
  // scratch for the largest grid of any candidate configuration
  static const int kGroups[] = {4, 8, 16, 32, 64, 128};
  static const int kBlocks[] = {128, 256, 512};
  int max_groups = 0;
  for (int G : kGroups)
    for (int block : kBlocks)
      if (block >= G) max_groups = std::max(max_groups, GridFor(p, G, block) * (block / G));
  BCK(cudaMalloc((void**)&p->d_scratch, (size_t)max_groups * p->nbuf * p->cap * 4));
  // autotune on the batch itself: group size (a part of a warp, a warp, or
  // two or four warps of a CTA) x block shape with one item per fetch, then
  // the items per fetch for the winner
  int bestG = o.granularity == 2 ? 128 : o.granularity == 1 ? 32 : 8;
  int bestB = o.block_threads ? o.block_threads : 256;
  if (bestB < bestG) bestB = bestG;
  int bestC = 1;
  float best = 0;
  if (o.autotune) {
    best = 1e30f;
    p->chunk = 1;
    for (int G : kGroups)
      for (int block : kBlocks) {
        if (block < G) continue;
        float ms = TimeConfig(p, G, block);
        if (ms < best) {
          best = ms;
          bestG = G;
          bestB = block;
        }
      }
    for (int c : {4, 16}) {
      p->chunk = c;
      float ms = TimeConfig(p, bestG, bestB);
      if (ms < best) {
        best = ms;
        bestC = c;
      }
    }
  }
  p->G = bestG;
  p->block = bestB;
  p->chunk = bestC;
  p->tuned_ms = best;
  p->grid = GridFor(p, bestG, bestB);
  if (p->use_graph) {
    BCK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    Reset(p);
    Launch(p, p->G, p->block, p->grid);
    BCK(cudaStreamEndCapture(p->stream, &p->graph));
    BCK(cudaGraphInstantiate(&p->exec, p->graph, 0));
  }
  BCK(cudaStreamSynchronize(p->stream));
}

void Run(sme_batch_plan* p, uint64_t* counts, double* ms) {
  BCK(cudaSetDevice(p->device));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, p->stream);
  if (p->use_graph) {
    BCK(cudaGraphLaunch(p->exec, p->stream));
  } else {
    Reset(p);
    Launch(p, p->G, p->block, p->grid);
  }
  cudaEventRecord(e1, p->stream);
  BCK(cudaMemcpyAsync(counts, p->d_counts, p->num * sizeof(uint64_t), cudaMemcpyDeviceToHost, p->stream));
  BCK(cudaStreamSynchronize(p->stream));
  BCK(cudaGetLastError());
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t;
}

template <typename F>
sme_status BGuard(F&& f) {
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

sme_status sme_batch_opts_default(sme_batch_opts* o) {
  if (!o) return SME_ERR_INVALID_ARG;
  *o = sme_batch_opts{};
  o->autotune = 1;
  o->use_graph = 1;
  return SME_OK;
}

sme_status sme_batch_prepare(sme_graph* const* graphs, const int32_t* queries, uint64_t num,
                             const sme_batch_opts* opts, sme_batch_plan** out) {
  if (!graphs || !queries || !out) return SME_ERR_INVALID_ARG;
  return BGuard([&] {
    sme_batch_opts o;
    sme_batch_opts_default(&o);
    if (opts) o = *opts;
    // the batched plan extends in identity order with whole-ordered
    // conditions: on an oriented graph only the ordered cliques count right
    for (uint64_t i = 0; i < num; ++i)
      if (graphs[i] && graphs[i]->g.oriented && !IsOrderedClique(Query(queries[i], true)))
        Fail(SME_ERR_UNSUPPORTED_QUERY, "graph " + std::to_string(i) +
                                            " is oriented: only the clique queries (0, 3, 7, 11) count on it");
    std::unique_ptr<sme_batch_plan> p(new sme_batch_plan());
    Prepare(graphs, queries, num, o, p.get());
    *out = p.release();
  });
}

sme_status sme_batch_run(sme_batch_plan* p, uint64_t* counts, double* ms) {
  if (!p || !counts) return SME_ERR_INVALID_ARG;
  return BGuard([&] { Run(p, counts, ms); });
}

sme_status sme_batch_describe(const sme_batch_plan* p, int32_t* g, int32_t* block, uint64_t* items) {
  if (!p) return SME_ERR_INVALID_ARG;
  if (g) *g = p->G;
  if (block) *block = p->block;
  if (items) *items = p->nitems;
  return SME_OK;
}

sme_status sme_batch_tuning(const sme_batch_plan* p, int32_t* group_threads, int32_t* block_threads,
                            int32_t* items_per_fetch, double* tuned_ms) {
  if (!p) return SME_ERR_INVALID_ARG;
  if (group_threads) *group_threads = p->G;
  if (block_threads) *block_threads = p->block;
  if (items_per_fetch) *items_per_fetch = p->chunk;
  if (tuned_ms) *tuned_ms = p->tuned_ms;
  return SME_OK;
}

sme_status sme_batch_free(sme_batch_plan* p) {
  delete p;
  return SME_OK;
}

// Allocation-free count on a caller-owned device CSR (see include/sme.h): the
// only device memory touched besides the caller's is g_noalloc_scratch.
sme_status sme_count_noalloc(const uint64_t* d_row_ptrs, const uint32_t* d_cols, uint64_t n, int32_t query_type,
                             uint64_t* count) {
  if (!count) return SME_ERR_INVALID_ARG;
  return BGuard([&] { *count = CountNoAlloc(d_row_ptrs, d_cols, n, query_type); });
}

sme_status sme_batch_count(sme_graph* const* graphs, const int32_t* queries, uint64_t num,
                           const sme_batch_opts* opts, uint64_t* counts) {
  if (!graphs || !queries || !counts) return SME_ERR_INVALID_ARG;
  sme_batch_plan* p = nullptr;
  sme_status st = sme_batch_prepare(graphs, queries, num, opts, &p);
  if (st != SME_OK) return st;
  st = sme_batch_run(p, counts, nullptr);
  sme_batch_free(p);
  return st;
}

}  // extern "C"
