// Device engine: level-by-level extension of partial instances with
// memory-bounded batches, depth first over batches.
//
// Host control mirrors HybridGPUProcessor::ProcessLevel
// (src/gpu/impl/common/HybridGPUProcessor.cuh:14-50): per level, estimate each
// path's output (children estimate), split the frontier into batches that fit
// the level's memory budget (BatchManager::OrganizeBatch,
// src/gpu/utils/batch/BatchManager.cuh:42-110), execute the batch, recurse.
// Differences by design:
//   * one device allocation per context, used as a LIFO stack (no allocator
//     calls in the loop; the reference uses cnmem + per-op DeviceArray);
//   * intersections write in a single pass into a gapped buffer sized by the
//     children estimate, instead of count pass + scan + DToH + write pass
//     (GpsmBinSearch, src/gpu/utils/ops/intersect/GPSMBinSearch.cuh:144-197);
//   * candidate sets are (pointer, count) views: a set that is a sub-range of
//     an adjacency list or of an earlier set is not copied;
//   * counts accumulate on the device; the host reads one uint64 at the end.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <string>

#include "engine.h"
#include "kernels.cuh"

namespace sme {

using namespace dev;

#define CK(x)                                                                            \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) Fail(SME_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// sme_stats.phase_ms indices
constexpr int kPhaseCompute = 0, kPhaseMaterialize = 1, kPhaseFilter = 2, kPhaseComputeCount = 3,
              kPhasePathCount = 4, kPhaseCount = 5, kPhaseOrganize = 6, kPhaseExternal = 7;

// A timed region on the execution stream (two CUDA events) and its phase.
struct Timed {
  cudaEvent_t a, b;
  int phase;
};

// ---------------------------------------------------------------- kernels --
namespace {

__global__ void k_iota(uint32_t* out, uint32_t n, uint32_t start, uint32_t stride) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = start + i * stride;
}

// Children estimate of an intersection step: the smallest list (the pivot
// size), an upper bound of the candidate count (ThreadEstimatePathCount<MIN>,
// CheckConstraintsCommon.cuh:161-189).
// With `sumdeg`, also the bytes of adjacency lists the path reads (external
// mode: the subgraph a batch must load, EXTEstimateIntersectCost,
// src/gpu/impl/light/ext/EXTLIGHTOrganizeBatch.cuh:11-53).
__global__ void k_est_compute(DFront F, DStep s, const uintE* __restrict__ rp, uint64_t* est,
                              uint64_t* sumdeg) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.P; p += gridDim.x * blockDim.x) {
    uint64_t m = ~0ULL, sd = 0;
    for (int i = 0; i < s.nconn; ++i) {
      uint32_t v = F.inst[s.conn[i]][p];
      uint64_t d = rp[v + 1] - rp[v];
      m = min(m, d);
      sd += d;
    }
    if (sumdeg) sumdeg[p] = sd;
    if (s.reuse >= 0) {
      const uint32_t* ptr;
      uint32_t len;
      GetSet(F, s.reuse, p, ptr, len);
      m = min(m, (uint64_t)len);
    }
    est[p] = m == ~0ULL ? 0 : m;
  }
}

__global__ void k_est_set(DFront F, int u, uint64_t* est) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.P; p += gridDim.x * blockDim.x) {
    uint32_t s = SetIndex(F, u, p);
    est[p] = F.set[u].cnt[s];
  }
}

// ---- inclusive scan of uint64 (tile 4096 = 512 threads x 8) -------------
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr uint32_t SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ uint64_t BlockExclusiveScan(uint64_t v, uint64_t* total) {
  __shared__ uint64_t warp_tot[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    uint64_t t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t y = __shfl_up_sync(FULL, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) warp_tot[lane] = t;
  }
  __syncthreads();
  uint64_t warp_prefix = wid > 0 ? warp_tot[wid - 1] : 0;
  uint64_t excl = warp_prefix + x - v;
  if (total) *total = warp_tot[(blockDim.x >> 5) - 1];
  __syncthreads();
  return excl;
}

__global__ void k_scan_reduce(const uint64_t* __restrict__ in, uint32_t n, uint64_t* bs) {
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
  uint64_t s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    uint64_t i = base + (uint64_t)k * SCAN_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  __shared__ uint64_t red[SCAN_THREADS / 32];
  s = WarpSum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    uint64_t t = threadIdx.x < SCAN_THREADS / 32 ? red[threadIdx.x] : 0;
    t = WarpSum(t);
    if (threadIdx.x == 0) bs[blockIdx.x] = t;
  }
}

// Exclusive scan of the block sums in place (one block).
__global__ void k_scan_partials(uint64_t* bs, uint32_t nb) {
  uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
  uint32_t b = threadIdx.x * per, e = min(nb, b + per);
  uint64_t s = 0;
  for (uint32_t i = b; i < e; ++i) s += bs[i];
  uint64_t run = BlockExclusiveScan(s, nullptr);
  for (uint32_t i = b; i < e; ++i) {
    uint64_t v = bs[i];
    bs[i] = run;
    run += v;
  }
}

__global__ void k_scan_apply(uint64_t* data, uint32_t n, const uint64_t* __restrict__ bs) {
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
  uint64_t v[SCAN_ITEMS];
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    uint64_t i = base + k;
    v[k] = i < n ? data[i] : 0;
    s += v[k];
  }
  uint64_t run = BlockExclusiveScan(s, nullptr) + bs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    uint64_t i = base + k;
    run += v[k];
    if (i < n) data[i] = run;
  }
}

// Batch boundaries: for threshold k, the first path whose inclusive cost
// exceeds cost(start-1) + (k+1)*budget (SplitBatchKernel,
// src/gpu/utils/batch/SplitBatch.cuh:38-87).  cost(p) = pf*(p+1) + cf*est_incl[p].
__global__ void k_split(const uint64_t* __restrict__ incl, const uint64_t* __restrict__ incl2, uint32_t P,
                        uint32_t start, double pf, double cf, double cg, double budget, uint32_t K,
                        uint64_t* out) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  auto cost = [&](uint32_t p) {  // inclusive cost of paths [0, p]
    double c = pf * (double)(p + 1) + cf * (double)incl[p];
    if (incl2) c += cg * (double)incl2[p];
    return c;
  };
  double c0 = start == 0 ? 0.0 : cost(start - 1);
  double t = c0 + (double)(k + 1) * budget;
  uint32_t lo = start, hi = P;  // first p in [start,P) with cost(p) > t
  while (lo < hi) {
    uint32_t mid = lo + (hi - lo) / 2;
    double c = cost(mid);
    if (c > t) hi = mid;
    else lo = mid + 1;
  }
  out[2 * k] = lo;
  out[2 * k + 1] = lo == 0 ? 0 : incl[lo - 1];
  if (lo == start) {  // a single path above the budget: its own batch
    out[2 * k] = start + 1;
    out[2 * k + 1] = incl[start];
  }
}

// ---- paths grouped by the hub they probe ------------------------------------
// A count step's membership tests land on the dense bitmap of the hub whose
// list is searched.  Taken in frontier order, consecutive paths probe
// different hubs and every 4-byte test pulls a 32-byte sector from DRAM (the
// bitmaps do not fit L2); taken hub by hub, a hub's bitmap stays in L2 while
// its paths run.  A counting sort by hub slot (non-hubs in one last bucket)
// gives the order: warp-aggregated counts, a scan, a warp-aggregated scatter.
__global__ void k_hub_hist(DFront F, uint8_t kv, const int32_t* __restrict__ hub, uint32_t nb,
                           unsigned long long* cnt) {
  const int lane = threadIdx.x & 31;
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = w0; base < F.P; base += stride) {
    const uint32_t p = base + lane;
    uint32_t key = 0xffffffffu;
    if (p < F.P) {
      const int32_t h = __ldg(hub + F.inst[kv][p]);
      key = h < 0 ? nb - 1 : (uint32_t)h;
    }
    const unsigned same = __match_any_sync(FULL, key);
    if (key != 0xffffffffu && lane == __ffs(same) - 1) atomicAdd(cnt + key, (unsigned long long)__popc(same));
  }
}

__global__ void k_hub_cursor(const unsigned long long* __restrict__ incl, const unsigned long long* cnt,
                             uint32_t nb, unsigned long long* cur) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
    cur[b] = incl[b] - cnt[b];
}

__global__ void k_hub_scatter(DFront F, uint8_t kv, const int32_t* __restrict__ hub, uint32_t nb,
                              unsigned long long* cur, uint32_t* perm) {
  const int lane = threadIdx.x & 31;
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = w0; base < F.P; base += stride) {
    const uint32_t p = base + lane;
    uint32_t key = 0xffffffffu;
    if (p < F.P) {
      const int32_t h = __ldg(hub + F.inst[kv][p]);
      key = h < 0 ? nb - 1 : (uint32_t)h;
    }
    const unsigned same = __match_any_sync(FULL, key);
    const int leader = __ffs(same) - 1;
    unsigned long long at = 0;
    if (key != 0xffffffffu && lane == leader) at = atomicAdd(cur + key, (unsigned long long)__popc(same));
    at = __shfl_sync(FULL, at, leader);
    if (key != 0xffffffffu) perm[at + __popc(same & ((1u << lane) - 1))] = p;
  }
}

// ---- mapped reuse: the sibling path's cached intersection ----------------
// In the reuse plan the level-1 paths of a root M[0] are its neighbours N(M[0])
// in order (one contiguous run per root; the compiler checks level 1 has no
// condition), and the level-2 store holds, per level-1 path (M[0], y) of the
// current batch, the intersection N(M[0]) ∩ N(y).  A path whose ancestor is
// (M[0], M[1]) at store index s finds the sibling (M[0], M[x]) at index
// s + rank(M[x]) - rank(M[1]), ranks taken in N(M[0]) (FastLocateCache over
// the prefix tree, src/gpu/impl/common/CheckConstraintsReuseCommon.cuh:114-289,
// reduced to two binary searches by that layout).  `sib` stays null when the
// sibling is not in the store (another batch), and the step intersects the
// lists instead.
__device__ __forceinline__ void SiblingSet(const DFront& F, const DStep& s, const DGraph& G, uint32_t p,
                                           const uint32_t*& sib, uint32_t& sibn) {
  sib = nullptr;
  sibn = 0;
  if (s.msrc < 0) return;
  const uint32_t m0 = F.inst[0][p], m1 = F.inst[1][p], mx = F.inst[s.mx][p];
  if ((s.mop == 0 && !(mx < m0)) || (s.mop == 1 && !(mx > m0))) return;  // not a level-1 candidate
  const uint32_t* n0;
  uint32_t d0;
  AdjList(G, m0, n0, d0);
  const uint32_t ia = LowerBound(n0, d0, m1), ib = LowerBound(n0, d0, mx);
  if (ib >= d0 || __ldg(n0 + ib) != mx) return;
  const int64_t s2 = (int64_t)SetIndex(F, s.msrc, p) + (int64_t)ib - (int64_t)ia;
  if (s2 < 0 || s2 >= (int64_t)F.nset[s.msrc]) return;
  sib = reinterpret_cast<const uint32_t*>(F.set[s.msrc].ptr[s2]);
  sibn = F.set[s.msrc].cnt[s2];
}

// ---- intersection (COMPUTE / COMPUTE_COUNT / COMPUTE_PATH_COUNT) ---------
// One warp per path.  The pivot is the smallest list (ThreadChoosePivotLevel,
// CheckConstraintsCommon.cuh:10-29); < and > conditions clip the pivot to a
// sub-range by binary search before the scan; every pivot element is checked
// in the other lists by a per-lane binary search whose lower end advances with
// the lane's previous hit (each lane sees increasing candidates).
// MODE 0 writes the sorted candidate set, MODE 1 counts (optionally ranked
// into a partner set), MODE 2 stores only the per-path count.  MINB is the
// minimum resident blocks per SM asked of the register allocator (the
// kernels are latency bound: more resident warps, more searches in flight).
// NLM bounds the lists a step intersects (backward lists + cached set), so a
// step with two or three lists keeps fewer values live; NEX = 0 is for steps
// without `!=` conditions (no exclusion array).  The launcher guarantees
// both bounds.
// DEFER (two lists, no `!=`): a path whose clipped pivot holds at least
// hv.min_len elements is queued for k_compute_cta instead.  MAPPED (reuse
// plan, s.msrc >= 0): the set cached by the sibling path replaces the lists
// of s.mmask when the sibling is in the current batch (see SiblingSet).
template <int MODE, int MINB = 1, int NLM = MAXV, int NEX = MAXV, bool DEFER = false, bool MAPPED = false,
          bool PERM = false>
__global__ void __launch_bounds__(WARP_BLOCK, MINB) k_compute(
    DFront F, DStep s, DGraph G, const uint64_t* __restrict__ est_incl, uint32_t b0, uint64_t* out_ptr,
    uint32_t* out_cnt, uint32_t* out_data, uint64_t out_cap, unsigned long long* acc, uint32_t* err,
    DHeavy hv) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const unsigned lt = (1u << lane) - 1;
  unsigned long long local = 0, bytes = 0, hits = 0;
  const uint64_t base = b0 == 0 ? 0 : est_incl[b0 - 1];

  for (uint32_t pi = gw; pi < F.P; pi += nw) {
    const uint32_t p = PERM ? __ldg(hv.perm + pi) : pi;
    const uint32_t* L[NLM];
    const uint32_t* B[NLM];  // hub bitmap of the list (null: binary search)
    uint32_t N[NLM];
    int nl = 0;
    const uint32_t* sib = nullptr;
    uint32_t sibn = 0;
    if constexpr (MAPPED) SiblingSet(F, s, G, p, sib, sibn);
    if (MAPPED && sib) {
      // the lists outside the mask, then the sibling's cached set
#pragma unroll
      for (int i = 0; i < NLM; ++i) {
        if (i < s.nconn && !((s.mmask >> i) & 1)) {
          const uint32_t v = F.inst[s.conn[i]][p];
          const uint32_t* lp;
          uint32_t ln;
          AdjList(G, v, lp, ln);
#pragma unroll
          for (int t = 0; t < NLM; ++t)
            if (t == nl) {
              L[t] = lp;
              N[t] = ln;
              B[t] = HubBitmap(G, v);
            }
          ++nl;
        }
      }
#pragma unroll
      for (int t = 0; t < NLM; ++t)
        if (t == nl) {
          L[t] = sib;
          N[t] = sibn;
          B[t] = nullptr;
        }
      ++nl;
      if (lane == 0) ++hits;
    } else {
#pragma unroll
      for (int i = 0; i < NLM; ++i) {
        B[i] = nullptr;
        if (i < s.nconn) {
          uint32_t v = F.inst[s.conn[i]][p];
          AdjList(G, v, L[i], N[i]);
          B[i] = HubBitmap(G, v);
          nl = i + 1;
        }
      }
    }
    if (s.reuse >= 0) {
#pragma unroll
      for (int i = 0; i < NLM; ++i)
        if (i == nl) GetSet(F, s.reuse, p, L[i], N[i]);
      ++nl;
    }
    if (lane == 0) bytes += 12ULL * s.nconn;  // row pointers + gathered instance vertices
    // pivot to slot 0
#pragma unroll
    for (int i = 1; i < NLM; ++i) {
      if (i < nl && N[i] < N[0]) {
        const uint32_t* tp = L[0];
        L[0] = L[i];
        L[i] = tp;
        tp = B[0];
        B[0] = B[i];
        B[i] = tp;
        uint32_t tn = N[0];
        N[0] = N[i];
        N[i] = tn;
      }
    }
    BoundsT<NEX> bd = MakeBounds<NEX>(s.cond, F, p);
    uint32_t r0 = 0, r1 = 0;
    if (nl > 0) WarpRange(L[0], N[0], bd, r0, r1);
    if (DEFER && nl == 2 && r1 - r0 >= hv.min_len) {
      uint32_t slot = 0;
      if (lane == 0) slot = atomicAdd(hv.q, 1u);
      slot = __shfl_sync(FULL, slot, 0);
      if (slot < hv.cap) {
        if (lane == 0) hv.q[1 + slot] = p;
        continue;
      }
    }

    uint64_t out_off = 0;
    if (MODE == 0) {
      out_off = (p + b0 == 0 ? 0 : est_incl[p + b0 - 1]) - base;
      if (nl == 1 && !s.noview) {
        // single list: the candidate set is a sub-range unless an excluded
        // value falls inside it
        uint32_t ex[MAXV];
        int ne = Exclusions(L[0], r0, r1, bd, ex);
        if (ne == 0) {
          if (lane == 0) {
            out_ptr[p] = (uint64_t)(L[0] + r0);
            out_cnt[p] = r1 - r0;
          }
          continue;
        }
      }
    }
    // partner set for ranked counting
    const uint32_t* W = nullptr;
    uint32_t WN = 0;
    if (MODE == 1 && s.with_u >= 0) GetSet(F, s.with_u, p, W, WN);

    // every element of the clipped pivot is read once and tested against
    // each other list (one bitmap word or one list element answers a test)
    if (lane == 0) bytes += 4ULL * (r1 - r0) * (uint64_t)nl;
    uint32_t cur[NLM];
#pragma unroll
    for (int i = 0; i < NLM; ++i) cur[i] = 0;
    uint32_t written = 0;
    for (uint32_t bi = r0; bi < r1; bi += 32) {
      uint32_t i = bi + lane;
      bool ok = i < r1;
      uint32_t x = ok ? __ldg(L[0] + i) : 0;
#pragma unroll
      for (int k = 0; k < NEX; ++k)
        if (k < bd.nne && x == bd.ne[k]) ok = false;
#pragma unroll
      for (int j = 1; j < NLM; ++j) {
        if (j < nl && ok) {
          if (B[j]) {
            ok = BitTest(B[j], x);
          } else {
            uint32_t pos = cur[j] + LowerBound(L[j] + cur[j], N[j] - cur[j], x);
            cur[j] = pos;
            ok = pos < N[j] && __ldg(L[j] + pos) == x;
          }
        }
      }
      unsigned mask = __ballot_sync(FULL, ok);
      if (MODE == 0) {
        uint64_t o = out_off + written + __popc(mask & lt);
        if (ok) {
          if (o < out_cap) out_data[o] = x;
          else atomicOr(err, ENGINE_ERR_BOUNDS);
        }
      } else if (MODE == 1) {
        if (W != nullptr) {
          if (ok) local += RankCount(W, WN, x, s.with_op);
        } else if (lane == 0) {
          local += __popc(mask);
        }
      }
      written += __popc(mask);
    }
    if (lane == 0) {
      if (MODE == 0) {
        out_ptr[p] = (uint64_t)(out_data + out_off);
        out_cnt[p] = written;
        bytes += 4ULL * written;
      } else if (MODE == 2) {
        out_ptr[p] = 0;
        out_cnt[p] = written;
      }
    }
  }
  if (MODE == 1) {
    local = WarpSum(local);
    if (lane == 0 && local) atomicAdd(acc, local);
  }
  if (lane == 0 && bytes) atomicAdd(acc + 1, bytes);
  if (MAPPED && lane == 0 && hits) atomicAdd(acc + 5, hits);
}

// ---- intersection of the root's list with one other list -------------------
// Steps that intersect exactly two adjacency lists, one of them the list of
// the plan's first vertex (the root of the task: the 4-cycle's and the
// triangle's count steps, the diamond's path count, the 4-clique's second
// level).  The frontier keeps the paths of a root together (materialisation
// preserves the parents' order), so a CTA holds the root's list as an n-bit
// bitmap in shared memory and rebuilds it only when the root changes between
// runs of paths.  Per path a warp then takes the cheapest of: walking the
// other list's clipped range and testing each element in the shared bitmap
// (no search at all), walking the root's clipped range and testing the other
// vertex's hub bitmap (one load each), or walking the root's clipped range
// with a binary search in the other list (the warp kernel's way).  Costs are
// compared in warp iterations, a binary search counting log2 of the list.
// Results equal k_compute's: MODE 0 writes the sorted set (both walks visit
// ascending values), MODE 1 counts, MODE 2 stores the count.  CTAs take
// chunks of RM_CHUNK paths from a counter.
constexpr int RM_THREADS = 1024;
constexpr int RM_WARPS = RM_THREADS / 32;
constexpr uint32_t RM_CHUNK = 2048;
constexpr uint32_t kRootMapMaxBytes = 200u << 10;  // bitmaps up to n = 1 638 400
constexpr uint32_t kNoRoot = 0xFFFFFFFFu;

template <int MODE, int NEX>
__global__ void __launch_bounds__(RM_THREADS, 2) k_compute_rootmap(
    DFront F, DStep s, DGraph G, int ru, int other, const uint64_t* __restrict__ est_incl, uint32_t b0,
    uint64_t* out_ptr, uint32_t* out_cnt, uint32_t* out_data, uint64_t out_cap, unsigned long long* acc,
    uint32_t* err, uint32_t* next_chunk, uint32_t words) {
  extern __shared__ uint32_t rmap[];
  __shared__ uint32_t s_chunk, s_end;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1;
  for (uint32_t i = threadIdx.x; i < words; i += RM_THREADS) rmap[i] = 0;
  unsigned long long local = 0, bytes = 0;
  const uint64_t base = (MODE == 0 && b0 > 0) ? est_incl[b0 - 1] : 0;
  const uint32_t* rootcol = F.inst[ru];
  const uint32_t* othercol = F.inst[other];
  uint32_t cur_root = kNoRoot;
  __syncthreads();
  while (true) {
    if (threadIdx.x == 0) s_chunk = atomicAdd(next_chunk, 1u);
    __syncthreads();
    const uint64_t c0 = (uint64_t)s_chunk * RM_CHUNK;
    __syncthreads();  // s_chunk is rewritten only after the next barrier pair
    if (c0 >= F.P) break;
    const uint32_t c1 = (uint32_t)(c0 + RM_CHUNK < F.P ? c0 + RM_CHUNK : F.P);
    uint32_t p = (uint32_t)c0;
    while (p < c1) {
      const uint32_t r = __ldg(rootcol + p);
      if (threadIdx.x == 0) s_end = c1;
      __syncthreads();
      for (uint32_t q = p + threadIdx.x; q < c1; q += RM_THREADS)
        if (__ldg(rootcol + q) != r) {
          atomicMin(&s_end, q);
          break;
        }
      __syncthreads();
      const uint32_t e = s_end;
      if (r != cur_root) {
        const uint32_t* L;
        uint32_t N;
        if (cur_root != kNoRoot) {
          AdjList(G, cur_root, L, N);
          for (uint32_t i = threadIdx.x; i < N; i += RM_THREADS) rmap[__ldg(L + i) >> 5] = 0;
          __syncthreads();
        }
        AdjList(G, r, L, N);
        for (uint32_t i = threadIdx.x; i < N; i += RM_THREADS) {
          const uint32_t x = __ldg(L + i);
          atomicOr(rmap + (x >> 5), 1u << (x & 31));
        }
        __syncthreads();
        cur_root = r;
      }
      const uint32_t* Lr;
      uint32_t Nr;
      AdjList(G, r, Lr, Nr);
      for (uint32_t pp = p + wid; pp < e; pp += RM_WARPS) {
        const uint32_t v = __ldg(othercol + pp);
        const uint32_t* Lv;
        uint32_t Nv;
        AdjList(G, v, Lv, Nv);
        const uint32_t* Bv = HubBitmap(G, v);
        const uint32_t* Cv = HubCoarse(G, v);
        BoundsT<NEX> bd = MakeBounds<NEX>(s.cond, F, pp);
        uint32_t a0, a1, v0, v1;
        WarpRange(Lr, Nr, bd, a0, a1);
        WarpRange(Lv, Nv, bd, v0, v1);
        // algorithmic bytes as the warp kernel counts them: the smaller
        // list is the pivot, its clipped range read and tested once
        if (lane == 0) bytes += 24ULL + 8ULL * (Nv < Nr ? v1 - v0 : a1 - a0);
        const uint32_t wv = (v1 - v0 + 31) >> 5, wr = (a1 - a0 + 31) >> 5;
        int how = 0;  // 0: walk v's range, test the shared bitmap
        if (Bv) {
          if (wr < wv) how = 1;  // walk the root's range, test v's hub bitmap
        } else {
          const uint32_t lg = 32 - __clz(Nv | 1u);
          if (wr * lg < wv) how = 2;  // walk the root's range, search v's list
        }
        const uint32_t* W = how == 0 ? Lv : Lr;
        const uint32_t w0 = how == 0 ? v0 : a0, w1 = how == 0 ? v1 : a1;
        uint64_t out_off = 0;
        if (MODE == 0) out_off = (pp + b0 == 0 ? 0 : est_incl[pp + b0 - 1]) - base;
        uint32_t cur = 0, written = 0;
        for (uint32_t bi = w0; bi < w1; bi += 32) {
          const uint32_t i = bi + lane;
          bool ok = i < w1;
          const uint32_t x = ok ? __ldg(W + i) : 0;
#pragma unroll
          for (int k = 0; k < NEX; ++k)
            if (k < bd.nne && x == bd.ne[k]) ok = false;
          if (ok) {
            if (how == 0) {
              ok = (rmap[x >> 5] >> (x & 31)) & 1u;
            } else if (how == 1) {
              ok = BitTest2(Bv, Cv, x);
            } else {
              const uint32_t pos = cur + LowerBound(Lv + cur, Nv - cur, x);
              cur = pos;
              ok = pos < Nv && __ldg(Lv + pos) == x;
            }
          }
          const unsigned mask = __ballot_sync(FULL, ok);
          if (MODE == 0) {
            const uint64_t o = out_off + written + __popc(mask & lt);
            if (ok) {
              if (o < out_cap) out_data[o] = x;
              else atomicOr(err, ENGINE_ERR_BOUNDS);
            }
          } else if (MODE == 1 && lane == 0) {
            local += __popc(mask);
          }
          written += __popc(mask);
        }
        if (lane == 0) {
          if (MODE == 0) {
            out_ptr[pp] = (uint64_t)(out_data + out_off);
            out_cnt[pp] = written;
            bytes += 4ULL * written;
          } else if (MODE == 2) {
            out_ptr[pp] = 0;
            out_cnt[pp] = written;
          }
        }
      }
      __syncthreads();  // the bitmap may change for the next run
      p = e;
    }
  }
  if (MODE == 1) {
    local = WarpSum(local);
    if (lane == 0 && local) atomicAdd(acc, local);
  }
  if (lane == 0 && bytes) atomicAdd(acc + 1, bytes);
}

// ---- intersection, one CTA per long-pivot path ----------------------------
// The paths k_compute<..., DEFER> queued: two lists, no `!=` conditions, a
// clipped pivot of at least DHeavy::min_len elements.  All CTA_THREADS
// threads walk one path's pivot.  When the other list is not a hub (no
// bitmap), its window between the pivot's first and last value is staged in
// shared memory first: the 16-byte-aligned interior by one bulk copy
// (cp.async.bulk global -> shared, completion on an mbarrier, the source this
// GPU's own memory), the at most three elements on either ragged end by plain
// loads; every binary search then probes shared memory instead of L2.  The
// window is staged only when it fits `win_cap` elements and holds at most
// kStageRatio elements per pivot element (else the copy would read more than
// the searches).  Results equal k_compute's: MODE 0 writes the sorted set at
// the path's offset (block-ordered compaction), MODE 1 counts (ranked into a
// partner set when the step has one), MODE 2 stores the count.
constexpr int CTA_THREADS = 512;
constexpr int CTA_WARPS = CTA_THREADS / 32;
constexpr uint32_t kStageRatio = 16;
constexpr uint32_t kMbarSpins = 1u << 22;

__device__ __forceinline__ uint32_t LowerBoundShared(const uint32_t* a, uint32_t n, uint32_t x) {
  if (n == 0) return 0;
  const uint32_t* base = a;
  while (n > 1) {
    const uint32_t half = n >> 1;
    base = base[half] < x ? base + half : base;
    n -= half;
  }
  return (uint32_t)(base - a) + (base[0] < x ? 1u : 0u);
}

__device__ __forceinline__ bool MbarTryWait(uint32_t bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(bar), "r"(phase)
      : "memory");
  return done != 0;
}

// Waits (bounded) for the phase of `bar` to complete; false if it gave up.
__device__ __forceinline__ bool MbarWait(uint32_t bar, uint32_t phase) {
  for (uint32_t i = 0; i < kMbarSpins; ++i)
    if (MbarTryWait(bar, phase)) return true;
  return false;
}

template <int MODE>
__global__ void __launch_bounds__(CTA_THREADS, 2) k_compute_cta(
    DFront F, DStep s, DGraph G, const uint64_t* __restrict__ est_incl, uint32_t b0, uint64_t* out_ptr,
    uint32_t* out_cnt, uint32_t* out_data, uint64_t out_cap, unsigned long long* acc, uint32_t* err,
    const uint32_t* __restrict__ hq, uint32_t hq_cap, uint32_t win_cap) {
  extern __shared__ __align__(128) uint32_t win[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t wtot[CTA_WARPS];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t phase = 0;
  unsigned long long local = 0, bytes = 0;
  const uint64_t base = (MODE == 0 && b0 > 0) ? est_incl[b0 - 1] : 0;
  const uint32_t nheavy = min(hq[0], hq_cap);
  for (uint32_t i = blockIdx.x; i < nheavy; i += gridDim.x) {
    const uint32_t p = hq[1 + i];
    // the two lists (backward lists, then the reused set), pivot first
    const uint32_t* L[2];
    const uint32_t* Bm[2] = {nullptr, nullptr};
    uint32_t N[2];
    int nl = 0;
    for (int k = 0; k < 2 && k < s.nconn; ++k) {
      const uint32_t v = F.inst[s.conn[k]][p];
      AdjList(G, v, L[k], N[k]);
      Bm[k] = HubBitmap(G, v);
      nl = k + 1;
    }
    if (s.reuse >= 0 && nl < 2) {
      GetSet(F, s.reuse, p, L[nl], N[nl]);
      Bm[nl] = nullptr;
      ++nl;
    }
    if (N[1] < N[0]) {
      const uint32_t* t = L[0];
      L[0] = L[1];
      L[1] = t;
      t = Bm[0];
      Bm[0] = Bm[1];
      Bm[1] = t;
      const uint32_t tn = N[0];
      N[0] = N[1];
      N[1] = tn;
    }
    BoundsT<0> bd = MakeBounds<0>(s.cond, F, p);
    uint32_t r0 = 0, r1 = 0;
    Range(L[0], N[0], bd, r0, r1);
    if (tid == 0) bytes += 4ULL * (r1 - r0) * 2ULL;
    // the other list's window [a, e) over the pivot's value range
    const uint32_t* W = L[1];
    uint32_t WN = N[1];
    bool staged = false;
    uint32_t pad = 0;
    if (!Bm[1] && r1 > r0) {
      const uint32_t a = LowerBound(L[1], N[1], __ldg(L[0] + r0));
      const uint32_t e = a + LowerBound(L[1] + a, N[1] - a, __ldg(L[0] + r1 - 1) + 1);
      W = L[1] + a;
      WN = e - a;
      const uintptr_t lo = (uintptr_t)W, hi = (uintptr_t)(W + WN);
      const uintptr_t alo = (lo + 15) & ~(uintptr_t)15, ahi = hi & ~(uintptr_t)15;
      const uint32_t head = (uint32_t)((alo - lo) >> 2);  // elements before the aligned interior
      pad = (4 - (head & 3)) & 3;
      staged = WN >= 64 && pad + WN <= win_cap && WN <= kStageRatio * (r1 - r0) && ahi > alo;
      if (staged) {
        const uint32_t bytes_in = (uint32_t)(ahi - alo);
        if (tid == 0) {
          // shared memory the previous path read is overwritten by the async proxy
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes_in)
                       : "memory");
          const uint32_t dst = (uint32_t)__cvta_generic_to_shared(win + pad + head);
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
              "l"(alo), "r"(bytes_in), "r"(bar)
              : "memory");
        }
        // ragged ends by plain loads
        const uint32_t tail0 = (uint32_t)((ahi - lo) >> 2);
        if (tid < (int)head) win[pad + tid] = __ldg(W + tid);
        if (tid >= 4 && tid < 4 + (int)(WN - tail0)) win[pad + tail0 + (tid - 4)] = __ldg(W + tail0 + (tid - 4));
        const bool done = MbarWait(bar, phase);
        // one decision for the whole CTA (and the ragged ends made visible)
        if (__syncthreads_or(!done)) {
          // the copy did not complete: flag it, give it one more bounded
          // wait (it writes this CTA's shared memory) and stop this CTA
          if (tid == 0) atomicOr(err, ENGINE_ERR_TIMEOUT);
          MbarWait(bar, phase);
          return;
        }
        phase ^= 1;
      }
    }
    const uint32_t* Ws = staged ? win + pad : W;
    const uint32_t* Bo = Bm[1];
    const uint32_t* P2 = nullptr;  // ranked-count partner set
    uint32_t P2N = 0;
    if (MODE == 1 && s.with_u >= 0) GetSet(F, s.with_u, p, P2, P2N);
    const uint64_t out_off = MODE == 0 ? (p + b0 == 0 ? 0 : est_incl[p + b0 - 1]) - base : 0;
    uint32_t cur = 0, written = 0;
    for (uint32_t bi = r0; bi < r1; bi += CTA_THREADS) {
      const uint32_t k = bi + tid;
      bool ok = k < r1;
      const uint32_t x = ok ? __ldg(L[0] + k) : 0;
      if (ok && nl == 2) {
        if (Bo) {
          ok = BitTest(Bo, x);
        } else if (staged) {
          const uint32_t pos = cur + LowerBoundShared(Ws + cur, WN - cur, x);
          cur = pos;
          ok = pos < WN && Ws[pos] == x;
        } else {
          const uint32_t pos = cur + LowerBound(Ws + cur, WN - cur, x);
          cur = pos;
          ok = pos < WN && __ldg(Ws + pos) == x;
        }
      }
      const unsigned mask = __ballot_sync(FULL, ok);
      if (MODE == 1) {
        if (ok) local += P2 ? RankCount(P2, P2N, x, s.with_op) : 1ULL;
      } else {
        if (lane == 0) wtot[wid] = __popc(mask);
        __syncthreads();
        uint32_t before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < CTA_WARPS; ++w) {
          const uint32_t c = wtot[w];
          before += w < wid ? c : 0;
          total += c;
        }
        if (MODE == 0 && ok) {
          const uint64_t o = out_off + written + before + __popc(mask & ((1u << lane) - 1));
          if (o < out_cap) out_data[o] = x;
          else atomicOr(err, ENGINE_ERR_BOUNDS);
        }
        written += total;
        __syncthreads();  // wtot is rewritten by the next chunk
      }
    }
    if (tid == 0 && MODE != 1) {
      out_ptr[p] = MODE == 0 ? (uint64_t)(out_data + out_off) : 0;
      out_cnt[p] = written;
      if (MODE == 0) bytes += 4ULL * written;
    }
    __syncthreads();  // the window is free for the next path
  }
  if (MODE == 1) {
    local = WarpSum(local);
    if (lane == 0 && local) atomicAdd(acc, local);
  }
  if (tid == 0 && bytes) atomicAdd(acc + 1, bytes);
}

// ---- intersection, flattened over 32 paths per warp ------------------------
// Same result as k_compute.  Each lane first prepares one path (lists, pivot,
// clipped pivot range, excluded values) into shared memory; the warp then
// walks the concatenation of the 32 pivot ranges 32 elements at a time, so
// short pivots (the common case on skewed graphs) keep every lane busy.  A
// lane finds its element's path by binary search over the 32 range offsets.
// Sets stay sorted and compact per path: the rank of an element is its path's
// running count plus the valid lanes before it in the same path segment.
template <int NLM, int NEX>
struct FlatPath {
  const uint32_t* L[NLM];  // L[0] = pivot (already offset by r0); others cut to the pivot's value range
  const uint32_t* B[NLM];  // hub bitmaps (null: binary search)
  uint32_t N[NLM];
  uint32_t ne[NEX > 0 ? NEX : 1];
  const uint32_t* W;       // ranked-count partner set
  uint32_t WN;
  uint64_t out_off;
  uint32_t written;
  uint8_t nl, nne;
};
constexpr int FLAT_WARPS = WARP_BLOCK / 32;

// Specialised like k_compute: NLM bounds the intersected lists, NEX = 0 for
// steps without `!=` conditions (the launcher guarantees both).
template <int MODE, int MINB = 1, int NLM = MAXV, int NEX = MAXV>
__global__ void __launch_bounds__(WARP_BLOCK, MINB) k_compute_flat(
    DFront F, DStep s, DGraph G, const uint64_t* __restrict__ est_incl, uint32_t b0, uint64_t* out_ptr,
    uint32_t* out_cnt, uint32_t* out_data, uint64_t out_cap, unsigned long long* acc, uint32_t* err) {
  __shared__ FlatPath<NLM, NEX> sp[FLAT_WARPS][32];
  __shared__ uint32_t soff[FLAT_WARPS][33];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  unsigned long long local = 0, bytes = 0;
  const uint64_t base = (MODE == 0 && b0 > 0) ? est_incl[b0 - 1] : 0;
  for (uint32_t p0 = gw * 32; p0 < F.P; p0 += nw * 32) {
    const uint32_t p = p0 + lane;
    uint32_t len = 0;
    bool view = false;
    if (p < F.P) {
      FlatPath<NLM, NEX>& fp = sp[wl][lane];
      const uint32_t* L[NLM];
      const uint32_t* B[NLM];
      uint32_t N[NLM];
      int nl = 0;
#pragma unroll
      for (int i = 0; i < NLM; ++i) {
        B[i] = nullptr;
        if (i < s.nconn) {
          uint32_t v = F.inst[s.conn[i]][p];
          AdjList(G, v, L[i], N[i]);
          B[i] = HubBitmap(G, v);
          nl = i + 1;
        }
      }
      if (s.reuse >= 0) {
#pragma unroll
        for (int i = 0; i < NLM; ++i)
          if (i == nl) GetSet(F, s.reuse, p, L[i], N[i]);
        ++nl;
      }
      uint64_t b = 12ULL * s.nconn;  // row pointers + gathered instance vertices
#pragma unroll
      for (int i = 1; i < NLM; ++i) {
        if (i < nl && N[i] < N[0]) {
          const uint32_t* tp = L[0];
          L[0] = L[i];
          L[i] = tp;
          tp = B[0];
          B[0] = B[i];
          B[i] = tp;
          uint32_t tn = N[0];
          N[0] = N[i];
          N[i] = tn;
        }
      }
      BoundsT<NEX> bd = MakeBounds<NEX>(s.cond, F, p);
      uint32_t r0 = 0, r1 = 0;
      if (nl > 0) Range(L[0], N[0], bd, r0, r1);
      if (MODE == 0) {
        fp.out_off = (p + b0 == 0 ? 0 : est_incl[p + b0 - 1]) - base;
        if (nl == 1 && !s.noview) {
          uint32_t ex[MAXV];
          if (Exclusions(L[0], r0, r1, bd, ex) == 0) {
            out_ptr[p] = (uint64_t)(L[0] + r0);
            out_cnt[p] = r1 - r0;
            view = true;
          }
        }
      }
      if (!view) b += 4ULL * (r1 - r0) * (uint64_t)nl;  // pivot elements x lists tested
      bytes += b;
      fp.W = nullptr;
      fp.WN = 0;
      if (MODE == 1 && s.with_u >= 0) GetSet(F, s.with_u, p, fp.W, fp.WN);
      fp.L[0] = L[0] + r0;
      fp.N[0] = r1 - r0;
      // the other lists only matter between the pivot's first and last value
      const uint32_t lo_v = r1 > r0 ? __ldg(L[0] + r0) : 0, hi_v = r1 > r0 ? __ldg(L[0] + r1 - 1) : 0;
#pragma unroll
      for (int i = 1; i < NLM; ++i) {
        fp.B[i] = B[i];
        fp.L[i] = L[i];
        fp.N[i] = N[i];
        if (i < nl && !B[i] && r1 > r0) {
          const uint32_t a = LowerBound(L[i], N[i], lo_v);
          const uint32_t e = a + LowerBound(L[i] + a, N[i] - a, hi_v + 1);
          fp.L[i] = L[i] + a;
          fp.N[i] = e - a;
        }
      }
#pragma unroll
      for (int i = 0; i < NEX; ++i) fp.ne[i] = bd.ne[i];
      fp.nne = (uint8_t)bd.nne;
      fp.nl = (uint8_t)nl;
      fp.written = 0;
      len = view ? 0 : r1 - r0;
    }
    // exclusive scan of the pivot ranges of the 32 paths
    uint32_t x = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(FULL, x, o);
      if (lane >= o) x += y;
    }
    soff[wl][lane] = x - len;
    const uint32_t total = __shfl_sync(FULL, x, 31);
    if (lane == 31) soff[wl][32] = total;
    __syncwarp();
    for (uint32_t fb = 0; fb < total; fb += 32) {
      const uint32_t f = fb + lane;
      const bool in = f < total;
      // path of element f: last j with soff[j] <= f
      int j = 0;
      if (in) {
        int lo = 0, hi = 31;
        while (lo < hi) {
          int mid = (lo + hi + 1) >> 1;
          if (soff[wl][mid] <= f) lo = mid;
          else hi = mid - 1;
        }
        j = lo;
      }
      const FlatPath<NLM, NEX>& fp = sp[wl][j];
      bool ok = in;
      uint32_t v = 0;
      if (ok) {
        v = __ldg(fp.L[0] + (f - soff[wl][j]));
#pragma unroll
        for (int k = 0; k < NEX; ++k)
          if (k < fp.nne && v == fp.ne[k]) ok = false;
#pragma unroll
        for (int q = 1; q < NLM; ++q) {
          if (q < fp.nl && ok) {
            if (fp.B[q]) {
              ok = BitTest(fp.B[q], v);
            } else {
              uint32_t pos = LowerBound(fp.L[q], fp.N[q], v);
              ok = pos < fp.N[q] && __ldg(fp.L[q] + pos) == v;
            }
          }
        }
      }
      const unsigned valid = __ballot_sync(FULL, ok);
      if (MODE == 1) {
        if (ok) local += fp.W ? RankCount(fp.W, fp.WN, v, s.with_op) : 1;
      } else {
        // segments of lanes that belong to the same path
        const int jprev = __shfl_up_sync(FULL, j, 1);
        const unsigned start = __ballot_sync(FULL, in && (lane == 0 || jprev != j));
        const unsigned le = (lane == 31) ? FULL : ((2u << lane) - 1);
        const int seg = 31 - __clz(start & le);
        const unsigned segmask = (lane == 31 ? FULL : ((2u << lane) - 1)) & ~((1u << seg) - 1);
        const uint32_t before = __popc(valid & segmask & ((1u << lane) - 1));
        const uint32_t w0 = in ? sp[wl][j].written : 0;
        if (MODE == 0 && ok) {
          uint64_t o = fp.out_off + w0 + before;
          if (o < out_cap) out_data[o] = v;
          else atomicOr(err, ENGINE_ERR_BOUNDS);
        }
        __syncwarp();
        // the last lane of each segment advances its path's running count
        const int jnext = __shfl_down_sync(FULL, j, 1);
        const bool last = in && (lane == 31 || f + 1 >= total || jnext != j);
        if (last) sp[wl][j].written = w0 + before + (ok ? 1 : 0);
        __syncwarp();
      }
      (void)valid;
    }
    if (MODE != 1 && p < F.P && !view) {  // views were published above
      const FlatPath<NLM, NEX>& fp = sp[wl][lane];
      out_ptr[p] = MODE == 0 ? (uint64_t)(out_data + fp.out_off) : 0;
      out_cnt[p] = fp.written;
      if (MODE == 0) bytes += 4ULL * fp.written;
    }
    __syncwarp();
  }
  if (MODE == 1) {
    local = WarpSum(local);
    if (lane == 0 && local) atomicAdd(acc, local);
  }
  bytes = WarpSum(bytes);
  if (lane == 0 && bytes) atomicAdd(acc + 1, bytes);
}

// ---- MATERIALIZE ---------------------------------------------------------
// Valid children per path: set range clipped by < / >, minus excluded values.
__global__ void k_mat_count(DFront F, int u, DCond c, uint64_t* cnt) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.P; p += gridDim.x * blockDim.x) {
    const uint32_t* a;
    uint32_t n;
    GetSet(F, u, p, a, n);
    Bounds bd = MakeBounds(c, F, p);
    uint32_t r0, r1, ex[MAXV];
    Range(a, n, bd, r0, r1);
    int ne = Exclusions(a, r0, r1, bd, ex);
    cnt[p] = (uint64_t)(r1 - r0 - ne);
  }
}

// Expands each path's valid candidates into child rows: materialised columns
// (broadcast from the parent) plus the new vertex, and the set index of every
// live candidate set (Materialize, src/gpu/impl/light/op/LIGHTMaterialize.cuh:23-162,
// fused: expand + filter + compact + per-column gather in one pass).  Work is
// cut by child rows, not by parents: a warp takes kMatChunk consecutive rows,
// finds the parent of the first one with a warp-cooperative search over the
// inclusive child counts, and walks forward through the parents the chunk
// covers; the k-th child of a parent is its k-th candidate in the clipped
// range that is not excluded.  A parent with tens of thousands of children
// (a hub's list) is spread over many warps instead of holding one.  Only
// parents of more than `big` children are expanded here (the rest, whose
// per-parent set-up a chunk would serialise, take k_mat_write); the parents
// a chunk covers are scanned 32 at a time, one coalesced load per lane.
constexpr uint32_t kMatChunk = 1024;
constexpr uint64_t kMatBig = 2048;

// First p in [0, n) with a[p] > c, by the whole warp (`a` non-decreasing).
__device__ __forceinline__ uint32_t WarpUpperBound64(const uint64_t* __restrict__ a, uint32_t n, uint64_t c) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t lo = 0, len = n;
  while (len > 32) {
    const uint32_t step = (len + 31) / 32;
    const uint32_t idx = lo + lane * step;
    const bool le = idx < lo + len && __ldg(a + idx) <= c;
    const uint32_t k = __popc(__ballot_sync(0xffffffffu, le));
    if (k == 0) return lo;
    const uint32_t nlo = lo + (k - 1) * step + 1;
    const uint32_t nhi = min(lo + k * step, lo + len);
    lo = nlo;
    len = nhi - nlo;
  }
  const bool le = lane < len && __ldg(a + lo + lane) <= c;
  return lo + __popc(__ballot_sync(0xffffffffu, le));
}

__global__ void __launch_bounds__(WARP_BLOCK) k_mat_write_big(DFront F, DCond c, DMatOut o,
                                                              const uint64_t* __restrict__ incl,
                                                              uint64_t total, uint64_t big, uint32_t* err) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const int u = o.u;
  for (uint64_t c0 = (uint64_t)gw * kMatChunk; c0 < total; c0 += (uint64_t)nw * kMatChunk) {
    const uint64_t c1 = c0 + kMatChunk < total ? c0 + kMatChunk : total;
    // the parents overlapping [c0, c1) start at the parent of row c0; they
    // are scanned 32 at a time and only the large ones expanded
    uint32_t p = WarpUpperBound64(incl, F.P, c0);
    while (p < F.P) {
      const uint32_t q = p + lane;
      bool cand = false, past = false;
      if (q < F.P) {
        const uint64_t qe = __ldg(incl + q), qo = q == 0 ? 0 : __ldg(incl + q - 1);
        past = qo >= c1;
        cand = !past && qe - qo > big;  // qe > c0 holds for every q at or after the first parent
      }
      const unsigned mp = __ballot_sync(FULL, past);
      unsigned todo = __ballot_sync(FULL, cand);
      if (mp) todo &= (1u << (__ffs(mp) - 1)) - 1;
      while (todo) {
        const uint32_t pp = p + (__ffs(todo) - 1);
        todo &= todo - 1;
        const uint64_t off = pp == 0 ? 0 : __ldg(incl + pp - 1);
        const uint64_t end = __ldg(incl + pp);
        const uint32_t* a;
        uint32_t n;
        GetSet(F, u, pp, a, n);
        Bounds bd = MakeBounds(c, F, pp);
        uint32_t r0, r1, ex[MAXV];
        WarpRange(a, n, bd, r0, r1);
        int ne = Exclusions(a, r0, r1, bd, ex);
        uint32_t vals[MAXV], idx[MAXV];
#pragma unroll
        for (int i = 0; i < MAXV; ++i) {
          vals[i] = 0;
          idx[i] = 0;
          if (i < o.nmat && o.mat[i] != u) vals[i] = F.inst[o.mat[i]][pp];
          if (i < o.nsets) idx[i] = SetIndex(F, o.sets[i], pp);
        }
        const uint64_t s0 = off > c0 ? off : c0, s1 = end < c1 ? end : c1;
        for (uint64_t w = s0 + lane; w < s1; w += 32) {
          // the (w - off)-th candidate of [r0, r1) that is not excluded
          uint32_t j = r0 + (uint32_t)(w - off);
#pragma unroll
          for (int k = 0; k < MAXV; ++k)
            if (k < ne && ex[k] <= j) ++j;
          if (j >= r1) {
            atomicOr(err, ENGINE_ERR_BOUNDS);
            continue;
          }
          const uint32_t x = __ldg(a + j);
#pragma unroll
          for (int i = 0; i < MAXV; ++i) {
            if (i < o.nmat) o.inst[o.mat[i]][w] = o.mat[i] == u ? x : vals[i];
            if (i < o.nsets) o.cidx[o.sets[i]][w] = idx[i];
          }
        }
      }
      if (mp) break;
      p += 32;
    }
  }
}

// Parents of at most `big` children: one warp each (the large ones are
// k_mat_write_big's).
__global__ void __launch_bounds__(WARP_BLOCK) k_mat_write(DFront F, DCond c, DMatOut o,
                                                          const uint64_t* __restrict__ incl,
                                                          uint64_t total, uint64_t big, uint32_t* err) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const int u = o.u;
  for (uint32_t p = gw; p < F.P; p += nw) {
    if ((p == 0 ? incl[0] : incl[p] - incl[p - 1]) > big) continue;  // k_mat_write_big's
    const uint32_t* a;
    uint32_t n;
    GetSet(F, u, p, a, n);
    Bounds bd = MakeBounds(c, F, p);
    uint32_t r0, r1, ex[MAXV];
    Range(a, n, bd, r0, r1);
    int ne = Exclusions(a, r0, r1, bd, ex);
    uint64_t off = (p == 0 ? 0 : incl[p - 1]);
    uint32_t vals[MAXV], idx[MAXV];
#pragma unroll
    for (int i = 0; i < MAXV; ++i) {
      vals[i] = 0;
      idx[i] = 0;
      if (i < o.nmat && o.mat[i] != u) vals[i] = F.inst[o.mat[i]][p];
      if (i < o.nsets) idx[i] = SetIndex(F, o.sets[i], p);
    }
    for (uint32_t j = r0 + lane; j < r1; j += 32) {
      int before = 0;
      bool skip = false;
#pragma unroll
      for (int k = 0; k < MAXV; ++k) {
        if (k < ne) {
          if (ex[k] == j) skip = true;
          if (ex[k] < j) ++before;
        }
      }
      if (skip) continue;
      uint64_t w = off + (j - r0) - before;
      if (w >= total) {
        atomicOr(err, ENGINE_ERR_BOUNDS);
        continue;
      }
      uint32_t x = __ldg(a + j);
#pragma unroll
      for (int i = 0; i < MAXV; ++i) {
        if (i < o.nmat) o.inst[o.mat[i]][w] = o.mat[i] == u ? x : vals[i];
        if (i < o.nsets) o.cidx[o.sets[i]][w] = idx[i];
      }
    }
  }
}

// ---- FILTER_COMPUTE ------------------------------------------------------
// Re-applies conditions to a computed set (FilterCandidate,
// src/gpu/impl/light/op/LIGHTFilterCompute.cuh:22-155).  A filtered set with
// no excluded value inside its range is a view of the old set.
__global__ void __launch_bounds__(WARP_BLOCK) k_filter(DFront F, int u, DCond c,
                                                       const uint64_t* __restrict__ est_incl, uint32_t b0,
                                                       uint64_t* out_ptr, uint32_t* out_cnt,
                                                       uint32_t* out_data, uint64_t out_cap, uint32_t* err) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint64_t base = b0 == 0 ? 0 : est_incl[b0 - 1];
  for (uint32_t p = gw; p < F.P; p += nw) {
    const uint32_t* a;
    uint32_t n;
    GetSet(F, u, p, a, n);
    Bounds bd = MakeBounds(c, F, p);
    uint32_t r0, r1, ex[MAXV];
    Range(a, n, bd, r0, r1);
    int ne = Exclusions(a, r0, r1, bd, ex);
    if (ne == 0) {
      if (lane == 0) {
        out_ptr[p] = (uint64_t)(a + r0);
        out_cnt[p] = r1 - r0;
      }
      continue;
    }
    uint64_t off = (p + b0 == 0 ? 0 : est_incl[p + b0 - 1]) - base;
    for (uint32_t j = r0 + lane; j < r1; j += 32) {
      int before = 0;
      bool skip = false;
      for (int k = 0; k < ne; ++k) {
        if (ex[k] == j) skip = true;
        if (ex[k] < j) ++before;
      }
      if (skip) continue;
      uint64_t w = off + (j - r0) - before;
      if (w < out_cap) out_data[w] = __ldg(a + j);
      else atomicOr(err, ENGINE_ERR_BOUNDS);
    }
    if (lane == 0) {
      out_ptr[p] = (uint64_t)(out_data + off);
      out_cnt[p] = r1 - r0 - ne;
    }
  }
}

// ---- COUNT (LIGHTCount / LIGHTDirectCount) -------------------------------
// One unmaterialised vertex: sum of set sizes.
__global__ void k_count1(DFront F, int u, unsigned long long* acc) {
  unsigned long long s = 0;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.P; p += gridDim.x * blockDim.x)
    s += F.set[u].cnt[SetIndex(F, u, p)];
  s = WarpSum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(acc, s);
}

// Two unmaterialised vertices u0,u1 with condition (x0 op x1): each element of
// the smaller set is ranked in the larger one
// (GeneralCountTwoComputedVertices, src/gpu/impl/light/op/LIGHTCount.cuh:22-116).
__global__ void __launch_bounds__(WARP_BLOCK) k_count2(DFront F, int u0, int u1, uint8_t op,
                                                       unsigned long long* acc) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  unsigned long long s = 0;
  for (uint32_t p = gw; p < F.P; p += nw) {
    const uint32_t *A, *B;
    uint32_t na, nb;
    GetSet(F, u0, p, A, na);
    GetSet(F, u1, p, B, nb);
    if (na <= nb) {
      for (uint32_t i = lane; i < na; i += 32) s += RankCount(B, nb, __ldg(A + i), op);
    } else {
      // count x in A with (x op y) for each y in B
      uint8_t rop = op == 0 ? 1 : (op == 1 ? 0 : 2);
      for (uint32_t i = lane; i < nb; i += 32) s += RankCount(A, na, __ldg(B + i), rop);
    }
  }
  s = WarpSum(s);
  if (lane == 0 && s) atomicAdd(acc, s);
}

// Closed forms over candidate-set sizes (ThreadDirectCount,
// src/gpu/impl/light/op/LIGHTDirectCount.cuh:21-79).
__device__ unsigned long long DirectCount(const unsigned long long* c, int q) {
  unsigned long long r = 0;
  switch (q) {
    case 0: r = c[2]; break;
    case 1: r = c[3]; break;
    case 2: r = c[1] > 0 ? c[1] * (c[1] - 1) / 2 : 0; break;
    case 3: r = c[3]; break;
    case 5:
      r = c[1] * c[3] * c[5];
      if (r > 0) r = r - c[3] * (c[1] - 1 + c[5] - 1) - c[3] * c[3];
      break;
    case 6:
      if (c[4] > 0 && c[2] > 0) r = c[4] * c[2] - c[2];
      break;
    case 7: r = c[4]; break;
    case 8: r = c[4]; break;
    case 10: r = c[2] > 0 ? c[2] * (c[2] - 1) / 2 : 0; break;
    case 11: r = c[5]; break;
    default: r = 0;
  }
  return r;
}

__global__ void k_count_direct(DFront F, uint8_t nu, uint8_t u0, uint8_t u1, uint8_t u2, int q,
                               unsigned long long* acc) {
  unsigned long long s = 0;
  const uint8_t us[3] = {u0, u1, u2};
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.P; p += gridDim.x * blockDim.x) {
    unsigned long long c[MAXV] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < nu; ++i) c[us[i]] = F.set[us[i]].cnt[SetIndex(F, us[i], p)];
    s += DirectCount(c, q);
  }
  s = WarpSum(s);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(acc, s);
}

// ---- external mode: per-batch subgraph ------------------------------------
// Marks the adjacency lists a batch's intersections read
// (InspectRequiredAdjLists, src/gpu/impl/common/ext/EXTGraphGPUCommon.cuh:157-184).
// External mode keeps the adjacency lists a batch reads in a device list
// cache: coff[v] is the first element of v's list in the cache, kAbsent when
// it is not there.  A batch claims the lists it needs that are missing
// (IncInspectRequiredAdjLists, src/gpu/impl/common/ext/EXTIncGraphGPUCommon.cuh:20-75:
// lists already in device memory are not loaded again), places them after
// the cache's last list and gathers them from pinned, mapped host memory;
// lists stay for later batches and steps until the cache is full, when it
// starts over.  Only the lists of a batch cross the host link, and no work
// scales with the vertex count except a start-over.
constexpr uint64_t kAbsent = ~0ULL, kPending = ~0ULL - 1;

__global__ void k_ext_claim(DFront F, DStep s, const uintE* __restrict__ rp, uint64_t* coff, uint32_t* newids,
                            unsigned int* nnew) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.P; p += gridDim.x * blockDim.x)
    for (int i = 0; i < s.nconn; ++i) {
      const uint32_t v = F.inst[s.conn[i]][p];
      if (rp[v + 1] == rp[v] || coff[v] != kAbsent) continue;
      if (atomicCAS(reinterpret_cast<unsigned long long*>(coff + v), kAbsent, kPending) == kAbsent)
        newids[atomicAdd(nnew, 1u)] = v;
    }
}

__global__ void k_ext_newdeg(const uint32_t* __restrict__ ids, uint32_t n, const uintE* __restrict__ rp,
                             uint64_t* deg) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    deg[k] = rp[ids[k] + 1] - rp[ids[k]];
}

__global__ void k_ext_place(const uint32_t* __restrict__ ids, uint32_t n, const uint64_t* __restrict__ deg_incl,
                            uint64_t used, uint64_t* coff) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    coff[ids[k]] = used + (k == 0 ? 0 : deg_incl[k - 1]);
}

// Copies the newly placed lists from pinned, mapped host memory into the
// cache (one warp per list, coalesced reads over the host link); replaces
// the host-thread gather + synchronous H2D of LoadSubgraph
// (src/gpu/impl/common/ext/LoadSubgraph.h:10-42, EXTGraphGPUCommon.cuh:60-149).
__global__ void __launch_bounds__(WARP_BLOCK) k_ext_gather(const uint32_t* __restrict__ ids, uint32_t nid,
                                                           const uintE* __restrict__ rp,
                                                           const uint32_t* __restrict__ host_cols,
                                                           const uint64_t* __restrict__ coff,
                                                           uint32_t* __restrict__ cache) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < nid; i += nw) {
    const uint32_t v = ids[i];
    const uintE b = rp[v], e = rp[v + 1];
    const uint64_t o = coff[v];
    for (uintE j = b + lane; j < e; j += 32) cache[o + (j - b)] = host_cols[j];
  }
}

// Writes complete instances (all vertices materialised), in output slots.
__global__ void k_emit(DFront F, uint8_t n, const uint8_t* __restrict__ slot_dummy, uint8_t s0,
                       uint8_t s1, uint8_t s2, uint8_t s3, uint8_t s4, uint8_t s5, uint32_t* out,
                       uint64_t cap, unsigned long long* counter) {
  const uint8_t slot[MAXV] = {s0, s1, s2, s3, s4, s5};
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < F.P; p += gridDim.x * blockDim.x) {
    unsigned long long pos = atomicAdd(counter, 1ULL);
    if (pos < cap)
      for (int v = 0; v < n; ++v) out[pos * n + slot[v]] = F.inst[v][p];
  }
  (void)slot_dummy;
}

}  // namespace

// ---------------------------------------------------------------- runtime --
void* Arena::Alloc(size_t bytes) {
  size_t b = (bytes + 255) & ~size_t(255);
  if (b > cap - top)
    Fail(SME_ERR_OOM, "device arena exhausted: need " + std::to_string(b) + " bytes, " +
                          std::to_string(cap - top) + " free of " + std::to_string(cap));
  void* p = base + top;
  top += b;
  peak = std::max(peak, top);
  return p;
}

int DeviceCount() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

DeviceContext::~DeviceContext() {}

DeviceContext* CreateContext(int device, uint64_t bytes) {
  if (DeviceCount() <= device || device < 0) Fail(SME_ERR_NO_DEVICE, "no CUDA device " + std::to_string(device));
  CK(cudaSetDevice(device));
  auto* c = new DeviceContext();
  c->device = device;
  try {
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (auto& e : c->copy_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    uint64_t want = bytes ? bytes : (uint64_t)(fr * 0.80);
    if (want > fr) want = (uint64_t)(fr * 0.95);
    CK(cudaMalloc((void**)&c->arena.base, want));
    c->arena.cap = want;
    c->pinned_words = 1 << 14;
    CK(cudaMallocHost((void**)&c->h_pinned, c->pinned_words * sizeof(uint64_t)));
  } catch (...) {
    DestroyContext(c);
    throw;
  }
  return c;
}

void DestroyContext(DeviceContext* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  if (c->arena.base) cudaFree(c->arena.base);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  for (auto e : c->copy_ev)
    if (e) cudaEventDestroy(e);
  delete c;
}

namespace {
__global__ void k_build_bitmaps(const uintE* __restrict__ rp, const uint32_t* __restrict__ cols,
                                const uint32_t* __restrict__ hubs, uint32_t words, uint32_t* bm) {
  const uint32_t v = hubs[blockIdx.x];
  uint32_t* row = bm + (size_t)blockIdx.x * words;
  for (uintE j = rp[v] + threadIdx.x; j < rp[v + 1]; j += blockDim.x) {
    uint32_t w = cols[j];
    atomicOr(row + (w >> 5), 1u << (w & 31));
  }
}

// One hub's bitmap per CTA, built in shared memory and written out whole in
// 16-byte stores (no memset of the bitmaps and no global atomics); for
// bitmaps of up to kSmemBitmapBytes.  `words` is a multiple of 4.
constexpr uint32_t kSmemBitmapBytes = 200u << 10;
__global__ void __launch_bounds__(1024) k_build_bitmaps_smem(const uintE* __restrict__ rp,
                                                             const uint32_t* __restrict__ cols,
                                                             const uint32_t* __restrict__ hubs, uint32_t words,
                                                             uint32_t* bm, uint32_t* coarse, uint32_t cwords) {
  extern __shared__ uint4 row_v[];
  uint32_t* row_s = reinterpret_cast<uint32_t*>(row_v);
  const uint32_t quads = words / 4;
  for (uint32_t i = threadIdx.x; i < quads; i += blockDim.x) row_v[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  const uint32_t v = hubs[blockIdx.x];
  for (uintE j = rp[v] + threadIdx.x; j < rp[v + 1]; j += blockDim.x) {
    const uint32_t w = cols[j];
    atomicOr(row_s + (w >> 5), 1u << (w & 31));
  }
  __syncthreads();
  uint4* row = reinterpret_cast<uint4*>(bm + (size_t)blockIdx.x * words);
  for (uint32_t i = threadIdx.x; i < quads; i += blockDim.x) row[i] = row_v[i];
  // coarse row: bit b of word cw set when bitmap word 32 cw + b is not zero
  uint32_t* crow = coarse + (size_t)blockIdx.x * cwords;
  for (uint32_t cw = threadIdx.x; cw < cwords; cw += blockDim.x) {
    uint32_t bits = 0;
    for (uint32_t b = 0; b < 32; ++b) {
      const uint32_t wi = cw * 32 + b;
      if (wi < words && row_s[wi]) bits |= 1u << b;
    }
    crow[cw] = bits;
  }
}

__global__ void k_set_slots(const uint32_t* __restrict__ hubs, uint32_t nh, int32_t* slot) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x)
    slot[hubs[i]] = (int32_t)i;
}

// Bitmaps for the vertices of highest degree (>= kHubMinDegree) within a
// byte budget (SME_HUB_BITMAP_MB, default 1 GiB, at most a quarter of the
// device memory `room` the caller can spare); a bitmap is n bits.  Measured
// on R-MAT s20 (root blocks of the bench): 256 MiB 9.5e9, 512 MiB 9.8e9,
// 1 GiB 10.5e9, 2 GiB 10.7e9 instances/s, flat beyond; whole-graph counts
// flat from 512 MiB.  The hub choice is cached on the host graph; hubs take
// slots in id order, so the hubs of a vertex range are a slot range.
struct HubPlan {
  std::shared_ptr<const std::vector<uint32_t>> sel;  // sorted ids; slot i holds (*sel)[i]
  const std::vector<uint32_t>& hubs() const { return *sel; }
  uint32_t* d_hubs = nullptr;
  uint32_t words = 0;
  bool smem = false;
};

// Chooses the hubs, allocates slot index + bitmaps + hub list with `alloc`,
// and queues on `st` the hub-list copy, the slot fill and (global build only)
// the clearing of the bitmaps.  False when no vertex gets a bitmap.
template <typename Alloc>
bool PlanHubBitmaps(DeviceGraph* d, const HostGraph& g, cudaStream_t st, Alloc alloc, uint64_t room, HubPlan* hp) {
  uint64_t kHubMinDegree = 256;
  if (const char* e = std::getenv("SME_HUB_MIN_DEGREE")) kHubMinDegree = std::strtoull(e, nullptr, 10);
  uint64_t budget = 1024ULL << 20;
  if (const char* e = std::getenv("SME_HUB_BITMAP_MB")) budget = std::strtoull(e, nullptr, 10) << 20;
  budget = std::min<uint64_t>(budget, room / 4);
  // n bits, rounded up to whole 16-byte quads (rows start 16-byte aligned)
  const uint32_t words = (uint32_t)(((g.n + 31) / 32 + 3) & ~uint64_t(3));
  if (budget == 0 || words == 0) return false;
  const uint64_t max_hubs = budget / ((uint64_t)words * 4);
  if (max_hubs == 0) return false;
  hp->sel = g.HubSelection(kHubMinDegree, max_hubs);
  if (hp->sel->empty()) return false;
  const uint32_t nh = (uint32_t)hp->sel->size();
  hp->words = words;
  hp->smem = (uint64_t)words * 4 <= kSmemBitmapBytes;
  d->hub_slot = (int32_t*)alloc(g.n * sizeof(int32_t));
  d->bitmaps = (uint32_t*)alloc((size_t)nh * words * 4);
  if (hp->smem) {  // built beside the bitmap by the shared-memory builder
    d->cwords = (words + 31) / 32;
    d->coarse = (uint32_t*)alloc((size_t)nh * d->cwords * 4);
  }
  hp->d_hubs = (uint32_t*)alloc((size_t)nh * 4);
  CK(cudaMemcpyAsync(hp->d_hubs, hp->sel->data(), (size_t)nh * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(d->hub_slot, 0xFF, g.n * sizeof(int32_t), st));
  k_set_slots<<<std::min<uint32_t>((nh + 255) / 256, 1184), 256, 0, st>>>(hp->d_hubs, nh, d->hub_slot);
  if (!hp->smem) CK(cudaMemsetAsync(d->bitmaps, 0, (size_t)nh * words * 4, st));
  d->words = words;
  d->nhubs = nh;
  return true;
}

// Builds the bitmaps of slots [first, first + count) from the device lists.
void BuildHubRange(const DeviceGraph* d, const HubPlan& hp, uint32_t first, uint32_t count, cudaStream_t st) {
  if (!count) return;
  if (hp.smem) {
    CK(cudaFuncSetAttribute(k_build_bitmaps_smem, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)kSmemBitmapBytes));
    k_build_bitmaps_smem<<<count, 1024, (size_t)hp.words * 4, st>>>(
        d->row_ptrs, d->cols, hp.d_hubs + first, hp.words, d->bitmaps + (size_t)first * hp.words,
        d->coarse + (size_t)first * d->cwords, d->cwords);
  } else {
    k_build_bitmaps<<<count, 256, 0, st>>>(d->row_ptrs, d->cols, hp.d_hubs + first, hp.words,
                                           d->bitmaps + (size_t)first * hp.words);
  }
}

// Plan + build of every hub, synchronised.  `scratch_owned` frees the hub
// list afterwards (cudaMalloc'd).  Returns the host->device bytes.
template <typename Alloc>
uint64_t BuildHubBitmaps(DeviceGraph* d, const HostGraph& g, cudaStream_t stream, Alloc alloc, bool scratch_owned,
                         uint64_t room) {
  HubPlan hp;
  if (!PlanHubBitmaps(d, g, stream, alloc, room, &hp)) return 0;
  BuildHubRange(d, hp, 0, (uint32_t)hp.hubs().size(), stream);
  CK(cudaStreamSynchronize(stream));
  CK(cudaGetLastError());
  if (scratch_owned) cudaFree(hp.d_hubs);
  return (uint64_t)hp.hubs().size() * 4;
}

// ------------------------------------------------------------ packed lists --
// rp[0] = 0, rp[i + 1] = deg[i] (then an inclusive scan of rp + 1).
__global__ void k_deg_to_rp(const uint32_t* __restrict__ deg, uint64_t n, uintE* rp) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x)
    rp[i] = i ? deg[i - 1] : 0;
}

// Expands the packed lists (format: PackedLists, sme_internal.h) of lists
// [v0, v1) into cols; their segments after the first are segs[s0, s1).
// One warp per (list, segment): warps [0, v1 - v0) take segment 0 of list
// v0 + w, the next s1 - s0 warps the segments named in segs.  The warp reads
// the segment's block widths (one per lane), scans the blocks' byte sizes to
// place every block, then per block extracts one delta per lane and adds the
// running value through a warp scan.  Every offset read from the buffer is
// checked against the stream before use: a bad one sets *flag and skips the
// segment.
__global__ void __launch_bounds__(256) k_unpack_lists(const uint32_t* __restrict__ deg,
                                                      const uint32_t* __restrict__ woff,
                                                      const uint64_t* __restrict__ segs, uint64_t n, uint64_t v0,
                                                      uint64_t v1, uint64_t s0, uint64_t s1,
                                                      const uint32_t* __restrict__ stream, uint64_t stream_words,
                                                      const uintE* __restrict__ rp, uint64_t m, uintV* cols,
                                                      uint32_t* flag) {
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nv = v1 - v0;
  if (w >= nv + (s1 - s0)) return;  // uniform in the warp
  uint64_t v;
  uint32_t s;
  if (w < nv) {
    v = v0 + w;
    s = 0;
  } else {
    const uint64_t e = segs[s0 + (w - nv)];
    v = e >> 32;
    s = (uint32_t)e;
  }
  if (v >= n) {
    if (lane == 0) atomicOr(flag, 1u);
    return;
  }
  const uint64_t d = deg[v];
  const uint64_t nseg = (d + kPackSegment - 1) / kPackSegment;
  if (s >= nseg) {
    if (s > 0 && lane == 0) atomicOr(flag, 1u);
    return;
  }
  const uint64_t stream_bytes = stream_words * 4;
  const uint64_t list = (uint64_t)woff[v] * 4;
  uint32_t base = 0;
  uint64_t seg = list + 8 * (nseg - 1);
  if (s > 0) {
    const uint64_t ti = (list >> 2) + 2 * (uint64_t)(s - 1);
    if (ti + 1 >= stream_words) {
      if (lane == 0) atomicOr(flag, 1u);
      return;
    }
    base = stream[ti];
    seg = list + stream[ti + 1];
  }
  const uint64_t e0 = (uint64_t)s * kPackSegment;
  const uint32_t ne = (uint32_t)(d - e0 < kPackSegment ? d - e0 : kPackSegment);
  const uint32_t nb = (ne + 31) / 32;
  const uint64_t out0 = rp[v] + e0;
  if (seg + nb + 8 > stream_bytes || out0 + ne > m) {
    if (lane == 0) atomicOr(flag, 1u);
    return;
  }
  const uint8_t* bytes = reinterpret_cast<const uint8_t*>(stream);
  const uint32_t width = lane < nb ? bytes[seg + lane] : 0;
  const uint32_t cnt = lane < nb ? min(32u, ne - 32 * lane) : 0;
  const uint32_t sz = (cnt * width + 7) / 8;
  uint32_t incl = sz;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t total = __shfl_sync(FULL, incl, 31);
  if (__any_sync(FULL, width > 32) || seg + nb + total + 8 > stream_bytes) {
    if (lane == 0) atomicOr(flag, 1u);
    return;
  }
  const uint64_t off = seg + nb + (incl - sz);  // byte start of this lane's block
  uintV* out = cols + out0;
  uint32_t prev = base;
  for (uint32_t t = 0; t < nb; ++t) {
    const uint32_t b = __shfl_sync(FULL, width, t);
    const uint32_t c = __shfl_sync(FULL, cnt, t);
    const uint64_t o = __shfl_sync(FULL, (unsigned long long)off, t);
    uint32_t delta = 0;
    if (lane < c && b) {
      const uint64_t bit = o * 8 + (uint64_t)lane * b;
      const uint64_t wi = bit >> 5;
      delta = __funnelshift_r(stream[wi], stream[wi + 1], (uint32_t)bit & 31);
      if (b < 32) delta &= (1u << b) - 1u;
    }
#pragma unroll
    for (int o2 = 1; o2 < 32; o2 <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, delta, o2);
      if (lane >= o2) delta += y;
    }
    const uint32_t val = prev + delta;
    if (lane < c) out[32 * t + lane] = val;
    prev = __shfl_sync(FULL, val, 31);
  }
}

uint32_t ScanBlocks(uint64_t n) { return (uint32_t)((n + SCAN_TILE - 1) / SCAN_TILE); }

// row_ptrs from the packed degrees in `scratch` (copied there already).
void PackedRowPtrs(const PackedLists& pk, const uint8_t* scratch, uint64_t* bs, uintE* rp, cudaStream_t st) {
  const uint64_t n = pk.n;
  const uint32_t* deg = reinterpret_cast<const uint32_t*>(scratch + pk.deg_at);
  k_deg_to_rp<<<(unsigned)std::min<uint64_t>((n + 256) / 256, 148 * 8), 256, 0, st>>>(deg, n, rp);
  if (n) {
    const uint32_t nb = ScanBlocks(n);
    k_scan_reduce<<<nb, SCAN_THREADS, 0, st>>>(rp + 1, (uint32_t)n, bs);
    k_scan_partials<<<1, 1024, 0, st>>>(bs, nb);
    k_scan_apply<<<nb, SCAN_THREADS, 0, st>>>(rp + 1, (uint32_t)n, bs);
  }
}

// Expands lists [v0, v1) (segments segs[s0, s1)) from `scratch` into cols.
void UnpackRange(const PackedLists& pk, const uint8_t* scratch, const uintE* rp, uintV* cols, uint32_t* flag,
                 uint64_t v0, uint64_t v1, uint64_t s0, uint64_t s1, cudaStream_t st) {
  const uint64_t items = (v1 - v0) + (s1 - s0);
  if (!items) return;
  k_unpack_lists<<<(unsigned)((items * 32 + 255) / 256), 256, 0, st>>>(
      reinterpret_cast<const uint32_t*>(scratch + pk.deg_at), reinterpret_cast<const uint32_t*>(scratch + pk.woff_at),
      reinterpret_cast<const uint64_t*>(scratch + pk.segs_at), pk.n, v0, v1, s0, s1,
      reinterpret_cast<const uint32_t*>(scratch + pk.stream_at), pk.stream_bytes / 4, rp, pk.m, cols, flag);
}

// Copies the packed lists into `scratch` (device, pk.total bytes) and expands
// them into rp (n + 1) and cols (m) on `st`.  `bs` holds ScanBlocks(n) words,
// `flag` one word (set by a bad offset).
void UnpackLists(const PackedLists& pk, uint8_t* scratch, uint64_t* bs, uint32_t* flag, uintE* rp, uintV* cols,
                 cudaStream_t st) {
  CK(cudaMemcpyAsync(scratch, pk.base, pk.total, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(flag, 0, sizeof(uint32_t), st));
  PackedRowPtrs(pk, scratch, bs, rp, st);
  UnpackRange(pk, scratch, rp, cols, flag, 0, pk.n, 0, pk.nsegs, st);
  CK(cudaGetLastError());
}

void CheckPacked(const HostGraph& g, const PackedLists& pk) {
  if (pk.n != g.n || pk.m != g.m) Fail(SME_ERR_INVALID_ARG, "packed lists do not match the graph");
  if (pk.n > UINT32_MAX) Fail(SME_ERR_INVALID_ARG, "packed upload needs n < 2^32");
}

void FailOnFlag(uint32_t flag) {
  if (flag) Fail(SME_ERR_CUDA, "packed lists are corrupt: an offset points outside the stream");
}

// Per-call packed upload into the arena, copy and expansion overlapped: the
// header (degrees, list offsets, segment ids) and then kUploadChunks byte
// ranges of the stream, cut at list boundaries, go over the context's copy
// stream; the execution stream scans the degrees into row_ptrs, then, as each
// range lands, expands its lists and builds the bitmaps of its hubs.  Hub
// bitmaps are allocated below the copy's scratch, which is released when the
// upload is done.  Returns the host->device bytes beyond the packed buffer.
uint64_t UploadPackedPipelined(const HostGraph& g, const PackedLists& pk, DeviceGraph* d, DeviceContext& ctx,
                               uint32_t* flag) {
  auto arena_alloc = [&ctx](size_t b) { return ctx.arena.Alloc(b); };
  const uint64_t n = pk.n;
  const uint64_t scratch_bytes = pk.total + (uint64_t)ScanBlocks(n) * 8 + 512;
  HubPlan hp;
  const uint64_t room = ctx.arena.Free() > scratch_bytes ? ctx.arena.Free() - scratch_bytes : 0;
  const bool hubs = PlanHubBitmaps(d, g, ctx.stream, arena_alloc, room, &hp);
  const size_t mark = ctx.arena.Mark();
  uint8_t* scratch = (uint8_t*)arena_alloc(pk.total);
  uint64_t* bs = (uint64_t*)arena_alloc((size_t)ScanBlocks(n) * 8);
  CK(cudaMemsetAsync(flag, 0, sizeof(uint32_t), ctx.stream));

  // chunk boundaries: list ids where the stream offset passes k/K of it
  const uint32_t* woff = reinterpret_cast<const uint32_t*>(pk.base + pk.woff_at);
  const uint64_t* segs = reinterpret_cast<const uint64_t*>(pk.base + pk.segs_at);
  const uint64_t lists_words = (pk.stream_bytes - 8) / 4;
  const int K = pk.stream_bytes >= (8ULL << 20) ? kUploadChunks : 1;
  uint64_t vb[kUploadChunks + 1];
  vb[0] = 0;
  vb[K] = n;
  for (int k = 1; k < K; ++k)
    vb[k] = std::max<uint64_t>(vb[k - 1],
                               (uint64_t)(std::lower_bound(woff, woff + n, (uint32_t)(lists_words * k / K)) - woff));
  auto byte_at = [&](uint64_t v) { return v < n ? (uint64_t)woff[v] * 4 : pk.stream_bytes; };
  auto seg_at = [&](uint64_t v) {
    return (uint64_t)(std::lower_bound(segs, segs + pk.nsegs, v << 32) - segs);
  };

  CK(cudaMemcpyAsync(scratch, pk.base, pk.stream_at, cudaMemcpyHostToDevice, ctx.copy_stream));
  CK(cudaEventRecord(ctx.copy_ev[0], ctx.copy_stream));
  for (int k = 0; k < K; ++k) {
    const uint64_t b0 = k == 0 ? 0 : byte_at(vb[k]), b1 = k + 1 == K ? pk.stream_bytes : byte_at(vb[k + 1]);
    if (b1 > b0)
      CK(cudaMemcpyAsync(scratch + pk.stream_at + b0, pk.base + pk.stream_at + b0, b1 - b0,
                         cudaMemcpyHostToDevice, ctx.copy_stream));
    CK(cudaEventRecord(ctx.copy_ev[k + 1], ctx.copy_stream));
  }
  CK(cudaStreamWaitEvent(ctx.stream, ctx.copy_ev[0], 0));
  PackedRowPtrs(pk, scratch, bs, d->row_ptrs, ctx.stream);
  for (int k = 0; k < K; ++k) {
    CK(cudaStreamWaitEvent(ctx.stream, ctx.copy_ev[k + 1], 0));
    UnpackRange(pk, scratch, d->row_ptrs, d->cols, flag, vb[k], vb[k + 1], seg_at(vb[k]), seg_at(vb[k + 1]),
                ctx.stream);
    if (hubs) {
      const std::vector<uint32_t>& H = hp.hubs();
      const uint32_t h0 = (uint32_t)(std::lower_bound(H.begin(), H.end(), (uint32_t)vb[k]) - H.begin());
      const uint32_t h1 = vb[k + 1] >= n ? (uint32_t)H.size()
                                         : (uint32_t)(std::lower_bound(H.begin(), H.end(), (uint32_t)vb[k + 1]) -
                                                      H.begin());
      BuildHubRange(d, hp, h0, h1 - h0, ctx.stream);
    }
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx.stream));
  ctx.arena.Release(mark);
  return hubs ? (uint64_t)hp.hubs().size() * 4 : 0;
}
}  // namespace

DeviceGraph* UploadGraph(const HostGraph& g, int device, cudaStream_t stream, uint64_t* h2d) {
  CK(cudaSetDevice(device));
  auto* d = new DeviceGraph();
  d->device = device;
  d->n = g.n;
  d->m = g.m;
  uint64_t bytes = 0;
  std::shared_ptr<const PackedLists> pk = g.packed;
  uint8_t* scratch = nullptr;
  try {
    CK(cudaMalloc((void**)&d->row_ptrs, (g.n + 1) * sizeof(uintE)));
    CK(cudaMalloc((void**)&d->cols, std::max<uint64_t>(g.m, 1) * sizeof(uintV)));
    if (pk) {
      CheckPacked(g, *pk);
      const uint64_t bs_at = (pk->total + 15) & ~uint64_t(15);
      CK(cudaMalloc((void**)&scratch, bs_at + (uint64_t)ScanBlocks(g.n) * 8 + 16));
      uint32_t* flag = reinterpret_cast<uint32_t*>(scratch + bs_at + (uint64_t)ScanBlocks(g.n) * 8);
      UnpackLists(*pk, scratch, reinterpret_cast<uint64_t*>(scratch + bs_at), flag, d->row_ptrs, d->cols, stream);
      uint32_t h_flag = 0;
      CK(cudaMemcpyAsync(&h_flag, flag, 4, cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      cudaFree(scratch);
      scratch = nullptr;
      FailOnFlag(h_flag);
      bytes = pk->total;
    } else {
      CK(cudaMemcpyAsync(d->row_ptrs, g.row_ptrs, (g.n + 1) * sizeof(uintE), cudaMemcpyHostToDevice, stream));
      if (g.m) CK(cudaMemcpyAsync(d->cols, g.cols, g.m * sizeof(uintV), cudaMemcpyHostToDevice, stream));
      CK(cudaStreamSynchronize(stream));
      bytes = (g.n + 1) * sizeof(uintE) + g.m * sizeof(uintV);
    }
    auto dev_alloc = [](size_t b) {
      void* p = nullptr;
      CK(cudaMalloc(&p, b));
      return p;
    };
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    bytes += BuildHubBitmaps(d, g, stream, dev_alloc, true, fr);
  } catch (...) {
    if (scratch) cudaFree(scratch);
    FreeDeviceGraph(d);
    throw;
  }
  if (h2d) *h2d += bytes;
  return d;
}

DeviceGraph* UploadGraphToArena(const HostGraph& g, DeviceContext& ctx, uint64_t* h2d) {
  CK(cudaSetDevice(ctx.device));
  auto* d = new DeviceGraph();
  d->device = ctx.device;
  d->n = g.n;
  d->m = g.m;
  d->in_arena = true;
  uint64_t bytes = 0;
  std::shared_ptr<const PackedLists> pk = g.packed;
  try {
    auto arena_alloc = [&ctx](size_t b) { return ctx.arena.Alloc(b); };
    d->row_ptrs = (uintE*)arena_alloc((g.n + 1) * sizeof(uintE));
    d->cols = (uintV*)arena_alloc(std::max<uint64_t>(g.m, 1) * sizeof(uintV));
    uint32_t* flag = nullptr;
    if (pk) {
      CheckPacked(g, *pk);
      flag = (uint32_t*)arena_alloc(sizeof(uint32_t));
      bytes = pk->total + UploadPackedPipelined(g, *pk, d, ctx, flag);
    } else {
      CK(cudaMemcpyAsync(d->row_ptrs, g.row_ptrs, (g.n + 1) * sizeof(uintE), cudaMemcpyHostToDevice, ctx.stream));
      if (g.m) CK(cudaMemcpyAsync(d->cols, g.cols, g.m * sizeof(uintV), cudaMemcpyHostToDevice, ctx.stream));
      bytes = (g.n + 1) * sizeof(uintE) + g.m * sizeof(uintV);
      bytes += BuildHubBitmaps(d, g, ctx.stream, arena_alloc, false, ctx.arena.Free());
    }
    if (flag) {
      CK(cudaMemcpyAsync(ctx.h_pinned, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx.stream));
      CK(cudaStreamSynchronize(ctx.stream));
      FailOnFlag(*reinterpret_cast<const uint32_t*>(ctx.h_pinned));
    }
    CK(cudaStreamSynchronize(ctx.stream));
  } catch (...) {
    delete d;
    throw;
  }
  if (h2d) *h2d += bytes;
  return d;
}

void FreeDeviceGraph(DeviceGraph* d) {
  if (!d) return;
  if (d->in_arena) {  // released with the arena mark taken before the upload
    delete d;
    return;
  }
  cudaSetDevice(d->device);
  if (d->row_ptrs) cudaFree(d->row_ptrs);
  if (d->cols && !d->host_mapped) cudaFree(d->cols);
  if (d->hub_slot) cudaFree(d->hub_slot);
  if (d->bitmaps) cudaFree(d->bitmaps);
  if (d->coarse) cudaFree(d->coarse);
  delete d;
}

// --------------------------------------------------------------- executor --
namespace {

int SmCount(int device) {
  static int cached[64] = {0};
  if (device >= 0 && device < 64 && cached[device]) return cached[device];
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  if (device >= 0 && device < 64) cached[device] = v;
  return v;
}

DCond ToDCond(const std::vector<StepCond>& c) {
  DCond d{};
  d.n = (uint8_t)c.size();
  for (size_t i = 0; i < c.size(); ++i) {
    d.op[i] = c[i].op;
    d.operand[i] = c[i].operand;
  }
  return d;
}

DStep ToDStep(const Step& s) {
  DStep d{};
  d.u = s.u;
  d.nconn = (uint8_t)s.conn.size();
  for (size_t i = 0; i < s.conn.size(); ++i) d.conn[i] = s.conn[i];
  d.reuse = s.reuse_src;
  d.cond = ToDCond(s.cond);
  d.with_u = s.with_u;
  d.with_op = s.with_op;
  d.msrc = s.map_src;
  d.mx = s.map_x;
  d.mmask = s.map_mask;
  d.mop = s.map_op;
  return d;
}

class Executor {
 public:
  Executor(const Program& prog, const DeviceGraph& g, DeviceContext& ctx, uint32_t* d_out, uint64_t cap)
      : prog_(prog), g_(g), ctx_(ctx), A_(ctx.arena), st_(ctx.stream), out_(d_out), cap_(cap) {
    sms_ = SmCount(ctx.device);
  }

  // External mode: adjacency lists are read from `host_cols` (pinned and
  // mapped host memory) into a per-batch device subgraph; g_.row_ptrs holds
  // the global row pointers on the device (GraphDevTracker,
  // src/gpu/graph/GraphDevTracker.cuh:12-79).
  void SetExternal(const uint32_t* host_cols) { ext_cols_ = host_cols; }
  uint64_t ext_h2d_bytes() const { return ext_bytes_; }

  RunResult Run(const RootTask& task) {
    const uint32_t stride = task.stride ? task.stride : 1;
    auto t0 = std::chrono::steady_clock::now();
    size_t mark = A_.Mark();
    A_.peak = mark;  // high-water mark of this run
    ctrl_ = (unsigned long long*)A_.Alloc(8 * sizeof(unsigned long long));
    if (ext_cols_) AllocExternalCache();
    cudaEvent_t ev0, ev1;
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    CK(cudaEventRecord(ev0, st_));
    CK(cudaMemsetAsync(ctrl_, 0, 8 * sizeof(unsigned long long), st_));
    const Step& s0 = prog_.steps[0];
    // roots: inst column + next level estimate + scan temporaries
    const uint64_t per_root = 4 + 8 + 8;
    uint64_t chunk = std::max<uint64_t>(1, Budget(0) / per_root);
    chunk = std::min<uint64_t>(chunk, 0x7fffffffULL);
    // the task's roots in chunks of `chunk` roots
    const uint64_t nroots = task.Count();
    for (uint64_t i0 = 0; i0 < nroots; i0 += chunk) {
      uint32_t P = (uint32_t)std::min<uint64_t>(chunk, nroots - i0);
      size_t m = A_.Mark();
      uint32_t* col = (uint32_t*)A_.Alloc((size_t)P * 4);
      if (task.list) {
        CK(cudaMemcpyAsync(col, task.list + i0, (size_t)P * 4, cudaMemcpyHostToDevice, st_));
        root_h2d_ += (uint64_t)P * 4;
      } else {
        k_iota<<<Grid(P, 256), 256, 0, st_>>>(col, P, (uint32_t)(task.begin + i0 * stride), stride);
        Launched();
      }
      DFront F{};
      F.P = P;
      F.inst[s0.u] = col;
      ++batches_;
      Level(1, F);
      A_.Release(m);
    }
    CK(cudaEventRecord(ev1, st_));
    unsigned long long h[8];
    CK(cudaMemcpyAsync(h, ctrl_, sizeof(h), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    float dev_ms = 0;
    cudaEventElapsedTime(&dev_ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    CK(cudaGetLastError());
    if (h[3])
      Fail(SME_ERR_CUDA, std::string(h[3] & ENGINE_ERR_BOUNDS ? "device bounds check failed" : "") +
                             (h[3] & ENGINE_ERR_TIMEOUT ? " bulk-copy wait gave up" : "") + " (engine error flags " +
                             std::to_string(h[3]) + ")");
    RunResult r;
    r.count = prog_.enumerate ? h[2] : h[0];
    r.emitted = h[2];
    r.stats.algorithmic_bytes = h[1];
    r.stats.reuse_hits = h[5];
    r.stats.kernel_launches = launches_;
    r.stats.batches = batches_;
    r.stats.peak_device_bytes = A_.peak;
    r.stats.paths_processed = paths_;
    double phase[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (auto& e : events_) {
      float ms = 0;
      cudaEventElapsedTime(&ms, e.a, e.b);
      phase[e.phase] += ms;
      cudaEventDestroy(e.a);
      cudaEventDestroy(e.b);
    }
    events_.clear();
    for (int i = 0; i < 8; ++i) r.stats.phase_ms[i] = phase[i];
    // the intersection kernels: COMPUTE, COMPUTE_COUNT, COMPUTE_PATH_COUNT
    r.stats.kernel_ms = phase[kPhaseCompute] + phase[kPhaseComputeCount] + phase[kPhasePathCount];
    r.stats.device_ms = dev_ms;
    r.stats.hot_launches = hot_;
    r.stats.h2d_bytes = root_h2d_;
    r.stats.elapsed_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    A_.Release(mark);
    return r;
  }

 private:
  const Program& prog_;
  const DeviceGraph& g_;
  DeviceContext& ctx_;
  Arena& A_;
  cudaStream_t st_;
  uint32_t* out_;
  uint64_t cap_;
  int sms_ = 148;
  unsigned long long* ctrl_ = nullptr;  // [0] count [1] bytes [2] emitted [3] error flags [5] reuse hits
  uint64_t launches_ = 0, batches_ = 0, paths_ = 0, hot_ = 0, root_h2d_ = 0;
  const uint32_t* ext_cols_ = nullptr;
  uint64_t ext_bytes_ = 0;
  uint64_t* ext_off_ = nullptr;      // per vertex: list offset in the cache
  uint32_t* ext_cache_ = nullptr;    // device list cache
  uint64_t ext_cap_ = 0, ext_used_ = 0, ext_restarts_ = 0;

  // Loads, for the paths of Fb, the adjacency lists step `ds` intersects into
  // a device subgraph allocated in the current arena frame (it stays valid
  // while deeper levels use candidate sets that point into it).
  // The resident graph with its hub bitmaps (`use_bitmaps_` false: lists only).
  DGraph Resident() const {
    if (use_bitmaps_ && g_.hub_slot)
      return DGraph{g_.row_ptrs, g_.cols, g_.hub_slot, g_.bitmaps, g_.words, nullptr, g_.coarse, g_.cwords};
    return DGraph{g_.row_ptrs, g_.cols, nullptr, nullptr, 0, nullptr, nullptr, 0};
  }

  DGraph LoadSubgraph(const DFront& Fb, const DStep& ds) {
    if (!ext_cols_) return Resident();
    Timed tl = TimerStart();
    const size_t mark = A_.Mark();
    uint32_t* newids = (uint32_t*)A_.Alloc(std::max<size_t>((size_t)Fb.P * std::max<int>(ds.nconn, 1), 1) * 4);
    unsigned int* nnew = (unsigned int*)A_.Alloc(sizeof(unsigned int));
    uint64_t total = 0;
    uint32_t K = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      CK(cudaMemsetAsync(nnew, 0, sizeof(unsigned int), st_));
      k_ext_claim<<<Grid(Fb.P, 256), 256, 0, st_>>>(Fb, ds, g_.row_ptrs, ext_off_, newids, nnew);
      Launched();
      K = (uint32_t)ReadU32(nnew);
      if (K == 0) break;
      uint64_t* deg = (uint64_t*)A_.Alloc((size_t)K * 8);
      k_ext_newdeg<<<Grid(K, 256), 256, 0, st_>>>(newids, K, g_.row_ptrs, deg);
      Launched();
      Scan(deg, K);
      total = ReadU64(deg + K - 1);
      if (ext_used_ + total <= ext_cap_) {
        k_ext_place<<<Grid(K, 256), 256, 0, st_>>>(newids, K, deg, ext_used_, ext_off_);
        k_ext_gather<<<WarpGrid(K), WARP_BLOCK, 0, st_>>>(newids, K, g_.row_ptrs, ext_cols_, ext_off_, ext_cache_);
        launches_ += 2;
        ext_used_ += total;
        ext_bytes_ += total * 4;
        break;
      }
      if (attempt == 1)
        Fail(SME_ERR_OOM, "external mode: the lists one batch reads (" + std::to_string(total * 4) +
                              " bytes) exceed the device list cache (" + std::to_string(ext_cap_ * 4) + " bytes)");
      // the cache is full: start over with this batch's lists
      CK(cudaMemsetAsync(ext_off_, 0xff, (size_t)(g_.n + 1) * 8, st_));
      ext_used_ = 0;
      ++ext_restarts_;
    }
    A_.Release(mark);
    TimerStop(tl, kPhaseExternal);
    return DGraph{g_.row_ptrs, ext_cache_, nullptr, nullptr, 0, ext_off_, nullptr, 0};
  }

  uint64_t ReadU32(const unsigned int* d) {
    CK(cudaMemcpyAsync(ctx_.h_pinned, d, sizeof(unsigned int), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    return *reinterpret_cast<const unsigned int*>(ctx_.h_pinned);
  }

  // External mode: the device list cache takes about half of the arena that
  // is free when the run starts (the frontiers keep the rest).
  void AllocExternalCache() {
    ext_off_ = (uint64_t*)A_.Alloc((size_t)(g_.n + 1) * 8);
    CK(cudaMemsetAsync(ext_off_, 0xff, (size_t)(g_.n + 1) * 8, st_));
    const uint64_t bytes = std::max<uint64_t>(A_.Free() / 2, 1 << 20) & ~uint64_t(255);
    ext_cache_ = (uint32_t*)A_.Alloc(bytes);
    ext_cap_ = bytes / 4;
    ext_used_ = 0;
  }

  // Batch cost of an external step in frontier-budget units: the subgraph
  // bytes count against the list cache (cg scales them so that frontier
  // bytes / budget + list bytes / cache <= 1).
  double ExtListCost(uint64_t budget) const {
    return ext_cols_ && ext_cap_ ? 4.0 * (double)std::max<uint64_t>(budget, 1 << 20) / (double)(ext_cap_ * 4) : 0.0;
  }
  std::vector<Timed> events_;

  void Launched() { ++launches_; }

  unsigned Grid(uint64_t items, int per_block) const {
    uint64_t b = (items + per_block - 1) / per_block;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)sms_ * 16));
  }
  unsigned WarpGrid(uint64_t paths) const { return Grid(paths * 32, WARP_BLOCK); }

  // The order in which a count step takes its paths: grouped by the hub
  // slot of the step's last list vertex (the most recently materialised one,
  // which changes fastest along the frontier), or nullptr to keep the
  // frontier order (no bitmaps, a small frontier, no room, or turned off).
  const uint32_t* GroupByHub(const DFront& F, const DStep& ds) {
    if (!group_by_hub_ || !use_bitmaps_ || !g_.hub_slot || g_.nhubs == 0 || ds.nconn == 0 || F.P < (1u << 16))
      return nullptr;
    const uint32_t nb = g_.nhubs + 1;
    const size_t need = (size_t)F.P * 4 + (size_t)nb * 24 + (((size_t)nb + SCAN_TILE - 1) / SCAN_TILE) * 8 + 4096;
    if (A_.Free() < need + (16u << 20)) return nullptr;
    Timed to = TimerStart();
    const uint8_t kv = ds.conn[ds.nconn - 1];
    unsigned long long* cnt = (unsigned long long*)A_.Alloc((size_t)nb * 8);
    unsigned long long* incl = (unsigned long long*)A_.Alloc((size_t)nb * 8);
    unsigned long long* cur = (unsigned long long*)A_.Alloc((size_t)nb * 8);
    uint32_t* perm = (uint32_t*)A_.Alloc((size_t)F.P * 4);
    CK(cudaMemsetAsync(cnt, 0, (size_t)nb * 8, st_));
    k_hub_hist<<<Grid(F.P, 256), 256, 0, st_>>>(F, kv, g_.hub_slot, nb, cnt);
    CK(cudaMemcpyAsync(incl, cnt, (size_t)nb * 8, cudaMemcpyDeviceToDevice, st_));
    Scan(reinterpret_cast<uint64_t*>(incl), nb);
    k_hub_cursor<<<Grid(nb, 256), 256, 0, st_>>>(incl, cnt, nb, cur);
    k_hub_scatter<<<Grid(F.P, 256), 256, 0, st_>>>(F, kv, g_.hub_slot, nb, cur, perm);
    launches_ += 3;
    TimerStop(to, kPhaseOrganize);
    return perm;
  }

  // Window of k_compute_cta in dynamic shared memory (64 KiB: two CTAs of
  // 512 threads per SM), the attribute set once per device.
  template <int MODE>
  size_t CtaWindowBytes() {
    constexpr size_t kBytes = 64 << 10;
    // per device, once (server slots on several host threads may race here;
    // setting the attribute twice is harmless)
    static std::atomic<bool> set[64];
    const int d = ctx_.device;
    if (d >= 0 && d < 64 && !set[d].load(std::memory_order_acquire)) {
      CK(cudaFuncSetAttribute(k_compute_cta<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBytes));
      set[d].store(true, std::memory_order_release);
    }
    return kBytes;
  }

  template <int MODE, int MINB, int NLM>
  void LaunchWarp(bool ne, const DFront& F, const DStep& ds, const DGraph& G, const uint64_t* est, uint32_t b0,
                  uint64_t* ptr, uint32_t* cnt, uint32_t* data, uint64_t cap, unsigned long long* acc,
                  uint32_t* err) {
    if (ne)
      k_compute<MODE, MINB, NLM, MAXV><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(F, ds, G, est, b0, ptr, cnt, data,
                                                                             cap, acc, err, DHeavy{});
    else
      k_compute<MODE, MINB, NLM, 0><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(F, ds, G, est, b0, ptr, cnt, data, cap,
                                                                          acc, err, DHeavy{});
  }

  template <int MODE, int MINB, int NLM>
  void LaunchFlat(bool ne, const DFront& F, const DStep& ds, const DGraph& G, const uint64_t* est, uint32_t b0,
                  uint64_t* ptr, uint32_t* cnt, uint32_t* data, uint64_t cap, unsigned long long* acc,
                  uint32_t* err) {
    const unsigned grid = WarpGrid((F.P + 31) / 32);
    if (ne)
      k_compute_flat<MODE, MINB, NLM, MAXV><<<grid, WARP_BLOCK, 0, st_>>>(F, ds, G, est, b0, ptr, cnt, data, cap,
                                                                         acc, err);
    else
      k_compute_flat<MODE, MINB, NLM, 0><<<grid, WARP_BLOCK, 0, st_>>>(F, ds, G, est, b0, ptr, cnt, data, cap, acc,
                                                                      err);
  }

  // The root's list as a shared-memory bitmap (k_compute_rootmap), the
  // attribute for its dynamic shared memory set once per device.
  template <int MODE, int NEX>
  void LaunchRootMapAs(int ru, int other, const DFront& F, const DStep& ds, const DGraph& G, const uint64_t* est,
                       uint32_t b0, uint64_t* ptr, uint32_t* cnt, uint32_t* data, uint64_t cap,
                       unsigned long long* acc, uint32_t* err) {
    // per device, once (server slots on several host threads may race here;
    // setting the attribute twice is harmless)
    static std::atomic<bool> set[64];
    const int d = ctx_.device;
    if (d >= 0 && d < 64 && !set[d].load(std::memory_order_acquire)) {
      CK(cudaFuncSetAttribute(k_compute_rootmap<MODE, NEX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kRootMapMaxBytes));
      set[d].store(true, std::memory_order_release);
    }
    const uint32_t words = (uint32_t)((g_.n + 31) / 32);
    const size_t bytes = (size_t)words * 4;
    const size_t mark = A_.Mark();
    uint32_t* next = (uint32_t*)A_.Alloc(4);
    CK(cudaMemsetAsync(next, 0, 4, st_));
    // two CTAs of 1024 threads per SM while two bitmaps fit shared memory
    const uint64_t per_sm = bytes <= (112u << 10) ? 2 : 1;
    const unsigned grid =
        (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(sms_ * per_sm, (F.P + RM_CHUNK - 1) / RM_CHUNK));
    k_compute_rootmap<MODE, NEX><<<grid, RM_THREADS, bytes, st_>>>(F, ds, G, ru, other, est, b0, ptr, cnt, data,
                                                                    cap, acc, err, next, words);
    A_.Release(mark);
  }

  // Intersection launch: warp per path, specialised (granularity 0 auto, 3),
  // warp per path generic (1) or flattened over 32 paths per warp (2); in the
  // auto launches, a two-list step that reads the root's list takes
  // k_compute_rootmap (SME_ROOT_MAP=0 turns it off).
  template <int MODE>
  void Compute(const DFront& F, const DStep& ds, const DGraph& G, const uint64_t* est, uint32_t b0, uint64_t* ptr,
               uint32_t* cnt, uint32_t* data, uint64_t cap, const uint32_t* perm = nullptr) {
    unsigned long long* acc = ctrl_;
    uint32_t* err = (uint32_t*)(ctrl_ + 3);
    Timed t = TimerStart();
    const int gran = gran_;
    const int nlists = ds.nconn + (ds.reuse >= 0 ? 1 : 0);
    bool has_ne = false;
    for (int i = 0; i < ds.cond.n; ++i) has_ne |= ds.cond.op[i] == 2;
    const int ru = prog_.steps[0].u;
    int ri = -1;
    for (int i = 0; i < ds.nconn; ++i)
      if (ds.conn[i] == ru) ri = i;
    // the bitmap pays only where a root has many paths (its rebuild and the
    // CTA's barriers are per run of paths): three or more materialised
    // vertices (the 4-cycle's count step, not the diamond's or the
    // 4-clique's second level, measured 3.4x and 2.2x slower there)
    int nmat = 0;
    for (int v = 0; v < MAXV; ++v) nmat += F.inst[v] != nullptr;
    const bool rootmap = root_map_ && nmat >= 3 && !perm && ds.msrc < 0 && ds.reuse < 0 && ds.nconn == 2 && ri >= 0 &&
                         (gran == 0 || gran == 3) && (MODE != 1 || ds.with_u < 0) && !G.coff && g_.n > 0 &&
                         (g_.n + 31) / 32 * 4 <= kRootMapMaxBytes && F.inst[ru] && F.inst[ds.conn[1 - ri]];
    if (rootmap) {
      const int other = ds.conn[1 - ri];
      if (has_ne)
        LaunchRootMapAs<MODE, MAXV>(ru, other, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
      else
        LaunchRootMapAs<MODE, 0>(ru, other, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
    } else if (MODE == 1 && perm && ds.msrc < 0 && (gran == 0 || gran == 3) && nlists <= 3) {
      // count step, paths taken hub by hub (see k_hub_hist)
      if constexpr (MODE == 1) {
        DHeavy hv{};
        hv.perm = perm;
        if (nlists <= 2) {
          if (has_ne)
            k_compute<1, 8, 2, MAXV, false, false, true><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(
                F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, hv);
          else
            k_compute<1, 8, 2, 0, false, false, true><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(
                F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, hv);
        } else {
          if (has_ne)
            k_compute<1, 8, 3, MAXV, false, false, true><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(
                F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, hv);
          else
            k_compute<1, 8, 3, 0, false, false, true><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(
                F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, hv);
        }
      }
    } else if (ds.msrc >= 0) {
      // mapped reuse: the warp kernel that looks up the sibling's set
      if (has_ne)
        k_compute<MODE, 4, MAXV, MAXV, false, true><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(
            F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, DHeavy{});
      else
        k_compute<MODE, 4, MAXV, 0, false, true><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(
            F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, DHeavy{});
    } else if (gran == 4 && nlists == 2 && !has_ne) {
      // warp per path; paths with a long clipped pivot go to a CTA each
      const size_t mark = A_.Mark();
      const uint32_t qcap = (uint32_t)std::min<uint64_t>(F.P, 1u << 16);
      uint32_t* q = (uint32_t*)A_.Alloc(((size_t)qcap + 1) * 4);
      CK(cudaMemsetAsync(q, 0, 4, st_));
      k_compute<MODE, 8, 2, 0, true><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(
          F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, DHeavy{q, qcap, heavy_min_});
      Launched();
      const size_t win_bytes = CtaWindowBytes<MODE>();
      k_compute_cta<MODE><<<(unsigned)sms_ * 2, CTA_THREADS, win_bytes, st_>>>(
          F, ds, G, est, b0, ptr, cnt, data, cap, acc, err, q, qcap, (uint32_t)(win_bytes / 4));
      hot_ += 1;
      A_.Release(mark);
    } else if (gran == 0 || gran == 3 || gran == 4) {
      // warp per path, specialised on the number of intersected lists and
      // on the presence of `!=` conditions; fewer live values let more warps
      // reside, which is what counts: the searches are L2-latency bound.
      // Auto: eight blocks per SM for two or three lists, six otherwise
      // (measured fastest on every plan at R-MAT s20); 3: six throughout.
      const int nl = ds.nconn + (ds.reuse >= 0 ? 1 : 0);
      bool ne = false;
      for (int i = 0; i < ds.cond.n; ++i) ne |= ds.cond.op[i] == 2;
      const bool dense = gran != 3;
      if (nl <= 2)
        dense ? LaunchWarp<MODE, 8, 2>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err)
              : LaunchWarp<MODE, 6, 2>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
      else if (nl <= 3)
        dense ? LaunchWarp<MODE, 8, 3>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err)
              : LaunchWarp<MODE, 6, 3>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
      else
        LaunchWarp<MODE, 6, MAXV>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
    } else if (gran == 1) {
      k_compute<MODE><<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(F, ds, G, est, b0, ptr, cnt, data, cap, acc, err,
                                                             DHeavy{});
    } else {
      // flattened, specialised the same way
      const int nl = ds.nconn + (ds.reuse >= 0 ? 1 : 0);
      bool ne = false;
      for (int i = 0; i < ds.cond.n; ++i) ne |= ds.cond.op[i] == 2;
      if (nl <= 2)
        LaunchFlat<MODE, 8, 2>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
      else if (nl <= 3)
        LaunchFlat<MODE, 6, 3>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
      else
        LaunchFlat<MODE, 4, MAXV>(ne, F, ds, G, est, b0, ptr, cnt, data, cap, acc, err);
    }
    TimerStop(t, MODE == 0 ? kPhaseCompute : MODE == 1 ? kPhaseComputeCount : kPhasePathCount);
    Launched();
  }

 public:
  int gran_ = 0;
  uint32_t heavy_min_ = 2048;  // granularity 4: shortest pivot that gets a CTA
  bool group_by_hub_ = false;  // count steps take their paths hub by hub
  bool use_bitmaps_ = true;
  bool root_map_ = true;  // two-list steps on the root's list: k_compute_rootmap

 private:

  uint64_t Budget(size_t k) const {
    size_t rem = prog_.steps.size() - k + 1;
    return (uint64_t)((double)A_.Free() * 0.85 / (double)rem);
  }

  Timed TimerStart() {
    Timed e;
    cudaEventCreate(&e.a);
    cudaEventCreate(&e.b);
    cudaEventRecord(e.a, st_);
    e.phase = 0;
    return e;
  }
  // Records the end of a timed region of `phase` (sme_stats.phase_ms index).
  void TimerStop(Timed e, int phase) {
    cudaEventRecord(e.b, st_);
    e.phase = phase;
    events_.push_back(e);
    if (phase == kPhaseCompute || phase == kPhaseComputeCount || phase == kPhasePathCount) ++hot_;
  }

  void Scan(uint64_t* d, uint32_t n) {
    if (n == 0) return;
    uint32_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    size_t m = A_.Mark();
    uint64_t* bs = (uint64_t*)A_.Alloc((size_t)nb * 8);
    k_scan_reduce<<<nb, SCAN_THREADS, 0, st_>>>(d, n, bs);
    k_scan_partials<<<1, 1024, 0, st_>>>(bs, nb);
    k_scan_apply<<<nb, SCAN_THREADS, 0, st_>>>(d, n, bs);
    launches_ += 3;
    A_.Release(m);
  }

  uint64_t ReadU64(const uint64_t* d) {
    CK(cudaMemcpyAsync(ctx_.h_pinned, d, 8, cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    return ctx_.h_pinned[0];
  }

  struct Batch {
    uint32_t b0, b1;
    uint64_t e0, e1;  // inclusive estimate before b0 / at b1-1
  };

  std::vector<Batch> Split(const uint64_t* incl, uint32_t P, double pf, double cf, uint64_t budget,
                           const uint64_t* incl2 = nullptr, double cg = 0) {
    std::vector<Batch> out;
    if (P == 0) return out;
    budget = std::max<uint64_t>(budget, 1 << 20);
    const uint32_t K = (uint32_t)std::min<size_t>(ctx_.pinned_words / 2, 4096);
    size_t m = A_.Mark();
    uint64_t* d = (uint64_t*)A_.Alloc((size_t)K * 16);
    uint32_t start = 0;
    uint64_t e_start = 0;
    while (start < P) {
      k_split<<<(K + 255) / 256, 256, 0, st_>>>(incl, incl2, P, start, pf, cf, cg, (double)budget, K, d);
      Launched();
      CK(cudaMemcpyAsync(ctx_.h_pinned, d, (size_t)K * 16, cudaMemcpyDeviceToHost, st_));
      CK(cudaStreamSynchronize(st_));
      const uint64_t* h = ctx_.h_pinned;
      for (uint32_t k = 0; k < K && start < P; ++k) {
        uint32_t end = (uint32_t)std::min<uint64_t>(h[2 * k], P);
        if (end <= start) continue;
        uint64_t e_end = h[2 * k + 1];
        out.push_back(Batch{start, end, e_start, e_end});
        start = end;
        e_start = e_end;
      }
    }
    A_.Release(m);
    return out;
  }

  static DFront Slice(const DFront& F, uint32_t b0, uint32_t b1) {
    DFront G = F;
    G.P = b1 - b0;
    for (int v = 0; v < MAXV; ++v) {
      if (F.inst[v]) G.inst[v] = F.inst[v] + b0;
      if (F.cidx[v]) G.cidx[v] = F.cidx[v] + b0;
      else G.ident_off[v] = F.ident_off[v] + b0;
    }
    return G;
  }

  void Emit(const DFront& F) {
    uint8_t sl[MAXV] = {0, 0, 0, 0, 0, 0};
    for (int v = 0; v < prog_.n; ++v) sl[v] = prog_.out_slot[v];
    k_emit<<<Grid(F.P, 256), 256, 0, st_>>>(F, (uint8_t)prog_.n, nullptr, sl[0], sl[1], sl[2], sl[3],
                                            sl[4], sl[5], out_, cap_, ctrl_ + 2);
    Launched();
  }

  void Level(size_t k, const DFront& F) {
    if (F.P == 0) return;
    if (k == prog_.steps.size()) {
      if (prog_.enumerate) Emit(F);
      return;
    }
    const Step& s = prog_.steps[k];
    DStep ds = ToDStep(s);
    ds.noview = ext_cols_ != nullptr;
    unsigned long long* acc = ctrl_;
    uint32_t* err = (uint32_t*)(ctrl_ + 3);
    switch (s.kind) {
      case S_COMPUTE_COUNT: {
        paths_ += F.P;
        if (!ext_cols_) {
          const size_t mg = A_.Mark();
          const uint32_t* perm = GroupByHub(F, ds);
          Compute<1>(F, ds, Resident(), nullptr, 0, nullptr, nullptr, nullptr, 0, perm);
          A_.Release(mg);
          return;
        }
        // external: batches whose required lists fit the level budget
        const size_t m0 = A_.Mark();
        uint64_t* est = (uint64_t*)A_.Alloc((size_t)F.P * 8);
        uint64_t* sd = (uint64_t*)A_.Alloc((size_t)F.P * 8);
        k_est_compute<<<Grid(F.P, 256), 256, 0, st_>>>(F, ds, g_.row_ptrs, est, sd);
        Launched();
        Scan(sd, F.P);
        const uint64_t bk = Budget(k);
        std::vector<Batch> bs = Split(sd, F.P, 12.0, 0.0, bk, sd, ExtListCost(bk));
        for (const Batch& b : bs) {
          const size_t mk = A_.Mark();
          DFront Fb = Slice(F, b.b0, b.b1);
          ++batches_;
          DGraph gv = LoadSubgraph(Fb, ds);
          Compute<1>(Fb, ds, gv, nullptr, 0, nullptr, nullptr, nullptr, 0);
          A_.Release(mk);
        }
        A_.Release(m0);
        return;
      }
      case S_ALIAS: {
        DFront Fn = F;
        const int a = s.alias_of;
        Fn.set[s.u] = F.set[a];
        Fn.cidx[s.u] = F.cidx[a];
        Fn.ident_off[s.u] = F.ident_off[a];
        Fn.nset[s.u] = F.nset[a];
        Level(k + 1, Fn);
        return;
      }
      case S_COUNT: {
        Timed tc = TimerStart();
        if (s.direct) {
          uint8_t us[3] = {0, 0, 0};
          for (size_t i = 0; i < s.unmat.size() && i < 3; ++i) us[i] = s.unmat[i];
          k_count_direct<<<Grid(F.P, 256), 256, 0, st_>>>(F, (uint8_t)s.unmat.size(), us[0], us[1], us[2],
                                                          prog_.query_type, acc);
        } else if (s.unmat.size() == 1) {
          k_count1<<<Grid(F.P, 256), 256, 0, st_>>>(F, s.unmat[0], acc);
        } else {
          k_count2<<<WarpGrid(F.P), WARP_BLOCK, 0, st_>>>(F, s.unmat[0], s.unmat[1], s.pair_op, acc);
        }
        TimerStop(tc, kPhaseCount);
        Launched();
        return;
      }
      default:
        break;
    }
    const size_t mark0 = A_.Mark();
    uint64_t* est = (uint64_t*)A_.Alloc((size_t)F.P * 8);
    uint64_t* sumdeg = nullptr;  // external mode: subgraph bytes per path
    double pf = 0, cf = 0;
    Timed to = TimerStart();
    if (s.kind == S_COMPUTE || s.kind == S_PATH_COUNT) {
      if (ext_cols_) sumdeg = (uint64_t*)A_.Alloc((size_t)F.P * 8);
      k_est_compute<<<Grid(F.P, 256), 256, 0, st_>>>(F, ds, g_.row_ptrs, est, sumdeg);
      pf = 12 + 16;
      cf = s.kind == S_COMPUTE ? 4 : 0;
    } else {  // MATERIALIZE, FILTER
      k_est_set<<<Grid(F.P, 256), 256, 0, st_>>>(F, s.u, est);
      if (s.kind == S_FILTER) {
        pf = 12 + 16;
        cf = 4;
      } else {
        pf = 16;
        cf = 4.0 * (s.mat_after.size() + s.sets_after.size()) + 16;
      }
    }
    Launched();
    Scan(est, F.P);
    if (sumdeg) Scan(sumdeg, F.P);
    TimerStop(to, kPhaseOrganize);
    uint64_t budget = Budget(k);
    // keep child counts of a batch within 31-bit path indices
    budget = std::min<uint64_t>(budget, (uint64_t)(std::max(cf, 1.0) * 2.0e9));
    std::vector<Batch> batches = Split(est, F.P, pf, cf, budget, sumdeg, ExtListCost(budget));
    for (const Batch& b : batches) {
      const size_t mark = A_.Mark();
      DFront Fb = Slice(F, b.b0, b.b1);
      const uint32_t Pb = b.b1 - b.b0;
      ++batches_;
      switch (s.kind) {
        case S_COMPUTE:
        case S_PATH_COUNT: {
          paths_ += Pb;
          uint64_t* ptr = (uint64_t*)A_.Alloc((size_t)Pb * 8);
          uint32_t* cnt = (uint32_t*)A_.Alloc((size_t)Pb * 4);
          uint64_t cap = s.kind == S_COMPUTE ? b.e1 - b.e0 : 0;
          uint32_t* data = cap ? (uint32_t*)A_.Alloc(cap * 4) : nullptr;
          DGraph gv = LoadSubgraph(Fb, ds);
          if (s.kind == S_COMPUTE)
            Compute<0>(Fb, ds, gv, est, b.b0, ptr, cnt, data, cap);
          else
            Compute<2>(Fb, ds, gv, est, b.b0, ptr, cnt, nullptr, 0);
          DFront Fn = Fb;
          Fn.set[s.u] = DSet{ptr, cnt};
          Fn.nset[s.u] = Pb;
          Fn.cidx[s.u] = nullptr;
          Fn.ident_off[s.u] = 0;
          Level(k + 1, Fn);
          break;
        }
        case S_FILTER: {
          uint64_t* ptr = (uint64_t*)A_.Alloc((size_t)Pb * 8);
          uint32_t* cnt = (uint32_t*)A_.Alloc((size_t)Pb * 4);
          uint64_t cap = b.e1 - b.e0;
          uint32_t* data = cap ? (uint32_t*)A_.Alloc(cap * 4) : nullptr;
          Timed tf = TimerStart();
          k_filter<<<WarpGrid(Pb), WARP_BLOCK, 0, st_>>>(Fb, s.u, ToDCond(s.cond), est, b.b0, ptr, cnt, data,
                                                         cap, err);
          TimerStop(tf, kPhaseFilter);
          Launched();
          DFront Fn = Fb;
          Fn.set[s.u] = DSet{ptr, cnt};
          Fn.nset[s.u] = Pb;
          Fn.cidx[s.u] = nullptr;
          Fn.ident_off[s.u] = 0;
          Level(k + 1, Fn);
          break;
        }
        case S_MATERIALIZE: {
          DCond dc = ToDCond(s.cond);
          uint64_t* cnt = (uint64_t*)A_.Alloc((size_t)Pb * 8);
          Timed tm = TimerStart();
          k_mat_count<<<Grid(Pb, 256), 256, 0, st_>>>(Fb, s.u, dc, cnt);
          Launched();
          Scan(cnt, Pb);
          uint64_t C = ReadU64(cnt + Pb - 1);
          if (C == 0) break;
          if (C > 0x7fffffffULL) Fail(SME_ERR_OOM, "materialised batch exceeds 2^31 partial instances");
          DMatOut o{};
          o.u = s.u;
          o.keep = s.keep_set;
          o.nmat = (uint8_t)s.mat_after.size();
          for (size_t i = 0; i < s.mat_after.size(); ++i) {
            o.mat[i] = s.mat_after[i];
            o.inst[s.mat_after[i]] = (uint32_t*)A_.Alloc(C * 4);
          }
          o.nsets = (uint8_t)s.sets_after.size();
          for (size_t i = 0; i < s.sets_after.size(); ++i) {
            o.sets[i] = s.sets_after[i];
            o.cidx[s.sets_after[i]] = (uint32_t*)A_.Alloc(C * 4);
          }
          k_mat_write<<<WarpGrid(Pb), WARP_BLOCK, 0, st_>>>(Fb, dc, o, cnt, C, kMatBig, err);
          k_mat_write_big<<<WarpGrid((C + kMatChunk - 1) / kMatChunk), WARP_BLOCK, 0, st_>>>(Fb, dc, o, cnt, C,
                                                                                             kMatBig, err);
          Launched();
          TimerStop(tm, kPhaseMaterialize);
          Launched();
          DFront Fn{};
          Fn.P = (uint32_t)C;
          for (int v = 0; v < MAXV; ++v) Fn.inst[v] = o.inst[v];
          for (uint8_t w : s.sets_after) {
            Fn.set[w] = Fb.set[w];
            Fn.nset[w] = Fb.nset[w];
            Fn.cidx[w] = o.cidx[w];
          }
          Level(k + 1, Fn);
          break;
        }
        default:
          Fail(SME_ERR_INVALID_ARG, "unexpected step kind");
      }
      A_.Release(mark);
    }
    A_.Release(mark0);
  }
};

}  // namespace

RunResult RunProgram(const Program& prog, const DeviceGraph& g, DeviceContext& ctx, const RootTask& task,
                     uint32_t* d_out, uint64_t cap, int tuning) {
  CK(cudaSetDevice(ctx.device));
  RootTask t = task;
  if (!t.list) {
    if (t.end > g.n) t.end = g.n;
    if (t.begin > t.end) t.begin = t.end;
  }
  Executor ex(prog, g, ctx, d_out, cap);
  ex.gran_ = tuning & 0xff;
  ex.use_bitmaps_ = !(tuning & 0x100);
  if (const char* e = std::getenv("SME_HEAVY_PIVOT")) ex.heavy_min_ = (uint32_t)std::max(32L, std::atol(e));
  if (const char* e = std::getenv("SME_GROUP_BY_HUB")) ex.group_by_hub_ = std::atoi(e) != 0;
  if (const char* e = std::getenv("SME_ROOT_MAP")) ex.root_map_ = std::atoi(e) != 0;
  return ex.Run(t);
}

// EXTERNAL_GPU: the graph stays in host memory.
//   EXT_CACHE  global row pointers on the device; for every intersection
//              batch, the required adjacency lists are gathered by the GPU
//              from pinned, mapped host memory into a device subgraph
//              (EXTLIGHTGPUProcessor::PrepareBatch/LoadSubgraph,
//              src/gpu/impl/light/ext/EXTLIGHTGPUProcessor.cuh:20-90).
//   EXT_UMA    the adjacency lists live in managed memory and migrate on
//              demand (EXTUMALIGHTGPUComp, src/gpu/impl/light/ext/uma/).
RunResult RunProgramExternal(const Program& prog, const HostGraph& hg, DeviceContext& ctx, const RootTask& task,
                             int ext_variant, uint64_t graph_budget_bytes) {
  (void)graph_budget_bytes;
  CK(cudaSetDevice(ctx.device));
  RootTask t = task;
  if (!t.list) {
    if (t.end > hg.n) t.end = hg.n;
    if (t.begin > t.end) t.begin = t.end;
  }
  DeviceGraph dg;
  dg.device = ctx.device;
  dg.n = hg.n;
  dg.m = hg.m;
  uint64_t h2d = (hg.n + 1) * sizeof(uintE);
  CK(cudaMalloc((void**)&dg.row_ptrs, (hg.n + 1) * sizeof(uintE)));
  RunResult r;
  bool registered = false;
  uint32_t* managed = nullptr;
  try {
    CK(cudaMemcpyAsync(dg.row_ptrs, hg.row_ptrs, (hg.n + 1) * sizeof(uintE), cudaMemcpyHostToDevice, ctx.stream));
    if (ext_variant == SME_EXT_UMA) {
      CK(cudaMallocManaged((void**)&managed, std::max<uint64_t>(hg.m, 1) * sizeof(uintV)));
      if (hg.m) std::memcpy(managed, hg.cols, hg.m * sizeof(uintV));
      dg.cols = managed;
      Executor ex(prog, dg, ctx, nullptr, 0);
      r = ex.Run(t);
      h2d += hg.m * sizeof(uintV);
    } else {
      const uint32_t* dcols = nullptr;
      if (hg.m) {
        cudaError_t e = cudaHostRegister(hg.cols, hg.m * sizeof(uintV), cudaHostRegisterMapped | cudaHostRegisterReadOnly);
        if (e == cudaSuccess) {
          registered = true;
        } else if (e == cudaErrorHostMemoryAlreadyRegistered) {
          cudaGetLastError();
        } else {
          Fail(SME_ERR_CUDA, std::string("cudaHostRegister: ") + cudaGetErrorString(e));
        }
        CK(cudaHostGetDevicePointer((void**)&dcols, hg.cols, 0));
      }
      Executor ex(prog, dg, ctx, nullptr, 0);
      ex.SetExternal(dcols);
      r = ex.Run(t);
      h2d += ex.ext_h2d_bytes();
    }
  } catch (...) {
    cudaStreamSynchronize(ctx.stream);
    if (registered) cudaHostUnregister(hg.cols);
    if (managed) cudaFree(managed);
    cudaFree(dg.row_ptrs);
    throw;
  }
  if (registered) cudaHostUnregister(hg.cols);
  if (managed) cudaFree(managed);
  cudaFree(dg.row_ptrs);
  r.stats.h2d_bytes += h2d;
  return r;
}

}  // namespace sme
