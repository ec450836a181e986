// Device kernels of the enumeration engine (sm_100a, integer SIMT).
//
// A level frontier is a set of partial instances ("paths").  For each
// pattern vertex it holds either a materialised column (one data vertex per
// path) or a candidate set per path.  Candidate sets are (pointer, count)
// pairs: the pointer is an absolute device address, so a set can be a
// sub-range of an adjacency list or of a parent's set (zero copy) or live in
// a level's own data buffer.
#pragma once

#include <cstdint>

namespace sme {
namespace dev {

constexpr int MAXV = 6;  // kMaxQueryVerticesNum, src/Meta.h:30
constexpr unsigned FULL = 0xffffffffu;
constexpr int WARP_BLOCK = 256;  // threads per block of warp-per-path kernels
constexpr uint32_t ENGINE_ERR_BOUNDS = 1u;   // a write would leave its buffer
constexpr uint32_t ENGINE_ERR_TIMEOUT = 2u;  // a bounded wait on a bulk copy gave up

// Paths whose clipped pivot is long are handed from the warp-per-path
// intersection to a CTA per path: `q[0]` counts the deferred paths, their
// indices follow (at most `cap`); a path that finds the queue full stays
// with its warp.  q == nullptr: nothing is deferred.
struct DHeavy {
  uint32_t* q;
  uint32_t cap;
  uint32_t min_len;
  // PERM launches: the order in which the paths are taken (path i of the
  // launch is perm[i]); a count is the same in any order
  const uint32_t* perm;
};

struct DSet {
  const uint64_t* ptr;  // absolute device address of the first element
  const uint32_t* cnt;
};

struct DFront {
  uint32_t P;                     // paths in this view
  const uint32_t* inst[MAXV];     // materialised columns (null if none)
  const uint32_t* cidx[MAXV];     // set index per path (null: identity)
  uint32_t ident_off[MAXV];       // identity index offset (after slicing)
  DSet set[MAXV];                 // candidate-set stores
  uint32_t nset[MAXV];            // sets in each store
};

struct DCond {
  uint8_t n;
  uint8_t op[MAXV];       // 0 <, 1 >, 2 !=
  uint8_t operand[MAXV];  // materialised pattern vertex
};

struct DStep {
  uint8_t u;
  uint8_t nconn;
  uint8_t conn[MAXV];
  int8_t reuse;   // vertex whose candidate set joins the intersection
  DCond cond;
  int8_t with_u;  // COMPUTE_COUNT rank partner (-1 none)
  uint8_t with_op;
  // reuse plan, a mapped reuse meta: the sibling path (M[0], M[mx]) of the
  // current path's level-1 ancestor holds, in the cached store of vertex
  // msrc, the intersection that replaces the lists conn[i] with bit i of
  // mmask set (msrc < 0: none)
  int8_t msrc;
  uint8_t mx;
  uint8_t mmask;
  uint8_t mop;  // level 1's order against M[0] the sibling's vertex obeys (0 <, 1 >, else none)
  // 1: a single-list set is copied, never a view into the list (external
  // mode: the list cache is reused by later batches while the set lives on)
  uint8_t noview;
};

struct DMatOut {
  uint32_t* inst[MAXV];
  uint32_t* cidx[MAXV];
  uint8_t nmat, mat[MAXV];
  uint8_t nsets, sets[MAXV];
  uint8_t u;
  uint8_t keep;
};

// Graph as seen by the intersection kernels.  Vertices of the highest degree
// also have a dense adjacency bitmap (`words` uint32 per hub): membership in
// their lists is one load instead of a binary search over a long list.
struct DGraph {
  const uint64_t* rp;
  const uint32_t* cols;
  const int32_t* hub;  // hub slot per vertex, -1 none; null: no bitmaps
  const uint32_t* bm;
  uint32_t words;
  // external mode: the lists live in a device cache; coff[v] is v's first
  // element in `cols` (null: cols is the CSR and rp indexes it)
  const uint64_t* coff;
  // per hub, one bit per 32-vertex block of its bitmap (null: none)
  const uint32_t* cbm;
  uint32_t cwords;
};

// Adjacency list of v: its first element and length.
__device__ __forceinline__ void AdjList(const DGraph& g, uint32_t v, const uint32_t*& ptr, uint32_t& len) {
  const uint64_t b = __ldg(g.rp + v);
  len = (uint32_t)(__ldg(g.rp + v + 1) - b);
  ptr = g.cols + (g.coff ? (len ? __ldg(g.coff + v) : 0) : b);
}

__device__ __forceinline__ const uint32_t* HubBitmap(const DGraph& g, uint32_t v) {
  if (!g.hub) return nullptr;
  int32_t s = __ldg(g.hub + v);
  return s < 0 ? nullptr : g.bm + (size_t)s * g.words;
}

__device__ __forceinline__ bool BitTest(const uint32_t* bm, uint32_t x) {
  return (__ldg(bm + (x >> 5)) >> (x & 31)) & 1u;
}

// The coarse bitmap of v (null: v is no hub, or none was built).
__device__ __forceinline__ const uint32_t* HubCoarse(const DGraph& g, uint32_t v) {
  if (!g.hub || !g.cbm) return nullptr;
  int32_t s = __ldg(g.hub + v);
  return s < 0 ? nullptr : g.cbm + (size_t)s * g.cwords;
}

// Membership in a hub's list: the coarse bit of x's 32-vertex block first
// (the coarse bitmaps are small enough to stay in L2), the bitmap word only
// when the block holds a neighbour.
__device__ __forceinline__ bool BitTest2(const uint32_t* bm, const uint32_t* coarse, uint32_t x) {
  if (coarse && !((__ldg(coarse + (x >> 10)) >> ((x >> 5) & 31)) & 1u)) return false;
  return BitTest(bm, x);
}

__device__ __forceinline__ uint32_t SetIndex(const DFront& F, int u, uint32_t p) {
  const uint32_t* c = F.cidx[u];
  return c ? c[p] : p + F.ident_off[u];
}

__device__ __forceinline__ void GetSet(const DFront& F, int u, uint32_t p, const uint32_t*& ptr,
                                       uint32_t& len) {
  uint32_t s = SetIndex(F, u, p);
  ptr = reinterpret_cast<const uint32_t*>(F.set[u].ptr[s]);
  len = F.set[u].cnt[s];
}

// First index i in a[0,n) with a[i] >= x (GpuUtils::BinSearch::BinSearch,
// src/gpu/utils/ops/GPUBinSearch.cuh:18-31), written with a select instead
// of a branch in the loop (the branch-free lower bound of Khuong and Morin,
// "Array layouts for comparison-based searching", 2017): lanes searching
// different values do not diverge inside the loop (2-4% on the count steps).
__device__ __forceinline__ uint32_t LowerBound(const uint32_t* __restrict__ a, uint32_t n, uint32_t x) {
  if (n == 0) return 0;
  const uint32_t* base = a;
  while (n > 1) {
    const uint32_t half = n >> 1;
    base = __ldg(base + half) < x ? base + half : base;
    n -= half;
  }
  return (uint32_t)(base - a) + (__ldg(base) < x ? 1u : 0u);
}

// Conditions of a candidate against materialised vertices reduce, on a sorted
// list, to an interval [lo, hi) minus up to NE excluded values.  NE = 0 is
// for steps whose conditions hold no `!=` (the caller checks): the exclusion
// array then takes no registers.
template <int NE>
struct BoundsT {
  uint64_t lo, hi;
  uint32_t ne[NE > 0 ? NE : 1];
  int nne;
};
using Bounds = BoundsT<MAXV>;

template <int NE = MAXV>
__device__ __forceinline__ BoundsT<NE> MakeBounds(const DCond& c, const DFront& F, uint32_t p) {
  static_assert(NE == 0 || NE == MAXV, "exclusion slots: none or one per condition");
  BoundsT<NE> b;
  b.lo = 0;
  b.hi = 1ULL << 32;
  b.nne = 0;
#pragma unroll
  for (int i = 0; i < MAXV; ++i) {
    if (i < c.n) {
      uint32_t v = F.inst[c.operand[i]][p];
      if (c.op[i] == 0) {
        b.hi = min(b.hi, (uint64_t)v);
      } else if (c.op[i] == 1) {
        b.lo = max(b.lo, (uint64_t)v + 1);
      } else if (NE > 0) {
        b.ne[b.nne++] = v;
      }
    }
  }
  return b;
}

template <int NE>
__device__ __forceinline__ void Range(const uint32_t* a, uint32_t n, const BoundsT<NE>& b, uint32_t& r0,
                                      uint32_t& r1) {
  if (b.lo >= b.hi) {
    r0 = r1 = 0;
    return;
  }
  r0 = b.lo == 0 ? 0 : (b.lo > 0xffffffffULL ? n : LowerBound(a, n, (uint32_t)b.lo));
  r1 = b.hi > 0xffffffffULL ? n : LowerBound(a, n, (uint32_t)b.hi);
  if (r1 < r0) r1 = r0;
}

// First index i in a[0,n) with a[i] >= x, found by the whole warp (every lane
// calls it with the same arguments): each round the 32 lanes probe 32 evenly
// spaced elements and a ballot narrows the range 32-fold, so a list of up to
// 1024 elements takes two dependent rounds instead of ten loads in a row.
__device__ __forceinline__ uint32_t WarpLowerBound(const uint32_t* __restrict__ a, uint32_t n, uint32_t x) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t lo = 0, len = n;  // the answer lies in [lo, lo + len]
  while (len > 32) {
    const uint32_t step = (len + 31) / 32;
    const uint32_t idx = lo + lane * step;
    const bool lt = idx < lo + len && __ldg(a + idx) < x;
    const uint32_t c = __popc(__ballot_sync(0xffffffffu, lt));  // samples below x: a prefix
    if (c == 0) return lo;
    const uint32_t nlo = lo + (c - 1) * step + 1;
    const uint32_t nhi = min(lo + c * step, lo + len);
    lo = nlo;
    len = nhi - nlo;
  }
  const bool lt = lane < len && __ldg(a + lo + lane) < x;
  return lo + __popc(__ballot_sync(0xffffffffu, lt));
}

// Range with the warp's lower bound (same result; warp-uniform arguments).
template <int NE>
__device__ __forceinline__ void WarpRange(const uint32_t* a, uint32_t n, const BoundsT<NE>& b, uint32_t& r0,
                                          uint32_t& r1) {
  if (b.lo >= b.hi) {
    r0 = r1 = 0;
    return;
  }
  r0 = b.lo == 0 ? 0 : (b.lo > 0xffffffffULL ? n : WarpLowerBound(a, n, (uint32_t)b.lo));
  r1 = b.hi > 0xffffffffULL ? n : WarpLowerBound(a, n, (uint32_t)b.hi);
  if (r1 < r0) r1 = r0;
}

// Positions (ascending) of excluded values present in a[r0,r1).
template <int NE>
__device__ __forceinline__ int Exclusions(const uint32_t* a, uint32_t r0, uint32_t r1, const BoundsT<NE>& b,
                                          uint32_t* ex) {
  int k = 0;
#pragma unroll
  for (int i = 0; i < NE; ++i) {
    if (i < b.nne) {
      uint32_t pos = r0 + LowerBound(a + r0, r1 - r0, b.ne[i]);
      if (pos < r1 && __ldg(a + pos) == b.ne[i]) ex[k++] = pos;
    }
  }
  for (int i = 1; i < k; ++i)  // insertion sort, k <= MAXV
    for (int j = i; j > 0 && ex[j - 1] > ex[j]; --j) {
      uint32_t t = ex[j];
      ex[j] = ex[j - 1];
      ex[j - 1] = t;
    }
  return k;
}

// Count of elements y of sorted s[0,n) with (x op y); op as CondOperator
// (ThreadCountWithComputedVertex, src/gpu/impl/common/CheckConstraintsCommon.cuh:131-155).
__device__ __forceinline__ uint64_t RankCount(const uint32_t* s, uint32_t n, uint32_t x, uint8_t op) {
  if (n == 0) return 0;
  uint32_t pos = LowerBound(s, n, x);
  bool eq = pos < n && __ldg(s + pos) == x;
  if (op == 0) return n - pos - (eq ? 1 : 0);  // x < y
  if (op == 1) return pos;                     // x > y
  return n - (eq ? 1 : 0);                     // x != y
}

__device__ __forceinline__ unsigned long long WarpSum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
  return v;
}

}  // namespace dev
}  // namespace sme
