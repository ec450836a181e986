// Packed adjacency lists for uploads over the host link (sme_graph_pack).
//
// A graph that is not resident on the device is copied into the call's arena
// on every call, and its uint32 lists are nearly all of those bytes.  The
// packed copy (format in sme_internal.h, PackedLists) stores each list as
// deltas in blocks of 32 with one bit width per block: on R-MAT graphs about
// 0.41x the bytes of the lists.  The device expands it (k_unpack_lists,
// engine.cu) at HBM speed after the copy.  No reference counterpart: the
// reference copies the uint32 CSR (CSRGraph::ToGPU via cudaMemcpy).
#include <algorithm>
#include <cstdlib>

#include <cuda_runtime.h>

#include "sme_internal.h"

namespace sme {

namespace {

inline uint32_t BitWidth(uint32_t x) { return x ? 32u - (uint32_t)__builtin_clz(x) : 0u; }

inline uint32_t Delta(const uintV* c, uint64_t i) { return i ? c[i] - c[i - 1] : c[0]; }

inline uint32_t BlockWidth(const uintV* c, uint64_t b, uint64_t e) {
  uint32_t w = 0;
  for (uint64_t i = b; i < e; ++i) w = std::max(w, BitWidth(Delta(c, i)));
  return w;
}

inline uint64_t Segments(uint64_t d) { return (d + kPackSegment - 1) / kPackSegment; }

// Bytes of one packed list (before the 4-byte alignment of the next list).
uint64_t ListBytes(const uintV* c, uint64_t d) {
  const uint64_t S = Segments(d);
  uint64_t bytes = S ? 8 * (S - 1) : 0;
  for (uint64_t e = 0; e < d; e += 32) {
    const uint64_t cnt = std::min<uint64_t>(32, d - e);
    bytes += 1 + (cnt * BlockWidth(c, e, e + cnt) + 7) / 8;
  }
  return bytes;
}

// Writes one packed list at `out`; returns the bytes written (== ListBytes).
uint64_t WriteList(const uintV* c, uint64_t d, uint8_t* out) {
  const uint64_t S = Segments(d);
  uint8_t* p = out + (S ? 8 * (S - 1) : 0);
  for (uint64_t s = 0; s < S; ++s) {
    const uint64_t e0 = s * kPackSegment, ne = std::min<uint64_t>(kPackSegment, d - e0);
    const uint64_t nb = (ne + 31) / 32;
    if (s > 0) {
      uint32_t entry[2] = {c[e0 - 1], (uint32_t)(p - out)};
      std::memcpy(out + 8 * (s - 1), entry, 8);
    }
    uint8_t* widths = p;
    p += nb;
    for (uint64_t b = 0; b < nb; ++b) {
      const uint64_t lo = e0 + 32 * b, hi = std::min<uint64_t>(lo + 32, e0 + ne);
      const uint32_t w = BlockWidth(c, lo, hi);
      widths[b] = (uint8_t)w;
      if (w == 0) continue;
      uint64_t acc = 0;
      uint32_t bits = 0;
      for (uint64_t i = lo; i < hi; ++i) {
        acc |= (uint64_t)Delta(c, i) << bits;
        bits += w;
        while (bits >= 8) {
          *p++ = (uint8_t)acc;
          acc >>= 8;
          bits -= 8;
        }
      }
      if (bits) *p++ = (uint8_t)acc;
    }
  }
  return (uint64_t)(p - out);
}

}  // namespace

PackedLists::~PackedLists() {
  if (!base) return;
  if (pinned)
    cudaFreeHost(base);
  else
    std::free(base);
}

std::shared_ptr<const PackedLists> PackLists(const HostGraph& g) {
  const uint64_t n = g.n;
  std::vector<uint64_t> at(n + 1, 0);  // byte start of each list, 4-byte aligned
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)n; ++u)
    at[u + 1] = (ListBytes(g.cols + g.row_ptrs[u], g.row_ptrs[u + 1] - g.row_ptrs[u]) + 3) & ~uint64_t(3);
  for (uint64_t u = 0; u < n; ++u) {
    if (at[u + 1] > UINT32_MAX) Fail(SME_ERR_INVALID_ARG, "a packed list exceeds 4 GiB; upload the plain CSR");
    at[u + 1] += at[u];
  }
  const uint64_t stream_bytes = at[n] + 8;
  if (at[n] / 4 > UINT32_MAX)
    Fail(SME_ERR_INVALID_ARG, "packed lists exceed 16 GiB; upload the plain CSR");
  uint64_t nsegs = 0;
  for (uint64_t u = 0; u < n; ++u) {
    const uint64_t S = Segments(g.row_ptrs[u + 1] - g.row_ptrs[u]);
    nsegs += S ? S - 1 : 0;
  }

  auto pk = std::make_shared<PackedLists>();
  pk->n = n;
  pk->m = g.m;
  pk->nsegs = nsegs;
  pk->deg_at = 0;
  pk->woff_at = 4 * n;
  pk->segs_at = (8 * n + 7) & ~uint64_t(7);
  pk->stream_at = (pk->segs_at + 8 * nsegs + 15) & ~uint64_t(15);
  pk->stream_bytes = stream_bytes;
  pk->total = pk->stream_at + stream_bytes;
  // pinned, so the upload is one DMA at link speed; plain memory where no
  // device is present (the copy then stages through the driver)
  if (cudaMallocHost((void**)&pk->base, pk->total) == cudaSuccess) {
    pk->pinned = true;
  } else {
    cudaGetLastError();
    pk->base = (uint8_t*)std::malloc(pk->total);
    if (!pk->base) Fail(SME_ERR_OOM, "cannot allocate the packed lists");
  }
  uint32_t* deg = (uint32_t*)(pk->base + pk->deg_at);
  uint32_t* woff = (uint32_t*)(pk->base + pk->woff_at);
  uint64_t* segs = (uint64_t*)(pk->base + pk->segs_at);
  uint8_t* stream = pk->base + pk->stream_at;
  std::memset(pk->base + pk->woff_at + 4 * n, 0, pk->segs_at - (pk->woff_at + 4 * n));
  std::memset(pk->base + pk->segs_at + 8 * nsegs, 0, pk->stream_at - (pk->segs_at + 8 * nsegs));
  std::memset(stream + at[n], 0, 8);
  uint64_t k = 0;
  for (uint64_t u = 0; u < n; ++u) {
    const uint64_t d = g.row_ptrs[u + 1] - g.row_ptrs[u];
    if (d > UINT32_MAX) Fail(SME_ERR_INVALID_ARG, "a list longer than 2^32 - 1 cannot be packed");
    deg[u] = (uint32_t)d;
    woff[u] = (uint32_t)(at[u] / 4);
    for (uint64_t s = 1; s < Segments(d); ++s) segs[k++] = ((uint64_t)u << 32) | s;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)n; ++u) {
    uint8_t* out = stream + at[u];
    const uint64_t w = WriteList(g.cols + g.row_ptrs[u], g.row_ptrs[u + 1] - g.row_ptrs[u], out);
    std::memset(out + w, 0, at[u + 1] - at[u] - w);  // alignment padding
  }
  return pk;
}

}  // namespace sme
