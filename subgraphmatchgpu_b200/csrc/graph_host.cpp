// Host CSR graphs: the BIN/SNAP formats, the preprocessing step and the seeded
// synthetic generators.
//
// Format and semantics follow the reference's graph layer:
//   BIN read/write   src/graph/GraphIO.h:88-136, :356-387
//   SNAP read        src/graph/GraphIO.h:195-270 (+ SortCSRArray :437-450)
//   preprocess       src/preprocess/PreprocessGraph.h:13-95
//   validate         src/graph/GraphIO.h:459-485
// The reader does one bulk read per array instead of one fread per element.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <unordered_map>

#include "sme_internal.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace sme {

uint64_t HostGraph::MaxDegree() const {
  uint64_t d = 0;
  for (uint64_t u = 0; u < n; ++u) d = std::max<uint64_t>(d, row_ptrs[u + 1] - row_ptrs[u]);
  return d;
}

bool HostGraph::LoopFree() const {
  int f = loop_free.load(std::memory_order_relaxed);
  if (f < 0) {
    uint64_t loops = 0;
    // a thread team only for large graphs: server workers call this for
    // every attached graph, and teams spawned from several workers at once
    // oversubscribe the host
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : loops) if (m > (1ULL << 22))
    for (uint64_t u = 0; u < n; ++u)
      for (uintE j = row_ptrs[u]; j < row_ptrs[u + 1]; ++j) loops += cols[j] == u;
    f = loops == 0 ? 1 : 0;
    loop_free.store(f, std::memory_order_relaxed);
  }
  return f == 1;
}

std::shared_ptr<const std::vector<uint32_t>> HostGraph::HubSelection(uint64_t min_degree, uint64_t max_hubs) const {
  std::lock_guard<std::mutex> lock(hub_mu_);
  if (hub_sel_ && hub_sel_min_ == min_degree && hub_sel_max_ == max_hubs) return hub_sel_;
  std::vector<std::pair<uint64_t, uint32_t>> cand;
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t deg = row_ptrs[u + 1] - row_ptrs[u];
    if (deg >= min_degree) cand.emplace_back(deg, (uint32_t)u);
  }
  std::sort(cand.begin(), cand.end(), [](const std::pair<uint64_t, uint32_t>& a,
                                         const std::pair<uint64_t, uint32_t>& b) {
    return a.first != b.first ? a.first > b.first : a.second < b.second;
  });
  if (cand.size() > max_hubs) cand.resize(max_hubs);
  auto sel = std::make_shared<std::vector<uint32_t>>(cand.size());
  for (size_t i = 0; i < cand.size(); ++i) (*sel)[i] = cand[i].second;
  std::sort(sel->begin(), sel->end());
  hub_sel_ = sel;
  hub_sel_min_ = min_degree;
  hub_sel_max_ = max_hubs;
  return hub_sel_;
}

void HostGraph::Adopt(std::vector<uintE>&& r, std::vector<uintV>&& c) {
  loop_free.store(-1, std::memory_order_relaxed);
  packed.reset();
  {
    std::lock_guard<std::mutex> lock(hub_mu_);
    hub_sel_.reset();
  }
  row_store = std::move(r);
  col_store = std::move(c);
  n = row_store.empty() ? 0 : row_store.size() - 1;
  m = col_store.size();
  if (row_store.empty()) row_store.assign(1, 0);
  row_ptrs = row_store.data();
  cols = col_store.data();
  borrowed = false;
}

// ------------------------------------------------------------------- BIN --
void ReadBinFile(const std::string& path, HostGraph& g) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) Fail(SME_ERR_BAD_FILE, "cannot open " + path);
  uint64_t hdr[4];
  if (std::fread(hdr, sizeof(uint64_t), 4, f) != 4) {
    std::fclose(f);
    Fail(SME_ERR_BAD_FILE, "truncated BIN header: " + path);
  }
  if (hdr[0] != sizeof(uintV) || hdr[1] != sizeof(uintE)) {
    std::fclose(f);
    Fail(SME_ERR_BAD_FILE, "BIN header has uintV_size/uintE_size " +
                               std::to_string(hdr[0]) + "/" + std::to_string(hdr[1]) +
                               ", expected 4/8: " + path);
  }
  const uint64_t n = hdr[2], m = hdr[3];
  std::fseek(f, 0, SEEK_END);
  const long long fsize = std::ftell(f);
  const long long want = 32LL + 8LL * (long long)(n + 1) + 4LL * (long long)m;
  if (n > (1ULL << 32) || fsize != want) {
    std::fclose(f);
    Fail(SME_ERR_BAD_FILE, "BIN size mismatch: file has " + std::to_string(fsize) +
                               " bytes, header implies " + std::to_string(want) + ": " + path);
  }
  std::fseek(f, 32, SEEK_SET);
  std::vector<uintE> r(n + 1);
  std::vector<uintV> c(m);
  bool ok = std::fread(r.data(), sizeof(uintE), n + 1, f) == n + 1 &&
            (m == 0 || std::fread(c.data(), sizeof(uintV), m, f) == m);
  std::fclose(f);
  if (!ok) Fail(SME_ERR_BAD_FILE, "short read: " + path);
  if (r[0] != 0 || r[n] != m) Fail(SME_ERR_BAD_FILE, "row_ptrs do not span cols: " + path);
  for (uint64_t u = 0; u < n; ++u)
    if (r[u] > r[u + 1]) Fail(SME_ERR_BAD_FILE, "row_ptrs not monotone: " + path);
  for (uint64_t j = 0; j < m; ++j)
    if (c[j] >= n) Fail(SME_ERR_BAD_FILE, "column id out of range: " + path);
  g.Adopt(std::move(r), std::move(c));
}

void WriteBinFile(const std::string& path, const HostGraph& g) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) Fail(SME_ERR_BAD_FILE, "cannot create " + path);
  uint64_t hdr[4] = {sizeof(uintV), sizeof(uintE), g.n, g.m};
  bool ok = std::fwrite(hdr, sizeof(uint64_t), 4, f) == 4 &&
            std::fwrite(g.row_ptrs, sizeof(uintE), g.n + 1, f) == g.n + 1 &&
            (g.m == 0 || std::fwrite(g.cols, sizeof(uintV), g.m, f) == g.m);
  if (std::fclose(f) != 0) ok = false;
  if (!ok) Fail(SME_ERR_BAD_FILE, "write failed: " + path);
}

// ------------------------------------------------------------------ SNAP --
static void SortLists(uint64_t n, const uintE* r, uintV* c) {
#pragma omp parallel for schedule(dynamic, 1024)
  for (long long u = 0; u < (long long)n; ++u) std::sort(c + r[u], c + r[u + 1]);
}

void ReadSnapFile(const std::string& path, bool directed, HostGraph& g) {
  std::ifstream in(path);
  if (!in) Fail(SME_ERR_BAD_FILE, "cannot open " + path);
  std::vector<std::pair<uintV, uintV>> e;
  std::string line;
  uintV lo = UINT32_MAX, hi = 0;
  while (std::getline(in, line)) {
    if (line.empty() || !std::isdigit((unsigned char)line[0])) continue;
    std::istringstream iss(line);
    unsigned long long a, b;
    if (!(iss >> a >> b) || a > UINT32_MAX || b > UINT32_MAX)
      Fail(SME_ERR_BAD_FILE, "malformed edge line in " + path + ": " + line);
    e.emplace_back((uintV)a, (uintV)b);
    lo = std::min(lo, (uintV)std::min(a, b));
    hi = std::max(hi, (uintV)std::max(a, b));
  }
  if (e.empty()) {
    g.Adopt(std::vector<uintE>(1, 0), std::vector<uintV>());
    return;
  }
  const uint64_t n = (uint64_t)hi - lo + 1;
  std::vector<uintE> r(n + 1, 0);
  for (auto& p : e) {
    p.first -= lo;
    p.second -= lo;
    r[p.first + 1]++;
    if (!directed) r[p.second + 1]++;
  }
  for (uint64_t u = 0; u < n; ++u) r[u + 1] += r[u];
  std::vector<uintV> c(r[n]);
  std::vector<uintE> pos(r.begin(), r.end() - 1);
  for (auto& p : e) {
    c[pos[p.first]++] = p.second;
    if (!directed) c[pos[p.second]++] = p.first;
  }
  SortLists(n, r.data(), c.data());
  g.Adopt(std::move(r), std::move(c));
}

// SNAP edge list with arbitrary vertex names (GraphIO::ReadSNAPLargeVIDFile,
// src/graph/GraphIO.h:142-230): every run of digits on a line that starts
// with a digit is a vertex name; names get dense ids in order of first
// appearance (the exact string: "007" and "7" are two vertices); the names
// pair up into edges in order.  Lists are sorted; nothing is deduplicated.
void ReadSnapLvidFile(const std::string& path, bool directed, HostGraph& g) {
  std::ifstream in(path);
  if (!in) Fail(SME_ERR_BAD_FILE, "cannot open " + path);
  std::unordered_map<std::string, uintV> ids;
  std::vector<uintV> ends;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || !std::isdigit((unsigned char)line[0])) continue;
    size_t i = 0;
    while (i < line.size()) {
      while (i < line.size() && !std::isdigit((unsigned char)line[i])) ++i;
      size_t j = i;
      while (j < line.size() && std::isdigit((unsigned char)line[j])) ++j;
      if (j > i) {
        auto it = ids.emplace(line.substr(i, j - i), (uintV)ids.size()).first;
        ends.push_back(it->second);
      }
      i = j;
    }
  }
  if (ends.size() % 2) Fail(SME_ERR_BAD_FILE, "odd number of vertex names in " + path);
  const uint64_t n = ids.size();
  std::vector<uintE> r(n + 1, 0);
  for (size_t k = 0; k < ends.size(); k += 2) {
    r[ends[k] + 1]++;
    if (!directed) r[ends[k + 1] + 1]++;
  }
  for (uint64_t u = 0; u < n; ++u) r[u + 1] += r[u];
  std::vector<uintV> c(r[n]);
  std::vector<uintE> pos(r.begin(), r.end() - 1);
  for (size_t k = 0; k < ends.size(); k += 2) {
    c[pos[ends[k]]++] = ends[k + 1];
    if (!directed) c[pos[ends[k + 1]]++] = ends[k];
  }
  SortLists(n, r.data(), c.data());
  g.Adopt(std::move(r), std::move(c));
}

// GraphIO::WriteCSRSNAPFile (src/graph/GraphIO.h:389-413): "u v" per stored
// pair with u < v, in CSR order.
void WriteSnapFile(const std::string& path, const HostGraph& g) {
  std::ofstream out(path);
  if (!out) Fail(SME_ERR_BAD_FILE, "cannot create " + path);
  for (uint64_t u = 0; u < g.n; ++u)
    for (uintE j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j)
      if (u < g.cols[j]) out << u << " " << g.cols[j] << "\n";
  if (!out) Fail(SME_ERR_BAD_FILE, "write failed: " + path);
}

// GraphIO::WriteCSRAdjFile (src/graph/GraphIO.h:414-436), the partitioner's
// input: per vertex "u<TAB>" then "v " per neighbour, then a newline; and
// `path`.info holding "n m".
void WriteAdjFile(const std::string& path, const HostGraph& g) {
  {
    std::ofstream out(path);
    if (!out) Fail(SME_ERR_BAD_FILE, "cannot create " + path);
    for (uint64_t u = 0; u < g.n; ++u) {
      out << u << "\t";
      for (uintE j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j) out << g.cols[j] << " ";
      out << "\n";
    }
    if (!out) Fail(SME_ERR_BAD_FILE, "write failed: " + path);
  }
  std::ofstream info(path + ".info");
  if (!info) Fail(SME_ERR_BAD_FILE, "cannot create " + path + ".info");
  info << g.n << " " << g.m;
  if (!info) Fail(SME_ERR_BAD_FILE, "write failed: " + path + ".info");
}

// ------------------------------------------------------------ preprocess --
// Removes self loops and parallel edges (adjacent duplicates of a sorted
// list), then dangling vertices, relabelling the rest densely in id order.
void Preprocess(HostGraph& g) {
  const uint64_t n = g.n;
  std::vector<uintE> keep(n + 1, 0);
  for (uint64_t u = 0; u < n; ++u) {
    uintE cnt = 0;
    for (uintE j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j) {
      uintV v = g.cols[j];
      bool par = j > g.row_ptrs[u] && v == g.cols[j - 1];
      if (!par && v != u) ++cnt;
    }
    keep[u + 1] = cnt;
  }
  for (uint64_t u = 0; u < n; ++u) keep[u + 1] += keep[u];
  std::vector<uintV> id(n);
  uintV next = 0;
  for (uint64_t u = 0; u < n; ++u) id[u] = keep[u + 1] > keep[u] ? next++ : (uintV)n;
  std::vector<uintE> r(next + 1, 0);
  std::vector<uintV> c(keep[n]);
  for (uint64_t u = 0; u < n; ++u) {
    if (id[u] == (uintV)n) continue;
    r[id[u]] = keep[u];
    uintE o = keep[u];
    for (uintE j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j) {
      uintV v = g.cols[j];
      bool par = j > g.row_ptrs[u] && v == g.cols[j - 1];
      if (!par && v != u) c[o++] = id[v];
    }
  }
  r[next] = keep[n];
  g.Adopt(std::move(r), std::move(c));
}

void Validate(const HostGraph& g) {
  uint64_t dangling = 0, loops = 0, par = 0, unsorted = 0;
  for (uint64_t u = 0; u < g.n; ++u) {
    if (g.row_ptrs[u] == g.row_ptrs[u + 1]) ++dangling;
    for (uintE j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j) {
      if (g.cols[j] == u) ++loops;
      if (j > g.row_ptrs[u] && g.cols[j] == g.cols[j - 1]) ++par;
      if (j > g.row_ptrs[u] && g.cols[j] < g.cols[j - 1]) ++unsorted;
    }
  }
  if (dangling || loops || par || unsorted)
    Fail(SME_ERR_INVALID_ARG, "graph invalid: dangling=" + std::to_string(dangling) +
                                  " self_loops=" + std::to_string(loops) +
                                  " parallel_edges=" + std::to_string(par) +
                                  " unsorted=" + std::to_string(unsorted));
}

// Renumbers vertices by (degree, id) ascending, so that under a total order
// of the pattern (the clique queries) every candidate set N(u) ∩ {> u} holds
// only neighbours of higher degree — the degree orientation that bounds those
// sets by O(sqrt(m)).  A counting sort by degree keeps ties in id order, so
// the result is deterministic.  `orient` keeps, per vertex, only the
// neighbours with a higher new id (each undirected edge once).
void DegreeOrder(const HostGraph& in, bool orient, HostGraph& out, std::vector<uintV>* new_to_old) {
  const uint64_t n = in.n;
  uint64_t dmax = 0;
  for (uint64_t u = 0; u < n; ++u) dmax = std::max<uint64_t>(dmax, in.row_ptrs[u + 1] - in.row_ptrs[u]);
  std::vector<uint64_t> start(dmax + 2, 0);
  for (uint64_t u = 0; u < n; ++u) ++start[in.row_ptrs[u + 1] - in.row_ptrs[u] + 1];
  for (uint64_t d = 0; d <= dmax; ++d) start[d + 1] += start[d];
  std::vector<uintV> old_of(n), new_of(n);
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t x = start[in.row_ptrs[u + 1] - in.row_ptrs[u]]++;
    old_of[x] = (uintV)u;
    new_of[u] = (uintV)x;
  }
  std::vector<uintE> r(n + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
  for (uint64_t x = 0; x < n; ++x) {
    const uint64_t v = old_of[x];
    uintE k = in.row_ptrs[v + 1] - in.row_ptrs[v];
    if (orient) {
      k = 0;
      for (uintE j = in.row_ptrs[v]; j < in.row_ptrs[v + 1]; ++j) k += new_of[in.cols[j]] > x;
    }
    r[x + 1] = k;
  }
  for (uint64_t x = 0; x < n; ++x) r[x + 1] += r[x];
  std::vector<uintV> c(r[n]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (uint64_t x = 0; x < n; ++x) {
    const uint64_t v = old_of[x];
    uintE o = r[x];
    for (uintE j = in.row_ptrs[v]; j < in.row_ptrs[v + 1]; ++j) {
      uintV w = new_of[in.cols[j]];
      if (!orient || w > x) c[o++] = w;
    }
    std::sort(c.begin() + r[x], c.begin() + r[x + 1]);
  }
  out.Adopt(std::move(r), std::move(c));
  out.oriented = orient;
  if (new_to_old) *new_to_old = std::move(old_of);
}

// GraphIO::ReadPartitionFile (src/graph/GraphIO.h:66-86): one partition id
// per vertex, whitespace separated; a single partition or no file puts every
// vertex in partition 0.  The reference asserts that the largest id is
// partition_num - 1; here that, a short file and an id out of range are
// errors.
void ReadPartitionFile(const std::string& path, uint64_t n, uint32_t partition_num, uint32_t* map) {
  if (partition_num == 0) Fail(SME_ERR_INVALID_ARG, "partition_num must be >= 1");
  if (partition_num == 1 || path.empty()) {
    std::fill(map, map + n, 0u);
    return;
  }
  std::ifstream in(path);
  if (!in) Fail(SME_ERR_BAD_FILE, "cannot open partition file " + path);
  uint64_t max_pid = 0;
  for (uint64_t u = 0; u < n; ++u) {
    unsigned long long pid;
    if (!(in >> pid)) Fail(SME_ERR_BAD_FILE, "partition file " + path + " ends after " + std::to_string(u) +
                                                 " of " + std::to_string(n) + " vertices");
    if (pid >= partition_num)
      Fail(SME_ERR_BAD_FILE, "partition id " + std::to_string(pid) + " of vertex " + std::to_string(u) +
                                 " is not below partition_num " + std::to_string(partition_num));
    map[u] = (uint32_t)pid;
    max_pid = std::max<uint64_t>(max_pid, pid);
  }
  if (max_pid + 1 != partition_num)
    Fail(SME_ERR_BAD_FILE, "partition file " + path + " has " + std::to_string(max_pid + 1) +
                               " partitions, partition_num is " + std::to_string(partition_num));
}

// The subgraph induced by the vertices of partition `p`, renumbered in
// ascending global id so lists stay sorted and the symmetry-breaking order is
// the global one (GraphPartition::BuildIntraPartition,
// src/graph/GraphPartition.h:36-95).
void InducedPartition(const HostGraph& g, const uint32_t* map, uint32_t p, HostGraph& out,
                      std::vector<uintV>* local_to_global) {
  const uint64_t n = g.n;
  std::vector<uintV> local(n, (uintV)-1), global;
  for (uint64_t u = 0; u < n; ++u)
    if (map[u] == p) {
      local[u] = (uintV)global.size();
      global.push_back((uintV)u);
    }
  const uint64_t k = global.size();
  std::vector<uintE> r(k + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
  for (uint64_t i = 0; i < k; ++i) {
    const uintV u = global[i];
    uintE c = 0;
    for (uintE j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j) c += map[g.cols[j]] == p;
    r[i + 1] = c;
  }
  for (uint64_t i = 0; i < k; ++i) r[i + 1] += r[i];
  std::vector<uintV> c(r[k]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (uint64_t i = 0; i < k; ++i) {
    const uintV u = global[i];
    uintE o = r[i];
    for (uintE j = g.row_ptrs[u]; j < g.row_ptrs[u + 1]; ++j)
      if (map[g.cols[j]] == p) c[o++] = local[g.cols[j]];
  }
  out.Adopt(std::move(r), std::move(c));
  if (local_to_global) *local_to_global = std::move(global);
}

void BuildFromEdges(uint64_t n, std::vector<std::pair<uintV, uintV>>& edges, HostGraph& g) {
  std::vector<uintE> r(n + 1, 0);
  for (auto& p : edges) {
    r[p.first + 1]++;
    r[p.second + 1]++;
  }
  for (uint64_t u = 0; u < n; ++u) r[u + 1] += r[u];
  std::vector<uintV> c(r[n]);
  {
    std::vector<uintE> pos(r.begin(), r.end() - 1);
    for (auto& p : edges) {
      c[pos[p.first]++] = p.second;
      c[pos[p.second]++] = p.first;
    }
  }
  std::vector<std::pair<uintV, uintV>>().swap(edges);
  SortLists(n, r.data(), c.data());
  g.Adopt(std::move(r), std::move(c));
  Preprocess(g);
}

// ------------------------------------------------------------ generators --
// Counter-based generator: every draw is a function of (seed, stream, index),
// so outputs do not depend on the number of host threads.
static inline uint64_t Mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static inline double Unit(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

void GenerateRmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                  HostGraph& g) {
  if (scale < 1 || scale > 31 || edge_factor < 1) Fail(SME_ERR_INVALID_ARG, "bad R-MAT size");
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12)
    Fail(SME_ERR_INVALID_ARG, "bad R-MAT probabilities");
  const uint64_t n = 1ULL << scale;
  const uint64_t ne = n * (uint64_t)edge_factor;
  std::vector<std::pair<uintV, uintV>> e(ne);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)ne; ++i) {
    uint64_t st = Mix64(seed ^ Mix64((uint64_t)i * 0x632BE59BD9B4E019ULL + 0x1234567ULL));
    uintV u = 0, v = 0;
    for (int lvl = 0; lvl < scale; ++lvl) {
      st = Mix64(st);
      double r = Unit(st);
      uint32_t bu, bv;
      if (r < a) { bu = 0; bv = 0; }
      else if (r < ab) { bu = 0; bv = 1; }
      else if (r < abc) { bu = 1; bv = 0; }
      else { bu = 1; bv = 1; }
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    e[i] = std::make_pair(u, v);
  }
  BuildFromEdges(n, e, g);
}

void GenerateER(uint64_t n, double avg_degree, uint64_t seed, HostGraph& g) {
  if (n < 2) Fail(SME_ERR_INVALID_ARG, "ER graph needs n >= 2");
  const double p = std::min(1.0, avg_degree / (double)(n - 1));
  std::vector<std::pair<uintV, uintV>> e;
  if (p <= 0) {
    BuildFromEdges(n, e, g);
    return;
  }
  // Geometric skipping over the n(n-1)/2 vertex pairs (Batagelj & Brandes 2005).
  const double lq = std::log(1.0 - p);
  uint64_t st = Mix64(seed ^ 0xE5E5E5E5ULL);
  long long v = 1, w = -1;
  while (v < (long long)n) {
    st = Mix64(st);
    double r = Unit(st);
    long long skip = p >= 1.0 ? 0 : (long long)std::floor(std::log(1.0 - r) / lq);
    w = w + 1 + skip;
    while (w >= v && v < (long long)n) {
      w -= v;
      ++v;
    }
    if (v < (long long)n) e.emplace_back((uintV)v, (uintV)w);
  }
  BuildFromEdges(n, e, g);
}

void GenerateBA(uint64_t n, uint32_t m_attach, uint64_t seed, HostGraph& g) {
  if (m_attach < 1 || n <= m_attach) Fail(SME_ERR_INVALID_ARG, "BA graph needs n > m >= 1");
  std::vector<std::pair<uintV, uintV>> e;
  std::vector<uintV> ends;  // every edge endpoint once: degree-proportional draw
  // seed clique on m_attach+1 vertices
  for (uintV u = 0; u <= m_attach; ++u)
    for (uintV v = u + 1; v <= m_attach; ++v) {
      e.emplace_back(u, v);
      ends.push_back(u);
      ends.push_back(v);
    }
  uint64_t st = Mix64(seed ^ 0xBABABABAULL);
  std::vector<uintV> pick;
  for (uint64_t u = m_attach + 1; u < n; ++u) {
    pick.clear();
    while (pick.size() < m_attach) {
      st = Mix64(st);
      uintV t = ends[st % ends.size()];
      if (std::find(pick.begin(), pick.end(), t) == pick.end()) pick.push_back(t);
    }
    for (uintV t : pick) {
      e.emplace_back((uintV)u, t);
      ends.push_back((uintV)u);
      ends.push_back(t);
    }
  }
  BuildFromEdges(n, e, g);
}

void GenerateClique(uint64_t n, HostGraph& g) {
  std::vector<uintE> r(n + 1, 0);
  std::vector<uintV> c;
  c.reserve(n * (n ? n - 1 : 0));
  for (uint64_t u = 0; u < n; ++u) {
    for (uint64_t v = 0; v < n; ++v)
      if (v != u) c.push_back((uintV)v);
    r[u + 1] = c.size();
  }
  g.Adopt(std::move(r), std::move(c));
}

}  // namespace sme
