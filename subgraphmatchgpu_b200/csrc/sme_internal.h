// Internal host-side declarations of libsme: graph container, pattern
// registry, the three query plans and the compiled level program that the
// device engine executes.
#pragma once

#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/sme.h"

namespace sme {

typedef uint32_t uintV;  // vertex ids (src/Meta.h:8)
typedef uint64_t uintE;  // edge offsets (src/Meta.h:9)

constexpr int kMaxQueryVertices = 6;  // src/Meta.h:30

// Error carried to the C-ABI as a status code plus message.
struct Error : public std::runtime_error {
  sme_status status;
  Error(sme_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};
[[noreturn]] inline void Fail(sme_status s, const std::string& m) {
  throw Error(s, m);
}
void SetLastError(const std::string& msg);

// ---------------------------------------------------------------- graphs --
// Packed copy of a graph's adjacency lists in pinned host memory
// (sme_graph_pack): what an upload of a non-resident graph copies over the
// host link, expanded on the device by k_unpack_lists (engine.cu).
//
// One contiguous buffer:
//   deg[n]    uint32 list lengths
//   woff[n]   uint32 start of each list in `stream`, in 4-byte words
//   segs[ns]  uint64 (vertex << 32 | segment) for every segment >= 1 of every
//             list (8-byte aligned)
//   stream    the lists, each on a 4-byte boundary, then 8 zero bytes
// A list of d elements is cut into segments of kPackSegment elements.  A list
// of S segments starts with S-1 table entries (uint32 value of the element
// before the segment, uint32 byte offset of the segment from the list start),
// then its segments.  A segment holds its blocks of 32 elements (the last one
// shorter): one width byte per block, then each block's deltas at `width`
// bits apiece, least significant bit first, every block on a byte boundary.
// An element's delta is its difference from the element before it in the
// list (from 0 for the first), modulo 2^32, so any list round-trips and
// sorted lists pack small.
constexpr uint32_t kPackSegment = 1024;
struct PackedLists {
  uint64_t n = 0, m = 0, nsegs = 0;
  uint8_t* base = nullptr;  // the buffer
  uint64_t total = 0;       // bytes of the buffer (what an upload copies)
  uint64_t deg_at = 0, woff_at = 0, segs_at = 0, stream_at = 0, stream_bytes = 0;  // byte offsets / size
  bool pinned = false;
  ~PackedLists();
};
struct HostGraph;
std::shared_ptr<const PackedLists> PackLists(const HostGraph& g);

// Host CSR.  Owns its arrays unless `borrowed`.
struct DeviceGraph;  // engine.cu
struct HostGraph {
  uint64_t n = 0, m = 0;
  uintE* row_ptrs = nullptr;
  uintV* cols = nullptr;
  bool borrowed = false;
  bool oriented = false;       // each edge once, towards the higher id
  // 1 no vertex lists itself, 0 some vertex does, -1 not yet checked
  // (server workers may ask concurrently: the flag is atomic)
  mutable std::atomic<int> loop_free{-1};
  bool LoopFree() const;
  std::vector<uintE> row_store;
  std::vector<uintV> col_store;
  DeviceGraph* dev = nullptr;  // resident device copy (may be null)
  // packed lists an upload copies instead of the CSR (null = plain CSR)
  std::shared_ptr<const PackedLists> packed;
  uint64_t MaxDegree() const;
  void Adopt(std::vector<uintE>&& r, std::vector<uintV>&& c);
  // The (at most) max_hubs vertices of highest degree among those of degree
  // >= min_degree (ties by id), sorted by id; computed once per graph and
  // arguments and shared by every upload.
  std::shared_ptr<const std::vector<uint32_t>> HubSelection(uint64_t min_degree, uint64_t max_hubs) const;

 private:
  mutable std::mutex hub_mu_;
  mutable std::shared_ptr<const std::vector<uint32_t>> hub_sel_;
  mutable uint64_t hub_sel_min_ = 0, hub_sel_max_ = 0;
};

void ReadBinFile(const std::string& path, HostGraph& g);
void ReadSnapFile(const std::string& path, bool directed, HostGraph& g);
void WriteBinFile(const std::string& path, const HostGraph& g);
void ReadSnapLvidFile(const std::string& path, bool directed, HostGraph& g);
void WriteSnapFile(const std::string& path, const HostGraph& g);
void WriteAdjFile(const std::string& path, const HostGraph& g);
void Preprocess(HostGraph& g);
void Validate(const HostGraph& g);
// Builds a sorted undirected CSR from an edge list (both directions stored),
// then applies Preprocess().
void BuildFromEdges(uint64_t n, std::vector<std::pair<uintV, uintV>>& edges,
                    HostGraph& g);
// Partition map of n vertices from a partition file (GraphIO::ReadPartitionFile).
void ReadPartitionFile(const std::string& path, uint64_t n, uint32_t partition_num, uint32_t* map);
// Subgraph induced by partition p, ascending global ids (GraphPartition).
void InducedPartition(const HostGraph& g, const uint32_t* map, uint32_t p, HostGraph& out,
                      std::vector<uintV>* local_to_global);
// Degree-ordered copy (vertices renumbered by (degree, id) ascending),
// optionally oriented towards the higher id; new_to_old[new] = old id.
void DegreeOrder(const HostGraph& in, bool orient, HostGraph& out, std::vector<uintV>* new_to_old);
void GenerateRmat(int scale, int edge_factor, double a, double b, double c,
                  uint64_t seed, HostGraph& g);
void GenerateER(uint64_t n, double avg_degree, uint64_t seed, HostGraph& g);
void GenerateBA(uint64_t n, uint32_t m_attach, uint64_t seed, HostGraph& g);
void GenerateClique(uint64_t n, HostGraph& g);

// ----------------------------------------------------------------- query --
enum CondOp : uint8_t { LESS_THAN = 0, LARGER_THAN = 1, NON_EQUAL = 2, OP_NONE = 3 };
typedef std::vector<uintV> ConnType;
typedef std::vector<ConnType> AllConnType;
typedef std::pair<CondOp, uintV> CondType;
typedef std::vector<std::vector<CondType>> AllCondType;
typedef std::vector<uintV> SearchSequence;

struct Query {
  int type = 0;
  int n = 0;
  AllConnType con;    // per-vertex neighbour lists, reference order
  AllCondType order;  // per-vertex symmetry-breaking conditions
  bool enable_ordering = true;
  Query(int query_type, bool enable_ordering = true);
};

// Plan helpers with the reference's semantics (src/query/common/Plan.h).
CondOp GetConditionType(uintV l1, uintV l2, const AllCondType& order);
void GetBackwardConnectivity(AllConnType& ret, const AllConnType& con,
                             const SearchSequence& seq);

// ------------------------------------------------------------ LIGHT plan --
enum LazyOp : uint8_t {
  L_COMPUTE = 0, L_COMPUTE_PATH_COUNT = 1, L_MATERIALIZE = 2,
  L_FILTER_COMPUTE = 3, L_COUNT = 4, L_COMPUTE_COUNT = 5
};
typedef std::pair<LazyOp, uintV> LazyEntry;

struct LazyPlan {
  const Query* q;
  int compress_level;  // effective intra-partition level
  SearchSequence seq;
  std::vector<LazyEntry> exec;
  std::vector<std::vector<uintV>> materialized;             // before level i
  std::vector<std::vector<uintV>> computed_unmaterialized;  // before level i
  AllCondType compute_cond, materialize_cond, filter_cond, count_to_mat_cond;
  AllConnType backward_conn;
  LazyPlan(const Query& q, int compress_level);
  std::string Describe() const;
};
// Per-level materialised/computed sets and the compute, materialise and
// filter conditions of an execute sequence (LazyTraversalPlanUtils.h:40-158).
void LightConstraintsFor(LazyPlan& p);

// ------------------------------------------------------------ reuse plan --
struct ReuseConnMeta {
  ConnType conn;         // sorted, index based
  uintV source_vertex;   // index based
  ConnType source_conn;  // sorted, index based
  std::vector<uintV> mapping;  // size n, n = none
};
struct VertexReusePlan {
  std::vector<ReuseConnMeta> reuse;
  ConnType separate;
};
struct ReusePlan {
  const Query* q;
  bool autogen;
  SearchSequence seq;
  AllConnType con;     // relabelled by seq (index based)
  AllCondType order;   // relabelled by seq
  std::vector<VertexReusePlan> levels;
  std::vector<bool> cache_required;
  ReusePlan(const Query& q, bool autogen);
  std::string Describe() const;
};
bool HasHardcodedReusePlan(int query_type);

// -------------------------------------------------------- traversal plan --
struct TraversalPlan {
  const Query* q;
  AllConnType ordered_conn;  // backward neighbours (smaller ids)
  AllCondType ordered_order; // GetOrderedOrdering
  AllCondType whole_order;   // GetWholeOrderedOrdering (NON_EQUAL filled)
  explicit TraversalPlan(const Query& q);
  std::string Describe() const;
};

// ------------------------------------------------ compiled level program --
// The device engine runs every plan as a sequence of these steps.  Vertex ids
// in a program are the plan's pattern-vertex ids; `out_slot` maps them to the
// output tuple position (u0..u_{k-1}, original query ids).
enum StepKind : uint8_t {
  S_INIT = 0,          // roots of the task: inst[u] = begin + i
  S_COMPUTE = 1,       // candidate set of u per path
  S_MATERIALIZE = 2,   // expand u's candidate sets into new partial instances
  S_FILTER = 3,        // re-filter u's candidate sets (FILTER_COMPUTE)
  S_COMPUTE_COUNT = 4, // count candidates of u (optionally ranked into with_u)
  S_PATH_COUNT = 5,    // per-path candidate count only (COMPUTE_PATH_COUNT)
  S_COUNT = 6,         // LIGHTCount / LIGHTDirectCount over unmaterialised sets
  S_ALIAS = 7          // u's set is an earlier step's identical set (no work)
};
struct StepCond { uint8_t op; uint8_t operand; };
struct Step {
  StepKind kind;
  uint8_t u = 0;
  std::vector<uint8_t> conn;      // materialised vertices: adjacency lists
  int8_t reuse_src = -1;          // vertex whose cached set is intersected
  int8_t alias_of = -1;           // S_ALIAS: vertex whose live set u shares
  std::vector<uint8_t> full_conn; // fallback when no cache (reuse plan)
  int8_t map_src = -1;            // reuse plan: mapped meta's cached level
  uint8_t map_x = 0;              //   vertex in the sibling's level-1 place
  uint8_t map_mask = 0;           //   conn entries the cached set replaces
  uint8_t map_op = OP_NONE;       //   level 1's order condition against M[0]
  std::vector<StepCond> cond;     // conditions vs materialised vertices
  bool keep_set = false;          // MATERIALIZE keeps u's set as a cache
  int8_t with_u = -1;             // COMPUTE_COUNT rank partner
  uint8_t with_op = OP_NONE;
  bool direct = false;            // COUNT: closed form (LIGHTDirectCount)
  std::vector<uint8_t> unmat;     // COUNT: unmaterialised vertices
  uint8_t pair_op = OP_NONE;      // COUNT with 2 unmaterialised vertices
  // state after this step (for the engine's bookkeeping)
  std::vector<uint8_t> mat_after;   // materialised vertices
  std::vector<uint8_t> sets_after;  // vertices with live candidate sets
  std::string label;
};
struct Program {
  int query_type = 0;
  int n = 0;               // pattern vertices
  int algo = SME_GPU_LIGHT;
  std::vector<Step> steps;
  std::vector<uint8_t> out_slot;  // plan vertex -> tuple position
  bool enumerate = false;
  std::string Describe() const;
};
// Builds the level program of a query under one of the three GPU plans.
// `loop_free`: the graph has no self loop, so a candidate drawn from N(M[v])
// differs from M[v] without a check.
Program Compile(const sme_opts& o, bool enumerate, bool loop_free = false);
// A clique query whose symmetry breaking is the total order u0 < u1 < ...
bool IsOrderedClique(const Query& q);
// Fails unless `p` counts correctly on an oriented graph: an ordered clique
// whose every adjacency list read belongs to an earlier vertex of the order.
void RequireOrientable(const Program& p, bool enable_ordering);

}  // namespace sme

// Opaque handle of the C-ABI (include/sme.h).
struct sme_graph {
  sme::HostGraph g;
};
