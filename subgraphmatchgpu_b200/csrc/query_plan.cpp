// Pattern registry and the three query plans of the enumeration path.
//
//   Query Q0..Q13          src/query/common/Query.h:84-434
//   Plan helpers           src/query/common/Plan.h:32-217
//   TraversalPlan (GPSM)   src/query/TraversalPlan.h:193-233 +
//                          src/gpu/plan/DevTraversalPlan.cuh:9-16
//   LazyTraversalPlan      src/query/LazyTraversalPlan.h:13-197,
//     (LIGHT)              src/query/optimizer/LazyTraversalPlanGenerator.h:11-300,
//                          LazyTraversalPlanHardCode.h:59-116,
//                          LazyTraversalPlanUtils.h:40-158
//   ReuseTraversalPlan     src/query/ReuseTraversalPlan.h:11-76,
//                          src/query/optimizer/ReuseTraversalPlanHardCode.h,
//                          ReuseTraversalOptimizer.h:12-174,
//                          ReusePlanGenerator.h:21-380
// The pattern tables, the per-vertex neighbour order and the search orders
// must match the reference exactly: the LIGHT execute sequence depends on the
// order in which backward neighbours are visited.
#include <algorithm>
#include <cassert>
#include <cmath>
#include <sstream>

#include "sme_internal.h"

namespace sme {

// ----------------------------------------------------------------- Query --
namespace {
struct QueryDef {
  int n;
  std::vector<std::vector<int>> con;
  // per vertex: list of (op, operand); op 'L' less than, 'G' larger than
  std::vector<std::vector<std::pair<char, int>>> order;
};

const std::vector<QueryDef>& Registry() {
  static const std::vector<QueryDef> defs = {
      // Q0 triangle
      {3, {{1, 2}, {0, 2}, {0, 1}}, {{{'L', 1}}, {{'G', 0}, {'L', 2}}, {{'G', 1}}}},
      // Q1 square (4-cycle)
      {4, {{1, 3}, {0, 2}, {1, 3}, {0, 2}},
       {{{'L', 1}, {'L', 2}, {'L', 3}}, {{'G', 0}, {'L', 3}}, {{'G', 0}}, {{'G', 0}, {'G', 1}}}},
      // Q2 chordal square (diamond)
      {4, {{1, 2, 3}, {0, 2}, {0, 1, 3}, {0, 2}}, {{{'L', 2}}, {{'L', 3}}, {{'G', 0}}, {{'G', 1}}}},
      // Q3 4-clique
      {4, {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}},
       {{{'L', 1}}, {{'G', 0}, {'L', 2}}, {{'G', 1}, {'L', 3}}, {{'G', 2}}}},
      // Q4 house
      {5, {{1, 2}, {0, 2, 3}, {0, 1, 4}, {1, 4}, {2, 3}}, {{}, {{'L', 2}}, {{'G', 1}}, {}, {}}},
      // Q5 quad triangle
      {6, {{1, 2, 3, 4, 5}, {0, 2}, {0, 1, 3}, {0, 2, 4}, {0, 3, 5}, {0, 4}},
       {{}, {}, {{'L', 4}}, {}, {{'G', 2}}, {}}},
      // Q6 near-5-clique
      {5, {{1, 2, 3, 4}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2, 4}, {0, 3}},
       {{{'L', 3}}, {{'L', 2}}, {{'G', 1}}, {{'G', 0}}, {}}},
      // Q7 5-clique
      {5, {{1, 2, 3, 4}, {0, 2, 3, 4}, {0, 1, 3, 4}, {0, 1, 2, 4}, {0, 1, 2, 3}},
       {{{'L', 1}}, {{'G', 0}, {'L', 2}}, {{'G', 1}, {'L', 3}}, {{'G', 2}, {'L', 4}}, {{'G', 3}}}},
      // Q8 chordal roof
      {5, {{1, 2, 3}, {0, 2, 3}, {0, 1, 4}, {0, 1, 4}, {2, 3}},
       {{{'L', 1}}, {{'G', 0}}, {{'L', 3}}, {{'G', 2}}, {}}},
      // Q9 three triangles
      {5, {{1, 2, 3, 4}, {0, 3, 2}, {0, 1, 4}, {0, 1}, {0, 2}}, {{}, {{'L', 2}}, {{'G', 1}}, {}, {}}},
      // Q10 solar square
      {5, {{1, 2, 3, 4}, {0, 2, 4}, {0, 1, 3}, {0, 2, 4}, {0, 1, 3}},
       {{}, {{'L', 2}, {'L', 3}, {'L', 4}}, {{'L', 4}, {'G', 1}}, {{'G', 1}}, {{'G', 1}, {'G', 2}}}},
      // Q11 6-clique
      {6,
       {{1, 2, 3, 4, 5}, {0, 2, 3, 4, 5}, {0, 1, 3, 4, 5}, {0, 1, 2, 4, 5}, {0, 1, 2, 3, 5},
        {0, 1, 2, 3, 4}},
       {{{'L', 1}},
        {{'G', 0}, {'L', 2}},
        {{'G', 1}, {'L', 3}},
        {{'G', 2}, {'L', 4}},
        {{'G', 3}, {'L', 5}},
        {{'G', 4}}}},
      // Q12 near-near-5-clique
      {5, {{1, 2, 3, 4}, {0, 2, 3, 4}, {0, 1, 3}, {0, 1, 2, 4}, {0, 1, 3}},
       {{{'L', 1}}, {{'G', 0}}, {{'L', 4}}, {}, {{'G', 2}}}},
      // Q13 triangle in diamond
      {6, {{1, 2, 3, 5}, {0, 2, 3, 4}, {0, 1, 4, 5}, {0, 1}, {1, 2}, {0, 2}},
       {{{'L', 1}}, {{'L', 2}, {'G', 0}}, {{'G', 1}}, {}, {}, {}}},
  };
  return defs;
}
}  // namespace

Query::Query(int query_type, bool ordering) : type(query_type), enable_ordering(ordering) {
  if (query_type < 0 || query_type >= SME_NUM_QUERIES)
    Fail(SME_ERR_UNSUPPORTED_QUERY, "unknown query type " + std::to_string(query_type));
  const QueryDef& d = Registry()[query_type];
  n = d.n;
  con.resize(n);
  order.resize(n);
  for (int u = 0; u < n; ++u) {
    for (int v : d.con[u]) con[u].push_back((uintV)v);
    if (ordering)
      for (auto& p : d.order[u])
        order[u].push_back(CondType(p.first == 'L' ? LESS_THAN : LARGER_THAN, (uintV)p.second));
  }
}

// ---------------------------------------------------------- Plan helpers --
CondOp GetConditionType(uintV l1, uintV l2, const AllCondType& order) {
  for (auto& c : order[l1])
    if (c.second == l2) return c.first;
  return NON_EQUAL;
}

void GetBackwardConnectivity(AllConnType& ret, const AllConnType& con, const SearchSequence& seq) {
  size_t n = con.size();
  ret.assign(n, ConnType());
  std::vector<bool> vis(n, false);
  for (size_t i = 0; i < n; ++i) {
    uintV u = seq[i];
    for (uintV nu : con[u])
      if (vis[nu]) ret[u].push_back(nu);
    vis[u] = true;
  }
}

static void GetOrderedConnectivity(AllConnType& ret, const AllConnType& con) {
  ret.assign(con.size(), ConnType());
  for (uintV u = 0; u < con.size(); ++u)
    for (uintV v : con[u])
      if (v < u) ret[u].push_back(v);
}
static void GetOrderedOrdering(AllCondType& ret, const AllCondType& order) {
  ret.assign(order.size(), std::vector<CondType>());
  for (uintV u = 0; u < order.size(); ++u)
    for (auto& c : order[u])
      if (c.second < u) ret[u].push_back(c);
}
static void GetWholeOrderedOrdering(AllCondType& ret, const AllCondType& order) {
  ret.assign(order.size(), std::vector<CondType>());
  for (uintV u = 0; u < order.size(); ++u)
    for (uintV v = 0; v < u; ++v) ret[u].push_back(CondType(GetConditionType(u, v, order), v));
}
// Relabels connectivity/ordering so that vertex seq[i] becomes i
// (TraversalPlan::GenConstraints, TraversalPlan.h:203-233).
static void Relabel(const Query& q, const SearchSequence& seq, AllConnType& con, AllCondType& order) {
  size_t n = q.n;
  std::vector<uintV> otn(n);
  for (uintV i = 0; i < n; ++i) otn[seq[i]] = i;
  con.assign(n, ConnType());
  order.assign(n, std::vector<CondType>());
  for (uintV i = 0; i < n; ++i) {
    uintV ou = seq[i];
    for (uintV v : q.con[ou]) con[i].push_back(otn[v]);
    for (auto& c : q.order[ou]) order[i].push_back(CondType(c.first, otn[c.second]));
  }
}

static const char* OpName(CondOp op) {
  return op == LESS_THAN ? "<" : op == LARGER_THAN ? ">" : op == NON_EQUAL ? "!=" : "?";
}

// -------------------------------------------------------- TraversalPlan --
TraversalPlan::TraversalPlan(const Query& query) : q(&query) {
  GetOrderedConnectivity(ordered_conn, query.con);
  GetOrderedOrdering(ordered_order, query.order);
  GetWholeOrderedOrdering(whole_order, query.order);
}

std::string TraversalPlan::Describe() const {
  std::ostringstream os;
  os << "TraversalPlan Q" << q->type << " search sequence:";
  for (int u = 0; u < q->n; ++u) os << " " << u;
  os << "\n";
  for (int u = 0; u < q->n; ++u) {
    os << "level " << u << ": conn=(";
    for (size_t j = 0; j < ordered_conn[u].size(); ++j) os << (j ? "," : "") << ordered_conn[u][j];
    os << ") cond=(";
    for (size_t j = 0; j < whole_order[u].size(); ++j)
      os << (j ? "," : "") << OpName(whole_order[u][j].first) << whole_order[u][j].second;
    os << ")\n";
  }
  return os.str();
}

// --------------------------------------------------------------- LIGHT --
static size_t OpIndex(const std::vector<LazyEntry>& e, LazyOp op, uintV u) {
  for (size_t i = 0; i < e.size(); ++i)
    if (e[i].first == op && e[i].second == u) return i;
  return e.size();
}

static void LightSearchSequence(int type, SearchSequence& seq) {
  static const std::vector<std::vector<uintV>> orders = {
      {0, 1, 2},       {0, 1, 2, 3},    {0, 2, 1, 3},       {0, 1, 2, 3},    {1, 2, 3, 0, 4},
      {0, 2, 4, 1, 3, 5}, {0, 1, 3, 2, 4}, {0, 1, 2, 3, 4}, {0, 1, 2, 3, 4}, {0, 1, 2, 3, 4},
      {0, 1, 3, 2, 4}, {0, 1, 2, 3, 4, 5}, {0, 1, 3, 2, 4}, {0, 1, 2, 3, 4, 5}};
  seq = orders[type];
}

// Compute every pattern vertex, materialising backward neighbours on demand
// (GenerateComputeExecuteSequence, LazyTraversalPlanGenerator.h:124-154).
static void ComputeSequence(std::vector<LazyEntry>& e, const SearchSequence& seq, const AllConnType& con) {
  AllConnType bc;
  GetBackwardConnectivity(bc, con, seq);
  std::vector<bool> mat(seq.size(), false);
  e.push_back(LazyEntry(L_MATERIALIZE, seq[0]));
  mat[seq[0]] = true;
  for (size_t i = 1; i < seq.size(); ++i) {
    uintV u = seq[i];
    for (uintV p : bc[u])
      if (!mat[p]) {
        e.push_back(LazyEntry(L_MATERIALIZE, p));
        mat[p] = true;
      }
    e.push_back(LazyEntry(L_COMPUTE, u));
  }
}

static void InspectUnmaterialized(std::vector<uintV>& unmat, std::vector<bool>& need_filter,
                                  const std::vector<LazyEntry>& e, size_t n) {
  std::vector<bool> mat(n, false);
  for (auto& x : e)
    if (x.first == L_MATERIALIZE) mat[x.second] = true;
  for (uintV u = 0; u < n; ++u) {
    if (mat[u]) continue;
    unmat.push_back(u);
    size_t ind = OpIndex(e, L_COMPUTE, u);
    bool f = false;
    for (size_t i = ind + 1; i < e.size(); ++i)
      if (e[i].first == L_MATERIALIZE) f = true;
    need_filter.push_back(f);
  }
}

static void Count1(std::vector<LazyEntry>& e, size_t n, const std::vector<uintV>& um,
                   const std::vector<bool>& nf, int level) {
  if (level == SME_COMPRESS_MATERIALIZE || level == SME_COMPRESS_NON_MATERIALIZE) {
    if (nf[0]) e.push_back(LazyEntry(L_FILTER_COMPUTE, um[0]));
    e.push_back(LazyEntry(L_COUNT, (uintV)n));
  } else {
    if (nf[0]) {
      e.push_back(LazyEntry(L_FILTER_COMPUTE, um[0]));
      e.push_back(LazyEntry(L_COUNT, (uintV)n));
    } else {
      assert(e.back().second == um[0] && e.back().first == L_COMPUTE);
      e.back().first = L_COMPUTE_COUNT;
    }
  }
}

static void Count2(std::vector<LazyEntry>& e, size_t n, const std::vector<uintV>& um,
                   const std::vector<bool>& nf, int level) {
  if (level == SME_COMPRESS_MATERIALIZE) {
    e.push_back(LazyEntry(L_MATERIALIZE, um[0]));
    e.push_back(LazyEntry(L_FILTER_COMPUTE, um[1]));
    e.push_back(LazyEntry(L_COUNT, (uintV)n));
  } else if (level == SME_COMPRESS_NON_MATERIALIZE) {
    if (nf[0]) e.push_back(LazyEntry(L_FILTER_COMPUTE, um[0]));
    if (nf[1]) e.push_back(LazyEntry(L_FILTER_COMPUTE, um[1]));
    e.push_back(LazyEntry(L_COUNT, (uintV)n));
  } else {
    if (nf[0] && nf[1]) {
      e.push_back(LazyEntry(L_FILTER_COMPUTE, um[0]));
      e.push_back(LazyEntry(L_FILTER_COMPUTE, um[1]));
      e.push_back(LazyEntry(L_COUNT, (uintV)n));
    } else if (!nf[0] && !nf[1]) {
      // the later of the two (single) COMPUTE entries becomes COMPUTE_COUNT
      size_t i0 = OpIndex(e, L_COMPUTE, um[0]), i1 = OpIndex(e, L_COMPUTE, um[1]);
      size_t mx = std::max(i0, i1);
      assert(mx == e.size() - 1);
      e[mx].first = L_COMPUTE_COUNT;
    } else {
      uintV need = nf[0] ? um[0] : um[1];
      uintV other = nf[0] ? um[1] : um[0];
      e.erase(e.begin() + OpIndex(e, L_COMPUTE, other));
      e.push_back(LazyEntry(L_FILTER_COMPUTE, need));
      e.push_back(LazyEntry(L_COMPUTE_COUNT, other));
    }
  }
}

static void GenerateExecuteSequence(std::vector<LazyEntry>& e, const SearchSequence& seq,
                                    const AllConnType& con, size_t n, int level) {
  ComputeSequence(e, seq, con);
  std::vector<uintV> um;
  std::vector<bool> nf;
  InspectUnmaterialized(um, nf, e, n);
  if (um.size() == 1) {
    Count1(e, n, um, nf, level);
  } else if (um.size() == 2) {
    Count2(e, n, um, nf, level);
  } else {
    for (size_t i = 2; i < um.size(); ++i) e.push_back(LazyEntry(L_MATERIALIZE, um[i]));
    std::vector<uintV> rest(um.begin(), um.begin() + 2);
    Count2(e, n, rest, std::vector<bool>(2, true), level);
  }
}

static void SpecialExecuteSequence(std::vector<LazyEntry>& e, int type, const SearchSequence& seq,
                                   const AllConnType& con, size_t n) {
  ComputeSequence(e, seq, con);
  std::vector<uintV> um;
  std::vector<bool> nf;
  InspectUnmaterialized(um, nf, e, n);
  if (type == 2 || type == 6) {
    size_t l2 = e.size() - 2, l1 = e.size() - 1;
    assert(um.size() == 2 && e[l1].first == L_COMPUTE && e[l2].first == L_COMPUTE);
    e[l2].first = L_COMPUTE_PATH_COUNT;
    e[l1].first = L_COMPUTE_PATH_COUNT;
    e.push_back(LazyEntry(L_COUNT, (uintV)n));
  } else {  // Q5
    for (size_t i = 0; i < um.size(); ++i)
      if (nf[i]) e.push_back(LazyEntry(L_FILTER_COMPUTE, um[i]));
    e.push_back(LazyEntry(L_COUNT, (uintV)n));
  }
}

// Conditions per step kind (LazyTraversalPlanUtils.h:40-158).
void LightConstraintsFor(LazyPlan& p) {
  const size_t n = p.q->n;
  const auto& e = p.exec;
  std::vector<bool> mat(n, false);
  std::vector<uintV> all_mat, all_comp;
  p.materialized.assign(e.size(), {});
  p.computed_unmaterialized.assign(e.size(), {});
  for (size_t i = 0; i < e.size(); ++i) {
    p.materialized[i] = all_mat;
    for (uintV u : all_comp)
      if (!mat[u]) p.computed_unmaterialized[i].push_back(u);
    if (e[i].first == L_COMPUTE || e[i].first == L_COMPUTE_PATH_COUNT) {
      all_comp.push_back(e[i].second);
    } else if (e[i].first == L_MATERIALIZE) {
      all_mat.push_back(e[i].second);
      mat[e[i].second] = true;
    }
  }
  const AllCondType& order = p.q->order;
  p.compute_cond.assign(n, {});
  p.materialize_cond.assign(n, {});
  p.filter_cond.assign(n, {});
  std::vector<uintV> mats;
  for (size_t i = 0; i < e.size(); ++i) {
    LazyOp op = e[i].first;
    uintV u = e[i].second;
    if (op == L_COMPUTE || op == L_COMPUTE_COUNT || op == L_COMPUTE_PATH_COUNT) {
      p.compute_cond[u].clear();
      for (uintV pu : mats) p.compute_cond[u].push_back(CondType(GetConditionType(u, pu, order), pu));
    } else if (op == L_MATERIALIZE) {
      mats.push_back(u);
    }
    if (op == L_MATERIALIZE || op == L_FILTER_COMPUTE) {
      AllCondType& dst = op == L_MATERIALIZE ? p.materialize_cond : p.filter_cond;
      dst[u].clear();
      for (int j = (int)i - 1; j >= 0; --j) {
        if (e[j].first == L_COMPUTE && e[j].second == u) break;
        if (e[j].first == L_MATERIALIZE)
          dst[u].push_back(CondType(GetConditionType(u, e[j].second, order), e[j].second));
      }
    }
  }
  p.count_to_mat_cond.assign(n, {});
  for (uintV u = 0; u < n; ++u)
    for (auto& x : e)
      if (x.first == L_MATERIALIZE && x.second != u)
        p.count_to_mat_cond[u].push_back(CondType(GetConditionType(u, x.second, order), x.second));
}

LazyPlan::LazyPlan(const Query& query, int level) : q(&query) {
  LightSearchSequence(query.type, seq);
  const size_t n = query.n;
  if (level == SME_COMPRESS_SPECIAL && (query.type == 2 || query.type == 5 || query.type == 6)) {
    compress_level = SME_COMPRESS_SPECIAL;
    SpecialExecuteSequence(exec, query.type, seq, query.con, n);
  } else {
    compress_level = level;
    GenerateExecuteSequence(exec, seq, query.con, n,
                            level == SME_COMPRESS_SPECIAL ? SME_COMPRESS_NON_MATERIALIZE_OPT : level);
  }
  GetBackwardConnectivity(backward_conn, query.con, seq);
  LightConstraintsFor(*this);
}

static const char* LazyName(LazyOp op) {
  switch (op) {
    case L_COMPUTE: return "COMPUTE";
    case L_COMPUTE_PATH_COUNT: return "COMPUTE_PATH_COUNT";
    case L_MATERIALIZE: return "MATERIALIZE";
    case L_FILTER_COMPUTE: return "FILTER_COMPUTE";
    case L_COUNT: return "COUNT";
    case L_COMPUTE_COUNT: return "COMPUTE_COUNT";
  }
  return "";
}

std::string LazyPlan::Describe() const {
  std::ostringstream os;
  os << "LazyTraversalPlan Q" << q->type << " search sequence:";
  for (auto u : seq) os << " " << u;
  os << "\n";
  for (auto& x : exec) os << "(" << LazyName(x.first) << "," << x.second << "),";
  os << "\n";
  for (size_t i = 0; i < exec.size(); ++i) {
    os << "materialized vertices:(";
    for (size_t j = 0; j < materialized[i].size(); ++j) os << (j ? "," : "") << materialized[i][j];
    os << ")\ncomputed_unmaterialized_vertices:(";
    for (size_t j = 0; j < computed_unmaterialized[i].size(); ++j)
      os << (j ? "," : "") << computed_unmaterialized[i][j];
    os << ")\n";
  }
  return os.str();
}

// --------------------------------------------------------------- reuse --
namespace {
struct Element {  // ReuseVertexPlanElement (ReusePlanGenerator.h:12-19)
  ConnType covered;
  double cost = 0.0;
  std::vector<uintV> g;
  uintV uj = 0;
};

// Tree-index search cost (ReusePlanGenerator.h:248-280).
double TreeSearchCost(const SearchSequence& seq, uintV ui, uintV uj, const std::vector<uintV>& g,
                      double tree_node) {
  size_t n = seq.size();
  std::vector<uintV> rank(n, (uintV)n);
  for (size_t i = 0; i < n; ++i) rank[seq[i]] = (uintV)i;
  size_t w = 0;
  for (; w < rank[uj]; ++w)
    if (g[seq[w]] != seq[w]) break;
  if (w == 0) return rank[uj] * std::log2(tree_node);
  double ret = (double)rank[ui] - (double)w;
  size_t j = rank[uj];
  if (j > w) ret += (j - w) * std::log2(tree_node);
  return ret;
}

// Every order-preserving embedding g of P_j into P_i with g(u2) = u1 that
// keeps backward adjacency (ReusePlanGenerator.h:285-379).
void Subsume(const SearchSequence& seq, const AllConnType& con, uintV u1, uintV u2,
             std::vector<std::vector<uintV>>& out) {
  size_t n = seq.size();
  std::vector<uintV> rank(n, (uintV)n);
  for (size_t i = 0; i < n; ++i) rank[seq[i]] = (uintV)i;
  out.clear();
  if (rank[u1] < rank[u2]) return;
  AllConnType bc;
  GetBackwardConnectivity(bc, con, seq);
  std::string mask(rank[u2] + 1, 1);
  mask.resize(rank[u1] + 1, 0);
  do {
    std::vector<uintV> pos;
    for (size_t i = 0; i < mask.size(); ++i)
      if (mask[i]) pos.push_back((uintV)i);
    std::vector<uintV> g(n, (uintV)n);
    for (size_t j = 0; j < pos.size(); ++j) g[seq[j]] = seq[pos[j]];
    bool valid = g[u2] == u1;
    for (size_t j = 0; j <= rank[u2]; ++j) {
      uintV from = seq[j], to = g[from];
      for (uintV pu : bc[from]) {
        uintV tp = g[pu];
        if (std::find(bc[to].begin(), bc[to].end(), tp) == bc[to].end()) valid = false;
      }
    }
    for (size_t j = 0; j < rank[u2]; ++j)
      if (!(rank[g[seq[j]]] < rank[g[seq[j + 1]]])) valid = false;
    if (valid) out.push_back(g);
  } while (std::prev_permutation(mask.begin(), mask.end()));
}

// Exhaustive minimum set cover over <32 candidate elements
// (MinimumSetCoverSolver::MinSetCover, ReusePlanGenerator.h:23-85).  The
// cost accumulates once per covered vertex, as in the reference.
void MinSetCover(const ConnType& universe, const std::vector<Element>& cand, std::vector<Element>& ans) {
  size_t m = cand.size();
  uint64_t umask = 0;
  for (uintV u : universe) umask |= 1ULL << u;
  for (uintV u : universe) {
    Element e;
    e.covered.push_back(u);
    ans.push_back(e);
  }
  double best = 0.0;
  for (size_t k = 1; k <= universe.size(); ++k) {
    if (k > ans.size()) break;
    std::string mask(k, 1);
    mask.resize(m, 0);
    do {
      uint64_t cm = 0;
      double cost = 0.0;
      for (size_t i = 0; i < mask.size(); ++i)
        if (mask[i])
          for (uintV u : cand[i].covered) {
            cm |= 1ULL << u;
            cost += cand[i].cost;
          }
      if ((cm & umask) == umask && (k < ans.size() || (k == ans.size() && cost < best))) {
        ans.clear();
        for (size_t i = 0; i < mask.size(); ++i)
          if (mask[i]) ans.push_back(cand[i]);
        best = cost;
      }
    } while (std::prev_permutation(mask.begin(), mask.end()));
  }
}

void VertexPlan(const SearchSequence& seq, const AllConnType& con, size_t i, double tree_node,
                VertexReusePlan& vp) {
  AllConnType bc;
  GetBackwardConnectivity(bc, con, seq);
  std::vector<Element> cand;
  for (uintV u : bc[seq[i]]) {
    Element e;
    e.covered.push_back(u);
    cand.push_back(e);
  }
  for (size_t j = 0; j < i; ++j) {
    if (bc[seq[j]].size() <= 1) continue;
    std::vector<std::vector<uintV>> maps;
    Subsume(seq, con, seq[i], seq[j], maps);
    for (auto& g : maps) {
      Element e;
      for (uintV u : bc[seq[j]]) e.covered.push_back(g[u]);
      e.g = g;
      e.uj = seq[j];
      e.cost = TreeSearchCost(seq, seq[i], seq[j], g, tree_node);
      cand.push_back(e);
    }
  }
  std::vector<Element> ans;
  MinSetCover(bc[seq[i]], cand, ans);
  for (auto& e : ans) {
    if (e.covered.size() == 1) {
      vp.separate.push_back(e.covered[0]);
    } else {
      ReuseConnMeta r;
      r.conn = e.covered;
      r.source_vertex = e.uj;
      r.source_conn = bc[e.uj];
      r.mapping = e.g;
      std::sort(r.conn.begin(), r.conn.end());
      std::sort(r.source_conn.begin(), r.source_conn.end());
      vp.reuse.push_back(r);
    }
  }
}

double EstimateCost(const SearchSequence& seq, const std::vector<VertexReusePlan>& plan,
                    const AllConnType& con, double avg_degree, double ratio, double tree_node) {
  AllConnType bc;
  GetBackwardConnectivity(bc, con, seq);
  size_t n = seq.size();
  std::vector<double> inst;
  double cur = 1;
  for (size_t i = 0; i < n; ++i) {
    if (!bc[seq[i]].empty()) cur *= avg_degree / bc.size();  // bc.size() == n (reference)
    inst.push_back(cur);
  }
  double ret = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double tm = 3 * inst[i], tc = 0;
    if (i > 0) {
      double bs = std::log2(avg_degree);
      double candidates;
      if (plan[i].reuse.empty()) {
        candidates = avg_degree;
      } else {
        double scale = 1;
        for (auto& r : plan[i].reuse)
          if (r.conn.size() > scale) scale = (double)r.conn.size();
        candidates = avg_degree / scale;
      }
      double alpha = candidates * bs;
      double w = (double)plan[i].separate.size() + (double)plan[i].reuse.size() - 1;
      double lambda = 0;
      for (auto& r : plan[i].reuse) lambda += TreeSearchCost(seq, seq[i], r.source_vertex, r.mapping, avg_degree);
      tc = ratio * inst[i - 1] * (alpha * w + lambda);
    }
    ret += tm + tc;
  }
  (void)tree_node;
  return ret;
}

void TransformIndexBased(VertexReusePlan& vp, const SearchSequence& seq) {
  size_t n = seq.size();
  std::vector<uintV> otn(n, (uintV)n);
  for (uintV u = 0; u < n; ++u) otn[seq[u]] = u;
  for (auto& r : vp.reuse) {
    for (auto& x : r.conn) x = otn[x];
    for (auto& x : r.source_conn) x = otn[x];
    r.source_vertex = otn[r.source_vertex];
    std::vector<uintV> nm(n, (uintV)n);
    for (uintV u = 0; u < n; ++u)
      if (r.mapping[u] < n) nm[otn[u]] = otn[r.mapping[u]];
    r.mapping.swap(nm);
  }
  for (auto& x : vp.separate) x = otn[x];
}

// One reuse meta of a hard-coded plan: the intersection over `source_conn`
// cached at level `source` is reused as the intersection over `conn` here;
// `pairs` map source-side pattern vertices to this side (the rest map to n).
// Index based, as the reference's hard-coded plans are.
struct HardMeta {
  std::vector<uintV> conn, source_conn;
  uintV source;
  std::vector<std::pair<uintV, uintV>> pairs;
};
struct HardLevel {
  std::vector<uintV> separate;
  std::vector<HardMeta> reuse;
};
struct HardPlan {
  std::vector<uintV> seq;
  std::vector<HardLevel> levels;  // levels 1..n-1 (level 0 has nothing)
};

ReuseConnMeta MakeMeta(const HardMeta& h, size_t n) {
  ReuseConnMeta r;
  r.conn = h.conn;
  r.source_conn = h.source_conn;
  r.source_vertex = h.source;
  r.mapping.assign(n, (uintV)n);
  for (auto& pr : h.pairs) r.mapping[pr.first] = pr.second;
  std::sort(r.conn.begin(), r.conn.end());
  std::sort(r.source_conn.begin(), r.source_conn.end());
  return r;
}

// The plans GPU_GPSM_REUSE runs by default (ReuseTraversalPlanHardcode::
// Generate, src/query/optimizer/ReuseTraversalPlanHardCode.h:9-72): Q0
// :74-84, Q2 :86-110, Q3 :112-132, Q5 (its Auto variant) :178-218, Q6
// :220-255, Q7 :257-282, Q8 :284-310, Q9 :346-375, Q10 :434-468, Q11
// :523-556, Q12 (Auto) :583-612, Q13 (Auto) :669-705.  The level shape is
// the same in every plan: level 1 intersects {0}, level 2 {0, 1}, and the
// cliques chain the previous level's cache.  Q1 and Q4 have none (the
// reference asserts).
bool HardcodedPlan(int t, size_t n, HardPlan& hp) {
  using P = std::pair<uintV, uintV>;
  auto ancestor = [](std::vector<uintV> conn, uintV source, uintV target) {
    HardMeta m{conn, conn, source, {}};
    for (uintV u = 0; u < source; ++u) m.pairs.push_back(P(u, u));
    m.pairs.push_back(P(source, target));
    return m;
  };
  auto mapped = [](std::vector<uintV> conn, uintV source, std::vector<P> pairs) {
    return HardMeta{conn, {0, 1}, source, pairs};
  };
  hp.seq.resize(n);
  for (size_t i = 0; i < n; ++i) hp.seq[i] = (uintV)i;
  hp.levels.assign(n, HardLevel());
  if (n > 1) hp.levels[1].separate = {0};
  if (n > 2) hp.levels[2].separate = {0, 1};
  switch (t) {
    case 0:
      return true;
    case 2:
      hp.seq = {0, 2, 1, 3};
      hp.levels[3].reuse = {ancestor({0, 1}, 2, 3)};
      return true;
    case 3:
    case 7:
    case 11:
      for (size_t k = 3; k < n; ++k) {
        std::vector<uintV> c;
        for (uintV x = 0; x + 1 < k; ++x) c.push_back(x);
        hp.levels[k].reuse = {ancestor(c, (uintV)(k - 1), (uintV)k)};
        hp.levels[k].separate = {(uintV)(k - 1)};
      }
      return true;
    case 5:
      hp.seq = {0, 2, 3, 4, 5, 1};
      hp.levels[3].reuse = {mapped({0, 2}, 2, {P(0, 0), P(1, 2), P(2, 3)})};
      hp.levels[4].reuse = {mapped({0, 3}, 2, {P(0, 0), P(1, 3), P(2, 4)})};
      hp.levels[5].reuse = {ancestor({0, 1}, 2, 5)};
      return true;
    case 6:
      hp.seq = {0, 3, 1, 2, 4};
      hp.levels[3].reuse = {ancestor({0, 1}, 2, 3)};
      hp.levels[3].separate = {2};
      hp.levels[4].reuse = {ancestor({0, 1}, 2, 4)};
      return true;
    case 8:
      hp.levels[3].reuse = {ancestor({0, 1}, 2, 3)};
      hp.levels[4].separate = {2, 3};
      return true;
    case 9:
      hp.levels[3].reuse = {ancestor({0, 1}, 2, 3)};
      hp.levels[4].reuse = {mapped({0, 2}, 2, {P(0, 0), P(1, 2), P(2, 4)})};
      return true;
    case 10:
      hp.seq = {0, 1, 2, 4, 3};
      hp.levels[3].reuse = {ancestor({0, 1}, 2, 3)};
      hp.levels[4].reuse = {mapped({0, 3}, 2, {P(0, 0), P(1, 3), P(2, 4)})};
      hp.levels[4].separate = {2};
      return true;
    case 12:
      hp.seq = {0, 1, 3, 2, 4};
      hp.levels[3].reuse = {ancestor({0, 1}, 2, 3)};
      hp.levels[3].separate = {2};
      hp.levels[4].reuse = {ancestor({0, 1, 2}, 3, 4)};
      return true;
    case 13:
      hp.seq = {0, 1, 2, 5, 4, 3};
      hp.levels[3].reuse = {mapped({0, 2}, 2, {P(0, 0), P(1, 2), P(2, 3)})};
      hp.levels[4].reuse = {mapped({1, 2}, 2, {P(0, 1), P(1, 2), P(2, 4)})};
      hp.levels[5].reuse = {ancestor({0, 1}, 2, 5)};
      return true;
    default:
      return false;
  }
}
}  // namespace

bool HasHardcodedReusePlan(int t) {
  HardPlan hp;
  return HardcodedPlan(t, 6, hp);
}

static void HardcodedReuse(int t, size_t n, SearchSequence& seq, std::vector<VertexReusePlan>& lv) {
  HardPlan hp;
  HardcodedPlan(t, n, hp);
  seq.assign(hp.seq.begin(), hp.seq.end());
  lv.assign(n, VertexReusePlan());
  for (size_t k = 0; k < n; ++k) {
    lv[k].separate.assign(hp.levels[k].separate.begin(), hp.levels[k].separate.end());
    for (auto& h : hp.levels[k].reuse) lv[k].reuse.push_back(MakeMeta(h, n));
  }
}

ReusePlan::ReusePlan(const Query& query, bool use_autogen) : q(&query), autogen(use_autogen) {
  const size_t n = query.n;
  if (!autogen) {
    if (!HasHardcodedReusePlan(query.type))
      Fail(SME_ERR_UNSUPPORTED_QUERY,
           "no hard-coded reuse plan for Q" + std::to_string(query.type) + " (use reuse_autogen=1)");
    HardcodedReuse(query.type, n, seq, levels);
  } else {
    // ReuseTraversalOptimizer::GenerateOrder: every connected match order,
    // cheapest by the reference's cost model.
    SearchSequence s(n);
    for (size_t i = 0; i < n; ++i) s[i] = (uintV)i;
    bool have = false;
    double best = 0;
    do {
      bool connected = true;
      std::vector<bool> vis(n, false);
      vis[s[0]] = true;
      for (size_t i = 1; i < n && connected; ++i) {
        bool any = false;
        for (uintV nu : query.con[s[i]])
          if (vis[nu]) any = true;
        connected = any;
        vis[s[i]] = true;
      }
      if (!connected) continue;
      std::vector<VertexReusePlan> plan(n);
      for (size_t i = 0; i < n; ++i) VertexPlan(s, query.con, i, 12.0, plan[i]);
      double c = EstimateCost(s, plan, query.con, 12.0, 10.0, 12.0);
      if (!have || best > c) {
        have = true;
        best = c;
        seq = s;
        levels = plan;
      }
    } while (std::next_permutation(s.begin(), s.end()));
    for (auto& vp : levels) TransformIndexBased(vp, seq);
  }
  Relabel(query, seq, con, order);
  cache_required.assign(n, false);
  for (uintV u = 0; u < n; ++u)
    for (uintV u2 = u + 1; u2 < n; ++u2)
      for (auto& r : levels[u2].reuse)
        if (r.source_vertex == u) cache_required[u] = true;
}

std::string ReusePlan::Describe() const {
  std::ostringstream os;
  os << "ReuseTraversalPlan Q" << q->type << (autogen ? " (autogen)" : " (hard-coded)")
     << " search sequence:";
  for (auto u : seq) os << " " << u;
  os << "\n";
  for (size_t i = 0; i < levels.size(); ++i) {
    os << "level " << i << ", vertex=" << seq[i] << ":intersect: ";
    size_t cnt = 0;
    for (auto& r : levels[i].reuse) {
      if (cnt++) os << " ";
      os << "[source_vertex=" << r.source_vertex << ",conn=(";
      for (size_t j = 0; j < r.conn.size(); ++j) os << (j ? "," : "") << r.conn[j];
      os << "),source_conn=(";
      for (size_t j = 0; j < r.source_conn.size(); ++j) os << (j ? "," : "") << r.source_conn[j];
      os << ")]";
    }
    for (auto s : levels[i].separate) {
      if (cnt++) os << " ";
      os << s;
    }
    os << (cache_required[i] ? "  (cached)" : "") << "\n";
  }
  // each reuse meta's vertex mapping (source side -> this side; n = none)
  for (size_t i = 0; i < levels.size(); ++i)
    for (auto& r : levels[i].reuse) {
      os << "mapping level " << i << ":";
      for (auto x : r.mapping) os << " " << x;
      os << "\n";
    }
  return os.str();
}

}  // namespace sme
