// Compiles a query under one of the three GPU plans into the level program
// run by the device engine.  One step per reference execute level:
//
//   GPU_GPSM        per level: intersect backward lists with the whole-ordered
//                   conditions, then materialise (Gpsm::JoinPhase,
//                   src/gpu/impl/gpsm/GPSMCheckConstraints.cuh:40-105).  The
//                   final level is counted instead of materialised unless
//                   instances are requested; the count is the same number as
//                   the size of the last level (IsProcessOver,
//                   src/gpu/impl/gpsm/HybridGPSMGPUProcessor.cuh:23-33).
//   GPU_LIGHT       the LIGHT execute sequence, op by op
//                   (HybridLIGHTGPUProcessor::ExecuteBatch,
//                   src/gpu/impl/light/HybridLIGHTGPUProcessor.cuh:147-228).
//   GPU_GPSM_REUSE  per level: when a later level reuses this level's
//                   intersection, the intersection is computed without the
//                   ordering conditions and kept as a cache while the level is
//                   materialised with the conditions (the "intersect-only"
//                   and "overall" outputs of GpsmReuseBinSearch,
//                   src/gpu/utils/ops/intersect/GPSMReuseBinSearch.cuh:167-221);
//                   a reusing level starts from the cached set of its
//                   ancestor and intersects the separate lists
//                   (GpsmReuse::JoinPhase, GPSMReuseCheckConstraints.cuh:166-338).
#include <algorithm>
#include <sstream>

#include "sme_internal.h"

namespace sme {

namespace {
std::vector<StepCond> Conds(const std::vector<CondType>& c) {
  std::vector<StepCond> r;
  for (auto& x : c) r.push_back(StepCond{(uint8_t)x.first, (uint8_t)x.second});
  return r;
}
std::vector<uint8_t> U8(const std::vector<uintV>& v) {
  return std::vector<uint8_t>(v.begin(), v.end());
}

// Tracks which vertices are materialised / hold live candidate sets.
struct State {
  std::vector<uint8_t> mat, sets;
  void AddMat(uint8_t u) { mat.push_back(u); }
  void AddSet(uint8_t u) {
    if (std::find(sets.begin(), sets.end(), u) == sets.end()) sets.push_back(u);
  }
  void DropSet(uint8_t u) { sets.erase(std::remove(sets.begin(), sets.end(), u), sets.end()); }
  void Stamp(Step& s) const {
    s.mat_after = mat;
    s.sets_after = sets;
  }
};

const char* KindName(StepKind k) {
  switch (k) {
    case S_INIT: return "INIT";
    case S_COMPUTE: return "COMPUTE";
    case S_MATERIALIZE: return "MATERIALIZE";
    case S_FILTER: return "FILTER_COMPUTE";
    case S_COMPUTE_COUNT: return "COMPUTE_COUNT";
    case S_PATH_COUNT: return "COMPUTE_PATH_COUNT";
    case S_COUNT: return "COUNT";
    case S_ALIAS: return "ALIAS";
  }
  return "?";
}

Program CompileGpsm(const Query& q, bool enumerate) {
  TraversalPlan tp(q);
  Program p;
  State st;
  p.n = q.n;
  for (int u = 0; u < q.n; ++u) p.out_slot.push_back((uint8_t)u);
  Step s0;
  s0.kind = S_INIT;
  s0.u = 0;
  st.AddMat(0);
  st.Stamp(s0);
  p.steps.push_back(s0);
  for (int u = 1; u < q.n; ++u) {
    bool last = u == q.n - 1;
    Step c;
    c.kind = (last && !enumerate) ? S_COMPUTE_COUNT : S_COMPUTE;
    c.u = (uint8_t)u;
    c.conn = U8(tp.ordered_conn[u]);
    c.cond = Conds(tp.whole_order[u]);
    if (c.kind == S_COMPUTE) st.AddSet((uint8_t)u);
    st.Stamp(c);
    p.steps.push_back(c);
    if (c.kind == S_COMPUTE) {
      Step m;
      m.kind = S_MATERIALIZE;
      m.u = (uint8_t)u;
      st.DropSet((uint8_t)u);
      st.AddMat((uint8_t)u);
      st.Stamp(m);
      p.steps.push_back(m);
    }
  }
  return p;
}

Program CompileReuse(const Query& q, bool autogen, bool enumerate) {
  ReusePlan rp(q, autogen);
  TraversalPlan tp(q);  // only for the helpers; reuse uses relabelled con
  (void)tp;
  Program p;
  State st;
  const int n = q.n;
  p.n = n;
  p.out_slot.resize(n);
  for (int i = 0; i < n; ++i) p.out_slot[i] = (uint8_t)rp.seq[i];
  // ordered (backward) connectivity and whole ordering of the relabelled
  // pattern (DevTraversalPlan built from the relabelled TraversalPlan).
  AllConnType oc(n);
  AllCondType wo(n);
  for (int u = 0; u < n; ++u) {
    for (uintV v : rp.con[u])
      if ((int)v < u) oc[u].push_back(v);
    for (int v = 0; v < u; ++v) wo[u].push_back(CondType(GetConditionType(u, v, rp.order), (uintV)v));
  }
  Step s0;
  s0.kind = S_INIT;
  s0.u = 0;
  st.AddMat(0);
  st.Stamp(s0);
  p.steps.push_back(s0);
  for (int u = 1; u < n; ++u) {
    const VertexReusePlan& vp = rp.levels[u];
    bool last = u == n - 1;
    Step c;
    c.u = (uint8_t)u;
    c.full_conn = U8(oc[u]);
    // Reuse one ancestor cache (identity mapping on the prefix).  A meta
    // whose mapping keeps level 0 and moves level 1 to an earlier vertex x
    // (the intersection N(M[0]) ∩ N(M[x]) cached at level 2 by the sibling
    // path (M[0], M[x])) is located at run time (FindCacheOffsets,
    // src/gpu/impl/common/CheckConstraintsReuseCommon.cuh:14-112); its
    // adjacency lists stay in `conn` for the paths whose sibling is not in
    // the current batch.  Any other meta is intersected from its lists.
    std::vector<uint8_t> conn = U8(vp.separate);
    std::vector<uint8_t> others = conn;  // lists not covered by the mapped meta
    int src = -1;
    const ReuseConnMeta* sib = nullptr;
    for (auto& r : vp.reuse) {
      bool ancestor = r.source_vertex < (uintV)u && r.mapping.size() == (size_t)n &&
                      r.mapping[r.source_vertex] == (uintV)u;
      for (uintV x = 0; ancestor && x < r.source_vertex; ++x)
        if (r.mapping[x] != x) ancestor = false;
      const bool sibling = !ancestor && !sib && r.source_vertex == 2 && r.mapping.size() == (size_t)n &&
                           r.source_conn == ConnType{0, 1} && r.mapping[0] == 0 && r.mapping[1] >= 2 &&
                           r.mapping[1] < (uintV)u && rp.cache_required[2];
      if (ancestor && src < 0 && rp.cache_required[r.source_vertex]) {
        src = (int)r.source_vertex;
      } else {
        for (uintV x : r.conn) conn.push_back((uint8_t)x);
        if (sibling) sib = &r;
        else
          for (uintV x : r.conn) others.push_back((uint8_t)x);
      }
    }
    std::sort(conn.begin(), conn.end());
    conn.erase(std::unique(conn.begin(), conn.end()), conn.end());
    c.conn = conn;
    c.reuse_src = (int8_t)src;
    if (sib) {
      // the cached set replaces exactly the meta's lists, none of which any
      // other source of this step also asks for
      bool clash = false;
      for (uintV x : sib->conn) clash = clash || std::count(others.begin(), others.end(), (uint8_t)x) > 0;
      if (!clash) {
        c.map_src = 2;
        c.map_x = (uint8_t)sib->mapping[1];
        for (size_t i = 0; i < conn.size(); ++i)
          if (std::count(sib->conn.begin(), sib->conn.end(), (uintV)conn[i])) c.map_mask |= (uint8_t)(1u << i);
      }
    }
    if (rp.cache_required[u] && !last) {
      // intersect-only result kept as the cache; conditions at materialise
      c.kind = S_COMPUTE;
      st.AddSet((uint8_t)u);
      st.Stamp(c);
      p.steps.push_back(c);
      Step m;
      m.kind = S_MATERIALIZE;
      m.u = (uint8_t)u;
      m.cond = Conds(wo[u]);
      m.keep_set = true;
      st.AddMat((uint8_t)u);
      st.Stamp(m);
      p.steps.push_back(m);
    } else {
      c.kind = (last && !enumerate) ? S_COMPUTE_COUNT : S_COMPUTE;
      c.cond = Conds(wo[u]);
      if (c.kind == S_COMPUTE) st.AddSet((uint8_t)u);
      st.Stamp(c);
      p.steps.push_back(c);
      if (c.kind == S_COMPUTE) {
        Step m;
        m.kind = S_MATERIALIZE;
        m.u = (uint8_t)u;
        st.DropSet((uint8_t)u);
        st.AddMat((uint8_t)u);
        st.Stamp(m);
        p.steps.push_back(m);
      }
    }
    // caches no longer referenced by a later level are dropped
    for (uint8_t s : std::vector<uint8_t>(st.sets)) {
      bool used = false;
      for (int k = u + 1; k < n; ++k)
        for (auto& r : rp.levels[k].reuse)
          if (r.source_vertex == s) used = true;
      if (!used) {
        st.DropSet(s);
        p.steps.back().sets_after = st.sets;
      }
    }
  }
  return p;
}

bool HasCond(const std::vector<StepCond>& v, uint8_t op, uint8_t operand) {
  for (auto& c : v)
    if (c.op == op && c.operand == operand) return true;
  return false;
}

// True when every x satisfying `c` (conditions against materialised
// vertices) also satisfies `need`.  Facts grow by transitivity through
// materialised vertices: x > M[a] and M[a] > M[b] (a relation M[a] was
// checked against, `known[a]`) give x > M[b]; likewise for <.  A strict
// order against v also gives x != M[v].
bool Implies(const std::vector<StepCond>& c, const std::vector<StepCond>& need, const std::vector<bool>& mat,
             const std::vector<std::vector<StepCond>>& known) {
  std::vector<StepCond> facts = c;
  for (size_t k = 0; k < facts.size(); ++k) {
    const StepCond f = facts[k];
    if (f.op == NON_EQUAL || !mat[f.operand]) continue;
    for (const StepCond& r : known[f.operand])
      if (r.op == f.op && !HasCond(facts, f.op, r.operand)) facts.push_back(StepCond{f.op, r.operand});
  }
  for (const StepCond& x : need) {
    bool ok = HasCond(facts, x.op, x.operand) ||
              (x.op == NON_EQUAL && (HasCond(facts, LESS_THAN, x.operand) || HasCond(facts, LARGER_THAN, x.operand)));
    if (!ok) return false;
  }
  return true;
}

// Candidate-set reuse for the LIGHT sequence.  The reference computes every
// candidate set from adjacency lists.  When an earlier candidate set of w
// was intersected from lists T ⊆ S (S = the lists of u) and every condition
// that set was filtered by follows from u's own conditions, then
// set(u) = set(w) ∩ lists(S \ T) under u's conditions: the same set from
// fewer, shorter inputs.  On the clique queries this turns the k-way
// intersection at every level into one 2-way step.  Returns, per sequence
// entry, the vertex whose set the entry starts from (-1 none).
std::vector<int> PlanSetReuse(const LazyPlan& lp, const Query& q, std::vector<int>& last_use_after_mat,
                              std::vector<std::vector<uint8_t>>& covered) {
  const size_t E = lp.exec.size();
  std::vector<int> from(E, -1);
  covered.assign(E, {});
  std::vector<bool> mat(q.n, false), live(q.n, false), has(q.n, false);
  std::vector<std::vector<uint8_t>> lists(q.n);
  std::vector<std::vector<StepCond>> cset(q.n), known(q.n);
  last_use_after_mat.assign(q.n, -1);
  for (size_t i = 0; i < E; ++i) {
    const LazyOp op = lp.exec[i].first;
    const uint8_t u = (uint8_t)lp.exec[i].second;
    if (op == L_MATERIALIZE) {
      if (i > 0) {
        known[u] = cset[u];
        for (const StepCond& c : Conds(lp.materialize_cond[u])) known[u].push_back(c);
      }
      mat[u] = true;
      live[u] = false;
    } else if (op == L_FILTER_COMPUTE) {
      for (const StepCond& c : Conds(lp.filter_cond[u])) cset[u].push_back(c);
    } else if (op == L_COMPUTE || op == L_COMPUTE_PATH_COUNT || op == L_COMPUTE_COUNT) {
      const std::vector<uint8_t> S = U8(lp.backward_conn[u]);
      const std::vector<StepCond> C = Conds(lp.compute_cond[u]);
      int best = -1;
      for (int w = 0; w < q.n; ++w) {
        if (w == u || !has[w] || !(live[w] || mat[w])) continue;
        if (lists[w].size() < 2 || (best >= 0 && lists[w].size() <= lists[best].size())) continue;
        bool subset = true;
        for (uint8_t t : lists[w])
          if (std::find(S.begin(), S.end(), t) == S.end()) subset = false;
        if (subset && Implies(C, cset[w], mat, known)) best = w;
      }
      from[i] = best;
      if (best >= 0) covered[i] = lists[best];
      if (best >= 0 && mat[best]) last_use_after_mat[best] = (int)i;
      if (op == L_COMPUTE) {
        has[u] = live[u] = true;
        lists[u] = S;
        cset[u] = C;
        if (best >= 0)
          for (const StepCond& c : cset[best]) cset[u].push_back(c);
      }
    }
  }
  return from;
}

// Drops `!=` conditions that the strict ones already imply (x > M[w] with
// M[w] > M[v] gives x != M[v]): the clique plans fill every unordered pair
// with NON_EQUAL, yet their total order makes those checks dead.  Steps
// without `!=` run the intersection without an exclusion array.
void PruneImpliedExclusions(Program& p, bool loop_free) {
  const int n = p.n;
  std::vector<bool> mat(n, false);
  std::vector<std::vector<StepCond>> cset(n), known(n);
  for (Step& s : p.steps) {
    const uint8_t u = s.u;
    // facts every candidate of this step satisfies besides its own `!=`
    std::vector<StepCond> strict;
    for (const StepCond& c : s.cond)
      if (c.op != NON_EQUAL) strict.push_back(c);
    if (s.kind == S_MATERIALIZE || s.kind == S_FILTER)
      for (const StepCond& c : cset[u])
        if (c.op != NON_EQUAL) strict.push_back(c);
    // lists the candidates are drawn from (a reused set stands for its lists)
    const std::vector<uint8_t>& lists = s.full_conn.empty() ? s.conn : s.full_conn;
    const bool intersects = s.kind == S_COMPUTE || s.kind == S_COMPUTE_COUNT || s.kind == S_PATH_COUNT;
    std::vector<StepCond> kept;
    for (const StepCond& c : s.cond) {
      bool dead = c.op == NON_EQUAL && mat[c.operand] &&
                  (Implies(strict, {StepCond{LESS_THAN, c.operand}}, mat, known) ||
                   Implies(strict, {StepCond{LARGER_THAN, c.operand}}, mat, known));
      // x in N(M[v]) and no self loop: x != M[v]
      if (c.op == NON_EQUAL && loop_free && intersects &&
          std::find(lists.begin(), lists.end(), c.operand) != lists.end())
        dead = true;
      if (!dead) kept.push_back(c);
    }
    // bookkeeping uses the full condition lists (facts, not checks)
    switch (s.kind) {
      case S_INIT:
        mat[u] = true;
        break;
      case S_COMPUTE:
        cset[u] = s.cond;
        if (s.reuse_src >= 0)
          for (const StepCond& c : cset[s.reuse_src]) cset[u].push_back(c);
        break;
      case S_FILTER:
        for (const StepCond& c : s.cond) cset[u].push_back(c);
        break;
      case S_MATERIALIZE:
        known[u] = cset[u];
        for (const StepCond& c : s.cond) known[u].push_back(c);
        mat[u] = true;
        break;
      default:
        break;
    }
    s.cond = kept;
  }
}

// LIGHT: the reference execute sequence; for enumeration the counting tail
// is replaced by materialising every vertex (conditions recomputed by the
// same utilities, so each pair of pattern vertices is still checked once).
Program CompileLight(const Query& q, int compress_level, bool enumerate, bool set_reuse) {
  LazyPlan lp(q, compress_level);
  if (enumerate) {
    std::vector<LazyEntry> e;
    for (auto x : lp.exec) {
      if (x.first == L_COUNT) continue;
      if (x.first == L_COMPUTE_COUNT || x.first == L_COMPUTE_PATH_COUNT) x.first = L_COMPUTE;
      e.push_back(x);
    }
    std::vector<bool> mat(q.n, false);
    for (auto& x : e)
      if (x.first == L_MATERIALIZE) mat[x.second] = true;
    for (auto& x : std::vector<LazyEntry>(e))
      if (x.first == L_COMPUTE && !mat[x.second]) {
        e.push_back(LazyEntry(L_MATERIALIZE, x.second));
        mat[x.second] = true;
      }
    lp.exec = e;
    // recompute per-level sets and conditions for the new sequence
    LazyPlan fresh(q, compress_level);
    fresh.exec = e;
    LightConstraintsFor(fresh);
    lp = fresh;
  }
  Program p;
  State st;
  p.n = q.n;
  for (int u = 0; u < q.n; ++u) p.out_slot.push_back((uint8_t)u);
  const bool direct_ok = lp.compress_level == SME_COMPRESS_SPECIAL && q.type <= 11 && q.type != 4 &&
                         q.type != 9;  // CanDirectCount, LIGHTDirectCount.cuh:13-19
  std::vector<int> last_use(q.n, -1);
  std::vector<int> from(lp.exec.size(), -1);
  std::vector<std::vector<uint8_t>> covered(lp.exec.size());
  if (set_reuse) from = PlanSetReuse(lp, q, last_use, covered);
  // lists of a compute entry: all backward lists, or those its reused set
  // does not cover (full_conn keeps all of them)
  auto lists_of = [&](size_t i, uint8_t u, Step& s) {
    s.conn = U8(lp.backward_conn[u]);
    if (from[i] < 0) return;
    const uint8_t w = (uint8_t)from[i];
    s.full_conn = s.conn;
    s.reuse_src = (int8_t)w;
    std::vector<uint8_t> rest;
    for (uint8_t t : s.conn)
      if (std::find(covered[i].begin(), covered[i].end(), t) == covered[i].end()) rest.push_back(t);
    s.conn = rest;
  };
  for (size_t i = 0; i < lp.exec.size(); ++i) {
    LazyOp op = lp.exec[i].first;
    uint8_t u = (uint8_t)lp.exec[i].second;
    Step s;
    s.u = u;
    switch (op) {
      case L_MATERIALIZE:
        if (i == 0) {
          s.kind = S_INIT;
        } else {
          s.kind = S_MATERIALIZE;
          s.cond = Conds(lp.materialize_cond[u]);
          // a set reused after this point stays with the children
          s.keep_set = last_use[u] > (int)i;
          if (!s.keep_set) st.DropSet(u);
          for (int w = 0; w < q.n; ++w)
            if (w != u && last_use[w] >= 0 && last_use[w] < (int)i) st.DropSet((uint8_t)w);
        }
        st.AddMat(u);
        break;
      case L_COMPUTE:
      case L_COMPUTE_PATH_COUNT:
        s.kind = op == L_COMPUTE ? S_COMPUTE : S_PATH_COUNT;
        lists_of(i, u, s);
        s.cond = Conds(lp.compute_cond[u]);
        st.AddSet(u);
        break;
      case L_FILTER_COMPUTE:
        s.kind = S_FILTER;
        s.cond = Conds(lp.filter_cond[u]);
        break;
      case L_COMPUTE_COUNT: {
        s.kind = S_COMPUTE_COUNT;
        lists_of(i, u, s);
        s.cond = Conds(lp.compute_cond[u]);
        auto& um = lp.computed_unmaterialized[i];
        if (um.size() > 1) Fail(SME_ERR_UNSUPPORTED_QUERY, "COMPUTE_COUNT with >1 unmaterialized vertex");
        if (um.size() == 1) {
          s.with_u = (int8_t)um[0];
          s.with_op = (uint8_t)GetConditionType(u, um[0], q.order);
        }
        break;
      }
      case L_COUNT: {
        s.kind = S_COUNT;
        s.unmat = U8(lp.computed_unmaterialized[i]);
        s.direct = direct_ok;
        if (!s.direct && s.unmat.size() == 2)
          s.pair_op = (uint8_t)GetConditionType(s.unmat[0], s.unmat[1], q.order);
        if (!s.direct && (s.unmat.empty() || s.unmat.size() > 2))
          Fail(SME_ERR_UNSUPPORTED_QUERY, "COUNT over " + std::to_string(s.unmat.size()) +
                                              " unmaterialized vertices");
        break;
      }
    }
    st.Stamp(s);
    p.steps.push_back(s);
  }
  return p;
}
}  // namespace

// A mapped reuse step finds its sibling's cached set by the rank of the
// sibling's level-1 vertex in N(M[0]).  That holds only while the level-1
// candidates of a root are all of N(M[0]) in order (COMPUTE(1) over {0}
// with no condition, MATERIALIZE(1) with none) and the level-2 cache is the
// plain intersection N(M[0]) ∩ N(M[1]); otherwise the step keeps its lists.
// A COMPUTE or COMPUTE_PATH_COUNT that repeats an earlier step of the same
// kind (same lists, reused set and conditions) while that step's set is
// still live computes the same set for every path: it becomes an alias of
// that set.  The diamond's LIGHT plan counts N(u0) ∩ N(u2) twice
// (COMPUTE_PATH_COUNT for u1 and for u3, LazyTraversalPlanGenerator.h:266-274);
// the second is now free.
static void AliasRepeatedComputes(Program& p) {
  for (size_t k = 1; k < p.steps.size(); ++k) {
    Step& s = p.steps[k];
    if ((s.kind != S_COMPUTE && s.kind != S_PATH_COUNT) || s.with_u >= 0 || s.map_src >= 0) continue;
    const std::vector<uint8_t>& live = p.steps[k - 1].sets_after;
    for (size_t j = 0; j < k; ++j) {
      const Step& e = p.steps[j];
      if (e.kind != s.kind || e.conn != s.conn || e.reuse_src != s.reuse_src || e.map_src >= 0 ||
          std::find(live.begin(), live.end(), e.u) == live.end())
        continue;
      bool same = e.cond.size() == s.cond.size();
      for (size_t i = 0; same && i < s.cond.size(); ++i)
        same = e.cond[i].op == s.cond[i].op && e.cond[i].operand == s.cond[i].operand;
      if (!same) continue;
      s.kind = S_ALIAS;
      s.alias_of = (int8_t)e.u;
      break;
    }
  }
}

static void RequireSiblingLayout(Program& p) {
  auto find = [&](StepKind k, uint8_t u) -> const Step* {
    for (const Step& s : p.steps)
      if (s.kind == k && s.u == u) return &s;
    return nullptr;
  };
  const Step* c1 = find(S_COMPUTE, 1);
  const Step* m1 = find(S_MATERIALIZE, 1);
  const Step* c2 = find(S_COMPUTE, 2);
  // level 1 may clip N(M[0]) by one order condition against M[0] (the clip
  // cancels out of the rank difference once M[x] passes it)
  const bool clip = c1 && c1->cond.size() == 1 && c1->cond[0].operand == 0 && c1->cond[0].op != OP_NONE &&
                    c1->cond[0].op != 2;
  const bool ok = c1 && m1 && c2 && (c1->cond.empty() || clip) && m1->cond.empty() && c1->reuse_src < 0 &&
                  c1->conn == std::vector<uint8_t>{0} && c2->cond.empty() && c2->reuse_src < 0 &&
                  c2->conn == std::vector<uint8_t>{0, 1};
  for (Step& s : p.steps) {
    if (s.map_src < 0) continue;
    if (!ok) {
      s.map_src = -1;
      s.map_x = 0;
      s.map_mask = 0;
    } else {
      s.map_op = clip ? c1->cond[0].op : OP_NONE;
    }
  }
}

Program Compile(const sme_opts& o, bool enumerate, bool loop_free) {
  Query q(o.query_type, o.enable_ordering != 0);
  Program p;
  switch (o.algo) {
    case SME_GPU_GPSM:
      p = CompileGpsm(q, enumerate);
      break;
    case SME_GPU_GPSM_REUSE: {
      bool autogen = o.reuse_autogen == 1 || (o.reuse_autogen < 0 && !HasHardcodedReusePlan(q.type));
      p = CompileReuse(q, autogen, enumerate);
      break;
    }
    case SME_GPU_LIGHT:
      if (o.compress_level < 0 || o.compress_level > 3)
        Fail(SME_ERR_INVALID_ARG, "compress_level must be 0..3");
      p = CompileLight(q, o.compress_level, enumerate, o.no_set_reuse == 0);
      break;
    default:
      Fail(SME_ERR_INVALID_ARG, "algo must be 4 (GPU_GPSM), 5 (GPU_GPSM_REUSE) or 6 (GPU_LIGHT)");
  }
  p.query_type = q.type;
  p.algo = o.algo;
  p.enumerate = enumerate;
  PruneImpliedExclusions(p, loop_free);
  RequireSiblingLayout(p);
  if (!enumerate) AliasRepeatedComputes(p);
  for (auto& s : p.steps) {
    std::ostringstream os;
    os << KindName(s.kind) << "(" << (int)s.u << ")";
    s.label = os.str();
  }
  return p;
}

bool IsOrderedClique(const Query& q) {
  if (!q.enable_ordering) return false;
  for (int u = 0; u < q.n; ++u) {
    if ((int)q.con[u].size() != q.n - 1) return false;
    if (u + 1 < q.n && GetConditionType((uintV)u, (uintV)(u + 1), q.order) != LESS_THAN) return false;
  }
  return true;
}

void RequireOrientable(const Program& p, bool enable_ordering) {
  Query q(p.query_type, enable_ordering);
  if (!IsOrderedClique(q))
    Fail(SME_ERR_UNSUPPORTED_QUERY,
         "an oriented graph holds each edge once: only the clique queries (0, 3, 7, 11) with symmetry "
         "breaking count on it");
  // every list a step reads must belong to a vertex that precedes u in the
  // total order, so the forward list holds all of u's candidates
  for (const Step& s : p.steps) {
    auto before = [&](uint8_t w) { return p.out_slot[w] < p.out_slot[s.u]; };
    for (uint8_t w : s.conn)
      if (!before(w)) Fail(SME_ERR_UNSUPPORTED_QUERY, "plan reads a list against the orientation");
    for (uint8_t w : s.full_conn)
      if (!before(w)) Fail(SME_ERR_UNSUPPORTED_QUERY, "plan reads a list against the orientation");
  }
}

std::string Program::Describe() const {
  std::ostringstream os;
  os << "program Q" << query_type << " algo=" << algo << (enumerate ? " enumerate" : " count") << "\n";
  for (size_t i = 0; i < steps.size(); ++i) {
    const Step& s = steps[i];
    os << i << ": " << s.label;
    if (!s.conn.empty()) {
      os << " conn=(";
      for (size_t j = 0; j < s.conn.size(); ++j) os << (j ? "," : "") << (int)s.conn[j];
      os << ")";
    }
    if (s.reuse_src >= 0) os << " reuse=" << (int)s.reuse_src;
    if (s.map_src >= 0)
      os << " sibling=(" << (int)s.map_src << ",x=" << (int)s.map_x
         << (s.map_op == 0 ? ",<0" : s.map_op == 1 ? ",>0" : "") << ")";
    if (!s.cond.empty()) {
      os << " cond=(";
      for (size_t j = 0; j < s.cond.size(); ++j)
        os << (j ? "," : "") << (s.cond[j].op == 0 ? "<" : s.cond[j].op == 1 ? ">" : "!=")
           << (int)s.cond[j].operand;
      os << ")";
    }
    if (s.with_u >= 0) os << " with=" << (int)s.with_u;
    if (s.kind == S_ALIAS) os << " of=" << (int)s.alias_of;
    if (s.kind == S_COUNT) os << (s.direct ? " direct" : " general");
    if (s.keep_set) os << " keep";
    os << " | mat=(";
    for (size_t j = 0; j < s.mat_after.size(); ++j) os << (j ? "," : "") << (int)s.mat_after[j];
    os << ") sets=(";
    for (size_t j = 0; j < s.sets_after.size(); ++j) os << (j ? "," : "") << (int)s.sets_after[j];
    os << ")\n";
  }
  return os.str();
}

}  // namespace sme
