/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle of the subgraph-enumeration
 * path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load this library, and only as the checker.  The product (libsme.so)
 * never links or calls it.
 *
 * A plain-C restatement of the reference's CPU worst-case-optimal join
 * (CPU_WCOJ):
 *   DFS over pattern vertices in identity order      src/cpu/CPUWCOJ.h:77-106
 *   root loop, OpenMP dynamic schedule                src/cpu/CPUWCOJ.h:37-52
 *   m-way sorted merge intersection                   src/cpu/common/CPUIntersection.h:14-34, :177-212
 *   ordering check (< / >) and injectivity           src/cpu/common/CPUFilter.h:7-34
 *   backward connectivity / ordering (smaller ids)    src/query/common/Plan.h:60-88
 *   patterns Q0..Q13 and their symmetry breaking      src/query/common/Query.h:84-434
 *
 * Parity of this restatement is pinned against the reference's own
 * patternmatchcpu binary (built from source by oracle/Makefile into
 * oracle/_ref/) on the committed golden graphs: tests/golden/.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXQ 6

typedef struct {
  int n;
  int nbr[MAXQ][MAXQ]; /* adjacency, reference per-vertex order */
  int nn[MAXQ];
  char op[MAXQ][MAXQ]; /* op[u][v]: 'L' u<v, 'G' u>v, 0 none */
} pattern_t;

/* edge list + order pairs of each query, same tables as Query.h */
static void add_edge(pattern_t* p, int u, int v) { p->nbr[u][p->nn[u]++] = v; }
static void add_ord(pattern_t* p, int u, char o, int v) { p->op[u][v] = o; }

static int build_pattern(int q, pattern_t* p) {
  memset(p, 0, sizeof(*p));
#define E(u, v) add_edge(p, u, v)
#define O(u, o, v) add_ord(p, u, o, v)
  switch (q) {
    case 0:
      p->n = 3;
      E(0, 1); E(0, 2); E(1, 0); E(1, 2); E(2, 0); E(2, 1);
      O(0, 'L', 1); O(1, 'G', 0); O(1, 'L', 2); O(2, 'G', 1);
      break;
    case 1:
      p->n = 4;
      E(0, 1); E(0, 3); E(1, 0); E(1, 2); E(2, 1); E(2, 3); E(3, 0); E(3, 2);
      O(0, 'L', 1); O(0, 'L', 2); O(0, 'L', 3); O(1, 'G', 0); O(1, 'L', 3);
      O(2, 'G', 0); O(3, 'G', 0); O(3, 'G', 1);
      break;
    case 2:
      p->n = 4;
      E(0, 1); E(0, 2); E(0, 3); E(1, 0); E(1, 2); E(2, 0); E(2, 1); E(2, 3); E(3, 0); E(3, 2);
      O(0, 'L', 2); O(1, 'L', 3); O(2, 'G', 0); O(3, 'G', 1);
      break;
    case 3:
      p->n = 4;
      for (int u = 0; u < 4; ++u)
        for (int v = 0; v < 4; ++v)
          if (u != v) E(u, v);
      O(0, 'L', 1); O(1, 'G', 0); O(1, 'L', 2); O(2, 'G', 1); O(2, 'L', 3); O(3, 'G', 2);
      break;
    case 4:
      p->n = 5;
      E(0, 1); E(0, 2); E(1, 0); E(1, 2); E(1, 3); E(2, 0); E(2, 1); E(2, 4); E(3, 1); E(3, 4);
      E(4, 2); E(4, 3);
      O(1, 'L', 2); O(2, 'G', 1);
      break;
    case 5:
      p->n = 6;
      E(0, 1); E(0, 2); E(0, 3); E(0, 4); E(0, 5); E(1, 0); E(1, 2); E(2, 0); E(2, 1); E(2, 3);
      E(3, 0); E(3, 2); E(3, 4); E(4, 0); E(4, 3); E(4, 5); E(5, 0); E(5, 4);
      O(2, 'L', 4); O(4, 'G', 2);
      break;
    case 6:
      p->n = 5;
      E(0, 1); E(0, 2); E(0, 3); E(0, 4); E(1, 0); E(1, 2); E(1, 3); E(2, 0); E(2, 1); E(2, 3);
      E(3, 0); E(3, 1); E(3, 2); E(3, 4); E(4, 0); E(4, 3);
      O(0, 'L', 3); O(3, 'G', 0); O(1, 'L', 2); O(2, 'G', 1);
      break;
    case 7:
      p->n = 5;
      for (int u = 0; u < 5; ++u)
        for (int v = 0; v < 5; ++v)
          if (u != v) E(u, v);
      for (int i = 0; i < 4; ++i) {
        O(i, 'L', i + 1);
        O(i + 1, 'G', i);
      }
      break;
    case 8:
      p->n = 5;
      E(0, 1); E(0, 2); E(0, 3); E(1, 0); E(1, 2); E(1, 3); E(2, 0); E(2, 1); E(2, 4); E(3, 0);
      E(3, 1); E(3, 4); E(4, 2); E(4, 3);
      O(0, 'L', 1); O(1, 'G', 0); O(2, 'L', 3); O(3, 'G', 2);
      break;
    case 9:
      p->n = 5;
      for (int i = 1; i <= 4; ++i) {
        E(0, i);
        E(i, 0);
      }
      E(1, 3); E(3, 1); E(1, 2); E(2, 1); E(2, 4); E(4, 2);
      O(1, 'L', 2); O(2, 'G', 1);
      break;
    case 10:
      p->n = 5;
      E(0, 1); E(0, 2); E(0, 3); E(0, 4); E(1, 0); E(1, 2); E(1, 4); E(2, 0); E(2, 1); E(2, 3);
      E(3, 0); E(3, 2); E(3, 4); E(4, 0); E(4, 1); E(4, 3);
      O(1, 'L', 2); O(1, 'L', 3); O(1, 'L', 4); O(2, 'L', 4); O(2, 'G', 1); O(3, 'G', 1);
      O(4, 'G', 1); O(4, 'G', 2);
      break;
    case 11:
      p->n = 6;
      for (int u = 0; u < 6; ++u)
        for (int v = 0; v < 6; ++v)
          if (u != v) E(u, v);
      for (int i = 0; i < 5; ++i) {
        O(i, 'L', i + 1);
        O(i + 1, 'G', i);
      }
      break;
    case 12:
      p->n = 5;
      E(0, 1); E(0, 2); E(0, 3); E(0, 4); E(1, 0); E(1, 2); E(1, 3); E(1, 4); E(3, 0); E(3, 1);
      E(3, 2); E(3, 4); E(2, 0); E(2, 1); E(2, 3); E(4, 0); E(4, 1); E(4, 3);
      O(0, 'L', 1); O(2, 'L', 4); O(1, 'G', 0); O(4, 'G', 2);
      break;
    case 13:
      p->n = 6;
      E(0, 1); E(0, 2); E(0, 3); E(0, 5); E(1, 0); E(1, 2); E(1, 3); E(1, 4); E(2, 0); E(2, 1);
      E(2, 4); E(2, 5); E(3, 0); E(3, 1); E(4, 1); E(4, 2); E(5, 0); E(5, 2);
      O(0, 'L', 1); O(1, 'L', 2); O(1, 'G', 0); O(2, 'G', 1);
      break;
    default:
      return -1;
  }
#undef E
#undef O
  return 0;
}

typedef struct {
  int n;
  int nbk[MAXQ];       /* backward neighbours (smaller id), reference order */
  int bk[MAXQ][MAXQ];
  int ncond[MAXQ];     /* ordering vs smaller ids (GetOrderedOrdering) */
  char cop[MAXQ][MAXQ];
  int cvar[MAXQ][MAXQ];
} plan_t;

static void make_plan(const pattern_t* p, int ordering, plan_t* pl) {
  memset(pl, 0, sizeof(*pl));
  pl->n = p->n;
  for (int u = 0; u < p->n; ++u) {
    for (int j = 0; j < p->nn[u]; ++j)
      if (p->nbr[u][j] < u) pl->bk[u][pl->nbk[u]++] = p->nbr[u][j];
    if (!ordering) continue;
    for (int v = 0; v < u; ++v)
      if (p->op[u][v]) {
        pl->cop[u][pl->ncond[u]] = p->op[u][v];
        pl->cvar[u][pl->ncond[u]++] = v;
      }
  }
}

typedef struct {
  const uint64_t* rp;
  const uint32_t* cols;
  uint64_t nv;
  const plan_t* pl;
  uint32_t* out;     /* optional instance output */
  uint64_t cap;
  uint64_t* pos;     /* shared output cursor */
  double deadline;   /* omp_get_wtime() limit of a time-bounded sample (0: none) */
  int* aborted;      /* set when the deadline cut a root short (per thread) */
} ctx_t;

static int expired(const ctx_t* c) {
#ifdef _OPENMP
  return c->deadline > 0 && omp_get_wtime() > c->deadline;
#else
  (void)c;
  return 0;
#endif
}

/* two-pointer merge of sorted a and b into out; returns size */
static uint64_t merge(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb, uint32_t* out) {
  uint64_t i = 0, j = 0, k = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j]) ++i;
    else if (a[i] > b[j]) ++j;
    else {
      out[k++] = a[i];
      ++i;
      ++j;
    }
  }
  return k;
}

static uint64_t dfs(const ctx_t* c, int level, uint32_t* path, uint32_t* buf) {
  const plan_t* pl = c->pl;
  if (level == pl->n) {
    if (c->out) {
      uint64_t at;
#pragma omp atomic capture
      at = (*c->pos)++;
      if (at < c->cap) memcpy(c->out + at * pl->n, path, sizeof(uint32_t) * pl->n);
    }
    return 1;
  }
  /* candidates = intersection of backward neighbours' lists */
  uint64_t maxd = 0;
  for (int j = 0; j < pl->nbk[level]; ++j) {
    uint32_t v = path[pl->bk[level][j]];
    uint64_t d = c->rp[v + 1] - c->rp[v];
    if (d > maxd) maxd = d;
  }
  uint32_t* cand = buf;
  uint32_t* tmp = buf + maxd;
  uint32_t* next = buf + 2 * maxd;
  uint64_t nc = 0;
  if (pl->nbk[level] == 0) {
    return 0; /* every Q0..Q13 vertex has a smaller neighbour */
  }
  {
    uint32_t v = path[pl->bk[level][0]];
    nc = c->rp[v + 1] - c->rp[v];
    memcpy(cand, c->cols + c->rp[v], sizeof(uint32_t) * nc);
  }
  for (int j = 1; j < pl->nbk[level]; ++j) {
    uint32_t v = path[pl->bk[level][j]];
    nc = merge(c->cols + c->rp[v], c->rp[v + 1] - c->rp[v], cand, nc, tmp);
    uint32_t* t = cand;
    cand = tmp;
    tmp = t;
  }
  uint64_t ans = 0;
  for (uint64_t i = 0; i < nc; ++i) {
    uint32_t x = cand[i];
    int ok = 1;
    for (int k = 0; k < pl->ncond[level] && ok; ++k) {
      uint32_t y = path[pl->cvar[level][k]];
      if (pl->cop[level][k] == 'L' && !(x < y)) ok = 0;
      if (pl->cop[level][k] == 'G' && !(x > y)) ok = 0;
    }
    for (int k = 0; k < level && ok; ++k)
      if (path[k] == x) ok = 0;
    if (!ok) continue;
    if (level <= 2 && c->aborted && expired(c)) {
      *c->aborted = 1;
      return ans;
    }
    path[level] = x;
    ans += dfs(c, level + 1, path, next);
  }
  return ans;
}

static uint64_t max_degree(const uint64_t* rp, uint64_t nv) {
  uint64_t d = 0;
  for (uint64_t u = 0; u < nv; ++u)
    if (rp[u + 1] - rp[u] > d) d = rp[u + 1] - rp[u];
  return d;
}

/* Number of pattern vertices of query q, or -1. */
int oracle_query_size(int q) {
  pattern_t p;
  if (build_pattern(q, &p)) return -1;
  return p.n;
}

/*
 * Counts (and optionally lists) the instances of query q over roots
 * [root_begin, root_end) of the CSR graph.  Instances are written in DFS
 * order per root (not globally sorted) as q-vertex tuples u0..u_{k-1}; the
 * return value is the count (or (uint64)-1 on a bad query).  threads <= 0
 * uses the OpenMP default.
 */
uint64_t oracle_wcoj(const uint64_t* rp, const uint32_t* cols, uint64_t nv, int q, int ordering,
                     uint64_t root_begin, uint64_t root_end, int threads, uint32_t* out, uint64_t cap,
                     uint64_t* n_written) {
  pattern_t p;
  if (build_pattern(q, &p)) return (uint64_t)-1;
  plan_t pl;
  make_plan(&p, ordering, &pl);
  if (root_end > nv || root_end == 0) root_end = nv;
  uint64_t pos = 0;
  ctx_t c = {rp, cols, nv, &pl, out, cap, &pos};
  uint64_t maxd = max_degree(rp, nv);
  size_t per_thread = (size_t)(3 * maxd + 3) * (size_t)(MAXQ + 1);
  uint64_t total = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel reduction(+ : total)
  {
    uint32_t* buf = (uint32_t*)malloc(sizeof(uint32_t) * per_thread);
    uint32_t path[MAXQ];
#pragma omp for schedule(dynamic, 64)
    for (long long u = (long long)root_begin; u < (long long)root_end; ++u) {
      path[0] = (uint32_t)u;
      total += dfs(&c, 1, path, buf);
    }
    free(buf);
  }
  if (n_written) *n_written = pos;
  return total;
}

/*
 * Strided root sample: counts instances rooted at r = offset + k*stride for
 * all k with r < nv (the bounded CPU-baseline sample of a large graph).
 */
uint64_t oracle_wcoj_strided(const uint64_t* rp, const uint32_t* cols, uint64_t nv, int q, int ordering,
                             uint64_t stride, uint64_t offset, int threads) {
  pattern_t p;
  if (build_pattern(q, &p) || stride == 0) return (uint64_t)-1;
  plan_t pl;
  make_plan(&p, ordering, &pl);
  uint64_t pos = 0;
  ctx_t c = {rp, cols, nv, &pl, NULL, 0, &pos};
  uint64_t maxd = max_degree(rp, nv);
  size_t per_thread = (size_t)(3 * maxd + 3) * (size_t)(MAXQ + 1);
  uint64_t total = 0;
  long long cnt = offset < nv ? (long long)((nv - offset + stride - 1) / stride) : 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel reduction(+ : total)
  {
    uint32_t* buf = (uint32_t*)malloc(sizeof(uint32_t) * per_thread);
    uint32_t path[MAXQ];
#pragma omp for schedule(dynamic, 1)
    for (long long k = 0; k < cnt; ++k) {
      path[0] = (uint32_t)(offset + (uint64_t)k * stride);
      total += dfs(&c, 1, path, buf);
    }
    free(buf);
  }
  return total;
}

/*
 * Time-bounded sample for the CPU baseline: roots[0..nroots) are processed
 * (OpenMP dynamic schedule) until `budget_s` seconds have passed; a root the
 * deadline cuts short is discarded.  Returns the instances of the completed
 * roots; *done = completed roots, *elapsed = wall seconds spent.
 */
uint64_t oracle_wcoj_sample(const uint64_t* rp, const uint32_t* cols, uint64_t nv, int q, int ordering,
                            const uint32_t* roots, uint64_t nroots, int threads, double budget_s,
                            uint64_t* done, double* elapsed) {
  pattern_t p;
  if (build_pattern(q, &p)) return (uint64_t)-1;
  plan_t pl;
  make_plan(&p, ordering, &pl);
  uint64_t pos = 0;
  uint64_t maxd = max_degree(rp, nv);
  size_t per_thread = (size_t)(3 * maxd + 3) * (size_t)(MAXQ + 1);
  uint64_t total = 0, completed = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
  const double t0 = omp_get_wtime();
#else
  const double t0 = 0;
#endif
  const double deadline = t0 + budget_s;
#pragma omp parallel reduction(+ : total, completed)
  {
    int aborted = 0;
    ctx_t c = {rp, cols, nv, &pl, NULL, 0, &pos, deadline, &aborted};
    uint32_t* buf = (uint32_t*)malloc(sizeof(uint32_t) * per_thread);
    uint32_t path[MAXQ];
#pragma omp for schedule(dynamic, 1)
    for (long long k = 0; k < (long long)nroots; ++k) {
      if (expired(&c)) continue;
      aborted = 0;
      path[0] = roots[k];
      uint64_t a = dfs(&c, 1, path, buf);
      if (!aborted) {
        total += a;
        completed += 1;
      }
    }
    free(buf);
  }
#ifdef _OPENMP
  if (elapsed) *elapsed = omp_get_wtime() - t0;
#else
  if (elapsed) *elapsed = 0;
#endif
  if (done) *done = completed;
  return total;
}

/*
 * Writes an edge list as SNAP text ("u v\n" per edge, decimal), the input
 * format of the reference's preprocess_graph tool (GraphIO.h:232-270): a
 * fast writer for the benchmark's generated edge lists.  Returns 0 on
 * success.
 */
#include <stdio.h>
int oracle_write_edge_text(const uint32_t* u, const uint32_t* v, uint64_t ne, const char* path) {
  FILE* f = fopen(path, "wb");
  if (!f) return 1;
  enum { CAP = 1 << 22 };
  char* buf = (char*)malloc(CAP + 32);
  if (!buf) {
    fclose(f);
    return 1;
  }
  size_t len = 0;
  for (uint64_t i = 0; i < ne; ++i) {
    uint32_t x[2] = {u[i], v[i]};
    for (int k = 0; k < 2; ++k) {
      char tmp[12];
      int t = 0;
      uint32_t y = x[k];
      do {
        tmp[t++] = (char)('0' + y % 10);
        y /= 10;
      } while (y);
      while (t) buf[len++] = tmp[--t];
      buf[len++] = k == 0 ? ' ' : '\n';
    }
    if (len >= CAP) {
      if (fwrite(buf, 1, len, f) != len) {
        free(buf);
        fclose(f);
        return 1;
      }
      len = 0;
    }
  }
  int bad = len && fwrite(buf, 1, len, f) != len;
  free(buf);
  return fclose(f) != 0 || bad;
}
