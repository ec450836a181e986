/*
 * sme.h -- C-ABI of the B200 subgraph-enumeration engine (libsme.so).
 *
 * Drop-in boundary for the GPU enumeration path of guowentian/SubgraphMatchGPU.
 * Every entry point takes plain pointers and sizes; no C++ or torch types
 * cross this boundary.  All calls return an sme_status; the library never
 * exits or aborts the caller (the reference calls exit(-1) from CUDA_ERROR,
 * src/gpu/utils/GPUUtil.cuh:9-17, and asserts elsewhere).
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   graph loading      src/graph/GraphIO.h:26-136 (ReadDataFile/ReadCSRBinFile)
 *   graph writing      src/graph/GraphIO.h:356-387 (WriteCSRBinFile)
 *   preprocessing      src/preprocess/PreprocessGraph.h:13-95
 *   instance wiring    src/gpu/PatternMatchGPUInstance.cuh:26-176 (InitGPUInstance)
 *   execution          src/gpu/executor/PatternMatch.cuh:52-88 (Execute), the
 *                      plugin HybridGPUComponent (src/gpu/impl/common/HybridGPUComp.cuh:18-107)
 *                      and HybridGPUProcessor::ProcessLevel
 *                      (src/gpu/impl/common/HybridGPUProcessor.cuh:14-50)
 *   plan printing      src/query/TestPlan.cpp:8-51
 */
#ifndef SME_H_
#define SME_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace assert/exit in the reference) ---------------- */
typedef enum sme_status {
  SME_OK = 0,
  SME_ERR_INVALID_ARG = 1,
  SME_ERR_BAD_FILE = 2,
  SME_ERR_OOM = 3,
  SME_ERR_TIMEOUT = 4,
  SME_ERR_CUDA = 5,
  SME_ERR_UNSUPPORTED_QUERY = 6,
  SME_ERR_NO_DEVICE = 7,
  SME_ERR_CAPACITY = 8,  /* enumeration output buffer too small           */
  SME_ERR_BUSY = 9,      /* server queue full / request not finished yet  */
  SME_ERR_CANCELLED = 10
} sme_status;

/* ---- enums: same numeric values as src/Meta.h:47-124 -------------------- */
enum {
  SME_CPU_WCOJ = 0, SME_CPU_VF2 = 1, SME_CPU_BFS = 2, SME_CPU_RBFS = 3,
  SME_GPU_GPSM = 4, SME_GPU_GPSM_REUSE = 5, SME_GPU_LIGHT = 6
};
enum { SME_HYBRID_CPU_GPU = 0, SME_IN_MEMORY_GPU = 1, SME_EXTERNAL_GPU = 2 };
enum { SME_EXT_CACHE = 0, SME_EXT_UMA = 1 };
/* LazyTraversalCompressLevel, src/query/common/LazyTraversalCommon.h:38-76 */
enum {
  SME_COMPRESS_MATERIALIZE = 0,
  SME_COMPRESS_NON_MATERIALIZE = 1,
  SME_COMPRESS_NON_MATERIALIZE_OPT = 2,
  SME_COMPRESS_SPECIAL = 3
};
#define SME_NUM_QUERIES 14 /* Q0..Q13 */

typedef struct sme_graph sme_graph; /* opaque: host CSR + cached device copy */

/* Options of one enumeration run; mirrors the patternmatchgpu flags
 * (src/gpu/PatternMatchGPU.cu:17-37). */
typedef struct sme_opts {
  int32_t query_type;      /* -q : 0..13                                     */
  int32_t algo;            /* -a : 4 GPU_GPSM, 5 GPU_GPSM_REUSE, 6 GPU_LIGHT */
  int32_t execute_mode;    /* -m : 1 IN_MEMORY_GPU, 2 EXTERNAL_GPU           */
  int32_t compress_level;  /* -c : 0..3, default 3 (SPECIAL)                 */
  int32_t enable_ordering; /* -r : 1 (default) keeps symmetry breaking       */
  int32_t ext_variant;     /* -y : 0 EXT_CACHE, 1 EXT_UMA                    */
  int32_t reuse_autogen;   /* 0 hard-coded reuse plan, 1 cost-based autogen,
                              -1 (default) hard-coded when one exists       */
  int32_t device;          /* CUDA device ordinal                            */
  uint64_t mem_limit_bytes;/* device budget for frontiers+graph; 0 = auto    */
  uint64_t root_begin;     /* first-level vertex range [begin,end) (a task   */
  uint64_t root_end;       /*  of IntraPartScheduler); end==0 means all.
                              The first level is the plan's first pattern
                              vertex: u0, except in the LIGHT house plan
                              (Q4), whose search sequence starts at u1      */
  int32_t warp_granularity;/* intersection launch shape: 0 auto (warp per
                              path, specialised on list count, tuned
                              occupancy; on an oriented graph, whose lists
                              are short, as 2), 1 warp per path generic,
                              2 flattened (32 paths per warp), 3 as 0 with
                              six blocks per SM throughout, 4 as 0 with a
                              CTA per path whose clipped pivot is long
                              (two-list steps; the other list staged in
                              shared memory by a bulk copy)                 */
  int32_t list_only;       /* 1: membership by binary search only, no hub
                              bitmaps (comparison knob)                      */
  uint32_t root_stride;    /* roots are root_begin, +stride, ... < root_end
                              (0 or 1: every root); a strided task          */
  int32_t no_set_reuse;    /* LIGHT: 1 computes every candidate set from
                              adjacency lists, as the reference does; 0
                              (default) starts a set from an earlier
                              candidate set that covers some of its lists
                              when the conditions allow (same sets)        */
  const uint32_t* roots;   /* explicit root task: when num_roots > 0 the
                              first level is exactly roots[0..num_roots)
                              (host memory, ids below n; a root listed
                              twice counts twice) and root_begin / root_end
                              / root_stride are ignored                    */
  uint64_t num_roots;
} sme_opts;

/* Counters of the last sme_count/sme_enumerate call on this thread. */
typedef struct sme_stats {
  double elapsed_ms;          /* plan + device execution (+ graph H2D when it
                                 was not resident), as elapsed_time= in the
                                 reference (PatternMatch.cuh:77-87)          */
  double kernel_ms;           /* sum of CUDA-event time of the hot kernels   */
  uint64_t kernel_launches;   /* kernels of this library launched            */
  uint64_t batches;           /* level batches processed                    */
  uint64_t algorithmic_bytes; /* bytes the intersection steps must touch: per
                                 path 12 per backward list (row pointers +
                                 gathered vertex), 4 x clipped pivot length x
                                 lists intersected (each pivot element read
                                 once and tested once per other list), 4 per
                                 candidate written                           */
  uint64_t h2d_bytes;         /* host->device bytes moved by this call       */
  uint64_t d2h_bytes;
  uint64_t peak_device_bytes; /* high-water mark of the frontier arena       */
  uint64_t paths_processed;   /* partial instances entering compute steps    */
  double device_ms;           /* CUDA-event time on the library's stream from
                                 the first to the last kernel of the run      */
  uint64_t hot_launches;      /* launches of the intersection kernels         */
  /* CUDA-event time per phase (the reference's PROFILE phase timers,
   * src/gpu/impl/common/ProfilerHelper.cuh:9-75): [0] compute,
   * [1] materialize, [2] filter_compute, [3] compute_count,
   * [4] compute_path_count, [5] count, [6] organize_batch (estimates, scans),
   * [7] external subgraph load. */
  double phase_ms[8];
  uint64_t reuse_hits;        /* reuse plan: paths whose mapped reuse found the
                                 sibling's cached intersection (the rest
                                 intersected the adjacency lists)            */
} sme_stats;

/* ---- options ------------------------------------------------------------- */
sme_status sme_opts_default(sme_opts* opts);

/* ---- graphs (GraphIO.h / PreprocessGraph.h) ------------------------------ */
/* BIN CSR: 4 x size_t header (4, 8, n, m), uint64 row_ptrs[n+1], uint32 cols[m]
 * (GraphIO.h:88-136).  Read with one bulk read, validated. */
sme_status sme_graph_load_bin(const char* path, sme_graph** out);
/* SNAP edge list text (GraphIO.h:195-270); directed=0 stores both directions;
 * adjacency lists are sorted.  No preprocessing. */
sme_status sme_graph_load_snap(const char* path, int directed, sme_graph** out);
/* SNAP edge list whose vertex names are any digit strings
 * (GraphIO::ReadSNAPLargeVIDFile, GraphIO.h:142-230): names get dense ids in
 * order of first appearance; lists sorted; no preprocessing. */
sme_status sme_graph_load_snap_lvid(const char* path, int directed, sme_graph** out);
/* Dispatch on the file suffix like GraphIO::ReadDataFile (GraphIO.h:48-64):
 * .txt SNAP, .bin BIN, .lvid SNAP with large vertex ids. */
sme_status sme_graph_load(const char* path, int directed, sme_graph** out);
/* From caller CSR.  copy=1 copies; copy=0 borrows (caller keeps the arrays
 * alive and unchanged until sme_graph_free). */
sme_status sme_graph_from_csr(const uint64_t* row_ptrs, const uint32_t* cols,
                              uint64_t n, uint64_t m, int copy,
                              sme_graph** out);
sme_status sme_graph_info(const sme_graph* g, uint64_t* n, uint64_t* m,
                          uint64_t* max_degree);
sme_status sme_graph_csr(const sme_graph* g, const uint64_t** row_ptrs,
                         const uint32_t** cols);
/* Writes exactly the bytes of GraphIO::WriteCSRBinFile to `path`. */
sme_status sme_graph_write_bin(const sme_graph* g, const char* path);
/* Writes exactly the text of GraphIO::WriteCSRSNAPFile (GraphIO.h:389-413):
 * "u v" per edge with u < v.  The reference appends ".snap.txt" to its
 * input name; here `path` is used as given. */
sme_status sme_graph_write_snap(const sme_graph* g, const char* path);
/* Writes exactly the text of GraphIO::WriteCSRAdjFile (GraphIO.h:414-436),
 * the partitioner's input: "u<TAB>v v ... " per vertex, and `path`.info with
 * "n m".  The reference appends ".adj.txt"; here `path` is used as given. */
sme_status sme_graph_write_adj(const sme_graph* g, const char* path);
/* PreprocessGraph::Preprocess: drop self loops and parallel edges, then
 * dangling vertices with a dense order-preserving relabel. */
sme_status sme_graph_preprocess(sme_graph* g);
/* GraphIO::Validate: sorted, no self loop, no parallel edge, no dangling. */
sme_status sme_graph_validate(const sme_graph* g);
/* Degree-ordered copy of `g` in `*out`: vertices renumbered by (degree, id)
 * ascending, lists sorted.  A renumbering is an isomorphism, so every count
 * is unchanged; under the clique queries' total order the candidate sets
 * N(u) ∩ {> u} then hold only higher-degree neighbours.  orient = 1 also
 * keeps each edge once, towards the higher new id (half the lists); an
 * oriented graph counts only the clique queries 0, 3, 7, 11 with symmetry
 * breaking on (others return SME_ERR_UNSUPPORTED_QUERY) and cannot be
 * preprocessed.  new_to_old (n entries, may be NULL) receives each new id's
 * original id, to map enumerated instances back.
 * No counterpart in the reference, which stores both directions and relies
 * on the `<` conditions; the R-MAT s22 clique configuration of this path asks
 * for the degree-ordered orientation. */
sme_status sme_graph_degree_order(const sme_graph* g, int32_t orient, sme_graph** out,
                                  uint32_t* new_to_old);
/* 1 when `g` was made by sme_graph_degree_order with orient = 1. */
int32_t sme_graph_is_oriented(const sme_graph* g);
/* Copies the CSR to device memory of `device` and keeps it there; later runs
 * on that device reuse it (inputs resident in HBM). */
sme_status sme_graph_to_device(sme_graph* g, int device);
sme_status sme_graph_release_device(sme_graph* g);
/* Device addresses of the resident copy on `device` (after
 * sme_graph_to_device): uint64 row_ptrs[n+1] and uint32 cols[m], valid until
 * the copy is released; for sme_count_noalloc and the caller's own kernels.
 * SME_ERR_INVALID_ARG when the graph is not resident there.  The reference
 * keeps the same arrays in its GPU CSR (CSRGraph's device row_ptrs/cols). */
sme_status sme_graph_device_arrays(const sme_graph* g, int device, const uint64_t** row_ptrs,
                                   const uint32_t** cols);
/* Keeps a packed copy of the adjacency lists in pinned host memory; every
 * later upload of this graph (sme_graph_to_device, or a call on a graph that
 * is not resident) copies the packed lists and expands them on the device
 * into the same CSR.  Each list is stored as deltas from the previous element
 * in blocks of 32 with one bit width per block (about 0.4x the bytes of the
 * uint32 lists on R-MAT graphs), so the host->device copy shrinks by that
 * much.  The packed copy reflects the lists when this is called: a borrowed
 * CSR (sme_graph_from_csr, copy = 0) changed afterwards must be packed again.
 * enable = 0 drops it.  *packed_bytes (may be NULL) receives the bytes an
 * upload now copies.  No counterpart in the reference, which copies the
 * uint32 CSR. */
sme_status sme_graph_pack(sme_graph* g, int enable, uint64_t* packed_bytes);
sme_status sme_graph_free(sme_graph* g);

/* ---- seeded synthetic graphs (all passed through the preprocess step) ---- */
/* R-MAT(scale, edge_factor, a, b, c) with d = 1-a-b-c; undirected. */
sme_status sme_generate_rmat(int32_t scale, int32_t edge_factor, double a,
                             double b, double c, uint64_t seed,
                             sme_graph** out);
/* Erdos-Renyi G(n, p = avg_degree/(n-1)). */
sme_status sme_generate_er(uint64_t n, double avg_degree, uint64_t seed,
                           sme_graph** out);
/* Barabasi-Albert with m_attach edges per new vertex. */
sme_status sme_generate_ba(uint64_t n, uint32_t m_attach, uint64_t seed,
                           sme_graph** out);
/* Complete graph K_n (GenerateNClique, src/test/gpu/TestGPUCommon.cuh:32-49). */
sme_status sme_generate_clique(uint64_t n, sme_graph** out);

/* ---- enumeration (PatternMatch::Execute) --------------------------------- */
sme_status sme_count(sme_graph* g, const sme_opts* opts, uint64_t* count);
/* Writes up to cap instances, each query_vertex_count uint32 ids in pattern
 * vertex order (u0..u_{k-1}); *n_out = number of instances found (the call
 * fails with SME_ERR_CAPACITY when it exceeds cap, *n_out still valid). */
sme_status sme_enumerate(sme_graph* g, const sme_opts* opts, uint32_t* out,
                         uint64_t cap_instances, uint64_t* n_out);
/* Stats of the last sme_count/sme_enumerate issued by this thread. */
sme_status sme_last_stats(sme_stats* stats);

/* ---- partitioned graphs (HYBRID_CPU_GPU, -m 0 -e FILE -p P) ------------- */
/* GraphIO::ReadPartitionFile (src/graph/GraphIO.h:66-86): n partition ids,
 * one per vertex, whitespace separated, into vertex_partition[n].
 * partition_num == 1 or an empty path puts every vertex in partition 0.
 * A short file, an id >= partition_num or a largest id other than
 * partition_num - 1 (an assert in the reference) return SME_ERR_BAD_FILE. */
sme_status sme_read_partition_file(const char* path, uint64_t n, uint32_t partition_num,
                                   uint32_t* vertex_partition);
/* The subgraph induced by partition p, its vertices renumbered in ascending
 * global id (GraphPartition::BuildIntraPartition,
 * src/graph/GraphPartition.h:36-95). */
sme_status sme_graph_partition(const sme_graph* g, const uint32_t* vertex_partition, uint32_t p,
                               sme_graph** out);
/* The counts of -m 0 (HybridSeparatePatternMatch / Interplay / Coprocess,
 * src/gpu/executor/): *total over the whole graph, intra[p] (may be NULL)
 * the instances inside partition p; the inter-partition count is
 * total - sum(intra).  algo 5 or 6 as the reference allows for this mode;
 * execute_mode 0 or 1.  The whole graph runs in one in-memory pass on the
 * GPU (it fits in HBM), so the CPU/GPU work split of variants O0-O3 is not
 * reproduced; the counts are the same. */
sme_status sme_count_partitioned(sme_graph* g, const sme_opts* opts, const uint32_t* vertex_partition,
                                 uint32_t partition_num, uint64_t* total, uint64_t* intra);

/* Number of pattern vertices of query q (Query.h:84-434). */
int32_t sme_query_vertex_count(int32_t query_type);

/* ---- plans (TestPlan.cpp) ------------------------------------------------ */
/* plan_type: 0 TraversalPlan, 1 ReuseTraversalPlan (autogen as test_plan -t 1),
 * 2 LazyTraversalPlan (NON_MATERIALIZE_OPT as test_plan -t 2),
 * 3 ReuseTraversalPlan with the hard-coded plan (patternmatch default),
 * 4 LazyTraversalPlan with compress_level SPECIAL,
 * 5 the level programs the engine runs for algo 4, 5 and 6 (default options),
 * 6 as 5 for a graph without self loops (the usual case).
 * Writes a NUL-terminated text description; returns SME_ERR_CAPACITY when
 * `cap` is too small (*needed holds the size). */
sme_status sme_plan_describe(int32_t query_type, int32_t plan_type, char* buf,
                             uint64_t cap, uint64_t* needed);

/* ---- batched form: many small graphs, one persistent launch ------------- */
typedef struct sme_batch_opts {
  int32_t device;
  int32_t autotune;        /* 1: pick granularity/block shape by measuring   */
  int32_t granularity;     /* without autotuning: 0 eight lanes, 1 a warp,
                              2 a CTA group of 128 threads per root item     */
  int32_t block_threads;   /* 0 auto                                         */
  int32_t use_graph;       /* 1: capture the launch in a CUDA graph          */
  int32_t reserved[11];
} sme_batch_opts;
sme_status sme_batch_opts_default(sme_batch_opts* o);
/* counts[i] = count of queries[i] on graphs[i] (symmetry-broken, uint64). */
sme_status sme_batch_count(sme_graph* const* graphs, const int32_t* queries,
                           uint64_t num, const sme_batch_opts* opts,
                           uint64_t* counts);
typedef struct sme_batch_plan sme_batch_plan; /* resident packed batch */
sme_status sme_batch_prepare(sme_graph* const* graphs, const int32_t* queries,
                             uint64_t num, const sme_batch_opts* opts,
                             sme_batch_plan** out);
sme_status sme_batch_run(sme_batch_plan* p, uint64_t* counts, double* ms);
sme_status sme_batch_describe(const sme_batch_plan* p, int32_t* granularity,
                              int32_t* block_threads, uint64_t* work_items);
/* The configuration the autotuner kept: threads per group (4, 8, 16 lanes of
 * a warp, 32 a warp, 64 or 128 warps of a CTA working on one item), threads
 * per block, work items a group takes per fetch, and its measured time on
 * the batch (0 without autotuning).  No counterpart in the reference: the
 * batched form is new. */
sme_status sme_batch_tuning(const sme_batch_plan* p, int32_t* group_threads,
                            int32_t* block_threads, int32_t* items_per_fetch,
                            double* tuned_ms);
sme_status sme_batch_free(sme_batch_plan* p);

/* Allocation-free count of query `query_type` on one graph whose CSR the
 * caller already holds in device memory (d_row_ptrs: n+1 uint64 offsets,
 * d_cols: uint32 neighbour ids; every list strictly increasing, so sorted with
 * no duplicate neighbours, no self loops, ids below n, both directions
 * stored).  It has no counterpart in the reference.  It exists for callers
 * that must not call cudaMalloc: code running under a framework whose caching
 * allocator already owns the device memory, or latency-critical paths that
 * cannot afford an allocation and the synchronisation it implies.  Besides
 * the caller's buffers it uses only a 16 MiB array the library reserves in
 * device memory for the life of the process on every GPU that loads it;
 * nothing is allocated or freed.  Limit: the graph's maximum degree must be
 * at most 32768 and n below 2^31, else SME_ERR_CAPACITY / SME_ERR_INVALID_ARG;
 * a list that breaks the contract above returns SME_ERR_INVALID_ARG (checked
 * on the device in the same pass that finds the maximum degree).  The number
 * of thread groups the array holds falls as the maximum degree rises (about
 * 7 blocks of 16 groups at the limit), so hub-heavy graphs count slowly here.
 * The first call on a device looks up the array's device address, so make
 * that first call before any stream capture.  Every call clears the array's
 * header with cudaMemsetAsync on the legacy default stream, launches its
 * kernels there and reads results back with two blocking cudaMemcpy; it
 * returns when the count is known.  All calls share the one array, so calls
 * that overlap on the same GPU (from several host threads) race. */
sme_status sme_count_noalloc(const uint64_t* d_row_ptrs, const uint32_t* d_cols,
                             uint64_t n, int32_t query_type, uint64_t* count);

/* ---- served form: resident graphs + continuous batching ----------------- */
typedef struct sme_server sme_server;
typedef struct sme_server_opts {
  int32_t device;
  int32_t slots;             /* concurrent requests on the device           */
  uint64_t mem_budget_bytes; /* admission budget (estimated frontier bytes) */
  int32_t queue_capacity;
  int32_t reserved[9];
} sme_server_opts;
sme_status sme_server_opts_default(sme_server_opts* o);
sme_status sme_server_create(const sme_server_opts* o, sme_server** out);
/* Keeps `g` resident on the server's device; returns its graph id. */
sme_status sme_server_add_graph(sme_server* s, sme_graph* g, int32_t* gid);
/* Enqueue a request on a resident graph (gid) or on an attached graph
 * (gid = -1, `attached` non-NULL, owned by the caller until completion). */
sme_status sme_server_submit(sme_server* s, int32_t gid, sme_graph* attached,
                             const sme_opts* opts, uint64_t* request_id);
/* Non-blocking: SME_ERR_BUSY while pending; else the request's final status,
 * its count and its latency (submit -> result) in milliseconds. */
sme_status sme_server_poll(sme_server* s, uint64_t request_id, uint64_t* count,
                           double* latency_ms);
sme_status sme_server_wait(sme_server* s, uint64_t request_id,
                           uint64_t* count, double* latency_ms);
sme_status sme_server_stats(sme_server* s, uint64_t* completed,
                            uint64_t* max_inflight, uint64_t* rejected);
sme_status sme_server_destroy(sme_server* s);

/* ---- errors --------------------------------------------------------------- */
/* Message of the last failing call on this thread ("" if none). */
const char* sme_last_error(void);
const char* sme_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SME_H_ */
