/*
 * gst_b200.h -- C ABI of the B200 group Steiner tree (GST) engine.
 *
 * The engine is a drop-in for the per-query GPU solve of GPU4GST
 * (TrimCDP / D-TrimCDP and their -WB variants) and for the inputs those
 * programs read.  Every entry point takes plain pointers and sizes, returns a
 * gst_status and never exits the process.  Host buffers passed in are owned
 * by the caller; buffers handed out (gst_csr, gst_groups, gst_queries,
 * gst_result edge lists) are freed with the matching *_free call.
 *
 * Costs are exact integers.  A query's answer is the optimal group Steiner
 * tree cost (plain, D < 0) or the optimum of the diameter-bounded DP of
 * D-PrunedDP++ (D >= 0); the tree itself is returned as an edge list.
 */
#ifndef GST_B200_H
#define GST_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GST_OK = 0,
  GST_E_INVALID = 1,     /* bad argument (null pointer, id out of range, k out of range) */
  GST_E_IO = 2,          /* file cannot be opened or read */
  GST_E_FORMAT = 3,      /* file content does not parse */
  GST_E_CUDA = 4,        /* CUDA runtime error (message in gst_last_error) */
  GST_E_NOMEM = 5,       /* the request does not fit the device arena */
  GST_E_UNSUPPORTED = 6, /* e.g. k above GST_MAX_K */
  GST_E_LIMIT = 7,       /* a device-side bound was hit (round limit, buffer cap) */
  GST_E_STATE = 8,       /* call out of order (no graph loaded, unknown ticket) */
  GST_E_TIMEOUT = 9      /* gst_server_wait ran out of time */
} gst_status;

#define GST_MAX_K 7        /* groups per query handled by the device kernels */
#define GST_MAX_D 15       /* largest finite diameter bound */
#define GST_REF_INF 100000 /* the reference's infinity / infeasible cost */

/* Text of the last error raised on the calling thread (never NULL). */
const char* gst_last_error(void);

/* sizeof of a public struct of this header as the library was compiled
 * ("gst_result", "gst_stats", "gst_engine_config", "gst_profile", "gst_csr",
 * "gst_groups", "gst_queries"), -1 for another name.  Lets a binding check
 * that it lays the structs out as the library does.  No reference
 * counterpart. */
int64_t gst_sizeof(const char* type_name);

/* ---------------------------------------------------------------------------
 * Host-side inputs in the reference's formats
 * ------------------------------------------------------------------------- */

/* Undirected graph as CSR with both directions stored, rows sorted by
 * neighbour id (the order the reference's text loader produces). */
typedef struct {
  int64_t V;       /* vertices */
  int64_t E;       /* directed entries (2 x undirected edges) */
  int64_t* rowptr; /* V+1 */
  int32_t* col;    /* E */
  int32_t* w;      /* E, weights >= 0 */
} gst_csr;

/* Groups as CSR of member vertices; group g is members[ptr[g] .. ptr[g+1]). */
typedef struct {
  int64_t n;
  int64_t* ptr;     /* n+1 */
  int32_t* members; /* ptr[n], each group's members sorted */
} gst_groups;

/* Queries: query i is ids[ptr[i] .. ptr[i+1]) (0-based group ids). */
typedef struct {
  int64_t n;
  int64_t* ptr;
  int32_t* ids;
} gst_queries;

/* "<path><data>.in": header "V ...", then "u v w" per undirected edge; both
 * directions are stored and rows sorted.  Replaces read_input_graph
 * (code/PrunedDP++/include/graph_hash_of_mixed_weighted_read_for_GSTP.h:15-66)
 * and toCSR (code/TrimCDP/include/graph_v_of_v_idealID/csr_graph.hpp:39-128).
 * A missing file returns GST_E_IO instead of blocking on getchar(). */
gst_status gst_read_input_graph(const char* file, gst_csr* out);

/* "<data>_beg_pos.bin" (V+1 x int64), "_csr.bin" (E x int64),
 * "_weight.bin" (E x int64), narrowed to int32 ids/weights.  Replaces the
 * graph<long,long,long,...> constructor (code/TrimCDP-WB/include/graph.hpp:12-118).
 * Rows are used as stored (not re-sorted). */
gst_status gst_read_binary_csr(const char* beg_pos_file, const char* csr_file,
                               const char* weight_file, gst_csr* out);

/* "<path><data>.g": lines "gK:v v v", K 1-based -> group K-1, members sorted.
 * Replaces read_Group (graph_hash_of_mixed_weighted_read_for_GSTP.h:116-171,
 * code/TrimCDP-WB/include/read_group.hpp:9-50). */
gst_status gst_read_groups(const char* file, gst_groups* out);

/* "<path><data><k>.csv": one query per line, space-separated 0-based group
 * ids.  Replaces read_inquire (graph_hash_of_mixed_weighted_read_for_GSTP.h:172-218). */
gst_status gst_read_queries(const char* file, gst_queries* out);

void gst_csr_free(gst_csr* g);
void gst_groups_free(gst_groups* g);
void gst_queries_free(gst_queries* q);

/* ---------------------------------------------------------------------------
 * Engine: one per device; holds the graph and groups in HBM and a
 * pre-allocated arena for per-query DP tables.
 * ------------------------------------------------------------------------- */

typedef struct gst_engine gst_engine;

typedef struct {
  int device;              /* CUDA device ordinal */
  double arena_fraction;   /* share of free device memory for the arena (0 -> 0.85) */
  int64_t arena_bytes;     /* explicit arena size; overrides the fraction when > 0 */
  int max_slots;           /* queries resident at once (0 or above 1024 -> 1024) */
  int rounds_per_poll;     /* device rounds between host status checks (0 -> 8) */
  int max_rounds;          /* device rounds a query may take before it fails with
                              GST_E_LIMIT (0: unlimited) */
  int profile;             /* 1: time the grow and merge kernels with CUDA events */
  int bucket_shift;        /* plain grows run in cost buckets of width
                              max(typical lightest edge, best >> bucket_shift)
                              (0 -> 30: the lightest-edge width, best measured) */
} gst_engine_config;

/* Device waits of an engine are bounded: if a poll of the round sequence does
 * not complete within GST_WATCHDOG_S seconds (environment variable, default
 * 120), the call returns GST_E_CUDA and the engine refuses further work; the
 * process should then exit (which ends the device work with its context).
 * gst_engine_destroy of such an engine frees nothing. */
gst_status gst_engine_create(const gst_engine_config* cfg, gst_engine** out);
void gst_engine_destroy(gst_engine* e);

/* Launch and scheduling parameters of an engine.  The defaults were picked
 * by hand; gst_b200.autotune (Python) times candidates on a workload and
 * writes a parameter file that sets them.  A field left 0 keeps the current
 * value.  No reference counterpart (the reference fixes its launch shapes as
 * macros: code/TrimCDP-WB/include/util.h:19-33, header.h:14). */
typedef struct {
  int grow_lanes;      /* lanes relaxing one grow chunk: 8, 16 or 32 (default 16) */
  int rounds_per_poll; /* device rounds between host status checks (default 8) */
  int max_slots;       /* queries resident at once, 1..1024 */
  int chunk_pairs[GST_MAX_K + 1][2]; /* (edge, set) pairs per grow chunk by k and
                                        [0] plain / [1] diameter-bounded (default 1024) */
  int bucket_mult[GST_MAX_K + 1];    /* plain grows: cost-bucket width = this many times
                                        the typical lightest edge, by k (default 1) */
  int overlap;         /* 1: a round's merge and grow run one after the other (default);
                          2: they run as two branches of the round graph, on two streams
                          (they touch disjoint slots), so their kernels can share the GPU */
} gst_tuning;

gst_status gst_engine_set_tuning(gst_engine* e, const gst_tuning* t);
gst_status gst_engine_get_tuning(gst_engine* e, gst_tuning* out);

/* Uploads the graph (CSR as gst_csr describes) and checks it: ids in range,
 * weights in [0, 2^30).  Replaces the per-program CSR upload
 * (csr_graph.hpp:117-125; code/TrimCDP-WB/include/gpu_graph.cuh:10-57). */
gst_status gst_engine_load_graph(gst_engine* e, int64_t V, const int64_t* rowptr,
                                 const int32_t* col, const int32_t* w);

/* Uploads the groups (member lists, as gst_groups describes). */
gst_status gst_engine_load_groups(gst_engine* e, int64_t n, const int64_t* ptr,
                                  const int32_t* members);

typedef struct {
  int64_t rounds;       /* device rounds the query took part in */
  int64_t frontier;     /* frontier states expanded (grow sources) */
  int64_t relax;        /* edge relaxations attempted */
  int64_t improve;      /* successful table updates by the grow */
  int64_t merges;       /* merge partner pairs evaluated (past the lower-bound pre-filter) */
  int64_t merge_items;  /* (vertex, set) items the merges visited */
  int64_t merge_passed; /* of those, items past the lower-bound pre-filter */
  int64_t touched;      /* vertices that held a finite state */
  double device_ms;     /* device time from admission to answer */
  double queue_ms;      /* host time from submission to admission into a slot */
  double latency_ms;    /* host time from submission to the result being ready */
} gst_stats;

typedef struct {
  int64_t cost;      /* optimal cost; GST_REF_INF when infeasible */
  int32_t feasible;  /* 1 if a tree touching every queried group exists */
  int32_t root;      /* root vertex of the returned tree, -1 if infeasible */
  int32_t n_edges;   /* tree edges */
  int32_t* edges;    /* n_edges x (u, v, w); free with gst_result_free */
  gst_stats stats;
} gst_result;

void gst_result_free(gst_result* r);

/* One query, blocking: group ids (duplicates merged), k = number of ids,
 * D < 0 for the plain problem, 0 <= D <= GST_MAX_D for the diameter bound of
 * the D- variants.  Replaces DP_GPU (code/TrimCDP/include/DPQ.cuh:63,
 * code/TrimCDP/src/DPQ.cu:275-624) and DP_gpu (code/D-TrimCDP/include/DPQ.cuh:63,
 * code/D-TrimCDP/src/DPQ.cu:143-261), which return the cost only. */
gst_status gst_solve(gst_engine* e, const int32_t* group_ids, int k, int D, gst_result* out);

/* Many queries in one persistent launch sequence: query i has ids
 * ids[ptr[i] .. ptr[i+1]) and bound D[i] (NULL: all plain).  out has n
 * entries.  Per-query failures are reported in status_out (may be NULL);
 * the call itself fails only for argument or device errors.  No reference
 * counterpart: the reference solves one query per call. */
gst_status gst_solve_batch(gst_engine* e, int64_t n, const int64_t* ptr, const int32_t* ids,
                           const int32_t* D, gst_result* out, gst_status* status_out);

/* Device-side measurements of the most recent gst_solve / gst_solve_batch
 * call.  run_ms spans the call on the engine's stream (CUDA events); the
 * kernel times are filled when the engine was created with profile = 1.
 * No reference counterpart (the reference times with host clocks). */
typedef struct {
  double run_ms;            /* device time of the call */
  double grow_ms;           /* summed duration of the grow-kernel launches */
  int64_t grow_launches;
  double merge_ms;          /* summed duration of the merge-kernel launches */
  int64_t merge_launches;
  int64_t kernel_launches;  /* all engine kernel launches in the call */
  int64_t rounds;           /* device rounds run */
  int64_t h2d_bytes;        /* host-to-device bytes copied by the call */
  int64_t d2h_bytes;        /* device-to-host bytes copied by the call */
} gst_profile;

gst_status gst_engine_profile(gst_engine* e, gst_profile* out);

/* ---------------------------------------------------------------------------
 * Allocation-free solve.  No counterpart in the reference.
 * ------------------------------------------------------------------------- */

#define GST_NOALLOC_SCRATCH_BYTES (64ull << 20) /* static device scratch: 64 MiB */

/* One query (plain, D < 0, or diameter-bounded) for callers that cannot
 * allocate memory: processes that reserved all device memory up front, code
 * running in allocation-free sections, plugin hosts that forbid cudaMalloc
 * after start-up.  Nothing is allocated: the caller passes the graph and the
 * groups as device pointers it owns (d_adj holds E (neighbour, weight) int32
 * pairs, interleaved; d_rowptr V+1 int64 offsets; groups as int64 offsets and
 * int32 members), the queried group ids in host memory, and receives the
 * cost (GST_REF_INF when infeasible) and the root vertex in host variables.
 * All scratch lives in a file-scope static device array of
 * GST_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit; a query whose scratch would exceed it fails with GST_E_NOMEM.  Calls
 * share that array and it keeps the last call's contents: each call clears
 * what must start cleared, and the library serialises the calls of one
 * process (a call holds a lock until its work has finished), since calls that
 * overlapped on the GPU would race on the array.  The first call on a device
 * performs a one-time set-up on it (the array's device address, the subset
 * tables) and should come before any stream capture; a context that was reset
 * and re-created since is detected and set up again.  Device waits are
 * bounded by GST_WATCHDOG_S seconds (environment, default 120): a wait that
 * runs out fails the call with GST_E_CUDA and later calls on that device are
 * refused.  `stream` is a cudaStream_t (NULL: the legacy default stream); the
 * call returns after the stream has finished the query. */
gst_status gst_solve_noalloc(int64_t V, int64_t E, const int64_t* d_rowptr, const int32_t* d_adj,
                             int64_t n_groups, const int64_t* d_group_ptr,
                             const int32_t* d_group_members, const int32_t* group_ids, int k,
                             int D, void* stream, int64_t* cost_out, int32_t* root_out);

/* ---------------------------------------------------------------------------
 * Serving: continuous batching.  Requests submitted while others run are
 * admitted as slots and arena memory free up; their device work overlaps.
 * No reference counterpart.
 * ------------------------------------------------------------------------- */

typedef struct gst_server gst_server;

gst_status gst_server_start(gst_engine* e, gst_server** out);
/* Enqueues a query; *ticket identifies it in gst_server_wait. Thread-safe. */
gst_status gst_server_submit(gst_server* s, const int32_t* group_ids, int k, int D,
                             uint64_t* ticket);
/* Waits up to timeout_ms (< 0: forever) for the ticket's result; the result
 * is handed out once.  Per-query failure is the returned status. */
gst_status gst_server_wait(gst_server* s, uint64_t ticket, double timeout_ms, gst_result* out);
/* Stops the serving thread after finishing admitted work. */
void gst_server_stop(gst_server* s);

#ifdef __cplusplus
}
#endif
#endif /* GST_B200_H */
