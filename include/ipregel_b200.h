/*
 * ipregel_b200.h -- C ABI of libipregel_b200.so, the type-independent runtime
 * under the drop-in iPregel headers (include/iPregel.h).
 *
 * The reference is a header-only C library: every ip_* function is compiled
 * into the user's program, and the graph loader, vertex storage and the
 * OpenMP superstep loop live in its headers.  Here the typed part (the user's
 * ip_compute / ip_combine inlined into sm_100a kernels, and the superstep
 * loop of each version) stays in headers compiled by nvcc with the
 * application, while everything that does not depend on the user's types sits
 * behind this C ABI: graph loading and device-resident CSR/CSC, seeded graph
 * generators, frontier compaction, bitmap reductions and error reporting.
 *
 * Every function returns 0 on success or a negative IPG_E* code; the message
 * is available from ipg_last_error().  No function exits the process: the
 * drop-in header layer turns errors into the reference's print-and-exit(-1)
 * behaviour (src/iPregel_postamble.h:117-174).  Pointers named d_* are device
 * pointers; "stream" is a cudaStream_t passed as void*.
 */
#ifndef IPREGEL_B200_RUNTIME_H
#define IPREGEL_B200_RUNTIME_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IPG_ABI_VERSION 1

enum ipg_status {
    IPG_OK = 0,
    IPG_EINVAL = -1,     /* bad argument */
    IPG_ENOMEM = -2,     /* host or device allocation failed */
    IPG_EIO = -3,        /* file missing, short or malformed */
    IPG_ECUDA = -4,      /* CUDA runtime error */
    IPG_EDEVICE = -5,    /* a kernel reported an error word */
    IPG_EBUDGET = -6     /* request exceeds the configured HBM budget */
};

/* Message of the last failing call on this thread ("" if none). */
const char* ipg_last_error(void);
int ipg_abi_version(void);
/* Name and HBM capacity of the current device; 0 when a device is usable. */
int ipg_device_info(char* name, size_t name_len, uint64_t* hbm_bytes, int* sm_count);

/* Device memory accounting.  Every device allocation of the runtime and of
 * the engine state goes through ipg_dev_alloc, which refuses (IPG_EBUDGET)
 * any request that would take the bytes held above the budget (0 = no
 * budget; the IPG_HBM_BUDGET environment variable sets it at first use). */
int ipg_dev_alloc(void** d_ptr, uint64_t bytes);
int ipg_dev_free(void* d_ptr, uint64_t bytes);
int ipg_set_hbm_budget(uint64_t bytes);
uint64_t ipg_hbm_in_use(void);
/* Page-locked host buffers, for host<->device copies at full link speed. */
int ipg_host_alloc(void** ptr, uint64_t bytes);
int ipg_host_free(void* ptr);
/* Synchronous copy between any two of host and device memory. */
int ipg_memcpy(void* dst, const void* src, uint64_t bytes);

/* ------------------------------------------------------------------------
 * Graphs.  A graph is the reference loader's CSR (src/iPregel_postamble.h:
 * 244-421) made resident on the device: row[V+1] (u64, row[V] = E), adj[E]
 * (id_bytes each) and optional weights.  For directed graphs whose in-lists
 * are needed, the in-CSR (CSC) is built on the device in the order of the
 * reference's mirror loop (iPregel_postamble.h:429-487): each in-list sorted
 * by source vertex, ties in edge order.  For undirected graphs the in-lists
 * alias the rows, as in the reference (iPregel_postamble.h:368-372).
 * ------------------------------------------------------------------------ */
typedef struct ipg_graph ipg_graph;

typedef struct ipg_graph_view {
    uint64_t V;
    uint64_t E;
    int id_bytes;            /* 4 or 8 */
    int weight_bytes;        /* 0 when unweighted, else 1, 2, 4 or 8 */
    int directed;
    int has_in;              /* in_* are valid */
    const uint64_t* d_row;   /* V+1 */
    const void* d_adj;       /* E ids */
    const void* d_wgt;       /* E weights or NULL */
    const uint64_t* d_in_row;
    const void* d_in_adj;
    const void* d_in_wgt;
    uint64_t max_out_degree;
    uint64_t max_in_degree;
    uint64_t device_bytes;   /* HBM held by the graph */
    int symmetric;           /* every edge (u,v) has its reverse (v,u) with the
                                same weight: the rows are also the in-lists */
} ipg_graph_view;

/* Replaces ip_load_graph (src/iPregel_postamble.h:508-546): reads
 * <path>.config ("V E"), <path>.idx (V x idx_bytes row starts, no trailing E),
 * <path>.adj (E x id_bytes) and, when weighted, <path>.wgt (E x weight_bytes,
 * an extension: the reference never loads weights). */
int ipg_graph_load(const char* path, int id_bytes, int idx_bytes, int directed,
                   int weighted, int weight_bytes, int need_in, ipg_graph** out);

/* Same, from host buffers laid out as the files are (idx without trailing E). */
int ipg_graph_from_host(uint64_t V, uint64_t E, const void* idx, int idx_bytes,
                        const void* adj, int id_bytes, const void* wgt,
                        int weight_bytes, int directed, int need_in,
                        ipg_graph** out);

/* Loads new contents into a graph made by ipg_graph_from_host or
 * ipg_graph_load, in place: the same V, E and widths, host buffers laid out
 * as for ipg_graph_from_host.  The role of a second ip_load_graph
 * (src/iPregel_postamble.h:508-546) of a same-sized graph, without
 * allocating the graph again.  Derived data of the old contents are dropped:
 * degree classes, the symmetric declaration, and an in-CSR built for a
 * directed graph (rebuilt here).  Validation as at load; on a malformed
 * input the graph keeps the new contents and must not be run.  No engine may
 * be running on the graph, nor another refill of it; engines attached to it
 * attach again before their next run (a run without it fails with
 * IPG_EINVAL), and a request server must not hold it.  After a failed
 * refill every attach and run on the graph fails with IPG_EINVAL until a
 * refill succeeds.  The first call on a graph makes its stream and a few
 * small buffers; later calls allocate nothing and synchronise only that
 * stream, so one thread may refill a graph while kernels on another graph
 * run.  Degree classes (single_broadcast versions) and a directed graph's
 * in-CSR are derived data: the next attach of such a program rebuilds them,
 * and that rebuild allocates and synchronises the device. */
int ipg_graph_refill_host(ipg_graph* g, const void* idx, int idx_bytes,
                          const void* adj, const void* wgt);

/* The contents generation of a graph (0 at creation, +1 at every refill) and
 * whether its contents passed validation (1) or a refill failed (0).  The
 * engine records the generation at attach and checks both before each run. */
int ipg_graph_contents(const ipg_graph* g, uint64_t* generation, int* valid);

/* Wraps device buffers (row with V+1 entries) without copying; the caller
 * keeps them alive until ipg_graph_free. */
int ipg_graph_from_device(uint64_t V, uint64_t E, const uint64_t* d_row,
                          const void* d_adj, int id_bytes, const void* d_wgt,
                          int weight_bytes, int directed, int need_in,
                          ipg_graph** out);

/* Disjoint union of `count` graphs (no counterpart in the reference, which
 * loads one graph per program): a new graph whose vertices are those of
 * parts[0], then parts[1], ... with ids shifted by the vertex offsets voff
 * (count + 1 entries, host, nullable) and edges concatenated at the edge
 * offsets eoff (same).  A vertex-centric program run on the union gives each
 * part the result it gives alone, with ids shifted by the part's offset.
 * All parts share the id width and, if weighted, the weight width. */
int ipg_graph_concat(ipg_graph* const* parts, uint32_t count, int directed,
                     int need_in, ipg_graph** out, uint64_t* voff, uint64_t* eoff);

/* Several applications' captured superstep loops in one CUDA graph launch
 * (each application library adds its loop with ipg_app_loop_add).  The graph
 * is instantiated at the first launch; loops added later are not seen.
 * ipg_fused_launch is synchronous and returns the launch's device time. */
typedef struct ipg_fused ipg_fused;
int ipg_fused_create(ipg_fused** out);
void* ipg_fused_graph(ipg_fused* f);
int ipg_fused_launch(ipg_fused* f, void* stream, double* seconds);
void ipg_fused_free(ipg_fused* f);

/* Seeded generators on the device (counter-based SplitMix64, self-loops and
 * duplicates removed, vertex ids not permuted).  R-MAT: 2^scale vertices,
 * edge_factor * 2^scale sampled edges with quadrant probabilities a, b, c,
 * 1-a-b-c.  Erdos-Renyi: n vertices, m sampled edges.  undirected adds every
 * reverse edge.  wmax > 0 attaches u32 weights in [1, wmax], symmetric in
 * (u, v).  The CPU oracle produces the identical CSR for the same arguments. */
int ipg_graph_generate_rmat(uint32_t scale, uint32_t edge_factor, double a,
                            double b, double c, uint64_t seed, int undirected,
                            uint32_t wmax, int need_in, ipg_graph** out);
int ipg_graph_generate_er(uint64_t n, uint64_t m, uint64_t seed, int undirected,
                          uint32_t wmax, int need_in, ipg_graph** out);

int ipg_graph_view_get(const ipg_graph* g, ipg_graph_view* view);
/* Declares (1) or withdraws (0) that the stored graph is symmetric, weights
 * included.  The generators set it for undirected graphs; for other graphs
 * it is the caller's statement.  The push versions then may deliver a dense
 * superstep's broadcasts by pulling over the rows instead of pushing along
 * them; a wrong declaration gives wrong results, so the default is 0.
 * ipg_graph_check_symmetric verifies it on the device (rows must be sorted
 * by neighbour id; *result = 1 symmetric, 0 not, -1 rows unsorted). */
int ipg_graph_set_symmetric(ipg_graph* g, int symmetric);
int ipg_graph_check_symmetric(const ipg_graph* g, int* result);
/* The `directed` argument of ip_init (iPregel_preamble.h:298) for a graph
 * already resident: 0 makes the in-lists alias the rows (what the reference's
 * benchmarks load, pagerank.c:91), 1 makes them the transpose, built on the
 * next ipg_graph_build_in.  In-lists built for the other meaning are freed,
 * and a change bumps the contents generation (ipg_graph_contents): engines
 * attached before must attach again. */
int ipg_graph_set_directed(ipg_graph* g, int directed);
/* Builds the in-CSR if it is missing (no-op for undirected graphs). */
int ipg_graph_build_in(ipg_graph* g);
/* A renamed copy of g (no reference counterpart: an internal layout of the
 * engine).  Vertex n of the copy is vertex d_old_of_new[n] of g; the
 * vertices are numbered by descending count of occurrences in the rows
 * (ties by ascending id), so the most pushed-to or gathered-from vertices
 * share cache lines (every s-th edge counted when IPG_ORDER_SAMPLE sets
 * s; default every edge).  Every row keeps its edge order and weights, its ids
 * renamed; in-lists (present on g, or built first when need_in is set) are
 * renamed the same way, and degrees are unchanged.  d_new_of_old is the
 * inverse map (both 4-byte device arrays of V entries).  Row n of the copy
 * lists the same edges, in the same order, as row d_old_of_new[n] of g, so
 * a program reading neighbour ids reads g's row.  The copy and its maps are
 * cached on g and belong to it: a later call after a refill rebuilds them
 * in place (same size), one that asks for in-lists the copy lacks adds them
 * in place, and ipg_graph_free frees them; after ipg_graph_set_directed
 * changed the meaning the next call makes a new copy.  Needs V < 2^31. */
typedef struct ipg_order {
    ipg_graph* graph;
    const uint32_t* d_old_of_new;
    const uint32_t* d_new_of_old;
} ipg_order;
int ipg_graph_degree_order(ipg_graph* g, int need_in, ipg_order* out);
/* Copies the CSR back to host buffers in the file layout (idx: V x u64). */
int ipg_graph_to_host(const ipg_graph* g, uint64_t* idx, void* adj, void* wgt);
/* Writes <path>.config/.idx/.adj(/.wgt) in the reference loader's format. */
int ipg_graph_write(const ipg_graph* g, const char* path);
void ipg_graph_free(ipg_graph* g);

/* Static degree classes of all vertices (cached on the graph): list k holds
 * the vertices whose (in- or out-) degree d satisfies d <= t0 (k=0),
 * t0 < d <= t1 (k=1), d > t1 (k=2), each sorted by id.  Used by the
 * all-vertex gather of the single-broadcast version. */
typedef struct ipg_bins {
    const uint32_t* d_list[3];
    uint64_t count[3];
    uint64_t edges[3];       /* degree sum of each class */
    uint64_t t0, t1;
} ipg_bins;
int ipg_graph_bins(ipg_graph* g, int use_in, uint64_t t0, uint64_t t1,
                   ipg_bins* bins);

/* The same degree classes without allocating anything -- no counterpart in
 * the reference.  Meant for callers that must not call cudaMalloc: code
 * running while a stream is being captured, serving loops that cannot afford
 * the device-wide synchronisation an allocation may cause, and host programs
 * whose memory pool already owns all of HBM.  The caller passes the row
 * offsets (V+1 u64), d_lists (V u32: class 0, then class 1, then class 2,
 * each sorted by id, as ipg_graph_bins packs them) and d_totals (six u64 on
 * the device: the three class sizes, then their degree sums).  Scratch is a
 * static device array of 384 KiB that every GPU loading the library holds
 * until exit, so V is limited to 67,108,864 (IPG_EINVAL beyond).  The first
 * call on a device looks up the array's device address and keeps it for the
 * life of the process; make that first call before any stream capture.  A
 * cudaDeviceReset invalidates the kept address (the module is loaded anew),
 * so do not call this entry point on a device after resetting it.  All calls share the array: calls that overlap
 * on the GPU (different streams, or concurrent host threads) race and must be
 * serialised by the caller.  Asynchronous on `stream`. */
int ipg_degree_classes_noalloc(uint64_t V, const uint64_t* d_row, uint64_t t0,
                               uint64_t t1, uint32_t* d_lists, uint64_t* d_totals,
                               void* stream);

/* ------------------------------------------------------------------------
 * Frontier primitives (stream-ordered, no host synchronisation, safe to
 * capture in a CUDA graph).
 * ------------------------------------------------------------------------ */

/* Compacts the set bits of d_bitmap (NULL = all of [0, V)) into up to three
 * degree-class lists, as ipg_graph_bins does, appending at d_counts[k]
 * (u32, device, not reset here).  d_row gives degrees (NULL puts every vertex
 * in list 0).  d_edges (nullable, three u64 on the device) accumulates the
 * degree sum of each class.  clear != 0 zeroes the bitmap words it read. */
int ipg_compact(uint32_t* d_bitmap, uint64_t V, const uint64_t* d_row,
                uint64_t t0, uint64_t t1, uint32_t* d_list0, uint32_t* d_list1,
                uint32_t* d_list2, uint32_t* d_counts, uint64_t* d_edges,
                int clear, void* stream);

/* d_out (u64, device) += popcount(a | b) over nwords words (b nullable). */
int ipg_bitmap_popc_or(const uint32_t* d_a, const uint32_t* d_b, uint64_t nwords,
                       uint64_t* d_out, void* stream);

/* SM count of the current device (cached). */
int ipg_sm_count(void);


/* ------------------------------------------------------------------------
 * PageRank precision split -- no counterpart in the reference, whose
 * PageRank (benchmarks/pagerank.c:36-66,98-99, run by the single-broadcast
 * version, combiner_single_broadcast_postamble.h:57-89) is FP64 throughout.
 * Same formula and superstep structure: x = 1/V at superstep 0, then
 * x_v = (1-d)/V + d * sum over u in row(v) with deg u > 0 of x_u / deg u for
 * supersteps 1..rounds (the stored rows are the gather lists, as with the
 * reference's directed = false).  Values and broadcast quotients are FP32;
 * every gather sum is compensated (TwoSum-carried error, Neumaier's variant
 * of Kahan summation) when `compensated` != 0; diagnostics are FP64.
 * ------------------------------------------------------------------------ */
typedef struct ipg_pr_plan ipg_pr_plan;

/* Degree classes and scratch for runs on graph g (32-bit ids); holds
 * 12 bytes per vertex plus 8 bytes per 4096 hub edges of HBM until freed
 * (and builds the graph's in-lists if it is directed). */
int ipg_pr_plan_create(ipg_graph* g, ipg_pr_plan** plan);
void ipg_pr_plan_free(ipg_pr_plan* plan);
/* Vertices and edge sums of the thread / warp / hub classes, hub chunks. */
int ipg_pr_plan_info(const ipg_pr_plan* plan, uint64_t* class_counts, uint64_t* class_edges,
                     uint64_t* hub_chunks);

/* Runs rounds + 1 supersteps, leaving the values in d_values (V floats,
 * device).  d_diag (device, (rounds + 1) x 3 doubles) receives per superstep
 * {sum of x, sum of x over vertices without out-edges, sum |x - x_prev|}
 * (the last is 0 at superstep 0).  Asynchronous on `stream`; allocates and
 * synchronises nothing, so it can be captured into a CUDA graph. */
int ipg_pr_run_f32(ipg_pr_plan* plan, uint32_t rounds, double damping, int compensated,
                   float* d_values, double* d_diag, void* stream);

/* Per-vertex error of d_a (FP32) against d_ref (FP64), n entries on the
 * device: max abs, max rel (abs where ref is 0), mean abs, and the smallest
 * index with the max abs error.  Synchronous. */
int ipg_error_f32_f64(const float* d_a, const double* d_ref, uint64_t n, double* max_abs,
                      double* max_rel, double* mean_abs, uint64_t* argmax_abs, void* stream);

/* ------------------------------------------------------------------------
 * Request server -- no counterpart in the reference (one program, one graph
 * per process).  Resident graphs (32-bit ids, u32 weights for SSSP) answer
 * single-source shortest-path, connected-component and personalised-PageRank
 * queries.  Concurrent queries on one graph run as lanes of one fused
 * superstep kernel (64 min-plus lanes for SSSP, and for CC on graphs not
 * declared symmetric; 16 FP32 lanes for PPR); CC on a symmetric graph runs
 * as one union-find pass shared by the CC queries admitted together.
 * Queries join free lanes whenever their group finishes a superstep
 * (continuous batching), and lane groups plus result buffers are admitted
 * under an HBM budget.  Results: u32 per vertex (SSSP distance, UINT32_MAX
 * unreached; CC label = least vertex id reaching it, as benchmarks/cc.c), or
 * f32 per vertex (PPR after `ppr_rounds` gathers, as the ppr application).
 * ------------------------------------------------------------------------ */
typedef struct ipg_server ipg_server;
enum ipg_query_kind { IPG_QUERY_SSSP = 0, IPG_QUERY_PPR = 1, IPG_QUERY_CC = 2 };
enum ipg_query_state { IPG_QUERY_PENDING = 0, IPG_QUERY_RUNNING = 1, IPG_QUERY_FINISHING = 2, IPG_QUERY_DONE = 3 };
typedef struct ipg_server_stats {
    uint64_t submitted;
    uint64_t lanes_admitted;     /* CC queries admitted together share a lane */
    uint64_t supersteps;         /* fused supersteps launched, all groups */
    uint64_t kernel_launches;    /* superstep kernels launched */
    uint64_t groups_created;
    uint64_t groups_freed;
    uint64_t bytes_in_use;       /* lane groups and result buffers */
    uint64_t peak_bytes;
    uint64_t pull_supersteps;    /* min-plus supersteps relaxed by pulling */
} ipg_server_stats;

/* hbm_budget: bytes for lane groups and results (0 = unbounded).  The
 * environment variables IPG_SERVE_DELTA (near-far bucket width of SSSP lanes,
 * default 1024) and IPG_SERVE_PULL (0: min-plus supersteps never pull) are
 * read here. */
int ipg_server_create(uint64_t hbm_budget, uint32_t ppr_rounds, ipg_server** out);
void ipg_server_free(ipg_server* srv);
/* The graph stays owned by the caller and must outlive the server.  Builds
 * the graph's degree classes, which synchronises the device. */
int ipg_server_add_graph(ipg_server* srv, ipg_graph* g, int* gid);
/* Allocates and clears, now, the lane group that queries of `kind` on graph
 * gid run in (no-op when it exists), so that
 * their first arrivals find the device state resident; the group counts
 * against the HBM budget (IPG_EBUDGET when it does not fit) and, when idle,
 * may be evicted like any other.  Synchronous. */
int ipg_server_reserve(ipg_server* srv, int gid, int kind);
int ipg_server_submit(ipg_server* srv, int gid, int kind, uint64_t source, uint64_t* qid);
/* One scheduling pass: completed supersteps retire lanes, pending queries
 * take free lanes, next supersteps are launched.  Non-blocking.
 * *outstanding = queries not yet done. */
int ipg_server_poll(ipg_server* srv, uint64_t* outstanding);
/* State; latency (submit to result on the device) and queueing time, s. */
int ipg_server_query(ipg_server* srv, uint64_t qid, int* state, double* latency, double* queued);
int ipg_server_result(ipg_server* srv, uint64_t qid, void* host_out, uint64_t cap_bytes);
int ipg_server_result_device(ipg_server* srv, uint64_t qid, const void** d_ptr, uint64_t* bytes);
/* Forgets a done query; its result buffer returns to the server's pool. */
int ipg_server_release(ipg_server* srv, uint64_t qid);
int ipg_server_get_stats(ipg_server* srv, ipg_server_stats* out);
/* Per graph and group kind (0 min-plus, 1 PPR): summed device time of its
 * supersteps (groups run concurrently, so times overlap), supersteps, lanes
 * admitted, and for min-plus groups the lane-edge relaxations examined (an
 * edge relaxed for m lanes counts m).  Any output may be NULL. */
int ipg_server_group_stats(ipg_server* srv, int gid, int group_kind, double* busy_s,
                           uint64_t* supersteps, uint64_t* lanes, uint64_t* lane_edges);
/* Replays an arrival trace in real time (arrival[i] seconds from the start,
 * ascending): submits each query at its time, polls until all are done.
 * latency[i] counts from the scheduled arrival; keep_results = 0 releases
 * each result on completion. */
int ipg_server_run_trace(ipg_server* srv, uint64_t n, const double* arrival, const int* gid,
                         const int* kind, const uint64_t* source, int keep_results,
                         uint64_t* qids, double* latency, double* makespan);

#ifdef __cplusplus
}
#endif

#endif /* IPREGEL_B200_RUNTIME_H */
