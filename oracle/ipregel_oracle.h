/*
 * ipregel_oracle.h -- TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * A sequential, plain-C restatement of iPregel's superstep engine (the four
 * versions selected by IP_USE_SPREAD / IP_USE_SINGLE_BROADCAST) together with
 * the three benchmark applications, a weighted-SSSP and a personalised
 * PageRank application written in the same vertex-centric style, and the
 * seeded graph generators whose GPU counterparts live in the product library.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * call this code, and only as the checker.  Nothing in the product links it.
 *
 * Parity pin: tests/test_oracle_vs_reference.py runs the reference's own
 * OpenMP binaries (built from the reference sources into oracle/_ref/ by
 * oracle/Makefile) on the same graph files and compares dumps and the
 * per-superstep "ActiveVertexCount" lines; tests/golden/ holds fixtures made
 * the same way (tests/golden/make_golden.py).
 */
#ifndef IPREGEL_ORACLE_H
#define IPREGEL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Engine versions (reference: src/iPregel_preamble.h:319-331). */
enum og_version {
    OG_COMBINER = 0,                 /* src/combiner_postamble.h */
    OG_SINGLE_BROADCAST = 1,         /* src/combiner_single_broadcast_postamble.h */
    OG_SPREAD = 2,                   /* src/combiner_spread_postamble.h */
    OG_SPREAD_SINGLE_BROADCAST = 3   /* src/combiner_spread_single_broadcast_postamble.h */
};

/* Applications. */
enum og_app {
    OG_APP_CC = 0,        /* benchmarks/cc.c:31-63 */
    OG_APP_PAGERANK = 1,  /* benchmarks/pagerank.c:36-71 */
    OG_APP_SSSP = 2,      /* benchmarks/sssp.c:38-79 (hop count) */
    OG_APP_SSSP_W = 3,    /* integer-weight SSSP (no reference counterpart) */
    OG_APP_PPR = 4        /* personalised PageRank (no reference counterpart) */
};

typedef struct og_graph {
    uint64_t V;
    uint64_t E;
    const uint64_t* idx;   /* V row starts, the .idx layout (no trailing E) */
    const void* adj;       /* E vertex ids, 4 or 8 bytes each (.adj) */
    const uint32_t* wgt;   /* E weights parallel to adj, or NULL */
    int id_bytes;          /* 4 or 8 */
    int directed;          /* the ip_init "directed" argument */
} og_graph;

typedef struct og_params {
    int app;
    int version;
    uint64_t source;          /* SSSP / PPR source vertex */
    uint32_t rounds;          /* PageRank ROUND (benchmarks/pagerank.c:34) */
    double damping;           /* 0.85 in benchmarks/pagerank.c:51 */
    int truncate_push;        /* reproduce the u32 truncation of the 2nd+ message
                                 in the combiner versions' ip_cas
                                 (src/combiner_postamble.h:41) */
    uint64_t max_supersteps;  /* safety bound; 0 = unbounded */
} og_params;

typedef struct og_stats {
    uint64_t supersteps;      /* number of supersteps executed */
    uint64_t edges_traversed; /* broadcast deliveries + sends + gather reads */
} og_stats;

/* Runs one application under one engine version.  values_out receives V
 * values (u32 or u64 for integer apps as id_bytes says, double for PageRank
 * and PPR).  counts_out (capacity max_counts) receives the per-superstep
 * ActiveVertexCount that the reference prints.  Returns 0, or a negative
 * error code (-1 bad argument, -2 out of memory, -3 send_message under a
 * single-broadcast version, -4 superstep bound reached). */
int og_run(const og_graph* g, const og_params* p, void* values_out,
           uint64_t* counts_out, uint64_t max_counts, og_stats* stats);

/* Generators: seeded, counter-based, identical to the device generator in
 * the product library.  og_gen_* return the number of stored edges E and fill
 * idx (V entries) / adj (capacity max_edges u32 ids); NULL outputs only count.
 * kind 0 = R-MAT(scale, edge factor, a, b, c), kind 1 = Erdos-Renyi G(n, m). */
int64_t og_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b,
                    double c, uint64_t seed, int undirected, uint64_t* idx,
                    uint32_t* adj, uint64_t max_edges);
int64_t og_gen_er(uint64_t n, uint64_t m, uint64_t seed, int undirected,
                  uint64_t* idx, uint32_t* adj, uint64_t max_edges);
void og_gen_weights(uint64_t V, uint64_t E, const uint64_t* idx,
                    const uint32_t* adj, uint32_t wmax, uint64_t seed,
                    uint32_t* wgt);

/* Exact integer Dijkstra (binary heap) over out-edges; UINT32_MAX = unreached. */
int og_dijkstra(uint64_t V, uint64_t E, const uint64_t* idx,
                const uint32_t* adj, const uint32_t* wgt, uint64_t source,
                uint32_t* dist);

/* Writes <path>.config / .idx / .adj (and .wgt when wgt != NULL) in the
 * reference loader's format (src/iPregel_postamble.h:244-421). */
int og_write_graph(const char* path, uint64_t V, uint64_t E,
                   const uint64_t* idx, const uint32_t* adj,
                   const uint32_t* wgt);

#ifdef __cplusplus
}
#endif

#endif
