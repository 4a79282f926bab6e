/*
 * sssp_weighted.c -- integer-weight single-source shortest paths in the
 * iPregel interface (no counterpart in the reference, which never loads
 * weights).  A vertex whose distance drops broadcasts it; the weighted
 * broadcast extension (IP_BROADCAST_EDGE_MESSAGE) adds each out-edge's weight
 * on delivery, so each neighbour w hears dist + weight(v, w).  Min combines,
 * and (a + w) distributes over min, as the extension requires.
 *
 * Batch mode: with the parameter "batch_offsets" (the vertex offsets of a
 * disjoint union of graphs, ipg_graph_concat, on the device) every part's
 * vertex `source` (a local id) is a source, so one run computes every part's
 * shortest paths.
 */
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t IP_NEIGHBOUR_COUNT_TYPE;
typedef IP_VERTEX_ID_TYPE IP_MESSAGE_TYPE;
typedef IP_VERTEX_ID_TYPE IP_VALUE_TYPE;
typedef uint32_t IP_EDGE_WEIGHT_TYPE;
#define IP_NEEDS_OUT_NEIGHBOUR_WEIGHTS
#define IP_BROADCAST_EDGE_MESSAGE(m, w) ((IP_MESSAGE_TYPE)((m) + (w)))
#define IP_APP_PARAMS
#define IP_APP_PARAM_PTRS
#include "iPregel.h"

IP_GLOBAL IP_VERTEX_ID_TYPE sssp_source = 0;
IP_GLOBAL const uint64_t* sssp_batch = NULL; /* parts + 1 vertex offsets, or NULL */
IP_GLOBAL uint64_t sssp_batch_parts = 0;

IP_DEVICE static bool sssp_is_source(uint64_t id)
{
    if (!sssp_batch) return id == (uint64_t)sssp_source;
    uint64_t lo = 0, hi = sssp_batch_parts; /* sssp_batch[lo] <= id < sssp_batch[hi] */
    while (hi - lo > 1) {
        uint64_t mid = (lo + hi) / 2;
        if (sssp_batch[mid] <= id) lo = mid;
        else hi = mid;
    }
    return id == sssp_batch[lo] + (uint64_t)sssp_source && id < sssp_batch[lo + 1];
}

IP_DEVICE void ip_compute(struct ip_vertex_t* v)
{
    IP_MESSAGE_TYPE best = UINT_MAX;
    if (ip_is_first_superstep()) {
        v->value = UINT_MAX;
        if (sssp_is_source(v->id)) best = 0;
    } else {
        IP_MESSAGE_TYPE m;
        while (ip_get_next_message(v, &m))
            if (m < best) best = m;
    }
    if (best < v->value) {
        v->value = best;
        ip_broadcast(v, best);
    }
    ip_vote_to_halt(v);
}

IP_DEVICE void ip_combine(IP_MESSAGE_TYPE* a, IP_MESSAGE_TYPE b)
{
    if (b < *a) *a = b;
}

void ip_serialise_vertex(FILE* f, struct ip_vertex_t* v)
{
    fprintf(f, "%llu: %llu\n", (unsigned long long)v->id, (unsigned long long)v->value);
}

int ip_app_set_param(const char* key, double value)
{
    if (strcmp(key, "source") != 0) return -1;
    sssp_source = (IP_VERTEX_ID_TYPE)value;
    return 0;
}

int ip_app_set_param_ptr(const char* key, const void* ptr, uint64_t n)
{
    if (strcmp(key, "batch_offsets") != 0) return -1;
    sssp_batch = (const uint64_t*)ptr;
    sssp_batch_parts = (ptr && n > 1) ? n - 1 : 0;
    if (!sssp_batch_parts) sssp_batch = NULL;
    return 0;
}

int main(int argc, char* argv[])
{
    if (argc != 7) {
        printf("usage: %s <graph> <output> <threads> <schedule> <chunk> <source>\n", argv[0]);
        return -1;
    }
    sssp_source = (IP_VERTEX_ID_TYPE)strtoull(argv[6], NULL, 10);
    ip_init(argv[1], atoi(argv[3]), argv[4], atoi(argv[5]), false, true);
    ip_run();
    FILE* out = fopen(argv[2], "w");
    if (!out) return -1;
    ip_dump(out);
    fclose(out);
    return 0;
}
