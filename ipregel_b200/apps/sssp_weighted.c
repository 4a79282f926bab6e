/*
 * sssp_weighted.c -- integer-weight single-source shortest paths in the
 * iPregel interface (no counterpart in the reference, which never loads
 * weights).  A vertex whose distance drops broadcasts it; the weighted
 * broadcast extension (IP_BROADCAST_EDGE_MESSAGE) adds each out-edge's weight
 * on delivery, so each neighbour w hears dist + weight(v, w).  Min combines,
 * and (a + w) distributes over min, as the extension requires.
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
#include "iPregel.h"

IP_GLOBAL IP_VERTEX_ID_TYPE sssp_source = 0;

IP_DEVICE void ip_compute(struct ip_vertex_t* v)
{
    IP_MESSAGE_TYPE best = UINT_MAX;
    if (ip_is_first_superstep()) {
        v->value = UINT_MAX;
        if (v->id == sssp_source) best = 0;
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
