/*
 * cc.c -- connected components by minimum-label propagation, written against
 * the iPregel interface (same algorithm as the reference's benchmarks/cc.c:
 * every vertex starts with its own id as label, adopts the smallest label it
 * hears, and re-broadcasts when its label drops).
 */
#include <stdint.h>
#include <stdlib.h>

typedef uint64_t IP_NEIGHBOUR_COUNT_TYPE;
typedef IP_VERTEX_ID_TYPE IP_MESSAGE_TYPE;
typedef IP_VERTEX_ID_TYPE IP_VALUE_TYPE;
#include "iPregel.h"

IP_DEVICE void ip_compute(struct ip_vertex_t* v)
{
    const bool first = ip_is_first_superstep();
    IP_VALUE_TYPE label = first ? v->id : v->value;
    bool lowered = first;
    IP_MESSAGE_TYPE m;
    while (ip_get_next_message(v, &m)) {
        if (m < label) {
            label = m;
            lowered = true;
        }
    }
    v->value = label;
    if (lowered) ip_broadcast(v, label);
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

int main(int argc, char* argv[])
{
    if (argc != 6) {
        printf("usage: %s <graph> <output> <threads> <schedule> <chunk>\n", argv[0]);
        return -1;
    }
    ip_init(argv[1], atoi(argv[3]), argv[4], atoi(argv[5]), false, false);
    ip_run();
    FILE* out = fopen(argv[2], "w");
    if (!out) return -1;
    ip_dump(out);
    fclose(out);
    return 0;
}
