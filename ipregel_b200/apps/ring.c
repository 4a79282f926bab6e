/*
 * ring.c -- a test program of ip_send_message to ids that are not
 * neighbours: at superstep 0 every vertex sends its id to vertex
 * (id * mul + add) mod V; at superstep 1 each vertex keeps the least id it
 * received (UINT32_MAX when none) and halts.  Parameters "mul" (default 1)
 * and "add" (default 1); mul > 1 sends several ids to one vertex, which the
 * combiner folds with min.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t IP_NEIGHBOUR_COUNT_TYPE;
typedef uint32_t IP_MESSAGE_TYPE;
typedef uint32_t IP_VALUE_TYPE;
#define IP_APP_PARAMS
#include "iPregel.h"

IP_GLOBAL unsigned long long ring_mul = 1;
IP_GLOBAL unsigned long long ring_add = 1;

IP_DEVICE void ip_compute(struct ip_vertex_t* v)
{
    if (ip_is_first_superstep()) {
        v->value = UINT32_MAX;
        const unsigned long long V = ip_get_vertices_count();
        const unsigned long long to = ((unsigned long long)v->id * ring_mul + ring_add) % V;
        ip_send_message((IP_VERTEX_ID_TYPE)to, (IP_MESSAGE_TYPE)v->id);
    } else {
        IP_MESSAGE_TYPE m;
        while (ip_get_next_message(v, &m))
            if (m < v->value) v->value = m;
        ip_vote_to_halt(v);
    }
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
    if (strcmp(key, "mul") == 0) ring_mul = (unsigned long long)value;
    else if (strcmp(key, "add") == 0) ring_add = (unsigned long long)value;
    else return -1;
    return 0;
}

int main(int argc, char* argv[])
{
    (void)argc;
    (void)argv;
    return 0;
}
