/*
 * pagerank.c -- PageRank in the iPregel interface, the formula of the
 * reference's benchmarks/pagerank.c: x'(v) = 0.15/|V| + 0.85 * sum of the
 * shares x(u)/deg(u) received, a fixed number of rank updates (10 by
 * default, parameter "rounds"), vertices without out-edges send nothing.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t IP_NEIGHBOUR_COUNT_TYPE;
typedef double IP_MESSAGE_TYPE;
typedef double IP_VALUE_TYPE;
#define IP_NEEDS_OUT_NEIGHBOUR_COUNT
#define IP_APP_PARAMS
#include "iPregel.h"

IP_GLOBAL unsigned int pr_rounds = 10;
IP_GLOBAL double pr_damping = 0.85;

IP_DEVICE void ip_compute(struct ip_vertex_t* v)
{
    const double n = (double)ip_get_vertices_count();
    const double teleport = (pr_damping == 0.85) ? 0.15 : 1.0 - pr_damping;
    if (ip_is_first_superstep()) {
        v->value = 1.0 / n;
    } else {
        double sum = 0.0, share;
        while (ip_get_next_message(v, &share)) sum += share;
        v->value = teleport / n + pr_damping * sum;
    }
    if (ip_get_superstep() < pr_rounds) {
        if (v->out_neighbour_count > 0) ip_broadcast(v, v->value / v->out_neighbour_count);
    } else {
        ip_vote_to_halt(v);
    }
}

IP_DEVICE void ip_combine(IP_MESSAGE_TYPE* a, IP_MESSAGE_TYPE b) { *a += b; }

void ip_serialise_vertex(FILE* f, struct ip_vertex_t* v)
{
    fprintf(f, "%llu: %0.20f\n", (unsigned long long)v->id, v->value);
}

int ip_app_set_param(const char* key, double value)
{
    if (strcmp(key, "rounds") == 0) pr_rounds = (unsigned int)value;
    else if (strcmp(key, "damping") == 0) pr_damping = value;
    else return -1;
    return 0;
}

int main(int argc, char* argv[])
{
    if (argc != 6 && argc != 7) {
        printf("usage: %s <graph> <output> <threads> <schedule> <chunk> [rounds]\n", argv[0]);
        return -1;
    }
    if (argc == 7) pr_rounds = (unsigned int)atoi(argv[6]);
    ip_init(argv[1], atoi(argv[3]), argv[4], atoi(argv[5]), false, false);
    ip_run();
    FILE* out = fopen(argv[2], "w");
    if (!out) return -1;
    ip_dump(out);
    fclose(out);
    return 0;
}
