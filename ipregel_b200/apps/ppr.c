/*
 * ppr.c -- personalised PageRank in the iPregel interface (no counterpart in
 * the reference): the PageRank recurrence with all teleport mass on one seed,
 * x'(v) = 0.15 [v == seed] + 0.85 * sum of shares received; only vertices
 * holding mass broadcast, so the frontier grows from the seed.
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

IP_GLOBAL unsigned int ppr_rounds = 20;
IP_GLOBAL double ppr_damping = 0.85;
IP_GLOBAL IP_VERTEX_ID_TYPE ppr_seed = 0;

IP_DEVICE void ip_compute(struct ip_vertex_t* v)
{
    const double teleport = (ppr_damping == 0.85) ? 0.15 : 1.0 - ppr_damping;
    const bool is_seed = v->id == ppr_seed;
    if (ip_is_first_superstep()) {
        v->value = is_seed ? 1.0 : 0.0;
    } else {
        double sum = 0.0, share;
        while (ip_get_next_message(v, &share)) sum += share;
        v->value = (is_seed ? teleport : 0.0) + ppr_damping * sum;
    }
    if (ip_get_superstep() < ppr_rounds) {
        if (v->out_neighbour_count > 0 && v->value > 0.0) ip_broadcast(v, v->value / v->out_neighbour_count);
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
    if (strcmp(key, "rounds") == 0) ppr_rounds = (unsigned int)value;
    else if (strcmp(key, "damping") == 0) ppr_damping = value;
    else if (strcmp(key, "source") == 0) ppr_seed = (IP_VERTEX_ID_TYPE)value;
    else return -1;
    return 0;
}

int main(int argc, char* argv[])
{
    if (argc != 7) {
        printf("usage: %s <graph> <output> <threads> <schedule> <chunk> <seed>\n", argv[0]);
        return -1;
    }
    ppr_seed = (IP_VERTEX_ID_TYPE)strtoull(argv[6], NULL, 10);
    ip_init(argv[1], atoi(argv[3]), argv[4], atoi(argv[5]), false, false);
    ip_run();
    FILE* out = fopen(argv[2], "w");
    if (!out) return -1;
    ip_dump(out);
    fclose(out);
    return 0;
}
