/*
 * reserved.c -- a two-superstep FP64 broadcast program for the engine's
 * reserved-pattern check: at superstep 0 the vertex "source" broadcasts
 * 1.0, or (parameter "allones" = 1) the FP64 bit pattern with all 64 bits
 * set, which the single_broadcast engine keeps for "no broadcast" in its
 * 8-byte slots and must refuse; at superstep 1 every vertex adds what it
 * received to its value (0 at the start) and halts.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t IP_NEIGHBOUR_COUNT_TYPE;
typedef double IP_MESSAGE_TYPE;
typedef double IP_VALUE_TYPE;
#define IP_APP_PARAMS
#include "iPregel.h"

IP_GLOBAL unsigned long long rs_source = 0;
IP_GLOBAL int rs_allones = 0;

IP_DEVICE void ip_compute(struct ip_vertex_t* v)
{
    if (ip_is_first_superstep()) {
        v->value = 0.0;
        if (v->id == rs_source) {
            double m = 1.0;
            if (rs_allones) {
                const unsigned long long bits = ~0ULL;
                memcpy(&m, &bits, sizeof m);
            }
            ip_broadcast(v, m);
        }
    } else {
        double m;
        while (ip_get_next_message(v, &m)) v->value += m;
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
    if (strcmp(key, "source") == 0) rs_source = (unsigned long long)value;
    else if (strcmp(key, "allones") == 0) rs_allones = value != 0.0;
    else return -1;
    return 0;
}

int main(int argc, char* argv[])
{
    (void)argc;
    (void)argv;
    return 0;
}
