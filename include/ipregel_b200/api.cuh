/*
 * api.cuh -- the user-facing half of the drop-in headers: the reference's
 * public interface (src/iPregel_preamble.h:44-317) with the same names and
 * argument meaning, the vertex structure seen by ip_compute, and the
 * qualifier macros.  Included by include/iPregel.h.
 */
#ifndef IPREGEL_B200_API_CUH
#define IPREGEL_B200_API_CUH

#ifndef __CUDACC__
#error "iPregel-B200: compile the application with nvcc -x cu; ip_compute and ip_combine become device code."
#endif

#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "ipregel_b200.h"

/* Needs implications, as src/iPregel_preamble.h:32-38. */
#if defined(IP_NEEDS_OUT_NEIGHBOUR_IDS) && !defined(IP_NEEDS_OUT_NEIGHBOUR_COUNT)
#define IP_NEEDS_OUT_NEIGHBOUR_COUNT
#endif
#if defined(IP_NEEDS_IN_NEIGHBOUR_IDS) && !defined(IP_NEEDS_IN_NEIGHBOUR_COUNT)
#define IP_NEEDS_IN_NEIGHBOUR_COUNT
#endif

/* Version selection (src/iPregel_preamble.h:319-331) and the needs each
 * version forces (combiner_preamble.h:21-27, combiner_single_broadcast_
 * preamble.h:30-36, combiner_spread_preamble.h:28-34,
 * combiner_spread_single_broadcast_preamble.h:28-34). */
#define IPX_COMBINER 0
#define IPX_SINGLE_BROADCAST 1
#define IPX_SPREAD 2
#define IPX_SPREAD_SINGLE_BROADCAST 3
#if defined(IP_USE_SPREAD) && defined(IP_USE_SINGLE_BROADCAST)
#define IPX_VERSION IPX_SPREAD_SINGLE_BROADCAST
#elif defined(IP_USE_SPREAD)
#define IPX_VERSION IPX_SPREAD
#elif defined(IP_USE_SINGLE_BROADCAST)
#define IPX_VERSION IPX_SINGLE_BROADCAST
#else
#define IPX_VERSION IPX_COMBINER
#endif

#if IPX_VERSION == IPX_SINGLE_BROADCAST || IPX_VERSION == IPX_SPREAD_SINGLE_BROADCAST
#define IPX_PULL 1
#ifndef IP_NEEDS_IN_NEIGHBOUR_IDS
#define IP_NEEDS_IN_NEIGHBOUR_IDS
#endif
#ifndef IP_NEEDS_IN_NEIGHBOUR_COUNT
#define IP_NEEDS_IN_NEIGHBOUR_COUNT
#endif
#else
#define IPX_PULL 0
#ifndef IP_NEEDS_OUT_NEIGHBOUR_IDS
#define IP_NEEDS_OUT_NEIGHBOUR_IDS
#endif
#ifndef IP_NEEDS_OUT_NEIGHBOUR_COUNT
#define IP_NEEDS_OUT_NEIGHBOUR_COUNT
#endif
#endif

#if defined(IP_ID_OFFSET) && (IP_ID_OFFSET != 0) && !defined(IP_FORCE_DIRECT_MAPPING)
#error "iPregel-B200 supports direct id mapping only (IP_FORCE_DIRECT_MAPPING or IP_ID_OFFSET == 0)."
#endif

/* Qualifiers: the only source change an application needs.  IP_DEVICE goes
 * on ip_compute and ip_combine (and on any helper they call); IP_GLOBAL on
 * file-scope variables that ip_compute reads and main assigns. */
#define IP_DEVICE __device__
#define IP_GLOBAL __managed__

/* Combiner hint (compile flag, not a source change): lets message delivery use
 * the hardware atomic of the operator instead of a CAS loop around the user's
 * ip_combine.  ip_init checks the hint against ip_combine on the device and
 * stops with an error if they disagree. */
#define IP_COMBINE_GENERIC 0
#define IP_COMBINE_MIN 1
#define IP_COMBINE_MAX 2
#define IP_COMBINE_SUM 3
#ifndef IP_COMBINE_KIND
#define IP_COMBINE_KIND IP_COMBINE_GENERIC
#endif

/* Banner macros the reference's makefile defines (makefile:13, :29-46);
 * defaults so that a plain nvcc command line works. */
#ifndef VERSION
#define VERSION "1.0.0"
#endif
#ifndef COMMITS
#define COMMITS "ipregel-b200"
#endif
#ifndef IP_APPLICATION
#define IP_APPLICATION "unnamed"
#endif
#ifndef IP_MACHINE
#define IP_MACHINE "B200"
#endif
#ifndef COMPILATION_FLAGS
#define COMPILATION_FLAGS nvcc
#endif

/* Global state, as src/iPregel_preamble.h:44-57 (host side). */
size_t ip_superstep = 0;
size_t ip_edges_count = 0;
size_t ip_vertices_count = 0;
size_t ip_active_vertices = 0;
struct ip_vertex_t;
struct ip_vertex_t* ip_all_vertices = NULL;
int ip_thread_count;

/* Device mirrors read by ip_compute through the same accessor names.
 * ipd_superstep is the superstep the engine's kernels are in;
 * ipd_compute_superstep the one whose compute phase runs, which ip_compute
 * sees: the same, except in the single_broadcast version, whose fused kernel
 * gathers superstep s's broadcasts and runs the compute phase of s+1. */
__device__ size_t ipd_superstep;
__device__ size_t ipd_compute_superstep;
__device__ size_t ipd_vertices_count;
__device__ size_t ipd_edges_count;

/* The vertex seen by ip_compute: the reference's field names
 * (combiner_preamble.h:35-77 and the other versions' preambles), held in
 * registers for the duration of one ip_compute call.  Neighbour pointers are
 * device pointers into the resident CSR.  The ipx_* members are the engine's
 * per-call outbox. */
struct ip_vertex_t {
#ifdef IP_NEEDS_OUT_NEIGHBOUR_IDS
    IP_VERTEX_ID_TYPE* out_neighbours;
#endif
#ifdef IP_NEEDS_IN_NEIGHBOUR_IDS
    IP_VERTEX_ID_TYPE* in_neighbours;
#endif
#ifdef IP_NEEDS_OUT_NEIGHBOUR_COUNT
    IP_NEIGHBOUR_COUNT_TYPE out_neighbour_count;
#endif
#ifdef IP_NEEDS_IN_NEIGHBOUR_COUNT
    IP_NEIGHBOUR_COUNT_TYPE in_neighbour_count;
#endif
#ifdef IP_NEEDS_OUT_NEIGHBOUR_WEIGHTS
    IP_EDGE_WEIGHT_TYPE* out_neighbour_weights;
#endif
#ifdef IP_NEEDS_IN_NEIGHBOUR_WEIGHTS
    IP_EDGE_WEIGHT_TYPE* in_neighbour_weights;
#endif
    bool active;
    bool has_message;
    IP_VERTEX_ID_TYPE id;
    IP_MESSAGE_TYPE message;
    IP_VALUE_TYPE value;
    bool ipx_has_out;
    IP_MESSAGE_TYPE ipx_out;
};

/* The interface has C linkage, as the reference's (a C library): a C host or
 * a foreign-function binding calls ip_init / ip_run / ip_dump by name. */
#ifdef __cplusplus
extern "C" {
#endif

/* ---- accessors (src/iPregel_preamble.h:66-103) ---- */
__host__ __device__ size_t ip_get_superstep()
{
#ifdef __CUDA_ARCH__
    return __ldg((const unsigned long long*)&ipd_compute_superstep);
#else
    return ip_superstep;
#endif
}
__host__ __device__ bool ip_is_first_superstep() { return ip_get_superstep() == 0; }
__host__ __device__ size_t ip_get_vertices_count()
{
#ifdef __CUDA_ARCH__
    return __ldg((const unsigned long long*)&ipd_vertices_count);
#else
    return ip_vertices_count;
#endif
}
__host__ __device__ size_t ip_get_edges_count()
{
#ifdef __CUDA_ARCH__
    return __ldg((const unsigned long long*)&ipd_edges_count);
#else
    return ip_edges_count;
#endif
}
void ip_increment_superstep();
void ip_set_vertices_count(size_t vertices_count);
void ip_set_edges_count(size_t edges_count);
struct ip_vertex_t* ip_get_vertex_by_location(size_t location);
struct ip_vertex_t* ip_get_vertex_by_id(IP_VERTEX_ID_TYPE id);

/* ---- vertex functions, called from ip_compute (iPregel_preamble.h:105-166) ---- */
__device__ inline bool ip_has_message(struct ip_vertex_t* v) { return v->has_message; }
__device__ inline bool ip_get_next_message(struct ip_vertex_t* v, IP_MESSAGE_TYPE* message)
{
    /* One combined message per superstep (combiner_postamble.h:29-39). */
    if (v->has_message) {
        *message = v->message;
        v->has_message = false;
        return true;
    }
    return false;
}
__device__ inline void ip_send_message(IP_VERTEX_ID_TYPE id, IP_MESSAGE_TYPE message);
__device__ inline void ip_broadcast(struct ip_vertex_t* v, IP_MESSAGE_TYPE message);
__device__ inline void ip_vote_to_halt(struct ip_vertex_t* v);

void ip_init_vertex_range(IP_VERTEX_ID_TYPE first, IP_VERTEX_ID_TYPE last);
void ip_load_graph(const char* file_path, bool directed, bool weighted);

/* ---- safe functions (iPregel_preamble.h:177-250) ---- */
void* ip_safe_malloc(size_t size_to_malloc);
void* ip_safe_realloc(void* ptr, size_t size_to_realloc);
void ip_safe_free(void* ptr);
FILE* ip_safe_fopen(const char* file_path, const char* mode);
void ip_safe_fread(void* ptr, size_t size, size_t count, FILE* stream);
void ip_safe_fwrite(void* ptr, size_t size, size_t count, FILE* stream);

/* ---- user-defined functions (iPregel_preamble.h:262-290) ---- */
extern IP_DEVICE void ip_combine(IP_MESSAGE_TYPE* message_a, IP_MESSAGE_TYPE message_b);
extern void ip_serialise_vertex(FILE* f, struct ip_vertex_t* v);
extern IP_DEVICE void ip_compute(struct ip_vertex_t* v);

/* ---- running iPregel (iPregel_preamble.h:292-317) ---- */
void ip_init(const char* file_path, int number_of_threads, const char* schedule, int chunk_size, bool directed,
             bool weighted);
void ip_init_specific();
int ip_run();
void ip_dump(FILE* f);

#ifdef __cplusplus
}
#endif

#endif /* IPREGEL_B200_API_CUH */
