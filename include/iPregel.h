/*
 * iPregel.h -- drop-in replacement for the reference's src/iPregel.h:18-19,
 * running the superstep engine on an NVIDIA B200 (sm_100a).
 *
 * An application keeps the reference's structure: it defines the IP_* types,
 * includes this header, then defines ip_compute, ip_combine and
 * ip_serialise_vertex.  Two things change:
 *   - the program is compiled by nvcc as CUDA C++ (nvcc -x cu), linked with
 *     libipregel_b200.so, so that ip_compute and ip_combine are inlined into
 *     the engine's kernels;
 *   - the functions that run on the GPU carry IP_DEVICE, and the file-scope
 *     variables they read carry IP_GLOBAL (benchmarks/pagerank.c:32-33 and
 *     benchmarks/sssp.c:36 need it; cc.c needs only IP_DEVICE).
 * The version is chosen exactly as in the reference (src/iPregel_preamble.h:
 * 319-331): IP_USE_SPREAD and/or IP_USE_SINGLE_BROADCAST.
 */
#ifndef IPREGEL_B200_DROPIN_H
#define IPREGEL_B200_DROPIN_H

#include "ipregel_b200/api.cuh"
#include "ipregel_b200/engine.cuh"
#include "ipregel_b200/host.cuh"

#endif
