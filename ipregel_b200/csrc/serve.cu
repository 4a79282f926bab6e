// serve.cu -- a request server over resident graphs (no counterpart in the
// reference, which runs one program on one graph per process).
//
// Queries: single-source shortest paths (integer weights), connected
// components (labels as benchmarks/cc.c: the least vertex id that reaches a
// vertex), and personalised PageRank (x' = 0.15 [v == seed] + 0.85 * sum of
// x_u / deg u over the row, as the ppr application, in FP32 with compensated
// sums).  Graphs and per-query vertex state stay in HBM.  Concurrent queries
// on one graph share a lane group and advance together, one fused superstep
// kernel for all their lanes:
//
//   min-plus group (SSSP; CC on graphs not declared symmetric): 64 lanes;
//     dist[v][lane] (u32, 256 bytes per vertex, so the lanes of one vertex
//     are one coalesced line), a bit-packed frontier mask per vertex (u64, a
//     bit per lane) double-buffered, and the frontier as degree-class lists.
//     A vertex with few frontier lanes has a thread per edge relax all its
//     lanes; one with many has a thread per lane relax each edge in turn.
//     nd = dist[v][k] + w (w = 0 for a CC lane) goes into dist[u][k] by
//     atomicMin, and the improved lanes into u's next mask.  A lane whose
//     frontier empties is finished.
//   CC on a graph declared symmetric: union-find over the edges, one pass
//     (the labels of min-label propagation are the least id of each
//     component); CC queries admitted together share the pass.
//   PPR group: 32 lanes; the broadcast quotients b[v][lane] = x/deg (FP32,
//     128 bytes per vertex, one line) double-buffered; a pull gather over
//     every row: 8 threads per low-degree vertex, each reading one float4
//     quad of every in-neighbour's row, a warp per vertex of higher degree
//     (four rows per load instruction), hub rows in chunks.  64 lanes (two
//     lines per row) measured slower in the mixed serving workload: a
//     superstep cost about twice as much, for half the supersteps.  A lane runs exactly
//     `rounds` gathers after admission and writes its last values into the
//     query's result buffer.
//
// Continuous batching: each group advances on its own stream; whenever its
// superstep has completed, finished lanes retire and pending queries take the
// free lanes before the next superstep is launched, so queries join and leave
// while others are in flight, and groups of different graphs overlap on the
// device.  A lane's arithmetic depends on nothing but its own query (min-plus
// and union-find are order independent; the PPR sums run in a fixed
// per-vertex order whatever the other lanes do), so a query's result is the
// same alone and in any mix.
//
// Admission is bounded by an HBM budget over the server's lane groups and
// result buffers; groups without busy lanes are freed, least recently used
// first, when a new group needs room.
#include "ipregel_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

extern "C" int ipg_internal_fail(int code, const char* msg);

namespace {

constexpr int MP_K = 64;
constexpr int PP_K = 32;           // PPR lanes: a row of 32 FP32 quotients is one 128-byte line
constexpr int PP_Q = PP_K / 4;     // float4 quads per row
constexpr int PP_SLOTS = 32 / PP_Q;  // rows per warp load instruction
static_assert(PP_K <= 64 && PP_Q <= 16 && PP_K % 16 == 0, "PPR lanes: a warp covers whole rows");
constexpr int SRV_THREADS = 256;
constexpr uint64_t MP_T0 = 8, MP_T1 = 4096;
constexpr uint64_t PP_T0 = 64;                      // PPR: quads up to this degree, then warps
constexpr uint64_t PP_NOALLOC_MAX_V = 67108864ull;  // ipg_degree_classes_noalloc's vertex limit
constexpr uint32_t HUB_CHUNK = 1024;
constexpr uint32_t SRV_INF = 0xffffffffu;
constexpr unsigned FULL = 0xffffffffu;
// Up to MP_SPARSE lanes of a vertex: a thread per edge, each relaxing all.
constexpr int MP_SPARSE = 8;
// A min-plus superstep pulls (symmetric graphs) when its frontier holds at
// least E / MP_PULL_DIV edges and at least MP_PULL_LANES lanes are busy.  On
// R-MAT graphs of scale 22 and 25 with 32 busy lanes, the dense supersteps
// took 15-40 % less time pulled than pushed; with 5 lanes, 3-4 times more.
constexpr uint64_t MP_PULL_DIV = 4;
constexpr int MP_PULL_LANES = 16;
// Resident CTAs per SM the min-plus kernels are compiled for (64 registers).
#define MP_CTAS 4

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// Shared helpers
// ---------------------------------------------------------------------------

// Neighbour ids and weights a superstep reads once per edge: loaded
// evict-first (ld.global.cs), so the gigabytes of edge stream leave the L2 to
// the lane rows that edges read at random.
__device__ __forceinline__ uint32_t ld_edge(const uint32_t* p) { return __ldcs(p); }

// Status of a min-plus group after a superstep, copied to the host in one
// transfer: lane flags, list sizes, hub chunks of list 2, least deferred
// distance of each lane.
struct MpStatus {
    unsigned long long any;   // lanes that improved a distance
    unsigned long long near;  // lanes that relaxed a vertex below their threshold
    unsigned long long far;   // lanes that deferred a vertex
    uint32_t cnt[3];
    uint32_t chunks;
    uint32_t far_min[64];     // least deferred distance per lane
    unsigned long long work;  // lane-edge relaxations examined (edges x lanes relaxing them)
    unsigned long long esum[3];  // degree sums of the next frontier's classes
};

inline uint32_t warp_grid(uint64_t tasks)
{
    const uint64_t ctas = (tasks + (SRV_THREADS / 32) - 1) / (SRV_THREADS / 32);
    return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(ctas, 1), 0x7fffffffULL);
}

inline uint32_t thread_grid(uint64_t n)
{
    const uint64_t ctas = (n + SRV_THREADS - 1) / SRV_THREADS;
    return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(ctas, 1), 0x7fffffffULL);
}

// At most the CTAs of `kernel` resident at once on the device: the kernels
// stride over their work, and CTAs beyond that would run as a second wave.
template <class K>
uint32_t resident_cap(K kernel, uint32_t want)
{
    static std::mutex mu;
    static std::map<const void*, uint32_t> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find((const void*)kernel);
    if (it == cache.end()) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, SRV_THREADS, 0) != cudaSuccess || n <= 0) n = 1;
        it = cache.emplace((const void*)kernel, (uint32_t)(n * ipg_sm_count())).first;
    }
    return std::min(want, it->second);
}

// prefix[i] = sum over j < i of ceil(deg(list[j]) / HUB_CHUNK); prefix[n] =
// total, also written to *total when given.
__global__ void __launch_bounds__(1024) k_chunk_prefix(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                                                       const uint64_t* __restrict__ row, uint32_t* __restrict__ prefix,
                                                       uint32_t* __restrict__ total)
{
    __shared__ uint32_t s[1024];
    __shared__ uint32_t carry;
    const uint32_t n = *count;
    const int t = threadIdx.x;
    if (t == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += 1024) {
        const uint32_t i = base + t;
        uint32_t c = 0;
        if (i < n) {
            const uint64_t v = list[i];
            c = (uint32_t)((row[v + 1] - row[v] + HUB_CHUNK - 1) / HUB_CHUNK);
        }
        s[t] = c;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            const uint32_t x = t >= off ? s[t - off] : 0;
            __syncthreads();
            s[t] += x;
            __syncthreads();
        }
        if (i < n) prefix[i] = carry + s[t] - c;
        __syncthreads();
        if (t == 1023) carry += s[1023];
        __syncthreads();
    }
    if (t == 0) {
        prefix[n] = carry;
        if (total) *total = carry;
    }
}

__device__ __forceinline__ uint32_t hub_of_chunk(const uint32_t* __restrict__ prefix, uint32_t n, uint32_t c)
{
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= c) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Min-plus lanes (SSSP, CC by label propagation)
// ---------------------------------------------------------------------------
struct MpArgs {
    const uint64_t* __restrict__ row;
    const uint32_t* __restrict__ adj;
    const uint32_t* __restrict__ wgt;  // null for an unweighted graph (CC only)
    uint32_t* __restrict__ dist;
    const uint64_t* __restrict__ front;
    uint64_t* __restrict__ next;
    uint32_t* __restrict__ fbm;        // bit per vertex: in the next frontier
    const uint32_t* __restrict__ fcur; // bit per vertex: in this superstep's frontier
    const uint32_t* __restrict__ thr;  // per lane: distances below it relax now
    MpStatus* __restrict__ st;
    uint64_t wmask;                    // lanes whose edges carry their weight (SSSP)
    uint64_t busy;                     // lanes holding a query
};

// Per-thread flags of a superstep, reduced per CTA into the status.
struct MpAcc {
    unsigned long long any = 0, near = 0, far = 0, work = 0;
};

// Relaxes edge (v -> u, weight t) for the lanes ks[0..m) of v (distances
// ds); returns the lanes whose distance at u may have dropped.  The
// atomicMin is issued only when a plain read of u's distance (possibly stale,
// and then only larger) shows an improvement, and its result is not waited
// for: a lane another thread improved further meanwhile is marked needlessly,
// which costs one redundant relaxation and changes no distance.
template <int MAXL>
__device__ __forceinline__ unsigned long long mp_relax_edge(const MpArgs& a, uint32_t u, uint32_t t, int m,
                                                            const int* ks, const uint32_t* ds)
{
    uint32_t cur[MAXL];
#pragma unroll
    for (int j = 0; j < MAXL; j++) cur[j] = j < m ? a.dist[(uint64_t)u * MP_K + ks[j]] : 0u;
    unsigned long long bits = 0;
#pragma unroll
    for (int j = 0; j < MAXL; j++) {
        if (j >= m) break;
        const uint32_t nd = ds[j] + (((a.wmask >> ks[j]) & 1ULL) ? t : 0u);
        if (nd < cur[j]) {
            atomicMin(&a.dist[(uint64_t)u * MP_K + ks[j]], nd);
            bits |= 1ULL << ks[j];
        }
    }
    return bits;
}

// Lanes `bits` of u join the next frontier.
__device__ __forceinline__ void mp_mark(const MpArgs& a, uint32_t u, unsigned long long bits)
{
    atomicOr((unsigned long long*)&a.next[u], bits);
    const uint32_t fb = 1u << (u & 31);
    if (!(a.fbm[u >> 5] & fb)) atomicOr(&a.fbm[u >> 5], fb);
}

// Edges e0 + lane, e0 + lane + stride, ... of v for its m <= L lanes; L is
// the smallest of 1, 2, 4, 8 holding m, so no instruction is issued for
// lanes v does not have.
template <int L>
__device__ __forceinline__ void mp_edges_sparse(const MpArgs& a, uint64_t e0, uint64_t e1, uint64_t lane,
                                                uint64_t stride, int m, const int* ks, const uint32_t* ds,
                                                MpAcc& acc)
{
    for (uint64_t e = e0 + lane; e < e1; e += stride) {
        const uint32_t u = ld_edge(&a.adj[e]);
        const uint32_t t = a.wgt ? ld_edge(&a.wgt[e]) : 0u;
        acc.work += (unsigned)m;
        const unsigned long long bits = mp_relax_edge<L>(a, u, t, m, ks, ds);
        if (bits) {
            mp_mark(a, u, bits);
            acc.any |= bits;
        }
    }
}

__device__ __forceinline__ void mp_edges_sparse_any(const MpArgs& a, uint64_t e0, uint64_t e1, uint64_t lane,
                                                    uint64_t stride, int m, const int* ks, const uint32_t* ds,
                                                    MpAcc& acc)
{
    if (m == 1) mp_edges_sparse<1>(a, e0, e1, lane, stride, m, ks, ds, acc);
    else if (m == 2) mp_edges_sparse<2>(a, e0, e1, lane, stride, m, ks, ds, acc);
    else if (m <= 4) mp_edges_sparse<4>(a, e0, e1, lane, stride, m, ks, ds, acc);
    else mp_edges_sparse<MP_SPARSE>(a, e0, e1, lane, stride, m, ks, ds, acc);
}

// Near-far ordering per lane.  A frontier lane whose distance at v is below
// the lane's threshold relaxes v's edges now; one at or above it stays in the
// frontier untouched (deferred), and the least deferred distance of each lane
// is kept (s_fmin, per CTA).  A lane with no vertex below its threshold in a
// superstep has its threshold raised (host side); one with neither is done.
// Relaxing in rough distance order leaves fewer vertices to be relaxed again
// after their distance drops; the fixpoint, and so every result, is the same.
__device__ __forceinline__ void mp_defer(const MpArgs& a, uint32_t v, unsigned long long lanes, MpAcc& acc)
{
    mp_mark(a, v, lanes);
    acc.far |= lanes;
}

// One warp relaxes the edges [e0, e1) of v for all of v's frontier lanes
// below their thresholds: a thread per edge when few lanes remain, else a
// thread per lane.  The warp classifies the lanes itself (a lane each).
__device__ __forceinline__ void mp_relax(const MpArgs& a, uint64_t v, uint64_t e0, uint64_t e1, bool mark_deferred,
                                         MpAcc& acc, uint32_t* s_fmin)
{
    const int lane = threadIdx.x & 31;
    const uint64_t M = a.front[v];
    if (!M) return;
    const bool in0 = (M >> lane) & 1ULL, in1 = (M >> (lane + 32)) & 1ULL;
    const uint32_t d0 = in0 ? a.dist[v * MP_K + lane] : SRV_INF;
    const uint32_t d1 = in1 ? a.dist[v * MP_K + 32 + lane] : SRV_INF;
    const bool act0 = in0 && d0 < __ldg(&a.thr[lane]);
    const bool act1 = in1 && d1 < __ldg(&a.thr[lane + 32]);
    const uint32_t Mlo = __ballot_sync(FULL, act0), Mhi = __ballot_sync(FULL, act1);
    const uint32_t Dlo = __ballot_sync(FULL, in0 && !act0), Dhi = __ballot_sync(FULL, in1 && !act1);
    if (Dlo | Dhi) {
        if (in0 && !act0) atomicMin(&s_fmin[lane], d0);
        if (in1 && !act1) atomicMin(&s_fmin[lane + 32], d1);
        if (mark_deferred && lane == 0) mp_defer(a, (uint32_t)v, (unsigned long long)Dlo | ((unsigned long long)Dhi << 32), acc);
    }
    const unsigned long long R = (unsigned long long)Mlo | ((unsigned long long)Mhi << 32);
    if (!R) return;
    if (lane == 0) {
        acc.near |= R;
        if (__popcll(R) > MP_SPARSE) acc.work += (unsigned long long)__popcll(R) * (e1 - e0);
    }
    if (__popcll(R) <= MP_SPARSE) {
        int ks[MP_SPARSE];
        uint32_t ds[MP_SPARSE];
        int m = 0;
        unsigned long long rest = R;
        while (rest && m < MP_SPARSE) {
            const int k = __ffsll((long long)rest) - 1;
            rest &= rest - 1;
            ks[m] = k;
            ds[m] = __shfl_sync(FULL, k < 32 ? d0 : d1, k & 31);
            m++;
        }
        mp_edges_sparse_any(a, e0, e1, lane, 32, m, ks, ds, acc);
        return;
    }
    const bool w0 = ((uint32_t)a.wmask >> lane) & 1u, w1 = ((uint32_t)(a.wmask >> 32) >> lane) & 1u;
    for (uint64_t e = e0; e < e1; e += 32) {
        const uint64_t ee = e + lane;
        const uint32_t wj = ee < e1 ? ld_edge(&a.adj[ee]) : 0u;
        const uint32_t tj = (ee < e1 && a.wgt) ? ld_edge(&a.wgt[ee]) : 0u;
        const int nj = (int)((e1 - e) < 32 ? (e1 - e) : 32);
        for (int j0 = 0; j0 < nj; j0 += 4) {
            uint32_t u[4], t[4], c0[4], c1[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                u[q] = __shfl_sync(FULL, wj, (j0 + q) & 31);
                t[q] = __shfl_sync(FULL, tj, (j0 + q) & 31);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const bool ok = j0 + q < nj;
                c0[q] = (ok && act0) ? a.dist[(uint64_t)u[q] * MP_K + lane] : 0u;
                c1[q] = (ok && act1) ? a.dist[(uint64_t)u[q] * MP_K + 32 + lane] : 0u;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (j0 + q >= nj) break;
                bool i0 = false, i1 = false;
                if (act0) {
                    const uint32_t nd = d0 + (w0 ? t[q] : 0u);
                    if (nd < c0[q]) {
                        atomicMin(&a.dist[(uint64_t)u[q] * MP_K + lane], nd);
                        i0 = true;
                    }
                }
                if (act1) {
                    const uint32_t nd = d1 + (w1 ? t[q] : 0u);
                    if (nd < c1[q]) {
                        atomicMin(&a.dist[(uint64_t)u[q] * MP_K + 32 + lane], nd);
                        i1 = true;
                    }
                }
                const uint32_t b0 = Mlo ? __ballot_sync(FULL, i0) : 0u;
                const uint32_t b1 = Mhi ? __ballot_sync(FULL, i1) : 0u;
                if ((b0 | b1) && lane == 0) {
                    const unsigned long long bits = (unsigned long long)b0 | ((unsigned long long)b1 << 32);
                    mp_mark(a, u[q], bits);
                    acc.any |= bits;
                }
            }
        }
    }
}

// The CTA's flags and least deferred distances into the status.
__device__ __forceinline__ void mp_block_flush(MpAcc acc, const MpArgs& a, uint32_t* s_fmin)
{
    __shared__ unsigned long long s[4][SRV_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        acc.any |= __shfl_down_sync(FULL, acc.any, o);
        acc.near |= __shfl_down_sync(FULL, acc.near, o);
        acc.far |= __shfl_down_sync(FULL, acc.far, o);
        acc.work += __shfl_down_sync(FULL, acc.work, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s[0][threadIdx.x >> 5] = acc.any;
        s[1][threadIdx.x >> 5] = acc.near;
        s[2][threadIdx.x >> 5] = acc.far;
        s[3][threadIdx.x >> 5] = acc.work;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t |= s[threadIdx.x][w];
        unsigned long long* dst = threadIdx.x == 0 ? &a.st->any : (threadIdx.x == 1 ? &a.st->near : &a.st->far);
        if (t) atomicOr(dst, t);
    } else if (threadIdx.x == 3) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s[3][w];
        if (t) atomicAdd(&a.st->work, t);
    }
    if (threadIdx.x < MP_K && s_fmin[threadIdx.x] != SRV_INF) atomicMin(&a.st->far_min[threadIdx.x], s_fmin[threadIdx.x]);
}

__device__ __forceinline__ void mp_fmin_init(uint32_t* s_fmin)
{
    if (threadIdx.x < MP_K) s_fmin[threadIdx.x] = SRV_INF;
    __syncthreads();
}

// A thread per low-degree frontier vertex (class 0): its lanes one at a
// time, each over the vertex's few edges.
__global__ void __launch_bounds__(SRV_THREADS, MP_CTAS) k_mp_thread(MpArgs a, const uint32_t* __restrict__ list,
                                                                     const uint32_t* __restrict__ count)
{
    __shared__ uint32_t s_fmin[MP_K];
    mp_fmin_init(s_fmin);
    const uint32_t n = *count;
    MpAcc acc;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = list[i];
        uint64_t M = a.front[v];
        const uint64_t e0 = a.row[v], e1 = a.row[v + 1];
        unsigned long long deferred = 0;
        while (M) {
            const int k = __ffsll((long long)M) - 1;
            M &= M - 1;
            const unsigned long long bit = 1ULL << k;
            const uint32_t d = a.dist[(uint64_t)v * MP_K + k];
            if (d >= __ldg(&a.thr[k])) {
                deferred |= bit;
                atomicMin(&s_fmin[k], d);
                continue;
            }
            acc.near |= bit;
            acc.work += e1 - e0;
            const bool weighted = (a.wmask >> k) & 1ULL;
            for (uint64_t e = e0; e < e1; e++) {
                const uint32_t u = a.adj[e];
                const uint32_t nd = d + ((weighted && a.wgt) ? a.wgt[e] : 0u);
                uint32_t* p = &a.dist[(uint64_t)u * MP_K + k];
                if (nd < *p) {
                    atomicMin(p, nd);
                    mp_mark(a, u, bit);
                    acc.any |= bit;
                }
            }
        }
        if (deferred) mp_defer(a, v, deferred, acc);
    }
    __syncthreads();
    mp_block_flush(acc, a, s_fmin);
}

// A warp per frontier vertex (class 1).
__global__ void __launch_bounds__(SRV_THREADS, MP_CTAS) k_mp_vertices(MpArgs a, const uint32_t* __restrict__ list,
                                                                       const uint32_t* __restrict__ count)
{
    __shared__ uint32_t s_fmin[MP_K];
    mp_fmin_init(s_fmin);
    const uint32_t n = *count;
    MpAcc acc;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint64_t v = list[i];
        mp_relax(a, v, a.row[v], a.row[v + 1], true, acc, s_fmin);
    }
    __syncthreads();
    mp_block_flush(acc, a, s_fmin);
}

// A warp per HUB_CHUNK edges of a frontier hub (class 2); the chunk holding
// the hub's first edge marks its deferred lanes.
__global__ void __launch_bounds__(SRV_THREADS, MP_CTAS) k_mp_hubs(MpArgs a, const uint32_t* __restrict__ list,
                                                                   const uint32_t* __restrict__ count,
                                                                   const uint32_t* __restrict__ prefix)
{
    __shared__ uint32_t s_fmin[MP_K];
    mp_fmin_init(s_fmin);
    const uint32_t n = *count;
    MpAcc acc;
    if (n) {
        const uint32_t chunks = prefix[n];
        const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
        for (uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; c < chunks; c += warps) {
            const uint32_t i = hub_of_chunk(prefix, n, (uint32_t)c);
            const uint64_t v = list[i];
            const uint64_t e0 = a.row[v] + (uint64_t)((uint32_t)c - prefix[i]) * HUB_CHUNK;
            const uint64_t end = a.row[v + 1];
            mp_relax(a, v, e0, e0 + HUB_CHUNK < end ? e0 + HUB_CHUNK : end, (uint32_t)c == prefix[i], acc, s_fmin);
        }
    }
    __syncthreads();
    mp_block_flush(acc, a, s_fmin);
}

// Pull supersteps (direction-optimised relaxation, symmetric graphs: a
// vertex's row lists its in-neighbours).  When the frontier covers a large
// part of the graph, most edges are relaxed for many lanes at once and the
// push kernels' atomicMin traffic dominates; pulling, the warp that owns a
// vertex u gathers, over u's in-neighbours v in this superstep's frontier
// (bitmap fcur), the candidates dist[v][k] + w of v's frontier lanes k below
// their thresholds, and lowers dist[u][k] with a plain store: u has one owner,
// so no atomics.  A neighbour's distance that its own owner lowers during the
// same superstep is still a path length, and the lowered neighbour is in the
// next frontier anyway, so reading either value reaches the same fixpoint.
// Each vertex also classifies its own frontier lanes as the push kernels do:
// below the threshold they are consumed (near), at or above it deferred into
// the next frontier.

// Least candidates over in-edges [e0, e1) of the warp's vertex: lane k in b0,
// lane k + 32 in b1 (SRV_INF when none).  Frontier neighbours are found by a
// ballot over 32 edges at a time and taken 4 at a time.  Every busy lane of a
// frontier neighbour below its threshold is a candidate, whether or not the
// lane itself is in the neighbour's frontier: a lane outside it was relaxed
// at its current distance already, so its candidate lowers nothing, and not
// reading the neighbour's frontier mask saves a dependent load per edge.
// Work counts frontier in-edges.
__device__ __forceinline__ void mp_pull_edges(const MpArgs& a, uint64_t e0, uint64_t e1, uint32_t thr0, uint32_t thr1,
                                              bool w0, bool w1, uint32_t& b0, uint32_t& b1, MpAcc& acc)
{
    const int lane = threadIdx.x & 31;
    const bool live0 = (a.busy >> lane) & 1ULL, live1 = (a.busy >> (lane + 32)) & 1ULL;
    for (uint64_t e = e0; e < e1; e += 32) {
        const uint64_t ee = e + lane;
        const uint32_t vj = ee < e1 ? ld_edge(&a.adj[ee]) : 0u;
        const bool fr = ee < e1 && ((a.fcur[vj >> 5] >> (vj & 31)) & 1u);
        uint32_t fm = __ballot_sync(FULL, fr);
        if (!fm) continue;
        const uint32_t tj = (fr && a.wgt) ? ld_edge(&a.wgt[ee]) : 0u;
        while (fm) {
            int j[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                j[q] = fm ? __ffs(fm) - 1 : -1;
                fm &= fm ? fm - 1 : 0u;
            }
            uint32_t v[4], t[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                v[q] = __shfl_sync(FULL, vj, j[q] & 31);
                t[q] = __shfl_sync(FULL, tj, j[q] & 31);
            }
            uint32_t d0[4], d1[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                d0[q] = j[q] >= 0 && live0 ? a.dist[(uint64_t)v[q] * MP_K + lane] : SRV_INF;
                d1[q] = j[q] >= 0 && live1 ? a.dist[(uint64_t)v[q] * MP_K + 32 + lane] : SRV_INF;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (d0[q] < thr0) b0 = min(b0, d0[q] + (w0 ? t[q] : 0u));
                if (d1[q] < thr1) b1 = min(b1, d1[q] + (w1 ? t[q] : 0u));
            }
            if (lane == 0) acc.work += (unsigned long long)(j[0] >= 0) + (j[1] >= 0) + (j[2] >= 0) + (j[3] >= 0);
        }
    }
}

// Own frontier lanes of u (mask fu, distances du0/du1 read by the caller):
// near lanes into acc.near, deferred ones into acc.far, the least deferred
// distance per lane into s_fmin; returns the deferred lanes.
__device__ __forceinline__ unsigned long long mp_pull_own(unsigned long long fu, uint32_t du0, uint32_t du1,
                                                          uint32_t thr0, uint32_t thr1, MpAcc& acc, uint32_t* s_fmin)
{
    const int lane = threadIdx.x & 31;
    const bool in0 = (fu >> lane) & 1ULL, in1 = (fu >> (lane + 32)) & 1ULL;
    const bool far0 = in0 && du0 >= thr0, far1 = in1 && du1 >= thr1;
    if (far0) atomicMin(&s_fmin[lane], du0);
    if (far1) atomicMin(&s_fmin[lane + 32], du1);
    const unsigned long long N = (unsigned long long)__ballot_sync(FULL, in0 && !far0) |
                                 ((unsigned long long)__ballot_sync(FULL, in1 && !far1) << 32);
    const unsigned long long D = (unsigned long long)__ballot_sync(FULL, far0) |
                                 ((unsigned long long)__ballot_sync(FULL, far1) << 32);
    if (lane == 0) {
        acc.near |= N;
        acc.far |= D;
    }
    return D;
}

// A warp per vertex of degree <= MP_T1 (the graph's class lists 0 and 1,
// stored back to back).
__global__ void __launch_bounds__(SRV_THREADS, MP_CTAS) k_mp_pull(MpArgs a, const uint32_t* __restrict__ list,
                                                                   uint64_t n)
{
    __shared__ uint32_t s_fmin[MP_K];
    mp_fmin_init(s_fmin);
    MpAcc acc;
    const int lane = threadIdx.x & 31;
    const uint32_t thr0 = __ldg(&a.thr[lane]), thr1 = __ldg(&a.thr[lane + 32]);
    const bool w0 = (a.wmask >> lane) & 1ULL, w1 = (a.wmask >> (lane + 32)) & 1ULL;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint32_t u = list[i];
        uint32_t b0 = SRV_INF, b1 = SRV_INF;
        mp_pull_edges(a, a.row[u], a.row[u + 1], thr0, thr1, w0, w1, b0, b1, acc);
        const unsigned long long fu = ((a.fcur[u >> 5] >> (u & 31)) & 1u) ? a.front[u] : 0ULL;
        if (!fu && !__any_sync(FULL, (b0 & b1) != SRV_INF)) continue;
        const uint32_t du0 = a.dist[(uint64_t)u * MP_K + lane], du1 = a.dist[(uint64_t)u * MP_K + 32 + lane];
        const unsigned long long D = fu ? mp_pull_own(fu, du0, du1, thr0, thr1, acc, s_fmin) : 0ULL;
        const bool i0 = b0 < du0, i1 = b1 < du1;
        if (i0) a.dist[(uint64_t)u * MP_K + lane] = b0;
        if (i1) a.dist[(uint64_t)u * MP_K + 32 + lane] = b1;
        const unsigned long long I = (unsigned long long)__ballot_sync(FULL, i0) |
                                     ((unsigned long long)__ballot_sync(FULL, i1) << 32);
        if (lane == 0 && (I | D)) {
            acc.any |= I;
            a.next[u] = I | D;  // u's only writer in a pull superstep
            atomicOr(&a.fbm[u >> 5], 1u << (u & 31));
        }
    }
    __syncthreads();
    mp_block_flush(acc, a, s_fmin);
}

// A warp per HUB_CHUNK in-edges of a hub (degree > MP_T1): candidates lower
// dist[u] by atomicMin (several chunks per hub); the hub's first chunk
// classifies its own frontier lanes.
__global__ void __launch_bounds__(SRV_THREADS, MP_CTAS) k_mp_pull_hubs(MpArgs a, const uint32_t* __restrict__ list,
                                                                        uint32_t n, const uint32_t* __restrict__ prefix)
{
    __shared__ uint32_t s_fmin[MP_K];
    mp_fmin_init(s_fmin);
    MpAcc acc;
    const int lane = threadIdx.x & 31;
    const uint32_t thr0 = __ldg(&a.thr[lane]), thr1 = __ldg(&a.thr[lane + 32]);
    const bool w0 = (a.wmask >> lane) & 1ULL, w1 = (a.wmask >> (lane + 32)) & 1ULL;
    if (n) {
        const uint32_t chunks = prefix[n];
        const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
        for (uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; c < chunks; c += warps) {
            const uint32_t i = hub_of_chunk(prefix, n, (uint32_t)c);
            const uint32_t u = list[i];
            const uint64_t e0 = a.row[u] + (uint64_t)((uint32_t)c - prefix[i]) * HUB_CHUNK;
            const uint64_t end = a.row[u + 1];
            uint32_t b0 = SRV_INF, b1 = SRV_INF;
            mp_pull_edges(a, e0, e0 + HUB_CHUNK < end ? e0 + HUB_CHUNK : end, thr0, thr1, w0, w1, b0, b1, acc);
            unsigned long long D = 0;
            if ((uint32_t)c == prefix[i]) {
                const unsigned long long fu = ((a.fcur[u >> 5] >> (u & 31)) & 1u) ? a.front[u] : 0ULL;
                if (fu)
                    D = mp_pull_own(fu, a.dist[(uint64_t)u * MP_K + lane], a.dist[(uint64_t)u * MP_K + 32 + lane], thr0,
                                    thr1, acc, s_fmin);
            }
            const bool i0 = b0 != SRV_INF && b0 < atomicMin(&a.dist[(uint64_t)u * MP_K + lane], b0);
            const bool i1 = b1 != SRV_INF && b1 < atomicMin(&a.dist[(uint64_t)u * MP_K + 32 + lane], b1);
            const unsigned long long I = (unsigned long long)__ballot_sync(FULL, i0) |
                                         ((unsigned long long)__ballot_sync(FULL, i1) << 32);
            if (lane == 0 && (I | D)) {
                acc.any |= I;
                atomicOr((unsigned long long*)&a.next[u], I | D);
                atomicOr(&a.fbm[u >> 5], 1u << (u & 31));
            }
        }
    }
    __syncthreads();
    mp_block_flush(acc, a, s_fmin);
}

// After a superstep: the consumed frontier masks back to zero.
__global__ void k_mp_clear(uint64_t* __restrict__ front, const uint32_t* __restrict__ l0, const uint32_t* __restrict__ l1,
                           const uint32_t* __restrict__ l2, const uint32_t* __restrict__ cnt)
{
    const uint64_t n0 = cnt[0], n1 = cnt[1], n2 = cnt[2];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n0 + n1 + n2;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = i < n0 ? l0[i] : (i < n0 + n1 ? l1[i - n0] : l2[i - n0 - n1]);
        front[v] = 0ULL;
    }
}

// Lane k of every vertex to the vertex id, every vertex in lane k's frontier
// (CC by label propagation); with cc = 0, lane k to INF.
__global__ void k_mp_init_lane(uint32_t* __restrict__ dist, uint64_t* __restrict__ front, uint64_t V, int k, int cc)
{
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        dist[v * MP_K + k] = cc ? (uint32_t)v : SRV_INF;
        if (cc) front[v] |= 1ULL << k;
    }
}

// SSSP source s of lane k: distance 0 and into the current frontier lists.
__global__ void k_mp_admit_source(uint32_t* __restrict__ dist, uint64_t* __restrict__ front, uint32_t* __restrict__ fcur,
                                  const uint64_t* __restrict__ row, uint64_t s, int k, uint32_t* __restrict__ l0,
                                  uint32_t* __restrict__ l1, uint32_t* __restrict__ l2, uint32_t* __restrict__ cnt)
{
    dist[s * MP_K + k] = 0u;
    const unsigned long long old = front[s];
    front[s] = old | (1ULL << k);
    fcur[s >> 5] |= 1u << (s & 31);
    if (!old) {
        const uint64_t d = row[s + 1] - row[s];
        const int cls = d <= MP_T0 ? 0 : (d <= MP_T1 ? 1 : 2);
        const uint32_t at = cnt[cls]++;
        (cls == 0 ? l0 : cls == 1 ? l1 : l2)[at] = (uint32_t)s;
    }
}

// Every vertex with a nonzero frontier mask into the frontier bitmap.
__global__ void k_mp_mark_all(const uint64_t* __restrict__ front, uint64_t V, uint32_t* __restrict__ fbm)
{
    const uint64_t W = (V + 31) >> 5;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < W; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t bits = 0;
        for (int j = 0; j < 32; j++) {
            const uint64_t v = w * 32 + j;
            if (v < V && front[v]) bits |= 1u << j;
        }
        fbm[w] |= bits;
    }
}

// Lane k's values out, and the lane back to INF for its next query (so an
// SSSP admission writes only its source).
__global__ void k_mp_extract(uint32_t* __restrict__ dist, uint64_t V, int k, uint32_t* __restrict__ out)
{
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        out[v] = dist[v * MP_K + k];
        dist[v * MP_K + k] = SRV_INF;
    }
}

// ---------------------------------------------------------------------------
// Connected components of a symmetric graph by union-find
// ---------------------------------------------------------------------------
// On a symmetric graph min-label propagation (benchmarks/cc.c) ends with every
// vertex labelled by the least id of its component.  Union-find reaches the
// same labels in one pass over the edges: a root is only ever hooked under a
// smaller root (so parents point to smaller ids and the root of a component
// is its least id), then every vertex is pointed at its root.  Parents are
// read through L2 (__ldcg); a stale parent is still an ancestor, and a failed
// compare-and-swap returns the current parent.
constexpr uint32_t CC_RETRIES = 1u << 24;  // hook attempts before an error

__device__ __forceinline__ uint32_t cc_find(uint32_t* p, uint32_t v)
{
    uint32_t x = __ldcg(&p[v]);
    while (x != v) {
        const uint32_t y = __ldcg(&p[x]);
        if (y != x) p[v] = y;  // path halving: y is an ancestor of v too
        v = x;
        x = y;
    }
    return v;
}

__device__ __forceinline__ void cc_hook(uint32_t* p, uint32_t a, uint32_t b, uint32_t* err)
{
    uint32_t ra = cc_find(p, a), rb = cc_find(p, b);
    for (uint32_t tries = 0; ra != rb; tries++) {
        if (tries == CC_RETRIES) {
            atomicOr(err, 1u);
            return;
        }
        if (ra > rb) {
            const uint32_t t = ra;
            ra = rb;
            rb = t;
        }
        const uint32_t old = atomicCAS(&p[rb], rb, ra);
        if (old == rb) return;
        rb = cc_find(p, old);
        ra = cc_find(p, ra);
    }
}

__global__ void k_cc_init(uint32_t* __restrict__ p, uint64_t V, uint32_t* __restrict__ err)
{
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        p[v] = (uint32_t)v;
    if (blockIdx.x == 0 && threadIdx.x == 0) *err = 0;
}

// The union-find pass runs in three steps (the sampling idea of Sutton et
// al., "Optimizing Parallel Graph Connectivity Computation via Subgraph
// Sampling", 2018): hook every vertex to its first CC_SAMPLE neighbours,
// find the component most sampled vertices ended in (on R-MAT graphs the
// giant one), then hook the remaining edges of the vertices outside it only.
// An edge between two vertices of that component needs no hook, and an edge
// with one end outside is hooked from that end, so the components (and their
// least-id roots) are those of a full pass.
constexpr uint32_t CC_SAMPLE = 2;
constexpr uint32_t CC_PROBES = 1024;

__global__ void k_cc_sample(const uint64_t* __restrict__ row, const uint32_t* __restrict__ adj, uint64_t V, uint32_t* p,
                            uint32_t* err)
{
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e1 = row[v + 1];
        for (uint64_t e = row[v]; e < e1 && e < row[v] + CC_SAMPLE; e++) cc_hook(p, (uint32_t)v, adj[e], err);
    }
}

// *giant = the root shared by most of CC_PROBES spread vertices (ties: the
// smaller root).  One CTA of CC_PROBES threads; V > 0.
__global__ void __launch_bounds__(CC_PROBES) k_cc_giant(uint32_t* p, uint64_t V, uint32_t* __restrict__ giant)
{
    __shared__ uint32_t r[CC_PROBES];
    __shared__ unsigned long long best;
    const uint32_t t = threadIdx.x;
    if (t == 0) best = 0;
    r[t] = cc_find(p, (uint32_t)(((uint64_t)t * 2654435761ULL) % V));
    __syncthreads();
    uint32_t c = 0;
    for (uint32_t j = 0; j < CC_PROBES; j++) c += r[j] == r[t];
    atomicMax(&best, ((unsigned long long)c << 32) | (0xffffffffu - r[t]));
    __syncthreads();
    if (t == 0) *giant = 0xffffffffu - (uint32_t)best;
}

// The edges from index `skip` of each listed vertex: all of them when `giant`
// is given (vertices in that component are skipped), else the edges to smaller
// ids only (each undirected edge once).  A thread per vertex of class 0, a
// warp per vertex of class 1, a warp per HUB_CHUNK edges of a hub.
__device__ __forceinline__ bool cc_wanted(uint32_t v, uint32_t u, bool all) { return all || u < v; }

__global__ void k_cc_hook_thread(const uint64_t* __restrict__ row, const uint32_t* __restrict__ adj,
                                 const uint32_t* __restrict__ list, uint64_t n, uint32_t* p, uint32_t* err,
                                 const uint32_t* __restrict__ giant, uint32_t skip)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = list[i];
        if (giant && cc_find(p, v) == *giant) continue;
        for (uint64_t e = row[v] + skip; e < row[v + 1]; e++) {
            const uint32_t u = adj[e];
            if (cc_wanted(v, u, giant != nullptr)) cc_hook(p, v, u, err);
        }
    }
}

__global__ void k_cc_hook_warp(const uint64_t* __restrict__ row, const uint32_t* __restrict__ adj,
                               const uint32_t* __restrict__ list, uint64_t n, uint32_t* p, uint32_t* err,
                               const uint32_t* __restrict__ giant, uint32_t skip)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint32_t v = list[i];
        if (giant) {
            const uint32_t root = __shfl_sync(FULL, lane == 0 ? cc_find(p, v) : 0u, 0);
            if (root == *giant) continue;
        }
        for (uint64_t e = row[v] + skip + lane; e < row[v + 1]; e += 32) {
            const uint32_t u = adj[e];
            if (cc_wanted(v, u, giant != nullptr)) cc_hook(p, v, u, err);
        }
    }
}

__global__ void k_cc_hook_hub(const uint64_t* __restrict__ row, const uint32_t* __restrict__ adj,
                              const uint32_t* __restrict__ list, uint32_t n, const uint32_t* __restrict__ prefix,
                              uint32_t* p, uint32_t* err, const uint32_t* __restrict__ giant, uint32_t skip)
{
    if (!n) return;
    const int lane = threadIdx.x & 31;
    const uint32_t chunks = prefix[n];
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; c < chunks; c += warps) {
        const uint32_t i = hub_of_chunk(prefix, n, (uint32_t)c);
        const uint32_t v = list[i];
        if (giant) {
            const uint32_t root = __shfl_sync(FULL, lane == 0 ? cc_find(p, v) : 0u, 0);
            if (root == *giant) continue;
        }
        const uint64_t first = row[v] + skip;
        uint64_t e0 = row[v] + (uint64_t)((uint32_t)c - prefix[i]) * HUB_CHUNK;
        const uint64_t e1 = e0 + HUB_CHUNK < row[v + 1] ? e0 + HUB_CHUNK : row[v + 1];
        if (e0 < first) e0 = first;
        for (uint64_t e = e0 + lane; e < e1; e += 32) {
            const uint32_t u = adj[e];
            if (cc_wanted(v, u, giant != nullptr)) cc_hook(p, v, u, err);
        }
    }
}

__global__ void k_cc_compress(uint32_t* p, uint64_t V)
{
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        p[v] = cc_find(p, (uint32_t)v);
}

// ---------------------------------------------------------------------------
// PPR lanes
// ---------------------------------------------------------------------------
struct PpLanes {
    float* out[PP_K];       // result buffer of a lane in its last gather, else null
    uint32_t seed[PP_K];
    unsigned long long active;  // lanes gathering this superstep
};

struct PpArgs {
    const uint64_t* __restrict__ row;
    const uint32_t* __restrict__ adj;
    const float* __restrict__ b_cur;
    float* __restrict__ b_next;
    float2* __restrict__ partial;  // (sum, compensation) per hub chunk and lane
};

// Compensated summation; the value of a pair is s + c.  Per term, Kahan's
// algorithm (4 operations: the gathers issue one per lane and edge, and the
// ncu profile of the PPR kernels shows them issue-bound, not memory-bound);
// pairs of partial sums merge with Knuth's TwoSum, which is exact whatever
// their magnitudes.
__device__ __forceinline__ void pp_add(float& s, float& c, float x)
{
    const float y = __fadd_rn(x, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(y, __fsub_rn(t, s));
    s = t;
}

__device__ __forceinline__ void pp_merge(float& s, float& c, float s2, float c2)
{
    const float t = __fadd_rn(s, s2);
    const float bp = __fsub_rn(t, s);
    const float err = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(s2, bp));
    c = __fadd_rn(__fadd_rn(c, c2), err);
    s = t;
}

// x of lane k at v from its gathered sum (ppr application: 0.15 at the seed).
__device__ __forceinline__ float pp_value(const PpLanes& L, int k, uint64_t v, float sum)
{
    return __fadd_rn(L.seed[k] == (uint32_t)v ? 0.15f : 0.0f, __fmul_rn(0.85f, sum));
}

// Sum of up to four float4 terms, pairwise: (x0 + x1) + (x2 + x3), absent
// terms 0.  All terms are non-negative quotients, so the group's rounding
// error is at most 2 ulp of the group sum; the group then enters the
// compensated sum as one term.  This cuts the compensated additions per
// gathered row by four.
__device__ __forceinline__ float4 pp_sum4(float4 x0, float4 x1, float4 x2, float4 x3)
{
    return make_float4(__fadd_rn(__fadd_rn(x0.x, x1.x), __fadd_rn(x2.x, x3.x)),
                       __fadd_rn(__fadd_rn(x0.y, x1.y), __fadd_rn(x2.y, x3.y)),
                       __fadd_rn(__fadd_rn(x0.z, x1.z), __fadd_rn(x2.z, x3.z)),
                       __fadd_rn(__fadd_rn(x0.w, x1.w), __fadd_rn(x2.w, x3.w)));
}

__device__ __forceinline__ void pp_add4(float* s, float* c, float4 t)
{
    pp_add(s[0], c[0], t.x);
    pp_add(s[1], c[1], t.y);
    pp_add(s[2], c[2], t.z);
    pp_add(s[3], c[3], t.w);
}

// Quad q (lanes 4q..4q+3) of u's row: one 16-byte load.
__device__ __forceinline__ float4 pp_row(const PpArgs& a, uint32_t u, int q)
{
    return reinterpret_cast<const float4*>(a.b_cur + (uint64_t)u * PP_K)[q];
}

// Threads q < PP_Q of a group finish lanes 4q..4q+3 of vertex v from their
// compensated sums: x to the result buffer of a lane in its last gather,
// else the quotient x / deg into the next row.
__device__ __forceinline__ void pp_finish_quad(const PpArgs& a, const PpLanes& L, uint64_t v, uint64_t deg, int q,
                                               const float* s, const float* c)
{
    float bn[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int k = 4 * q + j;
        bn[j] = 0.0f;
        if ((L.active >> k) & 1ULL) {
            const float xn = pp_value(L, k, v, __fadd_rn(s[j], c[j]));
            if (L.out[k]) L.out[k][v] = xn;
            else if (deg) bn[j] = __fdiv_rn(xn, (float)deg);
        }
    }
    // a vertex without edges has quotient 0 in every lane, and both buffers
    // start zeroed: its row is never written (a third of R-MAT's vertices)
    if (deg) reinterpret_cast<float4*>(a.b_next + v * PP_K)[q] = make_float4(bn[0], bn[1], bn[2], bn[3]);
}

// A warp gathers [e0, e1): thread t takes lane quad t % PP_Q and edge slot
// t / PP_Q (PP_SLOTS slots), reading the neighbour's quad as one float4, so
// each load instruction reads PP_SLOTS whole rows.  Every 4 rows of a thread
// are summed pairwise and added compensated; the next 32 ids are loaded while
// the current rows are in flight.  Then the slots of each quad merge (TwoSum),
// and threads 0..PP_Q-1 hold the totals of their quads.  The order of a
// lane's terms depends on the edge list only, not on which lanes are active.
__device__ __forceinline__ void pp_gather_warp(const PpArgs& a, uint64_t e0, uint64_t e1, bool quad_on, float* s,
                                               float* c)
{
    const int lane = threadIdx.x & 31, slot = lane / PP_Q, q = lane % PP_Q;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 4; i++) s[i] = c[i] = 0.0f;
    uint32_t uj = (e0 + lane < e1) ? ld_edge(&a.adj[e0 + lane]) : 0u;
    for (uint64_t e = e0; e < e1; e += 32) {
        const uint32_t un = (e + 32 + lane < e1) ? ld_edge(&a.adj[e + 32 + lane]) : 0u;
        const int nj = (int)((e1 - e) < 32 ? (e1 - e) : 32);
#pragma unroll
        for (int h = 0; h < 32 / PP_SLOTS; h += 4) {
            float4 x[4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int jj = (h + r) * PP_SLOTS + slot;
                const uint32_t u = __shfl_sync(FULL, uj, jj);
                x[r] = (quad_on && jj < nj) ? pp_row(a, u, q) : z;
            }
            if (quad_on) pp_add4(s, c, pp_sum4(x[0], x[1], x[2], x[3]));
        }
        uj = un;
    }
#pragma unroll
    for (int off = PP_Q; off < 32; off <<= 1)
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const float s2 = __shfl_xor_sync(FULL, s[i], off), c2 = __shfl_xor_sync(FULL, c[i], off);
            pp_merge(s[i], c[i], s2, c2);
        }
}

// PP_Q threads per low-degree vertex (degree <= PP_T0): thread q of the group
// takes lane quad q of every in-neighbour's row, so a warp reads 32 / PP_Q
// whole rows per load instruction and no partial sums need merging.  Four
// threads of the group load four consecutive ids at a time and the group
// shares them by shuffle; the four rows are summed pairwise and added
// compensated, in edge order.
__global__ void __launch_bounds__(SRV_THREADS, 4) k_pp_rows(PpArgs a, PpLanes L, const uint32_t* __restrict__ list,
                                                         uint64_t n)
{
    const int lane = threadIdx.x & 31, q = lane % PP_Q, gb = lane - q;
    const unsigned gmask = ((1u << PP_Q) - 1u) << gb;
    const bool quad_on = (L.active >> (4 * q)) & 0xFULL;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint64_t groups = ((uint64_t)gridDim.x * blockDim.x) / PP_Q;
    // The next vertex's list entry, row bounds and first four ids are loaded
    // while this vertex's rows are gathered, and the next four ids of a row
    // while its current four rows are: the chain list -> offsets -> ids ->
    // rows leaves the critical path except for its last link.  The threads
    // of a group share i, so they leave the loop together.
    uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / PP_Q;
    uint64_t v = 0, e0 = 0, e1 = 0;
    uint32_t u0 = 0;
    if (i < n) {
        v = list[i];
        e0 = a.row[v];
        e1 = a.row[v + 1];
        u0 = (q < 4 && e0 + q < e1) ? a.adj[e0 + q] : 0u;
    }
    for (; i < n; i += groups) {
        const uint64_t in = i + groups;
        uint64_t vn = 0, e0n = 0, e1n = 0;
        uint32_t u0n = 0;
        if (in < n) {
            vn = list[in];
            e0n = a.row[vn];
            e1n = a.row[vn + 1];
            u0n = (q < 4 && e0n + q < e1n) ? a.adj[e0n + q] : 0u;
        }
        float s[4], c[4];
#pragma unroll
        for (int k = 0; k < 4; k++) s[k] = c[k] = 0.0f;
        uint32_t uj = u0;
        for (uint64_t e = e0; e < e1; e += 4) {
            const uint32_t un = (q < 4 && e + 4 + q < e1) ? a.adj[e + 4 + q] : 0u;
            const int ne = (int)((e1 - e) < 4 ? (e1 - e) : 4);
            float4 x[4];
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const uint32_t u = __shfl_sync(gmask, uj, gb + r);
                x[r] = (quad_on && r < ne) ? pp_row(a, u, q) : z;
            }
            if (quad_on) pp_add4(s, c, pp_sum4(x[0], x[1], x[2], x[3]));
            uj = un;
        }
        pp_finish_quad(a, L, v, e1 - e0, q, s, c);
        v = vn;
        e0 = e0n;
        e1 = e1n;
        u0 = u0n;
    }
}

// A warp per vertex of higher degree (up to MP_T1).
__global__ void __launch_bounds__(SRV_THREADS) k_pp_vertices(PpArgs a, PpLanes L, const uint32_t* __restrict__ list,
                                                             uint64_t n)
{
    const int lane = threadIdx.x & 31;
    const bool quad_on = (L.active >> (4 * (lane % PP_Q))) & 0xFULL;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint64_t v = list[i];
        const uint64_t e0 = a.row[v], e1 = a.row[v + 1];
        float s[4], c[4];
        pp_gather_warp(a, e0, e1, quad_on, s, c);
        if (lane < PP_Q) pp_finish_quad(a, L, v, e1 - e0, lane, s, c);
    }
}

// Hubs: a warp per HUB_CHUNK edges, partial sums per chunk and lane...
__global__ void __launch_bounds__(SRV_THREADS) k_pp_hub_chunks(PpArgs a, PpLanes L, const uint32_t* __restrict__ list,
                                                               uint32_t n, const uint32_t* __restrict__ prefix)
{
    if (!n) return;
    const int lane = threadIdx.x & 31;
    const bool quad_on = (L.active >> (4 * (lane % PP_Q))) & 0xFULL;
    const uint32_t chunks = prefix[n];
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; c < chunks; c += warps) {
        const uint32_t i = hub_of_chunk(prefix, n, (uint32_t)c);
        const uint64_t v = list[i];
        const uint64_t e0 = a.row[v] + (uint64_t)((uint32_t)c - prefix[i]) * HUB_CHUNK;
        const uint64_t end = a.row[v + 1];
        float s[4], cc[4];
        pp_gather_warp(a, e0, e0 + HUB_CHUNK < end ? e0 + HUB_CHUNK : end, quad_on, s, cc);
        if (lane < PP_Q)
#pragma unroll
            for (int j = 0; j < 4; j++) a.partial[c * PP_K + 4 * lane + j] = make_float2(s[j], cc[j]);
    }
}

// ...then a warp per hub merges its chunks' partials in chunk order (a
// thread per lane) and threads 0..PP_Q-1 finish the hub's quads.
__global__ void __launch_bounds__(SRV_THREADS) k_pp_hub_finish(PpArgs a, PpLanes L, const uint32_t* __restrict__ list,
                                                               uint32_t n, const uint32_t* __restrict__ prefix)
{
    __shared__ float2 sh[SRV_THREADS / 32][PP_K];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint64_t v = list[i];
        for (int k = lane; k < PP_K; k += 32) {
            float s = 0.0f, c = 0.0f;
            for (uint32_t ch = prefix[i]; ch < prefix[i + 1]; ch++) {
                const float2 p = a.partial[(uint64_t)ch * PP_K + k];
                pp_merge(s, c, p.x, p.y);
            }
            sh[w][k] = make_float2(s, c);
        }
        __syncwarp();
        if (lane < PP_Q) {
            float s4[4], c4[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                s4[j] = sh[w][4 * lane + j].x;
                c4[j] = sh[w][4 * lane + j].y;
            }
            pp_finish_quad(a, L, v, a.row[v + 1] - a.row[v], lane, s4, c4);
        }
        __syncwarp();
    }
}

// Seed s of lane k: the broadcast of superstep 0, x = 1 at the seed.
__global__ void k_pp_admit(float* __restrict__ b, const uint64_t* __restrict__ row, uint64_t s, int k)
{
    const uint64_t d = row[s + 1] - row[s];
    b[s * PP_K + k] = d ? __fdiv_rn(1.0f, (float)d) : 0.0f;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Query {
    uint64_t id = 0;
    int gid = 0, kind = 0;
    uint64_t src = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int state = 0;  // IPG_QUERY_*
    void* result = nullptr;
    uint64_t result_bytes = 0;
    cudaEvent_t ready = nullptr;  // result complete on the device
};

struct Group;

struct Graph {
    int gid = 0;
    ipg_graph* g = nullptr;
    ipg_graph_view gv{};
    Group* mp = nullptr;
    Group* pp = nullptr;
    // degree classes over all vertices and the chunk prefix of their hubs,
    // built at first use by the PPR gathers and the union-find pass
    ipg_bins bins{};
    uint32_t* hub_prefix = nullptr;  // nh + 1 entries, then the hub count and the union-find error word
    uint64_t hub_chunks = 0;
    uint32_t* cc_err = nullptr;
    uint32_t* cc_giant = nullptr;
    bool classes = false;
};

struct Group {
    int kind = 0;  // 0 min-plus, 1 PPR
    Graph* G = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;   // end of the superstep in flight
    cudaEvent_t ev0 = nullptr;  // its start
    bool running = false;
    uint64_t busy = 0;
    std::vector<std::vector<uint64_t>> lane_q;  // queries on each lane
    double last_used = 0;
    std::vector<std::pair<void*, uint64_t>> allocs;
    uint64_t bytes = 0;
    // min-plus
    uint32_t* dist = nullptr;
    uint64_t* front[2] = {nullptr, nullptr};
    int cur = 0;
    uint32_t* fbm[2] = {nullptr, nullptr};  // frontier bitmaps: [cur] this superstep's, [cur ^ 1] the next
    uint32_t* list[3] = {nullptr, nullptr, nullptr};
    uint64_t hesum = 0;                   // frontier edges of the next superstep (last status)
    uint32_t* cnt = nullptr;              // into stat_d
    uint32_t* prefix = nullptr;
    uint32_t* thr_d = nullptr;            // lane thresholds of the next superstep
    uint32_t* thr_pin = nullptr;          // their pinned staging copy
    uint32_t thr_h[MP_K];
    MpStatus* stat_d = nullptr;
    MpStatus* stat_h = nullptr;           // pinned copy after each superstep
    uint32_t hn[3] = {0, 0, 0};           // list sizes the host knows of
    uint32_t hchunks = 0;                 // hub chunks of list 2
    uint32_t appended = 0;                // sources appended since
    uint64_t wmask = 0;
    int cc_lane = -1;  // label-propagation CC lane admitted in this admission pass
    // PPR
    float* b[2] = {nullptr, nullptr};
    float2* partial = nullptr;
    // gather classes: quads for degree <= PP_T0, warps up to MP_T1 (hubs
    // above, from the graph's classes); null when the graph is too large for
    // ipg_degree_classes_noalloc, and then the graph's classes serve
    uint32_t* pp_list = nullptr;
    uint64_t* pp_tot = nullptr;
    uint64_t pp_n[2] = {0, 0};
    int it[PP_K] = {0};
    uint32_t seed[PP_K] = {0};
    uint64_t supersteps = 0;
};

template <class T>
int galloc(Group* G, T** p, uint64_t n)
{
    void* d = nullptr;
    const uint64_t bytes = (n ? n : 1) * sizeof(T);
    int r = ipg_dev_alloc(&d, bytes);
    if (r != IPG_OK) return r;
    G->allocs.push_back({d, bytes});
    G->bytes += bytes;
    *p = (T*)d;
    return IPG_OK;
}

}  // namespace

struct ipg_server {
    uint64_t budget = 0;
    uint64_t in_use = 0;
    // result buffers come from a stream-ordered pool that keeps freed memory
    // (release threshold unbounded): a query's result is allocated at
    // admission and freed at release without a cudaMalloc / cudaFree, each of
    // which costs about a millisecond and stalls the scheduling loop
    cudaMemPool_t rpool = nullptr;
    cudaStream_t rel_st = nullptr;  // stream of the frees (results released are complete)
    uint32_t rounds = 20;
    std::vector<std::unique_ptr<Graph>> graphs;
    std::vector<Group*> groups;
    std::map<uint64_t, Query> queries;
    std::vector<std::deque<uint64_t>> pending;  // per graph and group kind: gid * 2 + kind
    uint64_t n_pending = 0;
    std::vector<uint64_t> finishing;            // results being completed on the device
    std::vector<uint64_t> completed;            // done since the last drain
    std::vector<double> busy_s;                 // per graph and group kind: superstep device time
    std::vector<uint64_t> steps, lanes;         // supersteps, lanes admitted
    std::vector<uint64_t> work;                 // min-plus lane-edge relaxations examined
    uint64_t next_id = 1;
    // near-far bucket width of SSSP lanes (IPG_SERVE_DELTA); on R-MAT graphs
    // with weights in [1, 255], 256..1024 measured best, 7 % faster than none
    uint32_t delta = 1024;
    // dense min-plus supersteps on symmetric graphs pull (IPG_SERVE_PULL=0: never)
    bool pull = true;
    std::mutex mu;
    ipg_server_stats stats{};
};

namespace {

void free_group(ipg_server* S, Group* G)
{
    if (G->st) cudaStreamSynchronize(G->st);
    for (auto& a : G->allocs) ipg_dev_free(a.first, a.second);
    if (G->stat_h) cudaFreeHost(G->stat_h);
    if (G->thr_pin) cudaFreeHost(G->thr_pin);
    if (G->ev) cudaEventDestroy(G->ev);
    if (G->ev0) cudaEventDestroy(G->ev0);
    if (G->st) cudaStreamDestroy(G->st);
    S->in_use -= G->bytes;
    if (G->G->mp == G) G->G->mp = nullptr;
    if (G->G->pp == G) G->G->pp = nullptr;
    S->groups.erase(std::find(S->groups.begin(), S->groups.end(), G));
    S->stats.groups_freed++;
    delete G;
}

uint64_t group_bytes(const Graph* G, int kind)
{
    const uint64_t V = G->gv.V, E = G->gv.E;
    if (kind == 0) return V * (MP_K * 4 + 16 + 12) + V / 4 + (E / (MP_T1 + 1) + 2) * 4 + 4096;
    return V * (PP_K * 4 * 2 + 4) + (E / HUB_CHUNK + V / MP_T1 + 2) * (PP_K * 8) + 4096;
}

// Frees idle groups (least recently used first) until `need` more bytes fit
// the budget.
bool make_room(ipg_server* S, uint64_t need)
{
    if (!S->budget) return true;
    while (S->in_use + need > S->budget) {
        Group* victim = nullptr;
        for (Group* G : S->groups)
            if (!G->busy && !G->running && (!victim || G->last_used < victim->last_used)) victim = G;
        if (victim) {
            free_group(S, victim);
            continue;
        }
        return false;
    }
    return true;
}

// Degree classes of all vertices of a graph and the chunk prefix of its hubs
// (built once; the PPR gathers and the union-find pass use them).
int graph_classes(Graph* Gr, cudaStream_t st)
{
    if (Gr->classes) return IPG_OK;
    int r = ipg_graph_bins(Gr->g, 0, MP_T0, MP_T1, &Gr->bins);
    if (r != IPG_OK) return r;
    const uint64_t nh = Gr->bins.count[2];
    void* p = nullptr;
    if ((r = ipg_dev_alloc(&p, (nh + 5) * 4)) != IPG_OK) return r;
    Gr->hub_prefix = (uint32_t*)p;
    uint32_t* count = Gr->hub_prefix + nh + 2;
    Gr->cc_err = count + 1;
    Gr->cc_giant = count + 2;
    const uint32_t n2 = (uint32_t)nh;
    uint32_t chunks = 0;
    cudaMemcpyAsync(count, &n2, 4, cudaMemcpyHostToDevice, st);
    k_chunk_prefix<<<1, 1024, 0, st>>>(Gr->bins.d_list[2], count, Gr->gv.d_row, Gr->hub_prefix, nullptr);
    cudaMemcpyAsync(&chunks, Gr->hub_prefix + nh, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return ipg_internal_fail(IPG_ECUDA, "serve: hub prefix failed");
    Gr->hub_chunks = chunks;
    Gr->classes = true;
    return IPG_OK;
}

// Union-find CC of a symmetric graph into p (V labels).
void run_union_find(Graph* Gr, uint32_t* p, cudaStream_t st)
{
    const ipg_graph_view& gv = Gr->gv;
    const ipg_bins& B = Gr->bins;
    const uint32_t* adj = (const uint32_t*)gv.d_adj;
    k_cc_init<<<resident_cap(k_cc_init, thread_grid(gv.V)), SRV_THREADS, 0, st>>>(p, gv.V, Gr->cc_err);
    if (gv.V == 0) return;
    k_cc_sample<<<resident_cap(k_cc_sample, thread_grid(gv.V)), SRV_THREADS, 0, st>>>(gv.d_row, adj, gv.V, p,
                                                                                     Gr->cc_err);
    k_cc_compress<<<resident_cap(k_cc_compress, thread_grid(gv.V)), SRV_THREADS, 0, st>>>(p, gv.V);
    k_cc_giant<<<1, CC_PROBES, 0, st>>>(p, gv.V, Gr->cc_giant);
    if (B.count[0])
        k_cc_hook_thread<<<resident_cap(k_cc_hook_thread, thread_grid(B.count[0])), SRV_THREADS, 0, st>>>(
            gv.d_row, adj, B.d_list[0], B.count[0], p, Gr->cc_err, Gr->cc_giant, CC_SAMPLE);
    if (B.count[1])
        k_cc_hook_warp<<<resident_cap(k_cc_hook_warp, warp_grid(B.count[1])), SRV_THREADS, 0, st>>>(
            gv.d_row, adj, B.d_list[1], B.count[1], p, Gr->cc_err, Gr->cc_giant, CC_SAMPLE);
    if (B.count[2])
        k_cc_hook_hub<<<resident_cap(k_cc_hook_hub, warp_grid(Gr->hub_chunks)), SRV_THREADS, 0, st>>>(
            gv.d_row, adj, B.d_list[2], (uint32_t)B.count[2], Gr->hub_prefix, p, Gr->cc_err, Gr->cc_giant,
            CC_SAMPLE);
    k_cc_compress<<<resident_cap(k_cc_compress, thread_grid(gv.V)), SRV_THREADS, 0, st>>>(p, gv.V);
}

int create_group(ipg_server* S, Graph* Gr, int kind)
{
    const uint64_t need = group_bytes(Gr, kind);
    if (!make_room(S, need)) return IPG_EBUDGET;
    Group* G = new Group();
    G->kind = kind;
    G->G = Gr;
    G->lane_q.resize(kind == 0 ? MP_K : PP_K);
    const uint64_t V = Gr->gv.V, E = Gr->gv.E;
    int r = IPG_OK;
    // smaller graphs get higher-priority streams: their supersteps are short,
    // and their CTAs go first whenever SMs free up
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    int lg = 0;
    while ((1ULL << (lg + 1)) <= V) lg++;
    const int prio = std::min(least, greatest + std::max(0, lg - 18));
    cudaError_t e = cudaStreamCreateWithPriority(&G->st, cudaStreamNonBlocking, prio);
    if (e == cudaSuccess) e = cudaEventCreate(&G->ev);
    if (e == cudaSuccess) e = cudaEventCreate(&G->ev0);
    if (e != cudaSuccess) r = ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
    if (kind == 0) {
        if (r == IPG_OK) r = galloc(G, &G->dist, V * MP_K);
        if (r == IPG_OK) r = galloc(G, &G->front[0], V);
        if (r == IPG_OK) r = galloc(G, &G->front[1], V);
        if (r == IPG_OK) r = galloc(G, &G->fbm[0], (V + 31) / 32 + 1);
        if (r == IPG_OK) r = galloc(G, &G->fbm[1], (V + 31) / 32 + 1);
        for (int k = 0; k < 3 && r == IPG_OK; k++) r = galloc(G, &G->list[k], V);
        if (r == IPG_OK) r = galloc(G, &G->stat_d, 1);
        if (r == IPG_OK) G->cnt = G->stat_d->cnt;
        if (r == IPG_OK) r = galloc(G, &G->thr_d, MP_K);
        if (r == IPG_OK && cudaHostAlloc((void**)&G->thr_pin, MP_K * 4, cudaHostAllocDefault) != cudaSuccess)
            r = ipg_internal_fail(IPG_ENOMEM, "serve: pinned allocation failed");
        if (r == IPG_OK) r = galloc(G, &G->prefix, E / (MP_T1 + 1) + 2);
        if (r == IPG_OK && cudaHostAlloc((void**)&G->stat_h, sizeof(MpStatus), cudaHostAllocDefault) != cudaSuccess)
            r = ipg_internal_fail(IPG_ENOMEM, "serve: pinned allocation failed");
        if (r == IPG_OK) {
            cudaMemsetAsync(G->dist, 0xff, V * MP_K * 4, G->st);  // every lane INF
            cudaMemsetAsync(G->front[0], 0, V * 8, G->st);
            cudaMemsetAsync(G->front[1], 0, V * 8, G->st);
            cudaMemsetAsync(G->fbm[0], 0, ((V + 31) / 32 + 1) * 4, G->st);
            cudaMemsetAsync(G->fbm[1], 0, ((V + 31) / 32 + 1) * 4, G->st);
            cudaMemsetAsync(G->stat_d, 0, sizeof(MpStatus), G->st);
            cudaMemsetAsync(G->prefix, 0, 8, G->st);
        }
    } else {
        if (r == IPG_OK) r = graph_classes(Gr, G->st);
        if (r == IPG_OK) r = galloc(G, &G->b[0], V * PP_K);
        if (r == IPG_OK) r = galloc(G, &G->b[1], V * PP_K);
        if (r == IPG_OK) r = galloc(G, &G->partial, Gr->hub_chunks * PP_K);
        if (r == IPG_OK) {
            // quotients of idle lanes are 0: an admitted lane sets its seed only
            cudaMemsetAsync(G->b[0], 0, V * PP_K * 4, G->st);
            cudaMemsetAsync(G->b[1], 0, V * PP_K * 4, G->st);
        }
        if (r == IPG_OK && V <= PP_NOALLOC_MAX_V) {
            if (r == IPG_OK) r = galloc(G, &G->pp_list, V);
            if (r == IPG_OK) r = galloc(G, &G->pp_tot, 6);
            // the server's calls of ipg_degree_classes_noalloc are serialised
            // by this synchronisation (its scratch is shared)
            uint64_t tot[6] = {0, 0, 0, 0, 0, 0};
            if (r == IPG_OK) r = ipg_degree_classes_noalloc(V, Gr->gv.d_row, PP_T0, MP_T1, G->pp_list, G->pp_tot, G->st);
            if (r == IPG_OK && (cudaMemcpyAsync(tot, G->pp_tot, sizeof tot, cudaMemcpyDeviceToHost, G->st) != cudaSuccess ||
                                cudaStreamSynchronize(G->st) != cudaSuccess))
                r = ipg_internal_fail(IPG_ECUDA, "serve: PPR degree classes failed");
            if (r == IPG_OK && tot[2] != Gr->bins.count[2])
                r = ipg_internal_fail(IPG_EINVAL, "serve: PPR hub class differs from the graph's");
            G->pp_n[0] = tot[0];
            G->pp_n[1] = tot[1];
        }
    }
    if (r == IPG_OK && cudaGetLastError() != cudaSuccess) r = ipg_internal_fail(IPG_ECUDA, "serve: group setup failed");
    S->in_use += G->bytes;
    S->groups.push_back(G);
    if (r != IPG_OK) {
        free_group(S, G);
        return r;
    }
    (kind == 0 ? Gr->mp : Gr->pp) = G;
    G->last_used = now_s();
    S->stats.groups_created++;
    return IPG_OK;
}

// A query's result buffer is counted against the budget when the query is
// admitted (reserve_result) and allocated when it is first written
// (alloc_result): at admission for union-find CC and PPR, at extraction for
// min-plus lanes, whose distance column holds the result until then.
int reserve_result(ipg_server* S, Query& q, uint64_t bytes)
{
    if (!make_room(S, bytes)) return IPG_EBUDGET;
    S->in_use += bytes;
    q.result_bytes = bytes;
    return IPG_OK;
}

int alloc_result(ipg_server* S, Query& q, cudaStream_t st)
{
    if (q.result) return IPG_OK;
    if (cudaMallocFromPoolAsync(&q.result, q.result_bytes, S->rpool, st) != cudaSuccess) {
        cudaGetLastError();
        q.result = nullptr;
        return IPG_ENOMEM;  // the caller tries again later
    }
    return IPG_OK;
}

// st: a stream ordered after the allocation (the admitting group's stream,
// or any stream once the query is done)
void release_result(ipg_server* S, Query& q, cudaStream_t st = nullptr)
{
    if (q.result) cudaFreeAsync(q.result, st ? st : S->rel_st);
    S->in_use -= q.result_bytes;
    q.result_bytes = 0;
    q.result = nullptr;
}

void finishing(ipg_server* S, Query& q, cudaStream_t st)
{
    cudaEventCreateWithFlags(&q.ready, cudaEventDisableTiming);
    cudaEventRecord(q.ready, st);
    q.state = IPG_QUERY_FINISHING;
    S->finishing.push_back(q.id);
}

// Pending queries of group G's graph and kind take free lanes.
void admit(ipg_server* S, Group* G, double now)
{
    std::deque<uint64_t>& queue = S->pending[(size_t)G->G->gid * 2 + G->kind];
    const uint64_t V = G->G->gv.V;
    const int K = G->kind == 0 ? MP_K : PP_K;
    const uint64_t full = K == 64 ? ~0ULL : ((1ULL << K) - 1);
    G->cc_lane = -1;
    bool rebuild = false;
    void* cc_first = nullptr;  // result of this admission pass's union-find run
    for (auto it = queue.begin(); it != queue.end();) {
        Query& q = S->queries[*it];
        const bool union_find = q.kind == IPG_QUERY_CC && G->G->gv.symmetric;
        const bool joins_cc = q.kind == IPG_QUERY_CC && G->cc_lane >= 0;
        if (!union_find && !joins_cc && (G->busy & full) == full) break;  // no lane free
        const uint64_t rbytes = V * 4;
        // a union-find CC result is written now, so it is allocated at
        // admission; a PPR lane's is allocated before its last gather and a
        // min-plus lane's when the lane is extracted (its column holds it
        // until then), so running lanes hold no result memory
        if (reserve_result(S, q, rbytes) != IPG_OK) {
            ++it;
            continue;
        }
        if (union_find && alloc_result(S, q, G->st) != IPG_OK) {
            release_result(S, q, G->st);
            ++it;
            continue;
        }
        q.state = IPG_QUERY_RUNNING;
        q.t_start = now;
        if (union_find) {
            // CC queries admitted together share one union-find pass
            if (!cc_first) {
                if (graph_classes(G->G, G->st) != IPG_OK) {
                    release_result(S, q, G->st);
                    q.state = IPG_QUERY_PENDING;
                    ++it;
                    continue;
                }
                run_union_find(G->G, (uint32_t*)q.result, G->st);
                cc_first = q.result;
                S->stats.kernel_launches += 8;
            } else {
                cudaMemcpyAsync(q.result, cc_first, rbytes, cudaMemcpyDeviceToDevice, G->st);
            }
            finishing(S, q, G->st);
            it = queue.erase(it);
            S->n_pending--;
            continue;
        }
        int k;
        if (joins_cc) {
            k = G->cc_lane;
        } else {
            k = __builtin_ctzll(~G->busy);
            G->busy |= 1ULL << k;
            const uint32_t g = resident_cap(k_mp_init_lane, thread_grid(V));
            if (q.kind == IPG_QUERY_PPR) {
                k_pp_admit<<<1, 1, 0, G->st>>>(G->b[G->cur], G->G->gv.d_row, q.src, k);
                G->it[k] = 0;
                G->seed[k] = (uint32_t)q.src;
            } else if (q.kind == IPG_QUERY_CC) {
                k_mp_init_lane<<<g, SRV_THREADS, 0, G->st>>>(G->dist, G->front[G->cur], V, k, 1);
                G->wmask &= ~(1ULL << k);
                G->thr_h[k] = SRV_INF;  // labels are no distances: never deferred
                G->cc_lane = k;
                rebuild = true;
            } else {
                // the lane is INF everywhere (cleared when its last query was extracted)
                k_mp_admit_source<<<1, 1, 0, G->st>>>(G->dist, G->front[G->cur], G->fbm[G->cur], G->G->gv.d_row,
                                                       q.src, k, G->list[0], G->list[1], G->list[2], G->cnt);
                G->wmask |= 1ULL << k;
                G->thr_h[k] = S->delta;
                G->appended++;
            }
            S->stats.lanes_admitted++;
            S->lanes[(size_t)G->G->gid * 2 + G->kind]++;
        }
        G->lane_q[k].push_back(q.id);
        it = queue.erase(it);
        S->n_pending--;
    }
    if (rebuild) {
        // a label-propagation CC lane puts every vertex into the frontier:
        // rebuild the lists and read their sizes back (grids are sized by them)
        k_mp_mark_all<<<resident_cap(k_mp_mark_all, thread_grid((V + 31) / 32)), SRV_THREADS, 0, G->st>>>(
            G->front[G->cur], V, G->fbm[G->cur]);
        cudaMemsetAsync(G->cnt, 0, 12, G->st);
        cudaMemsetAsync(G->stat_d->esum, 0, sizeof G->stat_d->esum, G->st);
        ipg_compact(G->fbm[G->cur], V, G->G->gv.d_row, MP_T0, MP_T1, G->list[0], G->list[1], G->list[2], G->cnt,
                    (uint64_t*)G->stat_d->esum, 0, G->st);
        k_chunk_prefix<<<1, 1024, 0, G->st>>>(G->list[2], G->cnt + 2, G->G->gv.d_row, G->prefix, &G->stat_d->chunks);
        cudaMemcpyAsync(G->stat_h, G->stat_d, sizeof(MpStatus), cudaMemcpyDeviceToHost, G->st);
        cudaStreamSynchronize(G->st);
        for (int c = 0; c < 3; c++) G->hn[c] = G->stat_h->cnt[c];
        G->hchunks = G->stat_h->chunks;
        G->hesum = G->stat_h->esum[0] + G->stat_h->esum[1] + G->stat_h->esum[2];
        G->appended = 0;
    }
}

int launch_superstep(ipg_server* S, Group* G)
{
    const ipg_graph_view& gv = G->G->gv;
    cudaEventRecord(G->ev0, G->st);
    if (G->kind == 0) {
        MpArgs a;
        a.row = gv.d_row;
        a.adj = (const uint32_t*)gv.d_adj;
        a.wgt = (const uint32_t*)gv.d_wgt;
        a.dist = G->dist;
        a.front = G->front[G->cur];
        a.next = G->front[G->cur ^ 1];
        a.fbm = G->fbm[G->cur ^ 1];
        a.fcur = G->fbm[G->cur];
        a.thr = G->thr_d;
        a.st = G->stat_d;
        a.wmask = G->wmask;
        a.busy = G->busy;
        // grids from the list sizes of the last status plus the sources
        // appended since (each in some list; a hub one adds its chunks)
        const uint64_t add = G->appended;
        const uint64_t hub_chunks_max = (gv.max_out_degree + HUB_CHUNK - 1) / HUB_CHUNK;
        const uint64_t n0 = G->hn[0] + add, n1 = G->hn[1] + add;
        const uint64_t chunks = G->hchunks + add * hub_chunks_max;
        memcpy(G->thr_pin, G->thr_h, sizeof G->thr_h);  // the last copy finished with the last superstep
        cudaMemcpyAsync(G->thr_d, G->thr_pin, sizeof G->thr_h, cudaMemcpyHostToDevice, G->st);
        cudaMemsetAsync(G->stat_d, 0, 3 * sizeof(unsigned long long), G->st);
        cudaMemsetAsync(G->stat_d->far_min, 0xff, sizeof G->stat_d->far_min, G->st);
        cudaMemsetAsync(&G->stat_d->work, 0, sizeof G->stat_d->work, G->st);
        cudaMemsetAsync(G->stat_d->esum, 0, sizeof G->stat_d->esum, G->st);
        // direction: pull when the frontier's edges are a large part of the
        // graph and enough lanes are busy to share each row read
        const Graph* Gr = G->G;
        const bool pull = S->pull && gv.symmetric && Gr->classes && __builtin_popcountll(G->busy) >= MP_PULL_LANES &&
                          G->hesum * MP_PULL_DIV >= gv.E;
        if (pull) {
            const ipg_bins& B = Gr->bins;
            const uint64_t n01 = B.count[0] + B.count[1];
            if (n01)
                k_mp_pull<<<resident_cap(k_mp_pull, warp_grid(n01)), SRV_THREADS, 0, G->st>>>(a, B.d_list[0], n01);
            if (B.count[2])
                k_mp_pull_hubs<<<resident_cap(k_mp_pull_hubs, warp_grid(Gr->hub_chunks)), SRV_THREADS, 0, G->st>>>(
                    a, B.d_list[2], (uint32_t)B.count[2], Gr->hub_prefix);
            S->stats.kernel_launches += (n01 ? 1 : 0) + (B.count[2] ? 1 : 0);
        } else {
            if (add) k_chunk_prefix<<<1, 1024, 0, G->st>>>(G->list[2], G->cnt + 2, gv.d_row, G->prefix, nullptr);
            k_mp_thread<<<resident_cap(k_mp_thread, thread_grid(n0)), SRV_THREADS, 0, G->st>>>(a, G->list[0],
                                                                                            G->cnt + 0);
            k_mp_vertices<<<resident_cap(k_mp_vertices, warp_grid(n1)), SRV_THREADS, 0, G->st>>>(a, G->list[1],
                                                                                              G->cnt + 1);
            k_mp_hubs<<<resident_cap(k_mp_hubs, warp_grid(chunks)), SRV_THREADS, 0, G->st>>>(a, G->list[2],
                                                                                          G->cnt + 2, G->prefix);
            S->stats.kernel_launches += 3 + (add ? 1 : 0);
        }
        S->stats.pull_supersteps += pull ? 1 : 0;
        k_mp_clear<<<resident_cap(k_mp_clear, thread_grid(G->hn[0] + G->hn[1] + G->hn[2] + add)), SRV_THREADS, 0,
                     G->st>>>(G->front[G->cur], G->list[0], G->list[1], G->list[2], G->cnt);
        cudaMemsetAsync(G->cnt, 0, 12, G->st);
        // the next bitmap is kept (it is the next superstep's frontier bitmap);
        // this superstep's is cleared for reuse as the one after
        ipg_compact(G->fbm[G->cur ^ 1], gv.V, gv.d_row, MP_T0, MP_T1, G->list[0], G->list[1], G->list[2], G->cnt,
                    (uint64_t*)G->stat_d->esum, 0, G->st);
        cudaMemsetAsync(G->fbm[G->cur], 0, ((gv.V + 31) / 32 + 1) * 4, G->st);
        k_chunk_prefix<<<1, 1024, 0, G->st>>>(G->list[2], G->cnt + 2, gv.d_row, G->prefix, &G->stat_d->chunks);
        cudaMemcpyAsync(G->stat_h, G->stat_d, sizeof(MpStatus), cudaMemcpyDeviceToHost, G->st);
        G->cur ^= 1;
        S->stats.kernel_launches += 4;
    } else {
        const Graph* Gr = G->G;
        PpArgs a;
        a.row = gv.d_row;
        a.adj = (const uint32_t*)gv.d_adj;
        a.b_cur = G->b[G->cur];
        a.b_next = G->b[G->cur ^ 1];
        a.partial = G->partial;
        PpLanes L;
        L.active = G->busy;
        for (int k = 0; k < PP_K; k++) {
            L.seed[k] = G->seed[k];
            L.out[k] = nullptr;
            if (((G->busy >> k) & 1) && G->it[k] + 1 == (int)S->rounds) {
                // a lane's result buffer is allocated for its last gather; if
                // the memory is not there yet the superstep waits
                Query& q = S->queries[G->lane_q[k][0]];
                if (alloc_result(S, q, G->st) != IPG_OK) return IPG_ENOMEM;
                L.out[k] = (float*)q.result;
            }
        }
        const ipg_bins& B = Gr->bins;
        const uint32_t* l0 = G->pp_list ? G->pp_list : B.d_list[0];
        const uint64_t n0 = G->pp_list ? G->pp_n[0] : B.count[0];
        const uint32_t* l1 = G->pp_list ? G->pp_list + n0 : B.d_list[1];
        const uint64_t n1 = G->pp_list ? G->pp_n[1] : B.count[1];
        if (n0)
            k_pp_rows<<<resident_cap(k_pp_rows, thread_grid(n0 * PP_Q)), SRV_THREADS, 0, G->st>>>(a, L, l0, n0);
        if (n1)
            k_pp_vertices<<<resident_cap(k_pp_vertices, warp_grid(n1)), SRV_THREADS, 0, G->st>>>(a, L, l1, n1);
        if (B.count[2]) {
            k_pp_hub_chunks<<<resident_cap(k_pp_hub_chunks, warp_grid(Gr->hub_chunks)), SRV_THREADS, 0, G->st>>>(
                a, L, B.d_list[2], (uint32_t)B.count[2], Gr->hub_prefix);
            k_pp_hub_finish<<<resident_cap(k_pp_hub_finish, warp_grid(B.count[2])), SRV_THREADS, 0, G->st>>>(
                a, L, B.d_list[2], (uint32_t)B.count[2], Gr->hub_prefix);
        }
        G->cur ^= 1;
        S->stats.kernel_launches += 4;
    }
    cudaEventRecord(G->ev, G->st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
    G->running = true;
    G->supersteps++;
    S->stats.supersteps++;
    return IPG_OK;
}

// A completed superstep: retire finished lanes.
void retire(ipg_server* S, Group* G, double now)
{
    if (G->kind == 0) {
        const MpStatus& st = *G->stat_h;
        for (int c = 0; c < 3; c++) G->hn[c] = st.cnt[c];
        G->hchunks = st.chunks;
        S->work[(size_t)G->G->gid * 2] += st.work;
        G->hesum = st.esum[0] + st.esum[1] + st.esum[2];
        G->appended = 0;
        const uint64_t live = st.any | st.far;
        const uint64_t done = G->busy & ~live;
        // lanes with deferred vertices only: the threshold moves past the
        // least of them
        const uint64_t raise = G->busy & st.far & ~st.near;
        for (int k = 0; k < MP_K; k++)
            if ((raise >> k) & 1) {
                const uint64_t base = st.far_min[k] != SRV_INF ? st.far_min[k] : G->thr_h[k];
                G->thr_h[k] = (uint32_t)std::min<uint64_t>(base + S->delta, SRV_INF);
            }
        uint64_t extracted = 0;
        for (int k = 0; k < MP_K; k++) {
            if (!((done >> k) & 1)) continue;
            // every query on the lane needs its buffer; a lane whose buffers
            // do not fit yet stays busy (its frontier is empty, so its
            // supersteps do nothing) and is tried again after the next one
            bool ok = true;
            for (uint64_t qid : G->lane_q[k]) {
                Query& q = S->queries[qid];
                if (alloc_result(S, q, G->st) != IPG_OK) ok = false;
            }
            if (!ok) continue;
            const void* first = nullptr;
            for (uint64_t qid : G->lane_q[k]) {
                Query& q = S->queries[qid];
                if (!first) {
                    k_mp_extract<<<resident_cap(k_mp_extract, thread_grid(G->G->gv.V)), SRV_THREADS, 0, G->st>>>(
                        G->dist, G->G->gv.V, k, (uint32_t*)q.result);
                    first = q.result;
                } else {
                    cudaMemcpyAsync(q.result, first, q.result_bytes, cudaMemcpyDeviceToDevice, G->st);
                }
                finishing(S, q, G->st);
            }
            G->lane_q[k].clear();
            if (G->cc_lane == k) G->cc_lane = -1;
            extracted |= 1ULL << k;
        }
        G->busy &= ~extracted;
    } else {
        for (int k = 0; k < PP_K; k++) {
            if (!((G->busy >> k) & 1)) continue;
            if (++G->it[k] < (int)S->rounds) continue;
            Query& q = S->queries[G->lane_q[k][0]];
            q.state = IPG_QUERY_DONE;
            q.t_done = now;
            S->completed.push_back(q.id);
            G->lane_q[k].clear();
            G->busy &= ~(1ULL << k);
        }
    }
    G->last_used = now;
}

}  // namespace

extern "C" int ipg_server_create(uint64_t hbm_budget, uint32_t ppr_rounds, ipg_server** out)
{
    if (!out) return ipg_internal_fail(IPG_EINVAL, "ipg_server_create: null output");
    if (ppr_rounds < 1) return ipg_internal_fail(IPG_EINVAL, "ipg_server_create: ppr_rounds must be at least 1");
    ipg_server* S = new (std::nothrow) ipg_server();
    if (!S) return ipg_internal_fail(IPG_ENOMEM, "ipg_server_create: out of host memory");
    S->budget = hbm_budget;
    S->rounds = ppr_rounds;
    int dev = 0;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    cudaError_t e = cudaGetDevice(&dev);
    props.location.id = dev;
    if (e == cudaSuccess) e = cudaMemPoolCreate(&S->rpool, &props);
    uint64_t keep = UINT64_MAX;
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(S->rpool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->rel_st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (S->rpool) cudaMemPoolDestroy(S->rpool);
        delete S;
        return ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
    }
    if (const char* d = getenv("IPG_SERVE_DELTA"))
        if (*d) S->delta = (uint32_t)std::max(1UL, strtoul(d, nullptr, 10));
    if (const char* p = getenv("IPG_SERVE_PULL"))
        if (*p) S->pull = strtol(p, nullptr, 10) != 0;
    *out = S;
    return IPG_OK;
}

extern "C" void ipg_server_free(ipg_server* S)
{
    if (!S) return;
    while (!S->groups.empty()) free_group(S, S->groups.back());
    for (auto& kv : S->queries) {
        if (kv.second.ready) {
            cudaEventSynchronize(kv.second.ready);
            cudaEventDestroy(kv.second.ready);
        }
        if (kv.second.result) cudaFreeAsync(kv.second.result, S->rel_st);
    }
    cudaStreamSynchronize(S->rel_st);
    cudaStreamDestroy(S->rel_st);
    cudaMemPoolDestroy(S->rpool);
    for (auto& g : S->graphs)
        if (g->hub_prefix) ipg_dev_free(g->hub_prefix, (g->bins.count[2] + 5) * 4);
    delete S;
}

extern "C" int ipg_server_add_graph(ipg_server* S, ipg_graph* g, int* gid)
{
    if (!S || !g || !gid) return ipg_internal_fail(IPG_EINVAL, "ipg_server_add_graph: null argument");
    std::unique_ptr<Graph> G(new Graph());
    G->g = g;
    int r = ipg_graph_view_get(g, &G->gv);
    if (r != IPG_OK) return r;
    if (G->gv.id_bytes != 4) return ipg_internal_fail(IPG_EINVAL, "ipg_server_add_graph: 32-bit vertex ids only");
    if (G->gv.d_wgt && G->gv.weight_bytes != 4)
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_add_graph: weights must be u32");
    std::lock_guard<std::mutex> lk(S->mu);
    // degree classes and hub chunks (the PPR gathers, the union-find pass and
    // the pull supersteps walk them) are built now, before queries arrive:
    // building them synchronises the device
    if ((r = graph_classes(G.get(), nullptr)) != IPG_OK) {
        if (G->hub_prefix) ipg_dev_free(G->hub_prefix, (G->bins.count[2] + 5) * 4);
        return r;
    }
    *gid = (int)S->graphs.size();
    G->gid = *gid;
    S->graphs.push_back(std::move(G));
    S->pending.resize(S->graphs.size() * 2);
    S->busy_s.resize(S->graphs.size() * 2, 0.0);
    S->steps.resize(S->graphs.size() * 2, 0);
    S->lanes.resize(S->graphs.size() * 2, 0);
    S->work.resize(S->graphs.size() * 2, 0);
    return IPG_OK;
}

extern "C" int ipg_server_reserve(ipg_server* S, int gid, int kind)
{
    if (!S) return ipg_internal_fail(IPG_EINVAL, "ipg_server_reserve: null server");
    std::lock_guard<std::mutex> lk(S->mu);
    if (gid < 0 || gid >= (int)S->graphs.size()) return ipg_internal_fail(IPG_EINVAL, "ipg_server_reserve: no such graph");
    if (kind != IPG_QUERY_SSSP && kind != IPG_QUERY_PPR && kind != IPG_QUERY_CC)
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_reserve: unknown query kind");
    Graph* Gr = S->graphs[gid].get();
    // SSSP and CC queries run in the graph's min-plus group (union-find CC on
    // its stream), PPR queries in its PPR group
    const int gk = kind == IPG_QUERY_PPR ? 1 : 0;
    if (gk ? Gr->pp : Gr->mp) return IPG_OK;
    int r = create_group(S, Gr, gk);
    if (r == IPG_ENOMEM) {
        cudaMemPoolTrimTo(S->rpool, 0);
        r = create_group(S, Gr, gk);
    }
    if (r == IPG_EBUDGET) return ipg_internal_fail(IPG_EBUDGET, "ipg_server_reserve: the group does not fit the budget");
    if (r != IPG_OK) return r;
    Group* G = gk ? Gr->pp : Gr->mp;
    if (cudaStreamSynchronize(G->st) != cudaSuccess) return ipg_internal_fail(IPG_ECUDA, "ipg_server_reserve: failed");
    return IPG_OK;
}

extern "C" int ipg_server_submit(ipg_server* S, int gid, int kind, uint64_t source, uint64_t* qid)
{
    if (!S || !qid) return ipg_internal_fail(IPG_EINVAL, "ipg_server_submit: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    if (gid < 0 || gid >= (int)S->graphs.size()) return ipg_internal_fail(IPG_EINVAL, "ipg_server_submit: no such graph");
    const Graph* G = S->graphs[gid].get();
    if (kind != IPG_QUERY_SSSP && kind != IPG_QUERY_PPR && kind != IPG_QUERY_CC)
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_submit: unknown query kind");
    if (kind != IPG_QUERY_CC && source >= G->gv.V)
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_submit: source out of range");
    if (kind == IPG_QUERY_SSSP && !G->gv.d_wgt)
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_submit: SSSP needs a weighted graph");
    Query q;
    q.id = S->next_id++;
    q.gid = gid;
    q.kind = kind;
    q.src = source;
    q.t_submit = now_s();
    q.state = IPG_QUERY_PENDING;
    S->queries[q.id] = q;
    S->pending[(size_t)gid * 2 + (kind == IPG_QUERY_PPR ? 1 : 0)].push_back(q.id);
    S->n_pending++;
    S->stats.submitted++;
    *qid = q.id;
    return IPG_OK;
}

extern "C" int ipg_server_poll(ipg_server* S, uint64_t* outstanding)
{
    if (!S) return ipg_internal_fail(IPG_EINVAL, "ipg_server_poll: null server");
    std::lock_guard<std::mutex> lk(S->mu);
    const double now = now_s();
    // results completed on the device
    for (size_t i = 0; i < S->finishing.size();) {
        Query& q = S->queries[S->finishing[i]];
        if (cudaEventQuery(q.ready) != cudaSuccess) {
            i++;
            continue;
        }
        cudaEventDestroy(q.ready);
        q.ready = nullptr;
        const Graph* Gr = S->graphs[q.gid].get();
        if (q.kind == IPG_QUERY_CC && Gr->gv.symmetric && Gr->cc_err) {
            uint32_t err = 0;
            cudaMemcpy(&err, Gr->cc_err, 4, cudaMemcpyDeviceToHost);
            if (err) return ipg_internal_fail(IPG_EDEVICE, "ipg_server_poll: union-find hook retries exhausted");
        }
        q.state = IPG_QUERY_DONE;
        q.t_done = now;
        S->completed.push_back(q.id);
        S->finishing[i] = S->finishing.back();
        S->finishing.pop_back();
    }
    // groups for pending queries that have none (HBM budget permitting)
    for (size_t i = 0; i < S->pending.size(); i++) {
        if (S->pending[i].empty()) continue;
        Graph* Gr = S->graphs[i / 2].get();
        const int kind = (int)(i % 2);
        if (!(kind ? Gr->pp : Gr->mp)) {
            int r = create_group(S, Gr, kind);
            if (r == IPG_ENOMEM) {
                // memory the result pool keeps but does not use goes back first
                cudaMemPoolTrimTo(S->rpool, 0);
                r = create_group(S, Gr, kind);
            }
            if (r != IPG_OK && r != IPG_EBUDGET && r != IPG_ENOMEM) return r;
        }
    }
    // every group: retire, admit, launch
    for (size_t i = 0; i < S->groups.size(); i++) {
        Group* G = S->groups[i];
        if (G->running) {
            if (cudaEventQuery(G->ev) != cudaSuccess) continue;
            G->running = false;
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, G->ev0, G->ev) == cudaSuccess) {
                const size_t slot = (size_t)G->G->gid * 2 + G->kind;
                S->busy_s[slot] += ms * 1e-3;
                S->steps[slot]++;
            }
            retire(S, G, now);
        }
        admit(S, G, now);
        if (G->busy) {
            int r = launch_superstep(S, G);
            if (r != IPG_OK && r != IPG_ENOMEM) return r;  // ENOMEM: launched at a later poll
        }
    }
    uint64_t n = S->n_pending + S->finishing.size();
    for (Group* G : S->groups)
        for (auto& l : G->lane_q) n += l.size();
    if (outstanding) *outstanding = n;
    S->stats.bytes_in_use = S->in_use;
    if (S->in_use > S->stats.peak_bytes) S->stats.peak_bytes = S->in_use;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
    return IPG_OK;
}

extern "C" int ipg_server_query(ipg_server* S, uint64_t qid, int* state, double* latency, double* queued)
{
    if (!S) return ipg_internal_fail(IPG_EINVAL, "ipg_server_query: null server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->queries.find(qid);
    if (it == S->queries.end()) return ipg_internal_fail(IPG_EINVAL, "ipg_server_query: no such query");
    const Query& q = it->second;
    if (state) *state = q.state;
    if (latency) *latency = q.state == IPG_QUERY_DONE ? q.t_done - q.t_submit : 0.0;
    if (queued) *queued = q.t_start > 0 ? q.t_start - q.t_submit : 0.0;
    return IPG_OK;
}

extern "C" int ipg_server_result(ipg_server* S, uint64_t qid, void* out, uint64_t cap_bytes)
{
    if (!S || !out) return ipg_internal_fail(IPG_EINVAL, "ipg_server_result: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->queries.find(qid);
    if (it == S->queries.end()) return ipg_internal_fail(IPG_EINVAL, "ipg_server_result: no such query");
    const Query& q = it->second;
    if (q.state != IPG_QUERY_DONE || !q.result) return ipg_internal_fail(IPG_EINVAL, "ipg_server_result: not available");
    if (cap_bytes < q.result_bytes) return ipg_internal_fail(IPG_EINVAL, "ipg_server_result: buffer too small");
    if (cudaMemcpy(out, q.result, q.result_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        return ipg_internal_fail(IPG_ECUDA, "ipg_server_result: copy failed");
    return IPG_OK;
}

extern "C" int ipg_server_result_device(ipg_server* S, uint64_t qid, const void** d_ptr, uint64_t* bytes)
{
    if (!S || !d_ptr) return ipg_internal_fail(IPG_EINVAL, "ipg_server_result_device: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->queries.find(qid);
    if (it == S->queries.end() || it->second.state != IPG_QUERY_DONE)
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_result_device: not available");
    *d_ptr = it->second.result;
    if (bytes) *bytes = it->second.result_bytes;
    return IPG_OK;
}

extern "C" int ipg_server_release(ipg_server* S, uint64_t qid)
{
    if (!S) return ipg_internal_fail(IPG_EINVAL, "ipg_server_release: null server");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->queries.find(qid);
    if (it == S->queries.end()) return ipg_internal_fail(IPG_EINVAL, "ipg_server_release: no such query");
    if (it->second.state != IPG_QUERY_DONE) return ipg_internal_fail(IPG_EINVAL, "ipg_server_release: still running");
    release_result(S, it->second);
    S->queries.erase(it);
    return IPG_OK;
}

extern "C" int ipg_server_get_stats(ipg_server* S, ipg_server_stats* out)
{
    if (!S || !out) return ipg_internal_fail(IPG_EINVAL, "ipg_server_get_stats: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->stats;
    out->bytes_in_use = S->in_use;
    return IPG_OK;
}

extern "C" int ipg_server_group_stats(ipg_server* S, int gid, int group_kind, double* busy_s, uint64_t* supersteps,
                                      uint64_t* lanes, uint64_t* lane_edges)
{
    if (!S) return ipg_internal_fail(IPG_EINVAL, "ipg_server_group_stats: null server");
    std::lock_guard<std::mutex> lk(S->mu);
    if (gid < 0 || gid >= (int)S->graphs.size() || group_kind < 0 || group_kind > 1)
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_group_stats: no such group");
    const size_t slot = (size_t)gid * 2 + group_kind;
    if (busy_s) *busy_s = S->busy_s[slot];
    if (supersteps) *supersteps = S->steps[slot];
    if (lanes) *lanes = S->lanes[slot];
    if (lane_edges) *lane_edges = S->work[slot];
    return IPG_OK;
}

extern "C" int ipg_server_run_trace(ipg_server* S, uint64_t n, const double* arrival, const int* gid, const int* kind,
                                    const uint64_t* source, int keep_results, uint64_t* qids, double* latency,
                                    double* makespan)
{
    if (!S || (n && (!arrival || !gid || !kind || !source)))
        return ipg_internal_fail(IPG_EINVAL, "ipg_server_run_trace: null argument");
    std::vector<uint64_t> ids(n, 0);
    std::map<uint64_t, uint64_t> index;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->completed.clear();
    }
    const double t0 = now_s();
    double last_progress = t0;
    uint64_t next = 0, done = 0;
    while (done < n) {
        const double t = now_s() - t0;
        while (next < n && arrival[next] <= t) {
            int r = ipg_server_submit(S, gid[next], kind[next], source[next], &ids[next]);
            if (r != IPG_OK) return r;
            {
                // latency counts from the scheduled arrival
                std::lock_guard<std::mutex> lk(S->mu);
                S->queries[ids[next]].t_submit = t0 + arrival[next];
            }
            index[ids[next]] = next;
            next++;
        }
        uint64_t outstanding = 0;
        int r = ipg_server_poll(S, &outstanding);
        if (r != IPG_OK) return r;
        std::vector<uint64_t> fresh;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            fresh.swap(S->completed);
        }
        for (uint64_t qid : fresh) {
            auto it = index.find(qid);
            if (it == index.end()) continue;
            double lat = 0;
            ipg_server_query(S, qid, nullptr, &lat, nullptr);
            if (latency) latency[it->second] = lat;
            if (!keep_results) ipg_server_release(S, qid);
            done++;
            last_progress = now_s();
        }
        if (outstanding && next == n && now_s() - last_progress > 60.0)
            return ipg_internal_fail(IPG_EBUDGET, "ipg_server_run_trace: no progress for 60 s (HBM budget too small?)");
    }
    if (makespan) *makespan = now_s() - t0;
    if (qids)
        for (uint64_t i = 0; i < n; i++) qids[i] = ids[i];
    return IPG_OK;
}
