// pagerank_split.cu -- PageRank with FP32 values and compensated gather sums,
// FP64 diagnostics (no counterpart in the reference; its PageRank is FP64
// throughout).
//
// Formula and superstep structure follow benchmarks/pagerank.c:36-66,98-99
// run under the single-broadcast version (combiner_single_broadcast_
// postamble.h:57-89,185-201):
//   superstep 0:       x_v = 1/V
//   superstep s >= 1:  x_v = (1-d)/V + d * sum_{u in row(v), deg u > 0} x_u / deg u
//   a vertex broadcasts x_v / deg v while s < rounds and deg v > 0;
// rounds + 1 supersteps in all.  As in the reference's benchmarks (they load
// with directed = false, pagerank.c:91), the stored rows serve both as the
// gather lists and for the out-degrees; no dangling mass is redistributed.
//
// Precision split: the values x and the broadcast quotients are FP32 (4 bytes
// per vertex, so the gathered array of an R-MAT scale-24 graph, 64 MiB, stays
// in the 126 MB L2), and each gather sum is compensated: every lane keeps a
// (sum, compensation) pair updated with Knuth's TwoSum (the Kahan-Babuska
// refinement of Kahan summation due to Neumaier, 1974), and pairs of lanes,
// warps and hub chunks are merged with the same error-free transformation.
// The diagnostics of every superstep -- the mass sum x, the dangling mass (sum
// of x over vertices without out-edges) and the L1 residual sum |x - x_prev| --
// are reduced in FP64.
//
// Kernels per superstep: one gather+update kernel per degree class (thread
// per vertex up to t0 edges, warp per vertex up to t1 edges), and for the
// hubs a chunk kernel (one CTA per PR_CHUNK edges, partial pairs to scratch)
// followed by a finalising kernel that merges each hub's chunk partials in
// chunk order.  Everything is enqueued on one stream without host
// synchronisation or allocation, so a run can be captured into a CUDA graph.
#include "ipregel_b200.h"

#include <cuda_runtime.h>

#include <cstdlib>
#include <new>
#include <utility>
#include <vector>

extern "C" int ipg_internal_fail(int code, const char* msg);

#define PR_THREADS 256
#define PR_UNROLL 4
#define PR_CHUNK 4096
#ifndef PR_GROUP
#define PR_GROUP 16 /* lanes per vertex of the middle degree class */
#endif
#define PR_CTAS_PER_SM 8 /* upper bound; the resident count decides */

#define PR_CUDA(call)                                                      \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) return ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e_)); \
    } while (0)

#define PR_TRY(call)                       \
    do {                                   \
        int r_ = (call);                   \
        if (r_ != IPG_OK) return r_;       \
    } while (0)

struct ipg_pr_plan {
    ipg_graph* g = nullptr;
    ipg_graph_view gv{};
    ipg_bins bins{};
    float* b[2] = {nullptr, nullptr};  // broadcast quotients, by superstep parity
    float* xs = nullptr;               // values of every other superstep
    // on the graph's degree-ordered copy (ipg_graph_degree_order): the
    // supersteps write xs / xs2 in the copy's numbering, and a last gather
    // writes the values in the caller's (null: the graph's own numbering)
    const uint32_t* new_of_old = nullptr;
    float* xs2 = nullptr;
    uint32_t* hub_prefix = nullptr;    // first chunk of each hub, then the total
    uint32_t* hub_owner = nullptr;     // chunk -> index of its hub
    float2* partial = nullptr;         // (sum, compensation) of every hub chunk
    uint64_t chunks = 0;
    int sms = 148;
    uint32_t grid = 0;  // resident CTAs of the gather kernels, all SMs
    std::vector<std::pair<void*, uint64_t>> allocs;
};

namespace {

// ---- compensated FP32 accumulation ----------------------------------------
// The value of a pair is s + c.  TwoSum gives the exact rounding error of
// s + x, which is carried in c.  __fadd_rn/__fsub_rn keep the compiler from
// contracting or reordering the error terms.
template <bool COMP>
__device__ __forceinline__ void pr_add(float& s, float& c, float x)
{
    if constexpr (COMP) {
        const float t = __fadd_rn(s, x);
        const float bp = __fsub_rn(t, s);
        const float err = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(x, bp));
        c = __fadd_rn(c, err);
        s = t;
    } else {
        (void)c;
        s = __fadd_rn(s, x);
    }
}

template <bool COMP>
__device__ __forceinline__ void pr_merge(float& s, float& c, float s2, float c2)
{
    pr_add<COMP>(s, c, s2);
    if constexpr (COMP) c = __fadd_rn(c, c2);
}

template <bool COMP>
__device__ __forceinline__ void pr_warp_merge(float& s, float& c)
{
    for (int o = 16; o > 0; o >>= 1) {
        const float s2 = __shfl_down_sync(0xffffffffu, s, o);
        const float c2 = __shfl_down_sync(0xffffffffu, c, o);
        pr_merge<COMP>(s, c, s2, c2);
    }
}

struct PrStep {
    const uint64_t* __restrict__ row;     // out-rows: the degrees
    const uint64_t* __restrict__ in_row;  // gather lists (the rows themselves
    const uint32_t* __restrict__ in_adj;  // unless the graph is directed)
    const float* __restrict__ b_cur;  // read by the gathers
    float* __restrict__ b_next;       // written for the next superstep
    float* __restrict__ x_out;        // this superstep's values
    float ratio, damping;
};

// Sum of the vertex diagnostics over the CTA, added to diag[0..2].
__device__ __forceinline__ void pr_block_diag(double m, double d, double r, double* diag)
{
    __shared__ double sh[3][PR_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, o);
        d += __shfl_down_sync(0xffffffffu, d, o);
        r += __shfl_down_sync(0xffffffffu, r, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][warp] = m;
        sh[1][warp] = d;
        sh[2][warp] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, c = 0;
        for (int w = 0; w < PR_THREADS / 32; w++) {
            a += sh[0][w];
            b += sh[1][w];
            c += sh[2][w];
        }
        if (a != 0.0) atomicAdd(&diag[0], a);
        if (b != 0.0) atomicAdd(&diag[1], b);
        if (c != 0.0) atomicAdd(&diag[2], c);
    }
}

// Vertex update of pagerank.c:51-52 and the broadcast of :57-63.  The
// values are double-buffered: the gathers only write, and the diagnostics
// come from a separate streaming pass over both buffers (reading the old
// value here, one more dependent load per vertex, cost more than doubling
// the superstep on R-MAT scale 24).
template <bool LAST>
__device__ __forceinline__ void pr_finish(const PrStep& a, uint64_t v, uint64_t deg, float sum)
{
    const float xn = __fadd_rn(a.ratio, __fmul_rn(a.damping, sum));
    a.x_out[v] = xn;
    if constexpr (!LAST) a.b_next[v] = deg ? __fdiv_rn(xn, (float)deg) : 0.0f;
}

// Lane-strided compensated sum of b_cur over adj[e0, e1), PR_UNROLL loads in
// flight per lane (warps and blocks: pr_gather_v4).  Ids are loaded evict-first where a warp reads consecutive
// ids in one instruction (lanes >= 32); a thread walking a row alone comes
// back to the same line in its next loads, so it keeps the line cached.
template <bool COMP>
__device__ __forceinline__ void pr_gather_v4(const PrStep& a, uint64_t e0, uint64_t e1, uint64_t lane,
                                             uint64_t lanes, float& s, float& c)
{
    // a warp or block reads four consecutive ids per lane with one 128-bit
    // load; the up to 3 ids before the first 16-byte boundary and after the
    // last take a lane each
    uint64_t al = (e0 + 3) & ~3ULL;
    if (al > e1) al = e1;
    const uint64_t b = al + ((e1 - al) & ~3ULL);
    {
        const uint64_t nh = al - e0, nt = e1 - b;
        uint64_t e = e1;
        if (lane < nh) e = e0 + lane;
        else if (lane < nh + nt) e = b + (lane - nh);
        if (e < e1) pr_add<COMP>(s, c, __ldg(&a.b_cur[a.in_adj[e]]));
    }
    const uint4* __restrict__ q4 = reinterpret_cast<const uint4*>(a.in_adj + al);
    const uint64_t groups = (b - al) >> 2;
    for (uint64_t g = lane; g < groups; g += lanes) {
        const uint4 id = __ldcs(q4 + g);
        const float q0 = __ldg(&a.b_cur[id.x]), q1 = __ldg(&a.b_cur[id.y]);
        const float q2 = __ldg(&a.b_cur[id.z]), q3 = __ldg(&a.b_cur[id.w]);
        pr_add<COMP>(s, c, q0);
        pr_add<COMP>(s, c, q1);
        pr_add<COMP>(s, c, q2);
        pr_add<COMP>(s, c, q3);
    }
}

template <bool COMP>
__device__ __forceinline__ void pr_gather(const PrStep& a, uint64_t e0, uint64_t e1, uint64_t lane, uint64_t lanes,
                                          float& s, float& c)
{
    if (lanes >= 8 && (reinterpret_cast<uintptr_t>(a.in_adj) & 15) == 0) {
        pr_gather_v4<COMP>(a, e0, e1, lane, lanes, s, c);
        return;
    }
    for (uint64_t e = e0 + lane; e < e1; e += PR_UNROLL * lanes) {
        uint32_t u[PR_UNROLL];
        float q[PR_UNROLL];
#pragma unroll
        for (int k = 0; k < PR_UNROLL; k++) {
            const uint64_t ek = e + k * lanes;
            u[k] = ek < e1 ? (lanes >= 32 ? __ldcs(&a.in_adj[ek]) : a.in_adj[ek]) : 0u;
        }
#pragma unroll
        for (int k = 0; k < PR_UNROLL; k++) q[k] = (e + k * lanes < e1) ? __ldg(&a.b_cur[u[k]]) : 0.0f;
#pragma unroll
        for (int k = 0; k < PR_UNROLL; k++)
            if (e + k * lanes < e1) pr_add<COMP>(s, c, q[k]);
    }
}

// Out-degree of v whose gather list is in_adj[e0, e1).
__device__ __forceinline__ uint64_t pr_deg(const PrStep& a, uint64_t v, uint64_t e0, uint64_t e1)
{
    return a.row == a.in_row ? e1 - e0 : a.row[v + 1] - a.row[v];
}

// Superstep 0: x = 1/V, broadcast x/deg.
__global__ void __launch_bounds__(PR_THREADS) k_pr_init(PrStep a, uint64_t V, float x0)
{
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t deg = a.row[v + 1] - a.row[v];
        a.x_out[v] = x0;
        a.b_next[v] = deg ? __fdiv_rn(x0, (float)deg) : 0.0f;
    }
}

// FP64 diagnostics of a superstep: diag = {sum x, sum of x over vertices
// without out-edges, sum |x - x_prev|} (x_prev null at superstep 0).
__global__ void __launch_bounds__(PR_THREADS) k_pr_diag(const float* __restrict__ x, const float* __restrict__ x_prev,
                                                        const uint64_t* __restrict__ row, uint64_t V,
                                                        double* __restrict__ diag)
{
    double m = 0, d = 0, r = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const double xv = (double)x[v];
        m += xv;
        if (row[v + 1] == row[v]) d += xv;
        if (x_prev) r += fabs(xv - (double)x_prev[v]);
    }
    pr_block_diag(m, d, r, diag);
}

// out[i] = x[new_of_old[i]]: the values in the caller's numbering.
__global__ void k_pr_by_id(const float* __restrict__ x, const uint32_t* __restrict__ new_of_old, uint64_t V,
                           float* __restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = x[new_of_old[i]];
}

// Class 0: a thread per vertex.
template <bool COMP, bool LAST>
__global__ void __launch_bounds__(PR_THREADS) k_pr_thread(PrStep a, const uint32_t* __restrict__ list, uint64_t n)
{
    // the next vertex's list entry and row bounds are loaded while this
    // vertex's in-edges are gathered
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x, v = 0, e0 = 0, e1 = 0;
    if (i < n) {
        v = list[i];
        e0 = a.in_row[v];
        e1 = a.in_row[v + 1];
    }
    for (; i < n; i += stride) {
        uint64_t vn = 0, e0n = 0, e1n = 0;
        if (i + stride < n) {
            vn = list[i + stride];
            e0n = a.in_row[vn];
            e1n = a.in_row[vn + 1];
        }
        float s = 0.0f, c = 0.0f;
        pr_gather<COMP>(a, e0, e1, 0, 1, s, c);
        pr_finish<LAST>(a, v, pr_deg(a, v, e0, e1), __fadd_rn(s, c));
        v = vn;
        e0 = e0n;
        e1 = e1n;
    }
}

// Class 1: PR_GROUP lanes per vertex (most vertices of the class have a few
// dozen in-edges, which 16 lanes reading four ids each cover in a step or
// two; a whole warp per vertex left most lanes idle).
template <bool COMP, bool LAST>
__global__ void __launch_bounds__(PR_THREADS) k_pr_warp(PrStep a, const uint32_t* __restrict__ list, uint64_t n)
{
    constexpr int G = PR_GROUP;
    const int lane = threadIdx.x & 31, gl = lane & (G - 1);
    const unsigned mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
    const uint64_t groups = ((uint64_t)gridDim.x * blockDim.x) / G;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / G; i < n; i += groups) {
        const uint64_t v = list[i];
        const uint64_t e0 = a.in_row[v], e1 = a.in_row[v + 1];
        float s = 0.0f, c = 0.0f;
        pr_gather<COMP>(a, e0, e1, gl, G, s, c);
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            const float s2 = __shfl_down_sync(mask, s, o, G);
            const float c2 = __shfl_down_sync(mask, c, o, G);
            pr_merge<COMP>(s, c, s2, c2);
        }
        if (gl == 0) pr_finish<LAST>(a, v, pr_deg(a, v, e0, e1), __fadd_rn(s, c));
    }
}

// Class 2, pass 1: a warp per chunk of PR_CHUNK edges of a hub (no CTA-wide
// barriers per chunk: 15 - 20 % shorter in the FP64 engine's gather).
template <bool COMP>
__global__ void __launch_bounds__(PR_THREADS) k_pr_hub_chunks(PrStep a, const uint32_t* __restrict__ list, uint64_t n,
                                                              const uint32_t* __restrict__ prefix,
                                                              const uint32_t* __restrict__ owner,
                                                              float2* __restrict__ partial)
{
    if (n == 0) return;
    const uint32_t chunks = prefix[n];
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t ch = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; ch < chunks; ch += warps) {
        const uint64_t i = owner[ch];  // one load, not a binary search over the prefix
        const uint64_t v = list[i];
        const uint64_t end = a.in_row[v + 1];
        const uint64_t e0 = a.in_row[v] + (ch - prefix[i]) * (uint64_t)PR_CHUNK;
        const uint64_t e1 = e0 + PR_CHUNK < end ? e0 + PR_CHUNK : end;
        float s = 0.0f, c = 0.0f;
        pr_gather<COMP>(a, e0, e1, lane, 32, s, c);
        pr_warp_merge<COMP>(s, c);
        if (lane == 0) partial[ch] = make_float2(s, c);
    }
}

// Class 2, pass 2: a warp per hub merges its chunk partials in chunk order.
template <bool COMP, bool LAST>
__global__ void __launch_bounds__(PR_THREADS) k_pr_hub_finish(PrStep a, const uint32_t* __restrict__ list, uint64_t n,
                                                              const uint32_t* __restrict__ prefix,
                                                              const float2* __restrict__ partial)
{
    const int lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint64_t v = list[i];
        float s = 0.0f, c = 0.0f;
        for (uint32_t ch = prefix[i] + lane; ch < prefix[i + 1]; ch += 32) {
            const float2 p = partial[ch];
            pr_merge<COMP>(s, c, p.x, p.y);
        }
        pr_warp_merge<COMP>(s, c);
        if (lane == 0) pr_finish<LAST>(a, v, a.row[v + 1] - a.row[v], __fadd_rn(s, c));
    }
}

__global__ void k_pr_hub_chunk_counts(const uint32_t* __restrict__ list, uint64_t n, const uint64_t* __restrict__ row,
                                      uint32_t* __restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = list[i];
        out[i] = (uint32_t)((row[v + 1] - row[v] + PR_CHUNK - 1) / PR_CHUNK);
    }
}

template <bool COMP, bool LAST>
int pr_superstep(ipg_pr_plan* p, const PrStep& a, cudaStream_t st)
{
    const ipg_bins& b = p->bins;
    const uint32_t grid = p->grid;
    if (b.count[0]) k_pr_thread<COMP, LAST><<<grid, PR_THREADS, 0, st>>>(a, b.d_list[0], b.count[0]);
    if (b.count[1]) k_pr_warp<COMP, LAST><<<grid, PR_THREADS, 0, st>>>(a, b.d_list[1], b.count[1]);
    if (b.count[2]) {
        k_pr_hub_chunks<COMP><<<grid, PR_THREADS, 0, st>>>(a, b.d_list[2], b.count[2], p->hub_prefix, p->hub_owner,
                                                             p->partial);
        const uint32_t g2 = (uint32_t)((b.count[2] * 32 + PR_THREADS - 1) / PR_THREADS);
        k_pr_hub_finish<COMP, LAST><<<g2 < grid ? g2 : grid, PR_THREADS, 0, st>>>(a, b.d_list[2], b.count[2],
                                                                                  p->hub_prefix, p->partial);
    }
    PR_CUDA(cudaGetLastError());
    return IPG_OK;
}

// Grid-stride kernels get exactly the CTAs that are resident at once: more
// would run as a second wave after the first finished its static share.
template <class K>
int pr_occupancy(K kernel)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, PR_THREADS, 0) != cudaSuccess || n <= 0) n = 1;
    return n < PR_CTAS_PER_SM ? n : PR_CTAS_PER_SM;
}

int pr_min_occupancy()
{
    int n = PR_CTAS_PER_SM;
    auto low = [&](int k) { n = k < n ? k : n; };
    low(pr_occupancy(k_pr_init));
    low(pr_occupancy(k_pr_diag));
    low(pr_occupancy(k_pr_thread<true, false>));
    low(pr_occupancy(k_pr_thread<true, true>));
    low(pr_occupancy(k_pr_thread<false, false>));
    low(pr_occupancy(k_pr_thread<false, true>));
    low(pr_occupancy(k_pr_warp<true, false>));
    low(pr_occupancy(k_pr_warp<true, true>));
    low(pr_occupancy(k_pr_warp<false, false>));
    low(pr_occupancy(k_pr_warp<false, true>));
    low(pr_occupancy(k_pr_hub_chunks<true>));
    low(pr_occupancy(k_pr_hub_chunks<false>));
    return n;
}

template <class T>
int pr_alloc(ipg_pr_plan* p, T** out, uint64_t n)
{
    void* d = nullptr;
    const uint64_t bytes = (n ? n : 1) * sizeof(T);
    PR_TRY(ipg_dev_alloc(&d, bytes));
    p->allocs.push_back({d, bytes});
    *out = (T*)d;
    return IPG_OK;
}

// Error of an FP32 vector against an FP64 one: out[0] = max abs, out[1] =
// max rel (abs where the reference is 0), out[2] = sum of abs, as doubles.
// Non-negative doubles order as their bit patterns, so the maxima use integer
// atomics.
__global__ void k_err_f32_f64(const float* __restrict__ a, const double* __restrict__ ref, uint64_t n,
                              unsigned long long* __restrict__ out)
{
    double mabs = 0, mrel = 0, sabs = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double e = fabs((double)a[i] - ref[i]);
        const double r = ref[i] != 0.0 ? e / fabs(ref[i]) : e;
        mabs = e > mabs ? e : mabs;
        mrel = r > mrel ? r : mrel;
        sabs += e;
    }
    atomicMax(&out[0], (unsigned long long)__double_as_longlong(mabs));
    atomicMax(&out[1], (unsigned long long)__double_as_longlong(mrel));
    atomicAdd((double*)&out[2], sabs);
}

// out[3] = smallest index whose abs error equals the maximum.
__global__ void k_err_argmax(const float* __restrict__ a, const double* __restrict__ ref, uint64_t n,
                             unsigned long long* __restrict__ out)
{
    const double mabs = __longlong_as_double((long long)out[0]);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (fabs((double)a[i] - ref[i]) == mabs) atomicMin(&out[3], (unsigned long long)i);
}

}  // namespace

extern "C" int ipg_pr_plan_create(ipg_graph* g, ipg_pr_plan** out)
{
    if (!g || !out) return ipg_internal_fail(IPG_EINVAL, "ipg_pr_plan_create: null argument");
    *out = nullptr;
    ipg_pr_plan* p = new (std::nothrow) ipg_pr_plan();
    if (!p) return ipg_internal_fail(IPG_ENOMEM, "ipg_pr_plan_create: out of host memory");
    int r = IPG_OK;
    do {
        p->g = g;
        if ((r = ipg_graph_view_get(g, &p->gv)) != IPG_OK) break;
        if (p->gv.id_bytes != 4) {
            r = ipg_internal_fail(IPG_EINVAL, "ipg_pr_plan_create: the FP32 PageRank takes 32-bit vertex ids");
            break;
        }
        if (p->gv.V >= (1ULL << 32)) {
            r = ipg_internal_fail(IPG_EINVAL, "ipg_pr_plan_create: more than 2^32 - 1 vertices");
            break;
        }
        p->sms = ipg_sm_count();
        const char* t0s = getenv("IPG_PR_T0");
        const char* t1s = getenv("IPG_PR_T1");
        const uint64_t t0 = (t0s && *t0s) ? strtoull(t0s, nullptr, 10) : 16;
        const uint64_t t1 = (t1s && *t1s) ? strtoull(t1s, nullptr, 10) : 4096;
        // the gathers run on the degree-ordered copy unless IPG_ORDER=0 (or
        // the copy does not fit the HBM budget): the most gathered
        // quotients share cache lines
        ipg_graph* gw = g;
        const char* ord = getenv("IPG_ORDER");
        if (!(ord && *ord && strtoull(ord, nullptr, 10) == 0) && p->gv.V < (1ULL << 31)) {
            ipg_order o;
            const int ro = ipg_graph_degree_order(g, 1, &o);
            if (ro == IPG_OK) {
                gw = o.graph;
                p->new_of_old = o.d_new_of_old;
            } else if (ro != IPG_EBUDGET && ro != IPG_ENOMEM) {
                r = ro;
                break;
            }
        }
        // classes over the gather lists (builds the in-lists of a directed graph)
        if ((r = ipg_graph_bins(gw, 1, t0, t1, &p->bins)) != IPG_OK) break;
        if ((r = ipg_graph_view_get(gw, &p->gv)) != IPG_OK) break;
        p->grid = (uint32_t)p->sms * (uint32_t)pr_min_occupancy();
        const uint64_t V = p->gv.V, nh = p->bins.count[2];
        if ((r = pr_alloc(p, &p->b[0], V)) != IPG_OK) break;
        if ((r = pr_alloc(p, &p->b[1], V)) != IPG_OK) break;
        if ((r = pr_alloc(p, &p->xs, V)) != IPG_OK) break;
        if (p->new_of_old && (r = pr_alloc(p, &p->xs2, V)) != IPG_OK) break;
        if ((r = pr_alloc(p, &p->hub_prefix, nh + 1)) != IPG_OK) break;
        std::vector<uint32_t> cnt(nh + 1, 0);
        if (nh) {
            k_pr_hub_chunk_counts<<<(uint32_t)((nh + 255) / 256), 256>>>(p->bins.d_list[2], nh, p->gv.d_in_row,
                                                                       p->hub_prefix);
            cudaError_t e = cudaMemcpy(cnt.data(), p->hub_prefix, nh * 4, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                r = ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
                break;
            }
        }
        uint64_t total = 0;
        for (uint64_t i = 0; i < nh; i++) {
            const uint32_t c = cnt[i];
            cnt[i] = (uint32_t)total;
            total += c;
        }
        cnt[nh] = (uint32_t)total;
        if (total >= (1ULL << 32)) {
            r = ipg_internal_fail(IPG_EINVAL, "ipg_pr_plan_create: too many hub chunks");
            break;
        }
        p->chunks = total;
        cudaError_t e = cudaMemcpy(p->hub_prefix, cnt.data(), (nh + 1) * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            r = ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
            break;
        }
        if ((r = pr_alloc(p, &p->partial, total)) != IPG_OK) break;
        std::vector<uint32_t> owner(total);
        for (uint64_t i = 0; i < nh; i++)
            for (uint32_t ch = cnt[i]; ch < cnt[i + 1]; ch++) owner[ch] = (uint32_t)i;
        if ((r = pr_alloc(p, &p->hub_owner, total + 1)) != IPG_OK) break;
        if (total) {
            e = cudaMemcpy(p->hub_owner, owner.data(), total * 4, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                r = ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
                break;
            }
        }
    } while (0);
    if (r != IPG_OK) {
        ipg_pr_plan_free(p);
        return r;
    }
    *out = p;
    return IPG_OK;
}

extern "C" void ipg_pr_plan_free(ipg_pr_plan* p)
{
    if (!p) return;
    for (auto& a : p->allocs) ipg_dev_free(a.first, a.second);
    delete p;
}

extern "C" int ipg_pr_run_f32(ipg_pr_plan* p, uint32_t rounds, double damping, int compensated, float* d_values,
                              double* d_diag, void* stream)
{
    if (!p || !d_values || !d_diag) return ipg_internal_fail(IPG_EINVAL, "ipg_pr_run_f32: null argument");
    if (!(damping >= 0.0 && damping <= 1.0)) return ipg_internal_fail(IPG_EINVAL, "ipg_pr_run_f32: damping outside [0, 1]");
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t V = p->gv.V;
    PR_CUDA(cudaMemsetAsync(d_diag, 0, (uint64_t)(rounds + 1) * 3 * sizeof(double), st));
    if (V == 0) return IPG_OK;
    PrStep a;
    a.row = p->gv.d_row;
    a.in_row = p->gv.d_in_row;
    a.in_adj = (const uint32_t*)p->gv.d_in_adj;
    // superstep s writes its values to xbuf(s), so that the last one lands in
    // d_values (on the renamed copy: in xs2, gathered into d_values at the end)
    float* last = p->new_of_old ? p->xs2 : d_values;
    auto xbuf = [&](uint32_t s) { return ((rounds - s) & 1) ? p->xs : last; };
    a.ratio = (float)((1.0 - damping) / (double)V);  // pagerank.c:98 (0.15 / V)
    a.damping = (float)damping;
    a.b_cur = nullptr;
    a.b_next = p->b[0];
    a.x_out = xbuf(0);
    k_pr_init<<<p->grid, PR_THREADS, 0, st>>>(a, V, (float)(1.0 / (double)V));  // pagerank.c:99
    k_pr_diag<<<p->grid, PR_THREADS, 0, st>>>(a.x_out, nullptr, a.row, V, d_diag);
    PR_CUDA(cudaGetLastError());
    for (uint32_t s = 1; s <= rounds; s++) {
        a.b_cur = p->b[(s - 1) & 1];
        a.b_next = p->b[s & 1];
        a.x_out = xbuf(s);
        const bool last = s == rounds;
        int r;
        if (compensated) r = last ? pr_superstep<true, true>(p, a, st) : pr_superstep<true, false>(p, a, st);
        else r = last ? pr_superstep<false, true>(p, a, st) : pr_superstep<false, false>(p, a, st);
        PR_TRY(r);
        k_pr_diag<<<p->grid, PR_THREADS, 0, st>>>(a.x_out, xbuf(s - 1), a.row, V, d_diag + (uint64_t)s * 3);
        PR_CUDA(cudaGetLastError());
    }
    if (p->new_of_old) {
        k_pr_by_id<<<p->grid, PR_THREADS, 0, st>>>(last, p->new_of_old, V, d_values);
        PR_CUDA(cudaGetLastError());
    }
    return IPG_OK;
}

extern "C" int ipg_pr_plan_info(const ipg_pr_plan* p, uint64_t* class_counts, uint64_t* class_edges,
                                uint64_t* hub_chunks)
{
    if (!p) return ipg_internal_fail(IPG_EINVAL, "ipg_pr_plan_info: null plan");
    for (int k = 0; k < 3; k++) {
        if (class_counts) class_counts[k] = p->bins.count[k];
        if (class_edges) class_edges[k] = p->bins.edges[k];
    }
    if (hub_chunks) *hub_chunks = p->chunks;
    return IPG_OK;
}

extern "C" int ipg_error_f32_f64(const float* d_a, const double* d_ref, uint64_t n, double* max_abs, double* max_rel,
                                 double* mean_abs, uint64_t* argmax_abs, void* stream)
{
    if ((!d_a || !d_ref) && n) return ipg_internal_fail(IPG_EINVAL, "ipg_error_f32_f64: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long* d_out = nullptr;
    PR_TRY(ipg_dev_alloc((void**)&d_out, 4 * sizeof(unsigned long long)));
    unsigned long long h[4] = {0, 0, 0, ~0ULL};
    cudaError_t e = cudaMemcpyAsync(d_out, h, sizeof h, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && n) {
        const uint64_t blocks = (n + 255) / 256;
        const uint32_t grid = (uint32_t)(blocks < 1184 ? blocks : 1184);
        k_err_f32_f64<<<grid, 256, 0, st>>>(d_a, d_ref, n, d_out);
        k_err_argmax<<<grid, 256, 0, st>>>(d_a, d_ref, n, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_out, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    ipg_dev_free(d_out, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) return ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
    double v[3];
    for (int k = 0; k < 3; k++) {
        long long bits = (long long)h[k];
        v[k] = *reinterpret_cast<double*>(&bits);
    }
    if (max_abs) *max_abs = v[0];
    if (max_rel) *max_rel = v[1];
    if (mean_abs) *mean_abs = n ? v[2] / (double)n : 0.0;
    if (argmax_abs) *argmax_abs = n ? h[3] : 0;
    return IPG_OK;
}
