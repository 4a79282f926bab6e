// runtime.cu -- libipregel_b200.so: the type-independent runtime under the
// drop-in iPregel headers.  C ABI declared in include/ipregel_b200.h.
//
// Graph residency (replaces the reference loader, src/iPregel_postamble.h:
// 244-546), seeded device generators, the in-CSR build that reproduces the
// reference's in-neighbour mirror order (iPregel_postamble.h:429-487), and the
// frontier primitives (bitmap -> degree-class lists, bitmap popcounts) that
// the typed superstep kernels in include/ipregel_b200/engine.cuh call.

#include "ipregel_b200.h"

#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <atomic>
#include <cerrno>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <mutex>
#include <string>
#include <thread>
#include <unistd.h>
#include <vector>

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define IPG_CUDA(call)                                                          \
    do {                                                                        \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess)                                                  \
            return fail(IPG_ECUDA, "%s failed: %s (%s:%d)", #call,              \
                        cudaGetErrorString(e_), __FILE__, __LINE__);            \
    } while (0)

#define IPG_TRY(call)                                                           \
    do {                                                                        \
        int r_ = (call);                                                        \
        if (r_ != IPG_OK) return r_;                                            \
    } while (0)

extern "C" const char* ipg_last_error(void) { return g_err.c_str(); }

// Lets other translation units of this library report through ipg_last_error.
extern "C" __attribute__((visibility("hidden"))) int ipg_internal_fail(int code, const char* msg)
{
    return fail(code, "%s", msg);
}
extern "C" int ipg_abi_version(void) { return IPG_ABI_VERSION; }

static int g_sm_count = 0;

extern "C" int ipg_sm_count(void)
{
    if (g_sm_count == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return 148;
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            return 148;
        g_sm_count = n;
    }
    return g_sm_count;
}

extern "C" int ipg_device_info(char* name, size_t name_len, uint64_t* hbm_bytes, int* sm_count)
{
    int dev = 0;
    IPG_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    IPG_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (name && name_len) {
        strncpy(name, prop.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    if (hbm_bytes) *hbm_bytes = prop.totalGlobalMem;
    if (sm_count) *sm_count = prop.multiProcessorCount;
    return IPG_OK;
}

// ---------------------------------------------------------------------------
// Device memory accounting
// ---------------------------------------------------------------------------
static std::atomic<uint64_t> g_in_use{0};
static std::atomic<uint64_t> g_budget{0};
static std::once_flag g_budget_once;

static void init_budget()
{
    std::call_once(g_budget_once, [] {
        const char* e = getenv("IPG_HBM_BUDGET");
        if (e && *e) g_budget = strtoull(e, nullptr, 10);
    });
}

extern "C" int ipg_set_hbm_budget(uint64_t bytes)
{
    init_budget();
    g_budget = bytes;
    return IPG_OK;
}

extern "C" uint64_t ipg_hbm_in_use(void) { return g_in_use.load(); }

extern "C" int ipg_dev_alloc(void** d_ptr, uint64_t bytes)
{
    init_budget();
    if (!d_ptr) return fail(IPG_EINVAL, "ipg_dev_alloc: null output pointer");
    *d_ptr = nullptr;
    if (bytes == 0) bytes = 16;
    uint64_t budget = g_budget.load();
    uint64_t now = g_in_use.fetch_add(bytes) + bytes;
    if (budget && now > budget) {
        g_in_use.fetch_sub(bytes);
        return fail(IPG_EBUDGET, "HBM budget exceeded: %llu bytes requested, %llu of %llu in use",
                    (unsigned long long)bytes, (unsigned long long)(now - bytes),
                    (unsigned long long)budget);
    }
    cudaError_t e = cudaMalloc(d_ptr, bytes);
    if (e != cudaSuccess) {
        g_in_use.fetch_sub(bytes);
        *d_ptr = nullptr;
        cudaGetLastError();
        return fail(IPG_ENOMEM, "cudaMalloc(%llu) failed: %s", (unsigned long long)bytes,
                    cudaGetErrorString(e));
    }
    return IPG_OK;
}

extern "C" int ipg_dev_free(void* d_ptr, uint64_t bytes)
{
    if (!d_ptr) return IPG_OK;
    if (bytes == 0) bytes = 16;
    g_in_use.fetch_sub(bytes);
    IPG_CUDA(cudaFree(d_ptr));
    return IPG_OK;
}

extern "C" int ipg_host_alloc(void** ptr, uint64_t bytes)
{
    if (!ptr) return fail(IPG_EINVAL, "ipg_host_alloc: null output pointer");
    *ptr = nullptr;
    cudaError_t e = cudaHostAlloc(ptr, bytes ? bytes : 16, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return fail(IPG_ENOMEM, "cudaHostAlloc(%llu) failed: %s", (unsigned long long)bytes, cudaGetErrorString(e));
    }
    return IPG_OK;
}

extern "C" int ipg_host_free(void* ptr)
{
    if (ptr) IPG_CUDA(cudaFreeHost(ptr));
    return IPG_OK;
}

extern "C" int ipg_memcpy(void* dst, const void* src, uint64_t bytes)
{
    if (!bytes) return IPG_OK;
    if (!dst || !src) return fail(IPG_EINVAL, "ipg_memcpy: null pointer");
    IPG_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
    return IPG_OK;
}

// RAII device buffer for temporaries.
struct DevBuf {
    void* p = nullptr;
    uint64_t n = 0;
    int alloc(uint64_t bytes)
    {
        release();
        int r = ipg_dev_alloc(&p, bytes);
        if (r == IPG_OK) n = bytes;
        return r;
    }
    void release()
    {
        if (p) ipg_dev_free(p, n);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    template <class T> T* as() { return static_cast<T*>(p); }
};

// ---------------------------------------------------------------------------
// Graph object
// ---------------------------------------------------------------------------
struct ipg_graph {
    ipg_graph_view v;
    bool owns_out = true;
    void* row = nullptr;  uint64_t row_bytes = 0;
    void* adj = nullptr;  uint64_t adj_bytes = 0;
    void* wgt = nullptr;  uint64_t wgt_bytes = 0;
    void* in_row = nullptr; uint64_t in_row_bytes = 0;
    void* in_adj = nullptr; uint64_t in_adj_bytes = 0;
    void* in_wgt = nullptr; uint64_t in_wgt_bytes = 0;
    struct BinCache {
        bool valid = false;
        uint64_t t0 = 0, t1 = 0;
        void* lists = nullptr;
        uint64_t bytes = 0;
        ipg_bins bins;
    } bins[2];
    // ipg_graph_refill_host's own stream, device words (check bits, degree
    // maxima), pinned words and offset staging, made at its first call
    cudaStream_t refill_st = nullptr;
    void* refill_dev = nullptr;
    uint64_t* refill_host = nullptr;
    void* refill_stage = nullptr;
    uint64_t refill_stage_bytes = 0;
    // contents generation (bumped by every refill) and whether the contents
    // failed validation; engines record the generation at attach and refuse
    // to run after it changed or while the contents are bad
    uint64_t generation = 0;
    bool bad = false;
    // the degree-ordered copy (ipg_graph_degree_order) of the contents of
    // generation ord_generation, its 4-byte id maps and its build scratch
    ipg_graph* ord = nullptr;
    void* ord_old_of_new = nullptr;
    void* ord_new_of_old = nullptr;
    uint64_t ord_map_bytes = 0;
    void* ord_scratch = nullptr;
    uint64_t ord_scratch_bytes = 0;
    uint64_t ord_generation = 0;
    bool ord_valid = false;
    void drop_order()
    {
        delete ord;
        ord = nullptr;
        ipg_dev_free(ord_old_of_new, ord_map_bytes);
        ipg_dev_free(ord_new_of_old, ord_map_bytes);
        ipg_dev_free(ord_scratch, ord_scratch_bytes);
        ord_old_of_new = ord_new_of_old = ord_scratch = nullptr;
        ord_map_bytes = ord_scratch_bytes = 0;
        ord_valid = false;
    }
    ~ipg_graph()
    {
        drop_order();
        ipg_dev_free(refill_dev, 64);
        ipg_dev_free(refill_stage, refill_stage_bytes);
        if (refill_host) cudaFreeHost(refill_host);
        if (refill_st) cudaStreamDestroy(refill_st);
        if (owns_out) {
            ipg_dev_free(row, row_bytes);
            ipg_dev_free(adj, adj_bytes);
            ipg_dev_free(wgt, wgt_bytes);
        }
        ipg_dev_free(in_row, in_row_bytes);
        ipg_dev_free(in_adj, in_adj_bytes);
        ipg_dev_free(in_wgt, in_wgt_bytes);
        for (auto& b : bins) ipg_dev_free(b.lists, b.bytes);
    }
};

static uint32_t grid_for(uint64_t n, int threads, int per_sm = 8)
{
    uint64_t blocks = (n + threads - 1) / threads;
    uint64_t cap = (uint64_t)ipg_sm_count() * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    return (uint32_t)blocks;
}

// ---------------------------------------------------------------------------
// Kernels: layout conversion, validation, degree statistics
// ---------------------------------------------------------------------------
template <class I>
__global__ void k_widen_idx(const I* __restrict__ idx, uint64_t V, uint64_t E, uint64_t* __restrict__ row)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= V; i += (uint64_t)gridDim.x * blockDim.x)
        row[i] = (i < V) ? (uint64_t)idx[i] : E;
}

// err bits: 1 row not monotone / row[0] != 0 / row[V-1] > E, 2 id >= V
__global__ void k_check_row(const uint64_t* __restrict__ row, uint64_t V, uint32_t* err)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x) {
        if (row[i] > row[i + 1] || (i == 0 && row[0] != 0)) atomicOr(err, 1u);
    }
}

template <class T>
__global__ void k_check_ids(const T* __restrict__ adj, uint64_t E, uint64_t V, uint32_t* err)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < E; i += (uint64_t)gridDim.x * blockDim.x)
        if ((uint64_t)adj[i] >= V) atomicOr(err, 2u);
}

__global__ void k_max_degree(const uint64_t* __restrict__ row, uint64_t V, unsigned long long* out)
{
    unsigned long long m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < V; i += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long d = row[i + 1] - row[i];
        m = d > m ? d : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_down_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

static int finish_graph_stats(ipg_graph* g, cudaStream_t st)
{
    g->v.max_out_degree = 0;
    g->v.max_in_degree = 0;
    if (g->v.V == 0) return IPG_OK;
    DevBuf tmp;
    IPG_TRY(tmp.alloc(sizeof(unsigned long long) * 2));
    IPG_CUDA(cudaMemsetAsync(tmp.p, 0, 16, st));
    k_max_degree<<<grid_for(g->v.V, 256), 256, 0, st>>>(g->v.d_row, g->v.V, tmp.as<unsigned long long>());
    if (g->v.has_in && g->v.d_in_row != g->v.d_row)
        k_max_degree<<<grid_for(g->v.V, 256), 256, 0, st>>>(g->v.d_in_row, g->v.V, tmp.as<unsigned long long>() + 1);
    IPG_CUDA(cudaGetLastError());
    unsigned long long h[2];
    IPG_CUDA(cudaMemcpyAsync(h, tmp.p, 16, cudaMemcpyDeviceToHost, st));
    IPG_CUDA(cudaStreamSynchronize(st));
    g->v.max_out_degree = h[0];
    g->v.max_in_degree = (g->v.has_in && g->v.d_in_row != g->v.d_row) ? h[1] : h[0];
    return IPG_OK;
}

static int validate_graph(ipg_graph* g, cudaStream_t st)
{
    if (g->v.V == 0) return IPG_OK;
    DevBuf err;
    IPG_TRY(err.alloc(4));
    IPG_CUDA(cudaMemsetAsync(err.p, 0, 4, st));
    k_check_row<<<grid_for(g->v.V, 256), 256, 0, st>>>(g->v.d_row, g->v.V, err.as<uint32_t>());
    if (g->v.E) {
        if (g->v.id_bytes == 4)
            k_check_ids<<<grid_for(g->v.E, 256), 256, 0, st>>>((const uint32_t*)g->v.d_adj, g->v.E, g->v.V, err.as<uint32_t>());
        else
            k_check_ids<<<grid_for(g->v.E, 256), 256, 0, st>>>((const uint64_t*)g->v.d_adj, g->v.E, g->v.V, err.as<uint32_t>());
    }
    IPG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    IPG_CUDA(cudaMemcpyAsync(&h, err.p, 4, cudaMemcpyDeviceToHost, st));
    IPG_CUDA(cudaStreamSynchronize(st));
    if (h & 1) return fail(IPG_EIO, "malformed offsets: row starts must begin at 0, be non-decreasing and not exceed E");
    if (h & 2) return fail(IPG_EIO, "malformed adjacency: a neighbour id is >= the vertex count");
    return IPG_OK;
}

// ---------------------------------------------------------------------------
// In-CSR (CSC) build: stable sort of edges by destination.  The edge order
// is the CSR order, i.e. by increasing source, so the stable sort yields the
// reference's mirror order (iPregel_postamble.h:429-487).
// ---------------------------------------------------------------------------
__global__ void k_edge_src(const uint64_t* __restrict__ row, uint64_t V, uint64_t E, uint32_t* __restrict__ src)
{
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = V;  // largest v with row[v] <= e, row[v+1] > e
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) >> 1;
            if (row[mid] <= e) lo = mid; else hi = mid;
        }
        src[e] = (uint32_t)lo;
    }
}

template <class T>
__global__ void k_copy_ids(const T* __restrict__ in, uint64_t n, uint32_t* __restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)in[i];
}

__global__ void k_iota(uint32_t* __restrict__ out, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)i;
}

__global__ void k_fill_u64(uint64_t* __restrict__ out, uint64_t n, uint64_t v)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = v;
}

// row[v] = first index e with key(e) >= v, given keys sorted; row pre-filled with E.
template <class K>
__global__ void k_row_from_sorted(const K* __restrict__ keys, uint64_t E, int shift, uint64_t* __restrict__ row)
{
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = (uint64_t)(keys[e] >> shift);
        int64_t ps = e ? (int64_t)(keys[e - 1] >> shift) : -1;
        for (int64_t v = ps + 1; v <= (int64_t)s; v++) row[v] = e;
    }
}

template <class T>
__global__ void k_gather_ids(const uint32_t* __restrict__ perm, uint64_t n, const uint32_t* __restrict__ src,
                             T* __restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (T)src[perm[i]];
}

__global__ void k_gather_bytes(const uint32_t* __restrict__ perm, uint64_t n, const uint8_t* __restrict__ src,
                               uint8_t* __restrict__ out, int w)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        for (int b = 0; b < w; b++) out[i * w + b] = src[(uint64_t)perm[i] * w + b];
}

static int bits_for(uint64_t n)
{
    int b = 1;
    while (b < 64 && (1ULL << b) < n) b++;
    return b;
}

// ---- degree order ----
// occ[v] = occurrences of v among the edges e = 0, s, 2s, ... of the rows (its
// in-degree over the stored rows, sampled every s-th edge)
template <class T>
__global__ void k_occurrences(const T* __restrict__ adj, uint64_t E, uint64_t s, uint32_t* __restrict__ occ)
{
    const uint64_t n = (E + s - 1) / s;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&occ[(uint64_t)adj[i * s]], 1u);
}

// occ[v] = length of row v: the occurrences of v in the rows when every edge
// has its reverse (symmetric rows), or its in-degree when row = the in-lists
__global__ void k_occurrences_from_rows(const uint64_t* __restrict__ row, uint64_t V, uint32_t* __restrict__ occ)
{
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t d = row[v + 1] - row[v];
        occ[v] = d < 0xFFFFFFFFull ? (uint32_t)d : 0xFFFFFFFFu;
    }
}

__global__ void k_invert_perm(const uint32_t* __restrict__ old_of_new, uint64_t V, uint32_t* __restrict__ new_of_old)
{
    for (uint64_t n = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; n < V; n += (uint64_t)gridDim.x * blockDim.x)
        new_of_old[old_of_new[n]] = (uint32_t)n;
}

// deg[n] = length of row old_of_new[n], deg[V] = 0 (an exclusive scan makes the new rows)
__global__ void k_perm_degrees(const uint64_t* __restrict__ row, const uint32_t* __restrict__ old_of_new, uint64_t V,
                               uint64_t* __restrict__ deg)
{
    for (uint64_t n = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; n <= V; n += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t d = 0;
        if (n < V) {
            const uint64_t o = old_of_new[n];
            d = row[o + 1] - row[o];
        }
        deg[n] = d;
    }
}

// Row n of the copy = row old_of_new[n] of the source, in the same edge order,
// each neighbour id renamed by new_of_old.  The copy's edges are cut into
// tiles of ORD_TILE; tile_lo[t] is the row holding the tile's first edge.
#define ORD_TILE 2048
#define ORD_TILE_ROWS 2048
#define ORD_PER_THREAD (ORD_TILE / 256) /* k_perm_rows runs 256 threads */

__global__ void k_tile_rows(const uint64_t* __restrict__ nrow, uint64_t V, uint64_t tiles, uint32_t* __restrict__ tile_lo)
{
    for (uint64_t n = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; n < V; n += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t a = nrow[n], b = nrow[n + 1];
        for (uint64_t t = (a + ORD_TILE - 1) / ORD_TILE; t * ORD_TILE < b; t++) tile_lo[t] = (uint32_t)n;
        if (n == V - 1) tile_lo[tiles] = (uint32_t)n;
    }
}

// A CTA per tile: the rows the tile touches staged in shared memory (copy
// and source starts) with the row of every tile position (each non-empty
// row marks its first position, a block-wide running max fills the rest);
// reads follow the source rows, writes are coalesced.  A tile of more rows
// than the stage holds (long runs of empty rows) searches the copy's row
// starts instead.
template <class T, class W>
__global__ void __launch_bounds__(256) k_perm_rows(const uint64_t* __restrict__ row, const T* __restrict__ adj,
                                                   const W* __restrict__ wgt, const uint32_t* __restrict__ old_of_new,
                                                   const uint32_t* __restrict__ new_of_old, uint64_t E,
                                                   const uint64_t* __restrict__ nrow,
                                                   const uint32_t* __restrict__ tile_lo, T* __restrict__ nadj,
                                                   W* __restrict__ nwgt)
{
    __shared__ uint64_t s_dst[ORD_TILE_ROWS + 1];
    __shared__ uint64_t s_src[ORD_TILE_ROWS];
    __shared__ uint16_t s_rowof[ORD_TILE];
    __shared__ uint32_t s_warp[8];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t tiles = (E + ORD_TILE - 1) / ORD_TILE;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t p0 = t * ORD_TILE, p1 = (p0 + ORD_TILE < E) ? p0 + ORD_TILE : E;
        const uint64_t lo = tile_lo[t], cnt = (uint64_t)tile_lo[t + 1] - lo + 1;
        const bool staged = cnt <= ORD_TILE_ROWS;
        if (staged) {
            for (uint64_t i = tid; i <= cnt; i += 256) {
                s_dst[i] = nrow[lo + i];  // lo + cnt <= V: nrow holds V + 1 starts
                if (i < cnt) s_src[i] = row[old_of_new[lo + i]];
            }
#pragma unroll
            for (int j = 0; j < ORD_PER_THREAD; j++) s_rowof[tid * ORD_PER_THREAD + j] = 0;
        }
        __syncthreads();
        if (staged) {
            // row 0 holds p0; every later non-empty row starts inside (p0, p1]
            for (uint64_t i = 1 + tid; i < cnt; i += 256) {
                const uint64_t d = s_dst[i];
                if (s_dst[i + 1] > d && d < p1) s_rowof[d - p0] = (uint16_t)i;
            }
        }
        __syncthreads();
        if (staged) {
            // running max over the positions: ORD_PER_THREAD consecutive ones a thread
            uint32_t m = 0, v[ORD_PER_THREAD];
#pragma unroll
            for (int j = 0; j < ORD_PER_THREAD; j++) {
                const uint32_t x = s_rowof[tid * ORD_PER_THREAD + j];
                m = x > m ? x : m;
                v[j] = m;
            }
            uint32_t inc = m;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= (uint32_t)o) inc = y > inc ? y : inc;
            }
            if (lane == 31) s_warp[warp] = inc;
            uint32_t before = __shfl_up_sync(0xffffffffu, inc, 1);
            if (lane == 0) before = 0;
            __syncthreads();
            for (uint32_t w = 0; w < warp; w++) before = s_warp[w] > before ? s_warp[w] : before;
#pragma unroll
            for (int j = 0; j < ORD_PER_THREAD; j++)
                s_rowof[tid * ORD_PER_THREAD + j] = (uint16_t)(v[j] > before ? v[j] : before);
        }
        __syncthreads();
        // a thread's ORD_PER_THREAD edges: every source position first, then
        // every load, then every store (independent loads in flight together)
        uint64_t src[ORD_PER_THREAD];
#pragma unroll
        for (int k = 0; k < ORD_PER_THREAD; k++) {
            const uint64_t p = p0 + tid + (uint64_t)k * 256;
            src[k] = ~0ULL;
            if (p < p1) {
                if (staged) {
                    const uint32_t a = s_rowof[p - p0];
                    src[k] = s_src[a] + (p - s_dst[a]);
                } else {
                    // the last row of [lo, lo + cnt) with start <= p holds p
                    uint64_t a = 0, b = cnt;
                    while (b - a > 1) {
                        const uint64_t m = (a + b) >> 1;
                        if (nrow[lo + m] <= p) a = m;
                        else b = m;
                    }
                    src[k] = row[old_of_new[lo + a]] + (p - nrow[lo + a]);
                }
            }
        }
        T u[ORD_PER_THREAD];
        W w[ORD_PER_THREAD];
#pragma unroll
        for (int k = 0; k < ORD_PER_THREAD; k++) {
            u[k] = src[k] != ~0ULL ? adj[src[k]] : (T)0;
            w[k] = (wgt && src[k] != ~0ULL) ? wgt[src[k]] : (W)0;
        }
        uint32_t r[ORD_PER_THREAD];
#pragma unroll
        for (int k = 0; k < ORD_PER_THREAD; k++) r[k] = src[k] != ~0ULL ? new_of_old[(uint64_t)u[k]] : 0u;
#pragma unroll
        for (int k = 0; k < ORD_PER_THREAD; k++) {
            const uint64_t p = p0 + tid + (uint64_t)k * 256;
            if (src[k] != ~0ULL) {
                nadj[p] = (T)r[k];
                if (wgt) nwgt[p] = w[k];
            }
        }
        __syncthreads();
    }
}

extern "C" int ipg_graph_build_in(ipg_graph* g)
{
    if (!g) return fail(IPG_EINVAL, "ipg_graph_build_in: null graph");
    if (g->v.has_in) return IPG_OK;
    if (!g->v.directed) {
        g->v.has_in = 1;
        g->v.d_in_row = g->v.d_row;
        g->v.d_in_adj = g->v.d_adj;
        g->v.d_in_wgt = g->v.d_wgt;
        return IPG_OK;
    }
    const uint64_t V = g->v.V, E = g->v.E;
    if (E >= (1ULL << 32) || V >= (1ULL << 32))
        return fail(IPG_EINVAL, "in-CSR build supports fewer than 2^32 vertices and edges");
    cudaStream_t st = 0;
    IPG_TRY(ipg_dev_alloc(&g->in_row, (V + 1) * 8));
    g->in_row_bytes = (V + 1) * 8;
    IPG_TRY(ipg_dev_alloc(&g->in_adj, (E ? E : 1) * (uint64_t)g->v.id_bytes));
    g->in_adj_bytes = (E ? E : 1) * (uint64_t)g->v.id_bytes;
    if (g->v.d_wgt) {
        IPG_TRY(ipg_dev_alloc(&g->in_wgt, (E ? E : 1) * (uint64_t)g->v.weight_bytes));
        g->in_wgt_bytes = (E ? E : 1) * (uint64_t)g->v.weight_bytes;
    }
    k_fill_u64<<<grid_for(V + 1, 256), 256, 0, st>>>((uint64_t*)g->in_row, V + 1, E);
    if (E) {
        DevBuf keys, keys_alt, vals, vals_alt, src, temp;
        IPG_TRY(keys.alloc(E * 4));
        IPG_TRY(keys_alt.alloc(E * 4));
        IPG_TRY(vals.alloc(E * 4));
        IPG_TRY(vals_alt.alloc(E * 4));
        IPG_TRY(src.alloc(E * 4));
        if (g->v.id_bytes == 4)
            k_copy_ids<<<grid_for(E, 256), 256, 0, st>>>((const uint32_t*)g->v.d_adj, E, keys.as<uint32_t>());
        else
            k_copy_ids<<<grid_for(E, 256), 256, 0, st>>>((const uint64_t*)g->v.d_adj, E, keys.as<uint32_t>());
        k_iota<<<grid_for(E, 256), 256, 0, st>>>(vals.as<uint32_t>(), E);
        k_edge_src<<<grid_for(E, 256), 256, 0, st>>>(g->v.d_row, V, E, src.as<uint32_t>());
        IPG_CUDA(cudaGetLastError());
        cub::DoubleBuffer<uint32_t> dk(keys.as<uint32_t>(), keys_alt.as<uint32_t>());
        cub::DoubleBuffer<uint32_t> dv(vals.as<uint32_t>(), vals_alt.as<uint32_t>());
        size_t tb = 0;
        int endb = bits_for(V);
        IPG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, (int)E, 0, endb, st));
        IPG_TRY(temp.alloc(tb));
        IPG_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, tb, dk, dv, (int)E, 0, endb, st));
        k_row_from_sorted<<<grid_for(E, 256), 256, 0, st>>>(dk.Current(), E, 0, (uint64_t*)g->in_row);
        if (g->v.id_bytes == 4)
            k_gather_ids<<<grid_for(E, 256), 256, 0, st>>>(dv.Current(), E, src.as<uint32_t>(), (uint32_t*)g->in_adj);
        else
            k_gather_ids<<<grid_for(E, 256), 256, 0, st>>>(dv.Current(), E, src.as<uint32_t>(), (uint64_t*)g->in_adj);
        if (g->v.d_wgt)
            k_gather_bytes<<<grid_for(E, 256), 256, 0, st>>>(dv.Current(), E, (const uint8_t*)g->v.d_wgt,
                                                             (uint8_t*)g->in_wgt, g->v.weight_bytes);
        IPG_CUDA(cudaGetLastError());
        IPG_CUDA(cudaStreamSynchronize(st));
    }
    IPG_CUDA(cudaStreamSynchronize(st));
    g->v.has_in = 1;
    g->v.d_in_row = (const uint64_t*)g->in_row;
    g->v.d_in_adj = g->in_adj;
    g->v.d_in_wgt = g->in_wgt;
    g->v.device_bytes += g->in_row_bytes + g->in_adj_bytes + g->in_wgt_bytes;
    return finish_graph_stats(g, st);
}

// ---------------------------------------------------------------------------
// Construction from host buffers / files
// ---------------------------------------------------------------------------
static int alloc_out(ipg_graph* g, uint64_t V, uint64_t E, int id_bytes, int weight_bytes)
{
    g->row_bytes = (V + 1) * 8;
    g->adj_bytes = (E ? E : 1) * (uint64_t)id_bytes;
    IPG_TRY(ipg_dev_alloc(&g->row, g->row_bytes));
    IPG_TRY(ipg_dev_alloc(&g->adj, g->adj_bytes));
    if (weight_bytes) {
        g->wgt_bytes = (E ? E : 1) * (uint64_t)weight_bytes;
        IPG_TRY(ipg_dev_alloc(&g->wgt, g->wgt_bytes));
    }
    g->v.V = V;
    g->v.E = E;
    g->v.id_bytes = id_bytes;
    g->v.weight_bytes = weight_bytes;
    g->v.d_row = (const uint64_t*)g->row;
    g->v.d_adj = g->adj;
    g->v.d_wgt = g->wgt;
    g->v.device_bytes = g->row_bytes + g->adj_bytes + g->wgt_bytes;
    return IPG_OK;
}

static int upload_idx(ipg_graph* g, const void* idx_dev_or_host, int idx_bytes, bool host, cudaStream_t st)
{
    const uint64_t V = g->v.V, E = g->v.E;
    DevBuf raw;
    const void* src = idx_dev_or_host;
    if (host && V) {
        IPG_TRY(raw.alloc(V * (uint64_t)idx_bytes));
        IPG_CUDA(cudaMemcpyAsync(raw.p, idx_dev_or_host, V * (uint64_t)idx_bytes, cudaMemcpyHostToDevice, st));
        src = raw.p;
    }
    uint64_t* row = (uint64_t*)g->row;
    switch (idx_bytes) {
    case 8: k_widen_idx<<<grid_for(V + 1, 256), 256, 0, st>>>((const uint64_t*)src, V, E, row); break;
    case 4: k_widen_idx<<<grid_for(V + 1, 256), 256, 0, st>>>((const uint32_t*)src, V, E, row); break;
    case 2: k_widen_idx<<<grid_for(V + 1, 256), 256, 0, st>>>((const uint16_t*)src, V, E, row); break;
    case 1: k_widen_idx<<<grid_for(V + 1, 256), 256, 0, st>>>((const uint8_t*)src, V, E, row); break;
    default: return fail(IPG_EINVAL, "unsupported offset width %d", idx_bytes);
    }
    IPG_CUDA(cudaGetLastError());
    IPG_CUDA(cudaStreamSynchronize(st));
    return IPG_OK;
}

static int check_widths(int id_bytes, int weight_bytes)
{
    if (id_bytes != 4 && id_bytes != 8) return fail(IPG_EINVAL, "vertex id width must be 4 or 8 bytes, got %d", id_bytes);
    if (weight_bytes != 0 && weight_bytes != 1 && weight_bytes != 2 && weight_bytes != 4 && weight_bytes != 8)
        return fail(IPG_EINVAL, "edge weight width must be 1, 2, 4 or 8 bytes, got %d", weight_bytes);
    return IPG_OK;
}

static int finalize(ipg_graph* g, int need_in, ipg_graph** out)
{
    int r = validate_graph(g, 0);
    if (r == IPG_OK && need_in) r = ipg_graph_build_in(g);
    if (r == IPG_OK) r = finish_graph_stats(g, 0);
    if (r != IPG_OK) {
        delete g;
        return r;
    }
    *out = g;
    return IPG_OK;
}

// ---------------------------------------------------------------------------
// Degree-ordered copy
// ---------------------------------------------------------------------------
template <class T>
static void launch_perm_rows(const uint64_t* row, const void* adj, const void* wgt, int weight_bytes,
                             const uint32_t* old_of_new, const uint32_t* new_of_old, uint64_t E, const uint64_t* nrow,
                             const uint32_t* tile_lo, void* nadj, void* nwgt, cudaStream_t st)
{
    const uint32_t grid = grid_for(E, ORD_TILE);
    const T* a = (const T*)adj;
    T* na = (T*)nadj;
    switch (wgt ? weight_bytes : 0) {
    case 1: k_perm_rows<<<grid, 256, 0, st>>>(row, a, (const uint8_t*)wgt, old_of_new, new_of_old, E, nrow, tile_lo, na, (uint8_t*)nwgt); break;
    case 2: k_perm_rows<<<grid, 256, 0, st>>>(row, a, (const uint16_t*)wgt, old_of_new, new_of_old, E, nrow, tile_lo, na, (uint16_t*)nwgt); break;
    case 4: k_perm_rows<<<grid, 256, 0, st>>>(row, a, (const uint32_t*)wgt, old_of_new, new_of_old, E, nrow, tile_lo, na, (uint32_t*)nwgt); break;
    case 8: k_perm_rows<<<grid, 256, 0, st>>>(row, a, (const uint64_t*)wgt, old_of_new, new_of_old, E, nrow, tile_lo, na, (uint64_t*)nwgt); break;
    default: k_perm_rows<<<grid, 256, 0, st>>>(row, a, (const uint8_t*)nullptr, old_of_new, new_of_old, E, nrow, tile_lo, na, (uint8_t*)nullptr); break;
    }
}

// New rows (degree scan) and their edges, for the out- or the in-CSR.
static int perm_csr(const ipg_graph* g, const uint64_t* row, const void* adj, const void* wgt, uint64_t* nrow,
                    void* nadj, void* nwgt, const uint32_t* old_of_new, const uint32_t* new_of_old,
                    uint64_t* deg, uint32_t* tile_lo, void* temp, size_t temp_bytes, cudaStream_t st)
{
    const uint64_t V = g->v.V, E = g->v.E;
    k_perm_degrees<<<grid_for(V + 1, 256), 256, 0, st>>>(row, old_of_new, V, deg);
    size_t tb = temp_bytes;
    IPG_CUDA(cub::DeviceScan::ExclusiveSum(temp, tb, deg, nrow, (int)(V + 1), st));
    if (E && V) {
        const uint64_t tiles = (E + ORD_TILE - 1) / ORD_TILE;
        k_tile_rows<<<grid_for(V, 256), 256, 0, st>>>(nrow, V, tiles, tile_lo);
        if (g->v.id_bytes == 4)
            launch_perm_rows<uint32_t>(row, adj, wgt, g->v.weight_bytes, old_of_new, new_of_old, E, nrow, tile_lo,
                                       nadj, nwgt, st);
        else
            launch_perm_rows<uint64_t>(row, adj, wgt, g->v.weight_bytes, old_of_new, new_of_old, E, nrow, tile_lo,
                                       nadj, nwgt, st);
    }
    IPG_CUDA(cudaGetLastError());
    return IPG_OK;
}

static uint64_t align256(uint64_t x) { return (x + 255) & ~255ULL; }

// Every s-th edge is counted for the order: 1 (every edge) unless
// IPG_ORDER_SAMPLE sets s.  On undirected R-MAT scale 24 a sample of every
// 8th edge took 1.2 instead of 5.3 ms, but ordered the many low-degree
// vertices by noise and left CC + SSSP 6 % slower than exact counts.
static uint64_t ord_sample_stride()
{
    const char* env = getenv("IPG_ORDER_SAMPLE");
    const uint64_t s = (env && *env) ? strtoull(env, nullptr, 10) : 1;
    return s ? s : 1;
}

extern "C" int ipg_graph_degree_order(ipg_graph* g, int need_in, ipg_order* out)
{
    if (!g || !out) return fail(IPG_EINVAL, "ipg_graph_degree_order: null argument");
    memset(out, 0, sizeof *out);
    if (g->bad) return fail(IPG_EINVAL, "the graph's contents failed validation at its last refill");
    const uint64_t V = g->v.V, E = g->v.E;
    if (V >= (1ULL << 31)) return fail(IPG_EINVAL, "ipg_graph_degree_order: supports fewer than 2^31 vertices");
    if (need_in && !g->v.has_in) IPG_TRY(ipg_graph_build_in(g));
    const bool with_in = g->v.has_in != 0;
    const bool in_alias = with_in && g->v.d_in_row == g->v.d_row;
    // scratch: degrees (the occurrence counts before the sort), sorted
    // counts, ids, the sort / scan temporaries, the tile rows of the copy
    const uint64_t deg_bytes = align256((V + 1) * 8), map_bytes = (V ? V : 1) * 4;
    size_t sort_tb = 0, scan_tb = 0;
    IPG_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_tb, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                                       (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)V, 0, 32, 0));
    IPG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_tb, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                           (int)(V + 1), 0));
    const uint64_t temp_bytes = align256(std::max(sort_tb, scan_tb) + 1);
    const uint64_t tile_bytes = align256(((E + ORD_TILE - 1) / ORD_TILE + 1) * 4);
    const uint64_t scratch_bytes = deg_bytes + 2 * align256(map_bytes) + temp_bytes + tile_bytes;

    // The copy is only ever dropped when the graph's shape or meaning
    // changed (set_directed bumps the generation, so engines attached to it
    // re-attach first); in-lists asked for later are added to it in place.
    ipg_graph* o = g->ord;
    const bool shape = o && o->v.V == V && o->v.E == E && o->v.id_bytes == g->v.id_bytes &&
                       o->v.weight_bytes == g->v.weight_bytes && o->v.directed == g->v.directed &&
                       g->ord_scratch_bytes >= scratch_bytes;
    if (!shape) {
        g->drop_order();
        o = new ipg_graph();
        o->v.directed = g->v.directed;
        int r = alloc_out(o, V, E, g->v.id_bytes, g->v.weight_bytes);
        g->ord = o;
        g->ord_map_bytes = map_bytes;  // sizes first: drop_order frees what was allocated
        g->ord_scratch_bytes = scratch_bytes;
        if (r == IPG_OK) r = ipg_dev_alloc(&g->ord_old_of_new, map_bytes);
        if (r == IPG_OK) r = ipg_dev_alloc(&g->ord_new_of_old, map_bytes);
        if (r == IPG_OK) r = ipg_dev_alloc(&g->ord_scratch, scratch_bytes);
        if (r != IPG_OK) {
            g->drop_order();
            return r;
        }
    }
    if (with_in && !in_alias && !o->in_row) {
        int r = IPG_OK;
        o->in_row_bytes = (V + 1) * 8;
        o->in_adj_bytes = (E ? E : 1) * (uint64_t)g->v.id_bytes;
        r = ipg_dev_alloc(&o->in_row, o->in_row_bytes);
        if (r == IPG_OK) r = ipg_dev_alloc(&o->in_adj, o->in_adj_bytes);
        if (r == IPG_OK && g->v.d_in_wgt) {
            o->in_wgt_bytes = (E ? E : 1) * (uint64_t)g->v.weight_bytes;
            r = ipg_dev_alloc(&o->in_wgt, o->in_wgt_bytes);
        }
        if (r != IPG_OK) {  // the copy stays as it was, without in-lists
            ipg_dev_free(o->in_row, o->in_row_bytes);
            ipg_dev_free(o->in_adj, o->in_adj_bytes);
            ipg_dev_free(o->in_wgt, o->in_wgt_bytes);
            o->in_row = o->in_adj = o->in_wgt = nullptr;
            o->in_row_bytes = o->in_adj_bytes = o->in_wgt_bytes = 0;
            return r;
        }
        o->v.device_bytes += o->in_row_bytes + o->in_adj_bytes + o->in_wgt_bytes;
    }
    cudaStream_t st = 0;
    uint32_t* old_of_new = (uint32_t*)g->ord_old_of_new;
    uint32_t* new_of_old = (uint32_t*)g->ord_new_of_old;
    char* sc = (char*)g->ord_scratch;
    uint64_t* deg = (uint64_t*)sc;
    uint32_t* occ_sorted = (uint32_t*)(sc + deg_bytes);
    uint32_t* iota = (uint32_t*)(sc + deg_bytes + align256(map_bytes));
    void* temp = sc + deg_bytes + 2 * align256(map_bytes);
    uint32_t* tile_lo = (uint32_t*)(sc + deg_bytes + 2 * align256(map_bytes) + temp_bytes);
    const bool fresh = g->ord_valid && g->ord_generation == g->generation;
    const bool add_in = with_in && !o->v.has_in;
    if (!fresh) {
        g->ord_valid = false;
        o->v.has_in = 0;  // rebuilt below with the rows
        for (auto& b : o->bins) {  // derived from the old contents
            ipg_dev_free(b.lists, b.bytes);
            b = ipg_graph::BinCache();
        }
        if (V) {
            uint32_t* occ = (uint32_t*)deg;
            const uint64_t s = ord_sample_stride();
            if (s == 1 && g->v.symmetric) {
                k_occurrences_from_rows<<<grid_for(V, 256), 256, 0, st>>>(g->v.d_row, V, occ);
            } else if (s == 1 && with_in && !in_alias) {
                k_occurrences_from_rows<<<grid_for(V, 256), 256, 0, st>>>(g->v.d_in_row, V, occ);
            } else {
                IPG_CUDA(cudaMemsetAsync(occ, 0, V * 4, st));
                if (E && g->v.id_bytes == 4)
                    k_occurrences<<<grid_for(E / s + 1, 256), 256, 0, st>>>((const uint32_t*)g->v.d_adj, E, s, occ);
                else if (E)
                    k_occurrences<<<grid_for(E / s + 1, 256), 256, 0, st>>>((const uint64_t*)g->v.d_adj, E, s, occ);
            }
            k_iota<<<grid_for(V, 256), 256, 0, st>>>(iota, V);
            IPG_CUDA(cudaGetLastError());
            // descending occurrences; the sort is stable, so ties keep ascending ids
            size_t tb = temp_bytes;
            const int end_bit = E + 1 >= (1ULL << 32) ? 32 : bits_for(E + 1);
            IPG_CUDA(cub::DeviceRadixSort::SortPairsDescending(temp, tb, occ, occ_sorted, iota, old_of_new, (int)V, 0,
                                                               end_bit, st));
            k_invert_perm<<<grid_for(V, 256), 256, 0, st>>>(old_of_new, V, new_of_old);
            IPG_CUDA(cudaGetLastError());
        }
        IPG_TRY(perm_csr(g, g->v.d_row, g->v.d_adj, g->v.d_wgt, (uint64_t*)o->row, o->adj, o->wgt, old_of_new,
                         new_of_old, deg, tile_lo, temp, temp_bytes, st));
    }
    if ((!fresh || add_in) && with_in) {
        if (!in_alias)
            IPG_TRY(perm_csr(g, g->v.d_in_row, g->v.d_in_adj, g->v.d_in_wgt, (uint64_t*)o->in_row, o->in_adj,
                             o->in_wgt, old_of_new, new_of_old, deg, tile_lo, temp, temp_bytes, st));
        o->v.d_in_row = in_alias ? o->v.d_row : (const uint64_t*)o->in_row;
        o->v.d_in_adj = in_alias ? o->v.d_adj : o->in_adj;
        o->v.d_in_wgt = in_alias ? o->v.d_wgt : o->in_wgt;
    }
    IPG_CUDA(cudaStreamSynchronize(st));
    if (with_in) o->v.has_in = 1;
    o->v.max_out_degree = g->v.max_out_degree;  // a renaming keeps every degree
    o->v.max_in_degree = g->v.max_in_degree;
    o->v.symmetric = g->v.symmetric;
    g->ord_generation = g->generation;
    g->ord_valid = true;
    out->graph = o;
    out->d_old_of_new = (const uint32_t*)g->ord_old_of_new;
    out->d_new_of_old = (const uint32_t*)g->ord_new_of_old;
    return IPG_OK;
}

extern "C" int ipg_graph_from_host(uint64_t V, uint64_t E, const void* idx, int idx_bytes, const void* adj,
                                   int id_bytes, const void* wgt, int weight_bytes, int directed, int need_in,
                                   ipg_graph** out)
{
    if (!out) return fail(IPG_EINVAL, "ipg_graph_from_host: null output");
    *out = nullptr;
    if (!wgt && E) weight_bytes = 0; /* an edgeless graph may still be declared weighted */
    IPG_TRY(check_widths(id_bytes, weight_bytes));
    if ((V && !idx) || (E && !adj)) return fail(IPG_EINVAL, "ipg_graph_from_host: null buffer");
    if (V >= (1ULL << 32)) return fail(IPG_EINVAL, "at most 2^32-1 vertices are supported");
    ipg_graph* g = new ipg_graph();
    g->v.directed = directed;
    int r = alloc_out(g, V, E, id_bytes, weight_bytes);
    if (r == IPG_OK) r = upload_idx(g, idx, idx_bytes, true, 0);
    if (r == IPG_OK && E) {
        cudaError_t e = cudaMemcpy(g->adj, adj, E * (uint64_t)id_bytes, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && weight_bytes)
            e = cudaMemcpy(g->wgt, wgt, E * (uint64_t)weight_bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) r = fail(IPG_ECUDA, "upload failed: %s", cudaGetErrorString(e));
    }
    if (r != IPG_OK) {
        delete g;
        return r;
    }
    return finalize(g, need_in, out);
}

// Everything on the graph's own non-blocking stream, synchronising only that
// stream, with buffers made at the first call: a refill allocates nothing
// and waits for no other work on the device, so it can run on one thread
// while kernels of another graph run on another.
extern "C" int ipg_graph_refill_host(ipg_graph* g, const void* idx, int idx_bytes, const void* adj, const void* wgt)
{
    if (!g) return fail(IPG_EINVAL, "ipg_graph_refill_host: null graph");
    if (!g->owns_out) return fail(IPG_EINVAL, "ipg_graph_refill_host: the graph wraps buffers it does not own");
    const uint64_t V = g->v.V, E = g->v.E;
    if ((V && !idx) || (E && !adj) || (E && g->v.weight_bytes && !wgt))
        return fail(IPG_EINVAL, "ipg_graph_refill_host: null buffer");
    if (idx_bytes != 1 && idx_bytes != 2 && idx_bytes != 4 && idx_bytes != 8)
        return fail(IPG_EINVAL, "unsupported offset width %d", idx_bytes);
    if (!g->refill_st) IPG_CUDA(cudaStreamCreateWithFlags(&g->refill_st, cudaStreamNonBlocking));
    if (!g->refill_dev) IPG_TRY(ipg_dev_alloc(&g->refill_dev, 64));
    if (!g->refill_host) IPG_CUDA(cudaHostAlloc((void**)&g->refill_host, 64, cudaHostAllocDefault));
    if (idx_bytes != 8 && g->refill_stage_bytes < V * (uint64_t)idx_bytes) {
        ipg_dev_free(g->refill_stage, g->refill_stage_bytes);
        g->refill_stage = nullptr;
        g->refill_stage_bytes = 0;
        IPG_TRY(ipg_dev_alloc(&g->refill_stage, V * (uint64_t)idx_bytes));
        g->refill_stage_bytes = V * (uint64_t)idx_bytes;
    }
    // From here on the old contents are being replaced: engines attached to
    // them refuse to run (generation), and so does any engine while the new
    // contents are not validated (bad).
    g->generation++;
    g->bad = true;
    // derived data of the old contents
    for (auto& b : g->bins) {
        ipg_dev_free(b.lists, b.bytes);
        b = ipg_graph::BinCache();
    }
    g->v.symmetric = 0;
    const bool own_in = g->in_row != nullptr;
    if (own_in) {
        g->v.device_bytes -= g->in_row_bytes + g->in_adj_bytes + g->in_wgt_bytes;
        ipg_dev_free(g->in_row, g->in_row_bytes);
        ipg_dev_free(g->in_adj, g->in_adj_bytes);
        ipg_dev_free(g->in_wgt, g->in_wgt_bytes);
        g->in_row = g->in_adj = g->in_wgt = nullptr;
        g->in_row_bytes = g->in_adj_bytes = g->in_wgt_bytes = 0;
        g->v.has_in = 0;
        g->v.d_in_row = nullptr;
        g->v.d_in_adj = nullptr;
        g->v.d_in_wgt = nullptr;
    }
    cudaStream_t st = g->refill_st;
    uint64_t* row = (uint64_t*)g->row;
    uint64_t* h = g->refill_host;  // [0] = E for row[V]; [1..3] read back
    uint32_t* err = (uint32_t*)g->refill_dev;
    unsigned long long* maxdeg = (unsigned long long*)((char*)g->refill_dev + 8);
    h[0] = E;
    if (V) {
        if (idx_bytes == 8) {
            IPG_CUDA(cudaMemcpyAsync(row, idx, V * 8, cudaMemcpyHostToDevice, st));
        } else {
            IPG_CUDA(cudaMemcpyAsync(g->refill_stage, idx, V * (uint64_t)idx_bytes, cudaMemcpyHostToDevice, st));
            const void* src = g->refill_stage;
            switch (idx_bytes) {
            case 4: k_widen_idx<<<grid_for(V + 1, 256), 256, 0, st>>>((const uint32_t*)src, V, E, row); break;
            case 2: k_widen_idx<<<grid_for(V + 1, 256), 256, 0, st>>>((const uint16_t*)src, V, E, row); break;
            default: k_widen_idx<<<grid_for(V + 1, 256), 256, 0, st>>>((const uint8_t*)src, V, E, row); break;
            }
        }
    }
    IPG_CUDA(cudaMemcpyAsync(row + V, &h[0], 8, cudaMemcpyHostToDevice, st));
    if (E) {
        IPG_CUDA(cudaMemcpyAsync(g->adj, adj, E * (uint64_t)g->v.id_bytes, cudaMemcpyHostToDevice, st));
        if (g->v.weight_bytes)
            IPG_CUDA(cudaMemcpyAsync(g->wgt, wgt, E * (uint64_t)g->v.weight_bytes, cudaMemcpyHostToDevice, st));
    }
    IPG_CUDA(cudaMemsetAsync(g->refill_dev, 0, 16, st));
    if (V) {
        k_check_row<<<grid_for(V, 256), 256, 0, st>>>(row, V, err);
        k_max_degree<<<grid_for(V, 256), 256, 0, st>>>(row, V, maxdeg);
    }
    if (E) {
        if (g->v.id_bytes == 4)
            k_check_ids<<<grid_for(E, 256), 256, 0, st>>>((const uint32_t*)g->adj, E, V, err);
        else
            k_check_ids<<<grid_for(E, 256), 256, 0, st>>>((const uint64_t*)g->adj, E, V, err);
    }
    IPG_CUDA(cudaGetLastError());
    IPG_CUDA(cudaMemcpyAsync(&h[1], g->refill_dev, 16, cudaMemcpyDeviceToHost, st));
    IPG_CUDA(cudaStreamSynchronize(st));
    const uint32_t bits = (uint32_t)h[1];
    if (bits & 1) return fail(IPG_EIO, "malformed offsets: row starts must begin at 0, be non-decreasing and not exceed E");
    if (bits & 2) return fail(IPG_EIO, "malformed adjacency: a neighbour id is >= the vertex count");
    g->v.max_out_degree = h[2];
    // without an in-CSR the in-degrees are the out-degrees only for a graph
    // whose rows are its in-lists; 0 = unknown, as the loader leaves it
    g->v.max_in_degree = g->v.directed ? 0 : h[2];
    if (own_in) {
        IPG_TRY(ipg_graph_build_in(g));  // allocates: directed graphs only
        IPG_TRY(finish_graph_stats(g, 0));
    }
    g->bad = false;
    return IPG_OK;
}

extern "C" int ipg_graph_contents(const ipg_graph* g, uint64_t* generation, int* valid)
{
    if (!g) return fail(IPG_EINVAL, "ipg_graph_contents: null graph");
    if (generation) *generation = g->generation;
    if (valid) *valid = g->bad ? 0 : 1;
    return IPG_OK;
}

extern "C" int ipg_graph_from_device(uint64_t V, uint64_t E, const uint64_t* d_row, const void* d_adj, int id_bytes,
                                     const void* d_wgt, int weight_bytes, int directed, int need_in, ipg_graph** out)
{
    if (!out) return fail(IPG_EINVAL, "ipg_graph_from_device: null output");
    *out = nullptr;
    if (!d_wgt && E) weight_bytes = 0;
    IPG_TRY(check_widths(id_bytes, weight_bytes));
    if (!d_row || (E && !d_adj)) return fail(IPG_EINVAL, "ipg_graph_from_device: null buffer");
    ipg_graph* g = new ipg_graph();
    g->owns_out = false;
    g->v.V = V;
    g->v.E = E;
    g->v.id_bytes = id_bytes;
    g->v.weight_bytes = weight_bytes;
    g->v.directed = directed;
    g->v.d_row = d_row;
    g->v.d_adj = d_adj;
    g->v.d_wgt = d_wgt;
    return finalize(g, need_in, out);
}

// ---------------------------------------------------------------------------
// Disjoint union of graphs: concatenated CSR with offset tables.
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_offset_copy(const T* __restrict__ src, T* __restrict__ dst, uint64_t n, T add)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[i] + add;
}

extern "C" int ipg_graph_concat(ipg_graph* const* parts, uint32_t count, int directed, int need_in, ipg_graph** out,
                                uint64_t* voff, uint64_t* eoff)
{
    if (!out || (count && !parts)) return fail(IPG_EINVAL, "ipg_graph_concat: null argument");
    *out = nullptr;
    if (count == 0) return fail(IPG_EINVAL, "ipg_graph_concat: no graphs");
    const int id_bytes = parts[0] ? parts[0]->v.id_bytes : 0;
    const int wb = parts[0] ? parts[0]->v.weight_bytes : 0;
    uint64_t V = 0, E = 0;
    for (uint32_t i = 0; i < count; i++) {
        const ipg_graph* p = parts[i];
        if (!p) return fail(IPG_EINVAL, "ipg_graph_concat: graph %u is null", i);
        if (p->v.id_bytes != id_bytes) return fail(IPG_EINVAL, "ipg_graph_concat: graph %u has another id width", i);
        if (p->v.weight_bytes != wb && p->v.E)
            return fail(IPG_EINVAL, "ipg_graph_concat: graph %u has another weight width", i);
        if (voff) voff[i] = V;
        if (eoff) eoff[i] = E;
        V += p->v.V;
        E += p->v.E;
    }
    if (voff) voff[count] = V;
    if (eoff) eoff[count] = E;
    if (id_bytes == 4 && V >= (1ULL << 32)) return fail(IPG_EINVAL, "ipg_graph_concat: more than 2^32-1 vertices");
    ipg_graph* g = new ipg_graph();
    g->v.directed = directed;
    int r = alloc_out(g, V, E, id_bytes, wb);
    uint64_t v0 = 0, e0 = 0;
    for (uint32_t i = 0; i < count && r == IPG_OK; i++) {
        const ipg_graph* p = parts[i];
        const uint64_t n = p->v.V, m = p->v.E;
        if (n)
            k_offset_copy<uint64_t><<<grid_for(n, 256), 256>>>(p->v.d_row, (uint64_t*)g->row + v0, n, e0);
        if (m) {
            if (id_bytes == 4)
                k_offset_copy<uint32_t><<<grid_for(m, 256), 256>>>((const uint32_t*)p->v.d_adj,
                                                                   (uint32_t*)g->adj + e0, m, (uint32_t)v0);
            else
                k_offset_copy<uint64_t><<<grid_for(m, 256), 256>>>((const uint64_t*)p->v.d_adj,
                                                                   (uint64_t*)g->adj + e0, m, v0);
            if (wb) {
                cudaError_t e = cudaMemcpyAsync((char*)g->wgt + e0 * wb, p->v.d_wgt, m * (uint64_t)wb,
                                                cudaMemcpyDeviceToDevice, 0);
                if (e != cudaSuccess) r = fail(IPG_ECUDA, "ipg_graph_concat: %s", cudaGetErrorString(e));
            }
        }
        if (cudaGetLastError() != cudaSuccess) r = fail(IPG_ECUDA, "ipg_graph_concat: copy kernel failed");
        v0 += n;
        e0 += m;
    }
    if (r == IPG_OK) {
        k_fill_u64<<<1, 32>>>((uint64_t*)g->row + V, 1, E);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) r = fail(IPG_ECUDA, "ipg_graph_concat: %s", cudaGetErrorString(e));
    }
    if (r != IPG_OK) {
        delete g;
        return r;
    }
    // symmetric parts give a symmetric union
    bool sym = true;
    for (uint32_t i = 0; i < count; i++) sym = sym && parts[i]->v.symmetric;
    g->v.symmetric = sym ? 1 : 0;
    return finalize(g, need_in, out);
}

// ---------------------------------------------------------------------------
// One CUDA graph holding several applications' superstep loops.
// ---------------------------------------------------------------------------
struct ipg_fused {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

extern "C" void ipg_fused_free(ipg_fused* f)
{
    if (!f) return;
    if (f->exec) cudaGraphExecDestroy(f->exec);
    if (f->graph) cudaGraphDestroy(f->graph);
    for (auto e : f->ev)
        if (e) cudaEventDestroy(e);
    delete f;
}

extern "C" int ipg_fused_create(ipg_fused** out)
{
    if (!out) return fail(IPG_EINVAL, "ipg_fused_create: null output");
    ipg_fused* f = new ipg_fused();
    cudaError_t e = cudaGraphCreate(&f->graph, 0);
    if (e == cudaSuccess) e = cudaEventCreate(&f->ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&f->ev[1]);
    if (e != cudaSuccess) {
        ipg_fused_free(f);
        return fail(IPG_ECUDA, "ipg_fused_create: %s", cudaGetErrorString(e));
    }
    *out = f;
    return IPG_OK;
}

extern "C" void* ipg_fused_graph(ipg_fused* f) { return f ? (void*)f->graph : nullptr; }

extern "C" int ipg_fused_launch(ipg_fused* f, void* stream, double* seconds)
{
    if (!f) return fail(IPG_EINVAL, "ipg_fused_launch: null argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (!f->exec) IPG_CUDA(cudaGraphInstantiate(&f->exec, f->graph, 0));
    IPG_CUDA(cudaEventRecord(f->ev[0], st));
    IPG_CUDA(cudaGraphLaunch(f->exec, st));
    IPG_CUDA(cudaEventRecord(f->ev[1], st));
    IPG_CUDA(cudaEventSynchronize(f->ev[1]));
    float ms = 0.f;
    IPG_CUDA(cudaEventElapsedTime(&ms, f->ev[0], f->ev[1]));
    if (seconds) *seconds = ms * 1e-3;
    return IPG_OK;
}

// Parallel pread of [off, off+bytes) into dst.
static int read_range(int fd, uint64_t off, uint64_t bytes, void* dst)
{
    const unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    std::vector<std::thread> ts;
    std::atomic<int> bad{0};
    const uint64_t per = (bytes + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        uint64_t b0 = t * per, b1 = std::min(bytes, b0 + per);
        if (b0 >= b1) break;
        ts.emplace_back([=, &bad] {
            uint64_t done = b0;
            while (done < b1) {
                ssize_t n = pread(fd, (char*)dst + done, b1 - done, off + done);
                if (n <= 0) {
                    bad = 1;
                    return;
                }
                done += (uint64_t)n;
            }
        });
    }
    for (auto& t : ts) t.join();
    return bad ? -1 : 0;
}

// Streams a file section to the device through two pinned staging buffers.
static int file_to_device(const char* name, uint64_t bytes, void* d_dst)
{
    int fd = open(name, O_RDONLY);
    if (fd < 0) return fail(IPG_EIO, "Cannot open the file \"%s\" in mode \"rb\".", name);
    off_t size = lseek(fd, 0, SEEK_END);
    if (size < 0 || (uint64_t)size < bytes) {
        close(fd);
        return fail(IPG_EIO, "Failed to read %llu bytes from \"%s\" (file holds %lld).",
                    (unsigned long long)bytes, name, (long long)size);
    }
    const uint64_t chunk = 64ULL << 20;
    void* stage[2] = {nullptr, nullptr};
    cudaEvent_t ev[2];
    cudaStream_t st;
    if (cudaHostAlloc(&stage[0], chunk, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&stage[1], chunk, cudaHostAllocDefault) != cudaSuccess) {
        if (stage[0]) cudaFreeHost(stage[0]);
        close(fd);
        cudaGetLastError();
        return fail(IPG_ENOMEM, "pinned staging allocation failed");
    }
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    int r = IPG_OK;
    uint64_t done = 0;
    for (int k = 0; done < bytes; k ^= 1) {
        uint64_t n = std::min(chunk, bytes - done);
        cudaEventSynchronize(ev[k]);
        if (read_range(fd, done, n, stage[k]) != 0) {
            r = fail(IPG_EIO, "Failed to read %llu bytes from \"%s\".", (unsigned long long)n, name);
            break;
        }
        if (cudaMemcpyAsync((char*)d_dst + done, stage[k], n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaEventRecord(ev[k], st) != cudaSuccess) {
            r = fail(IPG_ECUDA, "upload of \"%s\" failed", name);
            break;
        }
        done += n;
    }
    cudaStreamSynchronize(st);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    cudaStreamDestroy(st);
    cudaFreeHost(stage[0]);
    cudaFreeHost(stage[1]);
    close(fd);
    return r;
}

extern "C" int ipg_graph_load(const char* path, int id_bytes, int idx_bytes, int directed, int weighted,
                              int weight_bytes, int need_in, ipg_graph** out)
{
    if (!out || !path) return fail(IPG_EINVAL, "ipg_graph_load: null argument");
    *out = nullptr;
    if (!weighted) weight_bytes = 0;
    IPG_TRY(check_widths(id_bytes, weight_bytes));
    std::string base(path);
    std::string cfg = base + ".config";
    FILE* f = fopen(cfg.c_str(), "r");
    if (!f) return fail(IPG_EIO, "Cannot open the file \"%s\" in mode \"r\".", cfg.c_str());
    unsigned long long V = 0, E = 0;
    // iPregel_postamble.h:257 reads "%zu %zu" and ignores anything after.
    int got = fscanf(f, "%llu %llu", &V, &E);
    fclose(f);
    if (got != 2) return fail(IPG_EIO, "\t- Failure in reading the number of vertices and edges. Abort...");
    if (V >= (1ULL << 32)) return fail(IPG_EINVAL, "at most 2^32-1 vertices are supported");
    ipg_graph* g = new ipg_graph();
    g->v.directed = directed;
    int r = alloc_out(g, V, E, id_bytes, weight_bytes);
    DevBuf rawidx;
    if (r == IPG_OK && V) {
        r = rawidx.alloc(V * (uint64_t)idx_bytes);
        if (r == IPG_OK) r = file_to_device((base + ".idx").c_str(), V * (uint64_t)idx_bytes, rawidx.p);
    }
    if (r == IPG_OK) r = upload_idx(g, rawidx.p, idx_bytes, false, 0);
    if (r == IPG_OK && E) r = file_to_device((base + ".adj").c_str(), E * (uint64_t)id_bytes, g->adj);
    if (r == IPG_OK && E && weight_bytes)
        r = file_to_device((base + ".wgt").c_str(), E * (uint64_t)weight_bytes, g->wgt);
    rawidx.release();
    if (r != IPG_OK) {
        delete g;
        return r;
    }
    return finalize(g, need_in, out);
}

// ---------------------------------------------------------------------------
// Generators.  Keys are (src << vbits) | dst; self-loops become a sentinel
// that sorts last and is dropped after the unique pass.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t d_mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}

static uint64_t h_mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}

__device__ __forceinline__ uint64_t d_draw(uint64_t seedk, uint64_t i, uint32_t l)
{
    return d_mix64(seedk + ((i << 6) | l) * 0x9E3779B97F4A7C15ULL);
}

__global__ void k_gen_rmat(uint64_t M, uint32_t scale, uint64_t ta, uint64_t tab, uint64_t tabc, uint64_t seedk,
                           int undirected, uint64_t sentinel, uint64_t* __restrict__ keys)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < M; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = 0, d = 0;
        for (uint32_t l = 0; l < scale; l++) {
            uint64_t r = d_draw(seedk, i, l) >> 32;
            uint64_t sb = r >= tab;
            uint64_t db = (r >= ta && r < tab) || r >= tabc;
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        bool loop = (s == d);
        if (undirected) {
            keys[2 * i] = loop ? sentinel : (s << scale) | d;
            keys[2 * i + 1] = loop ? sentinel : (d << scale) | s;
        } else {
            keys[i] = loop ? sentinel : (s << scale) | d;
        }
    }
}

__global__ void k_gen_er(uint64_t M, uint64_t n, int vbits, uint64_t seedk, int undirected, uint64_t sentinel,
                         uint64_t* __restrict__ keys)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < M; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = ((d_draw(seedk, i, 0) >> 32) * n) >> 32;
        uint64_t d = ((d_draw(seedk, i, 1) >> 32) * n) >> 32;
        bool loop = (s == d);
        if (undirected) {
            keys[2 * i] = loop ? sentinel : (s << vbits) | d;
            keys[2 * i + 1] = loop ? sentinel : (d << vbits) | s;
        } else {
            keys[i] = loop ? sentinel : (s << vbits) | d;
        }
    }
}

__global__ void k_keys_to_adj(const uint64_t* __restrict__ keys, uint64_t E, int vbits, uint32_t* __restrict__ adj,
                              uint32_t* __restrict__ wgt, uint32_t wmax, uint64_t wk)
{
    const uint64_t mask = (1ULL << vbits) - 1;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k = keys[e];
        uint64_t u = k >> vbits, v = k & mask;
        adj[e] = (uint32_t)v;
        if (wgt) {
            uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
            wgt[e] = 1u + (uint32_t)(d_mix64(wk ^ ((lo << 32) | hi)) % wmax);
        }
    }
}

static int build_from_keys(uint64_t V, int vbits, DevBuf& keys, uint64_t n, int undirected, uint32_t wmax,
                           int need_in, ipg_graph** out)
{
    (void)undirected;
    cudaStream_t st = 0;
    if (n >= (1ULL << 31)) return fail(IPG_EINVAL, "generator: too many sampled edges for one sort (%llu)",
                                       (unsigned long long)n);
    DevBuf alt, temp, nsel;
    IPG_TRY(alt.alloc(n * 8 + 8));
    IPG_TRY(nsel.alloc(8));
    cub::DoubleBuffer<uint64_t> db(keys.as<uint64_t>(), alt.as<uint64_t>());
    size_t tb1 = 0, tb2 = 0;
    int endb = 2 * vbits + 1;
    IPG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb1, db, (int)n, 0, endb, st));
    IPG_CUDA(cub::DeviceSelect::Unique(nullptr, tb2, keys.as<uint64_t>(), alt.as<uint64_t>(), (int*)nsel.p, (int)n, st));
    IPG_TRY(temp.alloc(std::max(tb1, tb2)));
    IPG_CUDA(cub::DeviceRadixSort::SortKeys(temp.p, tb1, db, (int)n, 0, endb, st));
    uint64_t* sorted = db.Current();
    uint64_t* uniq = (sorted == keys.as<uint64_t>()) ? alt.as<uint64_t>() : keys.as<uint64_t>();
    IPG_CUDA(cub::DeviceSelect::Unique(temp.p, tb2, sorted, uniq, (int*)nsel.p, (int)n, st));
    int hn = 0;
    IPG_CUDA(cudaMemcpyAsync(&hn, nsel.p, 4, cudaMemcpyDeviceToHost, st));
    IPG_CUDA(cudaStreamSynchronize(st));
    uint64_t E = (uint64_t)hn;
    if (E) {
        uint64_t last = 0;
        IPG_CUDA(cudaMemcpy(&last, uniq + (E - 1), 8, cudaMemcpyDeviceToHost));
        if (last == (1ULL << (2 * vbits))) E--;
    }
    ipg_graph* g = new ipg_graph();
    g->v.directed = !undirected;
    g->v.symmetric = undirected ? 1 : 0; /* every reverse edge was added, weights are symmetric */
    int r = alloc_out(g, V, E, 4, wmax ? 4 : 0);
    if (r == IPG_OK) {
        k_fill_u64<<<grid_for(V + 1, 256), 256, 0, st>>>((uint64_t*)g->row, V + 1, E);
        if (E) {
            k_row_from_sorted<<<grid_for(E, 256), 256, 0, st>>>(uniq, E, vbits, (uint64_t*)g->row);
            k_keys_to_adj<<<grid_for(E, 256), 256, 0, st>>>(uniq, E, vbits, (uint32_t*)g->adj, (uint32_t*)g->wgt,
                                                             wmax, 0);
        }
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) r = fail(IPG_ECUDA, "generator kernels failed: %s", cudaGetErrorString(e));
    }
    if (r != IPG_OK) {
        delete g;
        return r;
    }
    return finalize(g, need_in, out);
}

static int attach_weights(ipg_graph* g, uint32_t wmax, uint64_t seed);

extern "C" int ipg_graph_generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                                       uint64_t seed, int undirected, uint32_t wmax, int need_in, ipg_graph** out)
{
    if (!out) return fail(IPG_EINVAL, "ipg_graph_generate_rmat: null output");
    *out = nullptr;
    if (scale == 0 || scale > 31) return fail(IPG_EINVAL, "R-MAT scale must be in [1, 31]");
    const uint64_t V = 1ULL << scale;
    const uint64_t M = (uint64_t)edge_factor << scale;
    const uint64_t n = M * (undirected ? 2 : 1);
    const uint64_t ta = (uint64_t)(a * 4294967296.0);
    const uint64_t tab = (uint64_t)((a + b) * 4294967296.0);
    const uint64_t tabc = (uint64_t)((a + b + c) * 4294967296.0);
    const uint64_t seedk = h_mix64(seed ^ 0x5851F42D4C957F2DULL);
    DevBuf keys;
    IPG_TRY(keys.alloc(n * 8 + 8));
    if (M) {
        k_gen_rmat<<<grid_for(M, 256, 32), 256>>>(M, scale, ta, tab, tabc, seedk, undirected,
                                                   1ULL << (2 * scale), keys.as<uint64_t>());
        IPG_CUDA(cudaGetLastError());
    }
    ipg_graph* g = nullptr;
    IPG_TRY(build_from_keys(V, (int)scale, keys, n, undirected, 0, 0, &g));
    keys.release();
    int r = wmax ? attach_weights(g, wmax, seed) : IPG_OK;
    if (r == IPG_OK && need_in) r = ipg_graph_build_in(g);
    if (r != IPG_OK) {
        delete g;
        return r;
    }
    *out = g;
    return IPG_OK;
}

extern "C" int ipg_graph_generate_er(uint64_t n, uint64_t m, uint64_t seed, int undirected, uint32_t wmax,
                                     int need_in, ipg_graph** out)
{
    if (!out) return fail(IPG_EINVAL, "ipg_graph_generate_er: null output");
    *out = nullptr;
    if (n == 0 || n >= (1ULL << 31)) return fail(IPG_EINVAL, "Erdos-Renyi vertex count must be in [1, 2^31)");
    const int vbits = bits_for(n);
    const uint64_t seedk = h_mix64(seed ^ 0x5851F42D4C957F2DULL);
    const uint64_t cnt = m * (undirected ? 2 : 1);
    DevBuf keys;
    IPG_TRY(keys.alloc(cnt * 8 + 8));
    if (m) {
        k_gen_er<<<grid_for(m, 256, 32), 256>>>(m, n, vbits, seedk, undirected, 1ULL << (2 * vbits),
                                                 keys.as<uint64_t>());
        IPG_CUDA(cudaGetLastError());
    }
    ipg_graph* g = nullptr;
    IPG_TRY(build_from_keys(n, vbits, keys, cnt, undirected, 0, 0, &g));
    keys.release();
    int r = wmax ? attach_weights(g, wmax, seed) : IPG_OK;
    if (r == IPG_OK && need_in) r = ipg_graph_build_in(g);
    if (r != IPG_OK) {
        delete g;
        return r;
    }
    *out = g;
    return IPG_OK;
}

__global__ void k_weights(const uint64_t* __restrict__ row, uint64_t V, uint64_t E, const uint32_t* __restrict__ adj,
                          uint32_t wmax, uint64_t wk, uint32_t* __restrict__ wgt)
{
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = V;
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) >> 1;
            if (row[mid] <= e) lo = mid; else hi = mid;
        }
        uint64_t u = lo, v = adj[e];
        uint64_t a = u < v ? u : v, b = u < v ? v : u;
        wgt[e] = 1u + (uint32_t)(d_mix64(wk ^ ((a << 32) | b)) % wmax);
    }
}

// Weights as the oracle's og_gen_weights: w(u,v) = 1 + mix(key ^ (min<<32|max)) % wmax.
static int attach_weights(ipg_graph* g, uint32_t wmax, uint64_t seed)
{
    if (g->wgt) return IPG_OK;
    g->wgt_bytes = (g->v.E ? g->v.E : 1) * 4;
    IPG_TRY(ipg_dev_alloc(&g->wgt, g->wgt_bytes));
    g->v.weight_bytes = 4;
    g->v.d_wgt = g->wgt;
    g->v.device_bytes += g->wgt_bytes;
    if (g->v.E) {
        k_weights<<<grid_for(g->v.E, 256), 256>>>(g->v.d_row, g->v.V, g->v.E, (const uint32_t*)g->v.d_adj, wmax,
                                                  h_mix64(seed ^ 0x77ULL), (uint32_t*)g->wgt);
        IPG_CUDA(cudaGetLastError());
        IPG_CUDA(cudaDeviceSynchronize());
    }
    return IPG_OK;
}

// ---------------------------------------------------------------------------
// Views, host copies, files
// ---------------------------------------------------------------------------
extern "C" int ipg_graph_view_get(const ipg_graph* g, ipg_graph_view* view)
{
    if (!g || !view) return fail(IPG_EINVAL, "ipg_graph_view_get: null argument");
    *view = g->v;
    return IPG_OK;
}

extern "C" int ipg_graph_to_host(const ipg_graph* g, uint64_t* idx, void* adj, void* wgt)
{
    if (!g) return fail(IPG_EINVAL, "ipg_graph_to_host: null graph");
    if (idx && g->v.V) IPG_CUDA(cudaMemcpy(idx, g->v.d_row, g->v.V * 8, cudaMemcpyDeviceToHost));
    if (adj && g->v.E) IPG_CUDA(cudaMemcpy(adj, g->v.d_adj, g->v.E * (uint64_t)g->v.id_bytes, cudaMemcpyDeviceToHost));
    if (wgt && g->v.E && g->v.d_wgt)
        IPG_CUDA(cudaMemcpy(wgt, g->v.d_wgt, g->v.E * (uint64_t)g->v.weight_bytes, cudaMemcpyDeviceToHost));
    return IPG_OK;
}

static int write_all(const std::string& name, const void* p, uint64_t bytes)
{
    FILE* f = fopen(name.c_str(), "wb");
    if (!f) return fail(IPG_EIO, "Cannot open the file \"%s\" in mode \"wb\".", name.c_str());
    uint64_t done = 0;
    while (done < bytes) {
        size_t n = fwrite((const char*)p + done, 1, (size_t)std::min<uint64_t>(bytes - done, 1ULL << 30), f);
        if (n == 0) {
            fclose(f);
            return fail(IPG_EIO, "Failed to write.");
        }
        done += n;
    }
    fclose(f);
    return IPG_OK;
}

extern "C" int ipg_graph_write(const ipg_graph* g, const char* path)
{
    if (!g || !path) return fail(IPG_EINVAL, "ipg_graph_write: null argument");
    std::string base(path);
    FILE* f = fopen((base + ".config").c_str(), "w");
    if (!f) return fail(IPG_EIO, "Cannot open the file \"%s.config\" in mode \"w\".", path);
    fprintf(f, "%llu %llu\n", (unsigned long long)g->v.V, (unsigned long long)g->v.E);
    fclose(f);
    std::vector<uint64_t> idx(g->v.V);
    void* adj = nullptr;
    void* wgt = nullptr;
    if (g->v.E) {
        IPG_CUDA(cudaMallocHost(&adj, g->v.E * (uint64_t)g->v.id_bytes));
        if (g->v.d_wgt) IPG_CUDA(cudaMallocHost(&wgt, g->v.E * (uint64_t)g->v.weight_bytes));
    }
    int r = ipg_graph_to_host(g, idx.data(), adj, wgt);
    if (r == IPG_OK) r = write_all(base + ".idx", idx.data(), g->v.V * 8);
    if (r == IPG_OK) r = write_all(base + ".adj", adj, g->v.E * (uint64_t)g->v.id_bytes);
    if (r == IPG_OK && wgt) r = write_all(base + ".wgt", wgt, g->v.E * (uint64_t)g->v.weight_bytes);
    if (adj) cudaFreeHost(adj);
    if (wgt) cudaFreeHost(wgt);
    return r;
}

extern "C" void ipg_graph_free(ipg_graph* g) { delete g; }

extern "C" int ipg_graph_set_symmetric(ipg_graph* g, int symmetric)
{
    if (!g) return fail(IPG_EINVAL, "ipg_graph_set_symmetric: null graph");
    g->v.symmetric = symmetric ? 1 : 0;
    return IPG_OK;
}

extern "C" int ipg_graph_set_directed(ipg_graph* g, int directed)
{
    if (!g) return fail(IPG_EINVAL, "ipg_graph_set_directed: null graph");
    directed = directed ? 1 : 0;
    if (g->v.directed == directed) return IPG_OK;
    // in-lists and the degree classes over them belong to the old meaning
    g->v.device_bytes -= g->in_row_bytes + g->in_adj_bytes + g->in_wgt_bytes;
    ipg_dev_free(g->in_row, g->in_row_bytes);
    ipg_dev_free(g->in_adj, g->in_adj_bytes);
    ipg_dev_free(g->in_wgt, g->in_wgt_bytes);
    g->in_row = g->in_adj = g->in_wgt = nullptr;
    g->in_row_bytes = g->in_adj_bytes = g->in_wgt_bytes = 0;
    ipg_dev_free(g->bins[1].lists, g->bins[1].bytes);
    g->bins[1] = ipg_graph::BinCache();
    g->v.has_in = 0;
    g->v.d_in_row = nullptr;
    g->v.d_in_adj = nullptr;
    g->v.d_in_wgt = nullptr;
    g->v.max_in_degree = directed ? 0 : g->v.max_out_degree;  // 0: unknown until ipg_graph_build_in
    g->v.directed = directed;
    g->generation++;  // engines attached to the old meaning (and its in-lists) must attach again
    return IPG_OK;
}

// err bit 1: a row is not sorted; bit 2: an edge has no reverse (or the
// reverse has another weight).
template <class T>
__global__ void k_check_symmetric(const uint64_t* __restrict__ row, const T* __restrict__ adj,
                                  const uint32_t* __restrict__ wgt, uint64_t V, uint64_t E, uint32_t* err)
{
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = 0, hi = V;  // source u: row[u] <= e < row[u+1]
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) >> 1;
            if (row[mid] <= e) lo = mid; else hi = mid;
        }
        const uint64_t u = lo, v = (uint64_t)adj[e];
        if (e + 1 < row[u + 1] && (uint64_t)adj[e + 1] <= v) atomicOr(err, 1u);
        uint64_t a = row[v], b = row[v + 1];  // find u in row(v)
        while (a < b) {
            uint64_t mid = (a + b) >> 1;
            if ((uint64_t)adj[mid] < u) a = mid + 1; else b = mid;
        }
        if (a >= row[v + 1] || (uint64_t)adj[a] != u || (wgt && wgt[a] != wgt[e])) atomicOr(err, 2u);
    }
}

extern "C" int ipg_graph_check_symmetric(const ipg_graph* g, int* result)
{
    if (!g || !result) return fail(IPG_EINVAL, "ipg_graph_check_symmetric: null argument");
    *result = 1;
    if (g->v.E == 0) return IPG_OK;
    if (g->v.d_wgt && g->v.weight_bytes != 4) return fail(IPG_EINVAL, "symmetry check supports u32 weights only");
    DevBuf err;
    IPG_TRY(err.alloc(4));
    IPG_CUDA(cudaMemset(err.p, 0, 4));
    if (g->v.id_bytes == 4)
        k_check_symmetric<<<grid_for(g->v.E, 256), 256>>>(g->v.d_row, (const uint32_t*)g->v.d_adj,
                                                          (const uint32_t*)g->v.d_wgt, g->v.V, g->v.E, err.as<uint32_t>());
    else
        k_check_symmetric<<<grid_for(g->v.E, 256), 256>>>(g->v.d_row, (const uint64_t*)g->v.d_adj,
                                                          (const uint32_t*)g->v.d_wgt, g->v.V, g->v.E, err.as<uint32_t>());
    IPG_CUDA(cudaGetLastError());
    uint32_t h = 0;
    IPG_CUDA(cudaMemcpy(&h, err.p, 4, cudaMemcpyDeviceToHost));
    *result = (h & 1) ? -1 : ((h & 2) ? 0 : 1);
    return IPG_OK;
}

// ---------------------------------------------------------------------------
// Frontier compaction: bitmap -> up to three degree-class lists.
// A block of 256 threads owns a tile of 256 bitmap words (8192 vertices):
// pass 1 counts per class, one atomicAdd per class per tile reserves space,
// pass 2 writes the ids (sorted within the tile).
// ---------------------------------------------------------------------------
constexpr int CT_THREADS = 256;
constexpr int CT_WARPS = CT_THREADS / 32;

__device__ __forceinline__ int deg_class(uint64_t d, uint64_t t0, uint64_t t1)
{
    return d <= t0 ? 0 : (d <= t1 ? 1 : 2);
}

__global__ void __launch_bounds__(CT_THREADS) k_compact(uint32_t* __restrict__ bitmap, uint64_t V,
                                                        const uint64_t* __restrict__ row, uint64_t t0, uint64_t t1,
                                                        uint32_t* __restrict__ l0, uint32_t* __restrict__ l1,
                                                        uint32_t* __restrict__ l2, uint32_t* __restrict__ counts,
                                                        unsigned long long* __restrict__ edges, int clear)
{
    __shared__ uint32_t s_cnt[CT_WARPS][3];
    __shared__ uint32_t s_base[3];
    __shared__ unsigned long long s_edges[3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t nwords = (V + 31) >> 5;
    const uint64_t tiles = (nwords + CT_THREADS - 1) / CT_THREADS;
    if (threadIdx.x < 3) s_edges[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint64_t wbase = tile * CT_THREADS + (uint64_t)warp * 32;
        const uint64_t wi = wbase + lane;
        uint32_t word = 0;
        if (wi < nwords) {
            word = bitmap ? bitmap[wi] : 0xffffffffu;
            if (wi == nwords - 1 && (V & 31)) word &= (1u << (V & 31)) - 1u;
        }
        uint32_t c0 = 0, c1 = 0, c2 = 0;
        unsigned long long es[3] = {0, 0, 0};
        for (int j = 0; j < 32; j++) {
            uint32_t w = __shfl_sync(0xffffffffu, word, j);
            if (w == 0) continue;
            const uint64_t v = (wbase + j) * 32 + lane;
            const bool set = (w >> lane) & 1u;
            int cls = 0;
            if (set && row) {
                uint64_t d = row[v + 1] - row[v];
                cls = deg_class(d, t0, t1);
                es[cls] += d;
            }
            c0 += __popc(__ballot_sync(0xffffffffu, set && cls == 0));
            c1 += __popc(__ballot_sync(0xffffffffu, set && cls == 1));
            c2 += __popc(__ballot_sync(0xffffffffu, set && cls == 2));
        }
        for (int k = 0; k < 3; k++)
            for (int o = 16; o > 0; o >>= 1) es[k] += __shfl_down_sync(0xffffffffu, es[k], o);
        if (lane == 0) {
            s_cnt[warp][0] = c0;
            s_cnt[warp][1] = c1;
            s_cnt[warp][2] = c2;
            for (int k = 0; k < 3; k++)
                if (es[k]) atomicAdd(&s_edges[k], es[k]);
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            uint32_t tot = 0;
            for (int w = 0; w < CT_WARPS; w++) tot += s_cnt[w][threadIdx.x];
            s_base[threadIdx.x] = tot ? atomicAdd(&counts[threadIdx.x], tot) : 0u;
            if (edges && s_edges[threadIdx.x]) atomicAdd(&edges[threadIdx.x], s_edges[threadIdx.x]);
        }
        __syncthreads();
        uint32_t o0 = s_base[0], o1 = s_base[1], o2 = s_base[2];
        for (int w = 0; w < warp; w++) {
            o0 += s_cnt[w][0];
            o1 += s_cnt[w][1];
            o2 += s_cnt[w][2];
        }
        for (int j = 0; j < 32; j++) {
            uint32_t w = __shfl_sync(0xffffffffu, word, j);
            if (w == 0) continue;
            const uint64_t v = (wbase + j) * 32 + lane;
            const bool set = (w >> lane) & 1u;
            int cls = 0;
            if (set && row) cls = deg_class(row[v + 1] - row[v], t0, t1);
            uint32_t m0 = __ballot_sync(0xffffffffu, set && cls == 0);
            uint32_t m1 = __ballot_sync(0xffffffffu, set && cls == 1);
            uint32_t m2 = __ballot_sync(0xffffffffu, set && cls == 2);
            if (set) {
                if (cls == 0) l0[o0 + __popc(m0 & lt)] = (uint32_t)v;
                else if (cls == 1) l1[o1 + __popc(m1 & lt)] = (uint32_t)v;
                else l2[o2 + __popc(m2 & lt)] = (uint32_t)v;
            }
            o0 += __popc(m0);
            o1 += __popc(m1);
            o2 += __popc(m2);
        }
        if (clear && bitmap && wi < nwords && word) bitmap[wi] = 0;
        __syncthreads();
        if (threadIdx.x < 3) s_edges[threadIdx.x] = 0;
        __syncthreads();
    }
}

extern "C" int ipg_compact(uint32_t* d_bitmap, uint64_t V, const uint64_t* d_row, uint64_t t0, uint64_t t1,
                           uint32_t* d_list0, uint32_t* d_list1, uint32_t* d_list2, uint32_t* d_counts,
                           uint64_t* d_edges, int clear, void* stream)
{
    if (V == 0) return IPG_OK;
    if (!d_counts || !d_list0) return fail(IPG_EINVAL, "ipg_compact: null output");
    if (d_row && (!d_list1 || !d_list2)) return fail(IPG_EINVAL, "ipg_compact: three lists needed with degrees");
    const uint64_t nwords = (V + 31) >> 5;
    const uint64_t tiles = (nwords + CT_THREADS - 1) / CT_THREADS;
    uint64_t blocks = std::min<uint64_t>(tiles, (uint64_t)ipg_sm_count() * 8);
    k_compact<<<(uint32_t)blocks, CT_THREADS, 0, (cudaStream_t)stream>>>(
        d_bitmap, V, d_row, t0, t1, d_list0, d_list1, d_list2, d_counts, (unsigned long long*)d_edges, clear);
    IPG_CUDA(cudaGetLastError());
    return IPG_OK;
}

__global__ void k_popc_or(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint64_t nwords,
                          unsigned long long* __restrict__ out)
{
    __shared__ unsigned long long s[32];
    unsigned long long sum = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nwords; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t w = a[i];
        if (b) w |= b[i];
        sum += __popc(w);
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x < 32) {
        sum = (threadIdx.x < (blockDim.x >> 5)) ? s[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        if (threadIdx.x == 0 && sum) atomicAdd(out, sum);
    }
}

extern "C" int ipg_bitmap_popc_or(const uint32_t* d_a, const uint32_t* d_b, uint64_t nwords, uint64_t* d_out,
                                  void* stream)
{
    if (nwords == 0) return IPG_OK;
    k_popc_or<<<grid_for(nwords, 256, 4), 256, 0, (cudaStream_t)stream>>>(d_a, d_b, nwords,
                                                                          (unsigned long long*)d_out);
    IPG_CUDA(cudaGetLastError());
    return IPG_OK;
}

// ---------------------------------------------------------------------------
// Static degree bins of all vertices (cached per direction).
// ---------------------------------------------------------------------------
extern "C" int ipg_graph_bins(ipg_graph* g, int use_in, uint64_t t0, uint64_t t1, ipg_bins* bins)
{
    if (!g || !bins) return fail(IPG_EINVAL, "ipg_graph_bins: null argument");
    if (use_in && !g->v.has_in) IPG_TRY(ipg_graph_build_in(g));
    auto& c = g->bins[use_in ? 1 : 0];
    if (c.valid && c.t0 == t0 && c.t1 == t1) {
        *bins = c.bins;
        return IPG_OK;
    }
    ipg_dev_free(c.lists, c.bytes);
    c.lists = nullptr;
    c.valid = false;
    const uint64_t V = g->v.V;
    c.bytes = (V ? V : 1) * 4 + 64;
    IPG_TRY(ipg_dev_alloc(&c.lists, c.bytes));
    DevBuf cnt, l1, l2;
    IPG_TRY(cnt.alloc(64));
    IPG_TRY(l1.alloc((V ? V : 1) * 4));
    IPG_TRY(l2.alloc((V ? V : 1) * 4));
    IPG_CUDA(cudaMemset(cnt.p, 0, 64));
    const uint64_t* row = use_in ? g->v.d_in_row : g->v.d_row;
    uint64_t* d_esum = (uint64_t*)((char*)cnt.p + 32);
    IPG_TRY(ipg_compact(nullptr, V, row, t0, t1, (uint32_t*)c.lists, l1.as<uint32_t>(), l2.as<uint32_t>(),
                        cnt.as<uint32_t>(), d_esum, 0, nullptr));
    uint32_t h[3] = {0, 0, 0};
    uint64_t esum[3] = {0, 0, 0};
    IPG_CUDA(cudaMemcpy(h, cnt.p, 12, cudaMemcpyDeviceToHost));
    IPG_CUDA(cudaMemcpy(esum, d_esum, 24, cudaMemcpyDeviceToHost));
    // Pack the three lists back to back in one allocation.
    uint32_t* base = (uint32_t*)c.lists;
    if (h[1]) IPG_CUDA(cudaMemcpy(base + h[0], l1.p, (uint64_t)h[1] * 4, cudaMemcpyDeviceToDevice));
    if (h[2]) IPG_CUDA(cudaMemcpy(base + h[0] + h[1], l2.p, (uint64_t)h[2] * 4, cudaMemcpyDeviceToDevice));
    // Lists within a class come out tile-ordered, which is id order, since
    // each block claims its tiles' space in arbitrary order; sort each class
    // so that the gather walks the graph in id order.
    for (int k = 0; k < 3; k++) {
        uint64_t off = (k == 0) ? 0 : (k == 1 ? h[0] : (uint64_t)h[0] + h[1]);
        if (h[k] < 2) continue;
        DevBuf alt, temp;
        IPG_TRY(alt.alloc((uint64_t)h[k] * 4));
        cub::DoubleBuffer<uint32_t> db(base + off, alt.as<uint32_t>());
        size_t tb = 0;
        IPG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int)h[k], 0, bits_for(V)));
        IPG_TRY(temp.alloc(tb));
        IPG_CUDA(cub::DeviceRadixSort::SortKeys(temp.p, tb, db, (int)h[k], 0, bits_for(V)));
        if (db.Current() != base + off)
            IPG_CUDA(cudaMemcpy(base + off, db.Current(), (uint64_t)h[k] * 4, cudaMemcpyDeviceToDevice));
        IPG_CUDA(cudaDeviceSynchronize());
    }
    c.bins.d_list[0] = base;
    c.bins.d_list[1] = base + h[0];
    c.bins.d_list[2] = base + h[0] + h[1];
    for (int k = 0; k < 3; k++) {
        c.bins.count[k] = h[k];
        c.bins.edges[k] = esum[k];
    }
    c.bins.t0 = t0;
    c.bins.t1 = t1;
    c.t0 = t0;
    c.t1 = t1;
    c.valid = true;
    *bins = c.bins;
    return IPG_OK;
}
