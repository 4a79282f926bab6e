// noalloc.cu -- degree classes of all vertices without any device allocation.
//
// ipg_graph_bins (runtime.cu) builds the thread / warp / block degree classes
// that the single-broadcast gather walks; it allocates temporary lists and a
// sort buffer with cudaMalloc.  ipg_degree_classes_noalloc computes the same
// lists into memory the caller passes, keeping its only scratch -- one count
// and one degree sum per class for each tile of 8192 vertices -- in the
// file-scope array below.  The lists come out sorted by construction: tiles
// are placed by an exclusive scan over tile index, warps by warp index and
// lanes by lane rank, so no sort (and no sort buffer) is needed.
#include "ipregel_b200.h"

#include <cuda_runtime.h>

#include <mutex>

#define NA_THREADS 256
#define NA_WARPS (NA_THREADS / 32)
#define NA_TILE_VERTICES (NA_THREADS * 32)
#define NA_MAX_TILES 8192
#define NA_MAX_VERTICES ((uint64_t)NA_MAX_TILES * NA_TILE_VERTICES) /* 67,108,864 */
#define NA_SCAN_THREADS 1024

// Scratch layout (u64): [0, 3T) per-tile class counts, overwritten by their
// exclusive offsets; [3T, 6T) per-tile class degree sums; [6T, 6T+3) class
// sizes.  T = NA_MAX_TILES.  Every entry a call reads is written earlier in
// the same call, so nothing needs clearing between calls.
static __device__ __align__(256) unsigned long long ipg_noalloc_scratch[6 * NA_MAX_TILES + 8];

extern "C" int ipg_internal_fail(int code, const char* msg);

__device__ __forceinline__ int na_class(uint64_t d, uint64_t t0, uint64_t t1) { return d <= t0 ? 0 : (d <= t1 ? 1 : 2); }

// Bit j of the word a warp lane holds: vertices of [0, V) only.
__device__ __forceinline__ uint32_t na_word(uint64_t wi, uint64_t V)
{
    const uint64_t nwords = (V + 31) >> 5;
    if (wi >= nwords) return 0u;
    if (wi == nwords - 1 && (V & 31)) return (1u << (V & 31)) - 1u;
    return 0xffffffffu;
}

// Pass 1: per-tile class counts and degree sums.
__global__ void __launch_bounds__(NA_THREADS) na_count(uint64_t V, const uint64_t* __restrict__ row, uint64_t t0,
                                                       uint64_t t1, unsigned long long* __restrict__ scratch)
{
    __shared__ unsigned long long s_cnt[NA_WARPS][3], s_deg[NA_WARPS][3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t tile = blockIdx.x;
    const uint64_t wbase = tile * NA_THREADS + (uint64_t)warp * 32;
    const uint32_t word = na_word(wbase + lane, V);
    unsigned long long c[3] = {0, 0, 0}, d[3] = {0, 0, 0};
    for (int j = 0; j < 32; j++) {
        const uint32_t w = __shfl_sync(0xffffffffu, word, j);
        if (w == 0) continue;
        const uint64_t v = (wbase + j) * 32 + lane;
        const bool set = (w >> lane) & 1u;
        int k = 0;
        uint64_t deg = 0;
        if (set) {
            deg = row[v + 1] - row[v];
            k = na_class(deg, t0, t1);
        }
        for (int q = 0; q < 3; q++) {
            c[q] += __popc(__ballot_sync(0xffffffffu, set && k == q));
            unsigned long long dq = (set && k == q) ? deg : 0ULL;
            for (int o = 16; o > 0; o >>= 1) dq += __shfl_down_sync(0xffffffffu, dq, o);
            d[q] += dq;
        }
    }
    if (lane == 0)
        for (int q = 0; q < 3; q++) {
            s_cnt[warp][q] = c[q];
            s_deg[warp][q] = d[q];
        }
    __syncthreads();
    if (threadIdx.x < 3) {
        unsigned long long tc = 0, td = 0;
        for (int w = 0; w < NA_WARPS; w++) {
            tc += s_cnt[w][threadIdx.x];
            td += s_deg[w][threadIdx.x];
        }
        scratch[3 * tile + threadIdx.x] = tc;
        scratch[3 * NA_MAX_TILES + 3 * tile + threadIdx.x] = td;
    }
}

// Pass 2 (one block): exclusive scan of the tile counts of each class, class
// sizes and degree sums into the caller's totals.
__global__ void __launch_bounds__(NA_SCAN_THREADS) na_scan(uint64_t tiles, unsigned long long* __restrict__ scratch,
                                                           uint64_t* __restrict__ totals)
{
    __shared__ unsigned long long s_part[NA_SCAN_THREADS];
    const uint64_t per = (tiles + NA_SCAN_THREADS - 1) / NA_SCAN_THREADS;
    const uint64_t lo = threadIdx.x * per, hi = (lo + per < tiles) ? lo + per : tiles;
    for (int q = 0; q < 3; q++) {
        unsigned long long sum = 0, dsum = 0;
        for (uint64_t t = lo; t < hi; t++) {
            sum += scratch[3 * t + q];
            dsum += scratch[3 * NA_MAX_TILES + 3 * t + q];
        }
        s_part[threadIdx.x] = sum;
        __syncthreads();
        // inclusive Hillis-Steele scan of the per-thread sums
        for (int o = 1; o < NA_SCAN_THREADS; o <<= 1) {
            unsigned long long x = (threadIdx.x >= (unsigned)o) ? s_part[threadIdx.x - o] : 0ULL;
            __syncthreads();
            s_part[threadIdx.x] += x;
            __syncthreads();
        }
        unsigned long long run = s_part[threadIdx.x] - sum;
        for (uint64_t t = lo; t < hi; t++) {
            unsigned long long cnt = scratch[3 * t + q];
            scratch[3 * t + q] = run;
            run += cnt;
        }
        const unsigned long long total = s_part[NA_SCAN_THREADS - 1];
        __syncthreads();
        // degree sum of the class
        s_part[threadIdx.x] = dsum;
        __syncthreads();
        for (int o = NA_SCAN_THREADS / 2; o > 0; o >>= 1) {
            if (threadIdx.x < (unsigned)o) s_part[threadIdx.x] += s_part[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            totals[q] = total;
            totals[3 + q] = s_part[0];
            scratch[6 * NA_MAX_TILES + q] = total;
        }
        __syncthreads();
    }
}

// Pass 3: write each class's ids at class base + tile offset + warp offset + rank.
__global__ void __launch_bounds__(NA_THREADS) na_write(uint64_t V, const uint64_t* __restrict__ row, uint64_t t0,
                                                       uint64_t t1, const unsigned long long* __restrict__ scratch,
                                                       uint32_t* __restrict__ lists)
{
    __shared__ unsigned long long s_cnt[NA_WARPS][3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t tile = blockIdx.x;
    const uint64_t wbase = tile * NA_THREADS + (uint64_t)warp * 32;
    const uint32_t word = na_word(wbase + lane, V);
    unsigned long long c[3] = {0, 0, 0};
    for (int j = 0; j < 32; j++) {
        const uint32_t w = __shfl_sync(0xffffffffu, word, j);
        if (w == 0) continue;
        const uint64_t v = (wbase + j) * 32 + lane;
        const bool set = (w >> lane) & 1u;
        const int k = set ? na_class(row[v + 1] - row[v], t0, t1) : 0;
        for (int q = 0; q < 3; q++) c[q] += __popc(__ballot_sync(0xffffffffu, set && k == q));
    }
    if (lane == 0)
        for (int q = 0; q < 3; q++) s_cnt[warp][q] = c[q];
    __syncthreads();
    const unsigned long long n0 = scratch[6 * NA_MAX_TILES + 0], n1 = scratch[6 * NA_MAX_TILES + 1];
    unsigned long long off[3];
    off[0] = scratch[3 * tile + 0];
    off[1] = n0 + scratch[3 * tile + 1];
    off[2] = n0 + n1 + scratch[3 * tile + 2];
    for (int w = 0; w < warp; w++)
        for (int q = 0; q < 3; q++) off[q] += s_cnt[w][q];
    for (int j = 0; j < 32; j++) {
        const uint32_t w = __shfl_sync(0xffffffffu, word, j);
        if (w == 0) continue;
        const uint64_t v = (wbase + j) * 32 + lane;
        const bool set = (w >> lane) & 1u;
        const int k = set ? na_class(row[v + 1] - row[v], t0, t1) : 0;
        for (int q = 0; q < 3; q++) {
            const uint32_t m = __ballot_sync(0xffffffffu, set && k == q);
            if (set && k == q) lists[off[q] + __popc(m & lt)] = (uint32_t)v;
            off[q] += __popc(m);
        }
    }
}

// Device address of the scratch array, looked up once per device.
static std::mutex na_mutex;
static void* na_addr[64];

static int na_scratch(unsigned long long** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return ipg_internal_fail(IPG_EINVAL, "ipg_degree_classes_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(na_mutex);
    if (!na_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, ipg_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return ipg_internal_fail(IPG_ECUDA, "ipg_degree_classes_noalloc: cudaGetSymbolAddress of the scratch failed");
        }
        na_addr[dev] = p;
    }
    *out = (unsigned long long*)na_addr[dev];
    return IPG_OK;
}

extern "C" int ipg_degree_classes_noalloc(uint64_t V, const uint64_t* d_row, uint64_t t0, uint64_t t1,
                                          uint32_t* d_lists, uint64_t* d_totals, void* stream)
{
    if (V > NA_MAX_VERTICES)
        return ipg_internal_fail(IPG_EINVAL,
                                 "ipg_degree_classes_noalloc: at most 67108864 vertices (8192 tiles of 8192); "
                                 "use ipg_graph_bins for larger graphs");
    if (!d_totals || (V && (!d_row || !d_lists)))
        return ipg_internal_fail(IPG_EINVAL, "ipg_degree_classes_noalloc: null argument");
    unsigned long long* scratch = nullptr;
    int r = na_scratch(&scratch);
    if (r != IPG_OK) return r;
    cudaStream_t st = (cudaStream_t)stream;
    if (V == 0) {
        cudaError_t e = cudaMemsetAsync(d_totals, 0, 6 * sizeof(uint64_t), st);
        return e == cudaSuccess ? IPG_OK : ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
    }
    const uint64_t tiles = (V + NA_TILE_VERTICES - 1) / NA_TILE_VERTICES;
    na_count<<<(unsigned)tiles, NA_THREADS, 0, st>>>(V, d_row, t0, t1, scratch);
    na_scan<<<1, NA_SCAN_THREADS, 0, st>>>(tiles, scratch, d_totals);
    na_write<<<(unsigned)tiles, NA_THREADS, 0, st>>>(V, d_row, t0, t1, scratch, d_lists);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? IPG_OK : ipg_internal_fail(IPG_ECUDA, cudaGetErrorString(e));
}
