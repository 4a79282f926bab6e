// probe.cu -- the random-gather ceiling of the GPU.
//
// The engine's push and gather kernels spend their time on scattered reads:
// per pushed edge one 4-byte mailbox precheck, per gathered edge one 4- or
// 8-byte broadcast value (or a 64-byte lane row for the request server's PPR
// lanes), at addresses that the edge list decides.  A copy kernel's bandwidth
// is not their ceiling: every scattered element costs a whole L1/L2 request,
// so the rate of requests bounds them well before DRAM bandwidth does.
// ipg_measure_gather times exactly that access pattern on its own -- a
// coalesced stream of u32 indices, and for each index one read of a table
// element at a pseudo-random position -- so that the kernels' edge rates can
// be read against the rate the memory system sustains for the same pattern.
#include "ipregel_b200.h"
#include "ipregel_b200_probe.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

// The probe library's own last error (it links nothing of the runtime but
// its header's status codes).
static thread_local char pb_err[256];

static int pb_fail(int code, const char* msg)
{
    snprintf(pb_err, sizeof pb_err, "%s", msg);
    return code;
}

extern "C" const char* ipg_probe_last_error(void) { return pb_err; }

#define PB_THREADS 256
#define PB_UNROLL 8

#define PB_CU(call)                                                                     \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return pb_fail(IPG_ECUDA, cudaGetErrorString(e_)); \
    } while (0)

// A 32-bit mixing function (the finaliser of MurmurHash3, Appleby 2011):
// consecutive i give indices spread uniformly over the table.
__device__ __forceinline__ uint32_t pb_mix(uint64_t i)
{
    uint32_t h = (uint32_t)i ^ (uint32_t)(i >> 32) * 0x9e3779b9u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

__global__ void k_pb_indices(uint32_t* __restrict__ idx, uint64_t n, uint32_t rows, uint64_t salt)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        idx[i] = (uint32_t)(((uint64_t)pb_mix(i + salt) * rows) >> 32);
}

__global__ void k_pb_fill(uint32_t* __restrict__ t, uint64_t words)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x)
        t[i] = (uint32_t)i;
}

// 4-byte rows: thread j of the grid reads idx[j + u * stride] (coalesced) and
// then table[idx] for PB_UNROLL indices at once, so PB_UNROLL scattered loads
// are in flight per thread.
__global__ void __launch_bounds__(PB_THREADS) k_pb_gather4(const uint32_t* __restrict__ idx,
                                                           const uint32_t* __restrict__ table, uint64_t n,
                                                           uint32_t* __restrict__ sink)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t acc = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += stride * PB_UNROLL) {
        uint32_t j[PB_UNROLL];
#pragma unroll
        for (int u = 0; u < PB_UNROLL; u++) j[u] = (i + u * stride < n) ? __ldcs(idx + i + u * stride) : 0xffffffffu;
#pragma unroll
        for (int u = 0; u < PB_UNROLL; u++)
            if (j[u] != 0xffffffffu) acc += table[j[u]];
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;  // keeps the loads; practically never stores
}

// Rows of 16 * TPR bytes read as float4 quads by TPR consecutive threads (64
// bytes: the lane rows of the PPR lanes; 256 bytes: the distance rows of the
// min-plus lanes): a warp reads 32 / TPR rows per load instruction.
template <int TPR>
__global__ void __launch_bounds__(PB_THREADS) k_pb_gather_rows(const uint32_t* __restrict__ idx,
                                                               const uint4* __restrict__ table, uint64_t n,
                                                               uint32_t* __restrict__ sink)
{
    const uint64_t groups = ((uint64_t)gridDim.x * blockDim.x) / TPR;
    const int q = threadIdx.x % TPR;
    uint32_t acc = 0;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / TPR; i < n; i += groups * PB_UNROLL) {
        uint32_t j[PB_UNROLL];
#pragma unroll
        for (int u = 0; u < PB_UNROLL; u++) j[u] = (i + u * groups < n) ? __ldcs(idx + i + u * groups) : 0xffffffffu;
#pragma unroll
        for (int u = 0; u < PB_UNROLL; u++)
            if (j[u] != 0xffffffffu) {
                const uint4 x = table[(uint64_t)j[u] * TPR + q];
                acc += x.x ^ x.y ^ x.z ^ x.w;
            }
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;
}

extern "C" int ipg_measure_gather(uint64_t table_bytes, uint32_t row_bytes, uint64_t n, int reps,
                                  double* rows_per_s, double* gbs)
{
    if (!rows_per_s || !gbs) return pb_fail(IPG_EINVAL, "ipg_measure_gather: null output");
    if (row_bytes != 4 && row_bytes != 64 && row_bytes != 128 && row_bytes != 256)
        return pb_fail(IPG_EINVAL, "ipg_measure_gather: row_bytes must be 4, 64, 128 or 256");
    if (table_bytes < row_bytes || table_bytes / row_bytes > 0xffffffffull || n == 0 || n > (1ull << 31) || reps < 1)
        return pb_fail(IPG_EINVAL, "ipg_measure_gather: table of 1 .. 2^32 rows, 1 <= n <= 2^31, reps >= 1");
    const uint64_t rows = table_bytes / row_bytes;
    int dev = 0, sms = 0, per_sm = 0;
    PB_CU(cudaGetDevice(&dev));
    PB_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (row_bytes == 4) PB_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pb_gather4, PB_THREADS, 0));
    else PB_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pb_gather_rows<16>, PB_THREADS, 0));
    const uint32_t grid = (uint32_t)(sms * (per_sm > 0 ? per_sm : 1));

    uint32_t *idx = nullptr, *table = nullptr, *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = IPG_OK;
    float ms = 0.f;
    auto check = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == IPG_OK) rc = pb_fail(IPG_ECUDA, cudaGetErrorString(e));
        return rc == IPG_OK;
    };
    if (check(cudaMalloc(&idx, n * 4)) && check(cudaMalloc(&table, rows * row_bytes)) && check(cudaMalloc(&sink, 4)) &&
        check(cudaEventCreate(&e0)) && check(cudaEventCreate(&e1))) {
        k_pb_indices<<<grid, PB_THREADS>>>(idx, n, (uint32_t)rows, 0x5eedull);
        k_pb_fill<<<grid, PB_THREADS>>>(table, rows * row_bytes / 4);
        auto launch = [&]() {
            const uint4* t4 = reinterpret_cast<const uint4*>(table);
            if (row_bytes == 4) k_pb_gather4<<<grid, PB_THREADS>>>(idx, table, n, sink);
            else if (row_bytes == 64) k_pb_gather_rows<4><<<grid, PB_THREADS>>>(idx, t4, n, sink);
            else if (row_bytes == 128) k_pb_gather_rows<8><<<grid, PB_THREADS>>>(idx, t4, n, sink);
            else k_pb_gather_rows<16><<<grid, PB_THREADS>>>(idx, t4, n, sink);
        };
        launch();  // warm-up: brings a table that fits into L2
        if (check(cudaGetLastError()) && check(cudaEventRecord(e0))) {
            for (int r = 0; r < reps; r++) launch();
            if (check(cudaEventRecord(e1)) && check(cudaEventSynchronize(e1)) && check(cudaGetLastError()))
                check(cudaEventElapsedTime(&ms, e0, e1));
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(idx);
    cudaFree(table);
    cudaFree(sink);
    if (rc != IPG_OK) return rc;
    const double sec = ms * 1e-3 / reps;
    *rows_per_s = sec > 0 ? (double)n / sec : 0.0;
    *gbs = sec > 0 ? (double)n * (4.0 + row_bytes) / sec / 1e9 : 0.0;
    return IPG_OK;
}
