/*
 * host.cuh -- host half of the drop-in headers: ip_init / ip_run / ip_dump and
 * the other host-side functions of the reference's interface
 * (src/iPregel_postamble.h:43-546 and each version's ip_run), plus the C ABI
 * that every application library exports (ipg_app_*), used by the Python
 * package and the benchmark to drive the same code path without files.
 *
 * Errors follow the reference: a message on stdout and exit(-1)
 * (iPregel_postamble.h:117-174).  The ipg_app_* entry points return status
 * codes instead.
 */
#ifndef IPREGEL_B200_HOST_CUH
#define IPREGEL_B200_HOST_CUH

#include <sys/time.h>

#include <string>
#include <vector>

#define STRINGIFY(x) STRINGIFY_LITERAL(x)
#define STRINGIFY_LITERAL(x) #x

#ifdef IPG_APP_SHARED
/* The application's main, renamed by -Dmain=ipg_app_main, keeps C linkage. */
extern "C" int ipg_app_main(int argc, char* argv[]);
#endif
#ifdef IP_APP_PARAMS
/* Optional application hook: set a named parameter before ip_run. */
extern "C" int ip_app_set_param(const char* key, double value);
#endif
#ifdef IP_APP_PARAM_PTRS
/* Optional application hook: a named device array of n entries. */
extern "C" int ip_app_set_param_ptr(const char* key, const void* ptr, uint64_t n);
#endif

static bool ipx_env_flag(const char* name)
{
    const char* v = getenv(name);
    return v && *v && atoi(v) != 0;
}

static uint64_t ipx_env_u64(const char* name, uint64_t dflt)
{
    const char* v = getenv(name);
    return (v && *v) ? strtoull(v, nullptr, 10) : dflt;
}

static double ipx_wtime()
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

/* ---- engine host state ---- */
struct ipx_host_state {
    ipg_graph* g = nullptr;  /* the caller's graph (contents checks, ownership) */
    bool own_graph = false;
    /* the graph the kernels run on: g, or its degree-ordered copy (owned by
     * g), with the id maps of the copy (null for g) */
    ipg_graph* gw = nullptr;
    const uint32_t* vid_of = nullptr;
    const uint32_t* vindex_of = nullptr;
    /* run on the degree-ordered copy (ipg_app_set_order; IPG_ORDER=0 turns
     * the default off) */
    bool order = ipx_env_u64("IPG_ORDER", 1) != 0;
    ipx_val* values_by_id = nullptr; /* the values in the caller's numbering */
    ipg_graph_view gv;
    uint64_t graph_generation = 0; /* the graph's contents generation at attach */
    ipx_consts c;
    std::vector<std::pair<void*, uint64_t>> allocs;
    /* device buffers of the previous attachment, kept through a re-attach:
     * ipx_alloc takes one of exactly the size it needs before allocating,
     * so re-attaching a graph of the same shape allocates and frees nothing
     * (cudaFree synchronises the whole device) */
    std::vector<std::pair<void*, uint64_t>> spare;
    uint32_t* blist[3] = {nullptr, nullptr, nullptr};  /* broadcaster classes */
    uint32_t* tlist[3] = {nullptr, nullptr, nullptr};  /* frontier / target classes */
    uint32_t* lcnt = nullptr;                          /* [0..2] broadcaster, [4..6] targets */
    uint32_t* hub_prefix = nullptr;                    /* chunk prefix of the broadcaster hubs */
    uint32_t* pull_prefix = nullptr;                   /* chunk prefix of the static in-degree hubs */
    unsigned long long pull_threshold = 0;             /* pull when broadcaster edges exceed this */
    unsigned long long* h_ctr = nullptr;               /* pinned mirror of ctr */
    uint32_t* h_lcnt = nullptr;                        /* pinned mirror of lcnt */
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ipg_bins gbins;                                    /* static in-degree classes (pull) */
    std::vector<uint64_t> counts;
    double total_seconds = 0.0;
    uint64_t edges = 0;
    uint64_t pulled_supersteps = 0;
    bool quiet = false;
    bool ready = false;
    bool dirty = false;
    /* Runtime tuning, applied at the next attach: CTA size of the superstep
     * kernels, degree-class thresholds (thread up to t0 edges, warp up to
     * t1, CTAs beyond) and the pull switch of the push versions (pull when
     * the broadcasters' edges exceed E / pull_div; 0 never). */
    struct {
        int block = IPX_THREADS;
        uint64_t t0 = IPX_T0, t1 = IPX_T1;
        uint64_t pull_div = ipx_env_u64("IPG_PULL_DIV", 0);
    } tune;
    int tb = IPX_THREADS;      /* CTA size in use */
    uint32_t grid_compute = 0; /* resident CTAs of the compute kernel */
    uint32_t grid_edge = 0;    /* resident CTAs of the edge kernels */
    uint32_t grid_gather[3] = {0, 0, 0}; /* single_broadcast: of each class's fused kernel */
    std::vector<struct ip_vertex_t> host_vertices;
    bool host_valid = false;
    char err[512] = {0};
    /* profiling */
    bool profile = false;
    uint64_t prof_launches[IPX_K_N] = {0};
    uint64_t prof_timed[IPX_K_N] = {0};
    double prof_ms[IPX_K_N] = {0};
    double prof_bytes[IPX_K_N] = {0};
    double prof_edges[IPX_K_N] = {0};  /* edges walked (push, mark, gather kernels) */
#define IPX_PEV 32
    cudaEvent_t pev[2][IPX_PEV];
    int pkid[IPX_PEV];
    int npev = 0;
    bool pev_made = false;
    /* captured superstep loop */
    bool graph_loop = ipx_env_flag("IPG_GRAPH_LOOP"); /* read once, at load */
    cudaGraphExec_t gexec = nullptr;
    uint64_t body_launches[IPX_K_N] = {0};
    uint64_t graph_launches = 0;
};
static ipx_host_state ipx_h;

static int ipx_fail(int code, const char* msg)
{
    snprintf(ipx_h.err, sizeof ipx_h.err, "%s", msg);
    return code;
}

#define IPX_CU(call)                                                                   \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            snprintf(ipx_h.err, sizeof ipx_h.err, "%s: %s", #call, cudaGetErrorString(e_)); \
            return IPG_ECUDA;                                                          \
        }                                                                              \
    } while (0)

#define IPX_OK(call)                                                                   \
    do {                                                                               \
        int r_ = (call);                                                               \
        if (r_ != IPG_OK) {                                                            \
            if (!ipx_h.err[0]) snprintf(ipx_h.err, sizeof ipx_h.err, "%s", ipg_last_error()); \
            return r_;                                                                 \
        }                                                                              \
    } while (0)

template <class T>
static int ipx_alloc(T** p, uint64_t n)
{
    void* d = nullptr;
    uint64_t bytes = (n ? n : 1) * sizeof(T);
    for (size_t i = 0; i < ipx_h.spare.size(); i++)
        if (ipx_h.spare[i].second == bytes) {
            d = ipx_h.spare[i].first;
            ipx_h.spare[i] = ipx_h.spare.back();
            ipx_h.spare.pop_back();
            break;
        }
    int r = d ? IPG_OK : ipg_dev_alloc(&d, bytes);
    if (r != IPG_OK) {
        snprintf(ipx_h.err, sizeof ipx_h.err, "%s", ipg_last_error());
        return r;
    }
    ipx_h.allocs.push_back({d, bytes});
    *p = (T*)d;
    return IPG_OK;
}

static void ipx_free_spares()
{
    for (auto& a : ipx_h.spare) ipg_dev_free(a.first, a.second);
    ipx_h.spare.clear();
}

/* keep = true (a re-attach): the device buffers become spares for the next
 * setup instead of being freed. */
static void ipx_release_state(bool keep = false)
{
    if (keep) {
        ipx_h.spare.insert(ipx_h.spare.end(), ipx_h.allocs.begin(), ipx_h.allocs.end());
    } else {
        for (auto& a : ipx_h.allocs) ipg_dev_free(a.first, a.second);
        ipx_free_spares();
    }
    ipx_h.allocs.clear();
    if (ipx_h.gexec) cudaGraphExecDestroy(ipx_h.gexec);
    ipx_h.gexec = nullptr;
    if (!keep) { /* a re-attach keeps the stream, events and pinned words too */
        if (ipx_h.h_ctr) cudaFreeHost(ipx_h.h_ctr);
        if (ipx_h.h_lcnt) cudaFreeHost(ipx_h.h_lcnt);
        ipx_h.h_ctr = nullptr;
        ipx_h.h_lcnt = nullptr;
        if (ipx_h.ev0) cudaEventDestroy(ipx_h.ev0);
        if (ipx_h.ev1) cudaEventDestroy(ipx_h.ev1);
        if (ipx_h.st) cudaStreamDestroy(ipx_h.st);
        ipx_h.ev0 = ipx_h.ev1 = nullptr;
        ipx_h.st = nullptr;
    }
    if (ipx_h.g && ipx_h.own_graph) ipg_graph_free(ipx_h.g);
    ipx_h.g = nullptr;
    ipx_h.gw = nullptr;
    ipx_h.vid_of = ipx_h.vindex_of = nullptr;
    ipx_h.values_by_id = nullptr;
    ipx_h.ready = false;
    ipx_h.host_valid = false;
    ipx_h.host_vertices.clear();
    ipx_h.host_vertices.shrink_to_fit();
}

static uint32_t ipx_grid(int per_sm = 8) { return (uint32_t)(ipg_sm_count() * per_sm); }

/* Grid of a grid-stride kernel: the CTAs resident at once (at most per_sm
 * per SM); a larger grid would run a second wave after the first CTAs
 * finished their static shares. */
template <class K>
static uint32_t ipx_resident_grid(K kernel, int block, int per_sm)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, 0) != cudaSuccess || n <= 0) n = 1;
    return ipx_grid(n < per_sm ? n : per_sm);
}

/* First degree threshold of the broadcaster classes. */
static uint64_t ipx_push_t0() { return IPX_PUSH_EXPAND ? ipx_h.tune.t1 : ipx_h.tune.t0; }

/* ip_init_vertex_range (combiner_postamble.h:89-117 and the other versions):
 * every per-vertex flag back to its initial value. */
static int ipx_reset_vertex_state()
{
    const ipx_consts& c = ipx_h.c;
    const uint64_t V = c.V;
    [[maybe_unused]] const uint64_t W = c.W;
    cudaStream_t st = ipx_h.st;
    if (V) {
        ipx_k_init_values<<<ipx_grid(), IPX_THREADS, 0, st>>>(0, V - 1);
        IPX_CU(cudaGetLastError());
    }
#if IPX_VERSION == IPX_COMBINER
    if (W) ipx_k_fill_bits<<<ipx_grid(), IPX_THREADS, 0, st>>>(c.active_bm, V, W);
    IPX_CU(cudaMemsetAsync(c.hasmsg_bm, 0, W * 4 + 4, st));
    IPX_CU(cudaMemsetAsync(c.recv[0], 0, W * 4 + 4, st));
    IPX_CU(cudaMemsetAsync(c.recv[1], 0, W * 4 + 4, st));
    IPX_CU(cudaMemsetAsync(c.bcaster, 0, W * 4 + 4, st));
#elif IPX_VERSION == IPX_SPREAD
    IPX_CU(cudaMemsetAsync(c.recv[0], 0, W * 4 + 4, st));
    IPX_CU(cudaMemsetAsync(c.recv[1], 0, W * 4 + 4, st));
    IPX_CU(cudaMemsetAsync(c.bcaster, 0, W * 4 + 4, st));
#elif IPX_VERSION == IPX_SINGLE_BROADCAST
    /* every stamp IPX_NO_STAMP: no slot counts in any superstep */
    IPX_CU(cudaMemsetAsync(c.sbslot[0], 0xff, (V ? V : 1) * sizeof(ipx_sbslot), st));
    IPX_CU(cudaMemsetAsync(c.sbslot[1], 0xff, (V ? V : 1) * sizeof(ipx_sbslot), st));
    IPX_CU(cudaMemsetAsync(c.hub_arrived, 0, (ipx_h.gbins.count[2] + 1) * sizeof(uint32_t), st));
#else
    IPX_CU(cudaMemsetAsync(c.hasmsg_b, 0, V + 1, st));
    IPX_CU(cudaMemsetAsync(c.bslot[0], 0xff, (V ? V : 1) * sizeof(ipx_bslot), st));
    IPX_CU(cudaMemsetAsync(c.bt, 0, W * 4 + 4, st));
    IPX_CU(cudaMemsetAsync(c.bcaster, 0, W * 4 + 4, st));
#endif
    IPX_CU(cudaMemsetAsync(c.ctr, 0, IPX_NCTR * sizeof(unsigned long long), st));
    IPX_CU(cudaMemsetAsync(ipx_h.lcnt, 0, 8 * sizeof(uint32_t), st));
    IPX_CU(cudaStreamSynchronize(st));
    ip_superstep = 0;
    ip_active_vertices = V;
    ipx_h.counts.clear();
    ipx_h.total_seconds = 0.0;
    ipx_h.edges = 0;
    ipx_h.pulled_supersteps = 0;
    ipx_h.dirty = false;
    ipx_h.host_valid = false;
    return IPG_OK;
}

#if IPX_VERSION == IPX_SINGLE_BROADCAST
/* The flagged copy of the in-lists (ipx_consts::in_adj_hot): the vertices
 * gathered most often, as many as IPG_SB_HOT_KB kilobytes of slots hold
 * (0, the default: no copy; on directed R-MAT scale 25, FP64 PageRank took
 * 158 ms with 32 to 96 MiB flagged against 137 ms without), have IPX_HOT_BIT set in their ids.  Needs
 * 32-bit ids and V < 2^31; skipped, not failed, when the copy (4 bytes per
 * edge) does not fit. */
static int ipx_build_hot_ids(ipx_consts& c)
{
    c.in_adj_hot = nullptr;
    const uint64_t kb = ipx_env_u64("IPG_SB_HOT_KB", 0);
    if (sizeof(ipx_vid) != 4 || kb == 0 || c.V == 0 || c.E == 0 || c.V >= (1ULL << 31)) return IPG_OK;
    const uint64_t hot_vertices = (kb << 10) / sizeof(ipx_sbslot);
    void* cnt = nullptr;
    const uint64_t hist_off = (c.V * 4 + 7) & ~7ULL, tmp_bytes = hist_off + 33 * 8;
    if (ipg_dev_alloc(&cnt, tmp_bytes) != IPG_OK) return IPG_OK;
    unsigned long long* hist = (unsigned long long*)((char*)cnt + hist_off);
    uint32_t* out = nullptr;
    if (ipx_alloc(&out, c.E) != IPG_OK) {
        ipx_h.err[0] = 0;
        ipg_dev_free(cnt, tmp_bytes);
        return IPG_OK;
    }
    int r = IPG_OK;
    unsigned long long h[33];
    cudaError_t e = cudaMemset(cnt, 0, tmp_bytes);
    if (e == cudaSuccess) {
        ipx_k_count_occurrences<<<ipx_grid(8), 256>>>((const uint32_t*)c.in_adj, c.E, (uint32_t*)cnt);
        ipx_k_count_hist<<<ipx_grid(8), 256>>>((const uint32_t*)cnt, c.V, hist);
        e = cudaMemcpy(h, hist, sizeof h, cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess) {
        /* the least b whose classes [b, 32] hold at most hot_vertices */
        int b = 33;
        uint64_t n = 0;
        while (b > 1 && n + h[b - 1] <= hot_vertices) n += h[--b];
        const uint32_t threshold = b > 32 ? 0xffffffffu : (1u << (b - 1));
        ipx_k_flag_hot<<<ipx_grid(8), 256>>>((const uint32_t*)c.in_adj, c.E, (const uint32_t*)cnt, threshold, out);
        e = cudaDeviceSynchronize();
    }
    ipg_dev_free(cnt, tmp_bytes);
    if (e != cudaSuccess) r = ipx_fail(IPG_ECUDA, cudaGetErrorString(e));
    else c.in_adj_hot = out;
    return r;
}
#else
static int ipx_build_hot_ids(ipx_consts&) { return IPG_OK; }
#endif

/* Allocates the version's device state for the attached graph. */
static int ipx_setup_state()
{
    ipx_consts& c = ipx_h.c;
    memset(&c, 0, sizeof c);
    ipx_h.tb = ipx_h.tune.block;
    const ipg_graph_view& gv = ipx_h.gv;
    if (gv.id_bytes != (int)sizeof(ipx_vid)) return ipx_fail(IPG_EINVAL, "graph id width differs from IP_VERTEX_ID_TYPE");
    const uint64_t V = gv.V, W = (V + 31) / 32;
    c.V = V;
    c.E = gv.E;
    c.W = W;
    c.row = gv.d_row;
    c.adj = (const ipx_vid*)gv.d_adj;
    c.wgt = (const ipx_wgt*)gv.d_wgt;
    c.in_row = gv.has_in ? gv.d_in_row : gv.d_row;
    c.in_adj = (const ipx_vid*)(gv.has_in ? gv.d_in_adj : gv.d_adj);
    c.in_wgt = (const ipx_wgt*)(gv.has_in ? gv.d_in_wgt : gv.d_wgt);
    c.vid_of = ipx_h.vid_of;
    c.vindex_of = ipx_h.vindex_of;
    if (ipx_h.vid_of) {
        /* the caller's rows, for the neighbour ids ip_compute reads */
        ipg_graph_view u;
        IPX_OK(ipg_graph_view_get(ipx_h.g, &u));
        c.user_row = u.d_row;
        c.user_adj = (const ipx_vid*)u.d_adj;
        c.user_in_row = u.has_in ? u.d_in_row : u.d_row;
        c.user_in_adj = (const ipx_vid*)(u.has_in ? u.d_in_adj : u.d_adj);
    }
    if (IPX_WEIGHT_BYTES && !gv.d_wgt)
        return ipx_fail(IPG_EINVAL, "the application needs edge weights: load the graph with weighted = true");
    if (IPX_WEIGHT_BYTES && gv.weight_bytes != IPX_WEIGHT_BYTES)
        return ipx_fail(IPG_EINVAL, "graph weight width differs from IP_EDGE_WEIGHT_TYPE");
    if (!ipx_h.st) IPX_CU(cudaStreamCreateWithFlags(&ipx_h.st, cudaStreamNonBlocking));
    if (!ipx_h.ev0) IPX_CU(cudaEventCreate(&ipx_h.ev0));
    if (!ipx_h.ev1) IPX_CU(cudaEventCreate(&ipx_h.ev1));
    if (!ipx_h.h_ctr)
        IPX_CU(cudaHostAlloc((void**)&ipx_h.h_ctr, IPX_NCTR * sizeof(unsigned long long), cudaHostAllocDefault));
    if (!ipx_h.h_lcnt) IPX_CU(cudaHostAlloc((void**)&ipx_h.h_lcnt, 8 * sizeof(uint32_t), cudaHostAllocDefault));
    IPX_OK(ipx_alloc(&c.value, V));
    if (ipx_h.vindex_of) IPX_OK(ipx_alloc(&ipx_h.values_by_id, V));
    IPX_OK(ipx_alloc(&c.ctr, IPX_NCTR));
    c.err = (uint32_t*)(c.ctr + IPX_CTR_ERR);
    IPX_OK(ipx_alloc(&ipx_h.lcnt, 8));
    c.lcnt = ipx_h.lcnt;
    IPX_OK(ipx_alloc(&c.hist, (uint64_t)IPX_HIST * 4));
    IPX_OK(ipx_alloc(&ipx_h.hub_prefix, gv.E / (ipx_h.tune.t1 + 1) + 2));
#if !IPX_PULL || IPX_VERSION == IPX_SPREAD_SINGLE_BROADCAST
    {
        /* the chunks of this superstep's broadcaster hubs: at most E / chunk
         * + one partial chunk per hub */
        uint32_t* owner = nullptr;
        IPX_OK(ipx_alloc(&owner, gv.E / IPX_HUB_CHUNK + gv.E / (ipx_h.tune.t1 + 1) + 2));
        c.push_owner = owner;
    }
#endif
#if IPX_VERSION == IPX_COMBINER
    IPX_OK(ipx_alloc(&c.active_bm, W + 1));
    IPX_OK(ipx_alloc(&c.hasmsg_bm, W + 1));
    IPX_OK(ipx_alloc(&c.msg, V));
#endif
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SPREAD
    IPX_OK(ipx_alloc(&c.mbox[0], V));
    IPX_OK(ipx_alloc(&c.mbox[1], V));
    IPX_OK(ipx_alloc(&c.recv[0], W + 1));
#if IPX_VERSION == IPX_COMBINER
    IPX_OK(ipx_alloc(&c.recv[1], W + 1));
#else
    c.recv[1] = c.recv[0]; /* compacted (and cleared) every superstep */
#endif
    IPX_OK(ipx_alloc(&c.outbox, V));
    IPX_OK(ipx_alloc(&c.bcaster, W + 1));
    for (int k = 0; k < 3; k++) IPX_OK(ipx_alloc(&ipx_h.blist[k], V));
#endif
#if IPX_VERSION == IPX_SPREAD
    IPX_OK(ipx_alloc(&ipx_h.tlist[0], V));
#endif
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SPREAD
    /* Direction optimisation: a dense superstep may deliver by pulling over
     * the in-lists, when they list exactly the vertices that would push:
     * on a symmetric graph (weights included), whose rows are the in-lists,
     * or on a directed graph with its transpose built.  tune.pull_div (the
     * IPG_PULL_DIV environment variable by default) sets the switch point:
     * pull when the broadcasters' out-edges exceed E / pull_div.  Default 0,
     * never pull: on R-MAT scale 24 every threshold measured slower than
     * pushing with the cached precheck. */
    {
        const unsigned long long div = ipx_h.tune.pull_div;
        const bool in_exact = gv.symmetric || (gv.directed && gv.has_in);
        c.pull_ok = (in_exact && div > 0 && V > 0) ? 1 : 0;
        ipx_h.pull_threshold = div ? gv.E / div : ~0ULL;
    }
    if (c.pull_ok) {
        IPX_OK(ipg_graph_bins(ipx_h.gw, gv.directed ? 1 : 0, ipx_h.tune.t0, ipx_h.tune.t1, &ipx_h.gbins));
        IPX_OK(ipx_alloc(&ipx_h.pull_prefix, ipx_h.gbins.count[2] + 2));
        uint32_t* dcount = nullptr;
        IPX_OK(ipx_alloc(&dcount, 1));
        const uint32_t n2 = (uint32_t)ipx_h.gbins.count[2];
        IPX_CU(cudaMemcpy(dcount, &n2, 4, cudaMemcpyHostToDevice));
        uint32_t* owner = nullptr;
        IPX_OK(ipx_alloc(&owner, ipx_h.gbins.edges[2] / IPX_HUB_CHUNK + n2 + 1));
        ipx_k_hub_prefix<><<<1, 1024>>>(ipx_h.gbins.d_list[2], dcount, c.in_row, ipx_h.pull_prefix, owner);
        IPX_CU(cudaGetLastError());
        IPX_CU(cudaDeviceSynchronize());
        c.hub_owner = owner;
    }
#endif
#if IPX_VERSION == IPX_SPREAD_SINGLE_BROADCAST
    IPX_OK(ipx_alloc(&c.hasmsg_b, V + 1));
    IPX_OK(ipx_alloc(&c.msg, V));
    IPX_OK(ipx_alloc(&c.bslot[0], V));
#endif
#if IPX_VERSION == IPX_SINGLE_BROADCAST
    IPX_OK(ipx_alloc(&c.sbslot[0], V));
    IPX_OK(ipx_alloc(&c.sbslot[1], V));
    IPX_OK(ipx_alloc(&c.active_b, V + 1));
    IPX_OK(ipg_graph_bins(ipx_h.gw, 1, ipx_h.tune.t0, ipx_h.tune.t1, &ipx_h.gbins));
    {
        /* chunks of the hub class: prefix, partial folds, arrival counters */
        const ipg_bins& b = ipx_h.gbins;
        const uint64_t n2 = b.count[2];
        const uint64_t max_chunks = b.edges[2] / IPX_GATHER_CHUNK + n2 + 1;
        IPX_OK(ipx_alloc(&ipx_h.pull_prefix, n2 + 2));
        IPX_OK(ipx_alloc(&c.hub_part, max_chunks));
        IPX_OK(ipx_alloc(&c.hub_arrived, n2 + 1));
        IPX_CU(cudaMemset(c.hub_arrived, 0, (n2 + 1) * sizeof(uint32_t)));
        uint32_t* dcount = nullptr;
        IPX_OK(ipx_alloc(&dcount, 1));
        const uint32_t n2u = (uint32_t)n2;
        IPX_CU(cudaMemcpy(dcount, &n2u, 4, cudaMemcpyHostToDevice));
        uint32_t* owner = nullptr;
        IPX_OK(ipx_alloc(&owner, max_chunks));
        ipx_k_hub_prefix<IPX_GATHER_CHUNK><<<1, 1024>>>(b.d_list[2], dcount, c.in_row, ipx_h.pull_prefix, owner);
        IPX_CU(cudaGetLastError());
        IPX_CU(cudaDeviceSynchronize());
        c.hub_owner = owner;
    }
    IPX_OK(ipx_build_hot_ids(c));
#endif
#if IPX_VERSION == IPX_SPREAD_SINGLE_BROADCAST
    IPX_OK(ipx_alloc(&c.bt, W + 1));
    IPX_OK(ipx_alloc(&c.bcaster, W + 1));
    for (int k = 0; k < 3; k++) IPX_OK(ipx_alloc(&ipx_h.blist[k], V));
    for (int k = 0; k < 3; k++) IPX_OK(ipx_alloc(&ipx_h.tlist[k], V));
#endif
    IPX_CU(cudaMemcpyToSymbol(ipx_c, &c, sizeof c));
    size_t vc = V, ec = gv.E;
    IPX_CU(cudaMemcpyToSymbol(ipd_vertices_count, &vc, sizeof vc));
    IPX_CU(cudaMemcpyToSymbol(ipd_edges_count, &ec, sizeof ec));
#if IP_COMBINE_KIND != IP_COMBINE_GENERIC
    IPX_CU(cudaMemset(c.err, 0, 4));
    ipx_k_check_hint<<<16, IPX_THREADS>>>(IP_COMBINE_KIND);
    IPX_CU(cudaGetLastError());
    uint32_t herr = 0;
    IPX_CU(cudaMemcpy(&herr, c.err, 4, cudaMemcpyDeviceToHost));
    if (herr & IPX_ERR_COMBINE_HINT)
        return ipx_fail(IPG_EINVAL, "IP_COMBINE_KIND disagrees with ip_combine on sample messages");
#endif
    {
        const int tb = ipx_h.tb;
        const int per_sm = 2048 / tb;
#if IPX_VERSION == IPX_COMBINER
        ipx_h.grid_compute = ipx_resident_grid(ipx_k_compute_combiner, tb, per_sm);
        ipx_h.grid_edge = ipx_resident_grid(ipx_k_push<1>, tb, per_sm);
#elif IPX_VERSION == IPX_SPREAD
        ipx_h.grid_compute = ipx_resident_grid(ipx_k_compute_spread, tb, per_sm);
        ipx_h.grid_edge = ipx_resident_grid(ipx_k_push<1>, tb, per_sm);
#elif IPX_VERSION == IPX_SINGLE_BROADCAST
        ipx_h.grid_compute = ipx_resident_grid(ipx_k_compute_sb0, tb, per_sm);
        if (c.in_adj_hot) {
            ipx_h.grid_edge = ipx_resident_grid(ipx_k_gather_compute<1, true>, tb, per_sm);
            ipx_h.grid_gather[0] = ipx_resident_grid(ipx_k_gather_compute<0, true>, tb, per_sm);
            ipx_h.grid_gather[2] = ipx_resident_grid(ipx_k_gather_compute<2, true>, tb, per_sm);
        } else {
            ipx_h.grid_edge = ipx_resident_grid(ipx_k_gather_compute<1, false>, tb, per_sm);
            ipx_h.grid_gather[0] = ipx_resident_grid(ipx_k_gather_compute<0, false>, tb, per_sm);
            ipx_h.grid_gather[2] = ipx_resident_grid(ipx_k_gather_compute<2, false>, tb, per_sm);
        }
        ipx_h.grid_gather[1] = ipx_h.grid_edge;
#else
        ipx_h.grid_compute = ipx_resident_grid(ipx_k_compute_ssb, tb, per_sm);
        ipx_h.grid_edge = ipx_resident_grid(ipx_k_gather<1, false>, tb, per_sm);
#endif
    }
    ipx_h.ready = true;
    return ipx_reset_vertex_state();
}

static int ipx_attach(ipg_graph* g, bool own)
{
    ipx_release_state(true);
    ipx_h.err[0] = 0;
    ipx_h.g = g;
    ipx_h.own_graph = own;
    IPX_OK(ipg_graph_view_get(g, &ipx_h.gv));
    int valid = 1;
    IPX_OK(ipg_graph_contents(g, &ipx_h.graph_generation, &valid));
    if (!valid) {
        ipx_h.g = nullptr;
        ipx_h.own_graph = false;
        return ipx_fail(IPG_EINVAL, "the graph's contents failed validation at its last refill");
    }
    bool need_in = IPX_PULL
#if defined(IP_NEEDS_IN_NEIGHBOUR_IDS) || defined(IP_NEEDS_IN_NEIGHBOUR_COUNT) || IPX_IN_WEIGHTS
                   || true
#endif
        ;
    /* the push versions pull over the transpose of a directed graph */
    if (!IPX_PULL && ipx_h.tune.pull_div > 0 && ipx_h.gv.directed) need_in = true;
    ipx_h.gw = g;
    if (ipx_h.order && ipx_h.gv.V < (1ULL << 31)) {
        /* the kernels run on the degree-ordered copy; a copy that does not
         * fit the HBM budget leaves the graph's own numbering */
        ipg_order o;
        const int r = ipg_graph_degree_order(g, need_in ? 1 : 0, &o);
        if (r == IPG_OK) {
            ipx_h.gw = o.graph;
            ipx_h.vid_of = o.d_old_of_new;
            ipx_h.vindex_of = o.d_new_of_old;
        } else if (r != IPG_EBUDGET && r != IPG_ENOMEM) {
            return ipx_fail(r, ipg_last_error());
        }
    }
    if (need_in && ipx_h.gw == g && !ipx_h.gv.has_in) IPX_OK(ipg_graph_build_in(g));
    IPX_OK(ipg_graph_view_get(ipx_h.gw, &ipx_h.gv));
    ip_set_vertices_count(ipx_h.gv.V);
    ip_set_edges_count(ipx_h.gv.E);
    int r = ipx_setup_state();
    ipx_free_spares(); /* the previous attachment's buffers this one did not take */
    if (r != IPG_OK) {
        ipx_h.own_graph = own;
        ipx_release_state();
    }
    return r;
}

/* ---- superstep loop ---- */
static int ipx_set_superstep(uint64_t s)
{
    size_t v = s;
    IPX_CU(cudaMemcpyToSymbolAsync(ipd_superstep, &v, sizeof v, 0, cudaMemcpyHostToDevice, ipx_h.st));
    IPX_CU(cudaMemcpyToSymbolAsync(ipd_compute_superstep, &v, sizeof v, 0, cudaMemcpyHostToDevice, ipx_h.st));
    return IPG_OK;
}

static int ipx_push_class(int k, uint32_t g);
static int ipx_deliver_superstep(uint32_t ge);

/* ---- per-kernel profiling (the role of IP_ENABLE_THREAD_PROFILING in the
 * reference, e.g. combiner_spread_postamble.h:166-178, :353-401): every
 * launch is counted; with profiling on, each is bracketed by events and its
 * algorithmic bytes are added from the sizes read back after the superstep. */
static void ipx_k_begin(int kid)
{
    ipx_h.prof_launches[kid]++;
    if (ipx_h.profile && ipx_h.npev < IPX_PEV) {
        cudaEventRecord(ipx_h.pev[0][ipx_h.npev], ipx_h.st);
        ipx_h.pkid[ipx_h.npev] = kid;
    }
}

static void ipx_k_end()
{
    if (ipx_h.profile && ipx_h.npev < IPX_PEV) {
        cudaEventRecord(ipx_h.pev[1][ipx_h.npev], ipx_h.st);
        ipx_h.npev++;
    }
}

#define IPX_LAUNCH(kid, ...)       \
    do {                           \
        ipx_k_begin(kid);          \
        __VA_ARGS__;               \
        ipx_k_end();               \
    } while (0)

static int ipx_push_class(int k, uint32_t g)
{
    cudaStream_t st = ipx_h.st;
    uint32_t* pre = ipx_h.hub_prefix;
    if (k == 0) IPX_LAUNCH(IPX_K_PUSH0, ipx_k_push<0><<<g, ipx_h.tb, 0, st>>>(ipx_h.blist[0], ipx_h.lcnt + 0, pre));
    if (k == 1) IPX_LAUNCH(IPX_K_PUSH1, ipx_k_push<1><<<g, ipx_h.tb, 0, st>>>(ipx_h.blist[1], ipx_h.lcnt + 1, pre));
    if (k == 2) {
        IPX_LAUNCH(IPX_K_CTRL, ipx_k_hub_prefix<><<<1, 1024, 0, st>>>(ipx_h.blist[2], ipx_h.lcnt + 2, ipx_h.c.row, pre,
                                                                       (uint32_t*)ipx_h.c.push_owner));
        IPX_LAUNCH(IPX_K_PUSH2, ipx_k_push<2><<<g, ipx_h.tb, 0, st>>>(ipx_h.blist[2], ipx_h.lcnt + 2, pre));
    }
    IPX_CU(cudaGetLastError());
    return IPG_OK;
}

/* Delivery of the superstep's broadcasts (push versions): compact the
 * broadcasters into degree classes, then push along their rows, or, on a
 * symmetric graph when their out-edges pass the threshold, pull over every
 * row.  The direction is chosen on the device (ipx_k_decide); the kernels of
 * the other direction return at once. */
static int ipx_deliver_superstep(uint32_t ge)
{
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SPREAD
    const ipx_consts& c = ipx_h.c;
    cudaStream_t st = ipx_h.st;
    uint64_t* edges_b = (uint64_t*)(c.ctr + 8);
    IPX_LAUNCH(IPX_K_COMPACT_B, IPX_OK(ipg_compact(c.bcaster, c.V, c.row, ipx_push_t0(), ipx_h.tune.t1, ipx_h.blist[0],
                                                   ipx_h.blist[1], ipx_h.blist[2], ipx_h.lcnt, edges_b,
                                                   c.pull_ok ? 0 : 1, st)));
    if (c.pull_ok) IPX_LAUNCH(IPX_K_CTRL, ipx_k_decide<<<1, 1, 0, st>>>(ipx_h.pull_threshold));
    for (int k = 0; k < 3; k++) IPX_OK(ipx_push_class(k, ge));
    if (c.pull_ok) {
        const ipg_bins& b = ipx_h.gbins;
        IPX_LAUNCH(IPX_K_PULLD0, ipx_k_pull_deliver<0><<<ge, ipx_h.tb, 0, st>>>(b.d_list[0], b.count[0],
                                                                                   ipx_h.pull_prefix));
        IPX_LAUNCH(IPX_K_PULLD1, ipx_k_pull_deliver<1><<<ge, ipx_h.tb, 0, st>>>(b.d_list[1], b.count[1],
                                                                                   ipx_h.pull_prefix));
        IPX_LAUNCH(IPX_K_PULLD2, ipx_k_pull_deliver<2><<<ge, ipx_h.tb, 0, st>>>(b.d_list[2], b.count[2],
                                                                                   ipx_h.pull_prefix));
        IPX_CU(cudaMemsetAsync(c.bcaster, 0, c.W * 4 + 4, st));
    }
    IPX_CU(cudaGetLastError());
#else
    (void)ge;
#endif
    return IPG_OK;
}

/* Algorithmic bytes of the superstep's kernels: the data each must move once
 * (ids, row offsets, values, messages, mailbox read-modify-writes, bitmap
 * bits), from the list sizes and degree sums of this superstep. */
static void ipx_account_bytes(uint64_t s, uint64_t frontier)
{
    const double V = (double)ipx_h.c.V;
    const double ib = sizeof(ipx_vid), vb = sizeof(ipx_val), mb = sizeof(ipx_msg), sb = sizeof(ipx_slot);
    const double wb = IPX_EDGE_MSG ? (double)IPX_WEIGHT_BYTES : 0.0;
    [[maybe_unused]] const unsigned long long* ctr = ipx_h.h_ctr;
    [[maybe_unused]] const uint32_t* l = ipx_h.h_lcnt;
    double* B = ipx_h.prof_bytes;
    double* N = ipx_h.prof_edges;
    (void)s;
    (void)sb;
    (void)wb;
    (void)N;
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SPREAD
    const double nb = (double)l[0] + l[1] + l[2];
    B[IPX_K_COMPUTE] += (IPX_VERSION == IPX_COMBINER ? V * 3.0 / 8.0 : frontier * 4.0) +
                        frontier * (2 * vb + sb) + nb * mb;
    B[IPX_K_COMPACT_B] += V / 8.0 + nb * 20.0;
    if (ipx_h.c.pull_ok && ctr[IPX_CTR_MODE]) {
        /* pulled: every row once, messages of the broadcasting neighbours */
        const ipg_bins& b = ipx_h.gbins;
        const double bedges = (double)ctr[8] + ctr[9] + ctr[10];
        const double E = ipx_h.c.E ? (double)ipx_h.c.E : 1.0;
        for (int k = 0; k < 3; k++)
            B[IPX_K_PULLD0 + k] +=
                b.count[k] * (4.0 + 16.0 + sb) + b.edges[k] * (ib + 0.125) + bedges * (mb + wb) * (b.edges[k] / E);
        for (int k = 0; k < 3; k++) N[IPX_K_PULLD0 + k] += b.edges[k];
    } else {
        for (int k = 0; k < 3; k++) B[IPX_K_PUSH0 + k] += l[k] * (20.0 + mb) + ctr[8 + k] * (ib + sb + wb);
        for (int k = 0; k < 3; k++) N[IPX_K_PUSH0 + k] += ctr[8 + k];
    }
#if IPX_VERSION == IPX_COMBINER
    B[IPX_K_COUNT] += V / 4.0;
#else
    B[IPX_K_COMPACT_T] += V / 8.0 + l[4] * 4.0;
#endif
#elif IPX_VERSION == IPX_SINGLE_BROADCAST
    /* superstep 0's compute: activity, value read and write, broadcast;
     * the fused kernels: per vertex its list entry, in-row bounds, activity
     * and value read + write, out-row bounds and a broadcast (the compute
     * phase of the next superstep); per in-edge its id and the gathered
     * message */
    const ipg_bins& b = ipx_h.gbins;
    (void)frontier;
    if (s == 0) B[IPX_K_COMPUTE] += V * (1.0 + 2 * vb + 16.0 + mb);
    for (int k = 0; k < 3; k++)
        B[IPX_K_GATHER0 + k] += b.count[k] * (4.0 + 16.0 + 1.0 + 2 * vb + mb) + b.edges[k] * (ib + mb);
    for (int k = 0; k < 3; k++) N[IPX_K_GATHER0 + k] += b.edges[k];
#else
    const double nb = (double)l[0] + l[1] + l[2];
    B[IPX_K_COMPUTE] += frontier * (4.0 + 2 * vb + 1 + mb) + nb * mb;
    B[IPX_K_COMPACT_B] += V / 8.0 + nb * 20.0;
    for (int k = 0; k < 3; k++) B[IPX_K_MARK0 + k] += l[k] * 20.0 + ctr[8 + k] * (ib + 0.125);
    for (int k = 0; k < 3; k++) N[IPX_K_MARK0 + k] += ctr[8 + k];
    B[IPX_K_COMPACT_T] += V / 8.0 + ((double)l[4] + l[5] + l[6]) * 20.0;
    for (int k = 0; k < 3; k++)
        B[IPX_K_GATHER0 + k] += l[4 + k] * (4.0 + 16.0 + 1.0 + mb) + ctr[11 + k] * (ib + mb + 0.125);
    for (int k = 0; k < 3; k++) N[IPX_K_GATHER0 + k] += ctr[11 + k];
#endif
}

static int ipx_end_superstep(uint64_t s, uint64_t* count, uint64_t frontier)
{
    cudaStream_t st = ipx_h.st;
    IPX_CU(cudaMemcpyAsync(ipx_h.h_ctr, ipx_h.c.ctr, IPX_NCTR * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    IPX_CU(cudaMemcpyAsync(ipx_h.h_lcnt, ipx_h.lcnt, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    IPX_CU(cudaEventRecord(ipx_h.ev1, st));
    IPX_CU(cudaEventSynchronize(ipx_h.ev1));
    IPX_CU(cudaGetLastError());
    uint32_t err = (uint32_t)(ipx_h.h_ctr[IPX_CTR_ERR] & 0xffffffffu);
    if (err & IPX_ERR_SEND_IN_BROADCAST)
        return ipx_fail(IPG_EDEVICE,
                        "The function send_message should not be used in the SINGLE_BROADCAST version; only "
                        "broadcast() should be called, and once per superstep maximum.");
    if (err & IPX_ERR_COPY_TIMEOUT)
        return ipx_fail(IPG_EDEVICE, "a bulk copy into shared memory did not complete in time (results kept exact)");
    if (err & IPX_ERR_RESERVED_MESSAGE)
        return ipx_fail(IPG_EDEVICE, "a broadcast FP64 message had all 64 bits set, the pattern the single_broadcast "
                                     "engine reserves for 'no broadcast' (build with -DIPX_SB_DENSE=0 to allow it)");
    if (err) return ipx_fail(IPG_EDEVICE, "a kernel reported an error");
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SINGLE_BROADCAST
    *count = ipx_h.h_ctr[s & 3];
#elif IPX_VERSION == IPX_SPREAD
    *count = ipx_h.h_lcnt[4];
#else
    *count = (uint64_t)ipx_h.h_lcnt[4] + ipx_h.h_lcnt[5] + ipx_h.h_lcnt[6];
#endif
#if IPX_VERSION == IPX_SINGLE_BROADCAST
    ipx_h.edges += ipx_h.c.E;
#else
    if (ipx_h.c.pull_ok && ipx_h.h_ctr[IPX_CTR_MODE]) {
        ipx_h.edges += ipx_h.c.E; /* a pulled superstep reads every row */
        ipx_h.pulled_supersteps++;
    } else {
        for (int k = 8; k < 11; k++) ipx_h.edges += ipx_h.h_ctr[k];
    }
    for (int k = 11; k < 14; k++) ipx_h.edges += ipx_h.h_ctr[k];
#endif
    if (ipx_h.profile) {
        for (int i = 0; i < ipx_h.npev; i++) {
            float kms = 0.f;
            IPX_CU(cudaEventElapsedTime(&kms, ipx_h.pev[0][i], ipx_h.pev[1][i]));
            ipx_h.prof_ms[ipx_h.pkid[i]] += kms;
            ipx_h.prof_timed[ipx_h.pkid[i]]++;
        }
        ipx_h.npev = 0;
        ipx_account_bytes(s, frontier);
    }
    float ms = 0.f;
    IPX_CU(cudaEventElapsedTime(&ms, ipx_h.ev0, ipx_h.ev1));
    double sec = ms * 1e-3;
    ipx_h.total_seconds += sec;
    ipx_h.counts.push_back(*count);
    ip_active_vertices = *count;
    if (!ipx_h.quiet) {
        printf("Superstep%zuDuration:%f\n", (size_t)s, sec);
        printf("Superstep%zuActiveVertexCount:%zu\n", (size_t)s, (size_t)*count);
    }
    return IPG_OK;
}

/* Enqueues one superstep's kernels on the engine stream.  Nothing here
 * depends on host-side values of the superstep: kernels read it (and the
 * mailbox parity) from device memory, so the same sequence serves the host
 * loop and the captured loop. */
static int ipx_enqueue_superstep()
{
    const ipx_consts& c = ipx_h.c;
    cudaStream_t st = ipx_h.st;
    const uint32_t g = ipx_h.grid_compute;
    const uint32_t ge = ipx_h.grid_edge;
    const uint64_t V = c.V;
    (void)V;
    (void)ge;
#if IPX_VERSION == IPX_SINGLE_BROADCAST
    /* superstep 0's compute phase (returns at once later), before
     * ipx_k_begin_superstep moves ip_get_superstep() to the next superstep */
    IPX_LAUNCH(IPX_K_COMPUTE, ipx_k_compute_sb0<<<g, ipx_h.tb, 0, st>>>());
#endif
    IPX_LAUNCH(IPX_K_CTRL, ipx_k_begin_superstep<<<1, 1, 0, st>>>());
#if IPX_VERSION == IPX_COMBINER
    IPX_LAUNCH(IPX_K_COMPUTE, ipx_k_compute_combiner<<<g, ipx_h.tb, 0, st>>>());
    IPX_CU(cudaMemsetAsync(ipx_h.lcnt, 0, 4 * sizeof(uint32_t), st));
    IPX_OK(ipx_deliver_superstep(ge));
    IPX_LAUNCH(IPX_K_COUNT, ipx_k_count_combiner<<<ipx_grid(4), 256, 0, st>>>());
#elif IPX_VERSION == IPX_SPREAD
    IPX_LAUNCH(IPX_K_COMPUTE, ipx_k_compute_spread<<<g, ipx_h.tb, 0, st>>>(ipx_h.tlist[0], ipx_h.lcnt + 4));
    IPX_CU(cudaMemsetAsync(ipx_h.lcnt, 0, 8 * sizeof(uint32_t), st));
    IPX_OK(ipx_deliver_superstep(ge));
    /* spread keeps one received bitmap (recv[0] == recv[1]): its compaction
     * clears it before the next superstep's sends */
    IPX_LAUNCH(IPX_K_COMPACT_T, IPX_OK(ipg_compact(c.recv[0], V, nullptr, 0, 0, ipx_h.tlist[0], nullptr, nullptr,
                                                   ipx_h.lcnt + 4, nullptr, 1, st)));
#elif IPX_VERSION == IPX_SINGLE_BROADCAST
    {
        /* gather of this superstep fused with the next one's compute phase */
        const ipg_bins& b = ipx_h.gbins;
        const bool hot = ipx_h.c.in_adj_hot != nullptr;
        if (b.count[0])
            IPX_LAUNCH(IPX_K_GATHER0, hot ? ipx_k_gather_compute<0, true><<<ipx_h.grid_gather[0], ipx_h.tb, 0, st>>>(
                                                b.d_list[0], b.count[0], nullptr)
                                          : ipx_k_gather_compute<0, false><<<ipx_h.grid_gather[0], ipx_h.tb, 0, st>>>(
                                                b.d_list[0], b.count[0], nullptr));
        if (b.count[1])
            IPX_LAUNCH(IPX_K_GATHER1, hot ? ipx_k_gather_compute<1, true><<<ipx_h.grid_gather[1], ipx_h.tb, 0, st>>>(
                                                b.d_list[1], b.count[1], nullptr)
                                          : ipx_k_gather_compute<1, false><<<ipx_h.grid_gather[1], ipx_h.tb, 0, st>>>(
                                                b.d_list[1], b.count[1], nullptr));
        if (b.count[2])
            IPX_LAUNCH(IPX_K_GATHER2, hot ? ipx_k_gather_compute<2, true><<<ipx_h.grid_gather[2], ipx_h.tb, 0, st>>>(
                                                b.d_list[2], b.count[2], ipx_h.pull_prefix)
                                          : ipx_k_gather_compute<2, false><<<ipx_h.grid_gather[2], ipx_h.tb, 0, st>>>(
                                                b.d_list[2], b.count[2], ipx_h.pull_prefix));
    }
#else
    uint64_t* edges_b = (uint64_t*)(c.ctr + 8);
    uint64_t* edges_t = (uint64_t*)(c.ctr + 11);
    IPX_LAUNCH(IPX_K_COMPUTE, ipx_k_compute_ssb<<<g, ipx_h.tb, 0, st>>>(ipx_h.tlist[0], ipx_h.tlist[1],
                                                                            ipx_h.tlist[2], ipx_h.lcnt + 4));
    IPX_CU(cudaMemsetAsync(ipx_h.lcnt, 0, 8 * sizeof(uint32_t), st));
    IPX_LAUNCH(IPX_K_COMPACT_B, IPX_OK(ipg_compact(c.bcaster, V, c.row, ipx_push_t0(), ipx_h.tune.t1, ipx_h.blist[0],
                                                   ipx_h.blist[1], ipx_h.blist[2], ipx_h.lcnt, edges_b, 1, st)));
    IPX_LAUNCH(IPX_K_MARK0, ipx_k_mark<0><<<ge, ipx_h.tb, 0, st>>>(ipx_h.blist[0], ipx_h.lcnt + 0, ipx_h.hub_prefix));
    IPX_LAUNCH(IPX_K_MARK1, ipx_k_mark<1><<<ge, ipx_h.tb, 0, st>>>(ipx_h.blist[1], ipx_h.lcnt + 1, ipx_h.hub_prefix));
    IPX_LAUNCH(IPX_K_CTRL, ipx_k_hub_prefix<><<<1, 1024, 0, st>>>(ipx_h.blist[2], ipx_h.lcnt + 2, c.row, ipx_h.hub_prefix,
                                                                   (uint32_t*)c.push_owner));
    IPX_LAUNCH(IPX_K_MARK2, ipx_k_mark<2><<<ge, ipx_h.tb, 0, st>>>(ipx_h.blist[2], ipx_h.lcnt + 2, ipx_h.hub_prefix));
    IPX_LAUNCH(IPX_K_COMPACT_T, IPX_OK(ipg_compact(c.bt, V, c.in_row, ipx_h.tune.t0, ipx_h.tune.t1, ipx_h.tlist[0], ipx_h.tlist[1],
                                                   ipx_h.tlist[2], ipx_h.lcnt + 4, edges_t, 1, st)));
    IPX_LAUNCH(IPX_K_GATHER0, ipx_k_gather<0, false><<<ge, ipx_h.tb, 0, st>>>(ipx_h.tlist[0], ipx_h.lcnt + 4, 0));
    IPX_LAUNCH(IPX_K_GATHER1, ipx_k_gather<1, false><<<ge, ipx_h.tb, 0, st>>>(ipx_h.tlist[1], ipx_h.lcnt + 5, 0));
    IPX_LAUNCH(IPX_K_GATHER2, ipx_k_gather<2, false><<<ge, ipx_h.tb, 0, st>>>(ipx_h.tlist[2], ipx_h.lcnt + 6, 0));
#endif
    IPX_CU(cudaGetLastError());
    return IPG_OK;
}

static uint64_t ipx_max_supersteps()
{
    /* The reference loops until quiescence; a bound (IPG_MAX_SUPERSTEPS,
     * default 10^6) turns a program that never halts into an error. */
    const char* lim = getenv("IPG_MAX_SUPERSTEPS");
    const uint64_t n = (lim && *lim) ? strtoull(lim, nullptr, 10) : 1000000ULL;
    /* pull versions stamp broadcast slots with the superstep's low 32 bits */
    return (IPX_PULL && n > (uint64_t)IPX_NO_STAMP - 1) ? (uint64_t)IPX_NO_STAMP - 1 : n;
}

/* Host-driven loop: one synchronisation per superstep, which gives the
 * reference's per-superstep log lines with their durations. */
static int ipx_run_host_loop()
{
    const uint64_t V = ipx_h.c.V;
    uint64_t count = ip_active_vertices;
    const uint64_t max_supersteps = ipx_max_supersteps();
    for (uint64_t s = 0;; s++) {
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SINGLE_BROADCAST
        if (count == 0) break; /* while(ip_active_vertices != 0), combiner_postamble.h:134 */
#else
        if (s > 0 && count == 0) break; /* while(first || count > 0), combiner_spread_postamble.h:212 */
#endif
        if (s >= max_supersteps) return ipx_fail(IPG_EDEVICE, "superstep limit (IPG_MAX_SUPERSTEPS) reached");
        /* vertices the compute kernel runs: the frontier (spread versions) or
         * the active ones of the previous superstep */
        const uint64_t frontier = (s == 0) ? V : count;
        IPX_OK(ipx_set_superstep(s));
        IPX_CU(cudaEventRecord(ipx_h.ev0, ipx_h.st));
        IPX_OK(ipx_enqueue_superstep());
        IPX_OK(ipx_end_superstep(s, &count, frontier));
        ip_superstep = s + 1;
    }
    return IPG_OK;
}

/* Captured loop: the superstep's kernels, then ipx_k_advance, as the body of
 * a CUDA-graph while node; one launch runs the program to quiescence with no
 * host synchronisation between supersteps.  The graph is built once per
 * attached graph and reused by later runs. */
/* Adds the superstep loop as a root node of `graph`: a while node whose
 * body is one superstep's kernels followed by ipx_k_advance, which records
 * the superstep and sets the condition on the device. */
static int ipx_add_loop_node(cudaGraph_t graph)
{
    cudaGraphConditionalHandle handle;
    IPX_CU(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    IPX_CU(cudaGraphAddNode(&node, graph, nullptr, 0, &params));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    const bool prof = ipx_h.profile;
    ipx_h.profile = false; /* no event nodes inside the body */
    uint64_t before[IPX_K_N];
    memcpy(before, ipx_h.prof_launches, sizeof before);
    IPX_CU(cudaStreamBeginCaptureToGraph(ipx_h.st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int r = ipx_enqueue_superstep();
    IPX_LAUNCH(IPX_K_CTRL, ipx_k_advance<<<1, 1, 0, ipx_h.st>>>(handle, (unsigned long long)ipx_max_supersteps()));
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(ipx_h.st, &captured);
    ipx_h.profile = prof;
    for (int k = 0; k < IPX_K_N; k++) {
        ipx_h.body_launches[k] = ipx_h.prof_launches[k] - before[k];
        ipx_h.prof_launches[k] = before[k];
    }
    if (r != IPG_OK) return r;
    if (e != cudaSuccess) return ipx_fail(IPG_ECUDA, cudaGetErrorString(e));
    return IPG_OK;
}

/* The library's own captured loop: built once per attached graph. */
static int ipx_build_graph_loop()
{
    if (ipx_h.gexec) return IPG_OK;
    cudaGraph_t graph = nullptr;
    IPX_CU(cudaGraphCreate(&graph, 0));
    int r = ipx_add_loop_node(graph);
    if (r != IPG_OK) {
        cudaGraphDestroy(graph);
        return r;
    }
    cudaError_t e = cudaGraphInstantiate(&ipx_h.gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        ipx_h.gexec = nullptr;
        return ipx_fail(IPG_ECUDA, cudaGetErrorString(e));
    }
    return IPG_OK;
}

/* Before a launch of a captured loop: superstep 0 on the device. */
/* The attached graph still holds the contents the engine's derived state
 * (degree classes, in-CSR pointers) was built from, and they are valid. */
static int ipx_check_contents()
{
    uint64_t gen = 0;
    int valid = 1;
    IPX_OK(ipg_graph_contents(ipx_h.g, &gen, &valid));
    if (!valid) return ipx_fail(IPG_EINVAL, "the graph's contents failed validation at its last refill");
    if (gen != ipx_h.graph_generation)
        return ipx_fail(IPG_EINVAL, "the graph was refilled after this engine attached it: attach it again");
    return IPG_OK;
}

static int ipx_loop_prepare()
{
    if (!ipx_h.ready) return ipx_fail(IPG_EINVAL, "ip_run called before ip_init");
    IPX_OK(ipx_check_contents());
    if (ipx_h.dirty) IPX_OK(ipx_reset_vertex_state());
    ipx_h.dirty = true;
    size_t zero = 0;
    IPX_CU(cudaMemcpyToSymbol(ipd_superstep, &zero, sizeof zero));
    IPX_CU(cudaMemcpyToSymbol(ipd_compute_superstep, &zero, sizeof zero));
    return IPG_OK;
}

/* After a captured loop ran: the supersteps, their counts and the error word
 * from the device; `seconds` is the loop's device time. */
static int ipx_loop_collect(double seconds)
{
    size_t S = 0;
    IPX_CU(cudaMemcpyFromSymbol(&S, ipd_superstep, sizeof S));
    uint32_t err = 0;
    IPX_CU(cudaMemcpy(&err, ipx_h.c.err, 4, cudaMemcpyDeviceToHost));
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SINGLE_BROADCAST
    /* while(ip_active_vertices != 0): no superstep at all without vertices */
    if (ipx_h.c.V == 0) S = 0;
#endif
    ipx_h.total_seconds = seconds;
    const uint64_t kept = S < IPX_HIST ? S : IPX_HIST;
    std::vector<unsigned long long> hist(kept * 4);
    if (kept) IPX_CU(cudaMemcpy(hist.data(), ipx_h.c.hist, kept * 4 * 8, cudaMemcpyDeviceToHost));
    for (uint64_t s = 0; s < S; s++) {
        const unsigned long long* h = S <= IPX_HIST ? &hist[s * 4] : nullptr;
        const uint64_t count = h ? h[0] : 0;
        if (h) ipx_h.edges += h[1];
        if (h && h[2]) ipx_h.pulled_supersteps++;
        ipx_h.counts.push_back(count);
        if (!ipx_h.quiet) {
            /* one launch for all supersteps: durations are the loop's average */
            printf("Superstep%zuDuration:%f\n", (size_t)s, ipx_h.total_seconds / (double)S);
            printf("Superstep%zuActiveVertexCount:%zu\n", (size_t)s, (size_t)count);
        }
    }
    for (int k = 0; k < IPX_K_N; k++) ipx_h.prof_launches[k] += ipx_h.body_launches[k] * S;
    ipx_h.graph_launches++;
    ip_superstep = S;
    ip_active_vertices = ipx_h.counts.empty() ? 0 : ipx_h.counts.back();
    ipx_h.host_valid = false;
    if (err & IPX_ERR_SEND_IN_BROADCAST)
        return ipx_fail(IPG_EDEVICE,
                        "The function send_message should not be used in the SINGLE_BROADCAST version; only "
                        "broadcast() should be called, and once per superstep maximum.");
    if (err & IPX_ERR_SUPERSTEP_LIMIT) return ipx_fail(IPG_EDEVICE, "superstep limit (IPG_MAX_SUPERSTEPS) reached");
    if (err & IPX_ERR_COPY_TIMEOUT)
        return ipx_fail(IPG_EDEVICE, "a bulk copy into shared memory did not complete in time (results kept exact)");
    if (err & IPX_ERR_RESERVED_MESSAGE)
        return ipx_fail(IPG_EDEVICE, "a broadcast FP64 message had all 64 bits set, the pattern the single_broadcast "
                                     "engine reserves for 'no broadcast' (build with -DIPX_SB_DENSE=0 to allow it)");
    if (err) return ipx_fail(IPG_EDEVICE, "a kernel reported an error");
    return IPG_OK;
}

static int ipx_run_graph_loop()
{
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SINGLE_BROADCAST
    if (ip_active_vertices == 0) return IPG_OK;
#endif
    IPX_OK(ipx_build_graph_loop());
    cudaStream_t st = ipx_h.st;
    IPX_OK(ipx_set_superstep(0));
    IPX_CU(cudaEventRecord(ipx_h.ev0, st));
    IPX_CU(cudaGraphLaunch(ipx_h.gexec, st));
    IPX_CU(cudaEventRecord(ipx_h.ev1, st));
    IPX_CU(cudaEventSynchronize(ipx_h.ev1));
    IPX_CU(cudaGetLastError());
    float ms = 0.f;
    IPX_CU(cudaEventElapsedTime(&ms, ipx_h.ev0, ipx_h.ev1));
    return ipx_loop_collect(ms * 1e-3);
}

static int ipx_run_impl()
{
    if (!ipx_h.ready) return ipx_fail(IPG_EINVAL, "ip_run called before ip_init");
    IPX_OK(ipx_check_contents());
    if (ipx_h.dirty) IPX_OK(ipx_reset_vertex_state());
    ipx_h.dirty = true;
    IPX_OK(ipx_h.graph_loop ? ipx_run_graph_loop() : ipx_run_host_loop());
    if (!ipx_h.quiet) printf("Total time of supersteps: %fs.\n", ipx_h.total_seconds);
    ipx_h.host_valid = false;
    return IPG_OK;
}

/* ------------------------------------------------------------------------ */
/* The reference's host interface.                                          */
/* ------------------------------------------------------------------------ */
static void ipx_die(const char* msg)
{
    printf("%s\n", msg);
    exit(-1);
}

void ip_increment_superstep() { ip_superstep++; }
void ip_set_vertices_count(size_t vertices_count) { ip_vertices_count = vertices_count; }
void ip_set_edges_count(size_t edges_count) { ip_edges_count = edges_count; }

/* The values in the caller's numbering, on the device: the engine's own
 * array, or a copy gathered from it when the kernels run renamed. */
static int ipx_values_by_id(const ipx_val** out)
{
    if (!ipx_h.vindex_of || !ipx_h.c.V) {
        *out = ipx_h.c.value;
        return IPG_OK;
    }
    if (!ipx_h.values_by_id) IPX_OK(ipx_alloc(&ipx_h.values_by_id, ipx_h.c.V));
    ipx_k_values_by_id<<<ipx_grid(), IPX_THREADS, 0, ipx_h.st>>>(ipx_h.values_by_id);
    IPX_CU(cudaGetLastError());
    IPX_CU(cudaStreamSynchronize(ipx_h.st));
    *out = ipx_h.values_by_id;
    return IPG_OK;
}

/* Host copies of the vertices, filled from the device on first use. */
static int ipx_materialise()
{
    if (ipx_h.host_valid) return IPG_OK;
    const uint64_t V = ipx_h.c.V;
    std::vector<ipx_val> vals(V);
    std::vector<uint64_t> row(V + 1), in_row(V + 1);
    std::vector<uint32_t> index_of(ipx_h.vindex_of ? V : 0); /* id -> vertex of the renamed copy */
    if (V) {
        const ipx_val* v = nullptr;
        IPX_OK(ipx_values_by_id(&v));
        IPX_CU(cudaMemcpy(vals.data(), v, V * sizeof(ipx_val), cudaMemcpyDeviceToHost));
        IPX_CU(cudaMemcpy(row.data(), ipx_h.c.row, (V + 1) * 8, cudaMemcpyDeviceToHost));
        IPX_CU(cudaMemcpy(in_row.data(), ipx_h.c.in_row, (V + 1) * 8, cudaMemcpyDeviceToHost));
        if (ipx_h.vindex_of) IPX_CU(cudaMemcpy(index_of.data(), ipx_h.vindex_of, V * 4, cudaMemcpyDeviceToHost));
    }
    ipx_h.host_vertices.resize(V);
    for (uint64_t i = 0; i < V; i++) {
        struct ip_vertex_t& x = ipx_h.host_vertices[i];
        memset(&x, 0, sizeof x);
        x.id = (ipx_vid)i;
        x.value = vals[i];
        [[maybe_unused]] const uint64_t n = ipx_h.vindex_of ? index_of[i] : i;
#ifdef IP_NEEDS_OUT_NEIGHBOUR_COUNT
        x.out_neighbour_count = (IP_NEIGHBOUR_COUNT_TYPE)(row[n + 1] - row[n]);
#endif
#ifdef IP_NEEDS_IN_NEIGHBOUR_COUNT
        x.in_neighbour_count = (IP_NEIGHBOUR_COUNT_TYPE)(in_row[n + 1] - in_row[n]);
#endif
    }
    ip_all_vertices = ipx_h.host_vertices.data();
    ipx_h.host_valid = true;
    return IPG_OK;
}

struct ip_vertex_t* ip_get_vertex_by_location(size_t location)
{
    if (ipx_materialise() != IPG_OK) ipx_die(ipx_h.err);
    return &ip_all_vertices[location];
}

struct ip_vertex_t* ip_get_vertex_by_id(IP_VERTEX_ID_TYPE id) { return ip_get_vertex_by_location((size_t)id); }

void ip_dump(FILE* f)
{
    double t0 = ipx_wtime();
    if (ipx_materialise() != IPG_OK) ipx_die(ipx_h.err);
    for (size_t i = 0; i < ip_get_vertices_count(); i++) ip_serialise_vertex(f, &ip_all_vertices[i]);
    printf("DumpingTime:%f\n", ipx_wtime() - t0);
}

void* ip_safe_malloc(size_t size_to_malloc)
{
    void* ptr = malloc(size_to_malloc);
    if (ptr == NULL) {
        printf("Failed to allocate %zu bytes.\n", size_to_malloc);
        exit(-1);
    }
    return ptr;
}

void* ip_safe_realloc(void* ptr, size_t size_to_realloc)
{
    ptr = realloc(ptr, size_to_realloc);
    if (ptr == NULL) {
        printf("Failed to reallocate to %zu bytes.\n", size_to_realloc);
        exit(-1);
    }
    return ptr;
}

void ip_safe_free(void* ptr)
{
    if (ptr != NULL) free(ptr);
}

FILE* ip_safe_fopen(const char* file_path, const char* mode)
{
    FILE* f = fopen(file_path, mode);
    if (f == NULL) {
        printf("Cannot open the file \"%s\" in mode \"%s\".\n", file_path, mode);
        exit(-1);
    }
    return f;
}

void ip_safe_fread(void* ptr, size_t size, size_t count, FILE* stream)
{
    if (fread(ptr, size, count, stream) != count) {
        printf("Failed to read %zu elements of %zu bytes each.\n", count, size);
        exit(-1);
    }
}

void ip_safe_fwrite(void* ptr, size_t size, size_t count, FILE* stream)
{
    if (fwrite(ptr, size, count, stream) != count) {
        printf("Failed to write.'\n");
        exit(-1);
    }
}

void ip_init_vertex_range(IP_VERTEX_ID_TYPE first, IP_VERTEX_ID_TYPE last)
{
    if (!ipx_h.ready || last < first) return;
    ipx_k_init_values<<<ipx_grid(), IPX_THREADS, 0, ipx_h.st>>>((uint64_t)first, (uint64_t)last);
    cudaStreamSynchronize(ipx_h.st);
}

void ip_init_specific()
{
    if (ipx_h.ready && ipx_reset_vertex_state() != IPG_OK) ipx_die(ipx_h.err);
}

void ip_load_graph(const char* file_path, bool directed, bool weighted)
{
    double start = ipx_wtime();
    if (!ipx_h.quiet) {
        printf("[INFO] The application indicates that the graph must be %sdirected and %sweighted, so the graph "
               "passed is expected to be so.\n",
               directed ? "" : "un", weighted ? "" : "un");
        printf("[INFO] Starting graph loading.\n");
    }
    const bool need_in = directed && (IPX_PULL
#if defined(IP_NEEDS_IN_NEIGHBOUR_IDS) || defined(IP_NEEDS_IN_NEIGHBOUR_COUNT) || IPX_IN_WEIGHTS
                                      || true
#endif
                                     );
    const int wbytes = IPX_WEIGHT_BYTES ? IPX_WEIGHT_BYTES : 4;
    ipg_graph* g = nullptr;
    int r = ipg_graph_load(file_path, (int)sizeof(IP_VERTEX_ID_TYPE), (int)sizeof(IP_NEIGHBOUR_COUNT_TYPE),
                           directed, weighted, wbytes, need_in, &g);
    if (r != IPG_OK) ipx_die(ipg_last_error());
    r = ipx_attach(g, true);
    if (r != IPG_OK) ipx_die(ipx_h.err);
    if (!ipx_h.quiet) {
        printf("\t\t- %zu vertices\n\t\t- %zu edges\n", ip_get_vertices_count(), ip_get_edges_count());
        printf("LoadingTime:%f\n", ipx_wtime() - start);
    }
}

void ip_init(const char* file_path, int number_of_threads, const char* schedule, int chunk_size, bool directed,
             bool weighted)
{
    /* The OpenMP schedule arguments are accepted and checked as in
     * tmp_extract_runtime_schedule (iPregel_postamble.h:176-193); the GPU
     * engine has no use for them. */
    if (strcmp(schedule, "static") == 0) {
        if (!ipx_h.quiet) printf("Runtime schedule set to static(%d).\n", chunk_size);
    } else if (strcmp(schedule, "dynamic") == 0) {
        if (!ipx_h.quiet) printf("Runtime schedule set to dynamic(%d).\n", chunk_size);
    } else {
        printf("The schedule %s is unknown.\n", schedule);
        exit(-1);
    }
    double t0 = ipx_wtime();
    if (!ipx_h.quiet) {
        char dev[256] = "unknown";
        uint64_t hbm = 0;
        int sms = 0;
        ipg_device_info(dev, sizeof dev, &hbm, &sms);
        printf("Version:%s\n", VERSION);
        printf("Software:iPregel-B200\n");
        printf("FileCommits:%s\n", COMMITS);
        printf("Application:%s\n", IP_APPLICATION);
        printf("MpiProcessCount:0\n");
        printf("Machine:%s\n", IP_MACHINE);
        printf("Device:%s\n", dev);
        printf("CompilationFlags:%s\n", STRINGIFY(COMPILATION_FLAGS));
        time_t t = time(NULL);
        struct tm tm = *localtime(&t);
        printf("SubmissionDate:%02d/%02d/%d\n", tm.tm_mday, tm.tm_mon + 1, tm.tm_year + 1900);
        printf("SubmissionTime:%02d:%02d:%02d\n", tm.tm_hour, tm.tm_min, tm.tm_sec);
        const char* name = file_path;
        const char* tmp = strchr(name, '/');
        while (tmp != NULL) {
            name = tmp + 1;
            tmp = strchr(name, '/');
        }
        printf("Graph:%s\n", name);
        printf("OpenmpThreadCount:%d\n", number_of_threads);
    }
    ip_thread_count = number_of_threads;
    ip_load_graph(file_path, directed, weighted);
    if (!ipx_h.quiet) printf("InitialisationTime:%f\n", ipx_wtime() - t0);
}

int ip_run()
{
    int r = ipx_run_impl();
    if (r != IPG_OK) ipx_die(ipx_h.err);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* C ABI exported by every application library (no reference counterpart:  */
/* the reference is compiled into its application; these let a host program */
/* or a test drive the same engine with in-memory graphs).                  */
/* ------------------------------------------------------------------------ */
extern "C" {

int ipg_app_abi_version(void) { return IPG_ABI_VERSION; }

/* "key=value" pairs describing the instantiated types and version. */
int ipg_app_describe(char* buf, int len)
{
    const char* kind = std::is_floating_point<ipx_val>::value ? "f" : (std::is_signed<ipx_val>::value ? "i" : "u");
    const char* mkind = std::is_floating_point<ipx_msg>::value ? "f" : (std::is_signed<ipx_msg>::value ? "i" : "u");
    return snprintf(buf, (size_t)len,
                    "application=%s version=%d id_bytes=%d value_bytes=%d value_kind=%s message_bytes=%d "
                    "message_kind=%s combine_kind=%d weight_bytes=%d",
                    IP_APPLICATION, IPX_VERSION, (int)sizeof(ipx_vid), (int)sizeof(ipx_val), kind,
                    (int)sizeof(ipx_msg), mkind, IP_COMBINE_KIND, IPX_WEIGHT_BYTES);
}

const char* ipg_app_last_error(void) { return ipx_h.err; }

/* Attaches a resident graph (the caller keeps ownership). */
int ipg_app_attach(ipg_graph* g)
{
    if (!g) return ipx_fail(IPG_EINVAL, "ipg_app_attach: null graph");
    return ipx_attach(g, false);
}

/* ip_init from host buffers in the file layout (idx: V row starts, u64). */
int ipg_app_load_host(uint64_t V, uint64_t E, const uint64_t* idx, const void* adj, const void* wgt, int directed)
{
    ipx_h.err[0] = 0;
    const bool need_in = directed && (IPX_PULL
#if defined(IP_NEEDS_IN_NEIGHBOUR_IDS) || defined(IP_NEEDS_IN_NEIGHBOUR_COUNT) || IPX_IN_WEIGHTS
                                      || true
#endif
                                     );
    ipg_graph* g = nullptr;
    int r = ipg_graph_from_host(V, E, idx, 8, adj, (int)sizeof(ipx_vid), wgt, wgt ? (IPX_WEIGHT_BYTES ? IPX_WEIGHT_BYTES : 4) : 0,
                                directed, need_in, &g);
    if (r != IPG_OK) return ipx_fail(r, ipg_last_error());
    return ipx_attach(g, true);
}

int ipg_app_run(void) { return ipx_run_impl(); }

int ipg_app_values(void* out, uint64_t cap_bytes)
{
    const uint64_t bytes = ipx_h.c.V * sizeof(ipx_val);
    if (!ipx_h.ready) return ipx_fail(IPG_EINVAL, "no graph attached");
    if (cap_bytes < bytes) return ipx_fail(IPG_EINVAL, "output buffer too small");
    const ipx_val* v = nullptr;
    IPX_OK(ipx_values_by_id(&v));
    if (bytes) IPX_CU(cudaMemcpy(out, v, bytes, cudaMemcpyDeviceToHost));
    return IPG_OK;
}

/* Valid until the next run, attach or release of this library. */
int ipg_app_values_device(void** ptr)
{
    if (!ipx_h.ready) return ipx_fail(IPG_EINVAL, "no graph attached");
    const ipx_val* v = nullptr;
    IPX_OK(ipx_values_by_id(&v));
    *ptr = (void*)v;
    return IPG_OK;
}

uint64_t ipg_app_supersteps(void) { return ipx_h.counts.size(); }

int ipg_app_counts(uint64_t* out, uint64_t cap)
{
    uint64_t n = ipx_h.counts.size();
    for (uint64_t i = 0; i < n && i < cap; i++) out[i] = ipx_h.counts[i];
    return (int)n;
}

int ipg_app_stats(double* seconds, uint64_t* edges, uint64_t* supersteps)
{
    if (seconds) *seconds = ipx_h.total_seconds;
    if (edges) *edges = ipx_h.edges;
    if (supersteps) *supersteps = ipx_h.counts.size();
    return IPG_OK;
}

/* Launch stream of the engine (for callers timing it with their own events). */
void* ipg_app_stream(void) { return (void*)ipx_h.st; }

int ipg_app_set_quiet(int quiet)
{
    ipx_h.quiet = quiet != 0;
    return IPG_OK;
}

/* Per-kernel profiling: events around every launch while on (adds a few
 * microseconds per launch). */
int ipg_app_set_profile(int on)
{
    if (on && !ipx_h.pev_made) {
        for (int i = 0; i < IPX_PEV; i++) {
            IPX_CU(cudaEventCreate(&ipx_h.pev[0][i]));
            IPX_CU(cudaEventCreate(&ipx_h.pev[1][i]));
        }
        ipx_h.pev_made = true;
    }
    ipx_h.profile = on != 0;
    ipx_h.npev = 0;
    return IPG_OK;
}

/* Superstep loop mode: 0 drives supersteps from the host (one
 * synchronisation each, the reference's per-superstep log), 1 runs them as a
 * captured CUDA graph with a device-evaluated while condition (one launch per
 * ip_run).  Default from IPG_GRAPH_LOOP, else 0. */
int ipg_app_set_graph_loop(int on)
{
    ipx_h.graph_loop = on != 0;
    return IPG_OK;
}

int ipg_app_graph_loop(void) { return ipx_h.graph_loop ? 1 : 0; }

/* 1 (the default, unless IPG_ORDER=0): the next attach runs the kernels on
 * the graph's degree-ordered copy (ipg_graph_degree_order).  ip_compute
 * still sees the graph's own numbering (its id, its neighbours' ids, the
 * order of its edges), and so do ip_send_message, the values and ip_dump:
 * every result is the same.  A copy that does not fit the HBM budget leaves
 * the graph's own numbering.  ipg_app_order reports whether the attached
 * graph runs renamed. */
int ipg_app_set_order(int on)
{
    ipx_h.order = on != 0;
    return IPG_OK;
}

int ipg_app_order(void) { return (ipx_h.ready && ipx_h.vid_of) ? 1 : 0; }

/* Tuning of the superstep kernels, applied at the next attach: CTA size
 * (a multiple of 32, at most 256), degree-class thresholds t0 <= t1 (thread
 * per vertex up to t0 edges, warp up to t1, CTAs beyond) and the push
 * versions' pull switch (pull when the broadcasters' edges exceed
 * E / pull_div; 0 never; needs a symmetric graph or a directed one). */
int ipg_app_set_tuning(int block, uint64_t t0, uint64_t t1, uint64_t pull_div)
{
    if (block < 32 || block > IPX_THREADS || (block & 31))
        return ipx_fail(IPG_EINVAL, "ipg_app_set_tuning: block must be a multiple of 32 in [32, 256]");
    if (t0 < 1 || t1 < t0) return ipx_fail(IPG_EINVAL, "ipg_app_set_tuning: need 1 <= t0 <= t1");
    /* a warp of the pull gather sums the degrees of 32 vertices of the
     * middle class in 32 bits */
    if (t1 > (1ULL << 26)) return ipx_fail(IPG_EINVAL, "ipg_app_set_tuning: t1 above 2^26");
    ipx_h.tune.block = block;
    ipx_h.tune.t0 = t0;
    ipx_h.tune.t1 = t1;
    ipx_h.tune.pull_div = pull_div;
    return IPG_OK;
}

/* Several applications' loops in one CUDA graph launch.  ipg_app_loop_add
 * adds this library's superstep loop (a while node over one superstep's
 * kernels, its condition evaluated on the device) as a root node of the
 * caller's cudaGraph_t; nodes of different libraries share no dependency
 * and may run concurrently.  Before every launch of the caller's graph call
 * ipg_app_loop_prepare (resets the vertex state, superstep 0); after it
 * completed, ipg_app_loop_collect with the launch's device time (reads the
 * superstep history and the error word, as ip_run would report them).  The
 * node belongs to the attached graph: attach again, add again. */
int ipg_app_loop_add(void* cuda_graph)
{
    if (!ipx_h.ready) return ipx_fail(IPG_EINVAL, "ipg_app_loop_add: no graph attached");
    if (!cuda_graph) return ipx_fail(IPG_EINVAL, "ipg_app_loop_add: null graph");
    return ipx_add_loop_node((cudaGraph_t)cuda_graph);
}

int ipg_app_loop_prepare(void) { return ipx_loop_prepare(); }

int ipg_app_loop_collect(double seconds) { return ipx_loop_collect(seconds); }

int ipg_app_get_tuning(int* block, uint64_t* t0, uint64_t* t1, uint64_t* pull_div)
{
    if (block) *block = ipx_h.tune.block;
    if (t0) *t0 = ipx_h.tune.t0;
    if (t1) *t1 = ipx_h.tune.t1;
    if (pull_div) *pull_div = ipx_h.tune.pull_div;
    return IPG_OK;
}

void ipg_app_profile_reset(void)
{
    for (int k = 0; k < IPX_K_N; k++) {
        ipx_h.prof_launches[k] = ipx_h.prof_timed[k] = 0;
        ipx_h.prof_ms[k] = ipx_h.prof_bytes[k] = ipx_h.prof_edges[k] = 0.0;
    }
}

/* Kernel launches of this library since the last reset. */
uint64_t ipg_app_launches(void)
{
    uint64_t n = 0;
    for (int k = 0; k < IPX_K_N; k++) n += ipx_h.prof_launches[k];
    return n;
}

/* One line per kernel: "name launches timed_launches total_ms algorithmic_bytes
 * edges_walked" (edges_walked is 0 for kernels that walk no edge lists). */
int ipg_app_profile(char* buf, int len)
{
    int off = 0;
    for (int k = 0; k < IPX_K_N && off < len; k++) {
        if (!ipx_h.prof_launches[k]) continue;
        off += snprintf(buf + off, (size_t)(len - off), "%s %llu %llu %.6f %.0f %.0f\n", ipx_kname[k],
                        (unsigned long long)ipx_h.prof_launches[k], (unsigned long long)ipx_h.prof_timed[k],
                        ipx_h.prof_ms[k], ipx_h.prof_bytes[k], ipx_h.prof_edges[k]);
    }
    return off;
}

int ipg_app_set_param(const char* key, double value)
{
#ifdef IP_APP_PARAMS
    return ip_app_set_param(key, value);
#else
    (void)key;
    (void)value;
    return ipx_fail(IPG_EINVAL, "this application takes no parameters");
#endif
}

/* A named device array for the application (e.g. batch offsets); the
 * caller keeps it alive while runs use it. */
int ipg_app_set_param_ptr(const char* key, const void* ptr, uint64_t n)
{
#ifdef IP_APP_PARAM_PTRS
    if (ip_app_set_param_ptr(key, ptr, n) != 0) return ipx_fail(IPG_EINVAL, "unknown array parameter");
    return IPG_OK;
#else
    (void)key;
    (void)ptr;
    (void)n;
    return ipx_fail(IPG_EINVAL, "this application takes no array parameters");
#endif
}

void ipg_app_release(void) { ipx_release_state(); }

} /* extern "C" */

#endif /* IPREGEL_B200_HOST_CUH */
