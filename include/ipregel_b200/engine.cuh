/*
 * engine.cuh -- the typed superstep engine: sm_100a kernels instantiated with
 * the application's IP_* types, its ip_compute and its ip_combine.
 *
 * Versions (selected as in src/iPregel_preamble.h:319-331):
 *   combiner (push)                src/combiner_postamble.h:123-199
 *   single_broadcast (pull)        src/combiner_single_broadcast_postamble.h:125-259
 *   spread (frontier push)         src/combiner_spread_postamble.h:160-431
 *   spread + single_broadcast      src/combiner_spread_single_broadcast_postamble.h:145-399
 *
 * Device layout (structure of arrays, all resident in HBM):
 *   value[V]                       IP_VALUE_TYPE
 *   CSR row[V+1] (u64), adj[E]     the loader's layout; in-CSR for pulls
 *   active / has_message           bitmaps (combiner, written by warp ballot)
 *                                  or bytes (pulls, written by any thread)
 *   mailbox[2][V]                  push: combined message of the superstep,
 *                                  double-buffered by superstep parity
 *   received[2]                    push: bitmap of mailboxes that got mail
 *   outbox[V] + broadcaster bitmap push: ip_broadcast records here; delivery
 *                                  is a separate edge-parallel kernel
 *   bval[V] + has_bcast bitmap     pull: the externalised broadcast slot of
 *                                  combiner_single_broadcast_preamble.h:42-50
 * Messages become visible only at the next superstep in every version
 * (combiner_postamble.h:168-183), so recording broadcasts in an outbox and
 * delivering them after the compute kernel gives the reference's results;
 * ip_combine is associative and commutative by contract
 * (iPregel_preamble.h:256-262), so combining in a different order is allowed.
 */
#ifndef IPREGEL_B200_ENGINE_CUH
#define IPREGEL_B200_ENGINE_CUH

#include <cuda_runtime.h>

#include <limits>
#include <type_traits>

typedef IP_VERTEX_ID_TYPE ipx_vid;
typedef IP_MESSAGE_TYPE ipx_msg;
typedef IP_VALUE_TYPE ipx_val;

#ifdef IP_NEEDS_OUT_NEIGHBOUR_WEIGHTS
#define IPX_OUT_WEIGHTS 1
#else
#define IPX_OUT_WEIGHTS 0
#endif
#ifdef IP_NEEDS_IN_NEIGHBOUR_WEIGHTS
#define IPX_IN_WEIGHTS 1
#else
#define IPX_IN_WEIGHTS 0
#endif
#if IPX_OUT_WEIGHTS || IPX_IN_WEIGHTS
typedef IP_EDGE_WEIGHT_TYPE ipx_wgt;
#define IPX_WEIGHT_BYTES ((int)sizeof(IP_EDGE_WEIGHT_TYPE))
#else
typedef unsigned int ipx_wgt;
#define IPX_WEIGHT_BYTES 0
#endif

/* Weighted broadcast (extension, no reference counterpart): an application
 * that defines IP_BROADCAST_EDGE_MESSAGE(m, w) before including iPregel.h
 * makes ip_broadcast deliver IP_BROADCAST_EDGE_MESSAGE(m, weight) along each
 * out-edge (e.g. m + w for SSSP).  The transform must distribute over
 * ip_combine, because two broadcasts of one vertex in one superstep are
 * combined before delivery. */
#ifdef IP_BROADCAST_EDGE_MESSAGE
#define IPX_EDGE_MSG 1
#if !IPX_OUT_WEIGHTS
#error "IP_BROADCAST_EDGE_MESSAGE needs IP_NEEDS_OUT_NEIGHBOUR_WEIGHTS"
#endif
#if IPX_PULL
#error "IP_BROADCAST_EDGE_MESSAGE applies to the combiner and spread versions"
#endif
#else
#define IPX_EDGE_MSG 0
#endif

static_assert(sizeof(ipx_msg) <= 8, "iPregel-B200: IP_MESSAGE_TYPE must be at most 8 bytes");

#define IPX_FULL 0xffffffffu
/* Largest CTA the kernels are compiled for; the launch size is a runtime
 * tuning parameter (a multiple of 32 up to this). */
#define IPX_THREADS 256
/* Resident CTAs per SM the edge kernels (push, mark, gather) are compiled
 * for: 6 x 256 threads keeps their ~40 registers without spilling. */
#ifndef IPX_EDGE_CTAS
#define IPX_EDGE_CTAS 6
#endif
#define IPX_ERR_SEND_IN_BROADCAST 1u
#define IPX_ERR_COMBINE_HINT 2u
#define IPX_ERR_SUPERSTEP_LIMIT 4u
#define IPX_HIST 65536

/* Default degree-class thresholds for the thread / warp / block kernels
 * (runtime tuning parameters). */
#ifndef IPX_T0
#define IPX_T0 16
#endif
#ifndef IPX_T1
#define IPX_T1 4096
#endif

/* ------------------------------------------------------------------------ */
/* Mailbox policies: how a push delivers a message into mailbox[w].          */
/* deliver() returns true when the received bit of w may still be clear      */
/* (the CAS policies know exactly: this call filled an empty mailbox; the    */
/* hardware-atomic ones return true whenever they issued an update), and the */
/* caller then sets the bit with a fire-and-forget atomic OR.                */
/* ------------------------------------------------------------------------ */
template <class T>
struct ipx_word {
    typedef typename std::conditional<(sizeof(T) <= 4), unsigned int, unsigned long long>::type type;
};

template <class T>
__device__ __forceinline__ typename ipx_word<T>::type ipx_to_word(const T& x)
{
    typename ipx_word<T>::type w = 0;
    memcpy(&w, &x, sizeof(T));
    return w;
}

template <class T>
__device__ __forceinline__ T ipx_from_word(typename ipx_word<T>::type w)
{
    T x;
    memcpy(&x, &w, sizeof(T));
    return x;
}

/* Bitwise equality: a compute kernel writes a vertex's value back only when
 * ip_compute changed it (unchanged receivers are common in min-propagation
 * supersteps; each skipped store is a dirty sector less). */
template <class T>
__device__ __forceinline__ bool ipx_same_bits(const T& a, const T& b)
{
    if constexpr (sizeof(T) <= 8) {
        return ipx_to_word(a) == ipx_to_word(b);
    } else {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&a);
        const unsigned char* q = reinterpret_cast<const unsigned char*>(&b);
        for (size_t k = 0; k < sizeof(T); k++)
            if (p[k] != q[k]) return false;
        return true;
    }
}

template <class T>
__device__ __forceinline__ T ipx_shfl_down(T x, int o)
{
    typedef typename ipx_word<T>::type W;
    W w = ipx_to_word(x);
    w = __shfl_down_sync(IPX_FULL, w, o);
    return ipx_from_word<T>(w);
}

/* Read-modify-write by compare-and-swap on the message's bits, for operand
 * types without a hardware atomic of the operator. */
template <class T, class Op>
__device__ __forceinline__ void ipx_atomic_cas_op(T* a, T v, Op op)
{
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "combiner hints need a 4- or 8-byte message type");
    typedef typename std::conditional<sizeof(T) == 4, unsigned int, unsigned long long>::type W;
    W* p = reinterpret_cast<W*>(a);
    W old = *p;
    for (;;) {
        T cur;
        memcpy(&cur, &old, sizeof(T));
        T nv = op(cur, v);
        W nw;
        memcpy(&nw, &nv, sizeof(T));
        if (nw == old) return;
        W prev = atomicCAS(p, old, nw);
        if (prev == old) return;
        old = prev;
    }
}

template <class T>
__device__ __forceinline__ void ipx_atomic_min(T* a, T v)
{
    if constexpr (std::is_unsigned<T>::value && sizeof(T) == 4) atomicMin((unsigned int*)a, (unsigned int)v);
    else if constexpr (std::is_unsigned<T>::value && sizeof(T) == 8) atomicMin((unsigned long long*)a, (unsigned long long)v);
    else if constexpr (std::is_signed<T>::value && std::is_integral<T>::value && sizeof(T) == 4) atomicMin((int*)a, (int)v);
    else if constexpr (std::is_signed<T>::value && std::is_integral<T>::value && sizeof(T) == 8) atomicMin((long long*)a, (long long)v);
    else ipx_atomic_cas_op(a, v, [](T x, T y) { return y < x ? y : x; });
}

template <class T>
__device__ __forceinline__ void ipx_atomic_max(T* a, T v)
{
    if constexpr (std::is_unsigned<T>::value && sizeof(T) == 4) atomicMax((unsigned int*)a, (unsigned int)v);
    else if constexpr (std::is_unsigned<T>::value && sizeof(T) == 8) atomicMax((unsigned long long*)a, (unsigned long long)v);
    else if constexpr (std::is_signed<T>::value && std::is_integral<T>::value && sizeof(T) == 4) atomicMax((int*)a, (int)v);
    else if constexpr (std::is_signed<T>::value && std::is_integral<T>::value && sizeof(T) == 8) atomicMax((long long*)a, (long long)v);
    else ipx_atomic_cas_op(a, v, [](T x, T y) { return y > x ? y : x; });
}

template <class T>
__device__ __forceinline__ void ipx_atomic_add(T* a, T v)
{
    if constexpr (std::is_same<T, double>::value || std::is_same<T, float>::value) atomicAdd(a, v);
    else if constexpr (std::is_integral<T>::value && sizeof(T) == 4) atomicAdd((unsigned int*)a, (unsigned int)v);
    else if constexpr (std::is_integral<T>::value && sizeof(T) == 8) atomicAdd((unsigned long long*)a, (unsigned long long)v);
    else ipx_atomic_cas_op(a, v, [](T x, T y) { return x + y; });
}

/* Read of a mailbox for the precheck of a monotone combiner.  Within a
 * superstep a min (max) mailbox only falls (rises), so a stale read can only
 * let a redundant atomic through, never drop a message: the read may come
 * from L1 (IPX_PRECHECK_L1 = 1, each SM keeps its own copy of hot mailboxes
 * such as the hubs') or from L2 (0, fresher but every read of a hot mailbox
 * lands on one L2 slice). */
#ifndef IPX_PRECHECK_L1
#define IPX_PRECHECK_L1 1
#endif
template <class T>
__device__ __forceinline__ T ipx_peek(const T* p)
{
#if IPX_PRECHECK_L1
    return *p;
#else
    return __ldcg(p);
#endif
}

/* 128-bit compare-and-swap (sm_90+ atom.cas.b128) for the generic 8-byte path. */
struct __align__(16) ipx_slot128 {
    unsigned long long flag;
    unsigned long long bits;
};

__device__ __forceinline__ void ipx_cas128(ipx_slot128* addr, unsigned long long cmp_f, unsigned long long cmp_b,
                                           unsigned long long new_f, unsigned long long new_b,
                                           unsigned long long& old_f, unsigned long long& old_b)
{
    asm volatile(
        "{\n\t"
        ".reg .b128 c, n, o;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 n, {%4, %5};\n\t"
        "atom.global.cas.b128 o, [%6], c, n;\n\t"
        "mov.b128 {%0, %1}, o;\n\t"
        "}"
        : "=l"(old_f), "=l"(old_b)
        : "l"(cmp_f), "l"(cmp_b), "l"(new_f), "l"(new_b), "l"(addr)
        : "memory");
}

template <int KIND, int MSGBYTES>
struct ipx_mailbox;

/* Hardware min / max on the message itself (4 or 8 bytes).  The slot holds
 * no flag: whether a vertex received mail is its received bit, which the
 * caller sets whenever deliver/commit return true.  A message equal to the
 * empty value still passes the precheck and so still sets the bit.  Keeping
 * the slot at the message's width halves the mailboxes of 4-byte messages
 * (V x 4 bytes per parity), which then stay in L2 at larger scales. */
struct ipx_mailbox_min {
    typedef ipx_msg slot;
    __device__ static slot empty() { return std::numeric_limits<ipx_msg>::max(); }
    __device__ static bool precheck(slot* s, ipx_msg m)
    {
        const ipx_msg c = ipx_peek(s);
        return m < c || (m == c && c == empty());
    }
    __device__ static bool commit(slot* s, ipx_msg m)
    {
        ipx_atomic_min(s, m);
        return true;
    }
    __device__ static bool deliver(slot* s, ipx_msg m)
    {
        if (m < __ldcg(s)) ipx_atomic_min(s, m);
        return true;
    }
    __device__ static bool merge(slot* s, ipx_msg m)
    {
        if (m < *s) *s = m;
        return true;
    }
    __device__ static ipx_msg take(slot* s)
    {
        ipx_msg m = *s;
        *s = empty();
        return m;
    }
};

struct ipx_mailbox_max {
    typedef ipx_msg slot;
    __device__ static slot empty() { return std::numeric_limits<ipx_msg>::lowest(); }
    __device__ static bool precheck(slot* s, ipx_msg m)
    {
        const ipx_msg c = ipx_peek(s);
        return m > c || (m == c && c == empty());
    }
    __device__ static bool commit(slot* s, ipx_msg m)
    {
        ipx_atomic_max(s, m);
        return true;
    }
    __device__ static bool deliver(slot* s, ipx_msg m)
    {
        if (m > __ldcg(s)) ipx_atomic_max(s, m);
        return true;
    }
    __device__ static bool merge(slot* s, ipx_msg m)
    {
        if (m > *s) *s = m;
        return true;
    }
    __device__ static ipx_msg take(slot* s)
    {
        ipx_msg m = *s;
        *s = empty();
        return m;
    }
};

template <>
struct ipx_mailbox<IP_COMBINE_MIN, 4> : ipx_mailbox_min {};
template <>
struct ipx_mailbox<IP_COMBINE_MIN, 8> : ipx_mailbox_min {};
template <>
struct ipx_mailbox<IP_COMBINE_MAX, 4> : ipx_mailbox_max {};
template <>
struct ipx_mailbox<IP_COMBINE_MAX, 8> : ipx_mailbox_max {};

template <int MSGBYTES>
struct ipx_mailbox<IP_COMBINE_SUM, MSGBYTES> {
    typedef ipx_msg slot;
    __device__ static slot empty() { return (ipx_msg)0; }
    __device__ static bool precheck(slot*, ipx_msg) { return true; }
    __device__ static bool deliver(slot* s, ipx_msg m)
    {
        ipx_atomic_add(s, m);
        return true;
    }
    __device__ static bool commit(slot* s, ipx_msg m) { return deliver(s, m); }
    __device__ static bool merge(slot* s, ipx_msg m)
    {
        *s = *s + m;
        return true;
    }
    __device__ static ipx_msg take(slot* s)
    {
        ipx_msg m = *s;
        *s = (ipx_msg)0;
        return m;
    }
};

/* Generic, up to 4 bytes: {flag, bits} in one 64-bit word, CAS loop around
 * the user's ip_combine with the early exit of ip_cas (combiner_postamble.h:
 * 41-52): no write when combining leaves the mailbox unchanged. */
template <int MSGBYTES>
struct ipx_mailbox_generic32 {
    typedef unsigned long long slot;
    __device__ static slot empty() { return 0ULL; }
    __device__ static bool precheck(slot*, ipx_msg) { return true; }
    __device__ static bool commit(slot* s, ipx_msg m) { return deliver(s, m); }
    __device__ static bool deliver(slot* s, ipx_msg m)
    {
        unsigned long long old = __ldcg(s);
        for (;;) {
            unsigned long long nw;
            if (old >> 32) {
                ipx_msg cur = ipx_from_word<ipx_msg>((unsigned int)old);
                ipx_msg nv = cur;
                ip_combine(&nv, m);
                unsigned int nb = ipx_to_word(nv);
                if (nb == (unsigned int)old) return false;
                nw = (1ULL << 32) | nb;
            } else {
                nw = (1ULL << 32) | ipx_to_word(m);
            }
            unsigned long long prev = atomicCAS(s, old, nw);
            if (prev == old) return (old >> 32) == 0;
            old = prev;
        }
    }
    __device__ static bool merge(slot* s, ipx_msg m)
    {
        const unsigned long long old = *s;
        ipx_msg v = m;
        if (old >> 32) {
            v = ipx_from_word<ipx_msg>((unsigned int)old);
            ip_combine(&v, m);
        }
        *s = (1ULL << 32) | ipx_to_word(v);
        return true;
    }
    __device__ static ipx_msg take(slot* s)
    {
        unsigned long long w = *s;
        *s = 0ULL;
        return ipx_from_word<ipx_msg>((unsigned int)w);
    }
};

template <>
struct ipx_mailbox<IP_COMBINE_GENERIC, 1> : ipx_mailbox_generic32<1> {};
template <>
struct ipx_mailbox<IP_COMBINE_GENERIC, 2> : ipx_mailbox_generic32<2> {};
template <>
struct ipx_mailbox<IP_COMBINE_GENERIC, 4> : ipx_mailbox_generic32<4> {};

/* Generic, 8 bytes: {flag, bits} in a 16-byte slot with a 128-bit CAS. */
template <>
struct ipx_mailbox<IP_COMBINE_GENERIC, 8> {
    typedef ipx_slot128 slot;
    __device__ static slot empty() { return slot{0ULL, 0ULL}; }
    __device__ static bool precheck(slot*, ipx_msg) { return true; }
    __device__ static bool commit(slot* s, ipx_msg m) { return deliver(s, m); }
    __device__ static bool deliver(slot* s, ipx_msg m)
    {
        unsigned long long of = __ldcg(&s->flag), ob = __ldcg(&s->bits);
        for (;;) {
            unsigned long long nb;
            if (of) {
                ipx_msg cur = ipx_from_word<ipx_msg>(ob);
                ipx_msg nv = cur;
                ip_combine(&nv, m);
                nb = ipx_to_word(nv);
                if (nb == ob) return false;
            } else {
                nb = ipx_to_word(m);
            }
            unsigned long long pf, pb;
            ipx_cas128(s, of, ob, 1ULL, nb, pf, pb);
            if (pf == of && pb == ob) return of == 0;
            of = pf;
            ob = pb;
        }
    }
    __device__ static bool merge(slot* s, ipx_msg m)
    {
        ipx_msg v = m;
        if (s->flag) {
            v = ipx_from_word<ipx_msg>(s->bits);
            ip_combine(&v, m);
        }
        s->bits = ipx_to_word(v);
        s->flag = 1ULL;
        return true;
    }
    __device__ static ipx_msg take(slot* s)
    {
        slot w = *s;
        *s = slot{0ULL, 0ULL};
        return ipx_from_word<ipx_msg>(w.bits);
    }
};

template <>
struct ipx_mailbox<IP_COMBINE_MIN, 1> : ipx_mailbox_generic32<1> {};
template <>
struct ipx_mailbox<IP_COMBINE_MIN, 2> : ipx_mailbox_generic32<2> {};
template <>
struct ipx_mailbox<IP_COMBINE_MAX, 1> : ipx_mailbox_generic32<1> {};
template <>
struct ipx_mailbox<IP_COMBINE_MAX, 2> : ipx_mailbox_generic32<2> {};

typedef ipx_mailbox<IP_COMBINE_KIND, (int)sizeof(ipx_msg)> ipx_mb;
typedef typename ipx_mb::slot ipx_slot;

/* ------------------------------------------------------------------------ */
/* Device-resident engine state, read through the constant bank.            */
/* ------------------------------------------------------------------------ */
struct ipx_consts {
    uint64_t V, E, W;  /* W = bitmap words */
    const uint64_t* row;
    const ipx_vid* adj;
    const ipx_wgt* wgt;
    const uint64_t* in_row;
    const ipx_vid* in_adj;
    const ipx_wgt* in_wgt;
    ipx_val* value;
    /* combiner */
    uint32_t* active_bm;
    uint32_t* hasmsg_bm;
    /* pulls */
    uint8_t* active_b;
    uint8_t* hasmsg_b;
    ipx_msg* msg;
    /* push mail */
    ipx_slot* mbox[2];
    uint32_t* recv[2];
    ipx_msg* outbox;
    uint32_t* bcaster;
    /* pull broadcast slots */
    ipx_msg* bval;
    uint32_t* has_b;
    uint32_t* bt;
    /* counters: [0..3] active counts ring, [4] edges, [5] error word */
    unsigned long long* ctr;
    uint32_t* err;
    /* direction optimisation (push versions on symmetric graphs) */
    int pull_ok;
    /* list sizes ([0..2] broadcaster classes, [4..6] targets) and the
     * per-superstep history of a captured loop: hist[s % IPX_HIST][0..3] =
     * active count, edges traversed, direction, unused */
    uint32_t* lcnt;
    unsigned long long* hist;
};

__constant__ ipx_consts ipx_c;

/* The current superstep, from device memory: the host writes it before each
 * superstep (host loop), or the previous superstep's last kernel advances it
 * (captured loop), so every kernel of a superstep reads the same value. */
__device__ __forceinline__ uint64_t ipx_step() { return (uint64_t)__ldg((const unsigned long long*)&ipd_superstep); }
__device__ __forceinline__ int ipx_parity() { return (int)(ipx_step() & 1); }

/* ctr layout (u64): [0..3] active-count ring, [5] error word (low half),
 * [8..10] degree sums of the broadcaster classes, [11..13] of the target
 * classes, both reset every superstep. */
#define IPX_NCTR 16
#define IPX_CTR_ERR 5
/* [6]: delivery direction of the current superstep (0 push, 1 pull). */
#define IPX_CTR_MODE 6

/* Kernel ids for launch counting and per-kernel profiling. */
enum {
    IPX_K_COMPUTE,
    IPX_K_COMPACT_B,
    IPX_K_PUSH0,
    IPX_K_PUSH1,
    IPX_K_PUSH2,
    IPX_K_COMPACT_T,
    IPX_K_GATHER0,
    IPX_K_GATHER1,
    IPX_K_GATHER2,
    IPX_K_MARK0,
    IPX_K_MARK1,
    IPX_K_MARK2,
    IPX_K_COUNT,
    IPX_K_PULLD0,
    IPX_K_PULLD1,
    IPX_K_PULLD2,
    IPX_K_CTRL,
    IPX_K_N
};
static const char* const ipx_kname[IPX_K_N] = {
    "compute", "compact_broadcasters", "push_thread", "push_warp", "push_block", "compact_targets",
    "gather_thread", "gather_warp", "gather_block", "mark_thread", "mark_warp", "mark_block", "count_active",
    "pull_deliver_thread", "pull_deliver_warp", "pull_deliver_block",
    "superstep_control"};

__device__ __forceinline__ uint64_t ipx_gtid() { return blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint64_t ipx_gstride() { return (uint64_t)gridDim.x * blockDim.x; }
__device__ __forceinline__ bool ipx_test(const uint32_t* bm, uint64_t v) { return (bm[v >> 5] >> (v & 31)) & 1u; }

/* Load of an edge stream element (neighbour id, weight).  A superstep reads
 * each edge once, and the streams are gigabytes, so they are loaded
 * evict-first (ld.global.cs): the L2 stays with the vertex arrays that edges
 * read at random (mailboxes, broadcast values, bitmaps). */
template <class T>
__device__ __forceinline__ T ipx_ld_stream(const T* p)
{
    T r;
    if constexpr (sizeof(T) == 8) {
        const unsigned long long w = __ldcs(reinterpret_cast<const unsigned long long*>(p));
        memcpy(&r, &w, 8);
    } else if constexpr (sizeof(T) == 4) {
        const unsigned int w = __ldcs(reinterpret_cast<const unsigned int*>(p));
        memcpy(&r, &w, 4);
    } else if constexpr (sizeof(T) == 2) {
        const unsigned short w = __ldcs(reinterpret_cast<const unsigned short*>(p));
        memcpy(&r, &w, 2);
    } else if constexpr (sizeof(T) == 1) {
        const unsigned char w = __ldcs(reinterpret_cast<const unsigned char*>(p));
        memcpy(&r, &w, 1);
    } else {
        r = *p;
    }
    return r;
}

/* Edge element read by a loop whose lanes take every lanes-th edge: evict-
 * first only when a warp reads consecutive edges in one instruction (lanes
 * >= 32).  A thread walking a short row alone (lanes = 1) comes back to the
 * same line in its next steps, and an evict-first line is often gone by
 * then (measured: more DRAM traffic and a slower thread class). */
template <class T>
__device__ __forceinline__ T ipx_ld_edge(const T* p, uint64_t lanes)
{
    return lanes >= 32 ? ipx_ld_stream(p) : *p;
}

/* Sets bit v of a shared bitmap; lanes that hit the same word combine first. */
__device__ __forceinline__ void ipx_set_bit_agg(uint32_t* bm, uint64_t v)
{
    const unsigned act = __activemask();
    const unsigned long long word = v >> 5;
    const unsigned peers = __match_any_sync(act, word);
    const unsigned bits = __reduce_or_sync(peers, 1u << (v & 31));
    if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicOr(&bm[word], bits);
}

/* Sets bit v if it is clear; returns nothing (idempotent). */
__device__ __forceinline__ void ipx_mark(uint32_t* bm, uint64_t v)
{
    const uint32_t bit = 1u << (v & 31);
    if (!(__ldcg(&bm[v >> 5]) & bit)) atomicOr(&bm[v >> 5], bit);
}

/* Warp + block sum into a global counter (all threads of the block call). */
__device__ __forceinline__ void ipx_block_count(unsigned long long c, unsigned long long* dst)
{
    __shared__ unsigned long long s_part[IPX_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(IPX_FULL, c, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_part[w];
        if (t) atomicAdd(dst, t);
    }
}

/* Delivery of one message into mailbox parity p of vertex w. */
__device__ __forceinline__ void ipx_deliver(int p, uint64_t w, ipx_msg m)
{
    if (ipx_mb::deliver(&ipx_c.mbox[p][w], m)) atomicOr(&ipx_c.recv[p][w >> 5], 1u << (w & 31));
}

/* Edges per chunk of a high-degree vertex: the block class is split into
 * chunks that all CTAs share, so one hub does not leave a single CTA working
 * after the others have finished. */
#ifndef IPX_HUB_CHUNK
#define IPX_HUB_CHUNK 2048
#endif
#ifndef IPX_UNROLL
#define IPX_UNROLL 4
#endif
/* 1: sources of the thread and warp classes go through the warp-cooperative
 * expansion; 0: a thread per source (degree <= IPX_T0), a warp per source. */
#ifndef IPX_PUSH_EXPAND
#define IPX_PUSH_EXPAND 0
#endif

template <class T>
__device__ __forceinline__ T ipx_shfl_idx(T x, int src)
{
    typedef typename ipx_word<T>::type W;
    W w = ipx_to_word(x);
    w = __shfl_sync(IPX_FULL, w, src);
    return ipx_from_word<T>(w);
}

/* A visitor gets batches of U edges: edge index e[k], target w[k], the
 * source's message m[k] (outbox value) and ok[k] (lane holds an edge). */

/* Push visitor: prechecks a batch of mailboxes first, then commits. */
struct ipx_push_visit {
    static constexpr bool kNeedsMessage = true;
    int p;
    bool warp_wide; /* a warp or CTA walks each source's edges (weights loaded evict-first) */
    template <int U>
    __device__ __forceinline__ void batch(const uint64_t* e, const ipx_vid* w, const ipx_msg* m, const bool* ok) const
    {
        ipx_msg mk[U];
        bool go[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            go[k] = false;
            if (ok[k]) {
#if IPX_EDGE_MSG
                mk[k] = IP_BROADCAST_EDGE_MESSAGE(m[k], warp_wide ? ipx_ld_stream(&ipx_c.wgt[e[k]]) : ipx_c.wgt[e[k]]);
#else
                mk[k] = m[k];
#endif
                go[k] = ipx_mb::precheck(&ipx_c.mbox[p][(uint64_t)w[k]], mk[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            const uint64_t t = (uint64_t)w[k];
            if (go[k] && ipx_mb::commit(&ipx_c.mbox[p][t], mk[k])) atomicOr(&ipx_c.recv[p][t >> 5], 1u << (t & 31));
        }
    }
};

/* Target-marking visitor (spread+single_broadcast). */
struct ipx_mark_visit {
    static constexpr bool kNeedsMessage = false;
    template <int U>
    __device__ __forceinline__ void batch(const uint64_t* e, const ipx_vid* w, const ipx_msg* m, const bool* ok) const
    {
        (void)e;
        (void)m;
        uint32_t cur[U];
#pragma unroll
        for (int k = 0; k < U; k++) cur[k] = ok[k] ? __ldcg(&ipx_c.bt[(uint64_t)w[k] >> 5]) : IPX_FULL;
#pragma unroll
        for (int k = 0; k < U; k++) {
            const uint32_t bit = 1u << ((uint64_t)w[k] & 31);
            if (!(cur[k] & bit)) atomicOr(&ipx_c.bt[(uint64_t)w[k] >> 5], bit);
        }
    }
};

/* Visits edges [e0, e1) of one source lane-strided, IPX_UNROLL edges a lane
 * at a time, loading the ids of a batch before visiting any of it. */
template <class Visit>
__device__ __forceinline__ void ipx_edges_strided(const ipx_vid* __restrict__ adj, uint64_t e0, uint64_t e1,
                                                  uint64_t lane, uint64_t lanes, ipx_msg m, const Visit& visit)
{
    for (uint64_t e = e0 + lane; e < e1; e += IPX_UNROLL * lanes) {
        uint64_t ek[IPX_UNROLL];
        ipx_vid w[IPX_UNROLL];
        ipx_msg mk[IPX_UNROLL];
        bool ok[IPX_UNROLL];
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++) {
            ek[k] = e + k * lanes;
            ok[k] = ek[k] < e1;
            w[k] = ok[k] ? ipx_ld_edge(&adj[ek[k]], lanes) : (ipx_vid)0;
            mk[k] = m;
        }
        visit.template batch<IPX_UNROLL>(ek, w, mk, ok);
    }
}

/* Warp-cooperative expansion: a warp takes 32 sources of a list at once
 * (one coalesced read of their ids, row bounds and messages), scans their
 * degrees, and spreads the concatenated edges over its lanes, so every lane
 * has work whatever the degrees and the per-source load latency is paid once
 * per 32 sources.  Each lane finds its source by a 5-step search over the
 * warp's exclusive degree prefix (shuffles). */
template <class Visit>
__device__ __forceinline__ void ipx_warp_expand(const uint32_t* __restrict__ list, uint64_t n, const Visit& visit)
{
    const ipx_vid* __restrict__ adj = ipx_c.adj;
    const uint64_t* __restrict__ row = ipx_c.row;
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ipx_gstride() >> 5;
    for (uint64_t base = (ipx_gtid() >> 5) * 32; base < n; base += nwarps * 32) {
        uint64_t r0 = 0;
        uint32_t deg = 0;
        ipx_msg m = ipx_msg();
        if (base + lane < n) {
            const uint64_t u = list[base + lane];
            r0 = row[u];
            deg = (uint32_t)(row[u + 1] - r0);
            if constexpr (Visit::kNeedsMessage) m = ipx_c.outbox[u];
        }
        uint32_t inc = deg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(IPX_FULL, inc, o);
            if (lane >= o) inc += t;
        }
        const uint32_t excl = inc - deg;
        const uint32_t total = __shfl_sync(IPX_FULL, inc, 31);
        for (uint32_t t0 = 0; t0 < total; t0 += 32 * IPX_UNROLL) {
            uint64_t ek[IPX_UNROLL];
            ipx_vid w[IPX_UNROLL];
            ipx_msg mk[IPX_UNROLL];
            bool ok[IPX_UNROLL];
#pragma unroll
            for (int k = 0; k < IPX_UNROLL; k++) {
                const uint32_t pos = t0 + (uint32_t)(k * 32 + lane);
                int j = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const uint32_t ex = __shfl_sync(IPX_FULL, excl, j + step);
                    if (ex <= pos) j += step;
                }
                const uint64_t rj = __shfl_sync(IPX_FULL, r0, j);
                const uint32_t xj = __shfl_sync(IPX_FULL, excl, j);
                mk[k] = ipx_shfl_idx(m, j);
                ok[k] = pos < total;
                ek[k] = rj + (pos - xj);
                w[k] = ok[k] ? ipx_ld_stream(&adj[ek[k]]) : (ipx_vid)0;
            }
            visit.template batch<IPX_UNROLL>(ek, w, mk, ok);
        }
    }
}

/* Chunk prefix of the high-degree class: prefix[i] = chunks of the hubs before
 * i, prefix[n] = total (one block, a carried scan over tiles of its width). */
__global__ void __launch_bounds__(1024) ipx_k_hub_prefix(const uint32_t* __restrict__ list,
                                                         const uint32_t* __restrict__ count,
                                                         const uint64_t* __restrict__ row, uint32_t* __restrict__ prefix)
{
    __shared__ uint32_t s[1024];
    const uint64_t n = *count;
    uint32_t carry = 0;
    for (uint64_t base = 0; base < n; base += 1024) {
        const uint64_t i = base + threadIdx.x;
        uint32_t c = 0;
        if (i < n) {
            const uint64_t u = list[i];
            c = (uint32_t)((row[u + 1] - row[u] + IPX_HUB_CHUNK - 1) / IPX_HUB_CHUNK);
        }
        s[threadIdx.x] = c;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const uint32_t x = (threadIdx.x >= (unsigned)o) ? s[threadIdx.x - o] : 0u;
            __syncthreads();
            s[threadIdx.x] += x;
            __syncthreads();
        }
        if (i < n) prefix[i] = carry + s[threadIdx.x] - c;
        carry += s[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) prefix[n] = carry;
}

/* Hub index of chunk c: the last i with prefix[i] <= c. */
__device__ __forceinline__ uint64_t ipx_hub_of_chunk(const uint32_t* __restrict__ prefix, uint64_t n, uint32_t c)
{
    uint64_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= c) lo = mid;
        else hi = mid;
    }
    return lo;
}

/* ---- the vertex functions that depend on the version ---- */
__device__ inline void ip_broadcast(struct ip_vertex_t* v, IP_MESSAGE_TYPE message)
{
#if IPX_PULL
    /* single_broadcast: write the vertex's own slot (combiner_single_broadcast_
     * postamble.h:51-55); spread+single_broadcast also flags the out-neighbours
     * as targets (combiner_spread_single_broadcast_postamble.h:64-76), which the
     * engine does after the compute kernel. */
    v->ipx_has_out = true;
    v->ipx_out = message;
#else
    /* combiner / spread: every out-neighbour receives the message
     * (combiner_postamble.h:81-87); two broadcasts in one call are combined. */
    if (v->ipx_has_out) {
        ip_combine(&v->ipx_out, message);
    } else {
        v->ipx_has_out = true;
        v->ipx_out = message;
    }
#endif
}

__device__ inline void ip_send_message(IP_VERTEX_ID_TYPE id, IP_MESSAGE_TYPE message)
{
#if IPX_PULL
    /* Fatal in the single-broadcast versions (combiner_single_broadcast_
     * postamble.h:42-49): flagged here, reported and exited on the host. */
    (void)id;
    (void)message;
    atomicOr(ipx_c.err, IPX_ERR_SEND_IN_BROADCAST);
#else
    ipx_deliver((int)(ip_get_superstep() & 1), (uint64_t)id, message);
#endif
}

__device__ inline void ip_vote_to_halt(struct ip_vertex_t* v)
{
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SINGLE_BROADCAST
    v->active = false;
#else
    (void)v; /* spread versions ignore it (combiner_spread_postamble.h:433-436) */
#endif
}

/* Fills the neighbour fields of the proxy (loads the compiler drops when
 * ip_compute does not read them). */
__device__ __forceinline__ void ipx_fill_topology(struct ip_vertex_t& x, uint64_t v)
{
#if defined(IP_NEEDS_OUT_NEIGHBOUR_IDS) || defined(IP_NEEDS_OUT_NEIGHBOUR_COUNT) || IPX_OUT_WEIGHTS
    const uint64_t r0 = ipx_c.row[v], r1 = ipx_c.row[v + 1];
#endif
#ifdef IP_NEEDS_OUT_NEIGHBOUR_IDS
    x.out_neighbours = const_cast<ipx_vid*>(ipx_c.adj + r0);
#endif
#ifdef IP_NEEDS_OUT_NEIGHBOUR_COUNT
    x.out_neighbour_count = (IP_NEIGHBOUR_COUNT_TYPE)(r1 - r0);
#endif
#if IPX_OUT_WEIGHTS
    x.out_neighbour_weights = const_cast<ipx_wgt*>(ipx_c.wgt + r0);
#endif
#if defined(IP_NEEDS_IN_NEIGHBOUR_IDS) || defined(IP_NEEDS_IN_NEIGHBOUR_COUNT) || IPX_IN_WEIGHTS
    const uint64_t q0 = ipx_c.in_row[v], q1 = ipx_c.in_row[v + 1];
#endif
#ifdef IP_NEEDS_IN_NEIGHBOUR_IDS
    x.in_neighbours = const_cast<ipx_vid*>(ipx_c.in_adj + q0);
#endif
#ifdef IP_NEEDS_IN_NEIGHBOUR_COUNT
    x.in_neighbour_count = (IP_NEIGHBOUR_COUNT_TYPE)(q1 - q0);
#endif
#if IPX_IN_WEIGHTS
    x.in_neighbour_weights = const_cast<ipx_wgt*>(ipx_c.in_wgt + q0);
#endif
}

/* ------------------------------------------------------------------------ */
/* Push delivery over degree-class lists of broadcasters.                   */
/* MODE 0: a thread per broadcaster; 1: a warp; 2: a block.                 */
/* ------------------------------------------------------------------------ */
/* Runs a visitor over the out-edges of a degree-class list of sources:
 * MODE 0 and 1 by warp-cooperative expansion, MODE 2 (the hubs) a CTA per
 * IPX_HUB_CHUNK-edge chunk, chunks located through `prefix`. */
template <int MODE, class Visit>
__device__ __forceinline__ void ipx_over_sources(const uint32_t* __restrict__ list, uint64_t n,
                                                 const uint32_t* __restrict__ prefix, const Visit& visit)
{
    if constexpr ((MODE == 0 || MODE == 1) && IPX_PUSH_EXPAND) {
        ipx_warp_expand(list, n, visit);
    } else if constexpr (MODE == 0 && sizeof(ipx_vid) == 8) {
        /* 64-bit ids: the loop below would spill registers */
        const ipx_vid* __restrict__ adj = ipx_c.adj;
        const uint64_t* __restrict__ row = ipx_c.row;
        for (uint64_t i = ipx_gtid(); i < n; i += ipx_gstride()) {
            const uint64_t u = list[i];
            ipx_msg m = ipx_msg();
            if constexpr (Visit::kNeedsMessage) m = ipx_c.outbox[u];
            ipx_edges_strided(adj, row[u], row[u + 1], 0, 1, m, visit);
        }
    } else if constexpr (MODE == 0) {
        /* the next source's list entry, row bounds and message are loaded
         * while this source's edges are visited */
        const ipx_vid* __restrict__ adj = ipx_c.adj;
        const uint64_t* __restrict__ row = ipx_c.row;
        const uint64_t stride = ipx_gstride();
        uint64_t i = ipx_gtid(), r0 = 0, r1 = 0;
        ipx_msg m = ipx_msg();
        if (i < n) {
            const uint64_t u = list[i];
            r0 = row[u];
            r1 = row[u + 1];
            if constexpr (Visit::kNeedsMessage) m = ipx_c.outbox[u];
        }
        for (; i < n; i += stride) {
            uint64_t r0n = 0, r1n = 0;
            ipx_msg mn = ipx_msg();
            if (i + stride < n) {
                const uint64_t un = list[i + stride];
                r0n = row[un];
                r1n = row[un + 1];
                if constexpr (Visit::kNeedsMessage) mn = ipx_c.outbox[un];
            }
            ipx_edges_strided(adj, r0, r1, 0, 1, m, visit);
            r0 = r0n;
            r1 = r1n;
            m = mn;
        }
    } else if constexpr (MODE == 1) {
        const ipx_vid* __restrict__ adj = ipx_c.adj;
        const uint64_t* __restrict__ row = ipx_c.row;
        const uint64_t lane = threadIdx.x & 31;
        for (uint64_t i = ipx_gtid() >> 5; i < n; i += ipx_gstride() >> 5) {
            const uint64_t u = list[i];
            ipx_msg m = ipx_msg();
            if constexpr (Visit::kNeedsMessage) m = ipx_c.outbox[u];
            ipx_edges_strided(adj, row[u], row[u + 1], lane, 32, m, visit);
        }
    } else {
        if (n == 0) return;
        const ipx_vid* __restrict__ adj = ipx_c.adj;
        const uint64_t* __restrict__ row = ipx_c.row;
        const uint32_t chunks = prefix[n];
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint64_t i = ipx_hub_of_chunk(prefix, n, c);
            const uint64_t u = list[i];
            const uint64_t e0 = row[u] + (uint64_t)(c - prefix[i]) * IPX_HUB_CHUNK;
            const uint64_t end = row[u + 1];
            const uint64_t e1 = (e0 + IPX_HUB_CHUNK < end) ? e0 + IPX_HUB_CHUNK : end;
            ipx_msg m = ipx_msg();
            if constexpr (Visit::kNeedsMessage) m = ipx_c.outbox[u];
            ipx_edges_strided(adj, e0, e1, threadIdx.x, blockDim.x, m, visit);
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(IPX_THREADS, IPX_EDGE_CTAS) ipx_k_push(const uint32_t* __restrict__ list,
                                                          const uint32_t* __restrict__ count,
                                                          const uint32_t* __restrict__ prefix)
{
    if (ipx_c.pull_ok && __ldcg(&ipx_c.ctr[IPX_CTR_MODE])) return; /* this superstep pulls */
    ipx_over_sources<MODE>(list, *count, prefix, ipx_push_visit{ipx_parity(), MODE != 0});
}

/* Direction of the superstep's delivery: pull when the broadcasters' out-edges
 * (degree sums of the compaction) exceed `threshold`. */
__global__ void ipx_k_decide(unsigned long long threshold)
{
    const unsigned long long m = ipx_c.ctr[8] + ipx_c.ctr[9] + ipx_c.ctr[10];
    ipx_c.ctr[IPX_CTR_MODE] = (m > threshold) ? 1ULL : 0ULL;
}

/* Marks the out-neighbours of broadcasters as targets (spread+single_broadcast). */
template <int MODE>
__global__ void __launch_bounds__(IPX_THREADS, IPX_EDGE_CTAS) ipx_k_mark(const uint32_t* __restrict__ list,
                                                          const uint32_t* __restrict__ count,
                                                          const uint32_t* __restrict__ prefix)
{
    ipx_over_sources<MODE>(list, *count, prefix, ipx_mark_visit{});
}

/* ------------------------------------------------------------------------ */
/* Pull gather (ip_fetch_broadcast_messages, combiner_single_broadcast_      */
/* postamble.h:57-89): fold ip_combine over the in-neighbours that           */
/* broadcast.  MODE 0 folds in adjacency order, as the reference does; the   */
/* warp and block modes fold lane-strided runs in order and then combine the */
/* partial results in a tree.                                                */
/* ------------------------------------------------------------------------ */
__device__ __forceinline__ void ipx_fold(bool& has, ipx_msg& acc, bool oh, ipx_msg om)
{
    if (oh) {
        if (has) {
            ip_combine(&acc, om);
        } else {
            acc = om;
            has = true;
        }
    }
}

__device__ __forceinline__ void ipx_warp_fold(bool& has, ipx_msg& acc)
{
    for (int o = 16; o > 0; o >>= 1) {
        bool oh = __shfl_down_sync(IPX_FULL, has, o);
        ipx_msg om = ipx_shfl_down(acc, o);
        ipx_fold(has, acc, oh, om);
    }
}

/* Folds the broadcasts of the in-neighbours at edges e0 + lane, e0 + lane +
 * lanes, ... below e1, in that order.  IPX_UNROLL edges a step: their ids,
 * then their broadcast bits, then the values of the set bits are each loaded
 * for all IPX_UNROLL edges before the next level, so a lane has IPX_UNROLL
 * independent loads in flight instead of one three-load chain per edge. */
__device__ __forceinline__ void ipx_gather_fold_edges(const ipx_vid* __restrict__ adj, const uint32_t* __restrict__ hb,
                                                      const ipx_msg* __restrict__ bv, uint64_t e0, uint64_t e1,
                                                      uint64_t lane, uint64_t lanes, bool& has, ipx_msg& acc)
{
    for (uint64_t e = e0 + lane; e < e1; e += IPX_UNROLL * lanes) {
        uint64_t u[IPX_UNROLL];
        uint32_t word[IPX_UNROLL];
        bool on[IPX_UNROLL];
        ipx_msg m[IPX_UNROLL];
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++)
            u[k] = (e + k * lanes < e1) ? (uint64_t)ipx_ld_edge(&adj[e + k * lanes], lanes) : 0;
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++) word[k] = (e + k * lanes < e1) ? __ldg(&hb[u[k] >> 5]) : 0u;
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++) {
            on[k] = (word[k] >> (u[k] & 31)) & 1u;
            if (on[k]) m[k] = __ldg(&bv[u[k]]);
        }
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++)
            if (on[k]) ipx_fold(has, acc, true, m[k]);
    }
}

/* REACT: reactivate and count (single_broadcast) or not (spread+single_broadcast). */
template <int MODE, bool REACT>
__global__ void __launch_bounds__(IPX_THREADS, IPX_EDGE_CTAS) ipx_k_gather(const uint32_t* __restrict__ list,
                                                            const uint32_t* __restrict__ count_dev,
                                                            uint64_t count_host)
{
    const int ctr_slot = (int)(ipx_step() & 3);
    const uint64_t n = count_dev ? (uint64_t)*count_dev : count_host;
    const ipx_vid* __restrict__ adj = ipx_c.in_adj;
    const uint64_t* __restrict__ row = ipx_c.in_row;
    const uint32_t* __restrict__ hb = ipx_c.has_b;
    const ipx_msg* __restrict__ bv = ipx_c.bval;
    unsigned long long react = 0;
    if constexpr (MODE == 0) {
        /* the next vertex's list entry is loaded while this vertex's
         * in-edges are folded (its row bounds too would spill registers) */
        const uint64_t stride = ipx_gstride();
        uint64_t i = ipx_gtid(), v = (i < n) ? list[i] : 0;
        for (; i < n; i += stride) {
            const uint64_t vn = (i + stride < n) ? list[i + stride] : 0;
            bool has = false;
            ipx_msg acc;
            ipx_gather_fold_edges(adj, hb, bv, row[v], row[v + 1], 0, 1, has, acc);
            ipx_c.hasmsg_b[v] = has;
            if (has) {
                ipx_c.msg[v] = acc;
                if constexpr (REACT) {
                    if (!ipx_c.active_b[v]) {
                        ipx_c.active_b[v] = 1;
                        react++;
                    }
                }
            }
            v = vn;
        }
    } else if constexpr (MODE == 1) {
        const int lane = threadIdx.x & 31;
        for (uint64_t i = ipx_gtid() >> 5; i < n; i += ipx_gstride() >> 5) {
            const uint64_t v = list[i];
            bool has = false;
            ipx_msg acc;
            ipx_gather_fold_edges(adj, hb, bv, row[v], row[v + 1], lane, 32, has, acc);
            ipx_warp_fold(has, acc);
            if (lane == 0) {
                ipx_c.hasmsg_b[v] = has;
                if (has) {
                    ipx_c.msg[v] = acc;
                    if constexpr (REACT) {
                        if (!ipx_c.active_b[v]) {
                            ipx_c.active_b[v] = 1;
                            react++;
                        }
                    }
                }
            }
        }
    } else {
        __shared__ bool s_has[IPX_THREADS / 32];
        __shared__ ipx_msg s_acc[IPX_THREADS / 32];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (uint64_t i = blockIdx.x; i < n; i += gridDim.x) {
            const uint64_t v = list[i];
            bool has = false;
            ipx_msg acc;
            ipx_gather_fold_edges(adj, hb, bv, row[v], row[v + 1], threadIdx.x, blockDim.x, has, acc);
            ipx_warp_fold(has, acc);
            if (lane == 0) {
                s_has[warp] = has;
                s_acc[warp] = acc;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                has = false;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) ipx_fold(has, acc, s_has[w], s_acc[w]);
                ipx_c.hasmsg_b[v] = has;
                if (has) {
                    ipx_c.msg[v] = acc;
                    if constexpr (REACT) {
                        if (!ipx_c.active_b[v]) {
                            ipx_c.active_b[v] = 1;
                            react++;
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    if constexpr (REACT) ipx_block_count(react, &ipx_c.ctr[ctr_slot]);
}

/* ------------------------------------------------------------------------ */
/* Pull delivery for the push versions (direction optimisation).  On a       */
/* symmetric graph a vertex's row lists exactly the vertices that would push */
/* to it, so folding the messages of its broadcasting row-neighbours gives   */
/* the message a push would have left in its mailbox (the fold order differs */
/* only as ip_combine's contract allows).  Used in dense supersteps: it      */
/* streams every row once and needs no atomics except for the hubs' chunks.  */
/* MODE 0: thread per vertex, 1: warp per vertex, 2: CTA per 2048-edge chunk */
/* of a high-degree vertex, committed with the mailbox's atomic.             */
/* ------------------------------------------------------------------------ */
__device__ __forceinline__ void ipx_pull_fold_edges(uint64_t e0, uint64_t e1, uint64_t lane, uint64_t lanes, bool& has,
                                                    ipx_msg& acc)
{
    const ipx_vid* __restrict__ adj = ipx_c.in_adj;
    const uint32_t* __restrict__ bc = ipx_c.bcaster;
    const ipx_msg* __restrict__ ob = ipx_c.outbox;
    for (uint64_t e = e0 + lane; e < e1; e += IPX_UNROLL * lanes) {
        uint64_t u[IPX_UNROLL];
        uint32_t word[IPX_UNROLL];
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++) {
            const uint64_t ek = e + k * lanes;
            u[k] = (ek < e1) ? (uint64_t)ipx_ld_edge(&adj[ek], lanes) : 0;
            word[k] = (ek < e1) ? __ldg(&bc[u[k] >> 5]) : 0u;
        }
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++) {
            if ((word[k] >> (u[k] & 31)) & 1u) {
#if IPX_EDGE_MSG
                ipx_msg m = IP_BROADCAST_EDGE_MESSAGE(__ldg(&ob[u[k]]), ipx_ld_edge(&ipx_c.in_wgt[e + k * lanes], lanes));
#else
                ipx_msg m = __ldg(&ob[u[k]]);
#endif
                ipx_fold(has, acc, true, m);
            }
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(IPX_THREADS, IPX_EDGE_CTAS) ipx_k_pull_deliver(const uint32_t* __restrict__ list,
                                                                                uint64_t n,
                                                                                const uint32_t* __restrict__ prefix)
{
    if (!__ldcg(&ipx_c.ctr[IPX_CTR_MODE])) return; /* this superstep pushes */
    const int p = ipx_parity();
    const uint64_t* __restrict__ row = ipx_c.in_row;
    if constexpr (MODE == 0) {
        for (uint64_t i = ipx_gtid(); i < n; i += ipx_gstride()) {
            const uint64_t v = list[i];
            bool has = false;
            ipx_msg acc;
            ipx_pull_fold_edges(row[v], row[v + 1], 0, 1, has, acc);
            if (has && ipx_mb::merge(&ipx_c.mbox[p][v], acc)) ipx_set_bit_agg(ipx_c.recv[p], v);
        }
    } else if constexpr (MODE == 1) {
        const int lane = threadIdx.x & 31;
        for (uint64_t i = ipx_gtid() >> 5; i < n; i += ipx_gstride() >> 5) {
            const uint64_t v = list[i];
            bool has = false;
            ipx_msg acc;
            ipx_pull_fold_edges(row[v], row[v + 1], lane, 32, has, acc);
            ipx_warp_fold(has, acc);
            if (lane == 0 && has && ipx_mb::merge(&ipx_c.mbox[p][v], acc))
                atomicOr(&ipx_c.recv[p][v >> 5], 1u << (v & 31));
        }
    } else {
        __shared__ bool s_has[IPX_THREADS / 32];
        __shared__ ipx_msg s_acc[IPX_THREADS / 32];
        if (n == 0) return;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const uint32_t chunks = prefix[n];
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint64_t i = ipx_hub_of_chunk(prefix, n, c);
            const uint64_t v = list[i];
            const uint64_t e0 = row[v] + (uint64_t)(c - prefix[i]) * IPX_HUB_CHUNK;
            const uint64_t e1 = (e0 + IPX_HUB_CHUNK < row[v + 1]) ? e0 + IPX_HUB_CHUNK : row[v + 1];
            bool has = false;
            ipx_msg acc;
            ipx_pull_fold_edges(e0, e1, threadIdx.x, blockDim.x, has, acc);
            ipx_warp_fold(has, acc);
            if (lane == 0) {
                s_has[warp] = has;
                s_acc[warp] = acc;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                has = false;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) ipx_fold(has, acc, s_has[w], s_acc[w]);
                /* chunks of one hub meet in its mailbox: the atomic delivery */
                if (has && ipx_mb::deliver(&ipx_c.mbox[p][v], acc)) atomicOr(&ipx_c.recv[p][v >> 5], 1u << (v & 31));
            }
            __syncthreads();
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Compute kernels.                                                         */
/* ------------------------------------------------------------------------ */

/* Combiner (push): src/combiner_postamble.h:151-183.  One thread per vertex,
 * warp-aligned so that each warp owns whole bitmap words.  The mailbox swap
 * of the previous superstep (:168-183) happens here, for the vertex about to
 * run: a received message becomes the vertex's message and reactivates it. */
__global__ void __launch_bounds__(IPX_THREADS) ipx_k_compute_combiner()
{
    const uint64_t s = ipx_step();
    const uint64_t V = ipx_c.V;
    const uint64_t Vp = (V + 31) & ~31ULL;
    const int pprev = (int)((s + 1) & 1);  /* parity of superstep s-1 */
    const int lane = threadIdx.x & 31;
    for (uint64_t v = ipx_gtid(); v < Vp; v += ipx_gstride()) {
        const uint64_t wi = v >> 5;
        const uint32_t aw = ipx_c.active_bm[wi];
        const uint32_t hw = ipx_c.hasmsg_bm[wi];
        const uint32_t rw = s ? ipx_c.recv[pprev][wi] : 0u;
        if ((aw | hw | rw) == 0u) continue; /* warp-uniform */
        const uint32_t bit = 1u << lane;
        bool a = aw & bit, h = hw & bit, out = false;
        const bool r = rw & bit;
        if (v < V && (a || h || r)) {
            struct ip_vertex_t x;
            x.id = (ipx_vid)v;
            x.active = true;
            if (r) {
                x.has_message = true;
                x.message = ipx_mb::take(&ipx_c.mbox[pprev][v]);
            } else {
                x.has_message = h;
                if (h) x.message = ipx_c.msg[v];
            }
            const ipx_val v0 = ipx_c.value[v];
            x.value = v0;
            x.ipx_has_out = false;
            ipx_fill_topology(x, v);
            ip_compute(&x);
            if (!ipx_same_bits(x.value, v0)) ipx_c.value[v] = x.value;
            a = x.active;
            h = x.has_message;
            if (h) ipx_c.msg[v] = x.message;
            if (x.ipx_has_out) {
                ipx_c.outbox[v] = x.ipx_out;
                out = true;
            }
        }
        const uint32_t na = __ballot_sync(IPX_FULL, a), nh = __ballot_sync(IPX_FULL, h);
        const uint32_t no = __ballot_sync(IPX_FULL, out);
        if (lane == 0) {
            if (na != aw) ipx_c.active_bm[wi] = na;
            if (nh != hw) ipx_c.hasmsg_bm[wi] = nh;
            if (no) ipx_c.bcaster[wi] = no;
            if (rw) ipx_c.recv[pprev][wi] = 0u;
        }
    }
}

/* Spread (frontier push): src/combiner_spread_postamble.h:235-272 and the
 * mailbox update :331-342.  Superstep 0 runs every vertex, later supersteps
 * the vertices that received mail; a frontier vertex always has a message. */
__global__ void __launch_bounds__(IPX_THREADS) ipx_k_compute_spread(const uint32_t* __restrict__ frontier,
                                                                    const uint32_t* __restrict__ fcount)
{
    const uint64_t s = ipx_step();
    const uint64_t n = s ? (uint64_t)*fcount : ipx_c.V;
    const int pprev = (int)((s + 1) & 1);
    /* the next frontier entry is loaded while this vertex computes */
    const uint64_t stride = ipx_gstride();
    uint64_t i = ipx_gtid();
    uint64_t vn = (i < n) ? (s ? frontier[i] : i) : 0;
    for (; i < n; i += stride) {
        const uint64_t v = vn;
        vn = (i + stride < n) ? (s ? frontier[i + stride] : i + stride) : 0;
        struct ip_vertex_t x;
        x.id = (ipx_vid)v;
        x.active = true;
        x.has_message = s != 0;
        if (s) x.message = ipx_mb::take(&ipx_c.mbox[pprev][v]);
        const ipx_val v0 = ipx_c.value[v];
        x.value = v0;
        x.ipx_has_out = false;
        ipx_fill_topology(x, v);
        ip_compute(&x);
        if (!ipx_same_bits(x.value, v0)) ipx_c.value[v] = x.value;
        if (x.ipx_has_out) {
            ipx_c.outbox[v] = x.ipx_out;
            ipx_set_bit_agg(ipx_c.bcaster, v);
        }
    }
}

/* Single broadcast (pull) compute phase: combiner_single_broadcast_postamble.h:
 * 185-201.  Each warp rewrites whole has_broadcast words, which also clears
 * last superstep's flags. */
__global__ void __launch_bounds__(IPX_THREADS) ipx_k_compute_sb()
{
    const int ctr_slot = (int)(ipx_step() & 3);
    const uint64_t V = ipx_c.V;
    const uint64_t Vp = (V + 31) & ~31ULL;
    const int lane = threadIdx.x & 31;
    unsigned long long cnt = 0;
    for (uint64_t v = ipx_gtid(); v < Vp; v += ipx_gstride()) {
        bool a = (v < V) && ipx_c.active_b[v];
        bool out = false;
        if (a) {
            struct ip_vertex_t x;
            x.id = (ipx_vid)v;
            x.active = true;
            x.has_message = ipx_c.hasmsg_b[v];
            if (x.has_message) x.message = ipx_c.msg[v];
            const ipx_val v0 = ipx_c.value[v];
            x.value = v0;
            x.ipx_has_out = false;
            ipx_fill_topology(x, v);
            ip_compute(&x);
            if (!ipx_same_bits(x.value, v0)) ipx_c.value[v] = x.value;
            if (!x.active) ipx_c.active_b[v] = 0;
            a = x.active;
            if (x.ipx_has_out) {
                ipx_c.bval[v] = x.ipx_out;
                out = true;
            }
        }
        const uint32_t ob = __ballot_sync(IPX_FULL, out);
        const uint32_t ab = __ballot_sync(IPX_FULL, a);
        if (lane == 0) {
            ipx_c.has_b[v >> 5] = ob;
            cnt += __popc(ab);
        }
    }
    ipx_block_count(cnt, &ipx_c.ctr[ctr_slot]);
}

/* Spread + single broadcast compute phase: combiner_spread_single_broadcast_
 * postamble.h:228-237, over the targets (all vertices at superstep 0). */
__global__ void __launch_bounds__(IPX_THREADS) ipx_k_compute_ssb(const uint32_t* __restrict__ l0,
                                                                 const uint32_t* __restrict__ l1,
                                                                 const uint32_t* __restrict__ l2,
                                                                 const uint32_t* __restrict__ cnt)
{
    const uint64_t s = ipx_step();
    const uint64_t c0 = s ? cnt[0] : ipx_c.V, c1 = s ? cnt[1] : 0, c2 = s ? cnt[2] : 0;
    const uint64_t n = c0 + c1 + c2;
    for (uint64_t i = ipx_gtid(); i < n; i += ipx_gstride()) {
        const uint64_t v = !s ? i : (i < c0 ? l0[i] : (i < c0 + c1 ? l1[i - c0] : l2[i - c0 - c1]));
        struct ip_vertex_t x;
        x.id = (ipx_vid)v;
        x.active = true;
        x.has_message = ipx_c.hasmsg_b[v];
        if (x.has_message) x.message = ipx_c.msg[v];
        const ipx_val v0 = ipx_c.value[v];
        x.value = v0;
        x.ipx_has_out = false;
        ipx_fill_topology(x, v);
        ip_compute(&x);
        if (!ipx_same_bits(x.value, v0)) ipx_c.value[v] = x.value;
        if (x.ipx_has_out) {
            ipx_c.bval[v] = x.ipx_out;
            ipx_set_bit_agg(ipx_c.has_b, v);
            ipx_set_bit_agg(ipx_c.bcaster, v);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Initialisation kernels (ip_init_vertex_range of each version).           */
/* ------------------------------------------------------------------------ */
__global__ void ipx_k_init_values(uint64_t first, uint64_t last)
{
    for (uint64_t v = first + ipx_gtid(); v <= last && v < ipx_c.V; v += ipx_gstride()) {
        ipx_c.value[v] = ipx_val();
#if IPX_VERSION == IPX_SINGLE_BROADCAST
        ipx_c.active_b[v] = 1;
#endif
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SPREAD
        ipx_c.mbox[0][v] = ipx_mb::empty();
        ipx_c.mbox[1][v] = ipx_mb::empty();
#endif
    }
}

__global__ void ipx_k_fill_bits(uint32_t* bm, uint64_t V, uint64_t W)
{
    for (uint64_t w = ipx_gtid(); w < W; w += ipx_gstride()) {
        uint32_t x = IPX_FULL;
        if (w == W - 1 && (V & 31)) x = (1u << (V & 31)) - 1u;
        bm[w] = x;
    }
}

/* ------------------------------------------------------------------------ */
/* Superstep control on the device.                                         */
/* ------------------------------------------------------------------------ */

/* Zeroes the counters a superstep accumulates into. */
__global__ void ipx_k_begin_superstep()
{
    const uint64_t s = ipx_step();
    ipx_c.ctr[s & 3] = 0ULL;
    for (int k = 8; k < 14; k++) ipx_c.ctr[k] = 0ULL;
}

/* Combiner: active count of the superstep = |active or received|
 * (combiner_postamble.h:151-183), parity read on the device. */
__global__ void __launch_bounds__(IPX_THREADS) ipx_k_count_combiner()
{
    const uint64_t s = ipx_step();
    const uint32_t* __restrict__ a = ipx_c.active_bm;
    const uint32_t* __restrict__ r = ipx_c.recv[s & 1];
    unsigned long long c = 0;
    for (uint64_t i = ipx_gtid(); i < ipx_c.W; i += ipx_gstride()) c += __popc(a[i] | r[i]);
    ipx_block_count(c, &ipx_c.ctr[s & 3]);
}

/* Active count the reference prints for the superstep just run and tests in
 * its loop condition (each version's ip_run). */
__device__ __forceinline__ unsigned long long ipx_superstep_count(uint64_t s)
{
#if IPX_VERSION == IPX_COMBINER || IPX_VERSION == IPX_SINGLE_BROADCAST
    return ipx_c.ctr[s & 3];
#elif IPX_VERSION == IPX_SPREAD
    (void)s;
    return ipx_c.lcnt[4];
#else
    (void)s;
    return (unsigned long long)ipx_c.lcnt[4] + ipx_c.lcnt[5] + ipx_c.lcnt[6];
#endif
}

/* Last kernel of a captured superstep: records the superstep in the history,
 * advances the superstep and sets the loop's condition: continue while the
 * count is nonzero (combiner_postamble.h:134; spread versions test it after
 * superstep 0, combiner_spread_postamble.h:212), no kernel reported an error
 * and the superstep bound is not reached. */
__global__ void ipx_k_advance(cudaGraphConditionalHandle loop, unsigned long long max_supersteps)
{
    const uint64_t s = ipx_step();
    const unsigned long long count = ipx_superstep_count(s);
    unsigned long long edges = 0;
#if IPX_VERSION == IPX_SINGLE_BROADCAST
    edges = ipx_c.E;
#else
    const bool pulled = ipx_c.pull_ok && ipx_c.ctr[IPX_CTR_MODE];
    edges = pulled ? ipx_c.E : ipx_c.ctr[8] + ipx_c.ctr[9] + ipx_c.ctr[10];
    edges += ipx_c.ctr[11] + ipx_c.ctr[12] + ipx_c.ctr[13];
#endif
    unsigned long long* h = ipx_c.hist + (s % IPX_HIST) * 4;
    h[0] = count;
    h[1] = edges;
    h[2] = ipx_c.pull_ok ? ipx_c.ctr[IPX_CTR_MODE] : 0ULL;
    bool go = count != 0 && *ipx_c.err == 0;
    if (go && s + 1 >= max_supersteps) {
        atomicOr(ipx_c.err, IPX_ERR_SUPERSTEP_LIMIT);
        go = false;
    }
    ipd_superstep = s + 1;
    cudaGraphSetConditional(loop, go ? 1u : 0u);
}

/* Checks an IP_COMBINE_KIND hint against the user's ip_combine on sample
 * pairs before the hint is trusted. */
__global__ void ipx_k_check_hint(int kind)
{
    for (uint64_t i = ipx_gtid(); i < 4096; i += ipx_gstride()) {
        unsigned long long ra = (i * 0x9E3779B97F4A7C15ULL) ^ (i >> 3), rb = (i * 0xC2B2AE3D27D4EB4FULL) + 7;
        ipx_msg a, b;
        if constexpr (std::is_floating_point<ipx_msg>::value) {
            a = (ipx_msg)((double)(ra >> 11) * (1.0 / 9007199254740992.0));
            b = (ipx_msg)((double)(rb >> 11) * (1.0 / 9007199254740992.0));
        } else if constexpr (std::is_integral<ipx_msg>::value) {
            a = (ipx_msg)((i & 1) ? (ra & 0xFFFF) : ra);
            b = (ipx_msg)((i & 2) ? (rb & 0xFFFF) : rb);
        } else {
            return;
        }
        ipx_msg c = a;
        ip_combine(&c, b);
        ipx_msg e;
        if (kind == IP_COMBINE_MIN) e = (b < a) ? b : a;
        else if (kind == IP_COMBINE_MAX) e = (b > a) ? b : a;
        else e = a + b;
        if (!(c == e)) atomicOr(ipx_c.err, IPX_ERR_COMBINE_HINT);
    }
}

#endif /* IPREGEL_B200_ENGINE_CUH */
