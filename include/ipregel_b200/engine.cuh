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
 *   bslot[V]                       pull: the externalised broadcast slot of
 *                                  combiner_single_broadcast_preamble.h:42-50,
 *                                  {message, superstep stamp} in 8 or 16 bytes
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
#define IPX_ERR_COPY_TIMEOUT 8u
#define IPX_ERR_RESERVED_MESSAGE 16u
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
/* Pull broadcast slot.  The reference keeps {has_broadcast, message} per    */
/* vertex (combiner_single_broadcast_preamble.h:42-50) and clears the flags  */
/* every superstep.  Here a slot holds the message's bits and the superstep  */
/* in which it was broadcast: it counts in superstep s iff its stamp is s,   */
/* so no slot is ever cleared, and a gathered edge costs one 8-byte (message */
/* up to 4 bytes) or 16-byte (up to 8 bytes) load -- one L2 request -- where */
/* a flag bitmap costs a dependent bitmap-word load before the value.        */
/* ------------------------------------------------------------------------ */
typedef typename std::conditional<(sizeof(ipx_msg) <= 4), uint2, uint4>::type ipx_bslot;
/* Stamp of a slot that holds no broadcast (all bytes 0xff after a reset);
 * supersteps stay below it (ipx_max_supersteps). */
#define IPX_NO_STAMP 0xffffffffu

__device__ __forceinline__ void ipx_bslot_store(uint2* p, unsigned long long w, uint32_t stamp)
{
    *p = make_uint2((uint32_t)w, stamp);
}
__device__ __forceinline__ void ipx_bslot_store(uint4* p, unsigned long long w, uint32_t stamp)
{
    *p = make_uint4((uint32_t)w, (uint32_t)(w >> 32), stamp, 0u);
}
__device__ __forceinline__ unsigned long long ipx_bslot_bits(const uint2& w) { return w.x; }
__device__ __forceinline__ unsigned long long ipx_bslot_bits(const uint4& w)
{
    return ((unsigned long long)w.y << 32) | w.x;
}
__device__ __forceinline__ uint32_t ipx_bslot_stamp(const uint2& w) { return w.y; }
__device__ __forceinline__ uint32_t ipx_bslot_stamp(const uint4& w) { return w.z; }

/* A slot that holds no broadcast. */
__device__ __forceinline__ ipx_bslot make_ipx_nobslot()
{
    ipx_bslot w;
    memset(&w, 0xff, sizeof w);
    return w;
}

__device__ __forceinline__ void ipx_bslot_put(ipx_bslot* p, const ipx_msg& m, uint32_t stamp)
{
    ipx_bslot_store(p, (unsigned long long)ipx_to_word(m), stamp);
}

/* The message of a loaded slot; true when it was broadcast in superstep
 * `stamp`. */
__device__ __forceinline__ bool ipx_bslot_take(const ipx_bslot& w, uint32_t stamp, ipx_msg& m)
{
    m = ipx_from_word<ipx_msg>((typename ipx_word<ipx_msg>::type)ipx_bslot_bits(w));
    return ipx_bslot_stamp(w) == stamp;
}

/* The single_broadcast version with FP64 messages (PageRank) keeps 8-byte
 * slots without a stamp: its fused kernel visits every vertex each
 * superstep and writes every slot of the next buffer -- the broadcast, or
 * IPX_ABSENT64 when the vertex does not broadcast -- so a slot never holds
 * a message of an older superstep.  IPX_ABSENT64 (all bits set) is a NaN
 * that FP64 arithmetic does not produce; a broadcast of exactly that bit
 * pattern is reported as an error (IPX_ERR_RESERVED_MESSAGE).  Half the
 * bytes of a stamped 16-byte slot: twice as many vertices' slots fit in the
 * L2.  Other message types keep stamped slots. */
#ifndef IPX_SB_DENSE
#define IPX_SB_DENSE 1
#endif
#define IPX_ABSENT64 0xffffffffffffffffULL
typedef typename std::conditional<(IPX_SB_DENSE && std::is_same<ipx_msg, double>::value), unsigned long long,
                                  ipx_bslot>::type ipx_sbslot;

__device__ __forceinline__ bool ipx_slot_take(const ipx_bslot& w, uint32_t stamp, ipx_msg& m)
{
    return ipx_bslot_take(w, stamp, m);
}
__device__ __forceinline__ bool ipx_slot_take(const unsigned long long& w, uint32_t, ipx_msg& m)
{
    m = ipx_from_word<ipx_msg>((typename ipx_word<ipx_msg>::type)w);
    return w != IPX_ABSENT64;
}
template <class S>
__device__ __forceinline__ S ipx_no_slot()
{
    S w;
    memset(&w, 0xff, sizeof w);
    return w;
}

/* ---- L2 eviction policies for the gathered slots ----
 * The slots of a few million often-gathered vertices would fit the L2, but
 * the gather's cold accesses (most vertices are gathered a few times per
 * superstep) evict them.  The single_broadcast version can gather from a
 * copy of the in-lists whose ids carry a flag in bit 31 for the vertices
 * gathered most often (ipx_consts::in_adj_hot, built at attach): their
 * slots are loaded evict-last, all others evict-first. */
#define IPX_HOT_BIT 0x80000000u
__device__ __forceinline__ uint64_t ipx_policy(bool hot)
{
    uint64_t p;
    if (hot) asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long ipx_ld_policy(const unsigned long long* p, uint64_t pol)
{
    unsigned long long r;
    asm volatile("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(r) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ uint2 ipx_ld_policy(const uint2* p, uint64_t pol)
{
    uint2 r;
    asm volatile("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(r.x), "=r"(r.y) : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ uint4 ipx_ld_policy(const uint4* p, uint64_t pol)
{
    uint4 r;
    asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p), "l"(pol));
    return r;
}
/* The slot of the in-neighbour whose id word is w: HOT ids carry the flag. */
template <bool HOT, class S>
__device__ __forceinline__ S ipx_slot_ld(const S* __restrict__ bs, uint64_t w)
{
    if constexpr (HOT) {
        return ipx_ld_policy(&bs[w & (IPX_HOT_BIT - 1u)], ipx_policy((w & IPX_HOT_BIT) != 0));
    } else {
        return __ldg(&bs[w]);
    }
}

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
    /* pull broadcast slots: single_broadcast alternates bslot[s & 1] (its
     * fused kernel reads superstep s's slots while writing s+1's);
     * spread+single_broadcast uses bslot[0] */
    ipx_bslot* bslot[2];
    ipx_sbslot* sbslot[2];
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
    /* single_broadcast hub chunks: per chunk the partial fold ({message,
     * has} in a slot, has in the stamp word), per hub the chunks arrived */
    ipx_bslot* hub_part;
    uint32_t* hub_arrived;
    /* chunk -> index of its hub in the static hub class (built at attach) */
    const uint32_t* hub_owner;
    /* the in-lists with the flag of the most gathered vertices (null: none) */
    const uint32_t* in_adj_hot;
    /* push / mark: chunk -> index of its hub in this superstep's hub list
     * (null: found by a binary search over the prefix) */
    const uint32_t* push_owner;
    /* The kernels run on a degree-ordered copy of the graph: vid_of[v] is
     * the id of vertex v in the caller's numbering, vindex_of its inverse
     * (both null when the graph is not renamed). */
    const uint32_t* vid_of;
    const uint32_t* vindex_of;
    /* the caller's graph, whose row vid_of[v] holds the same edges in the
     * same order as row v of the copy: the neighbour ids ip_compute reads
     * (null when not renamed) */
    const uint64_t* user_row;
    const ipx_vid* user_adj;
    const uint64_t* user_in_row;
    const ipx_vid* user_in_adj;
};

__constant__ ipx_consts ipx_c;

/* The id ip_compute sees for vertex v (the caller's numbering). */
__device__ __forceinline__ ipx_vid ipx_user_id(uint64_t v)
{
    return (ipx_vid)(ipx_c.vid_of ? (uint64_t)__ldg(&ipx_c.vid_of[v]) : v);
}

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
/* 1: the hub class of the fused pull kernel takes a warp per chunk instead
 * of a CTA (no CTA-wide barriers per chunk); 0: a CTA per chunk, its ids
 * staged in shared memory (IPX_HUB_SMEM).  On directed R-MAT scale 25
 * (FP64 PageRank, 30 rounds) a warp per 4,096-edge chunk took 109 ms (8,192:
 * 105.9 ms), a CTA per 2,048-edge chunk, staged or not, 118.7 ms: the CTA
 * version waits at two barriers per chunk. */
#ifndef IPX_HUB_WARP
#define IPX_HUB_WARP 1
#endif
/* In-edges per chunk of the single_broadcast gather's hub class (a warp's
 * with IPX_HUB_WARP; 2,048 for a CTA's: the staging buffers of larger
 * chunks do not fit the 48 KB of static shared memory). */
#ifndef IPX_GATHER_CHUNK
#if IPX_HUB_WARP
#define IPX_GATHER_CHUNK 8192
#else
#define IPX_GATHER_CHUNK 2048
#endif
#endif
#ifndef IPX_UNROLL
#define IPX_UNROLL 4
#endif
/* 1: sources of the thread and warp classes go through the warp-cooperative
 * expansion; 0: a thread per source (degree <= IPX_T0), a warp per source. */
#ifndef IPX_PUSH_EXPAND
#define IPX_PUSH_EXPAND 0
#endif
/* Lanes per source in the warp class of push and mark (8, 16 or 32).  On
 * the degree-ordered copy of undirected R-MAT scale 24 (most sources of the
 * class have a few dozen out-edges), CC + SSSP ran at 63.7 - 63.9 GTEPS with
 * 16, 62.0 with 8 and 61.5 - 61.6 with 32. */
#ifndef IPX_PUSH_GROUP
#define IPX_PUSH_GROUP 16
#endif
/* Lanes per source in the thread class of push and mark (1, 2, 4 or 8). */
#ifndef IPX_PUSH_Q
#define IPX_PUSH_Q 1
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
    /* Four consecutive edges e0 .. e0+3 (e0 a multiple of 4) whose ids one
     * 128-bit load gave; 4-byte weights come the same way. */
    __device__ __forceinline__ void batch_v4(uint64_t e0, const uint4& id, const ipx_msg& m) const
    {
        const uint32_t w[4] = {id.x, id.y, id.z, id.w};
        ipx_msg mk[4];
#if IPX_EDGE_MSG
        if constexpr (sizeof(ipx_wgt) == 4) {
            const uint4 ww = __ldcs(reinterpret_cast<const uint4*>(ipx_c.wgt + e0));
            const uint32_t wk[4] = {ww.x, ww.y, ww.z, ww.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                ipx_wgt x;
                memcpy(&x, &wk[k], 4);
                mk[k] = IP_BROADCAST_EDGE_MESSAGE(m, x);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) mk[k] = IP_BROADCAST_EDGE_MESSAGE(m, ipx_ld_stream(&ipx_c.wgt[e0 + k]));
        }
#else
        (void)e0;
#pragma unroll
        for (int k = 0; k < 4; k++) mk[k] = m;
#endif
        bool go[4];
#pragma unroll
        for (int k = 0; k < 4; k++) go[k] = ipx_mb::precheck(&ipx_c.mbox[p][w[k]], mk[k]);
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (go[k] && ipx_mb::commit(&ipx_c.mbox[p][w[k]], mk[k])) atomicOr(&ipx_c.recv[p][w[k] >> 5], 1u << (w[k] & 31));
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
    __device__ __forceinline__ void batch_v4(uint64_t e0, const uint4& id, const ipx_msg& m) const
    {
        const uint64_t e[4] = {e0, e0 + 1, e0 + 2, e0 + 3};
        const ipx_vid w[4] = {(ipx_vid)id.x, (ipx_vid)id.y, (ipx_vid)id.z, (ipx_vid)id.w};
        const ipx_msg mk[4] = {m, m, m, m};
        const bool ok[4] = {true, true, true, true};
        batch<4>(e, w, mk, ok);
    }
};

/* Edges [e0, e1) of one source visited by a warp or block (lanes >= 32)
 * with 32-bit ids: the ids of four consecutive edges per lane come from one
 * 128-bit load (the weights too, when the visitor needs 4-byte weights),
 * the up to 3 edges before the first 16-byte boundary and after the last one
 * take a lane each. */
template <class Visit>
__device__ __forceinline__ void ipx_edges_v4(const uint32_t* __restrict__ adj, uint64_t e0, uint64_t e1,
                                             uint64_t lane, uint64_t lanes, ipx_msg m, const Visit& visit)
{
    uint64_t a = (e0 + 3) & ~3ULL;
    if (a > e1) a = e1;
    const uint64_t b = a + ((e1 - a) & ~3ULL);
    {
        const uint64_t nh = a - e0, nt = e1 - b;
        uint64_t e = e1;
        if (lane < nh) e = e0 + lane;
        else if (lane < nh + nt) e = b + (lane - nh);
        const uint64_t ek[1] = {e};
        const bool ok[1] = {e < e1};
        const ipx_vid w[1] = {ok[0] ? (ipx_vid)ipx_ld_stream(&adj[e]) : (ipx_vid)0};
        const ipx_msg mk[1] = {m};
        visit.template batch<1>(ek, w, mk, ok);
    }
    const uint4* __restrict__ q = reinterpret_cast<const uint4*>(adj + a);
    const uint64_t groups = (b - a) >> 2;
    for (uint64_t g = lane; g < groups; g += lanes) visit.batch_v4(a + 4 * g, __ldcs(q + g), m);
}

/* The 128-bit path needs 16-byte aligned id and weight arrays (always so for
 * arrays the runtime allocates; a caller's array may not be). */
__device__ __forceinline__ bool ipx_v4_ok(const void* adj)
{
    if constexpr (sizeof(ipx_vid) != 4) return false;
    if ((reinterpret_cast<uintptr_t>(adj) & 15) != 0) return false;
#if IPX_EDGE_MSG
    if ((reinterpret_cast<uintptr_t>(ipx_c.wgt) & 15) != 0) return false;
#endif
    return true;
}

/* Visits edges [e0, e1) of one source lane-strided, IPX_UNROLL edges a lane
 * at a time, loading the ids of a batch before visiting any of it (warps and
 * blocks over 32-bit ids: ipx_edges_v4). */
template <class Visit>
__device__ __forceinline__ void ipx_edges_strided(const ipx_vid* __restrict__ adj, uint64_t e0, uint64_t e1,
                                                  uint64_t lane, uint64_t lanes, ipx_msg m, const Visit& visit)
{
    if constexpr (sizeof(ipx_vid) == 4) {
        if (lanes >= 8 && ipx_v4_ok(adj)) {
            ipx_edges_v4(reinterpret_cast<const uint32_t*>(adj), e0, e1, lane, lanes, m, visit);
            return;
        }
    }
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
 * i, prefix[n] = total (one block, a carried scan over tiles of its width).
 * With owner, also owner[c] = i for every chunk c of hub i, so that a chunk
 * finds its hub with one load instead of a binary search over the prefix. */
template <uint32_t CHUNK = IPX_HUB_CHUNK>
__global__ void __launch_bounds__(1024) ipx_k_hub_prefix(const uint32_t* __restrict__ list,
                                                         const uint32_t* __restrict__ count,
                                                         const uint64_t* __restrict__ row, uint32_t* __restrict__ prefix,
                                                         uint32_t* __restrict__ owner = nullptr)
{
    __shared__ uint32_t s[1024];
    const uint64_t n = *count;
    uint32_t carry = 0;
    for (uint64_t base = 0; base < n; base += 1024) {
        const uint64_t i = base + threadIdx.x;
        uint32_t c = 0;
        if (i < n) {
            const uint64_t u = list[i];
            c = (uint32_t)((row[u + 1] - row[u] + CHUNK - 1) / CHUNK);
        }
        s[threadIdx.x] = c;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const uint32_t x = (threadIdx.x >= (unsigned)o) ? s[threadIdx.x - o] : 0u;
            __syncthreads();
            s[threadIdx.x] += x;
            __syncthreads();
        }
        if (i < n) {
            const uint32_t p = carry + s[threadIdx.x] - c;
            prefix[i] = p;
            if (owner)
                for (uint32_t k = 0; k < c; k++) owner[p + k] = (uint32_t)i;
        }
        carry += s[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) prefix[n] = carry;
}

/* ---- the flagged in-lists of the single_broadcast gather (attach time) ---- */
/* cnt[u] += 1 for every occurrence of u in the in-lists. */
__global__ void ipx_k_count_occurrences(const uint32_t* __restrict__ adj, uint64_t E, uint32_t* __restrict__ cnt)
{
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[adj[e]], 1u);
}

/* hist[b] = vertices whose occurrence count has b significant bits. */
__global__ void ipx_k_count_hist(const uint32_t* __restrict__ cnt, uint64_t V, unsigned long long* __restrict__ hist)
{
    __shared__ unsigned int h[33];
    if (threadIdx.x < 33) h[threadIdx.x] = 0;
    __syncthreads();
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < V; v += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[32 - __clz(cnt[v])], 1u);
    __syncthreads();
    if (threadIdx.x < 33 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], (unsigned long long)h[threadIdx.x]);
}

/* out[e] = adj[e], with IPX_HOT_BIT set when that vertex occurs at least
 * `threshold` times in the in-lists. */
__global__ void ipx_k_flag_hot(const uint32_t* __restrict__ adj, uint64_t E, const uint32_t* __restrict__ cnt,
                               uint32_t threshold, uint32_t* __restrict__ out)
{
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t u = adj[e];
        out[e] = u | (cnt[u] >= threshold ? IPX_HOT_BIT : 0u);
    }
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
    uint64_t w = (uint64_t)id;
    if (ipx_c.vindex_of && w < ipx_c.V) w = ipx_c.vindex_of[w]; /* the caller's id -> the copy's vertex */
    ipx_deliver((int)(ip_get_superstep() & 1), w, message);
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
    x.out_neighbours = const_cast<ipx_vid*>(ipx_c.user_adj ? ipx_c.user_adj + ipx_c.user_row[ipx_c.vid_of[v]]
                                                           : ipx_c.adj + r0);
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
    x.in_neighbours = const_cast<ipx_vid*>(ipx_c.user_in_adj ? ipx_c.user_in_adj + ipx_c.user_in_row[ipx_c.vid_of[v]]
                                                             : ipx_c.in_adj + q0);
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
    } else if constexpr (MODE == 0 && IPX_PUSH_Q > 1) {
        /* IPX_PUSH_Q consecutive lanes per source: a source's (at most
         * IPX_T0) ids are read by the group's lanes together, sectors shared */
        const ipx_vid* __restrict__ adj = ipx_c.adj;
        const uint64_t* __restrict__ row = ipx_c.row;
        const uint64_t q = threadIdx.x & (IPX_PUSH_Q - 1);
        for (uint64_t i = ipx_gtid() / IPX_PUSH_Q; i < n; i += ipx_gstride() / IPX_PUSH_Q) {
            const uint64_t u = list[i];
            ipx_msg m = ipx_msg();
            if constexpr (Visit::kNeedsMessage) m = ipx_c.outbox[u];
            ipx_edges_strided(adj, row[u], row[u + 1], q, IPX_PUSH_Q, m, visit);
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
        /* IPX_PUSH_GROUP lanes per source (a warp's worth, or fewer: most
         * sources of the class have a few dozen out-edges) */
        constexpr int G = IPX_PUSH_GROUP;
        const ipx_vid* __restrict__ adj = ipx_c.adj;
        const uint64_t* __restrict__ row = ipx_c.row;
        const uint64_t lane = threadIdx.x & (G - 1);
        for (uint64_t i = ipx_gtid() / G; i < n; i += ipx_gstride() / G) {
            const uint64_t u = list[i];
            ipx_msg m = ipx_msg();
            if constexpr (Visit::kNeedsMessage) m = ipx_c.outbox[u];
            ipx_edges_strided(adj, row[u], row[u + 1], lane, G, m, visit);
        }
    } else {
        if (n == 0) return;
        const ipx_vid* __restrict__ adj = ipx_c.adj;
        const uint64_t* __restrict__ row = ipx_c.row;
        const uint32_t chunks = prefix[n];
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint64_t i = ipx_c.push_owner ? ipx_c.push_owner[c] : ipx_hub_of_chunk(prefix, n, c);
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

/* The same over the G lanes of one group (G a power of two <= 32); `mask`
 * holds the group's lanes. */
template <int G>
__device__ __forceinline__ void ipx_group_fold(bool& has, ipx_msg& acc, unsigned mask)
{
    typedef typename ipx_word<ipx_msg>::type W;
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
        const bool oh = __shfl_down_sync(mask, has, o, G);
        const ipx_msg om = ipx_from_word<ipx_msg>(__shfl_down_sync(mask, ipx_to_word(acc), o, G));
        ipx_fold(has, acc, oh, om);
    }
}

/* Folds the broadcasts of the in-neighbours at edges e0 + lane, e0 + lane +
 * lanes, ... below e1, in that order.  IPX_UNROLL edges a step: their ids,
 * then their broadcast slots are each loaded for all IPX_UNROLL edges before
 * any is folded, so a lane has IPX_UNROLL independent slot loads in flight.
 * A warp or block (lanes >= 32) with 32-bit ids reads the ids 128 bits at a
 * time instead: four consecutive in-edges per lane and load instruction
 * (ipx_gather_fold_edges_v4). */
template <bool HOT = false, class S>
__device__ __forceinline__ void ipx_gather_fold_edges_v4(const uint32_t* __restrict__ adj,
                                                         const S* __restrict__ bs, uint32_t stamp,
                                                         uint64_t e0, uint64_t e1, uint64_t lane, uint64_t lanes,
                                                         bool& has, ipx_msg& acc)
{
    /* [e0, a): up to 3 edges before the first 16-byte boundary; [a, b): whole
     * groups of four; [b, e1): up to 3 edges after.  The 6 or fewer edges of
     * both ends take one lane each (lanes >= 8). */
    uint64_t a = (e0 + 3) & ~3ULL;
    if (a > e1) a = e1;
    const uint64_t b = a + ((e1 - a) & ~3ULL);
    {
        const uint64_t nh = a - e0, nt = e1 - b;
        uint64_t e = e1;
        if (lane < nh) e = e0 + lane;
        else if (lane < nh + nt) e = b + (lane - nh);
        if (e < e1) {
            const S w = ipx_slot_ld<HOT>(bs, adj[e]);
            ipx_msg m;
            if (ipx_slot_take(w, stamp, m)) ipx_fold(has, acc, true, m);
        }
    }
    const uint4* __restrict__ q = reinterpret_cast<const uint4*>(adj + a);
    const uint64_t groups = (b - a) >> 2;
    for (uint64_t g = lane; g < groups; g += lanes) {
        const uint4 id = __ldcs(q + g);
        S w[4];
        w[0] = ipx_slot_ld<HOT>(bs, id.x);
        w[1] = ipx_slot_ld<HOT>(bs, id.y);
        w[2] = ipx_slot_ld<HOT>(bs, id.z);
        w[3] = ipx_slot_ld<HOT>(bs, id.w);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            ipx_msg m;
            if (ipx_slot_take(w[k], stamp, m)) ipx_fold(has, acc, true, m);
        }
    }
}

template <bool HOT = false, class S>
__device__ __forceinline__ void ipx_gather_fold_edges(const ipx_vid* __restrict__ adj,
                                                      const S* __restrict__ bs, uint32_t stamp, uint64_t e0,
                                                      uint64_t e1, uint64_t lane, uint64_t lanes, bool& has,
                                                      ipx_msg& acc)
{
    if constexpr (sizeof(ipx_vid) == 4) {
        /* the vector path needs a 16-byte aligned id array (always so for
         * arrays the runtime allocates; a caller's array may not be) */
        if (lanes >= 8 && (reinterpret_cast<uintptr_t>(adj) & 15) == 0) {
            ipx_gather_fold_edges_v4<HOT>(reinterpret_cast<const uint32_t*>(adj), bs, stamp, e0, e1, lane, lanes, has,
                                          acc);
            return;
        }
    }
    for (uint64_t e = e0 + lane; e < e1; e += IPX_UNROLL * lanes) {
        uint64_t u[IPX_UNROLL];
        S w[IPX_UNROLL];
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++)
            u[k] = (e + k * lanes < e1) ? (uint64_t)ipx_ld_edge(&adj[e + k * lanes], lanes) : 0;
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++)
            w[k] = (e + k * lanes < e1) ? ipx_slot_ld<HOT>(bs, u[k]) : ipx_no_slot<S>();
#pragma unroll
        for (int k = 0; k < IPX_UNROLL; k++) {
            ipx_msg m;
            if (ipx_slot_take(w[k], stamp, m)) ipx_fold(has, acc, true, m);
        }
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
    const ipx_bslot* __restrict__ bs = ipx_c.bslot[0];
    const uint32_t stamp = (uint32_t)ipx_step();
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
            ipx_gather_fold_edges(adj, bs, stamp, row[v], row[v + 1], 0, 1, has, acc);
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
            ipx_gather_fold_edges(adj, bs, stamp, row[v], row[v + 1], lane, 32, has, acc);
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
            ipx_gather_fold_edges(adj, bs, stamp, row[v], row[v + 1], threadIdx.x, blockDim.x, has, acc);
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
            const uint64_t i = ipx_c.hub_owner ? ipx_c.hub_owner[c] : ipx_hub_of_chunk(prefix, n, c);
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
            x.id = ipx_user_id(v);
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
        x.id = ipx_user_id(v);
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

/* The single_broadcast version's record of a vertex's broadcast (or of
 * none) for the superstep `stamp`: a stamped slot is written only for a
 * broadcast; a dense slot every time. */
__device__ __forceinline__ void ipx_sb_put(ipx_bslot* p, bool out, const ipx_msg& m, uint32_t stamp)
{
    if (out) ipx_bslot_put(p, m, stamp);
}
__device__ __forceinline__ void ipx_sb_put(unsigned long long* p, bool out, const ipx_msg& m, uint32_t)
{
    unsigned long long w = IPX_ABSENT64;
    if (out) {
        w = (unsigned long long)ipx_to_word(m);
        if (w == IPX_ABSENT64) atomicOr(ipx_c.err, IPX_ERR_RESERVED_MESSAGE);
    }
    *p = w;
}

/* Single broadcast (pull), superstep 0's compute phase
 * (combiner_single_broadcast_postamble.h:185-201): every vertex is active and
 * has no message.  A broadcast writes the vertex's slot in buffer 0 stamped
 * 0.  Later supersteps' compute phases run inside ipx_k_gather_compute; this
 * kernel returns at once after superstep 0, so the same launch sequence
 * serves every superstep of a captured loop.  The count of superstep 0 is
 * made by the gather that follows. */
__global__ void __launch_bounds__(IPX_THREADS) ipx_k_compute_sb0()
{
    if (ipx_step() != 0) return;
    const uint64_t V = ipx_c.V;
    ipx_sbslot* __restrict__ out = ipx_c.sbslot[0];
    for (uint64_t v = ipx_gtid(); v < V; v += ipx_gstride()) {
        if (!ipx_c.active_b[v]) {
            ipx_sb_put(&out[v], false, ipx_msg(), 0u);
            continue;
        }
        struct ip_vertex_t x;
        x.id = ipx_user_id(v);
        x.active = true;
        x.has_message = false;
        const ipx_val v0 = ipx_c.value[v];
        x.value = v0;
        x.ipx_has_out = false;
        ipx_fill_topology(x, v);
        ip_compute(&x);
        if (!ipx_same_bits(x.value, v0)) ipx_c.value[v] = x.value;
        if (!x.active) ipx_c.active_b[v] = 0;
        ipx_sb_put(&out[v], x.ipx_has_out, x.ipx_out, 0u);
    }
}

/* After vertex v's gather of superstep s: whether v is active (it was after
 * compute(s), or a message reactivates it, :65-71), and if so its compute
 * phase of superstep s+1 (:185-201) with the gathered message; a broadcast
 * goes to `out` stamped s+1.  Returns the activity that superstep s counts. */
__device__ __forceinline__ bool ipx_sb_compute_next(uint64_t v, bool has, const ipx_msg& acc, ipx_sbslot* out,
                                                    uint32_t next_stamp)
{
    const bool a0 = ipx_c.active_b[v] != 0;
    if (!a0 && !has) {
        ipx_sb_put(&out[v], false, acc, next_stamp);
        return false;
    }
    struct ip_vertex_t x;
    x.id = ipx_user_id(v);
    x.active = true;
    x.has_message = has;
    if (has) x.message = acc;
    const ipx_val v0 = ipx_c.value[v];
    x.value = v0;
    x.ipx_has_out = false;
    ipx_fill_topology(x, v);
    ip_compute(&x);
    if (!ipx_same_bits(x.value, v0)) ipx_c.value[v] = x.value;
    if (x.active != a0) ipx_c.active_b[v] = x.active ? 1 : 0;
    ipx_sb_put(&out[v], x.ipx_has_out, x.ipx_out, next_stamp);
    return true;
}

/* ---- bulk copies into shared memory (cp.async.bulk, completed on an
 * mbarrier; one CTA, no cluster, no multicast) ---- */
__device__ __forceinline__ uint32_t ipx_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ipx_mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ipx_smem(bar)) : "memory");
}

/* The issuing thread's arrival on `bar`, expecting `bytes` from a bulk copy
 * (0: a plain arrival, which completes the phase). */
__device__ __forceinline__ void ipx_mbar_arrive_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ipx_smem(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void ipx_bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     ipx_smem(dst)),
                 "l"(src), "r"(bytes), "r"(ipx_smem(bar))
                 : "memory");
}

/* Waits for phase `parity` of `bar` to complete, at most `limit` polls. */
__device__ __forceinline__ bool ipx_mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t k = 0; k < limit; k++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(ipx_smem(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

/* Polls before a wait for a chunk's ids is given up (each try_wait may
 * suspend the thread for a while): an 8 KB copy lands in microseconds, so
 * this is reached only if the copy never completes. */
#define IPX_COPY_WAIT_LIMIT (1u << 22)

/* A hub chunk as thread 0 located it: the vertex, its hub index, the chunk's
 * edge range [e0, e1) and the 16-byte aligned range [a0, b) copied into
 * shared memory (b <= a0: nothing copied). */
struct ipx_hub_chunk {
    uint64_t v, e0, e1, a0, b;
    uint64_t i;
    uint32_t c, c0, nch, pad;
};

__device__ __forceinline__ void ipx_locate_chunk(const uint32_t* __restrict__ list, uint64_t n,
                                                 const uint32_t* __restrict__ prefix, const uint64_t* __restrict__ row,
                                                 uint32_t c, ipx_hub_chunk& h)
{
    h.c = c;
    h.i = ipx_c.hub_owner ? ipx_c.hub_owner[c] : ipx_hub_of_chunk(prefix, n, c);
    h.v = list[h.i];
    h.c0 = prefix[h.i];
    h.nch = prefix[h.i + 1] - h.c0;
    h.e0 = row[h.v] + (uint64_t)(c - h.c0) * IPX_GATHER_CHUNK;
    const uint64_t end = row[h.v + 1];
    h.e1 = (h.e0 + IPX_GATHER_CHUNK < end) ? h.e0 + IPX_GATHER_CHUNK : end;
    h.a0 = h.e0 & ~3ULL;
    h.b = h.e1 & ~3ULL;
}

/* The CTA's fold of one hub chunk is done (thread 0 holds it in has/acc;
 * every thread of the CTA calls this).  The fold is stored; the CTA whose
 * chunk arrives last folds the hub's partials in chunk order -- each thread
 * a contiguous run of them, then the runs in order through the warps and
 * the CTA -- and thread 0 runs the vertex's compute phase of the next
 * superstep.  s_has / s_acc: the caller's per-warp shared scratch, free
 * again when this is called.  Returns the count (thread 0). */
__device__ __forceinline__ unsigned long long ipx_hub_chunk_done(const ipx_hub_chunk& h, bool has, ipx_msg acc,
                                                                 ipx_sbslot* out, uint32_t next_stamp,
                                                                 bool* s_has, ipx_msg* s_acc)
{
    __shared__ int s_last;
    if (threadIdx.x == 0) {
        int last = 2; /* a hub of one chunk: its fold is the hub's */
        if (h.nch != 1) {
            ipx_bslot_put(&ipx_c.hub_part[h.c], acc, has ? 1u : 0u);
            __threadfence();
            last = atomicAdd(&ipx_c.hub_arrived[h.i], 1u) == h.nch - 1 ? 1 : 0;
        }
        s_last = last;
    }
    __syncthreads();
    const int last = s_last;
    if (last == 1) {
        __threadfence();
        const uint32_t nthr = blockDim.x, per = (h.nch + nthr - 1) / nthr;
        const uint32_t k0 = threadIdx.x * per, k1 = min(k0 + per, h.nch);
        bool hp = false;
        ipx_msg ap;
        for (uint32_t k = k0; k < k1; k++) {
            const ipx_bslot p = __ldcg(&ipx_c.hub_part[h.c0 + k]);
            ipx_msg m;
            if (ipx_bslot_take(p, 1u, m)) ipx_fold(hp, ap, true, m);
        }
        ipx_warp_fold(hp, ap);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) {
            s_has[warp] = hp;
            s_acc[warp] = ap;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            has = false;
            for (int w = 0; w < (int)(nthr >> 5); w++) ipx_fold(has, acc, s_has[w], s_acc[w]);
            ipx_c.hub_arrived[h.i] = 0; /* every chunk of the hub has arrived */
        }
    }
    if (threadIdx.x == 0 && last != 0) return (unsigned long long)ipx_sb_compute_next(h.v, has, acc, out, next_stamp);
    return 0ULL;
}

/* 1: the warp class of the fused pull kernel takes 32 vertices per warp and
 * spreads their concatenated in-edges over its lanes (ipx_gather_expand);
 * 0: a warp per vertex.  Measured on directed R-MAT scale 25 (FP64
 * PageRank, 30 rounds): 191 ms with the expansion against 135 ms without
 * (its shuffles and segmented folds cost more than the idle lanes of the
 * warp per vertex), so it is off. */
#ifndef IPX_GATHER_EXPAND
#define IPX_GATHER_EXPAND 0
#endif
#ifndef IPX_EXPAND_STEPS
#define IPX_EXPAND_STEPS 4
#endif

/* The warp class of ipx_k_gather_compute, edge-balanced.  Most vertices of
 * the class have a few dozen in-edges, so a warp per vertex leaves most
 * lanes idle and pays the list -> row -> ids -> slots chain once per vertex.
 * Here a warp takes 32 vertices of the list (lane j owns vertex j), scans
 * their in-degrees, and walks the concatenated edges 32 per step, lane by
 * lane: each lane finds its vertex by a 5-step search of the exclusive
 * degree prefix, loads the id and the slot (IPX_EXPAND_STEPS steps' loads
 * in flight), the lanes of each vertex fold their messages by a segmented
 * reduction (a lane folds in its right neighbour's partial while it belongs
 * to the same vertex), and the vertex's owner lane folds the segment's
 * result into its own.  A vertex's messages are folded in edge order within
 * a step, as a tree, and step after step: only the order of the ip_combine
 * calls differs from the reference's sequential fold.  Then every lane runs
 * the compute phase of its own vertex.  Degrees are below 2^32 / 32 (the
 * class bound t1). */
__device__ __forceinline__ unsigned long long ipx_gather_expand(const uint32_t* __restrict__ list, uint64_t n,
                                                                const ipx_vid* __restrict__ adj,
                                                                const uint64_t* __restrict__ row,
                                                                const ipx_sbslot* __restrict__ bs, uint32_t stamp,
                                                                ipx_sbslot* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ipx_gstride() >> 5;
    unsigned long long cnt = 0;
    for (uint64_t base = (ipx_gtid() >> 5) * 32; base < n; base += nwarps * 32) {
        const bool valid = base + lane < n;
        uint64_t v = 0, r0 = 0;
        uint32_t deg = 0;
        if (valid) {
            v = list[base + lane];
            r0 = row[v];
            deg = (uint32_t)(row[v + 1] - r0);
        }
        uint32_t inc = deg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(IPX_FULL, inc, o);
            if (lane >= o) inc += t;
        }
        const uint32_t excl = inc - deg;
        const uint32_t total = __shfl_sync(IPX_FULL, inc, 31);
        bool has = false;
        ipx_msg acc;
        for (uint32_t t0 = 0; t0 < total; t0 += 32 * IPX_EXPAND_STEPS) {
            int jk[IPX_EXPAND_STEPS];
            ipx_sbslot w[IPX_EXPAND_STEPS];
#pragma unroll
            for (int k = 0; k < IPX_EXPAND_STEPS; k++) {
                const uint32_t pos = t0 + (uint32_t)(32 * k + lane);
                int j = 0;
#pragma unroll
                for (int st = 16; st > 0; st >>= 1) {
                    const uint32_t ex = __shfl_sync(IPX_FULL, excl, j + st);
                    if (ex <= pos) j += st;
                }
                const uint64_t rj = __shfl_sync(IPX_FULL, r0, j);
                const uint32_t xj = __shfl_sync(IPX_FULL, excl, j);
                jk[k] = pos < total ? j : 32 + lane; /* past the end: a segment of its own */
                w[k] = ipx_no_slot<ipx_sbslot>();
                if (pos < total) {
                    const uint64_t u = (uint64_t)ipx_ld_stream(&adj[rj + (pos - xj)]);
                    w[k] = __ldg(&bs[u]);
                }
            }
#pragma unroll
            for (int k = 0; k < IPX_EXPAND_STEPS; k++) {
                ipx_msg m;
                bool h = ipx_slot_take(w[k], stamp, m);
                const int j = jk[k];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const bool h2 = __shfl_down_sync(IPX_FULL, h, o);
                    const ipx_msg m2 = ipx_shfl_down(m, o);
                    const int j2 = __shfl_down_sync(IPX_FULL, j, o);
                    if (lane + o < 32 && j2 == j) ipx_fold(h, m, h2, m2);
                }
                /* lane j's segment in this step starts at its first edge
                 * here (or at lane 0 when it began in an earlier step) */
                const uint32_t ts = t0 + 32u * k;
                const bool meets = deg && excl < ts + 32 && excl + deg > ts;
                const int src = meets ? (int)(excl > ts ? excl - ts : 0u) : lane;
                const bool hs = __shfl_sync(IPX_FULL, h, src);
                const ipx_msg ms = ipx_shfl_idx(m, src);
                if (meets) ipx_fold(has, acc, hs, ms);
            }
        }
        if (valid) cnt += ipx_sb_compute_next(v, has, acc, out, stamp + 1);
    }
    return cnt;
}

#ifndef IPX_HUB_SMEM
#define IPX_HUB_SMEM 1
#endif
/* In-edges a thread of the staged hub gather loads per step. */
#ifndef IPX_HUB_UNROLL
#define IPX_HUB_UNROLL 4
#endif
/* Lanes per vertex in the middle class of the fused pull kernel.  On
 * directed R-MAT scale 25 (FP64 PageRank, 30 rounds) 16 lanes took 118 ms,
 * 8 lanes 119 ms and a whole warp 135 ms: most vertices of the class have a
 * few dozen in-edges. */
#ifndef IPX_GATHER_GROUP
#define IPX_GATHER_GROUP 16
#endif

/* The hub class of ipx_k_gather_compute with ids staged in shared memory:
 * two id buffers, each filled by one bulk copy per chunk and completed on
 * its own mbarrier.  Thread 0 locates chunk k+1 and starts its copy before
 * the CTA waits for chunk k's.  Each iteration thread 0 arrives once on the
 * barrier of the chunk it issues (with the copy's byte count, or alone when
 * the chunk has no whole 16-byte group), so buffer j's barrier completes its
 * u-th phase at its u-th use.  Edges outside the copied range are read from
 * global memory.  A wait that gives up (never expected) sets
 * IPX_ERR_COPY_TIMEOUT, and the CTA reads ids from global memory for the
 * rest of the launch; results stay exact. */

/* The hub class with a warp per chunk: the warp folds its chunk, lane 0
 * stores the fold, and the warp whose chunk arrives last folds the hub's
 * partials -- each lane a contiguous run of them, then the runs in order by
 * shuffles -- and lane 0 runs the vertex's compute phase. */
template <bool HOT>
__device__ __forceinline__ unsigned long long ipx_gather_hubs_warp(
    const ipx_vid* __restrict__ adj, const uint64_t* __restrict__ row, const uint32_t* __restrict__ list, uint64_t n,
    const uint32_t* __restrict__ prefix, uint32_t chunks, const ipx_sbslot* __restrict__ bs, uint32_t stamp,
    ipx_sbslot* __restrict__ out)
{
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ipx_gstride() >> 5;
    unsigned long long cnt = 0;
    for (uint64_t c = ipx_gtid() >> 5; c < chunks; c += nwarps) {
        ipx_hub_chunk h;
        ipx_locate_chunk(list, n, prefix, row, (uint32_t)c, h);
        bool has = false;
        ipx_msg acc;
        ipx_gather_fold_edges<HOT>(adj, bs, stamp, h.e0, h.e1, lane, 32, has, acc);
        ipx_warp_fold(has, acc);
        int last = 2; /* a hub of one chunk: its fold is the hub's */
        if (lane == 0 && h.nch != 1) {
            ipx_bslot_put(&ipx_c.hub_part[h.c], acc, has ? 1u : 0u);
            __threadfence();
            last = atomicAdd(&ipx_c.hub_arrived[h.i], 1u) == h.nch - 1 ? 1 : 0;
        }
        last = __shfl_sync(IPX_FULL, last, 0);
        if (last == 1) {
            __threadfence();
            const uint32_t per = (h.nch + 31) / 32;
            const uint32_t k0 = (uint32_t)lane * per, k1 = min(k0 + per, h.nch);
            has = false;
            for (uint32_t k = k0; k < k1; k++) {
                const ipx_bslot p = __ldcg(&ipx_c.hub_part[h.c0 + k]);
                ipx_msg m;
                if (ipx_bslot_take(p, 1u, m)) ipx_fold(has, acc, true, m);
            }
            ipx_warp_fold(has, acc);
            if (lane == 0) ipx_c.hub_arrived[h.i] = 0; /* every chunk of the hub has arrived */
        }
        if (lane == 0 && last != 0) cnt += ipx_sb_compute_next(h.v, has, acc, out, stamp + 1);
    }
    return cnt;
}

template <bool HOT>
__device__ __forceinline__ unsigned long long ipx_gather_hubs_staged(
    const uint32_t* __restrict__ adj, const uint64_t* __restrict__ row, const uint32_t* __restrict__ list, uint64_t n,
    const uint32_t* __restrict__ prefix, uint32_t chunks, const ipx_sbslot* __restrict__ bs, uint32_t stamp,
    ipx_sbslot* __restrict__ out)
{
    __shared__ __align__(16) uint32_t s_ids[2][IPX_GATHER_CHUNK + 4];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ ipx_hub_chunk s_h[2];
    __shared__ bool s_has[IPX_THREADS / 32];
    __shared__ ipx_msg s_acc[IPX_THREADS / 32];
    __shared__ int s_fail;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nthr = blockDim.x;
    unsigned long long cnt = 0;
    bool pending[2] = {false, false}; /* thread 0: a copy issued and not yet waited for */
    if (threadIdx.x == 0) {
        ipx_mbar_init(&s_bar[0]);
        ipx_mbar_init(&s_bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    __syncthreads();
    auto issue = [&](uint32_t c, int buf) {
        ipx_hub_chunk& h = s_h[buf];
        ipx_locate_chunk(list, n, prefix, row, c, h);
        if (h.b > h.a0 && !s_fail) {
            const uint32_t bytes = (uint32_t)((h.b - h.a0) * 4);
            ipx_mbar_arrive_tx(&s_bar[buf], bytes);
            ipx_bulk_load(s_ids[buf], adj + h.a0, bytes, &s_bar[buf]);
            pending[buf] = true;
        } else {
            h.b = h.a0; /* nothing copied: every id from global memory */
            ipx_mbar_arrive_tx(&s_bar[buf], 0u);
        }
    };
    if (threadIdx.x == 0 && blockIdx.x < chunks) issue(blockIdx.x, 0);
    uint32_t it = 0;
    for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x, it++) {
        const int buf = (int)(it & 1);
        __syncthreads(); /* s_h[buf] is written; everyone is done with buffer buf ^ 1 */
        if (threadIdx.x == 0 && c + gridDim.x < chunks) issue(c + gridDim.x, buf ^ 1);
        bool staged = ipx_mbar_wait(&s_bar[buf], (it >> 1) & 1u, IPX_COPY_WAIT_LIMIT);
        if (!staged) {
            atomicOr(ipx_c.err, IPX_ERR_COPY_TIMEOUT);
            s_fail = 1;
        } else if (threadIdx.x == 0) {
            pending[buf] = false;
        }
        const ipx_hub_chunk h = s_h[buf];
        staged = staged && !s_fail;
        const uint64_t sb = staged ? h.b : h.e0; /* ids of [e0, sb) from shared memory */
        bool has = false;
        ipx_msg acc;
        for (uint64_t e = h.e0 + threadIdx.x; e < h.e1; e += IPX_HUB_UNROLL * (uint64_t)nthr) {
            uint32_t u[IPX_HUB_UNROLL];
            ipx_sbslot w[IPX_HUB_UNROLL];
#pragma unroll
            for (int k = 0; k < IPX_HUB_UNROLL; k++) {
                const uint64_t ek = e + (uint64_t)k * nthr;
                u[k] = (ek < sb) ? s_ids[buf][ek - h.a0] : (ek < h.e1 ? __ldcs(&adj[ek]) : 0u);
            }
#pragma unroll
            for (int k = 0; k < IPX_HUB_UNROLL; k++) {
                w[k] = (e + (uint64_t)k * nthr < h.e1) ? ipx_slot_ld<HOT>(bs, u[k]) : ipx_no_slot<ipx_sbslot>();
            }
#pragma unroll
            for (int k = 0; k < IPX_HUB_UNROLL; k++) {
                ipx_msg m;
                if (ipx_slot_take(w[k], stamp, m)) ipx_fold(has, acc, true, m);
            }
        }
        ipx_warp_fold(has, acc);
        if (lane == 0) {
            s_has[warp] = has;
            s_acc[warp] = acc;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            has = false;
            for (int w = 0; w < (int)(nthr >> 5); w++) ipx_fold(has, acc, s_has[w], s_acc[w]);
        }
        cnt += ipx_hub_chunk_done(h, has, acc, out, stamp + 1, s_has, s_acc);
    }
    /* a copy given up on may still be in flight: wait for it (bounded)
     * before the CTA's shared memory is released */
    if (threadIdx.x == 0) {
        for (int b = 0; b < 2; b++)
            if (pending[b]) {
                /* the phase in progress is the copy's: one of the two
                 * parities is the completed phase before it and returns at
                 * once, the other waits for the copy */
                ipx_mbar_wait(&s_bar[b], 0u, IPX_COPY_WAIT_LIMIT);
                ipx_mbar_wait(&s_bar[b], 1u, IPX_COPY_WAIT_LIMIT);
            }
    }
    __syncthreads();
    return cnt;
}

/* Single broadcast (pull), one superstep s >= 0 after its compute phase:
 * ip_fetch_broadcast_messages (combiner_single_broadcast_postamble.h:57-89)
 * for the vertices of one in-degree class, then, vertex by vertex, the
 * compute phase of superstep s+1.  The gather reads buffer s & 1 (slots
 * stamped s) and the compute writes buffer (s+1) & 1, which no gather of
 * superstep s reads, so the two phases need no grid-wide barrier between
 * them and the message goes from the fold to ip_compute in registers.
 * Count of superstep s: the vertices active after the gather.  When it is
 * 0 no vertex was active or received a message, so no compute phase of
 * superstep s+1 ran, and the loop ends (:164).  MODE 0: a thread per vertex,
 * folding in adjacency order as the reference does; 1: a warp; 2: a block
 * (lane-strided runs folded in order, then a tree, per chunk of a hub's
 * row; chunks folded in order: only the order of the ip_combine calls
 * differs). */
/* Resident CTAs per SM the fused pull kernel is compiled for: it carries
 * ip_compute besides the gather, which needs more registers than the other
 * edge kernels. */
#ifndef IPX_GATHER_CTAS
#define IPX_GATHER_CTAS 5
#endif

#ifndef IPX_EXPAND_CTAS
#define IPX_EXPAND_CTAS 4
#endif

template <int MODE, bool HOT>
__global__ void __launch_bounds__(IPX_THREADS, (MODE == 1 && IPX_GATHER_EXPAND) ? IPX_EXPAND_CTAS : IPX_GATHER_CTAS)
    ipx_k_gather_compute(const uint32_t* __restrict__ list,
                                                                                  uint64_t n,
                                                                                  const uint32_t* __restrict__ prefix)
{
    const uint64_t s = ipx_step();
    const uint32_t stamp = (uint32_t)s;
    /* HOT: ids of the in-lists carry the flag of the most gathered vertices */
    const ipx_vid* __restrict__ adj = HOT ? reinterpret_cast<const ipx_vid*>(ipx_c.in_adj_hot) : ipx_c.in_adj;
    const uint64_t* __restrict__ row = ipx_c.in_row;
    const ipx_sbslot* __restrict__ bs = ipx_c.sbslot[s & 1];
    ipx_sbslot* __restrict__ out = ipx_c.sbslot[(s + 1) & 1];
    unsigned long long cnt = 0;
    if constexpr (MODE == 0) {
        /* the next vertex's list entry is loaded while this vertex's
         * in-edges are folded */
        const uint64_t stride = ipx_gstride();
        uint64_t i = ipx_gtid(), v = (i < n) ? list[i] : 0;
        for (; i < n; i += stride) {
            const uint64_t vn = (i + stride < n) ? list[i + stride] : 0;
            bool has = false;
            ipx_msg acc;
            ipx_gather_fold_edges<HOT>(adj, bs, stamp, row[v], row[v + 1], 0, 1, has, acc);
            cnt += ipx_sb_compute_next(v, has, acc, out, stamp + 1);
            v = vn;
        }
    } else if constexpr (MODE == 1 && IPX_GATHER_EXPAND && !HOT) {
        cnt += ipx_gather_expand(list, n, adj, row, bs, stamp, out);
    } else if constexpr (MODE == 1 && IPX_GATHER_GROUP < 32) {
        /* IPX_GATHER_GROUP lanes per vertex: most vertices of the class have
         * a few dozen in-edges, which 8 lanes reading four ids each cover
         * in one or two steps, so a warp works on 32 / G vertices at once */
        constexpr int G = IPX_GATHER_GROUP;
        const int lane = threadIdx.x & 31, gl = lane & (G - 1);
        const unsigned mask = (G == 32) ? IPX_FULL : (((1u << G) - 1u) << (lane & ~(G - 1)));
        const uint64_t groups = ipx_gstride() / G;
        for (uint64_t i = ipx_gtid() / G; i < n; i += groups) {
            const uint64_t v = list[i];
            bool has = false;
            ipx_msg acc;
            ipx_gather_fold_edges<HOT>(adj, bs, stamp, row[v], row[v + 1], gl, G, has, acc);
            ipx_group_fold<G>(has, acc, mask);
            if (gl == 0) cnt += ipx_sb_compute_next(v, has, acc, out, stamp + 1);
        }
    } else if constexpr (MODE == 1) {
        /* the next vertex's list entry and row bounds are loaded while this
         * vertex's in-edges are folded */
        const int lane = threadIdx.x & 31;
        const uint64_t stride = ipx_gstride() >> 5;
        uint64_t i = ipx_gtid() >> 5, v = 0, r0 = 0, r1 = 0;
        if (i < n) {
            v = list[i];
            r0 = row[v];
            r1 = row[v + 1];
        }
        for (; i < n; i += stride) {
            uint64_t vn = 0, r0n = 0, r1n = 0;
            if (i + stride < n) {
                vn = list[i + stride];
                r0n = row[vn];
                r1n = row[vn + 1];
            }
            bool has = false;
            ipx_msg acc;
            ipx_gather_fold_edges<HOT>(adj, bs, stamp, r0, r1, lane, 32, has, acc);
            ipx_warp_fold(has, acc);
            if (lane == 0) cnt += ipx_sb_compute_next(v, has, acc, out, stamp + 1);
            v = vn;
            r0 = r0n;
            r1 = r1n;
        }
    } else {
        /* hubs in chunks of IPX_GATHER_CHUNK in-edges, spread over all CTAs
         * (one hub's row would otherwise keep one CTA busy long after the
         * others finished): each chunk's fold is stored, and the CTA whose
         * chunk arrives last folds the partials in chunk order, then runs
         * the compute phase (ipx_hub_chunk_done).  No CTA waits for another.
         * With 32-bit ids the chunk's ids are staged through shared memory:
         * while the CTA gathers one chunk, a bulk copy brings the ids of its
         * next chunk, so the slot loads are issued from shared memory
         * instead of behind a global id load each. */
        if (n == 0) return;
        const uint32_t chunks = prefix[n];
        if constexpr (IPX_HUB_WARP) {
            cnt += ipx_gather_hubs_warp<HOT>(adj, row, list, n, prefix, chunks, bs, stamp, out);
            ipx_block_count(cnt, &ipx_c.ctr[s & 3]);
            return;
        }
        if constexpr (sizeof(ipx_vid) == 4 && IPX_HUB_SMEM) {
            if ((reinterpret_cast<uintptr_t>(adj) & 15) == 0) {
                cnt += ipx_gather_hubs_staged<HOT>(reinterpret_cast<const uint32_t*>(adj), row, list, n, prefix, chunks,
                                              bs, stamp, out);
                ipx_block_count(cnt, &ipx_c.ctr[s & 3]);
                return;
            }
        }
        __shared__ bool s_has[IPX_THREADS / 32];
        __shared__ ipx_msg s_acc[IPX_THREADS / 32];
        __shared__ ipx_hub_chunk s_h;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            if (threadIdx.x == 0) ipx_locate_chunk(list, n, prefix, row, c, s_h);
            __syncthreads();
            const ipx_hub_chunk h = s_h;
            bool has = false;
            ipx_msg acc;
            ipx_gather_fold_edges<HOT>(adj, bs, stamp, h.e0, h.e1, threadIdx.x, blockDim.x, has, acc);
            ipx_warp_fold(has, acc);
            if (lane == 0) {
                s_has[warp] = has;
                s_acc[warp] = acc;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                has = false;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) ipx_fold(has, acc, s_has[w], s_acc[w]);
            }
            cnt += ipx_hub_chunk_done(h, has, acc, out, stamp + 1, s_has, s_acc);
            __syncthreads();
        }
    }
    ipx_block_count(cnt, &ipx_c.ctr[s & 3]);
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
        x.id = ipx_user_id(v);
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
            ipx_bslot_put(&ipx_c.bslot[0][v], x.ipx_out, (uint32_t)s);
            ipx_set_bit_agg(ipx_c.bcaster, v);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Initialisation kernels (ip_init_vertex_range of each version).           */
/* ------------------------------------------------------------------------ */
__global__ void ipx_k_init_values(uint64_t first, uint64_t last)
{
    /* [first, last] are ids in the caller's numbering: on a renamed graph
     * every vertex checks its own id */
    const bool renamed = ipx_c.vid_of != nullptr;
    const uint64_t lo = renamed ? 0 : first, hi = renamed ? ~0ULL : last;
    for (uint64_t v = lo + ipx_gtid(); v <= hi && v < ipx_c.V; v += ipx_gstride()) {
        if (renamed) {
            const uint64_t id = ipx_c.vid_of[v];
            if (id < first || id > last) continue;
        }
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

/* out[i] = value of the vertex whose id is i in the caller's numbering. */
__global__ void ipx_k_values_by_id(ipx_val* __restrict__ out)
{
    for (uint64_t i = ipx_gtid(); i < ipx_c.V; i += ipx_gstride()) out[i] = ipx_c.value[ipx_c.vindex_of[i]];
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
#if IPX_VERSION == IPX_SINGLE_BROADCAST
    /* the fused kernels of superstep s run the compute phase of s + 1
     * (superstep 0's own compute phase, ipx_k_compute_sb0, ran before) */
    ipd_compute_superstep = s + 1;
#endif
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
    ipd_compute_superstep = s + 1;
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
