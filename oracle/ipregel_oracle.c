/*
 * ipregel_oracle.c -- TEST INFRASTRUCTURE ONLY (the CPU oracle).
 *
 * Sequential restatement of iPregel's superstep engine.  Each version follows
 * the reference loop it cites, phase by phase, with OpenMP removed: the
 * reference's results do not depend on the thread count for these apps
 * (min combiners are order-free; the pull fold is sequential per vertex), so
 * a single-threaded pass in vertex order reproduces them.
 *
 * Checked against the reference's own binaries (oracle/_ref/, built by
 * oracle/Makefile from the reference sources) by tests/test_oracle_vs_reference.py
 * and against committed fixtures in tests/golden/.  Never linked into the
 * product; see ipregel_oracle.h for who may call it.
 */
#define _GNU_SOURCE
#include "ipregel_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Counter-based generator (same arithmetic as the device generator).       */
/* ------------------------------------------------------------------------ */

static inline uint64_t og_mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}

/* The n-th SplitMix64 output of a stream keyed by the seed, n = (i<<6)|l. */
static inline uint64_t og_draw(uint64_t seedk, uint64_t i, uint32_t l)
{
    return og_mix64(seedk + ((i << 6) | l) * 0x9E3779B97F4A7C15ULL);
}

static uint64_t og_seed_key(uint64_t seed)
{
    return og_mix64(seed ^ 0x5851F42D4C957F2DULL);
}

/* LSD radix sort of u64 keys, 16-bit digits, skipping constant digits. */
static int og_radix_sort(uint64_t* keys, uint64_t n)
{
    if (n < 2) return 0;
    uint64_t* tmp = (uint64_t*)malloc(n * sizeof(uint64_t));
    uint64_t* cnt = (uint64_t*)malloc(65536 * sizeof(uint64_t));
    if (!tmp || !cnt) { free(tmp); free(cnt); return -2; }
    uint64_t* src = keys;
    uint64_t* dst = tmp;
    for (int pass = 0; pass < 4; pass++) {
        int sh = pass * 16;
        memset(cnt, 0, 65536 * sizeof(uint64_t));
        for (uint64_t i = 0; i < n; i++) cnt[(src[i] >> sh) & 0xFFFF]++;
        if (cnt[(src[0] >> sh) & 0xFFFF] == n) continue;
        uint64_t acc = 0;
        for (int d = 0; d < 65536; d++) { uint64_t c = cnt[d]; cnt[d] = acc; acc += c; }
        for (uint64_t i = 0; i < n; i++) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
        uint64_t* t = src; src = dst; dst = t;
    }
    if (src != keys) memcpy(keys, src, n * sizeof(uint64_t));
    free(tmp);
    free(cnt);
    return 0;
}

/* Sort + dedup keys (src<<32|dst) and write CSR.  Returns E. */
static int64_t og_keys_to_csr(uint64_t* keys, uint64_t n, uint64_t V,
                              uint64_t* idx, uint32_t* adj, uint64_t max_edges)
{
    if (og_radix_sort(keys, n) != 0) return -2;
    uint64_t E = 0;
    for (uint64_t i = 0; i < n; i++) {
        if (i > 0 && keys[i] == keys[i - 1]) continue;
        keys[E++] = keys[i];
    }
    if (idx) {
        uint64_t e = 0;
        for (uint64_t v = 0; v < V; v++) {
            while (e < E && (keys[e] >> 32) < v) e++;
            idx[v] = e;
        }
    }
    if (adj) {
        if (E > max_edges) return -1;
        for (uint64_t e = 0; e < E; e++) adj[e] = (uint32_t)(keys[e] & 0xFFFFFFFFULL);
    }
    return (int64_t)E;
}

int64_t og_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b,
                    double c, uint64_t seed, int undirected, uint64_t* idx,
                    uint32_t* adj, uint64_t max_edges)
{
    if (scale == 0 || scale > 31) return -1;
    const uint64_t V = 1ULL << scale;
    const uint64_t M = (uint64_t)edge_factor << scale;
    const uint64_t ta = (uint64_t)(a * 4294967296.0);
    const uint64_t tab = (uint64_t)((a + b) * 4294967296.0);
    const uint64_t tabc = (uint64_t)((a + b + c) * 4294967296.0);
    const uint64_t sk = og_seed_key(seed);
    uint64_t* keys = (uint64_t*)malloc((undirected ? 2 : 1) * (M ? M : 1) * sizeof(uint64_t));
    if (!keys) return -2;
    uint64_t n = 0;
    for (uint64_t i = 0; i < M; i++) {
        uint64_t s = 0, d = 0;
        for (uint32_t l = 0; l < scale; l++) {
            uint64_t r = og_draw(sk, i, l) >> 32;
            uint64_t sb = r >= tab;
            uint64_t db = (r >= ta && r < tab) || r >= tabc;
            s = (s << 1) | sb;
            d = (d << 1) | db;
        }
        if (s == d) continue;
        keys[n++] = (s << 32) | d;
        if (undirected) keys[n++] = (d << 32) | s;
    }
    int64_t E = og_keys_to_csr(keys, n, V, idx, adj, max_edges);
    free(keys);
    return E;
}

int64_t og_gen_er(uint64_t V, uint64_t m, uint64_t seed, int undirected,
                  uint64_t* idx, uint32_t* adj, uint64_t max_edges)
{
    if (V == 0 || V > 4294967296ULL) return -1;
    const uint64_t sk = og_seed_key(seed);
    uint64_t* keys = (uint64_t*)malloc((undirected ? 2 : 1) * (m ? m : 1) * sizeof(uint64_t));
    if (!keys) return -2;
    uint64_t n = 0;
    for (uint64_t i = 0; i < m; i++) {
        uint64_t s = ((og_draw(sk, i, 0) >> 32) * V) >> 32;
        uint64_t d = ((og_draw(sk, i, 1) >> 32) * V) >> 32;
        if (s == d) continue;
        keys[n++] = (s << 32) | d;
        if (undirected) keys[n++] = (d << 32) | s;
    }
    int64_t E = og_keys_to_csr(keys, n, V, idx, adj, max_edges);
    free(keys);
    return E;
}

void og_gen_weights(uint64_t V, uint64_t E, const uint64_t* idx,
                    const uint32_t* adj, uint32_t wmax, uint64_t seed,
                    uint32_t* wgt)
{
    const uint64_t wk = og_mix64(seed ^ 0x77ULL);
    for (uint64_t u = 0; u < V; u++) {
        uint64_t end = (u + 1 < V) ? idx[u + 1] : E;
        for (uint64_t e = idx[u]; e < end; e++) {
            uint64_t v = adj[e];
            uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
            wgt[e] = 1u + (uint32_t)(og_mix64(wk ^ ((lo << 32) | hi)) % wmax);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Exact Dijkstra for the weighted-SSSP application.                        */
/* ------------------------------------------------------------------------ */

typedef struct { uint64_t d; uint64_t v; } og_hitem;

static void og_heap_push(og_hitem* h, uint64_t* n, og_hitem x)
{
    uint64_t i = (*n)++;
    while (i > 0) {
        uint64_t p = (i - 1) / 2;
        if (h[p].d <= x.d) break;
        h[i] = h[p];
        i = p;
    }
    h[i] = x;
}

static og_hitem og_heap_pop(og_hitem* h, uint64_t* n)
{
    og_hitem top = h[0];
    og_hitem x = h[--(*n)];
    uint64_t i = 0;
    for (;;) {
        uint64_t l = 2 * i + 1;
        if (l >= *n) break;
        uint64_t r = l + 1;
        uint64_t m = (r < *n && h[r].d < h[l].d) ? r : l;
        if (h[m].d >= x.d) break;
        h[i] = h[m];
        i = m;
    }
    if (*n > 0) h[i] = x;
    return top;
}

int og_dijkstra(uint64_t V, uint64_t E, const uint64_t* idx,
                const uint32_t* adj, const uint32_t* wgt, uint64_t source,
                uint32_t* dist)
{
    for (uint64_t v = 0; v < V; v++) dist[v] = 0xFFFFFFFFu;
    if (source >= V) return 0;
    og_hitem* h = (og_hitem*)malloc((E + 1) * sizeof(og_hitem));
    if (!h) return -2;
    uint64_t n = 0;
    dist[source] = 0;
    og_hitem s0 = { 0, source };
    og_heap_push(h, &n, s0);
    while (n > 0) {
        og_hitem it = og_heap_pop(h, &n);
        if (it.d != dist[it.v]) continue;
        uint64_t end = (it.v + 1 < V) ? idx[it.v + 1] : E;
        for (uint64_t e = idx[it.v]; e < end; e++) {
            uint64_t nd = it.d + wgt[e];
            if (nd < dist[adj[e]]) {
                dist[adj[e]] = (uint32_t)nd;
                og_hitem y = { nd, adj[e] };
                og_heap_push(h, &n, y);
            }
        }
    }
    free(h);
    return 0;
}

int og_write_graph(const char* path, uint64_t V, uint64_t E,
                   const uint64_t* idx, const uint32_t* adj,
                   const uint32_t* wgt)
{
    char name[4096];
    FILE* f;
    snprintf(name, sizeof name, "%s.config", path);
    if (!(f = fopen(name, "w"))) return -1;
    fprintf(f, "%llu %llu\n", (unsigned long long)V, (unsigned long long)E);
    fclose(f);
    snprintf(name, sizeof name, "%s.idx", path);
    if (!(f = fopen(name, "wb"))) return -1;
    if (V && fwrite(idx, sizeof(uint64_t), V, f) != V) { fclose(f); return -1; }
    fclose(f);
    snprintf(name, sizeof name, "%s.adj", path);
    if (!(f = fopen(name, "wb"))) return -1;
    if (E && fwrite(adj, sizeof(uint32_t), E, f) != E) { fclose(f); return -1; }
    fclose(f);
    if (wgt) {
        snprintf(name, sizeof name, "%s.wgt", path);
        if (!(f = fopen(name, "wb"))) return -1;
        if (E && fwrite(wgt, sizeof(uint32_t), E, f) != E) { fclose(f); return -1; }
        fclose(f);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Engine restatement.                                                      */
/* ------------------------------------------------------------------------ */

typedef union { uint64_t u; double d; } ogw;

typedef struct og_ctx {
    const og_params* p;
    uint64_t V, E;
    uint64_t* row;      /* V+1 out-row starts */
    uint64_t* adj;      /* E out-neighbour ids, widened */
    const uint32_t* wgt;
    uint64_t* in_row;   /* in-neighbour lists for the fetch phase */
    uint64_t* in_adj;
    int own_in;         /* in lists allocated (directed) or aliased (undirected) */
    uint64_t s;         /* ip_superstep */
    uint8_t *active, *has_message, *has_next, *has_b, *bt;
    ogw *message, *next, *bval, *value;
    uint64_t *list, list_size, *list_new, list_new_size;
    uint64_t edges;
    int fatal;
    int is_double;
    double teleport;
    uint64_t id_mask;   /* wrap-around of IP_MESSAGE_TYPE arithmetic */
} og_ctx;

static inline uint64_t og_outdeg(const og_ctx* c, uint64_t v) { return c->row[v + 1] - c->row[v]; }

/* ip_combine of each application: min (cc.c:57-63, sssp.c:73-79) or sum
 * (pagerank.c:68-71). */
static inline void og_combine(const og_ctx* c, ogw* a, ogw b)
{
    if (c->is_double) a->d += b.d;
    else if (a->u > b.u) a->u = b.u;
}

/* ip_send_message (combiner: src/combiner_postamble.h:54-79; spread:
 * src/combiner_spread_postamble.h:73-98).  The first message is stored, later
 * ones go through ip_cas (combiner_postamble.h:41-52), whose message parameter
 * has type IP_VERTEX_ID_TYPE. */
static void og_send(og_ctx* c, uint64_t id, ogw m)
{
    int v = c->p->version;
    if (v == OG_SINGLE_BROADCAST || v == OG_SPREAD_SINGLE_BROADCAST) {
        /* combiner_single_broadcast_postamble.h:42-49: fatal. */
        c->fatal = -3;
        return;
    }
    c->edges++;
    if (c->has_next[id]) {
        if (c->p->truncate_push && c->is_double) {
            if (c->id_mask == 0xFFFFFFFFULL) m.d = (double)(uint32_t)m.d;
            else m.d = (double)(uint64_t)m.d;
        }
        og_combine(c, &c->next[id], m);
    } else {
        c->next[id] = m;
        c->has_next[id] = 1;
        if (v == OG_SPREAD) c->list_new[c->list_new_size++] = id;  /* ip_add_spread_vertex */
    }
}

/* ip_broadcast of each version. */
static void og_broadcast(og_ctx* c, uint64_t v, ogw m)
{
    switch (c->p->version) {
    case OG_COMBINER:   /* combiner_postamble.h:81-87 */
    case OG_SPREAD:     /* combiner_spread_postamble.h:100-106 */
        for (uint64_t e = c->row[v]; e < c->row[v + 1]; e++) og_send(c, c->adj[e], m);
        break;
    case OG_SINGLE_BROADCAST:  /* combiner_single_broadcast_postamble.h:51-55 */
        c->has_b[v] = 1;
        c->bval[v] = m;
        break;
    case OG_SPREAD_SINGLE_BROADCAST:  /* combiner_spread_single_broadcast_postamble.h:64-76 */
        c->has_b[v] = 1;
        c->bval[v] = m;
        for (uint64_t e = c->row[v]; e < c->row[v + 1]; e++) c->bt[c->adj[e]] = 1;
        c->edges += og_outdeg(c, v);
        break;
    }
}

static inline int og_get_next_message(og_ctx* c, uint64_t v, ogw* m)
{
    if (c->has_message[v]) {
        *m = c->message[v];
        c->has_message[v] = 0;
        return 1;
    }
    return 0;
}

static inline void og_vote_to_halt(og_ctx* c, uint64_t v)
{
    if (c->p->version == OG_COMBINER || c->p->version == OG_SINGLE_BROADCAST) c->active[v] = 0;
    /* spread versions: no-op (combiner_spread_postamble.h:433-436) */
}

/* ---- applications ---- */

static void og_compute(og_ctx* c, uint64_t v)
{
    const uint64_t UMAX = 4294967295ULL;  /* UINT_MAX in sssp.c */
    ogw m;
    switch (c->p->app) {
    case OG_APP_CC: {  /* benchmarks/cc.c:31-55 */
        if (c->s == 0) {
            c->value[v].u = v;
            og_broadcast(c, v, c->value[v]);
        } else {
            uint64_t tmp = c->value[v].u;
            while (og_get_next_message(c, v, &m))
                if (c->value[v].u > m.u) c->value[v].u = m.u;
            if (tmp != c->value[v].u) og_broadcast(c, v, c->value[v]);
        }
        og_vote_to_halt(c, v);
        break;
    }
    case OG_APP_PAGERANK:  /* benchmarks/pagerank.c:36-66 */
    case OG_APP_PPR: {
        const double V = (double)c->V;
        int ppr = c->p->app == OG_APP_PPR;
        if (c->s == 0) {
            c->value[v].d = ppr ? (v == c->p->source ? 1.0 : 0.0) : 1.0 / V;
        } else {
            double sum = 0.0;
            while (og_get_next_message(c, v, &m)) sum += m.d;
            double base = ppr ? (v == c->p->source ? c->teleport : 0.0) : c->teleport / V;
            c->value[v].d = base + c->p->damping * sum;
        }
        if (c->s < c->p->rounds) {
            uint64_t deg = og_outdeg(c, v);
            if (deg > 0 && (!ppr || c->value[v].d > 0.0)) {
                ogw b;
                b.d = c->value[v].d / (double)deg;
                og_broadcast(c, v, b);
            }
        } else {
            og_vote_to_halt(c, v);
        }
        break;
    }
    case OG_APP_SSSP: {  /* benchmarks/sssp.c:38-71 */
        if (c->s == 0) {
            if (v == c->p->source) {
                c->value[v].u = 0;
                ogw b; b.u = 1;
                og_broadcast(c, v, b);
            } else {
                c->value[v].u = UMAX;
            }
        } else {
            uint64_t m0 = UMAX;
            while (og_get_next_message(c, v, &m))
                if (m0 > m.u) m0 = m.u;
            if (m0 < c->value[v].u) {
                c->value[v].u = m0;
                ogw b; b.u = (m0 + 1) & c->id_mask;
                og_broadcast(c, v, b);
            }
        }
        og_vote_to_halt(c, v);
        break;
    }
    case OG_APP_SSSP_W: {
        uint64_t m0;
        int go = 0;
        if (c->s == 0) {
            if (v == c->p->source) { c->value[v].u = 0; m0 = 0; go = 1; }
            else c->value[v].u = UMAX;
        } else {
            m0 = UMAX;
            while (og_get_next_message(c, v, &m))
                if (m0 > m.u) m0 = m.u;
            if (m0 < c->value[v].u) { c->value[v].u = m0; go = 1; }
        }
        if (go) {
            for (uint64_t e = c->row[v]; e < c->row[v + 1]; e++) {
                ogw b; b.u = (m0 + c->wgt[e]) & c->id_mask;
                og_send(c, c->adj[e], b);
            }
        }
        og_vote_to_halt(c, v);
        break;
    }
    }
}

/* ip_fetch_broadcast_messages: combiner_single_broadcast_postamble.h:57-89
 * (with reactivation) and combiner_spread_single_broadcast_postamble.h:78-104
 * (without).  Fold in in-neighbour order, seeded by the first broadcaster. */
static void og_fetch(og_ctx* c, uint64_t v, uint64_t* count, int reactivate)
{
    uint64_t i = c->in_row[v], end = c->in_row[v + 1];
    c->edges += end - i;
    while (i < end && !c->has_b[c->in_adj[i]]) i++;
    if (i >= end) {
        c->has_message[v] = 0;
        return;
    }
    if (reactivate && !c->active[v]) {
        (*count)++;
        c->active[v] = 1;
    }
    c->has_message[v] = 1;
    c->message[v] = c->bval[c->in_adj[i]];
    for (i++; i < end; i++)
        if (c->has_b[c->in_adj[i]]) og_combine(c, &c->message[v], c->bval[c->in_adj[i]]);
}

/* og_fetch with reactivation, for concurrent calls on distinct vertices:
 * the edges it reads are returned instead of added to c->edges, and the
 * reactivations are counted into the caller's *count. */
static uint64_t og_fetch_sb(og_ctx* c, uint64_t v, uint64_t* count)
{
    uint64_t i = c->in_row[v], end = c->in_row[v + 1];
    const uint64_t edges = end - i;
    while (i < end && !c->has_b[c->in_adj[i]]) i++;
    if (i >= end) {
        c->has_message[v] = 0;
        return edges;
    }
    if (!c->active[v]) {
        (*count)++;
        c->active[v] = 1;
    }
    c->has_message[v] = 1;
    c->message[v] = c->bval[c->in_adj[i]];
    for (i++; i < end; i++)
        if (c->has_b[c->in_adj[i]]) og_combine(c, &c->message[v], c->bval[c->in_adj[i]]);
    return edges;
}

static int og_record(og_ctx* c, uint64_t count, uint64_t* counts_out, uint64_t max_counts)
{
    if (counts_out && c->s < max_counts) counts_out[c->s] = count;
    c->s++;
    if (c->p->max_supersteps && c->s >= c->p->max_supersteps) return -4;
    return 0;
}

int og_run(const og_graph* g, const og_params* p, void* values_out,
           uint64_t* counts_out, uint64_t max_counts, og_stats* stats)
{
    if (!g || !p || (g->id_bytes != 4 && g->id_bytes != 8)) return -1;
    if (p->version < 0 || p->version > 3 || p->app < 0 || p->app > 4) return -1;
    if ((p->app == OG_APP_SSSP_W) && !g->wgt) return -1;
    og_ctx c;
    memset(&c, 0, sizeof c);
    c.p = p;
    c.V = g->V;
    c.E = g->E;
    c.wgt = g->wgt;
    c.is_double = (p->app == OG_APP_PAGERANK || p->app == OG_APP_PPR);
    c.teleport = (p->damping == 0.85) ? 0.15 : 1.0 - p->damping;
    c.id_mask = g->id_bytes == 4 ? 0xFFFFFFFFULL : ~0ULL;
    const uint64_t V = c.V, E = c.E;
    int rc = 0;

    c.row = (uint64_t*)malloc((V + 1) * sizeof(uint64_t));
    c.adj = (uint64_t*)malloc((E ? E : 1) * sizeof(uint64_t));
    size_t vb = V ? V : 1;
    c.active = (uint8_t*)calloc(vb, 1);
    c.has_message = (uint8_t*)calloc(vb, 1);
    c.has_next = (uint8_t*)calloc(vb, 1);
    c.has_b = (uint8_t*)calloc(vb, 1);
    c.bt = (uint8_t*)calloc(vb, 1);
    c.message = (ogw*)calloc(vb, sizeof(ogw));
    c.next = (ogw*)calloc(vb, sizeof(ogw));
    c.bval = (ogw*)calloc(vb, sizeof(ogw));
    c.value = (ogw*)calloc(vb, sizeof(ogw));
    c.list = (uint64_t*)malloc(vb * sizeof(uint64_t));
    c.list_new = (uint64_t*)malloc(vb * sizeof(uint64_t));
    if (!c.row || !c.adj || !c.active || !c.has_message || !c.has_next || !c.has_b || !c.bt ||
        !c.message || !c.next || !c.bval || !c.value || !c.list || !c.list_new) {
        rc = -2;
        goto done;
    }
    /* Row lengths: offset differences, last row E - idx[V-1]
     * (src/iPregel_postamble.h:383-421). */
    for (uint64_t v = 0; v < V; v++) c.row[v] = g->idx[v];
    c.row[V] = E;
    for (uint64_t e = 0; e < E; e++)
        c.adj[e] = g->id_bytes == 4 ? ((const uint32_t*)g->adj)[e] : ((const uint64_t*)g->adj)[e];

    if (!g->directed) {
        /* in_neighbours alias the stored rows (iPregel_postamble.h:368-372). */
        c.in_row = c.row;
        c.in_adj = c.adj;
    } else {
        /* Mirror: in-lists in order of increasing source, then edge order
         * (iPregel_postamble.h:429-487). */
        c.own_in = 1;
        c.in_row = (uint64_t*)calloc(V + 1, sizeof(uint64_t));
        c.in_adj = (uint64_t*)malloc((E ? E : 1) * sizeof(uint64_t));
        uint64_t* fill = (uint64_t*)calloc(vb, sizeof(uint64_t));
        if (!c.in_row || !c.in_adj || !fill) { free(fill); rc = -2; goto done; }
        for (uint64_t e = 0; e < E; e++) {
            if (c.adj[e] >= V) { free(fill); rc = -1; goto done; }
            c.in_row[c.adj[e] + 1]++;
        }
        for (uint64_t v = 0; v < V; v++) c.in_row[v + 1] += c.in_row[v];
        for (uint64_t u = 0; u < V; u++)
            for (uint64_t e = c.row[u]; e < c.row[u + 1]; e++) {
                uint64_t w = c.adj[e];
                c.in_adj[c.in_row[w] + fill[w]++] = u;
            }
        free(fill);
    }
    for (uint64_t e = 0; e < E; e++)
        if (c.adj[e] >= V) { rc = -1; goto done; }

    uint64_t count;
    switch (p->version) {
    case OG_COMBINER: {  /* src/combiner_postamble.h:89-199 */
        for (uint64_t v = 0; v < V; v++) c.active[v] = 1;
        count = V;  /* ip_active_vertices = V, iPregel_postamble.h:517 */
        while (count != 0) {
            count = 0;
            for (uint64_t v = 0; v < V; v++) {
                if (c.active[v] || c.has_message[v]) {
                    c.active[v] = 1;
                    og_compute(&c, v);
                    if (c.fatal) { rc = c.fatal; goto done; }
                    if (c.active[v]) count++;
                }
            }
            for (uint64_t v = 0; v < V; v++) {
                if (c.has_next[v]) {
                    c.has_message[v] = 1;
                    c.message[v] = c.next[v];
                    c.has_next[v] = 0;
                    if (!c.active[v]) { c.active[v] = 1; count++; }
                }
            }
            if ((rc = og_record(&c, count, counts_out, max_counts))) goto done;
        }
        break;
    }
    case OG_SINGLE_BROADCAST: {  /* src/combiner_single_broadcast_postamble.h:91-259 */
        /* Both phases are loops over independent vertices, as the
         * reference's `omp for` loops are (:185-201, :213-220): a vertex's
         * compute writes only its own value, flags and broadcast slot, and a
         * vertex's fetch folds its in-list sequentially into its own
         * message, so running them on several threads gives the same bits. */
        for (uint64_t v = 0; v < V; v++) c.active[v] = 1;
        count = V;
        while (count != 0) {
            uint64_t cnt = 0, edges = 0;
            int fatal = 0;
            #pragma omp parallel for schedule(dynamic, 4096) reduction(+:cnt) reduction(|:fatal)
            for (uint64_t v = 0; v < V; v++) {
                c.has_b[v] = 0;
                if (c.active[v]) {
                    og_compute(&c, v);
                    if (c.fatal) fatal = 1;
                    if (c.active[v]) cnt++;
                }
            }
            if (fatal) { rc = c.fatal; goto done; }
            #pragma omp parallel for schedule(dynamic, 4096) reduction(+:cnt, edges)
            for (uint64_t v = 0; v < V; v++) edges += og_fetch_sb(&c, v, &cnt);
            c.edges += edges;
            count = cnt;
            if ((rc = og_record(&c, count, counts_out, max_counts))) goto done;
        }
        break;
    }
    case OG_SPREAD: {  /* src/combiner_spread_postamble.h:137-431 */
        count = 0;
        while (c.s == 0 || count > 0) {
            count = 0;
            if (c.s == 0) {
                for (uint64_t v = 0; v < V; v++) {
                    og_compute(&c, v);
                    if (c.fatal) { rc = c.fatal; goto done; }
                }
            } else {
                for (uint64_t i = 0; i < c.list_size; i++) {
                    og_compute(&c, c.list[i]);
                    if (c.fatal) { rc = c.fatal; goto done; }
                }
            }
            count = c.list_new_size;
            uint64_t* t = c.list; c.list = c.list_new; c.list_new = t;
            c.list_size = c.list_new_size;
            c.list_new_size = 0;
            for (uint64_t i = 0; i < c.list_size; i++) {
                uint64_t v = c.list[i];
                c.has_message[v] = 1;
                c.message[v] = c.next[v];
                c.has_next[v] = 0;
            }
            if ((rc = og_record(&c, count, counts_out, max_counts))) goto done;
        }
        break;
    }
    case OG_SPREAD_SINGLE_BROADCAST: {  /* src/combiner_spread_single_broadcast_postamble.h:106-399 */
        for (uint64_t v = 0; v < V; v++) c.list[v] = v;
        c.list_size = V;
        while (c.s == 0 || c.list_size > 0) {
            for (uint64_t i = 0; i < c.list_size; i++) {
                og_compute(&c, c.list[i]);
                if (c.fatal) { rc = c.fatal; goto done; }
            }
            c.list_size = 0;
            for (uint64_t v = 0; v < V; v++)
                if (c.bt[v]) c.list[c.list_size++] = v;
            count = c.list_size;
            for (uint64_t i = 0; i < c.list_size; i++) {
                uint64_t v = c.list[i];
                if (c.bt[v]) {
                    og_fetch(&c, v, NULL, 0);
                    c.bt[v] = 0;
                }
            }
            for (uint64_t v = 0; v < V; v++) c.has_b[v] = 0;
            if ((rc = og_record(&c, count, counts_out, max_counts))) goto done;
        }
        break;
    }
    }

    if (values_out) {
        for (uint64_t v = 0; v < V; v++) {
            if (c.is_double) ((double*)values_out)[v] = c.value[v].d;
            else if (g->id_bytes == 4) ((uint32_t*)values_out)[v] = (uint32_t)c.value[v].u;
            else ((uint64_t*)values_out)[v] = c.value[v].u;
        }
    }
done:
    if (stats) {
        stats->supersteps = c.s;
        stats->edges_traversed = c.edges;
    }
    free(c.row); free(c.adj);
    if (c.own_in) { free(c.in_row); free(c.in_adj); }
    free(c.active); free(c.has_message); free(c.has_next); free(c.has_b); free(c.bt);
    free(c.message); free(c.next); free(c.bval); free(c.value);
    free(c.list); free(c.list_new);
    return rc;
}
