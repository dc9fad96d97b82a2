/* oracle.c -- CPU restatement of the deterministic synchronous multilevel
 * schedule (TEST INFRASTRUCTURE; see oracle.h).  Plain C, single threaded,
 * written for clarity: dense scratch arrays, no clever data structures.
 *
 * Reference citations are paths inside the KaHIP source tree.
 */
#include "oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum {
    TAG_CSUB = 1, TAG_CTIE = 2, TAG_RSUB = 3, TAG_RTIE = 4, TAG_RPRIO = 5,
    TAG_BTIE = 6, TAG_BCLS = 7, TAG_BPRIO = 8, TAG_IP = 9, TAG_IPM = 10, TAG_MATCH = 11, TAG_JTIE = 12,
    TAG_EVO = 13
};

#define BAL_CLASSES 256

static void* xcalloc(size_t n, size_t s) {
    void* p = calloc(n ? n : 1, s);
    if (!p) abort();
    return p;
}
static void* xmalloc(size_t n) {
    void* p = malloc(n ? n : 1);
    if (!p) abort();
    return p;
}

/* ------------------------------------------------------------------ hashing */

uint64_t or_mix64(uint64_t z) {
    /* splitmix64 output function (Steele, Lea & Flood 2014) */
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t or_stream(int seed, int tag, int level, int round) {
    uint64_t s = or_mix64((uint64_t)(uint32_t)seed ^ ((uint64_t)(uint32_t)tag << 40));
    s = or_mix64(s ^ (uint64_t)(uint32_t)level);
    return or_mix64(s ^ (uint64_t)(uint32_t)round);
}

uint32_t or_hash(uint64_t stream, uint32_t x) {
    /* murmur3-style 32-bit finaliser (MurmurHash3 fmix32, Appleby) keyed by
     * both halves of the stream key */
    uint32_t h = (x * 0x9E3779B1u) ^ (uint32_t)stream;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= (uint32_t)(stream >> 32) | 1u;
    h ^= h >> 16;
    return h;
}

/* uniform 32-bit hash -> [0, n) by multiply-shift */
static uint32_t or_range(uint32_t h, uint32_t n) {
    return (uint32_t)(((uint64_t)h * n) >> 32);
}

/* ------------------------------------------------------------------- knobs */

void or_derive_knobs(int n, const int* vwgt, int k, double imbalance, int seed, int mode,
                     or_knobs* o) {
    memset(o, 0, sizeof(*o));
    o->k = k;
    o->imbalance = imbalance;
    o->seed = seed;
    o->mode = mode;
    /* app/balance_configuration.h:19-24: W = sum of node weights (NodeWeight) */
    uint32_t W = 0;
    for (int v = 0; v < n; ++v) W += vwgt ? (uint32_t)vwgt[v] : 1u;
    o->total_weight = W;
    /* interface/kaHIP_interface.cpp:115 then balance_configuration.h:40-47 */
    double imbalance_pct = 100 * imbalance;
    double epsilon = imbalance_pct / 100.0;
    double per_block = ceil(W / (double)k);
    if (imbalance_pct == 0) {
        o->upper_bound = (uint32_t)((1 + epsilon + 0.01) * per_block);
        o->final_bound = (uint32_t)per_block;
    } else {
        o->upper_bound = (uint32_t)((1 + epsilon) * per_block);
        o->final_bound = o->upper_bound;
    }
    /* stop_rules.h:46-56 (simple_stop_rule, work_load = W) */
    double x = 60;
    double ns = (double)n / (2.0 * x * k);
    if (ns < 60.0 * k) ns = 60.0 * k;
    o->num_stop = (uint32_t)ns;
    o->max_vertex_weight = (uint32_t)(1.5 * W / o->num_stop);
    /* size_constraint_label_propagation.cpp:57 -- ceil(U / cluster_coarsening_factor)
     * with cf = 18 (app/configuration.h:422), capped so that no coarse node
     * exceeds max_vertex_weight (the matching bound of the fast/eco presets). */
    uint32_t cb = (uint32_t)ceil(o->upper_bound / 18.0);
    if (o->max_vertex_weight + 1u < cb) cb = o->max_vertex_weight + 1u;
    o->cluster_bound = cb;
    int fast = (mode == 0 || mode == 3);
    o->lpc_rounds = fast ? 5 : 10;
    o->lpc_subrounds = 2;
    o->ref_rounds = fast ? 10 : 25;
    o->ref_subrounds = 2;
    o->ref_classes = 16;
    o->bal_iters = 64;
    o->ip_reps = fast ? 1 : 2;
    o->ip_tries = fast ? 4 : 16;
    o->ip_fm_passes = fast ? 3 : 6;
    o->ip_fm_stall = 100;
    o->max_levels = 48;
    o->coarsening = 0;
    o->match_rounds = 16;
    o->refinement = (fast && k > 8) ? 0 : 1; /* configuration.h:108-118: pair refinement up to k = 8 */
    o->jet_iters = 32;
    o->jet_patience = 12;
    o->jet_c0 = 1;
    o->jet_c = 3;
    o->ip_mode = 1;
    o->ip_jet_iters = 20;
    o->ip_jet_patience = 8;
}

/* stop_rules.h:64-66: continue coarsening after a level that went from nf to
 * nc nodes? */
int or_stop_continue(const or_knobs* kn, int nf, int nc) {
    double rate = 1.0 * nf / (double)nc;
    return rate >= 1.1 && (uint32_t)nc >= kn->num_stop;
}

/* ----------------------------------------------------------------- metrics */

long long or_edge_cut(const or_graph* g, const int* part) {
    /* quality_metrics.cpp:23-37 (64-bit accumulation) */
    long long cut = 0;
    for (int v = 0; v < g->n; ++v)
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e)
            if (part[v] != part[g->adjncy[e]]) cut += g->adjwgt[e];
    return cut / 2;
}

void or_block_weights(const or_graph* g, const int* part, int k, uint32_t* bw) {
    memset(bw, 0, sizeof(uint32_t) * (size_t)k);
    for (int v = 0; v < g->n; ++v) bw[part[v]] += (uint32_t)g->vwgt[v];
}

double or_balance_ratio(const or_graph* g, const int* part, int k) {
    /* quality_metrics.cpp:265-288 */
    uint32_t* bw = xcalloc((size_t)k, sizeof(uint32_t));
    double total = 0;
    for (int v = 0; v < g->n; ++v) { bw[part[v]] += (uint32_t)g->vwgt[v]; total += g->vwgt[v]; }
    double per = ceil(total / (double)k), mx = -1;
    for (int b = 0; b < k; ++b) if (bw[b] > mx) mx = bw[b];
    free(bw);
    return mx / per;
}

void or_rate_expansion_star_2(const or_graph* g, double* rating) {
    /* edge_ratings.cpp:171-183: 1.0*w*w / (c(u)*c(v)), denominator as a
     * 32-bit unsigned product */
    for (int v = 0; v < g->n; ++v) {
        uint32_t cv = (uint32_t)g->vwgt[v];
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
            uint32_t cu = (uint32_t)g->vwgt[g->adjncy[e]];
            int w = g->adjwgt[e];
            rating[e] = 1.0 * w * w / (uint32_t)(cu * cv);
        }
    }
}

/* ------------------------------------------------------ heavy-edge matching */

/* Primary key of an entry: the rating's IEEE bits (order-preserving for
 * non-negative doubles; NaN from 0/0 counts as 0) or the supplied 32-bit
 * rating. */
static uint64_t match_primary(const or_graph* g, const uint32_t* rq, int e, uint32_t cv, uint32_t cu) {
    if (rq) return rq[e];
    int w = g->adjwgt[e];
    double r = 1.0 * w * w / (uint32_t)(cu * cv);
    if (r != r) r = 0.0;
    uint64_t b;
    memcpy(&b, &r, sizeof b);
    return b;
}

/* Secondary key: hash of the unordered pair, then the complement of the
 * endpoint sum (unique among the entries of one row). */
static uint64_t match_secondary(uint64_t ks, uint32_t a, uint32_t b) {
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    uint32_t h = or_hash(ks, or_hash(ks, lo) ^ hi);
    return ((uint64_t)h << 32) | (uint32_t)~(lo + hi);
}

void or_hem_match(const or_graph* g, const or_knobs* kn, int level, const uint32_t* rq, int* label) {
    const int n = g->n;
    const uint64_t ks = or_stream(kn->seed, TAG_MATCH, level, 0);
    /* state: >= 0 unmatched (its weight), -1 matched, -2 no eligible neighbour left */
    long long* state = xmalloc(sizeof(long long) * (size_t)(n ? n : 1));
    int* best = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* mate = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int v = 0; v < n; ++v) { state[v] = (uint32_t)g->vwgt[v]; mate[v] = -1; }
    for (int r = 0; r < kn->match_rounds; ++r) {
        for (int v = 0; v < n; ++v) {
            best[v] = -1;
            if (state[v] < 0) continue;
            const uint32_t cv = (uint32_t)state[v];
            uint64_t b1 = 0, b2 = 0;
            for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
                int u = g->adjncy[e];
                if (u == v || state[u] < 0) continue;
                if ((uint64_t)cv + (uint64_t)state[u] > kn->max_vertex_weight) continue;
                uint64_t k1 = match_primary(g, rq, e, cv, (uint32_t)state[u]);
                uint64_t k2 = match_secondary(ks, (uint32_t)v, (uint32_t)u);
                if (best[v] < 0 || k1 > b1 || (k1 == b1 && k2 > b2)) { best[v] = u; b1 = k1; b2 = k2; }
            }
        }
        int matched = 0;
        for (int v = 0; v < n; ++v) {
            if (state[v] < 0) continue;
            if (best[v] >= 0 && best[best[v]] == v) { mate[v] = best[v]; ++matched; }
        }
        for (int v = 0; v < n; ++v) {
            if (state[v] < 0) continue;
            if (mate[v] >= 0) state[v] = -1;
            else if (best[v] < 0) state[v] = -2;
        }
        if (!matched) break;
    }
    for (int v = 0; v < n; ++v) label[v] = mate[v] >= 0 && mate[v] < v ? mate[v] : v;
    free(state); free(best); free(mate);
}

/* ------------------------------------------------------ isolated vertices */

/* No rule of the reference merges a vertex without neighbours; these bundles
 * keep coarsening going on graphs with many of them (R-MAT). */
void or_bundle_isolated(const or_graph* g, uint32_t bound, int* label) {
    if (g->n < 2 || bound < 2) return;
    uint32_t count = 0, wmax = 0;
    for (int v = 0; v < g->n; ++v)
        if (g->xadj[v + 1] == g->xadj[v]) {
            ++count;
            if ((uint32_t)g->vwgt[v] > wmax) wmax = (uint32_t)g->vwgt[v];
        }
    uint32_t group = wmax == 0 ? count : (bound - 1) / wmax;
    if (count < 2 || group < 2) return;
    uint32_t rank = 0;
    int first = -1;
    for (int v = 0; v < g->n; ++v) {
        if (g->xadj[v + 1] != g->xadj[v]) continue;
        if (rank % group == 0) first = v;
        label[v] = first;
        ++rank;
    }
}

/* --------------------------------------------------- neighbourhood scratch */

typedef struct {
    uint32_t* acc;  /* dense accumulator indexed by label */
    int* touched;   /* labels with a live entry */
    int ntouched;
} or_acc;

static void acc_init(or_acc* a, int labels, int maxdeg) {
    a->acc = xcalloc((size_t)labels, sizeof(uint32_t));
    a->touched = xmalloc(sizeof(int) * (size_t)(maxdeg + 1));
    a->ntouched = 0;
}
static void acc_free(or_acc* a) { free(a->acc); free(a->touched); }

/* conn[b] = sum of w(v,u) over neighbours u with lab[u] == b.  A label is
 * recorded as touched the first time an edge to it is seen, so zero-weight
 * edges still make their label a candidate. */
static void acc_gather(or_acc* a, const or_graph* g, int v, const int* lab, char* seen) {
    a->ntouched = 0;
    for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
        int b = lab[g->adjncy[e]];
        if (!seen[b]) { seen[b] = 1; a->touched[a->ntouched++] = b; }
        a->acc[b] += (uint32_t)g->adjwgt[e];
    }
}
static void acc_clear(or_acc* a, char* seen) {
    for (int i = 0; i < a->ntouched; ++i) { a->acc[a->touched[i]] = 0; seen[a->touched[i]] = 0; }
    a->ntouched = 0;
}

static int max_degree(const or_graph* g) {
    int d = 0;
    for (int v = 0; v < g->n; ++v) if (g->xadj[v + 1] - g->xadj[v] > d) d = g->xadj[v + 1] - g->xadj[v];
    return d;
}

/* Candidate order shared by clustering and refinement: higher connection
 * wins; the current label wins ties against everything; among other labels
 * the smaller hash(tie stream, label) wins, then the smaller label.
 * (The reference breaks ties with a coin flip, random_functions.h:152-155.) */
static int beats(uint32_t cb, int b, uint32_t ca, int a, int own, uint64_t ks_tie) {
    if (cb != ca) return cb > ca;
    if (a == own) return 0;
    uint32_t hb = or_hash(ks_tie, (uint32_t)b), ha = or_hash(ks_tie, (uint32_t)a);
    if (hb != ha) return hb < ha;
    return b < a;
}

/* ----------------------------------------------------------- LP clustering */

/* One node's choice.  Rules of size_constraint_label_propagation.cpp:160-190:
 * start from the own cluster with its connection, move to a neighbouring
 * cluster b with a strictly larger connection when
 * cluster_weight[b] + c(v) < bound (:175); the own cluster is always
 * allowed. */
static int cluster_choice(const or_graph* g, int v, const int* label, const uint32_t* cw,
                          uint32_t bound, or_acc* a, char* seen, uint64_t ks_tie) {
    acc_gather(a, g, v, label, seen);
    int own = label[v];
    uint32_t cv = (uint32_t)g->vwgt[v];
    int best = own;
    uint32_t bestc = seen[own] ? a->acc[own] : 0;
    for (int i = 0; i < a->ntouched; ++i) {
        int b = a->touched[i];
        if (b == own) continue;
        uint32_t c = a->acc[b];
        if (c == 0) continue;
        if (!((uint64_t)cw[b] + cv < bound)) continue;
        if (beats(c, b, bestc, best, own, ks_tie)) { best = b; bestc = c; }
    }
    acc_clear(a, seen);
    return best;
}

void or_lp_cluster(const or_graph* g, const or_knobs* kn, int level, int* label) {
    const int n = g->n;
    uint32_t* cw = xmalloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    int* prop = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    uint64_t* incoming = xcalloc((size_t)n, sizeof(uint64_t));
    int* minv = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    char* seen = xcalloc((size_t)n, 1);
    or_acc a;
    acc_init(&a, n, max_degree(g));
    for (int v = 0; v < n; ++v) { label[v] = v; cw[v] = (uint32_t)g->vwgt[v]; minv[v] = INT_MAX; }
    for (int r = 0; r < kn->lpc_rounds; ++r) {
        uint64_t ks_sub = or_stream(kn->seed, TAG_CSUB, level, r);
        uint64_t ks_tie = or_stream(kn->seed, TAG_CTIE, level, r);
        /* round 0 runs as one fully synchronous sub-round (every cluster is
         * still a single node), later rounds in lpc_subrounds sub-rounds */
        const uint32_t S = r == 0 ? 1u : (uint32_t)kn->lpc_subrounds;
        for (uint32_t s = 0; s < S; ++s) {
            /* 1. every active node decides against the state at sub-round start */
            for (int v = 0; v < n; ++v) {
                prop[v] = -1;
                if (or_range(or_hash(ks_sub, (uint32_t)v), S) != s) continue;
                int b = cluster_choice(g, v, label, cw, kn->cluster_bound, &a, seen, ks_tie);
                if (b != label[v]) prop[v] = b;
            }
            /* 2. admission: all proposals into b if they fit together,
             *    otherwise only the one of the smallest node id (which fits
             *    on its own by the test in cluster_choice) */
            for (int v = 0; v < n; ++v) {
                int b = prop[v];
                if (b < 0) continue;
                incoming[b] += (uint32_t)g->vwgt[v];
                if (v < minv[b]) minv[b] = v;
            }
            for (int v = 0; v < n; ++v) {
                int b = prop[v];
                if (b < 0) continue;
                int ok = ((uint64_t)cw[b] + incoming[b] < kn->cluster_bound) || minv[b] == v;
                if (!ok) prop[v] = -2 - b; /* rejected, remember target for reset */
            }
            /* 3. apply */
            for (int v = 0; v < n; ++v) {
                int b = prop[v];
                if (b == -1) continue;
                int t = b >= 0 ? b : -2 - b;
                incoming[t] = 0;
                minv[t] = INT_MAX;
                if (b < 0) continue;
                cw[label[v]] -= (uint32_t)g->vwgt[v];
                cw[b] += (uint32_t)g->vwgt[v];
                label[v] = b;
            }
        }
    }
    acc_free(&a);
    free(cw); free(prop); free(incoming); free(minv); free(seen);
}

int or_lp_cluster_seq(const or_graph* g, uint32_t bound, int rounds, const int* order, int* label) {
    const int n = g->n;
    uint32_t* cw = xmalloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    char* seen = xcalloc((size_t)n, 1);
    or_acc a;
    acc_init(&a, n, max_degree(g));
    for (int v = 0; v < n; ++v) { label[v] = v; cw[v] = (uint32_t)g->vwgt[v]; }
    for (int r = 0; r < rounds; ++r)
        for (int i = 0; i < n; ++i) {
            int v = order[i];
            int b = cluster_choice(g, v, label, cw, bound, &a, seen, 0);
            cw[label[v]] -= (uint32_t)g->vwgt[v];
            cw[b] += (uint32_t)g->vwgt[v];
            label[v] = b;
        }
    /* remap_cluster_ids, size_constraint_label_propagation.cpp:207-232 */
    int* remap = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int v = 0; v < n; ++v) remap[v] = -1;
    int nc = 0;
    for (int v = 0; v < n; ++v) {
        if (remap[label[v]] < 0) remap[label[v]] = nc++;
        label[v] = remap[label[v]];
    }
    free(remap);
    acc_free(&a);
    free(cw); free(seen);
    return nc;
}

/* ------------------------------------------------------------- contraction */

static int cmp_int(const void* x, const void* y) {
    int a = *(const int*)x, b = *(const int*)y;
    return (a > b) - (a < b);
}

int or_contract(const or_graph* g, const int* label, int* cmap, int* cxadj, int* cadjncy,
                int* cadjwgt, int* cvwgt) {
    const int n = g->n;
    /* coarse ids in order of each cluster's smallest member = order of first
     * appearance, as remap_cluster_ids (size_constraint_label_propagation.cpp:
     * 207-232) and the matching leaders (random_matching.cpp:104-110) number them */
    int* cid = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int v = 0; v < n; ++v) cid[v] = -1;
    int nc = 0;
    for (int v = 0; v < n; ++v) {
        if (cid[label[v]] < 0) cid[label[v]] = nc++;
        cmap[v] = cid[label[v]];
    }
    free(cid);
    for (int c = 0; c < nc; ++c) cvwgt[c] = 0;
    for (int v = 0; v < n; ++v) cvwgt[cmap[v]] += g->vwgt[v];
    /* members of each coarse node */
    int* start = xcalloc((size_t)nc + 1, sizeof(int));
    int* mem = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int v = 0; v < n; ++v) start[cmap[v] + 1]++;
    for (int c = 0; c < nc; ++c) start[c + 1] += start[c];
    {
        int* fill = xmalloc(sizeof(int) * (size_t)(nc ? nc : 1));
        for (int c = 0; c < nc; ++c) fill[c] = start[c];
        for (int v = 0; v < n; ++v) mem[fill[cmap[v]]++] = v;
        free(fill);
    }
    /* contraction.h:60-82 / complete_boundary.h:538-556: drop edges inside a
     * coarse node, sum the weights of parallel edges.  Rows are emitted
     * sorted by target. */
    uint32_t* acc = xcalloc((size_t)nc, sizeof(uint32_t));
    char* seen = xcalloc((size_t)nc, 1);
    int* touched = xmalloc(sizeof(int) * (size_t)(nc ? nc : 1));
    int pos = 0;
    for (int c = 0; c < nc; ++c) {
        cxadj[c] = pos;
        int nt = 0;
        for (int i = start[c]; i < start[c + 1]; ++i) {
            int v = mem[i];
            for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
                int t = cmap[g->adjncy[e]];
                if (t == c) continue;
                if (!seen[t]) { seen[t] = 1; touched[nt++] = t; }
                acc[t] += (uint32_t)g->adjwgt[e];
            }
        }
        qsort(touched, (size_t)nt, sizeof(int), cmp_int);
        for (int i = 0; i < nt; ++i) {
            int t = touched[i];
            cadjncy[pos] = t;
            cadjwgt[pos] = (int)acc[t];
            ++pos;
            acc[t] = 0;
            seen[t] = 0;
        }
    }
    cxadj[nc] = pos;
    free(start); free(mem); free(acc); free(seen); free(touched);
    return nc;
}

/* ---------------------------------------------------------- LP refinement */

/* One node's choice, label_propagation_refinement.cpp:49-78: start from the
 * own block (connection counts only if the own block is within the bound,
 * :68), move to a neighbouring block with a strictly larger connection whose
 * weight stays below the bound (:67). */
static int refine_choice(const or_graph* g, int v, const int* part, const uint32_t* bw,
                         uint32_t bound, or_acc* a, char* seen, uint64_t ks_tie) {
    acc_gather(a, g, v, part, seen);
    int own = part[v];
    uint32_t cv = (uint32_t)g->vwgt[v];
    int own_ok = bw[own] <= bound;
    int best = own;
    uint32_t bestc = (own_ok && seen[own]) ? a->acc[own] : 0;
    for (int i = 0; i < a->ntouched; ++i) {
        int b = a->touched[i];
        if (b == own) continue;
        uint32_t c = a->acc[b];
        if (c == 0) continue;
        if (!((uint64_t)bw[b] + cv < bound)) continue;
        /* when the own block is infeasible bestc starts at 0 < c, so the
         * "own wins ties" rule of beats() only applies to a feasible own block */
        if (beats(c, b, bestc, best, own, ks_tie)) { best = b; bestc = c; }
    }
    acc_clear(a, seen);
    return best;
}

/* Threshold admission into capacity-limited targets: proposals carry a
 * priority class p in [0,P); classes are admitted in increasing order while
 * the cumulative weight fits into cap[b]; in the first class that does not
 * fit, only the proposal of the smallest node id is tried on its own. */
typedef struct {
    int P, nt;
    uint64_t* H;   /* nt * P */
    int* minv;     /* nt * P */
} or_admit;

static void admit_init(or_admit* A, int nt, int P) {
    A->P = P; A->nt = nt;
    A->H = xcalloc((size_t)nt * (size_t)P, sizeof(uint64_t));
    A->minv = xmalloc(sizeof(int) * (size_t)nt * (size_t)P);
    for (size_t i = 0; i < (size_t)nt * (size_t)P; ++i) A->minv[i] = INT_MAX;
}
static void admit_free(or_admit* A) { free(A->H); free(A->minv); }
static void admit_add(or_admit* A, int b, int p, int v, uint32_t w) {
    size_t i = (size_t)b * (size_t)A->P + (size_t)p;
    A->H[i] += w;
    if (v < A->minv[i]) A->minv[i] = v;
}
/* returns 1 if proposal (v,b,p,w) is admitted, given cap[b] >= 0 */
static int admit_test(const or_admit* A, int b, int p, int v, uint32_t w, int64_t cap) {
    const uint64_t* H = A->H + (size_t)b * (size_t)A->P;
    uint64_t cum = 0;
    int t = 0;
    while (t < A->P && (int64_t)(cum + H[t]) <= cap) { cum += H[t]; ++t; }
    if (p < t) return 1;
    if (p == t && A->minv[(size_t)b * (size_t)A->P + (size_t)t] == v && (int64_t)(cum + w) <= cap) return 1;
    return 0;
}
static void admit_reset(or_admit* A, int b) {
    for (int p = 0; p < A->P; ++p) {
        A->H[(size_t)b * (size_t)A->P + (size_t)p] = 0;
        A->minv[(size_t)b * (size_t)A->P + (size_t)p] = INT_MAX;
    }
}

void or_lp_refine(const or_graph* g, const or_knobs* kn, int level, uint32_t bound, int* part) {
    const int n = g->n, k = kn->k;
    uint32_t* bw = xcalloc((size_t)k, sizeof(uint32_t));
    or_block_weights(g, part, k, bw);
    char* active = xmalloc((size_t)(n ? n : 1));
    char* next_active = xcalloc((size_t)n, 1);
    int* prop = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* cls = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    char* seen = xcalloc((size_t)k, 1);
    or_acc a;
    acc_init(&a, k, max_degree(g));
    or_admit A;
    admit_init(&A, k, kn->ref_classes);
    memset(active, 1, (size_t)n);
    const uint32_t S = (uint32_t)kn->ref_subrounds;
    for (int r = 0; r < kn->ref_rounds; ++r) {
        uint64_t ks_sub = or_stream(kn->seed, TAG_RSUB, level, r);
        uint64_t ks_tie = or_stream(kn->seed, TAG_RTIE, level, r);
        uint64_t ks_prio = or_stream(kn->seed, TAG_RPRIO, level, r);
        long long moved = 0;
        memset(next_active, 0, (size_t)n);
        for (uint32_t s = 0; s < S; ++s) {
            for (int v = 0; v < n; ++v) {
                prop[v] = -1;
                if (!active[v] || or_range(or_hash(ks_sub, (uint32_t)v), S) != s) continue;
                int b = refine_choice(g, v, part, bw, bound, &a, seen, ks_tie);
                if (b != part[v]) {
                    prop[v] = b;
                    cls[v] = (int)or_range(or_hash(ks_prio, (uint32_t)v), (uint32_t)kn->ref_classes);
                    admit_add(&A, b, cls[v], v, (uint32_t)g->vwgt[v]);
                }
            }
            for (int v = 0; v < n; ++v) {
                int b = prop[v];
                if (b < 0) continue;
                int64_t cap = (int64_t)bound - 1 - (int64_t)bw[b];
                if (!admit_test(&A, b, cls[v], v, (uint32_t)g->vwgt[v], cap)) prop[v] = -2 - b;
            }
            for (int v = 0; v < n; ++v) {
                int b = prop[v];
                if (b == -1) continue;
                admit_reset(&A, b >= 0 ? b : -2 - b);
                if (b < 0) continue;
                bw[part[v]] -= (uint32_t)g->vwgt[v];
                bw[b] += (uint32_t)g->vwgt[v];
                part[v] = b;
                ++moved;
                /* label_propagation_refinement.cpp:84-92: neighbours of a moved
                 * node are visited again in the next round */
                for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) next_active[g->adjncy[e]] = 1;
            }
        }
        char* t = active; active = next_active; next_active = t;
        if (moved == 0) break;
    }
    acc_free(&a);
    admit_free(&A);
    free(bw); free(active); free(next_active); free(prop); free(cls); free(seen);
}

void or_lp_refine_seq(const or_graph* g, int k, uint32_t bound, int rounds, const int* order,
                      int* part) {
    /* label_propagation_refinement.cpp:21-98, queue semantics kept:
     * round 0 visits every node in `order`; later rounds visit, in push
     * order, the neighbours of nodes that changed block. */
    const int n = g->n;
    uint32_t* bw = xcalloc((size_t)k, sizeof(uint32_t));
    or_block_weights(g, part, k, bw);
    int* Q = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* NQ = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    char* nq_in = xcalloc((size_t)n, 1);
    char* seen = xcalloc((size_t)k, 1);
    or_acc a;
    acc_init(&a, k, max_degree(g));
    int qn = n;
    for (int i = 0; i < n; ++i) Q[i] = order[i];
    for (int r = 0; r < rounds; ++r) {
        int nqn = 0;
        for (int i = 0; i < qn; ++i) {
            int v = Q[i];
            int b = refine_choice(g, v, part, bw, bound, &a, seen, 0);
            int changed = b != part[v];
            bw[part[v]] -= (uint32_t)g->vwgt[v];
            bw[b] += (uint32_t)g->vwgt[v];
            part[v] = b;
            if (changed)
                for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
                    int u = g->adjncy[e];
                    if (!nq_in[u]) { nq_in[u] = 1; NQ[nqn++] = u; }
                }
        }
        int* t = Q; Q = NQ; NQ = t;
        qn = nqn;
        for (int i = 0; i < qn; ++i) nq_in[Q[i]] = 0;
    }
    acc_free(&a);
    free(bw); free(Q); free(NQ); free(nq_in); free(seen);
}

/* --------------------------------------------------------- balance repair */

static int loss_bucket(int64_t loss) {
    if (loss <= 0) return 0;
    int b = 1;
    while (b < 31 && (loss >> b) > 0) ++b; /* b = 1 + floor(log2 loss) */
    return b;
}

int or_balance(const or_graph* g, const or_knobs* kn, int level, uint32_t bound, int* part) {
    const int n = g->n, k = kn->k;
    uint32_t* bw = xcalloc((size_t)k, sizeof(uint32_t));
    int* tgt = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* cls = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    uint64_t* HS = xcalloc((size_t)k * BAL_CLASSES, sizeof(uint64_t));
    int* thr = xmalloc(sizeof(int) * (size_t)k);
    char* seen = xcalloc((size_t)k, 1);
    or_acc a;
    acc_init(&a, k, max_degree(g));
    or_admit A;
    admit_init(&A, k, kn->ref_classes);
    int ok = 0;
    for (int it = 0; it < kn->bal_iters; ++it) {
        or_block_weights(g, part, k, bw);
        int over = 0, lightest = 0;
        for (int b = 0; b < k; ++b) {
            if (bw[b] > bound) over = 1;
            if (bw[b] < bw[lightest]) lightest = b;
        }
        if (!over) { ok = 1; break; }
        uint64_t ks_tie = or_stream(kn->seed, TAG_BTIE, level, it);
        uint64_t ks_cls = or_stream(kn->seed, TAG_BCLS, level, it);
        uint64_t ks_prio = or_stream(kn->seed, TAG_BPRIO, level, it);
        /* 1. every node of an overloaded block picks the best target that can
         *    take it: the most connected feasible neighbouring block, else the
         *    lightest block */
        for (int v = 0; v < n; ++v) {
            tgt[v] = -1;
            int own = part[v];
            if (bw[own] <= bound) continue;
            uint32_t cv = (uint32_t)g->vwgt[v];
            acc_gather(&a, g, v, part, seen);
            int t = -1;
            uint32_t tc = 0;
            for (int i = 0; i < a.ntouched; ++i) {
                int b = a.touched[i];
                if (b == own) continue;
                if ((uint64_t)bw[b] + cv > bound) continue;
                uint32_t c = a.acc[b];
                int better;
                if (t < 0) better = 1;
                else if (c != tc) better = c > tc;
                else {
                    uint32_t hb = or_hash(ks_tie, (uint32_t)b), ht = or_hash(ks_tie, (uint32_t)t);
                    better = hb != ht ? hb < ht : b < t;
                }
                if (better) { t = b; tc = c; }
            }
            if (t < 0 && lightest != own && (uint64_t)bw[lightest] + cv <= bound) { t = lightest; tc = 0; }
            uint32_t cown = seen[own] ? a.acc[own] : 0;
            acc_clear(&a, seen);
            if (t < 0) continue;
            int64_t loss = (int64_t)cown - (int64_t)tc;
            tgt[v] = t;
            cls[v] = loss_bucket(loss) * 8 + (int)or_range(or_hash(ks_cls, (uint32_t)v), 8u);
            HS[(size_t)own * BAL_CLASSES + (size_t)cls[v]] += cv;
        }
        /* 2. each overloaded block releases its cheapest classes until the
         *    released weight covers its excess */
        for (int b = 0; b < k; ++b) {
            thr[b] = 0;
            if (bw[b] <= bound) continue;
            uint64_t excess = bw[b] - bound, cum = 0;
            int t = 0;
            while (t < BAL_CLASSES && cum < excess) { cum += HS[(size_t)b * BAL_CLASSES + (size_t)t]; ++t; }
            thr[b] = t;
        }
        /* 3. released nodes are admitted into their targets by priority class */
        for (int v = 0; v < n; ++v) {
            if (tgt[v] < 0) continue;
            if (cls[v] >= thr[part[v]]) { tgt[v] = -1; continue; }
            cls[v] = (int)or_range(or_hash(ks_prio, (uint32_t)v), (uint32_t)kn->ref_classes);
            admit_add(&A, tgt[v], cls[v], v, (uint32_t)g->vwgt[v]);
        }
        for (int v = 0; v < n; ++v) {
            int t = tgt[v];
            if (t < 0) continue;
            int64_t cap = (int64_t)bound - (int64_t)bw[t];
            if (!admit_test(&A, t, cls[v], v, (uint32_t)g->vwgt[v], cap)) tgt[v] = -2 - t;
        }
        for (int v = 0; v < n; ++v) {
            int t = tgt[v];
            if (t == -1) continue;
            admit_reset(&A, t >= 0 ? t : -2 - t);
            if (t < 0) continue;
            part[v] = t;
        }
        memset(HS, 0, sizeof(uint64_t) * (size_t)k * BAL_CLASSES);
    }
    if (!ok) {
        or_block_weights(g, part, k, bw);
        ok = 1;
        for (int b = 0; b < k; ++b) if (bw[b] > bound) ok = 0;
    }
    acc_free(&a);
    admit_free(&A);
    free(bw); free(tgt); free(cls); free(HS); free(thr); free(seen);
    return ok;
}

/* ------------------------------------------------------------ Jet refinement */

static uint64_t overload_of(const uint32_t* bw, int k, uint32_t bound) {
    uint64_t o = 0;
    for (int b = 0; b < k; ++b) if (bw[b] > bound) o += bw[b] - bound;
    return o;
}

/* Jet refinement (Gilbert, Madduri, Boman, Rajamanickam, "Jet: Multilevel
 * Graph Partitioning on GPUs", 2023) in synchronous iterations; it stands in
 * for the reference's k-way FM (kway_graph_refinement_core.cpp:47-171):
 *   1. every vertex not moved in the previous iteration picks its most
 *      connected other block d (ties as in refinement, stream TAG_JTIE); it
 *      is a candidate when 4 (conn(d) - conn(own)) >= -c4 conn(own)
 *      (c4 = jet_c0 on level 0, jet_c above): negative gains are allowed;
 *   2. afterburner: a candidate's gain is recomputed with every neighbour of
 *      higher priority (larger gain, then smaller id) already in its
 *      destination; it moves if that gain is >= 0;
 *   3. moves are applied, blocks above the bound are repaired (or_balance);
 *   4. the best partition by (overload, cut) is kept; the loop ends after
 *      jet_patience iterations without a better one, an iteration without
 *      moves, or jet_iters iterations. */
void or_jet_refine(const or_graph* g, const or_knobs* kn, int level, uint32_t bound, int* part) {
    const int n = g->n, k = kn->k;
    if (n == 0) return;
    uint32_t* bw = xcalloc((size_t)k, sizeof(uint32_t));
    int* best = xmalloc(sizeof(int) * (size_t)n);
    int* dest = xmalloc(sizeof(int) * (size_t)n);
    long long* gain = xmalloc(sizeof(long long) * (size_t)n);
    int* moved_at = xmalloc(sizeof(int) * (size_t)n);
    char* keep = xmalloc((size_t)n);
    char* seen = xcalloc((size_t)k, 1);
    or_acc a;
    acc_init(&a, k, max_degree(g));
    for (int v = 0; v < n; ++v) moved_at[v] = -2;
    memcpy(best, part, sizeof(int) * (size_t)n);
    or_block_weights(g, part, k, bw);
    uint64_t best_ov = overload_of(bw, k, bound);
    long long best_cut = or_edge_cut(g, part);
    const int c4 = level == 0 ? kn->jet_c0 : kn->jet_c;
    int since = 0;
    for (int it = 0; it < kn->jet_iters; ++it) {
        const uint64_t ks_tie = or_stream(kn->seed, TAG_JTIE, level, it);
        for (int v = 0; v < n; ++v) {
            dest[v] = -1;
            if (moved_at[v] == it - 1) continue;
            acc_gather(&a, g, v, part, seen);
            const int own = part[v];
            const long long co = seen[own] ? (long long)a.acc[own] : 0;
            int d = -1;
            uint32_t dc = 0;
            for (int i = 0; i < a.ntouched; ++i) {
                int b = a.touched[i];
                if (b == own) continue;
                uint32_t c = a.acc[b];
                if (c == 0) continue;
                if (d < 0 || beats(c, b, dc, d, -1, ks_tie)) { d = b; dc = c; }
            }
            acc_clear(&a, seen);
            if (d < 0) continue;
            const long long gv = (long long)dc - co;
            if (4 * gv >= -(long long)c4 * co) { dest[v] = d; gain[v] = gv; }
        }
        long long moved = 0;
        for (int v = 0; v < n; ++v) {
            keep[v] = 0;
            if (dest[v] < 0) continue;
            long long adj = 0;
            for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
                int u = g->adjncy[e];
                int bu = part[u];
                if (dest[u] >= 0 && (gain[u] > gain[v] || (gain[u] == gain[v] && u < v))) bu = dest[u];
                if (bu == dest[v]) adj += g->adjwgt[e];
                else if (bu == part[v]) adj -= g->adjwgt[e];
            }
            keep[v] = adj >= 0;
        }
        for (int v = 0; v < n; ++v) {
            if (!keep[v]) continue;
            bw[part[v]] -= (uint32_t)g->vwgt[v];
            bw[dest[v]] += (uint32_t)g->vwgt[v];
            part[v] = dest[v];
            moved_at[v] = it;
            ++moved;
        }
        uint32_t mx = 0;
        for (int b = 0; b < k; ++b) if (bw[b] > mx) mx = bw[b];
        if (mx > bound) {
            or_balance(g, kn, level, bound, part);
            or_block_weights(g, part, k, bw);
        }
        const uint64_t ov = overload_of(bw, k, bound);
        const long long cut = or_edge_cut(g, part);
        if (ov < best_ov || (ov == best_ov && cut < best_cut)) {
            best_ov = ov;
            best_cut = cut;
            memcpy(best, part, sizeof(int) * (size_t)n);
            since = 0;
        } else {
            ++since;
        }
        if (moved == 0 || since >= kn->jet_patience) break;
    }
    memcpy(part, best, sizeof(int) * (size_t)n);
    acc_free(&a);
    free(bw); free(best); free(dest); free(gain); free(moved_at); free(keep); free(seen);
}

/* ------------------------------------------------- initial partitioning */

/* max-heap of node ids keyed by (gain desc, id asc) with position index */
typedef struct {
    int* heap;
    int* pos;
    int64_t* key;
    int size;
} or_pq;

static void pq_init(or_pq* q, int n, int64_t* key) {
    q->heap = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    q->pos = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int i = 0; i < n; ++i) q->pos[i] = -1;
    q->key = key;
    q->size = 0;
}
static void pq_free(or_pq* q) { free(q->heap); free(q->pos); }
static int pq_less(const or_pq* q, int a, int b) { /* a has lower priority than b */
    if (q->key[a] != q->key[b]) return q->key[a] < q->key[b];
    return a > b;
}
static void pq_swap(or_pq* q, int i, int j) {
    int a = q->heap[i], b = q->heap[j];
    q->heap[i] = b; q->heap[j] = a;
    q->pos[b] = i; q->pos[a] = j;
}
static void pq_up(or_pq* q, int i) {
    while (i > 0) {
        int p = (i - 1) / 2;
        if (!pq_less(q, q->heap[p], q->heap[i])) break;
        pq_swap(q, i, p);
        i = p;
    }
}
static void pq_down(or_pq* q, int i) {
    for (;;) {
        int l = 2 * i + 1, r = l + 1, m = i;
        if (l < q->size && pq_less(q, q->heap[m], q->heap[l])) m = l;
        if (r < q->size && pq_less(q, q->heap[m], q->heap[r])) m = r;
        if (m == i) break;
        pq_swap(q, i, m);
        i = m;
    }
}
static void pq_push(or_pq* q, int v) {
    q->heap[q->size] = v;
    q->pos[v] = q->size++;
    pq_up(q, q->size - 1);
}
static int pq_pop(or_pq* q) {
    int v = q->heap[0];
    q->pos[v] = -1;
    --q->size;
    if (q->size > 0) {
        q->heap[0] = q->heap[q->size];
        q->pos[q->heap[0]] = 0;
        pq_down(q, 0);
    }
    return v;
}
static void pq_update(or_pq* q, int v) { /* key[v] changed */
    int i = q->pos[v];
    pq_up(q, i);
    pq_down(q, q->pos[v]);
}
static void pq_clear(or_pq* q) {
    for (int i = 0; i < q->size; ++i) q->pos[q->heap[i]] = -1;
    q->size = 0;
}

/* last node dequeued by a BFS from s (bipartition.cpp:125-146 grows from a
 * node found by repeated BFS the same way) */
static int bfs_last(const or_graph* g, int s, int* queue, char* mark) {
    int head = 0, tail = 0, last = s;
    queue[tail++] = s;
    mark[s] = 1;
    while (head < tail) {
        int v = queue[head++];
        last = v;
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
            int u = g->adjncy[e];
            if (!mark[u]) { mark[u] = 1; queue[tail++] = u; }
        }
    }
    for (int i = 0; i < tail; ++i) mark[queue[i]] = 0;
    return last;
}

static long long cut2(const or_graph* g, const char* side) {
    long long c = 0;
    for (int v = 0; v < g->n; ++v)
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e)
            if (side[v] != side[g->adjncy[e]]) c += g->adjwgt[e];
    return c / 2;
}

typedef struct {
    int n;
    int *xadj, *adjncy, *adjwgt, *vwgt;
    int* orig; /* node id in the coarsest graph */
} or_sub;

/* Greedy graph growing of side 0 from `start` (bipartition.cpp:147-222
 * restated with a gain queue): the frontier node with the largest
 * w(v,side0) - w(v,side1) joins next; nodes that would push side 0 above
 * max0 are skipped; stops once side 0 reaches target0. */
static void grow(const or_graph* g, int start, uint64_t target0, uint64_t max0, char* side,
                 int64_t* key, or_pq* q) {
    const int n = g->n;
    memset(side, 1, (size_t)n);
    char* excl = xcalloc((size_t)n, 1);
    for (int v = 0; v < n; ++v) {
        int64_t d = 0;
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) d += g->adjwgt[e];
        key[v] = -d;
    }
    uint64_t w0 = 0;
    int next_free = 0;
    int cur = start;
    while (w0 < target0) {
        int v;
        if (cur >= 0) { v = cur; cur = -1; }
        else if (q->size > 0) v = pq_pop(q);
        else {
            while (next_free < n && (side[next_free] == 0 || excl[next_free])) ++next_free;
            if (next_free >= n) break;
            v = next_free;
        }
        if (side[v] == 0 || excl[v]) continue;
        if (w0 + (uint64_t)g->vwgt[v] > max0) { excl[v] = 1; continue; }
        side[v] = 0;
        w0 += (uint64_t)g->vwgt[v];
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
            int u = g->adjncy[e];
            if (side[u] == 0 || excl[u]) continue;
            key[u] += 2 * (int64_t)g->adjwgt[e];
            if (q->pos[u] >= 0) pq_update(q, u);
            else pq_push(q, u);
        }
    }
    pq_clear(q);
    free(excl);
}

static uint64_t overload2(const uint64_t w[2], const uint64_t maxw[2]) {
    return (w[0] > maxw[0] ? w[0] - maxw[0] : 0) + (w[1] > maxw[1] ? w[1] - maxw[1] : 0);
}

/* 2-way FM (two_way_fm.cpp restated): per pass, boundary nodes by largest
 * cut reduction (ties: smaller id), each node moves at most once, a move is
 * allowed only if the receiving side stays within maxw; afterwards roll back
 * to the best prefix by (overload, cut).  Returns the cut. */
static long long fm2(const or_graph* g, char* side, const uint64_t maxw[2], int passes,
                     int stall_limit, int64_t* key, or_pq* q) {
    const int n = g->n;
    uint64_t w[2] = {0, 0};
    for (int v = 0; v < n; ++v) w[(int)side[v]] += (uint64_t)g->vwgt[v];
    char* locked = xcalloc((size_t)n, 1);
    int* moves = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    long long cut = cut2(g, side);
    for (int pass = 0; pass < passes; ++pass) {
        for (int v = 0; v < n; ++v) {
            int64_t in = 0, out = 0;
            for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
                if (side[g->adjncy[e]] == side[v]) in += g->adjwgt[e];
                else out += g->adjwgt[e];
            }
            key[v] = out - in;
            if (out > 0) pq_push(q, v);
        }
        int nm = 0, best_len = 0, stall = 0;
        long long cur_cut = cut, best_cut = cut;
        uint64_t best_ov = overload2(w, maxw);
        while (q->size > 0 && stall < stall_limit) {
            int v = pq_pop(q);
            int from = side[v], to = 1 - from;
            if (w[to] + (uint64_t)g->vwgt[v] > maxw[to]) continue;
            side[v] = (char)to;
            w[from] -= (uint64_t)g->vwgt[v];
            w[to] += (uint64_t)g->vwgt[v];
            cur_cut -= key[v];
            locked[v] = 1;
            moves[nm++] = v;
            for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
                int u = g->adjncy[e];
                if (locked[u]) continue;
                int64_t d = 2 * (int64_t)g->adjwgt[e];
                key[u] += side[u] == to ? -d : d;
                if (q->pos[u] >= 0) pq_update(q, u);
                else pq_push(q, u);
            }
            uint64_t ov = overload2(w, maxw);
            if (ov < best_ov || (ov == best_ov && cur_cut < best_cut)) {
                best_ov = ov; best_cut = cur_cut; best_len = nm; stall = 0;
            } else {
                ++stall;
            }
        }
        pq_clear(q);
        for (int i = nm - 1; i >= best_len; --i) {
            int v = moves[i];
            int from = side[v], to = 1 - from;
            side[v] = (char)to;
            w[from] -= (uint64_t)g->vwgt[v];
            w[to] += (uint64_t)g->vwgt[v];
        }
        for (int i = 0; i < nm; ++i) locked[moves[i]] = 0;
        cut = best_cut;
        if (best_len == 0) break;
    }
    free(locked);
    free(moves);
    return cut;
}

/* bipartition.cpp:24-75: several growing tries on the coarsest graph of a
 * bisection, each followed by FM; keep the best by (overload, cut). */
static void coarsest_bisect(const or_graph* g, uint64_t t0, const uint64_t maxw[2],
                            const or_knobs* kn, int bis_key, char* best_side) {
    const int n = g->n;
    char* side = xmalloc((size_t)(n ? n : 1));
    int64_t* key = xmalloc(sizeof(int64_t) * (size_t)(n ? n : 1));
    int* queue = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    char* mark = xcalloc((size_t)n, 1);
    or_pq q;
    pq_init(&q, n, key);
    long long best_cut = LLONG_MAX;
    uint64_t best_ov = UINT64_MAX;
    for (int t = 0; t < kn->ip_tries; ++t) {
        uint64_t ks = or_stream(kn->seed, TAG_IP, bis_key, t);
        int s0 = 0;
        uint32_t hbest = UINT32_MAX;
        for (int v = 0; v < n; ++v) {
            uint32_t h = or_hash(ks, (uint32_t)v);
            if (h < hbest) { hbest = h; s0 = v; }
        }
        int s1 = bfs_last(g, s0, queue, mark);
        int start = bfs_last(g, s1, queue, mark);
        grow(g, start, t0, maxw[0], side, key, &q);
        long long c = fm2(g, side, maxw, kn->ip_fm_passes, kn->ip_fm_stall, key, &q);
        uint64_t w[2] = {0, 0};
        for (int v = 0; v < n; ++v) w[(int)side[v]] += (uint64_t)g->vwgt[v];
        uint64_t ov = overload2(w, maxw);
        if (ov < best_ov || (ov == best_ov && c < best_cut)) {
            best_ov = ov; best_cut = c;
            memcpy(best_side, side, (size_t)n);
        }
    }
    pq_free(&q);
    free(side); free(key); free(queue); free(mark);
}

typedef struct { uint32_t h; int v; } or_hv;
static int cmp_hv(const void* x, const void* y) {
    const or_hv* a = (const or_hv*)x;
    const or_hv* b = (const or_hv*)y;
    if (a->h != b->h) return a->h < b->h ? -1 : 1;
    return (a->v > b->v) - (a->v < b->v);
}

/* Sequential heavy-edge matching on the expansion*^2 rating
 * (edge_ratings.cpp:171-183, weight bound as random_matching.cpp:85-96):
 * nodes in hash order; an unmatched node takes its unmatched neighbour of
 * largest rating (ties: smaller id) with c(u)+c(v) <= maxnode. */
static void hem(const or_graph* g, uint64_t ks, uint64_t maxnode, int* match) {
    const int n = g->n;
    or_hv* ord = xmalloc(sizeof(or_hv) * (size_t)(n ? n : 1));
    for (int v = 0; v < n; ++v) { ord[v].h = or_hash(ks, (uint32_t)v); ord[v].v = v; match[v] = -1; }
    qsort(ord, (size_t)n, sizeof(or_hv), cmp_hv);
    for (int i = 0; i < n; ++i) {
        int u = ord[i].v;
        if (match[u] >= 0) continue;
        uint32_t cu = (uint32_t)g->vwgt[u];
        int best = -1;
        double br = 0;
        for (int e = g->xadj[u]; e < g->xadj[u + 1]; ++e) {
            int v = g->adjncy[e];
            if (v == u || match[v] >= 0) continue;
            uint32_t cv = (uint32_t)g->vwgt[v];
            if ((uint64_t)cu + cv > maxnode) continue;
            int w = g->adjwgt[e];
            double r = 1.0 * w * w / (uint32_t)(cu * cv);
            if (best < 0 || r > br || (r == br && v < best)) { best = v; br = r; }
        }
        if (best < 0) match[u] = u;
        else { match[u] = best; match[best] = u; }
    }
    free(ord);
}

/* Multilevel bisection (graph_partitioner.cpp:110-145 runs a full k=2
 * multilevel partitioning): coarsen by matching while the graph has more
 * than 200 nodes and shrinks by >= 1.1 (multiple_k_stop_rule with
 * num_vert_stop_factor 100, stop_rules.h:86-112; node weight bound
 * 1.5*W/200), bisect the coarsest, then FM on every level on the way up. */
static void ml_bisect(const or_graph* g, uint64_t t0, const uint64_t maxw[2], const or_knobs* kn,
                      int bis_key, char* side_out) {
    enum { MAXL = 32 };
    or_graph H[MAXL + 1];
    or_sub own[MAXL + 1];
    int* cmaps[MAXL + 1];
    H[0] = *g;
    int L = 0;
    uint64_t W = 0;
    for (int v = 0; v < g->n; ++v) W += (uint64_t)g->vwgt[v];
    uint64_t maxnode = (uint64_t)(1.5 * (double)W / 200.0);
    while (L < MAXL && H[L].n > 200) {
        const or_graph* f = &H[L];
        int* match = xmalloc(sizeof(int) * (size_t)f->n);
        hem(f, or_stream(kn->seed, TAG_IPM, bis_key, L), maxnode, match);
        int* label = xmalloc(sizeof(int) * (size_t)f->n);
        for (int v = 0; v < f->n; ++v) label[v] = match[v] < v ? match[v] : v;
        free(match);
        int fm = f->xadj[f->n];
        or_sub* s = &own[L + 1];
        s->xadj = xmalloc(sizeof(int) * (size_t)(f->n + 1));
        s->adjncy = xmalloc(sizeof(int) * (size_t)(fm ? fm : 1));
        s->adjwgt = xmalloc(sizeof(int) * (size_t)(fm ? fm : 1));
        s->vwgt = xmalloc(sizeof(int) * (size_t)f->n);
        s->orig = NULL;
        cmaps[L] = xmalloc(sizeof(int) * (size_t)f->n);
        int nc = or_contract(f, label, cmaps[L], s->xadj, s->adjncy, s->adjwgt, s->vwgt);
        free(label);
        s->n = nc;
        if (1.0 * f->n / (double)nc < 1.1) {
            free(cmaps[L]);
            free(s->xadj); free(s->adjncy); free(s->adjwgt); free(s->vwgt);
            break;
        }
        H[L + 1].n = nc; H[L + 1].xadj = s->xadj; H[L + 1].adjncy = s->adjncy;
        H[L + 1].adjwgt = s->adjwgt; H[L + 1].vwgt = s->vwgt;
        ++L;
    }
    char* side = xmalloc((size_t)(H[L].n ? H[L].n : 1));
    coarsest_bisect(&H[L], t0, maxw, kn, bis_key, side);
    int64_t* key = xmalloc(sizeof(int64_t) * (size_t)(g->n ? g->n : 1));
    or_pq q;
    pq_init(&q, g->n, key);
    for (int l = L - 1; l >= 0; --l) {
        char* fs = xmalloc((size_t)(H[l].n ? H[l].n : 1));
        for (int v = 0; v < H[l].n; ++v) fs[v] = side[cmaps[l][v]];
        free(side);
        side = fs;
        fm2(&H[l], side, maxw, kn->ip_fm_passes, kn->ip_fm_stall, key, &q);
        free(cmaps[l]);
        free(own[l + 1].xadj); free(own[l + 1].adjncy); free(own[l + 1].adjwgt); free(own[l + 1].vwgt);
    }
    pq_free(&q);
    free(key);
    memcpy(side_out, side, (size_t)g->n);
    free(side);
}


static void sub_free(or_sub* s) {
    free(s->xadj); free(s->adjncy); free(s->adjwgt); free(s->vwgt); free(s->orig);
}

/* induced subgraph of the nodes with side[v] == which, ids kept in order */
static void extract(const or_graph* g, const int* orig, const char* side, int which, or_sub* s) {
    int* nid = xmalloc(sizeof(int) * (size_t)(g->n ? g->n : 1));
    int n = 0, m = 0;
    for (int v = 0; v < g->n; ++v) nid[v] = side[v] == which ? n++ : -1;
    for (int v = 0; v < g->n; ++v)
        if (side[v] == which)
            for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) m += side[g->adjncy[e]] == which;
    s->n = n;
    s->xadj = xmalloc(sizeof(int) * (size_t)(n + 1));
    s->adjncy = xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    s->adjwgt = xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    s->vwgt = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    s->orig = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int pos = 0;
    for (int v = 0; v < g->n; ++v) {
        if (side[v] != which) continue;
        int u = nid[v];
        s->xadj[u] = pos;
        s->vwgt[u] = g->vwgt[v];
        s->orig[u] = orig[v];
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
            int t = g->adjncy[e];
            if (side[t] != which) continue;
            s->adjncy[pos] = nid[t];
            s->adjwgt[pos] = g->adjwgt[e];
            ++pos;
        }
    }
    s->xadj[n] = pos;
    free(nid);
}

static int ceil_log2(int k) {
    int l = 0;
    while ((1 << l) < k) ++l;
    return l;
}

/* Recursive bisection (graph_partitioner.cpp:110-238 restated): the left
 * half gets ceil(k/2) blocks; each side may exceed its share of the weight
 * by eps_b = (1+eps)^(1/ceil(log2 k)) - 1. */
static void rb(const or_graph* g, const int* orig, int k, int offset, const or_knobs* kn,
               int rep, uint32_t node, int* out_part) {
    if (k == 1 || g->n == 0) {
        for (int v = 0; v < g->n; ++v) out_part[orig[v]] = offset;
        return;
    }
    const int n = g->n;
    /* bisections are numbered by their position in the recursion tree (root
     * 1, children 2i and 2i+1), so both halves can be computed independently */
    int bis_key = (int)(node * 64u + (uint32_t)rep);
    int kl = (k + 1) / 2, kr = k - kl;
    uint64_t W = 0;
    for (int v = 0; v < n; ++v) W += (uint64_t)g->vwgt[v];
    uint64_t t0 = W * (uint64_t)kl / (uint64_t)k;
    uint64_t t1 = W - t0;
    double eps = kn->imbalance > 0 ? kn->imbalance : 0.0;
    /* graph_partitioner.cpp:125-133 allows 1-2% per bisection; here the
     * adaptive (1+eps)^(1/depth)-1, but at least min(eps, 1%) */
    double eb = pow(1.0 + eps, 1.0 / ceil_log2(k)) - 1.0;
    double floor_eb = eps < 0.01 ? eps : 0.01;
    if (eb < floor_eb) eb = floor_eb;
    uint64_t maxw[2] = {(uint64_t)((1.0 + eb) * (double)t0), (uint64_t)((1.0 + eb) * (double)t1)};
    char* best_side = xmalloc((size_t)n);
    ml_bisect(g, t0, maxw, kn, bis_key, best_side);
    or_sub L, R;
    extract(g, orig, best_side, 0, &L);
    extract(g, orig, best_side, 1, &R);
    free(best_side);
    or_graph gl = {L.n, L.xadj, L.adjncy, L.adjwgt, L.vwgt};
    or_graph gr = {R.n, R.xadj, R.adjncy, R.adjwgt, R.vwgt};
    rb(&gl, L.orig, kl, offset, kn, rep, 2u * node, out_part);
    rb(&gr, R.orig, kr, offset + kl, kn, rep, 2u * node + 1u, out_part);
    sub_free(&L);
    sub_free(&R);
}

void or_initial_partition(const or_graph* g, const or_knobs* knobs, int* part) {
    /* initial_partitioning.cpp:66-99: several repetitions, keep the best cut */
    const int n = g->n;
    /* a dense coarsest graph (average degree > 64: skewed-degree inputs whose
     * coarsening stalls) gets one growing try and one FM pass per bisection;
     * its cut hardly depends on them and the FM's cost grows with the degree */
    or_knobs dense = *knobs;
    if ((long long)g->xadj[n] > 64LL * n) {
        dense.ip_tries = dense.ip_tries < 1 ? dense.ip_tries : 1;
        dense.ip_fm_passes = dense.ip_fm_passes < 1 ? dense.ip_fm_passes : 1;
    }
    const or_knobs* kn = &dense;
    int* orig = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* cand = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int v = 0; v < n; ++v) orig[v] = v;
    long long best = LLONG_MAX;
    for (int rep = 0; rep < kn->ip_reps; ++rep) {
        rb(g, orig, kn->k, 0, kn, rep, 1u, cand);
        long long c = or_edge_cut(g, cand);
        if (c < best) { best = c; memcpy(part, cand, sizeof(int) * (size_t)n); }
    }
    free(orig);
    free(cand);
}

/* ---------------------------- batched recursive bisection (the device's form) */

/* The device runs every bisection of one recursion depth together, one
 * thread block per block of the current partition, each on the subgraph
 * its block induces.  The recursion and its bounds are the host form's
 * (graph_partitioner.cpp:110-238 as restated in rb above): the left half
 * gets ceil(k/2) blocks, targets in proportion, per-side slack eb.  A
 * bisection runs `ip_tries` tries and keeps the best by (overload, cut),
 * the first on ties; a try:
 *   1. start: the reached node farthest from s0 by breadth-first search
 *      (bipartition.cpp:125-146 searches twice), ties to the smaller id,
 *      where s0 is the node of smallest (hash, id);
 *   2. growing (bipartition.cpp:147-222 grows by gain; here by distance):
 *      nodes in (BFS distance from the start, id) order, unreached nodes
 *      last by id; side 0 takes the order's prefix until it reaches t0 --
 *      the node that crosses t0 joins only if side 0 stays within max0;
 *   3. 2-way Jet refinement (the synchronous form of or_jet_refine with two
 *      labels and a bound per side) with a balance repair per side. */

static void bfs_dist(const or_graph* g, int s, int* dist, int* queue) {
    for (int v = 0; v < g->n; ++v) dist[v] = INT_MAX;
    int head = 0, tail = 0;
    dist[s] = 0;
    queue[tail++] = s;
    while (head < tail) {
        const int v = queue[head++];
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
            const int u = g->adjncy[e];
            if (dist[u] == INT_MAX) { dist[u] = dist[v] + 1; queue[tail++] = u; }
        }
    }
}

/* reached node of largest distance, ties to the smaller id */
static int farthest_node(const or_graph* g, const int* dist) {
    int best = 0, bd = -1;
    for (int v = 0; v < g->n; ++v)
        if (dist[v] != INT_MAX && dist[v] > bd) { bd = dist[v]; best = v; }
    return best;
}

static void grow_bfs(const or_graph* g, const int* dist, uint64_t t0, uint64_t max0, char* side) {
    const int n = g->n;
    int maxd = 0;
    for (int v = 0; v < n; ++v) if (dist[v] != INT_MAX && dist[v] > maxd) maxd = dist[v];
    /* layer of v: its distance, unreached nodes form layer maxd + 1 */
    uint64_t* lw = xcalloc((size_t)maxd + 2, sizeof(uint64_t));
    for (int v = 0; v < n; ++v) lw[dist[v] == INT_MAX ? maxd + 1 : dist[v]] += (uint64_t)g->vwgt[v];
    uint64_t cum = 0;
    int lc = 0;
    while (lc <= maxd + 1 && cum + lw[lc] < t0) cum += lw[lc++];
    for (int v = 0; v < n; ++v) {
        const int l = dist[v] == INT_MAX ? maxd + 1 : dist[v];
        side[v] = l < lc ? 0 : 1;
    }
    if (lc <= maxd + 1) {
        /* the crossing layer in id order: P = inclusive prefix weight */
        for (int v = 0; v < n; ++v) {
            const int l = dist[v] == INT_MAX ? maxd + 1 : dist[v];
            if (l != lc) continue;
            if (cum >= t0) break;
            const uint64_t p = cum + (uint64_t)g->vwgt[v];
            if (p <= max0) side[v] = 0;
            cum = p;
        }
    }
    free(lw);
}

static void side_weights(const or_graph* g, const char* side, uint64_t w[2]) {
    w[0] = w[1] = 0;
    for (int v = 0; v < g->n; ++v) w[(int)side[v]] += (uint64_t)g->vwgt[v];
}

/* connection of v to its own side (*co) and to the other side (*cx) */
static void side_conn(const or_graph* g, const char* side, int v, long long* co, long long* cx) {
    long long a = 0, b = 0;
    for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
        if (side[g->adjncy[e]] == side[v]) a += g->adjwgt[e];
        else b += g->adjwgt[e];
    }
    *co = a;
    *cx = b;
}

/* Moves nodes off side s until it is within maxw[s] (the balance repair of
 * or_balance for two labels): every node of s gets a class, log2 bucket of
 * its loss conn(own) - conn(other) times 8 hashed sub-classes; classes are
 * released in order until their weight covers the excess; released classes
 * move in order while the other side stays within its bound, and in the
 * first class that does not fit whole, its nodes in id order while the
 * running weight fits. */
static void balance2(const or_graph* g, char* side, int s, const uint64_t maxw[2], uint64_t ks_cls, int iters) {
    const int n = g->n;
    int* cls = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int it = 0; it < iters; ++it) {
        uint64_t w[2];
        side_weights(g, side, w);
        if (w[s] <= maxw[s]) break;
        const uint64_t excess = w[s] - maxw[s];
        const uint64_t cap = maxw[1 - s] > w[1 - s] ? maxw[1 - s] - w[1 - s] : 0;
        uint64_t HS[BAL_CLASSES];
        memset(HS, 0, sizeof(HS));
        const uint64_t ks = or_mix64(ks_cls ^ (uint64_t)it);
        for (int v = 0; v < n; ++v) {
            cls[v] = -1;
            if (side[v] != s) continue;
            long long co, cx;
            side_conn(g, side, v, &co, &cx);
            cls[v] = loss_bucket(co - cx) * 8 + (int)or_range(or_hash(ks, (uint32_t)v), 8u);
            HS[cls[v]] += (uint64_t)g->vwgt[v];
        }
        int T = 0;
        uint64_t rel = 0;
        while (T < BAL_CLASSES && rel < excess) rel += HS[T++];
        /* classes [0, full) move whole; class `full` (if < T) moves by id prefix */
        int full = 0;
        uint64_t used = 0;
        while (full < T && used + HS[full] <= cap) used += HS[full++];
        uint64_t run = used;
        int moved = 0;
        for (int v = 0; v < n; ++v) {
            if (cls[v] < 0) continue;
            if (cls[v] < full) { side[v] = (char)(1 - s); ++moved; continue; }
            if (cls[v] == full && full < T) {
                run += (uint64_t)g->vwgt[v];
                if (run <= cap) { side[v] = (char)(1 - s); ++moved; }
            }
        }
        if (!moved) break;
    }
    free(cls);
}

/* 2-way Jet refinement with a bound per side (or_jet_refine for two labels,
 * c4 = jet_c, at most ip_jet_iters iterations, patience ip_jet_patience);
 * returns the cut of the best (overload, cut) state kept */
static long long jet2(const or_graph* g, char* side, const uint64_t maxw[2], const or_knobs* kn, int bis_level,
                      int bis_round) {
    const int n = g->n;
    char* best = xmalloc((size_t)(n ? n : 1));
    char* dest = xcalloc((size_t)(n ? n : 1), 1);
    char* keep = xcalloc((size_t)(n ? n : 1), 1);
    long long* gain = xmalloc(sizeof(long long) * (size_t)(n ? n : 1));
    int* moved_at = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int v = 0; v < n; ++v) moved_at[v] = -2;
    memcpy(best, side, (size_t)n);
    uint64_t w[2];
    side_weights(g, side, w);
    uint64_t best_ov = overload2(w, maxw);
    long long best_cut = cut2(g, side);
    const int c4 = kn->jet_c;
    int since = 0;
    for (int it = 0; it < kn->ip_jet_iters; ++it) {
        for (int v = 0; v < n; ++v) {
            dest[v] = 0;
            if (moved_at[v] == it - 1) continue;
            long long co, cx;
            side_conn(g, side, v, &co, &cx);
            if (cx == 0) continue;
            const long long gv = cx - co;
            if (4 * gv >= -(long long)c4 * co) { dest[v] = 1; gain[v] = gv; }
        }
        long long moved = 0;
        for (int v = 0; v < n; ++v) {
            keep[v] = 0;
            if (!dest[v]) continue;
            long long adj = 0;
            for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
                const int u = g->adjncy[e];
                int su = side[u];
                if (dest[u] && (gain[u] > gain[v] || (gain[u] == gain[v] && u < v))) su = 1 - su;
                adj += su != side[v] ? g->adjwgt[e] : -(long long)g->adjwgt[e];
            }
            keep[v] = adj >= 0;
        }
        for (int v = 0; v < n; ++v) {
            if (!keep[v]) continue;
            side[v] = (char)(1 - side[v]);
            moved_at[v] = it;
            ++moved;
        }
        const uint64_t ks_cls = or_stream(kn->seed, TAG_BCLS, bis_level, bis_round * 64 + it);
        side_weights(g, side, w);
        for (int s2 = 0; s2 < 2; ++s2)
            if (w[s2] > maxw[s2]) balance2(g, side, s2, maxw, ks_cls, kn->bal_iters);
        side_weights(g, side, w);
        const uint64_t ov = overload2(w, maxw);
        const long long cut = cut2(g, side);
        if (ov < best_ov || (ov == best_ov && cut < best_cut)) {
            best_ov = ov;
            best_cut = cut;
            memcpy(best, side, (size_t)n);
            since = 0;
        } else {
            ++since;
        }
        if (moved == 0 || since >= kn->ip_jet_patience) break;
    }
    memcpy(side, best, (size_t)n);
    free(best); free(dest); free(keep); free(gain); free(moved_at);
    return best_cut;
}

/* One bisection of the batched form; bis_level / bis_round key its hash
 * streams (the block's offset, and (repetition, depth)). */
static void batched_bisect(const or_graph* g, uint64_t t0, const uint64_t maxw[2], const or_knobs* kn,
                           int bis_level, int bis_round, char* best_side) {
    const int n = g->n;
    char* side = xmalloc((size_t)(n ? n : 1));
    int* dist = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* queue = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    long long best_cut = LLONG_MAX;
    uint64_t best_ov = UINT64_MAX;
    for (int t = 0; t < kn->ip_tries; ++t) {
        const uint64_t ks = or_stream(kn->seed, TAG_IP, bis_level, bis_round * 64 + t);
        int s0 = 0;
        uint32_t hbest = UINT32_MAX;
        for (int v = 0; v < n; ++v) {
            const uint32_t h = or_hash(ks, (uint32_t)v);
            if (h < hbest) { hbest = h; s0 = v; }
        }
        bfs_dist(g, s0, dist, queue);
        const int start = farthest_node(g, dist);
        bfs_dist(g, start, dist, queue);
        grow_bfs(g, dist, t0, maxw[0], side);
        const long long c = jet2(g, side, maxw, kn, bis_level, bis_round * 64 + t);
        uint64_t w[2];
        side_weights(g, side, w);
        const uint64_t ov = overload2(w, maxw);
        if (ov < best_ov || (ov == best_ov && c < best_cut)) {
            best_ov = ov;
            best_cut = c;
            memcpy(best_side, side, (size_t)n);
        }
    }
    free(side); free(dist); free(queue);
}

/* Every bisection of a depth sees the partition at the depth's start; a
 * block is named by its offset o (its first final block id) and still
 * splits into kb[o] blocks. */
static void rb_batched(const or_graph* g, const or_knobs* kn, int rep, int* part) {
    const int n = g->n, k = kn->k;
    int* kb = xcalloc((size_t)k, sizeof(int));
    int* kb_next = xcalloc((size_t)k, sizeof(int));
    kb[0] = k;
    for (int v = 0; v < n; ++v) part[v] = 0;
    const double eps = kn->imbalance > 0 ? kn->imbalance : 0.0;
    int* nid = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    char* all = xcalloc((size_t)(n ? n : 1), 1);
    for (int depth = 0; depth < 32; ++depth) {
        int any = 0;
        memcpy(kb_next, kb, sizeof(int) * (size_t)k);
        for (int o = 0; o < k; ++o) {
            if (kb[o] <= 1) continue;
            any = 1;
            /* the block's subgraph, ids in increasing order */
            or_sub S;
            for (int v = 0; v < n; ++v) all[v] = part[v] == o ? 0 : 1;
            int* orig = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
            for (int v = 0; v < n; ++v) orig[v] = v;
            extract(g, orig, all, 0, &S);
            free(orig);
            const int kk = kb[o], kl = (kk + 1) / 2;
            uint64_t W = 0;
            for (int v = 0; v < S.n; ++v) W += (uint64_t)S.vwgt[v];
            const uint64_t t0 = W * (uint64_t)kl / (uint64_t)kk, t1 = W - t0;
            double eb = pow(1.0 + eps, 1.0 / ceil_log2(kk)) - 1.0;
            const double floor_eb = eps < 0.01 ? eps : 0.01;
            if (eb < floor_eb) eb = floor_eb;
            const uint64_t maxw[2] = {(uint64_t)((1.0 + eb) * (double)t0), (uint64_t)((1.0 + eb) * (double)t1)};
            char* side = xcalloc((size_t)(S.n ? S.n : 1), 1);
            if (S.n > 0) {
                or_graph sg = {S.n, S.xadj, S.adjncy, S.adjwgt, S.vwgt};
                batched_bisect(&sg, t0, maxw, kn, o, rep * 32 + depth, side);
            }
            for (int i = 0; i < S.n; ++i)
                if (side[i]) part[S.orig[i]] = o + kl;
            kb_next[o] = kl;
            kb_next[o + kl] = kk - kl;
            free(side);
            sub_free(&S);
        }
        memcpy(kb, kb_next, sizeof(int) * (size_t)k);
        if (!any) break;
    }
    free(kb); free(kb_next); free(nid); free(all);
}

void or_initial_partition_batched(const or_graph* g, const or_knobs* knobs, int* part) {
    const int n = g->n;
    or_knobs dense = *knobs;
    if ((long long)g->xadj[n] > 64LL * n) dense.ip_tries = dense.ip_tries < 1 ? dense.ip_tries : 1;
    const or_knobs* kn = &dense;
    int* cand = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    long long best = LLONG_MAX;
    for (int rep = 0; rep < kn->ip_reps; ++rep) {
        rb_batched(g, kn, rep, cand);
        const long long c = or_edge_cut(g, cand);
        if (c < best) { best = c; memcpy(part, cand, sizeof(int) * (size_t)n); }
    }
    free(cand);
}

/* ------------------------------------------------------------ full call */

typedef struct {
    or_graph g;
    int *xadj, *adjncy, *adjwgt, *vwgt; /* owned copies (NULL for level 0) */
    int* cmap;                          /* fine -> coarse of this level */
} or_level;

int or_kaffpa(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
              int nparts, double imbalance, int seed, int mode, long long* edgecut, int* part,
              or_stats* stats) {
    if (n < 0 || nparts < 1 || !xadj || (n > 0 && !adjncy) || imbalance < 0) return -1;
    or_knobs kn;
    or_derive_knobs(n, vwgt, nparts, imbalance, seed, mode, &kn);
    return or_kaffpa_knobs(n, vwgt, xadj, adjcwgt, adjncy, &kn, edgecut, part, stats);
}

/* The edges of f whose ends lie in the same block of both parents; the
 * clusterings of a combine run only on these (size_constraint_label_
 * propagation.cpp:175-178: graph_allready_partitioned / combine). */
static void parents_filter(const or_graph* f, const int* p1, const int* p2, or_graph* out, int** fx, int** fa,
                           int** fw) {
    const int n = f->n, m = f->xadj[n];
    *fx = xmalloc(sizeof(int) * (size_t)(n + 1));
    *fa = xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    *fw = xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    int c = 0;
    (*fx)[0] = 0;
    for (int v = 0; v < n; ++v) {
        for (int e = f->xadj[v]; e < f->xadj[v + 1]; ++e) {
            const int u = f->adjncy[e];
            if (p1[u] != p1[v] || p2[u] != p2[v]) continue;
            (*fa)[c] = u;
            (*fw)[c] = f->adjwgt[e];
            ++c;
        }
        (*fx)[v + 1] = c;
    }
    out->n = n; out->xadj = *fx; out->adjncy = *fa; out->adjwgt = *fw; out->vwgt = f->vwgt;
}

/* (overload against bound, cut) of a partition of g */
static void part_quality(const or_graph* g, const int* part, int k, uint32_t bound, uint64_t* ov, long long* cut) {
    uint32_t* bw = xcalloc((size_t)k, sizeof(uint32_t));
    or_block_weights(g, part, k, bw);
    *ov = overload_of(bw, k, bound);
    *cut = or_edge_cut(g, part);
    free(bw);
}

/* The multilevel driver.  With parents (p1 the better partition, p2 the
 * other) it is the KaFFPaE combine: coarsening never joins nodes that lie in
 * different blocks of either parent, the coarsest graph takes p1 instead of
 * an initial partitioning, and a result worse than p1 by (overload, cut) is
 * replaced by p1 (population.cpp:189-250). */
static int kaffpa_core(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                       const or_knobs* knobs, const int* p1_in, const int* p2_in, long long* edgecut, int* part,
                       or_stats* stats) {
    if (n < 0 || !knobs || knobs->k < 1 || !xadj || (n > 0 && !adjncy)) return -1;
    if (knobs->coarsening < 0 || knobs->coarsening > 1 || knobs->refinement < 0 || knobs->refinement > 1) return -1;
    const int nparts = knobs->k;
    const int combine = p1_in != NULL;
    int* P1[64];
    int* P2[64];
    memset(P1, 0, sizeof(P1));
    memset(P2, 0, sizeof(P2));
    const int m = xadj[n];
    int* vw = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* ew = xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    for (int v = 0; v < n; ++v) vw[v] = vwgt ? vwgt[v] : 1;
    for (int e = 0; e < m; ++e) ew[e] = adjcwgt ? adjcwgt[e] : 1;
    or_knobs kn = *knobs;
    or_stats st;
    memset(&st, 0, sizeof(st));

    or_level lv[64];
    memset(lv, 0, sizeof(lv));
    lv[0].g.n = n; lv[0].g.xadj = xadj; lv[0].g.adjncy = adjncy; lv[0].g.adjwgt = ew; lv[0].g.vwgt = vw;
    int L = 0;
    /* coarsening.cpp:60-91 level loop with stop_rules.h:64-66 */
    while (L + 1 < kn.max_levels && lv[L].g.n > 0) {
        or_graph* f = &lv[L].g;
        int* label = xmalloc(sizeof(int) * (size_t)f->n);
        /* a combine clusters on the edges inside both parents' blocks and
         * never bundles isolated nodes (they may lie in different blocks) */
        or_graph flt;
        int *fx = NULL, *fa = NULL, *fw = NULL;
        if (combine) {
            if (L == 0) {
                P1[0] = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
                P2[0] = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
                memcpy(P1[0], p1_in, sizeof(int) * (size_t)n);
                memcpy(P2[0], p2_in, sizeof(int) * (size_t)n);
            }
            parents_filter(f, P1[L], P2[L], &flt, &fx, &fa, &fw);
        }
        const or_graph* cg = combine ? &flt : f;
        if (kn.coarsening == 1) {
            or_hem_match(cg, &kn, L, NULL, label);
            if (!combine) or_bundle_isolated(cg, kn.max_vertex_weight + 1u, label);
            /* a matching that removes less than 40 % of the nodes (stars,
             * skewed degrees) gives way to LP clustering for this level */
            long long nc = 0;
            for (int v = 0; v < f->n; ++v) nc += label[v] == v;
            if (5 * nc > 3 * (long long)f->n) {
                or_lp_cluster(cg, &kn, L, label);
                if (!combine) or_bundle_isolated(cg, kn.cluster_bound, label);
            }
        } else {
            or_lp_cluster(cg, &kn, L, label);
            if (!combine) or_bundle_isolated(cg, kn.cluster_bound, label);
        }
        free(fx); free(fa); free(fw);
        or_level* c = &lv[L + 1];
        lv[L].cmap = xmalloc(sizeof(int) * (size_t)f->n);
        c->xadj = xmalloc(sizeof(int) * (size_t)(f->n + 1));
        int fm = f->xadj[f->n];
        c->adjncy = xmalloc(sizeof(int) * (size_t)(fm ? fm : 1));
        c->adjwgt = xmalloc(sizeof(int) * (size_t)(fm ? fm : 1));
        c->vwgt = xmalloc(sizeof(int) * (size_t)f->n);
        int nc = or_contract(f, label, lv[L].cmap, c->xadj, c->adjncy, c->adjwgt, c->vwgt);
        free(label);
        c->g.n = nc; c->g.xadj = c->xadj; c->g.adjncy = c->adjncy; c->g.adjwgt = c->adjwgt; c->g.vwgt = c->vwgt;
        if (combine) {
            /* every coarse node lies inside one block of each parent */
            P1[L + 1] = xmalloc(sizeof(int) * (size_t)(nc ? nc : 1));
            P2[L + 1] = xmalloc(sizeof(int) * (size_t)(nc ? nc : 1));
            for (int v = 0; v < f->n; ++v) {
                P1[L + 1][lv[L].cmap[v]] = P1[L][v];
                P2[L + 1][lv[L].cmap[v]] = P2[L][v];
            }
        }
        ++L;
        if (!or_stop_continue(&kn, f->n, nc)) break;
    }
    /* initial partition of the coarsest graph */
    int* cpart = xmalloc(sizeof(int) * (size_t)(lv[L].g.n ? lv[L].g.n : 1));
    if (combine) {
        if (L == 0 && !P1[0]) { /* no level was built (n == 0 or max_levels 1) */
            P1[0] = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
            memcpy(P1[0], p1_in, sizeof(int) * (size_t)n);
        }
        memcpy(cpart, P1[L], sizeof(int) * (size_t)lv[L].g.n);
    } else {
        if (kn.ip_mode == 1) or_initial_partition_batched(&lv[L].g, &kn, cpart);
        else or_initial_partition(&lv[L].g, &kn, cpart);
    }
    st.initial_cut = or_edge_cut(&lv[L].g, cpart);
    uint32_t* bw = xcalloc((size_t)nparts, sizeof(uint32_t));
    for (int l = L; l >= 0; --l) {
        or_graph* g = &lv[l].g;
        if (l < L) {
            /* graph_hierarchy.cpp:54-58 projection */
            int* fp = xmalloc(sizeof(int) * (size_t)(g->n ? g->n : 1));
            for (int v = 0; v < g->n; ++v) fp[v] = cpart[lv[l].cmap[v]];
            free(cpart);
            cpart = fp;
        }
        uint32_t bound = l == 0 ? kn.final_bound : kn.upper_bound;
        or_block_weights(g, cpart, nparts, bw);
        uint32_t mx = 0;
        for (int b = 0; b < nparts; ++b) if (bw[b] > mx) mx = bw[b];
        if (mx > bound) or_balance(g, &kn, l, bound, cpart);
        if (kn.refinement == 1) or_jet_refine(g, &kn, l, bound, cpart);
        else or_lp_refine(g, &kn, l, bound, cpart);
        or_block_weights(g, cpart, nparts, bw);
        mx = 0;
        for (int b = 0; b < nparts; ++b) if (bw[b] > mx) mx = bw[b];
        if (l < 64) {
            st.level_n[l] = g->n;
            st.level_m[l] = g->xadj[g->n];
            st.level_cut[l] = or_edge_cut(g, cpart);
            st.level_maxbw[l] = mx;
        }
        if (l == 0) st.balanced = mx <= bound;
    }
    st.levels = L + 1;
    memcpy(part, cpart, sizeof(int) * (size_t)n);
    *edgecut = st.level_cut[0];
    if (combine) {
        uint64_t ov_r, ov_p;
        long long cut_r, cut_p;
        part_quality(&lv[0].g, part, nparts, kn.final_bound, &ov_r, &cut_r);
        part_quality(&lv[0].g, p1_in, nparts, kn.final_bound, &ov_p, &cut_p);
        if (ov_p < ov_r || (ov_p == ov_r && cut_p < cut_r)) {
            memcpy(part, p1_in, sizeof(int) * (size_t)n);
            *edgecut = cut_p;
            st.balanced = ov_p == 0;
        }
    }
    for (int l = 0; l < 64; ++l) { free(P1[l]); free(P2[l]); }
    if (stats) *stats = st;
    free(cpart);
    free(bw);
    for (int l = 0; l <= L; ++l) {
        free(lv[l].cmap);
        if (l > 0) { free(lv[l].xadj); free(lv[l].adjncy); free(lv[l].adjwgt); free(lv[l].vwgt); }
    }
    free(vw);
    free(ew);
    return 0;
}

int or_kaffpa_knobs(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                    const or_knobs* knobs, long long* edgecut, int* part, or_stats* stats) {
    return kaffpa_core(n, vwgt, xadj, adjcwgt, adjncy, knobs, NULL, NULL, edgecut, part, stats);
}

int or_kaffpa_combine(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                      const or_knobs* knobs, const int* part_a, const int* part_b, long long* edgecut, int* part,
                      or_stats* stats) {
    if (n < 0 || !knobs || knobs->k < 1 || !xadj || (n > 0 && (!adjncy || !part_a || !part_b))) return -1;
    for (int v = 0; v < n; ++v)
        if (part_a[v] < 0 || part_a[v] >= knobs->k || part_b[v] < 0 || part_b[v] >= knobs->k) return -1;
    /* the better parent by (overload, cut); part_a on ties */
    const int m = xadj[n];
    int* vw = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* ew = xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    for (int v = 0; v < n; ++v) vw[v] = vwgt ? vwgt[v] : 1;
    for (int e = 0; e < m; ++e) ew[e] = adjcwgt ? adjcwgt[e] : 1;
    or_graph g = {n, xadj, adjncy, ew, vw};
    uint64_t ova, ovb;
    long long ca, cb;
    part_quality(&g, part_a, knobs->k, knobs->final_bound, &ova, &ca);
    part_quality(&g, part_b, knobs->k, knobs->final_bound, &ovb, &cb);
    free(vw);
    free(ew);
    const int b_first = ovb < ova || (ovb == ova && cb < ca);
    return kaffpa_core(n, vwgt, xadj, adjcwgt, adjncy, knobs, b_first ? part_b : part_a, b_first ? part_a : part_b,
                       edgecut, part, stats);
}

static int kaffpa_core_combine(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                               const or_knobs* knobs, const int* part_a, const int* part_b, long long* edgecut,
                               int* part) {
    return or_kaffpa_combine(n, vwgt, xadj, adjcwgt, adjncy, knobs, part_a, part_b, edgecut, part, NULL);
}

/* ------------------------------------------------ evolutionary partitioning */

typedef struct {
    uint64_t ov;
    long long cut;
} or_obj;

static int obj_less(or_obj a, or_obj b) { return a.ov < b.ov || (a.ov == b.ov && a.cut < b.cut); }

/* directed entries whose cut status differs between two partitions (twice
 * the size of the symmetric difference of their cut-edge sets) */
static long long cut_difference(const or_graph* g, const int* a, const int* b) {
    long long d = 0;
    for (int v = 0; v < g->n; ++v)
        for (int e = g->xadj[v]; e < g->xadj[v + 1]; ++e) {
            const int u = g->adjncy[e];
            d += (a[v] != a[u]) != (b[v] != b[u]);
        }
    return d;
}

/* the better of two members by (objective, index) */
static int fitter(const or_obj* obj, int a, int b) {
    if (obj_less(obj[a], obj[b])) return a;
    if (obj_less(obj[b], obj[a])) return b;
    return a < b ? a : b;
}

static void or_evo_select(const or_obj* obj, int P, uint64_t ks, int* first, int* second) {
    const int x0 = (int)or_range(or_hash(ks, 0), (uint32_t)P), x1 = (int)or_range(or_hash(ks, 1), (uint32_t)P);
    const int x2 = (int)or_range(or_hash(ks, 2), (uint32_t)P), x3 = (int)or_range(or_hash(ks, 3), (uint32_t)P);
    const int f = fitter(obj, x0, x1);
    int s2 = fitter(obj, x2, x3);
    if (s2 == f) s2 = s2 == x2 ? x3 : x2;
    if (s2 == f) s2 = (f + 1) % P;
    *first = f;
    *second = s2;
}

int or_kaffpae(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
               const or_knobs* knobs, int population, int generations, int per_generation, long long* edgecut,
               int* part, long long* history) {
    if (n < 0 || !knobs || knobs->k < 1 || population < 1 || generations < 0 || per_generation < 1) return -1;
    const int P = population, W = per_generation, k = knobs->k;
    const int m = xadj[n];
    int* vw = xmalloc(sizeof(int) * (size_t)(n ? n : 1));
    int* ew = xmalloc(sizeof(int) * (size_t)(m ? m : 1));
    for (int v = 0; v < n; ++v) vw[v] = vwgt ? vwgt[v] : 1;
    for (int e = 0; e < m; ++e) ew[e] = adjcwgt ? adjcwgt[e] : 1;
    or_graph g = {n, xadj, adjncy, ew, vw};
    const size_t nn = (size_t)(n ? n : 1);
    int* pop = xmalloc(sizeof(int) * nn * (size_t)P);
    int* off = xmalloc(sizeof(int) * nn * (size_t)W);
    or_obj* obj = xmalloc(sizeof(or_obj) * (size_t)P);
    or_obj* oobj = xmalloc(sizeof(or_obj) * (size_t)W);
    int rc = 0;
    /* population: member i is the plain partitioner with seed + i */
    for (int i = 0; i < P && !rc; ++i) {
        or_knobs kn = *knobs;
        kn.seed = knobs->seed + i;
        long long c;
        rc = kaffpa_core(n, vwgt, xadj, adjcwgt, adjncy, &kn, NULL, NULL, &c, pop + (size_t)i * nn, NULL);
        part_quality(&g, pop + (size_t)i * nn, k, knobs->final_bound, &obj[i].ov, &obj[i].cut);
    }
    int best = 0;
    for (int i = 1; i < P; ++i) best = fitter(obj, best, i);
    if (history) history[0] = obj[best].cut;
    for (int t = 0; t < generations && !rc; ++t) {
        if (P >= 2) {
            /* every offspring of a generation reads the population at its start */
            for (int j = 0; j < W && !rc; ++j) {
                int a, b;
                or_evo_select(obj, P, or_stream(knobs->seed, TAG_EVO, t, j), &a, &b);
                or_knobs kn = *knobs;
                kn.seed = knobs->seed + P + t * W + j;
                long long c;
                rc = kaffpa_core_combine(n, vwgt, xadj, adjcwgt, adjncy, &kn, pop + (size_t)a * nn,
                                         pop + (size_t)b * nn, &c, off + (size_t)j * nn);
                part_quality(&g, off + (size_t)j * nn, k, knobs->final_bound, &oobj[j].ov, &oobj[j].cut);
            }
            /* population.cpp:120-173: an offspring worse than the worst member
             * is dropped; otherwise it replaces the member most similar to it
             * (fewest differing cut edges) among those not better than it */
            for (int j = 0; j < W && !rc; ++j) {
                int worst = 0;
                for (int i = 1; i < P; ++i)
                    if (obj_less(obj[worst], obj[i])) worst = i;
                if (obj_less(obj[worst], oobj[j])) continue;
                int pick = -1;
                long long pd = 0;
                for (int i = 0; i < P; ++i) {
                    if (obj_less(obj[i], oobj[j])) continue;
                    const long long d = cut_difference(&g, pop + (size_t)i * nn, off + (size_t)j * nn);
                    if (pick < 0 || d < pd) { pick = i; pd = d; }
                }
                memcpy(pop + (size_t)pick * nn, off + (size_t)j * nn, sizeof(int) * (size_t)n);
                obj[pick] = oobj[j];
            }
        }
        best = 0;
        for (int i = 1; i < P; ++i) best = fitter(obj, best, i);
        if (history) history[t + 1] = obj[best].cut;
    }
    if (!rc) {
        memcpy(part, pop + (size_t)best * nn, sizeof(int) * (size_t)n);
        *edgecut = obj[best].cut;
    }
    free(pop); free(off); free(obj); free(oobj); free(vw); free(ew);
    return rc;
}
