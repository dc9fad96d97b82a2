// lp.cu -- label-propagation sweeps on the device: size-constrained LP
// clustering (coarsening), LP refinement (uncoarsening) and the candidate
// selection of the exact balance repair.
//
// Rules (restated from the reference):
//   clustering  size_constraint_label_propagation.cpp:134-194
//   refinement  label_propagation_refinement.cpp:21-98
// Schedule (this library's, deterministic): synchronous sub-rounds chosen by
// a counter hash; every decision of a sub-round reads the state at its start;
// ties broken by hash(tie stream, label) then label id; moves are admitted
// into capacity-limited targets without sorting (see decide kernels).
//
// Work distribution: a warp takes 32 consecutive vertex ids, ballots which of
// them take part in this sub-round, and hands them to groups of G lanes
// (G = 8/16/32 by average degree).  A group aggregates one vertex's
// neighbourhood: degree <= G in registers (match_any + redux), degree <=
// kTable/2 in a per-group shared-memory hash table, larger degrees are
// deferred to a block-per-vertex kernel with a global-memory table.
#include "lp.cuh"
#include "prims.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <climits>
#include <vector>

namespace kb {

namespace cg = cooperative_groups;

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kThreads = 256;
constexpr int kBalClasses = 256;

enum Mode { CLUSTER = 0, REFINE = 1, BALANCE = 2 };

// A list filled by many warps without contention: warp w appends to stripe
// w % kStripes through that stripe's counter.  Every stripe has a capacity
// `cap` computed on the host from the number of warps of the producing
// kernels and the work each warp can be given.
constexpr int kStripes = 128;
struct SList {
    int* data;        // kStripes * cap entries
    unsigned* counts; // kStripes counters
    long long cap;
};

// Everything a sweep reads or writes; passed by value.
struct SweepArgs {
    int n;
    const int* __restrict__ xadj;
    const int* __restrict__ adjncy;
    const int* __restrict__ adjwgt;
    const int* __restrict__ vwgt;
    const int* __restrict__ lab;        // cluster id or block id per vertex
    const uint32_t* __restrict__ lw;    // weight per label (cluster / block)
    const uint8_t* __restrict__ active; // REFINE: vertex may move this round (null: every vertex)
    const int* vlist;                   // REFINE: sweep only these vertices (null: ids 0 .. n-1)
    const unsigned* vcount;             // their number
    uint32_t bound;
    uint32_t S, s;                      // sub-rounds, this sub-round
    uint64_t ks_sub, ks_tie, ks_prio;
    int P;                              // admission classes
    // outputs
    int* pt; int* pc;                   // per vertex: proposed target / class (-1: none)
    uint32_t* inc;                      // CLUSTER: incoming weight per target
    int* minv;                          // CLUSTER: smallest proposer per target
    uint32_t* H;                        // REFINE/BALANCE: weight per (target, class)
    int* minvP;                         // smallest proposer per (target, class)
    int* heavy; unsigned* hcount;       // deferred high-degree vertices
    SList plist;                        // vertices that proposed a move this sub-round
    int* hplist; unsigned* hpcount;     // proposals of high-degree vertices
    int singletons;                     // every label is its own vertex id and rows have
                                        // strictly increasing targets (clustering round 0)
    const uint32_t* tie;                // singletons: hash32(ks_tie, u) per vertex
    int all_fit;                        // singletons: every neighbour cluster fits (2 max c(v) < bound)
    int admit_all;                      // CLUSTER: every target takes all its proposers
                                        // (max c(v) (max degree + 1) < bound): no admission data
    int fuse_apply;                     // singletons + all_fit + admit_all, no row above kWin:
                                        // moves are applied in the sweep (nothing reads labels
                                        // or cluster weights of others in that round)
    int* label_w;                       // fuse_apply: labels, written by their own vertex
    uint32_t* cw_w;                     // fuse_apply: cluster weights
    int stash;                          // host: sweep with lane_vertex's label stash
    unsigned long long* work;           // [0] vertices, [1] edges
    int* err;                           // set when an invariant breaks
    // BALANCE
    const int* lightest;
    uint32_t* HS;                       // release weight per (own block, class)
};

__device__ __forceinline__ uint32_t table_slot(uint32_t key, int cap) {
    return (key * 0x9E3779B1u) >> (32 - __ffs(cap) + 1);
}

// Linear probing; the caller guarantees fewer distinct keys than cap/2, so
// the probe ends within cap steps.  The bound only guards against a broken
// invariant: the key is then dropped and *err is set.
__device__ __forceinline__ void table_insert(uint32_t* tk, uint32_t* tv, int cap, uint32_t key,
                                             uint32_t val, int* err) {
    uint32_t s = table_slot(key, cap);
    for (int probe = 0; probe < cap; ++probe) {
        uint32_t prev = atomicCAS(&tk[s], kEmpty, key);
        if (prev == kEmpty || prev == key) {
            atomicAdd(&tv[s], val);
            return;
        }
        s = (s + 1) & (uint32_t)(cap - 1);
    }
    atomicOr(err, 1);
}

// candidate key: larger connection first, then smaller tie hash; id breaks
// the remaining ties (smaller wins)
__device__ __forceinline__ uint64_t cand_key(uint32_t conn, uint64_t ks_tie, uint32_t label) {
    return ((uint64_t)conn << 32) | (uint32_t)~hash32(ks_tie, label);
}

__device__ __forceinline__ void better(uint64_t& k, uint32_t& id, uint64_t k2, uint32_t id2) {
    if (k2 > k || (k2 == k && id2 < id)) { k = k2; id = id2; }
}

template <int G>
__device__ __forceinline__ void group_argmax(uint64_t& k, uint32_t& id, unsigned gmask) {
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) {
        uint64_t k2 = __shfl_xor_sync(gmask, k, o);
        uint32_t i2 = __shfl_xor_sync(gmask, id, o);
        better(k, id, k2, i2);
    }
}

// Is label b (connection c) a candidate for vertex of weight cv?
template <int MODE>
__device__ __forceinline__ bool cand_ok(const SweepArgs& a, uint32_t b, uint32_t c, uint32_t cv) {
    if (MODE == BALANCE) return (uint64_t)a.lw[b] + cv <= a.bound;
    return c > 0 && (uint64_t)a.lw[b] + cv < a.bound;
}

__device__ __forceinline__ int loss_bucket(long long loss) {
    if (loss <= 0) return 0;
    int b = 1;
    while (b < 31 && (loss >> b) > 0) ++b;
    return b;
}

// Final decision for vertex v (executed by one lane).
// Returns true when v proposes a move (pt[v] = target; the caller lists v).
template <int MODE>
__device__ bool decide_emit(const SweepArgs& a, int v, uint32_t own, uint32_t cv, uint32_t conn_own,
                            uint64_t key, uint32_t id) {
    if (MODE == CLUSTER) {
        if (id == kEmpty || (uint32_t)(key >> 32) <= conn_own) return false;
        a.pt[v] = (int)id;
        if (!a.admit_all) {
            atomicAdd(&a.inc[id], cv);
            atomicMin(&a.minv[id], v);
        }
    } else if (MODE == REFINE) {
        uint32_t base = a.lw[own] <= a.bound ? conn_own : 0u;
        if (id == kEmpty || (uint32_t)(key >> 32) <= base) return false;
        int cls = (int)hash_range(hash32(a.ks_prio, (uint32_t)v), (uint32_t)a.P);
        a.pt[v] = (int)id;
        a.pc[v] = cls;
        size_t h = (size_t)id * a.P + cls;
        atomicAdd(&a.H[h], cv);
        atomicMin(&a.minvP[h], v);
    } else {  // BALANCE
        uint32_t t = id, tc = (uint32_t)(key >> 32);
        if (t == kEmpty) {
            int L = *a.lightest;
            if ((uint32_t)L == own || (uint64_t)a.lw[L] + cv > a.bound) return false;
            t = (uint32_t)L;
            tc = 0;
        }
        long long loss = (long long)conn_own - (long long)tc;
        int cls = loss_bucket(loss) * 8 + (int)hash_range(hash32(a.ks_sub, (uint32_t)v), 8u);
        a.pt[v] = (int)t;
        a.pc[v] = cls;
        atomicAdd(&a.HS[(size_t)own * kBalClasses + cls], cv);
    }
    return true;
}

__device__ __forceinline__ int warp_global_id() {
    return (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
}

// warp-aggregated append to a plain list (one atomic per warp call)
__device__ __forceinline__ void append_aggregated(bool pred, int v, int* list, unsigned* count) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) list[base + __popc(m & lanemask_lt())] = v;
}

// warp-aggregated append to this warp's stripe of a striped list
__device__ __forceinline__ void append_striped(bool pred, int v, const SList& L) {
    const int stripe = warp_global_id() % kStripes;
    append_aggregated(pred, v, L.data + (long long)stripe * L.cap, L.counts + stripe);
}

template <int MODE>
__device__ __forceinline__ bool member(const SweepArgs& a, int v) {
    if (MODE == BALANCE) return a.lw[a.lab[v]] > a.bound;
    if (MODE == REFINE && a.active && !a.active[v]) return false;
    return hash_range(hash32(a.ks_sub, (uint32_t)v), a.S) == a.s;
}

// ------------------------------------------------ chunk-cooperative path

constexpr int kWin = 128;                 // edges per window (<= 4 batches)
constexpr int kBatches = kWin / 32;
constexpr int kTab = 2 * kWin;            // table slots per warp (load <= 1/2)
constexpr unsigned long long kEmpty64 = ~0ull;
constexpr int kWarpsPerBlock = kThreads / 32;

// Labels (and weights) that lane_vertex stashes per lane: column `lane` of a
// row-major [kStash][32] array, so that lanes never share a bank.  The stash
// overlays the chunk table, which chunk_process clears before each use.
constexpr int kStashUnit = 24;  // unit edge weights: labels only
constexpr int kStashWgt = 12;   // labels, then weights

struct WarpTable {
    union {
        struct {
            unsigned long long key[kTab];  // (member lane << 32) | label
            uint32_t val[kTab];
        };
        uint32_t stash[3 * kTab];
    };
    uint16_t used[kWin];           // slots filled in the current window
    unsigned long long bkey[32];   // per member: best candidate key
    uint32_t bid[32];              // per member: best candidate label
    uint32_t cown[32];             // per member: connection to its own label
    uint32_t own[32];
    uint32_t cv[32];
    uint32_t nused;
};

__device__ __forceinline__ uint32_t slot64(unsigned long long k) {
    return (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> (64 - 8)) & (kTab - 1);  // kTab == 256
}

// Decides up to 32 vertices (lane i: vertex v when mem) with the per-warp
// shared table: the members' edges are laid back to back (warp prefix sum of
// degrees) and processed in windows of at most kWin edges; every lane takes
// one edge slot per 32-edge batch, all adjacency loads of a window are issued
// before the label gathers, (member, label) pairs are merged with a 64-bit
// match_any and summed into the table, and each member's best candidate is
// found with shared-memory atomicMax / atomicMin.  Used for the vertices
// whose neighbours carry more distinct labels than the lane path's slots.
template <int MODE>
__device__ void chunk_process(const SweepArgs& a, WarpTable& T, bool mem, int v, unsigned& wv, unsigned& we,
                              unsigned& wo) {
    const int lane = threadIdx.x & 31;
    int beg = 0, deg = 0;
    bool heavy = false;
    if (mem) {
        beg = a.xadj[v];
        deg = a.xadj[v + 1] - beg;
        if (deg > kWin) {  // high degree: block-per-vertex kernel decides it
            a.heavy[atomicAdd(a.hcount, 1u)] = v;
            deg = 0;
            heavy = true;
        } else {
            wv += 1;
            we += (unsigned)deg;
            wo += 1;
        }
        T.own[lane] = (uint32_t)a.lab[v];
        T.cv[lane] = (uint32_t)a.vwgt[v];
    }
    const bool light = mem && !heavy;
    // inclusive prefix sum of degrees over the chunk
    int incl = deg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int off = incl - deg;
    const unsigned lightmask = __ballot_sync(0xffffffffu, light);
    if (!lightmask) return;
    // the table doubles as lane_vertex's stash: clear it before use
    for (int i = lane; i < kTab; i += 32) {
        T.key[i] = kEmpty64;
        T.val[i] = 0;
    }
    __syncwarp();
    int wstart = __ffs(lightmask) - 1;
    while (wstart < 32) {
        // window: lanes [wstart, wend) whose edges fit into kWin slots
        const int base = __shfl_sync(0xffffffffu, off, wstart);
        const bool inwin = lane >= wstart && incl - base <= kWin;
        const unsigned wmask = __ballot_sync(0xffffffffu, inwin);
        const int wend = 32 - __clz(wmask);
        const int E = __shfl_sync(0xffffffffu, incl, wend - 1) - base;
        const bool wmember = light && lane >= wstart && lane < wend;
        if (wmember) {
            T.bkey[lane] = 0;
            T.bid[lane] = kEmpty;
            T.cown[lane] = 0;
        }
        // gather the window's edges: all adjacency loads, then all labels
        int own_lane[kBatches];
        int tgt[kBatches];
        uint32_t wgt[kBatches];
#pragma unroll
        for (int b = 0; b < kBatches; ++b) {
            const int q = b * 32 + lane;
            // largest window lane o with off[o] - base <= q (binary lifting)
            int o = wstart;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int c = o + step;
                const int oc = __shfl_sync(0xffffffffu, off, c < 32 ? c : 31) - base;
                if (c < wend && oc <= q) o = c;
            }
            const int ob = __shfl_sync(0xffffffffu, beg, o);
            const int oo = __shfl_sync(0xffffffffu, off, o) - base;
            own_lane[b] = o;
            tgt[b] = -1;
            wgt[b] = 0;
            if (q < E) {
                const int e = ob + (q - oo);
                tgt[b] = a.adjncy[e];
                wgt[b] = (uint32_t)a.adjwgt[e];
            }
        }
#pragma unroll
        for (int b = 0; b < kBatches; ++b)
            if (tgt[b] >= 0) tgt[b] = a.lab[tgt[b]];
#pragma unroll
        for (int b = 0; b < kBatches; ++b) {
            if (b * 32 >= E) break;
            const bool ok = tgt[b] >= 0;
            const unsigned long long key =
                ok ? (((unsigned long long)own_lane[b] << 32) | (uint32_t)tgt[b]) : kEmpty64;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            const uint32_t sum = __reduce_add_sync(peers, wgt[b]);
            if (ok && (peers & lanemask_lt()) == 0) {
                uint32_t sl = slot64(key);
                for (int probe = 0; probe < kTab; ++probe) {
                    const unsigned long long prev = atomicCAS(&T.key[sl], kEmpty64, key);
                    if (prev == kEmpty64) {
                        T.used[atomicAdd(&T.nused, 1u)] = (uint16_t)sl;
                        atomicAdd(&T.val[sl], sum);
                        break;
                    }
                    if (prev == key) {
                        atomicAdd(&T.val[sl], sum);
                        break;
                    }
                    sl = (sl + 1) & (kTab - 1);
                    if (probe == kTab - 1) atomicOr(a.err, 1);
                }
            }
            __syncwarp();
        }
        // per member: connection to its own label and the best candidate
        const uint32_t nused = T.nused;
        for (uint32_t i = lane; i < nused; i += 32) {
            const uint32_t sl = T.used[i];
            const unsigned long long k = T.key[sl];
            const int o = (int)(k >> 32);
            const uint32_t l = (uint32_t)k;
            const uint32_t c = T.val[sl];
            if (l == T.own[o]) T.cown[o] = c;
            else if (cand_ok<MODE>(a, l, c, T.cv[o])) atomicMax(&T.bkey[o], cand_key(c, a.ks_tie, l));
        }
        __syncwarp();
        for (uint32_t i = lane; i < nused; i += 32) {
            const uint32_t sl = T.used[i];
            const unsigned long long k = T.key[sl];
            const int o = (int)(k >> 32);
            const uint32_t l = (uint32_t)k;
            const uint32_t c = T.val[sl];
            if (l != T.own[o] && cand_ok<MODE>(a, l, c, T.cv[o]) && cand_key(c, a.ks_tie, l) == T.bkey[o])
                atomicMin(&T.bid[o], l);
            T.key[sl] = kEmpty64;
            T.val[sl] = 0;
        }
        __syncwarp();
        if (lane == 0) T.nused = 0;
        bool prop = false;
        if (wmember) prop = decide_emit<MODE>(a, v, T.own[lane], T.cv[lane], T.cown[lane], T.bkey[lane], T.bid[lane]);
        append_striped(prop, v, a.plist);
        __syncwarp();
        // next window starts at the first light lane at or after wend
        const unsigned rest = lightmask & (wend < 32 ? (~0u << wend) : 0u);
        wstart = rest ? __ffs(rest) - 1 : 32;
    }
}

// ------------------------------------------------------ lane-per-vertex sweep
//
// The main sweep: a warp takes 32 * kSpan consecutive vertex ids, compacts the
// members of the sub-round onto its lanes, and every lane aggregates its own
// vertex's neighbourhood in kSlots register slots (connection per label; the
// own label is kept apart), four edges at a time with all loads issued
// before use.  A vertex whose neighbours carry more distinct labels than
// slots is queued per warp and decided by chunk_process in the same kernel;
// one of degree > kWin goes to the high-degree list (heavy_kernel).

constexpr int kSlots = 6;  // 4: ~5 % of RGG rows overflow; 6: 0.6 %, fastest measured
constexpr int kSpan = 2;  // chunks of 32 ids per warp task (2 measured 3 % faster than 4)

// r-th set bit (0-based) of mask
__device__ __forceinline__ int nth_set_bit(unsigned mask, int r) {
    int lo = 0, hi = 31;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const unsigned below = mid == 31 ? mask : (mask & ((2u << mid) - 1u));
        if (__popc(below) > r) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// 0: decided (stays), 3: decided (proposes a move), 1: too many distinct
// labels for NS slots, 2: degree above kWin
template <int MODE, int NS, bool UNIT, bool STASH>
__device__ int lane_vertex(const SweepArgs& a, int v, uint32_t* st, unsigned& wv, unsigned& we) {
    const int beg = a.xadj[v], end = a.xadj[v + 1];
    if (end - beg > kWin) return 2;
    // clustering round 0 (singletons): every label is its own vertex id
    const uint32_t own = (MODE == CLUSTER && a.singletons) ? (uint32_t)v : (uint32_t)a.lab[v];
    const uint32_t cv = (uint32_t)a.vwgt[v];
    uint32_t cown = 0;
    if (MODE == CLUSTER && a.singletons && UNIT && a.all_fit) {
        // unit weights: every neighbour cluster has connection 1, so the best
        // is the neighbour of smallest (tie hash, id) -- one 64-bit minimum
        // per entry
        uint64_t bk = ~0ull;
        for (int e = beg; e < end; e += 4) {
            int u[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) u[t] = e + t < end ? a.adjncy[e + t] : -1;
            uint32_t h[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) h[t] = u[t] >= 0 ? a.tie[u[t]] : 0u;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (u[t] < 0) continue;
                if ((uint32_t)u[t] == own) { cown += 1; continue; }
                const uint64_t k = ((uint64_t)h[t] << 32) | (uint32_t)u[t];
                bk = k < bk ? k : bk;
            }
        }
        wv += 1;
        we += (unsigned)(end - beg);
        const uint32_t id = bk == ~0ull ? kEmpty : (uint32_t)bk;
        if (a.fuse_apply) {
            if (id == kEmpty || 1u <= cown) return 0;
            a.label_w[v] = (int)id;
            atomicSub(&a.cw_w[own], cv);
            atomicAdd(&a.cw_w[id], cv);
            return 0;
        }
        const uint64_t key = id == kEmpty ? 0ull : (1ull << 32);
        return decide_emit<MODE>(a, v, own, cv, cown, key, id) ? 3 : 0;
    }
    if (MODE == CLUSTER && a.singletons) {
        // label[u] == u and no target repeats: the connection to cluster u is
        // exactly w(v,u), so the best candidate is a running maximum; the
        // tie hashes come precomputed per vertex, and the size test is
        // skipped when every pair of node weights fits under the bound
        uint64_t key = 0;
        uint32_t id = kEmpty;
        for (int e = beg; e < end; e += 4) {
            int u[4];
            uint32_t w[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                u[t] = -1;
                w[t] = 0;
                if (e + t < end) {
                    u[t] = a.adjncy[e + t];
                    w[t] = UNIT ? 1u : (uint32_t)a.adjwgt[e + t];
                }
            }
            uint32_t h[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) h[t] = u[t] >= 0 ? a.tie[u[t]] : 0u;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (u[t] < 0) continue;
                const uint32_t l = (uint32_t)u[t];
                if (l == own) { cown += w[t]; continue; }
                if (a.all_fit ? w[t] > 0 : cand_ok<MODE>(a, l, w[t], cv))
                    better(key, id, ((uint64_t)w[t] << 32) | (uint32_t)~h[t], l);
            }
        }
        wv += 1;
        we += (unsigned)(end - beg);
        return decide_emit<MODE>(a, v, own, cv, cown, key, id) ? 3 : 0;
    }
    // NS register slots (label, connection); a new label enters at slot 0 and
    // shifts the others up, so slot NS-1 filled means the slots are full
    uint32_t sl[NS], sc[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) { sl[i] = kEmpty; sc[i] = 0; }
    bool overflow = false;
    auto add_label = [&](uint32_t lt, uint32_t wt) {
        bool hit = false;
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            const bool m = sl[j] == lt;
            sc[j] += m ? wt : 0u;
            hit |= m;
        }
        if (!hit) {
            overflow |= sl[NS - 1] != kEmpty;
#pragma unroll
            for (int j = NS - 1; j > 0; --j) { sl[j] = sl[j - 1]; sc[j] = sc[j - 1]; }
            sl[0] = lt;
            sc[0] = wt;
        }
    };
    // STASH: two passes -- the gather pass adds entries of the own label to
    // cown and stashes the others in shared memory, the slot pass merges the
    // stash into the slots.  Once most entries carry the own label the slot
    // search then runs over far fewer entries than the row has (without the
    // stash every lane's slot search runs whenever one lane of the warp needs
    // it).
    constexpr int kStash = UNIT ? kStashUnit : kStashWgt;
    uint32_t* const stl = st;
    uint32_t* const stw = st + kStashWgt * 32;  // weights (not UNIT)
    int ns = 0;
    auto slot_pass = [&]() {
        for (int i = 0; i < ns && !overflow; ++i) add_label(stl[i * 32], UNIT ? 1u : stw[i * 32]);
        ns = 0;
    };
    // software pipeline: the row entries of the next group of four are
    // loaded while the labels of the current group are gathered
    int un[4];
    uint32_t wn[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        un[t] = -1;
        wn[t] = 0;
        if (beg + t < end) {
            un[t] = a.adjncy[beg + t];
            wn[t] = UNIT ? 1u : (uint32_t)a.adjwgt[beg + t];
        }
    }
    for (int e = beg; e < end && !overflow; e += 4) {
        int u[4];
        uint32_t w[4], l[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            u[t] = un[t];
            w[t] = wn[t];
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) l[t] = u[t] >= 0 ? (uint32_t)a.lab[u[t]] : kEmpty;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            un[t] = -1;
            wn[t] = 0;
            if (e + 4 + t < end) {
                un[t] = a.adjncy[e + 4 + t];
                wn[t] = UNIT ? 1u : (uint32_t)a.adjwgt[e + 4 + t];
            }
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if (l[t] == kEmpty) continue;  // past the row's end (labels are < n)
            if (l[t] == own) {
                cown += w[t];
            } else if (STASH) {
                stl[ns * 32] = l[t];
                if (!UNIT) stw[ns * 32] = w[t];
                ++ns;
            } else {
                add_label(l[t], w[t]);
            }
        }
        if (STASH && ns > kStash - 4) slot_pass();  // room for the next group of four
    }
    if (STASH) slot_pass();
    if (overflow) return 1;
    wv += 1;
    we += (unsigned)(end - beg);
    // best candidate: largest connection, ties by smaller tie hash, then
    // smaller label; hashes are computed only for ties
    uint32_t ok[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) ok[i] = sl[i] != kEmpty && cand_ok<MODE>(a, sl[i], sc[i], cv);
    uint32_t bc = 0, id = kEmpty;
#pragma unroll
    for (int i = 0; i < NS; ++i) {
        if (!ok[i]) continue;
        if (id == kEmpty || sc[i] > bc) {
            bc = sc[i];
            id = sl[i];
        } else if (sc[i] == bc) {
            const uint32_t hi = hash32(a.ks_tie, sl[i]), hb = hash32(a.ks_tie, id);
            if (hi < hb || (hi == hb && sl[i] < id)) id = sl[i];
        }
    }
    // decide_emit reads the connection (upper half) of the key only
    const uint64_t key = id == kEmpty ? 0ull : ((uint64_t)bc << 32);
    return decide_emit<MODE>(a, v, own, cv, cown, key, id) ? 3 : 0;
}


template <int MODE, bool UNIT, bool STASH>
__global__ void __launch_bounds__(kThreads, 4) lane_kernel(SweepArgs a) {
    static_assert(kTab == 256, "slot64 assumes 256 slots");
    // per-warp queue of members still to be processed, so that every pass
    // over the lanes is full, and of vertices that overflowed the slots
    __shared__ int queue[kWarpsPerBlock][32 * kSpan + 32];
    __shared__ int oqueue[kWarpsPerBlock][64];
    __shared__ WarpTable tabs[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    int* q = queue[threadIdx.x >> 5];
    int* oq = oqueue[threadIdx.x >> 5];
    WarpTable& T = tabs[threadIdx.x >> 5];
    if (lane == 0) T.nused = 0;
    __syncwarp();
    int qn = 0, oqn = 0;  // warp-uniform
    // per-lane work counts (32 bits: a lane never sees more than m < 2^31 entries)
    unsigned wv = 0, we = 0, wo = 0;
    const long long span = 32LL * kSpan;
    // the swept items: vertex ids 0 .. n-1, or the entries of vlist
    const long long nitems = a.vlist ? (long long)*a.vcount : (long long)a.n;
    const long long ntasks = (nitems + span - 1) / span;
    const long long warp = ((long long)blockIdx.x * kThreads + threadIdx.x) / 32;
    const long long nwarps = (long long)gridDim.x * kThreads / 32;
    auto overflow_pass = [&]() {
        const bool mem = lane < oqn && lane < 32;
        const int v = mem ? oq[lane] : 0;
        __syncwarp();
        for (int i = lane; i + 32 < oqn; i += 32) oq[i] = oq[i + 32];
        __syncwarp();
        oqn = oqn > 32 ? oqn - 32 : 0;
        chunk_process<MODE>(a, T, mem, v, wv, we, wo);
    };
    auto pass = [&](int v) {
        int status = 0;
        if (v >= 0) status = lane_vertex<MODE, kSlots, UNIT, STASH>(a, v, T.stash + lane, wv, we);
        const unsigned om = __ballot_sync(0xffffffffu, status == 1);
        if (status == 1) oq[oqn + __popc(om & lanemask_lt())] = v;
        oqn += __popc(om);
        __syncwarp();
        append_aggregated(status == 2, v, a.heavy, a.hcount);
        append_striped(status == 3, v, a.plist);
        if (oqn >= 32) overflow_pass();
    };
    for (long long task = warp; task < ntasks; task += nwarps) {
        const long long base = task * span;
#pragma unroll
        for (int c = 0; c < kSpan; ++c) {
            const long long vv = base + c * 32 + lane;
            const bool valid = vv < nitems;
            const int v = valid ? (a.vlist ? a.vlist[vv] : (int)vv) : 0;
            const bool mem = valid && member<MODE>(a, v);
            const unsigned m = __ballot_sync(0xffffffffu, mem);
            if (mem) q[qn + __popc(m & lanemask_lt())] = v;
            qn += __popc(m);
        }
        __syncwarp();
        while (qn >= 32) {
            const int v = q[lane];
            __syncwarp();
            for (int i = lane; i + 32 < qn; i += 32) q[i] = q[i + 32];
            __syncwarp();
            qn -= 32;
            pass(v);
        }
    }
    if (qn > 0) pass(lane < qn ? q[lane] : -1);
    while (oqn > 0) overflow_pass();
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        wv += __shfl_xor_sync(0xffffffffu, wv, o);
        we += __shfl_xor_sync(0xffffffffu, we, o);
        wo += __shfl_xor_sync(0xffffffffu, wo, o);
    }
    if (lane == 0 && (wv | we)) {
        atomicAdd(&a.work[0], (unsigned long long)wv);
        atomicAdd(&a.work[1], (unsigned long long)we);
        if (wo) atomicAdd(&a.work[2], (unsigned long long)wo);
    }
}

// High-degree vertices: one block per vertex.  Its connections aggregate in
// a hash table in shared memory (rows up to kSmemTab / 2 entries) or, for
// longer rows, in the block's global-memory table of `gcap` slots
// (gcap >= 2 * maxdeg, power of two; gtk may be null when every row fits
// the shared table).
constexpr int kSmemTab = 4096;

// BT threads per block (more for the longest rows).
// `which`: 0 = every listed vertex, 1 = only those whose table fits in
// shared memory, 2 = only the others (the two kinds can run as separate
// launches with different grids; the decisions do not depend on the order).
// The shared-memory table (stab slots, a power of two, keys then values) is
// dynamic shared memory: kSmemTab slots in the many-block launches, more in
// the launch of the longest rows, whose rows up to stab / 2 entries then
// stay out of the global table.
template <int MODE, int BT>
__global__ void __launch_bounds__(BT) heavy_kernel(SweepArgs a, uint32_t* gtk, uint32_t* gtv, int gcap, int which,
                                                   int stab) {
    __shared__ uint64_t sk[BT / 32];
    __shared__ uint32_t sid[BT / 32];
    __shared__ uint32_t sco;
    extern __shared__ uint32_t htab[];
    uint32_t* stk = htab;
    uint32_t* stv = htab + stab;
    for (int s = threadIdx.x; s < stab; s += BT) {
        stk[s] = kEmpty;
        stv[s] = 0;
    }
    __syncthreads();
    uint32_t* gk = gtk ? gtk + (size_t)blockIdx.x * gcap : nullptr;
    uint32_t* gv = gtv ? gtv + (size_t)blockIdx.x * gcap : nullptr;
    const unsigned count = *a.hcount;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (unsigned i = blockIdx.x; i < count; i += gridDim.x) {
        const int v = a.heavy[i];
        const int beg = a.xadj[v], end = a.xadj[v + 1];
        const uint32_t own = (uint32_t)a.lab[v];
        const uint32_t cv = (uint32_t)a.vwgt[v];
        // this vertex uses the first cap entries of the block's table (a
        // power of two >= 2 * degree, at most gcap), so inserting, scanning
        // and clearing cost O(degree), not O(max degree)
        int cap = 256;
        while (cap < 2 * (end - beg) && cap < gcap) cap <<= 1;
        if ((which == 1 && cap > kSmemTab) || (which == 2 && cap <= kSmemTab)) continue;
        uint32_t* tk = cap <= stab ? stk : gk;
        uint32_t* tv = cap <= stab ? stv : gv;
        if (threadIdx.x == 0) {
            sco = 0;
            atomicAdd(&a.work[0], 1ull);
            atomicAdd(&a.work[1], (unsigned long long)(end - beg));
        }
        for (int c = beg; c < end; c += BT) {
            int e = c + threadIdx.x;
            uint32_t l = kEmpty, wt = 0;
            if (e < end) {
                wt = (uint32_t)a.adjwgt[e];
                l = (uint32_t)a.lab[a.adjncy[e]];
            }
            unsigned peers = __match_any_sync(0xffffffffu, l);
            uint32_t sum = __reduce_add_sync(peers, wt);
            if (e < end && (peers & lanemask_lt()) == 0) table_insert(tk, tv, cap, l, sum, a.err);
        }
        __syncthreads();
        uint64_t key = 0;
        uint32_t id = kEmpty;
        for (int s = threadIdx.x; s < cap; s += BT) {
            uint32_t l = tk[s];
            if (l == kEmpty) continue;
            uint32_t c = tv[s];
            tk[s] = kEmpty;
            tv[s] = 0;
            if (l == own) sco = c;
            else if (cand_ok<MODE>(a, l, c, cv)) better(key, id, cand_key(c, a.ks_tie, l), l);
        }
        group_argmax<32>(key, id, 0xffffffffu);
        if (lane == 0) { sk[w] = key; sid[w] = id; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int j = 1; j < BT / 32; ++j) better(key, id, sk[j], sid[j]);
            if (decide_emit<MODE>(a, v, own, cv, sco, key, id)) a.hplist[atomicAdd(a.hpcount, 1u)] = v;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- admission

// Iterates the proposals of a sub-round: the stripes of the lane/chunk list
// plus the high-degree list (treated as stripe kStripes).  Blocks take
// stripes round-robin; the threads of the blocks sharing a stripe stride over
// its entries.  The body's `continue` moves on to the next proposal.
// The grid must be a multiple of kStripes + 1 blocks (admit_blocks()).
#define FOR_EACH_PROPOSAL(pl, hpl, hpc, v)                                                              \
    for (unsigned s_ = blockIdx.x % (kStripes + 1), G_ = gridDim.x / (kStripes + 1),                   \
                  i_ = (blockIdx.x / (kStripes + 1)) * blockDim.x + threadIdx.x,                       \
                  n_ = s_ < kStripes ? (pl).counts[s_] : *(hpc);                                       \
         i_ < n_; i_ += G_ * blockDim.x)                                                               \
        for (int v = s_ < kStripes ? (pl).data[(long long)s_ * (pl).cap + i_] : (hpl)[i_], once_ = 1;     \
             once_; once_ = 0)

// Proposal encoding per vertex: pt[v] = target (>= 0), -1 = no proposal,
// -2 - target = rejected (its accumulators still need resetting).

// Clustering: all proposals into b are admitted if they fit together;
// otherwise only the smallest proposer (which fits by itself).
__global__ void cluster_decide(SList pl, const int* hpl, const unsigned* hpc, int* pt, const uint32_t* cw,
                               const uint32_t* inc, const int* minv, uint32_t bound) {
    FOR_EACH_PROPOSAL(pl, hpl, hpc, v) {
        int b = pt[v];
        if (b < 0) continue;
        bool ok = ((uint64_t)cw[b] + inc[b] < bound) || minv[b] == v;
        if (!ok) pt[v] = -2 - b;
    }
}

// reset = 0: no admission data was gathered (every proposal is admitted)
__global__ void cluster_apply(SList pl, const int* hpl, const unsigned* hpc, const int* pt, const int* vwgt,
                              int* label, uint32_t* cw, uint32_t* inc, int* minv, int reset) {
    FOR_EACH_PROPOSAL(pl, hpl, hpc, v) {
        int t = pt[v];
        if (t == -1) continue;
        int b = t >= 0 ? t : -2 - t;
        if (reset) {
            inc[b] = 0;
            minv[b] = INT_MAX;
        }
        if (t < 0) continue;
        uint32_t cv = (uint32_t)vwgt[v];
        atomicSub(&cw[label[v]], cv);
        atomicAdd(&cw[t], cv);
        label[v] = t;
    }
}

// Threshold admission: classes of target b are admitted in increasing order
// while the cumulative weight stays <= cap(b); in the first class that does
// not fit, only its smallest proposer is tried alone.
__device__ __forceinline__ bool admit(const uint32_t* H, const int* minvP, int P, int b, int c, int v,
                                      uint32_t cv, long long cap) {
    const uint32_t* h = H + (size_t)b * P;
    unsigned long long cum = 0;
    int t = 0;
    while (t < P && (long long)(cum + h[t]) <= cap) { cum += h[t]; ++t; }
    if (c < t) return true;
    return c == t && minvP[(size_t)b * P + t] == v && (long long)(cum + cv) <= cap;
}

// strict: cap = bound - 1 - w[b] (refinement keeps blocks < bound);
// otherwise cap = bound - w[b] (balance repair fills up to bound)
__global__ void class_decide(SList pl, const int* hpl, const unsigned* hpc, int* pt, const int* pc,
                             const int* vwgt, const uint32_t* bw, const uint32_t* H, const int* minvP, int P,
                             uint32_t bound, int strict) {
    FOR_EACH_PROPOSAL(pl, hpl, hpc, v) {
        int b = pt[v];
        if (b < 0) continue;
        int c = pc[v];
        if (c < 0) continue;
        long long cap = (long long)bound - (strict ? 1 : 0) - (long long)bw[b];
        if (!admit(H, minvP, P, b, c, v, (uint32_t)vwgt[v], cap)) pt[v] = -2 - b;
    }
}

// The vertices a refinement round sweeps next: the neighbours of the ones it
// moves, as flags (a round that moves many vertices) or as a list in which
// each is listed once (the first thread to raise its stamp to this round's
// tag appends it; appends are aggregated over the coalesced lanes).
struct NextActive {
    uint8_t* flags;   // non-null: flags[u] = 1
    uint32_t* stamp;  // per vertex: the tag of the last round that listed it
    uint32_t tag;     // this round's tag, larger than every earlier one
    int* list;        // null (and no flags): nothing is kept
    unsigned* count;
    int* hubs;        // non-null: moved vertices of degree > kHubMark are listed
    unsigned* nhubs;  // here instead, for mark_hubs (a warp per vertex)
};

// (a thread marks at most this many neighbours itself: in list mode every
// mark waits for its atomic's result)
constexpr int kHubMark = 32;

// Marks (or lists) the neighbours of one moved vertex, row entries
// [e0, e1), by the threads t, t + nt, ...
__device__ __forceinline__ void mark_row(const NextActive& na, const int* adjncy, int e0, int e1, int t, int nt) {
    if (na.flags) {
        for (int e = e0 + t; e < e1; e += nt) na.flags[adjncy[e]] = 1;
    } else if (na.list) {
        for (int e = e0 + t; e < e1; e += nt) {
            const int u = adjncy[e];
            if (atomicMax(&na.stamp[u], na.tag) < na.tag) {
                cg::coalesced_group g = cg::coalesced_threads();
                unsigned at = 0;
                if (g.thread_rank() == 0) at = atomicAdd(na.count, g.size());
                at = g.shfl(at, 0);
                na.list[at + g.thread_rank()] = u;
            }
        }
    }
}

__global__ void class_apply(SList pl, const int* hpl, const unsigned* hpc, const int* pt, const int* pc,
                            const int* xadj, const int* adjncy, const int* vwgt, int* part, uint32_t* bw,
                            uint32_t* H, int* minvP, int P, NextActive na, unsigned* moved) {
    unsigned mv = 0;
    FOR_EACH_PROPOSAL(pl, hpl, hpc, v) {
        int t = pt[v];
        if (t == -1) continue;
        int c = pc[v];
        if (c < 0) continue;  // dropped before admission (balance)
        int b = t >= 0 ? t : -2 - t;
        H[(size_t)b * P + c] = 0;
        minvP[(size_t)b * P + c] = INT_MAX;
        if (t < 0) continue;
        uint32_t cv = (uint32_t)vwgt[v];
        atomicSub(&bw[part[v]], cv);
        atomicAdd(&bw[t], cv);
        part[v] = t;
        ++mv;
        if (!na.flags && !na.list) continue;
        // a longer row is marked by a whole warp later (mark_hubs), not by
        // this one thread
        const int e0 = xadj[v], e1 = xadj[v + 1];
        if (na.hubs && e1 - e0 > kHubMark) na.hubs[atomicAdd(na.nhubs, 1u)] = v;
        else mark_row(na, adjncy, e0, e1, 0, 1);
    }
    mv = __reduce_add_sync(0xffffffffu, mv);
    if ((threadIdx.x & 31) == 0 && mv) atomicAdd(moved, mv);
}

// the neighbours of the listed moved vertices with long rows, a warp each
__global__ void mark_hubs(NextActive na, const int* xadj, const int* adjncy) {
    const unsigned n = *na.nhubs;
    const unsigned w = (blockIdx.x * blockDim.x + threadIdx.x) / 32, nw = gridDim.x * blockDim.x / 32;
    for (unsigned i = w; i < n; i += nw) {
        const int v = na.hubs[i];
        mark_row(na, adjncy, xadj[v], xadj[v + 1], (int)(threadIdx.x & 31), 32);
    }
}

// Balance: per overloaded block, the release threshold class.
__global__ void balance_threshold(const uint32_t* bw, const uint32_t* HS, int k, uint32_t bound,
                                  int* thr) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= k) return;
    int t = 0;
    if (bw[b] > bound) {
        unsigned long long excess = bw[b] - bound, cum = 0;
        while (t < kBalClasses && cum < excess) { cum += HS[(size_t)b * kBalClasses + t]; ++t; }
    }
    thr[b] = t;
}

// Balance: released candidates get an admission class; others are dropped.
__global__ void balance_release(SList pl, const int* hpl, const unsigned* hpc, const int* pt, int* pc,
                                const int* part, const int* vwgt, const int* thr, uint32_t* H, int* minvP, int P,
                                uint64_t ks_prio) {
    FOR_EACH_PROPOSAL(pl, hpl, hpc, v) {
        int t = pt[v];
        if (t < 0) continue;
        if (pc[v] >= thr[part[v]]) { pc[v] = -1; continue; }
        int c = (int)hash_range(hash32(ks_prio, (uint32_t)v), (uint32_t)P);
        pc[v] = c;
        size_t h = (size_t)t * P + c;
        atomicAdd(&H[h], (uint32_t)vwgt[v]);
        atomicMin(&minvP[h], v);
    }
}

// lightest block (ties: smaller id) and whether any block exceeds bound
// (skip != nullptr and *skip != 0: report no overload, the caller is done)
__global__ void block_scan_kernel(const uint32_t* bw, int k, uint32_t bound, int* lightest,
                                  int* over, const int* skip) {
    if (skip && *skip) {
        if (threadIdx.x == 0) {
            *lightest = 0;
            *over = 0;
        }
        return;
    }
    __shared__ unsigned long long best[32];
    __shared__ int ov[32];
    unsigned long long mine = ~0ull;
    int o = 0;
    for (int b = threadIdx.x; b < k; b += blockDim.x) {
        unsigned long long key = ((unsigned long long)bw[b] << 32) | (unsigned)b;
        if (key < mine) mine = key;
        if (bw[b] > bound) o = 1;
    }
    for (int s = 16; s >= 1; s >>= 1) {
        unsigned long long x = __shfl_xor_sync(0xffffffffu, mine, s);
        if (x < mine) mine = x;
        o |= __shfl_xor_sync(0xffffffffu, o, s);
    }
    if ((threadIdx.x & 31) == 0) { best[threadIdx.x >> 5] = mine; ov[threadIdx.x >> 5] = o; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            if (best[w] < mine) mine = best[w];
            o |= ov[w];
        }
        *lightest = (int)(mine & 0xffffffffu);
        *over = o;
    }
}

// ------------------------------------------------------------- host helpers

struct SweepBuffers {
    int *pt, *pc;
    unsigned* counters;  // [0, kStripes) unused, [kStripes, 2 kStripes) proposals,
                         // [2 kStripes] heavy, [+1] heavy proposals, [+2] moved
    int* heavy;
    int* hplist;
    SList plist;
    int lblocks;
    uint32_t *gtk, *gtv;
    int gcap, hblocks;
    unsigned long long* work;
    int* err;
};

constexpr int kCntHeavy = 2 * kStripes, kCntHeavyProp = 2 * kStripes + 1, kCntMoved = 2 * kStripes + 2;

int admit_blocks() { return (kStripes + 1) * 4; }

SweepBuffers make_buffers(Ctx& ctx, const DevGraph& g) {
    SweepBuffers b;
    Arena& A = ctx.scratch;
    const long long n = std::max(g.n, 1);
    b.pt = A.alloc<int>((size_t)n);
    b.pc = A.alloc<int>((size_t)n);
    b.heavy = A.alloc<int>((size_t)n);
    b.hplist = A.alloc<int>((size_t)n);
    b.counters = A.alloc<unsigned>(2 * kStripes + 8);
    // stripe capacities from the producers' warp counts and per-warp work
    const long long tasks = (n + 32 * kSpan - 1) / (32 * kSpan);
    // one wave: 64 registers and 37 KB of shared memory per 256-thread
    // block leave room for 4 blocks per SM
    b.lblocks = (int)std::max<long long>(1, std::min<long long>(div_up(tasks, kWarpsPerBlock), kNumSMs * 4LL));
    const long long wl = (long long)b.lblocks * kWarpsPerBlock;
    const long long cap_l = ((wl + kStripes - 1) / kStripes) * ((tasks + wl - 1) / wl) * 32 * kSpan;
    b.plist = SList{A.alloc<int>((size_t)(kStripes * cap_l)), b.counters + kStripes, cap_l};
    b.work = ctx.work;
    b.err = ctx.dscalars + 60;
    b.gcap = 0;
    b.hblocks = 0;
    b.gtk = b.gtv = nullptr;
    if (g.maxdeg > kWin) {
        int cap = 1;
        while (cap < 2 * g.maxdeg) cap <<= 1;
        b.gcap = cap;
        if (cap <= kSmemTab) {
            // every row fits the blocks' shared-memory tables
            b.hblocks = 8 * kNumSMs;
        } else {
            // per-block global tables within min(1 GiB, 8 B per directed entry of the level)
            long long per = (long long)cap * 8;
            long long budget = std::min<long long>(1LL << 30, 8LL * g.m);
            b.hblocks = (int)std::max<long long>(1, std::min<long long>(8LL * kNumSMs, budget / per));
            b.gtk = A.alloc<uint32_t>((size_t)cap * b.hblocks);
            b.gtv = A.alloc<uint32_t>((size_t)cap * b.hblocks);
            fill_u32(b.gtk, (long long)cap * b.hblocks, kEmpty, ctx.stream);
            fill_u32(b.gtv, (long long)cap * b.hblocks, 0u, ctx.stream);
        }
    }
    return b;
}

const char* family(int mode, int part) {
    static const char* names[3][3] = {{"lp_cluster_sweep", "lp_cluster_overflow", "lp_cluster_heavy"},
                                      {"lp_refine_sweep", "lp_refine_overflow", "lp_refine_heavy"},
                                      {"balance_sweep", "balance_overflow", "balance_heavy"}};
    return names[mode][part];
}

// Shared-memory slots of the longest rows' launch: rows up to kBigTab / 2
// entries aggregate in shared memory (128 KiB of the block's), longer ones in
// the global table.  The launch needs the larger dynamic shared memory
// allowed once per device; without it the launch keeps kSmemTab slots.
constexpr int kBigTab = 16384;

template <int MODE>
bool big_tab_ok() {
    static int state[64];  // per device: 0 unknown, 1 allowed, -1 refused
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (state[dev] == 0)
        state[dev] = cudaFuncSetAttribute(heavy_kernel<MODE, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          8 * kBigTab) == cudaSuccess ? 1 : -1;
    if (state[dev] < 0) (void)cudaGetLastError();
    return state[dev] > 0;
}

template <int MODE>
void launch_sweep(Ctx& ctx, const DevGraph& g, SweepArgs a, const SweepBuffers& b, double bytes) {
    KB_CUDA(cudaMemsetAsync(b.counters, 0, sizeof(unsigned) * kCntMoved, ctx.stream));
    {
        PhaseScope ps(ctx, family(MODE, 0), bytes);
        if (a.stash) {
            if (g.unit_weights) lane_kernel<MODE, true, true><<<b.lblocks, kThreads, 0, ctx.stream>>>(a);
            else lane_kernel<MODE, false, true><<<b.lblocks, kThreads, 0, ctx.stream>>>(a);
        } else {
            if (g.unit_weights) lane_kernel<MODE, true, false><<<b.lblocks, kThreads, 0, ctx.stream>>>(a);
            else lane_kernel<MODE, false, false><<<b.lblocks, kThreads, 0, ctx.stream>>>(a);
        }
        KB_LAUNCH();
    }
    if (b.gcap > 0) {
        PhaseScope ps(ctx, family(MODE, 2), 0);
        if (b.gcap <= kSmemTab) {
            heavy_kernel<MODE, kThreads><<<b.hblocks, kThreads, 8 * kSmemTab, ctx.stream>>>(a, nullptr, nullptr, b.gcap,
                                                                                           0, kSmemTab);
            KB_LAUNCH();
        } else {
            // rows that fit the shared tables on many blocks, the longest
            // rows on the blocks that own a global table
            heavy_kernel<MODE, kThreads><<<8 * kNumSMs, kThreads, 8 * kSmemTab, ctx.stream>>>(a, nullptr, nullptr,
                                                                                              b.gcap, 1, kSmemTab);
            KB_LAUNCH();
            const int tab = big_tab_ok<MODE>() ? kBigTab : kSmemTab;
            heavy_kernel<MODE, 1024><<<b.hblocks, 1024, 8 * tab, ctx.stream>>>(a, b.gtk, b.gtv, b.gcap, 2, tab);
            KB_LAUNCH();
        }
    }
}

SweepArgs base_args(const DevGraph& g, const SweepBuffers& b) {
    SweepArgs a{};
    a.n = g.n;
    a.xadj = g.xadj;
    a.adjncy = g.adjncy;
    a.adjwgt = g.adjwgt;
    a.vwgt = g.vwgt;
    a.pt = b.pt;
    a.pc = b.pc;
    a.hcount = b.counters + kCntHeavy;
    a.heavy = b.heavy;
    a.plist = b.plist;
    a.hplist = b.hplist;
    a.hpcount = b.counters + kCntHeavyProp;
    a.work = b.work;
    a.err = b.err;
    return a;
}

double sweep_bytes(const DevGraph& g, double frac) {
    // per directed entry: adjncy + label gather (+ adjwgt unless all weights
    // are 1, then the sweep does not read it); per node: xadj, own label,
    // node weight, target weight, label write, weight update
    return frac * ((g.unit_weights ? 8.0 : 12.0) * (double)g.m + 24.0 * (double)g.n);
}

}  // namespace

// --------------------------------------------------------------- clustering

__global__ void tie_hash_kernel(int n, uint64_t ks, uint32_t* tie) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        tie[v] = hash32(ks, (uint32_t)v);
}

void lp_cluster(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, int* label) {
    const size_t mk = ctx.scratch.mark();
    cudaStream_t st = ctx.stream;
    const size_t n = (size_t)std::max(g.n, 1);
    uint32_t* cw = ctx.scratch.alloc<uint32_t>(n);
    uint32_t* inc = ctx.scratch.alloc<uint32_t>(n);
    int* minv = ctx.scratch.alloc<int>(n);
    SweepBuffers b = make_buffers(ctx, g);
    init_labels(ctx, g, label, cw);
    fill_u32(inc, g.n, 0u, st);
    fill_i32(minv, g.n, INT_MAX, st);
    SweepArgs a = base_args(g, b);
    a.lab = label;
    a.lw = cw;
    a.bound = kn.cluster_bound;
    a.S = (uint32_t)kn.lpc_subrounds;
    a.inc = inc;
    a.minv = minv;
    const bool sorted_rows = g.rows_sorted >= 0 ? g.rows_sorted == 1 : rows_strictly_increasing(ctx, g);
    for (int r = 0; r < kn.lpc_rounds; ++r) {
        a.ks_sub = stream_key(kn.seed, TAG_CSUB, level, r);
        a.ks_tie = stream_key(kn.seed, TAG_CTIE, level, r);
        // round 0 is one fully synchronous sub-round (every cluster is still a
        // single node), later rounds use lpc_subrounds sub-rounds
        a.S = r == 0 ? 1u : (uint32_t)kn.lpc_subrounds;
        // in round 0 every vertex is its own cluster; with no repeated
        // targets per row nothing needs aggregating
        a.singletons = (r == 0 && sorted_rows) ? 1 : 0;
        // from round 2 on most neighbours share the vertex's cluster: the
        // stash measured faster there, slower in round 1
        a.stash = r >= 2 ? 1 : 0;
        a.tie = nullptr;
        a.all_fit = 0;
        // round 0: a target's proposers are its neighbours, so with
        // max c(v) (max degree + 1) < bound every target takes them all
        a.admit_all = (r == 0 && (unsigned long long)g.maxvw * ((unsigned long long)g.maxdeg + 1) <
                                     (unsigned long long)a.bound) ? 1 : 0;
        if (a.singletons && g.n > 0) {
            uint32_t* tie = ctx.scratch.alloc<uint32_t>(n);
            tie_hash_kernel<<<(int)std::min<long long>(div_up(g.n, kThreads), (long long)kNumSMs * 16), kThreads, 0,
                              st>>>(g.n, a.ks_tie, tie);
            KB_LAUNCH();
            a.tie = tie;
            a.all_fit = 2ull * g.maxvw < (unsigned long long)a.bound ? 1 : 0;
        }
        // unit weights, every target fitting and taking all its proposers and
        // no row for the high-degree kernel: the sweep applies the moves itself
        a.fuse_apply = (a.singletons && a.all_fit && a.admit_all && g.unit_weights && g.maxdeg <= kWin) ? 1 : 0;
        a.label_w = label;
        a.cw_w = cw;
        for (uint32_t s = 0; s < a.S; ++s) {
            a.s = s;
            launch_sweep<CLUSTER>(ctx, g, a, b, sweep_bytes(g, 1.0 / a.S));
            if (a.fuse_apply) continue;
            PhaseScope ps(ctx, "lp_cluster_admit", 0);
            if (!a.admit_all) {
                cluster_decide<<<admit_blocks(), kThreads, 0, st>>>(b.plist, b.hplist, a.hpcount, b.pt, cw, inc, minv,
                                                                    a.bound);
                KB_LAUNCH();
            }
            cluster_apply<<<admit_blocks(), kThreads, 0, st>>>(b.plist, b.hplist, a.hpcount, b.pt, g.vwgt, label, cw,
                                                               inc, minv, a.admit_all ? 0 : 1);
            KB_LAUNCH();
        }
    }
    ctx.scratch.release(mk);
}

// --------------------------------------------------------------- refinement

void lp_refine(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, uint32_t bound, int* part,
               uint32_t* bw, const uint8_t* active0) {
    if (g.n == 0) return;
    const size_t mk = ctx.scratch.mark();
    cudaStream_t st = ctx.stream;
    const int k = kn.k, P = kn.ref_classes;
    uint32_t* H = ctx.scratch.alloc<uint32_t>((size_t)k * P);
    int* minvP = ctx.scratch.alloc<int>((size_t)k * P);
    // round 0 sweeps every vertex (or active0); round r > 0 the neighbours of
    // the vertices round r - 1 moved: as flags over all ids when many moved
    // (round 0, or a round after one that moved more than n / 64), else as a
    // list (no pass over all ids; every listing waits for an atomic)
    uint8_t* flagbuf[2] = {ctx.scratch.alloc<uint8_t>((size_t)g.n), ctx.scratch.alloc<uint8_t>((size_t)g.n)};
    uint32_t* stamp = ctx.scratch.alloc<uint32_t>((size_t)g.n);
    int* alist[2] = {ctx.scratch.alloc<int>((size_t)g.n), ctx.scratch.alloc<int>((size_t)g.n)};
    unsigned* acount = ctx.scratch.alloc<unsigned>(2);
    // moved vertices of degree > kHubMark mark their neighbours a warp each
    // (levels with rows of more than 128 entries; elsewhere the few such
    // rows cost less than the extra launches)
    int* hubs = g.maxdeg > 128 ? ctx.scratch.alloc<int>((size_t)g.n) : nullptr;
    unsigned* nhubs = hubs ? ctx.scratch.alloc<unsigned>(1) : nullptr;
    SweepBuffers b = make_buffers(ctx, g);
    fill_u32(H, (long long)k * P, 0u, st);
    fill_i32(minvP, (long long)k * P, INT_MAX, st);
    fill_u32(stamp, g.n, 0u, st);
    SweepArgs a = base_args(g, b);
    a.lab = part;
    a.lw = bw;
    a.bound = bound;
    a.S = (uint32_t)kn.ref_subrounds;
    a.P = P;
    a.H = H;
    a.minvP = minvP;
    a.stash = 1;  // most neighbours lie in the vertex's own block
    // Small levels read each round's move count one round late: round r + 1
    // is queued before the host waits for round r's count (a round after one
    // without moves sweeps an empty set), so the GPU is not idle while the
    // host reads it.  On large levels the extra round costs more than the
    // wait (measured).
    const bool late = g.n <= (1 << 18);
    unsigned* moved_r = ctx.scratch.alloc<unsigned>(2);
    cudaEvent_t counted[2] = {ctx.ev(), ctx.ev()};
    bool flags_in = false;               // this round's set came as flags
    unsigned long long moved_prev = ~0ull;  // latest move count known to the host
    for (int r = 0; r < kn.ref_rounds; ++r) {
        unsigned* moved = moved_r + (r & 1);
        a.active = r == 0 ? active0 : flags_in ? flagbuf[r & 1] : nullptr;
        a.vlist = r > 0 && !flags_in ? alist[r & 1] : nullptr;
        a.vcount = acount + (r & 1);
        const bool flags_out = moved_prev == ~0ull || moved_prev * 64 > (unsigned long long)g.n;
        uint8_t* fo = flagbuf[(r + 1) & 1];
        if (flags_out) fill_u8(fo, g.n, 0, st);
        const NextActive na{flags_out ? fo : nullptr, stamp, (uint32_t)r + 1u, alist[(r + 1) & 1],
                            acount + ((r + 1) & 1), hubs, nhubs};
        a.ks_sub = stream_key(kn.seed, TAG_RSUB, level, r);
        a.ks_tie = stream_key(kn.seed, TAG_RTIE, level, r);
        a.ks_prio = stream_key(kn.seed, TAG_RPRIO, level, r);
        KB_CUDA(cudaMemsetAsync(na.count, 0, sizeof(unsigned), st));
        KB_CUDA(cudaMemsetAsync(moved, 0, sizeof(unsigned), st));
        for (uint32_t s = 0; s < a.S; ++s) {
            a.s = s;
            launch_sweep<REFINE>(ctx, g, a, b, sweep_bytes(g, 1.0 / a.S));
            PhaseScope ps(ctx, "lp_refine_admit", 0);
            class_decide<<<admit_blocks(), kThreads, 0, st>>>(b.plist, b.hplist, a.hpcount, b.pt, b.pc, g.vwgt, bw,
                                                              H, minvP, P, bound, 1);
            KB_LAUNCH();
            if (hubs) KB_CUDA(cudaMemsetAsync(nhubs, 0, sizeof(unsigned), st));
            class_apply<<<admit_blocks(), kThreads, 0, st>>>(b.plist, b.hplist, a.hpcount, b.pt, b.pc, g.xadj,
                                                             g.adjncy, g.vwgt, part, bw, H, minvP, P, na, moved);
            KB_LAUNCH();
            if (hubs) {
                mark_hubs<<<4 * kNumSMs, kThreads, 0, st>>>(na, g.xadj, g.adjncy);
                KB_LAUNCH();
            }
        }
        // large levels wait for this round's count before queueing the next
        // (read one round late there, the queued round after the last one
        // cost more than the synchronisation it hid); small levels read it
        // one round late
        KB_CUDA(cudaMemcpyAsync(ctx.pinned + 20 + (r & 1), moved, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        flags_in = flags_out;
        if (!late) {
            KB_CUDA(cudaStreamSynchronize(st));
            if (ctx.pinned[20 + (r & 1)] == 0) break;
            moved_prev = ctx.pinned[20 + (r & 1)];
            continue;
        }
        KB_CUDA(cudaEventRecord(counted[r & 1], st));
        if (r > 0) {
            KB_CUDA(cudaEventSynchronize(counted[(r - 1) & 1]));
            const unsigned mp = ctx.pinned[20 + ((r - 1) & 1)];
            if (mp == 0) break;  // round r (queued) has nothing to sweep
            moved_prev = mp;
        }
    }
    ctx.ev_free.push_back(counted[0]);
    ctx.ev_free.push_back(counted[1]);
    ctx.scratch.release(mk);
}

// ------------------------------------------------------------------ balance

bool balance(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, uint32_t bound, int* part,
             uint32_t* bw, const int* skip, bool* moved) {
    if (moved) *moved = false;
    const size_t mk = ctx.scratch.mark();
    cudaStream_t st = ctx.stream;
    const int k = kn.k, P = kn.ref_classes;
    int* flags = ctx.scratch.alloc<int>(2);  // [0] lightest, [1] over
    // the first check before any set-up: most calls find every block within
    // the bound
    block_scan_kernel<<<1, 1024, 0, st>>>(bw, k, bound, flags, flags + 1, skip);
    KB_LAUNCH();
    KB_CUDA(cudaMemcpyAsync(ctx.pinned, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    if (ctx.pinned[0] == 0) {
        ctx.scratch.release(mk);
        return true;
    }
    if (moved) *moved = true;
    uint32_t* H = ctx.scratch.alloc<uint32_t>((size_t)k * P);
    int* minvP = ctx.scratch.alloc<int>((size_t)k * P);
    uint32_t* HS = ctx.scratch.alloc<uint32_t>((size_t)k * kBalClasses);
    int* thr = ctx.scratch.alloc<int>((size_t)k);
    SweepBuffers b = make_buffers(ctx, g);
    fill_u32(H, (long long)k * P, 0u, st);
    fill_i32(minvP, (long long)k * P, INT_MAX, st);
    SweepArgs a = base_args(g, b);
    a.lab = part;
    a.lw = bw;
    a.bound = bound;
    a.P = P;
    a.HS = HS;
    a.lightest = flags;
    a.stash = 1;
    bool ok = false;
    for (int it = 0; it < kn.bal_iters; ++it) {
        if (it > 0) {  // iteration 0's check ran above
            block_scan_kernel<<<1, 1024, 0, st>>>(bw, k, bound, flags, flags + 1, nullptr);
            KB_LAUNCH();
            KB_CUDA(cudaMemcpyAsync(ctx.pinned, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            KB_CUDA(cudaStreamSynchronize(st));
            if (ctx.pinned[0] == 0) { ok = true; break; }
        }
        PhaseScope ps(ctx, "balance", 0);
        a.ks_tie = stream_key(kn.seed, TAG_BTIE, level, it);
        a.ks_sub = stream_key(kn.seed, TAG_BCLS, level, it);  // release class stream
        uint64_t ks_prio = stream_key(kn.seed, TAG_BPRIO, level, it);
        fill_u32(HS, (long long)k * kBalClasses, 0u, st);
        launch_sweep<BALANCE>(ctx, g, a, b, 0);
        balance_threshold<<<div_up(k, 256), 256, 0, st>>>(bw, HS, k, bound, thr);
        KB_LAUNCH();
        balance_release<<<admit_blocks(), kThreads, 0, st>>>(b.plist, b.hplist, a.hpcount, b.pt, b.pc, part, g.vwgt,
                                                             thr, H, minvP, P, ks_prio);
        KB_LAUNCH();
        class_decide<<<admit_blocks(), kThreads, 0, st>>>(b.plist, b.hplist, a.hpcount, b.pt, b.pc, g.vwgt, bw, H,
                                                          minvP, P, bound, 0);
        KB_LAUNCH();
        class_apply<<<admit_blocks(), kThreads, 0, st>>>(b.plist, b.hplist, a.hpcount, b.pt, b.pc, g.xadj, g.adjncy,
                                                         g.vwgt, part, bw, H, minvP, P, NextActive{}, b.counters + kCntMoved);
        KB_LAUNCH();
    }
    if (!ok) {
        block_scan_kernel<<<1, 1024, 0, st>>>(bw, k, bound, flags, flags + 1, nullptr);
        KB_LAUNCH();
        KB_CUDA(cudaMemcpyAsync(ctx.pinned, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaStreamSynchronize(st));
        ok = ctx.pinned[0] == 0;
    }
    ctx.scratch.release(mk);
    return ok;
}

}  // namespace kb
