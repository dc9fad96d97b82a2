// ip_device.cu -- initial partitioning of the coarsest graph on the device:
// recursive bisection with every bisection of one recursion depth in one
// launch, one thread block per block of the current partition.
//
// The recursion and its bounds follow graph_partitioner.cpp:110-238: the
// left half of a block that still splits into kk blocks gets ceil(kk/2) of
// them, the side targets are in proportion, each side may exceed its target
// by max((1+eps)^(1/ceil log2 kk) - 1, min(eps, 1%)).  A block is named by
// its offset o, the first final block id it covers, so part[] holds final
// block ids once the recursion ends.  A bisection runs `tries` tries and
// keeps the best by (overload, cut), the first on ties.  A try:
//   1. start node: the reached node farthest from s0 by breadth-first search
//      (bipartition.cpp:125-146 searches twice), ties to the smaller id,
//      where s0 is the node of smallest (hash, id);
//   2. growing: nodes in (BFS distance from the start, id) order, unreached
//      nodes last; side 0 takes the prefix until it reaches its target, and
//      the node that crosses the target joins only if side 0 then stays
//      within its bound (bipartition.cpp:147-222 grows by gain instead);
//   3. 2-way Jet refinement in synchronous iterations: candidate moves with
//      a negative-gain tolerance, the afterburner, a balance repair of an
//      overloaded side by loss classes, the best (overload, cut) kept.
// Per depth: one thread block per splitting block builds its subgraph
// (members in id order, edges inside the block) from the coarsest graph;
// one thread block per (block, try) runs the try; one per block keeps the
// best try and writes the new block ids.  Every step is deterministic: BFS
// distances, reductions over (key, id) and prefix sums in id order do not
// depend on the order threads run in.
#include "ip_device.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "hash.h"

#include "prims.cuh"

namespace kb {

namespace {

constexpr int kBT = 256;              // threads per block of the small kernels
constexpr int kMaxBW = 32;            // warps per block at most (reduction buffers)
constexpr int kTryMaxBT = 512;        // threads per block of ip_try at most
constexpr int kIpClasses = 256;       // balance repair classes (loss bucket x 8)
constexpr int kDenseRows = 16;        // average degree from which a warp walks each row
constexpr int kIpSmemPerNode = 36;    // shared-memory bytes per node of a try's working state
constexpr int kIpSmemLean = 22;       // ... without row starts, lengths and node weights
constexpr int kIpSmemBfs = 12;        // breadth-first distances and queues only
constexpr int kIpSmem = 200 * 1024;   // dynamic shared memory of the try kernel

struct IpArgs {
    int n;
    const int* xadj;
    const int* adjncy;
    const int* adjwgt;
    const int* vwgt;
    int* part;        // [reps][n]: current block offset per node
    int nsplit, reps;
    const int* split_o;  // [nsplit] offsets of the blocks that split at this depth
    const int* split_k;  // [nsplit] their block counts
    const double* split_eb;  // [nsplit] their per-side slack (computed on the host)
    const int* sidx;     // [k] split index of a block offset, -1 when it does not split
    unsigned* cnt;       // [reps][nsplit] members
    unsigned* deg;       // [reps][nsplit] members' degrees
    unsigned* nbase;     // [reps][nsplit] start of the split's node slots (members + 2 each)
    unsigned* ebase;     // [reps][nsplit] start of its edge slots
    long long NS, ES;    // node / edge slots per repetition
    int* lid;            // [reps][n]
    int* nsub;           // [reps][nsplit] nodes of each split's subgraph
    int *orig, *lbeg, *ldeg, *lcw;  // [reps][NS] subgraphs (lcw: node weights)
    int *ladj, *lw;      // [reps][ES]
    // per (repetition, try): node slots of the try's working state
    int *dist, *qa, *qb, *moved_at, *cls;  // [reps * tries][NS]
    uint8_t *side, *best, *dest, *keep;    // [reps * tries][NS]
    long long* gain;                       // [reps * tries][NS]
    unsigned long long* layer;             // [reps * tries][NS]
    unsigned long long* try_ov;            // [reps][nsplit][tries]
    long long* try_cut;                    // [reps][nsplit][tries]
    int seed, depth, tries, jet_iters, jet_patience, jet_c, bal_iters;
    double eps;
    int smem_bytes;      // dynamic shared memory of ip_try
    int* err;
};

struct Acc2 {
    long long a, b;
};

__device__ __forceinline__ long long warp_sum_ll(long long x) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Block-wide reductions; every thread gets the result.  `sh` holds kMaxBW + 1
// words and is free again when the call returns.
__device__ unsigned long long block_sum(unsigned long long x, unsigned long long* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
        sh[kMaxBW] = t;
    }
    __syncthreads();
    const unsigned long long r = sh[kMaxBW];
    __syncthreads();
    return r;
}

__device__ unsigned long long block_min(unsigned long long x, unsigned long long* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = ~0ull;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = min(t, sh[w]);
        sh[kMaxBW] = t;
    }
    __syncthreads();
    const unsigned long long r = sh[kMaxBW];
    __syncthreads();
    return r;
}

__device__ unsigned long long block_max(unsigned long long x, unsigned long long* sh) {
    return ~block_min(~x, sh);
}

// Exclusive prefix sum over the block's threads in thread order; *total =
// the sum.  `sh` as above.
__device__ unsigned long long block_scan(unsigned long long x, unsigned long long* total, unsigned long long* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) sh[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long run = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            const unsigned long long t = sh[w];
            sh[w] = run;
            run += t;
        }
        sh[kMaxBW] = run;
    }
    __syncthreads();
    const unsigned long long r = sh[wid] + incl - x;
    *total = sh[kMaxBW];
    __syncthreads();
    return r;
}

// Per-row sums over the local subgraph: entry(i, e, acc) for every entry e
// of row i, then row(i, acc) once per row (a warp per row when WARP, the
// warp's lane 0 calling row; a thread per row otherwise).
// every row by default; take(i) false: row i's entries are not read (row(i)
// still runs, with zero sums)
struct AllRows {
    __device__ bool operator()(int) const { return true; }
};

template <bool WARP, class F, class G, class Q = AllRows>
__device__ __forceinline__ void for_rows(int n_o, const int* lbeg, const int* ldeg, const int* __restrict__ ladj,
                                         const int* __restrict__ lw, bool vec, F entry, G row, Q take = Q()) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (WARP) {
        for (int i = wid; i < n_o; i += (int)(blockDim.x >> 5)) {
            Acc2 s{0, 0};
            const int b = lbeg[i], d = take(i) ? ldeg[i] : 0;
            if (vec && d >= 64) {
                // 16-byte loads of four entries (and weights) per lane, from
                // the 16-byte boundary at or before the row start; entries
                // outside the row are skipped (rows in global memory only:
                // the first load may start up to three entries before the
                // row, the last end up to three after it, inside the arrays'
                // allocation)
                const int e1 = b + d;
                const int a0 = b - (int)(((uintptr_t)(ladj + b) >> 2) & 3);
                for (int c = a0 + 4 * lane; c < e1; c += 128) {
                    const int4 u4 = *reinterpret_cast<const int4*>(ladj + c);
                    const int4 w4 = *reinterpret_cast<const int4*>(lw + c);
                    if (c >= b) entry(i, u4.x, w4.x, s);
                    if (c + 1 >= b && c + 1 < e1) entry(i, u4.y, w4.y, s);
                    if (c + 2 >= b && c + 2 < e1) entry(i, u4.z, w4.z, s);
                    if (c + 3 >= b && c + 3 < e1) entry(i, u4.w, w4.w, s);
                }
            } else {
                int t = lane;
                for (; t + 96 < d; t += 128) {  // four entries per lane in flight
                    const int e = b + t;
                    const int u0 = ladj[e], u1 = ladj[e + 32], u2 = ladj[e + 64], u3 = ladj[e + 96];
                    const int w0 = lw[e], w1 = lw[e + 32], w2 = lw[e + 64], w3 = lw[e + 96];
                    entry(i, u0, w0, s);
                    entry(i, u1, w1, s);
                    entry(i, u2, w2, s);
                    entry(i, u3, w3, s);
                }
                for (; t < d; t += 32) entry(i, ladj[b + t], lw[b + t], s);
            }
            s.a = warp_sum_ll(s.a);
            s.b = warp_sum_ll(s.b);
            if (lane == 0) row(i, s);
        }
    } else {
        for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) {
            Acc2 s{0, 0};
            const int b = lbeg[i], d = take(i) ? ldeg[i] : 0;
            int t = 0;
            for (; t + 4 <= d; t += 4) {  // four independent entries in flight
                const int e = b + t;
                const int u0 = ladj[e], u1 = ladj[e + 1], u2 = ladj[e + 2], u3 = ladj[e + 3];
                const int w0 = lw[e], w1 = lw[e + 1], w2 = lw[e + 2], w3 = lw[e + 3];
                entry(i, u0, w0, s);
                entry(i, u1, w1, s);
                entry(i, u2, w2, s);
                entry(i, u3, w3, s);
            }
            for (; t < d; ++t) entry(i, ladj[b + t], lw[b + t], s);
            row(i, s);
        }
    }
}

// Breadth-first distances from s (INT_MAX = unreached).  One barrier per
// level: level L counts its next frontier in sh_next[L % 3], and thread 0
// clears sh_next[(L + 1) % 3] during level L -- every thread read that
// counter before the barrier of level L - 1.
__device__ __forceinline__ void bfs_visit(int u, int next, int* dist, int* qb, unsigned* cnt) {
    if (atomicCAS(&dist[u], INT_MAX, next) == INT_MAX) qb[atomicAdd(cnt, 1u)] = u;
}

template <bool WARP>
__device__ void bfs(int n_o, int s, int* dist, int* qa, int* qb, const int* lbeg, const int* ldeg,
                    const int* ladj, unsigned* sh_next) {
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) dist[i] = INT_MAX;
    if (threadIdx.x == 0) {
        sh_next[0] = 0;
        sh_next[1] = 0;
        sh_next[2] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        dist[s] = 0;
        qa[0] = s;
    }
    __syncthreads();
    int cnt = 1, level = 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    while (cnt > 0) {
        unsigned* nx = sh_next + level % 3;
        const int next = level + 1;
        if (WARP) {
            for (int f = wid; f < cnt; f += (int)(blockDim.x >> 5)) {
                const int v = qa[f], b = lbeg[v], d = ldeg[v];
                for (int t = lane; t < d; t += 32) bfs_visit(ladj[b + t], next, dist, qb, nx);
            }
        } else {
            for (int f = threadIdx.x; f < cnt; f += (int)blockDim.x) {
                const int v = qa[f], b = lbeg[v], d = ldeg[v];
                int t = 0;
                for (; t + 4 <= d; t += 4) {  // four row entries loaded together
                    const int u0 = ladj[b + t], u1 = ladj[b + t + 1], u2 = ladj[b + t + 2], u3 = ladj[b + t + 3];
                    bfs_visit(u0, next, dist, qb, nx);
                    bfs_visit(u1, next, dist, qb, nx);
                    bfs_visit(u2, next, dist, qb, nx);
                    bfs_visit(u3, next, dist, qb, nx);
                }
                for (; t < d; ++t) bfs_visit(ladj[b + t], next, dist, qb, nx);
            }
        }
        if (threadIdx.x == 0) sh_next[(level + 1) % 3] = 0;
        __syncthreads();
        cnt = (int)*nx;
        int* tq = qa;
        qa = qb;
        qb = tq;
        ++level;
    }
    __syncthreads();
}

// reached node of largest distance, ties to the smaller id
__device__ int farthest(int n_o, const int* dist, unsigned long long* sh) {
    unsigned long long best = 0;
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x)
        if (dist[i] != INT_MAX) {
            const unsigned long long key = ((unsigned long long)(unsigned)dist[i] << 32) | (0xffffffffu - (unsigned)i);
            best = max(best, key);
        }
    best = block_max(best, sh);
    return (int)(0xffffffffu - (unsigned)(best & 0xffffffffu));
}

// A bisection's subgraph in local ids: row starts and lengths, entries and
// their weights, node weights.
struct Sub {
    int n_o;
    const int *lbeg, *ldeg;
    const int* __restrict__ ladj;
    const int* __restrict__ lw;
    const int* cw;
    bool vec;  // rows in global memory, ladj and lw 16-byte aligned alike: 16-byte row loads
    __device__ uint32_t c(int i) const { return (uint32_t)cw[i]; }
};

__device__ void side_weights(const Sub& S, const uint8_t* side, unsigned long long w[2], unsigned long long* sh) {
    unsigned long long a = 0, b = 0;
    for (int i = threadIdx.x; i < S.n_o; i += (int)blockDim.x) (side[i] ? b : a) += S.c(i);
    w[0] = block_sum(a, sh);
    w[1] = block_sum(b, sh);
}

__device__ __forceinline__ unsigned long long overload2(const unsigned long long w[2], const unsigned long long mw[2]) {
    return (w[0] > mw[0] ? w[0] - mw[0] : 0ull) + (w[1] > mw[1] ? w[1] - mw[1] : 0ull);
}

template <bool WARP>
__device__ long long cut_of(const Sub& S, const uint8_t* side, unsigned long long* sh) {
    long long mine = 0;
    for_rows<WARP>(S.n_o, S.lbeg, S.ldeg, S.ladj, S.lw, S.vec,
                   [&](int i, int u, int w, Acc2& s) { if (side[u] != side[i]) s.a += w; },
                   [&](int, const Acc2& s) { mine += s.a; });
    return (long long)block_sum((unsigned long long)mine, sh) / 2;
}

__device__ __forceinline__ int loss_bucket_d(long long loss) {
    if (loss <= 0) return 0;
    int b = 1;
    while (b < 31 && (loss >> b) > 0) ++b;
    return b;
}

// Moves nodes off side s until it is within mw[s]: classes (log2 bucket of
// conn(own) - conn(other)) x 8 hashed sub-classes; classes are released in
// order until their weight covers the excess; released classes move whole
// while the other side stays within its bound, and in the first class that
// does not fit, its nodes in id order while the running weight fits.
__device__ void block_sum4(unsigned long long v[4], unsigned long long* sh);

// Release threshold T (classes [0, T) cover the excess) and the whole classes
// that fit the other side, [0, full), with their weight `used`, from the
// class weights HS[0 .. kIpClasses): warp 0, eight classes per lane.
__device__ void class_thresholds(const unsigned long long* HS, unsigned long long excess, unsigned long long cap,
                                 int* T_out, int* full_out, unsigned long long* used_out) {
    const int L = threadIdx.x;  // warp 0 only
    unsigned long long h[8], sum = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        h[q] = HS[L * 8 + q];
        sum += h[q];
    }
    unsigned long long incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (L >= o) incl += y;
    }
    const unsigned long long excl = incl - sum;
    // T = the first t with (weight of classes before t) >= excess, else kIpClasses
    int myT = kIpClasses, myF = kIpClasses;
    unsigned long long run = excl;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        if (myT == kIpClasses && run >= excess) myT = L * 8 + q;
        if (myF == kIpClasses && run + h[q] > cap) myF = L * 8 + q;
        run += h[q];
    }
    const int T = (int)__reduce_min_sync(0xffffffffu, (unsigned)myT);
    const int full = min(T, (int)__reduce_min_sync(0xffffffffu, (unsigned)myF));
    // used = weight of the classes before `full`
    unsigned long long u = 0;
    const bool owner = full < kIpClasses ? (full >> 3) == L : L == 31;
    if (owner) {
        if (full < kIpClasses) {
            u = excl;
#pragma unroll
            for (int q = 0; q < 8; ++q)
                if (L * 8 + q < full) u += h[q];
        } else {
            u = incl;
        }
    }
    const unsigned long long used = __shfl_sync(0xffffffffu, u, full < kIpClasses ? (full >> 3) : 31);
    if (L == 0) {
        *T_out = T;
        *full_out = full;
        *used_out = used;
    }
}

// Moves nodes off side s until it is within mw[s]: classes (log2 bucket of
// conn(own) - conn(other)) x 8 hashed sub-classes; classes are released in
// order until their weight covers the excess; released classes move whole
// while the other side stays within its bound, and in the first class that
// does not fit, its nodes in id order while the running weight fits.  w[]
// (the side weights, exact on entry) is kept up to date.
template <bool WARP>
__device__ void balance2(const Sub& S, uint8_t* side, int* cls, int s, const unsigned long long mw[2],
                         unsigned long long w[2], uint64_t ks_cls, int iters, unsigned long long* HS,
                         unsigned long long* sh, unsigned long long* sh4, int* sh_int) {
    for (int it = 0; it < iters; ++it) {
        if (w[s] <= mw[s]) break;
        const unsigned long long excess = w[s] - mw[s];
        const unsigned long long cap = mw[1 - s] > w[1 - s] ? mw[1 - s] - w[1 - s] : 0ull;
        for (int t = threadIdx.x; t < kIpClasses; t += (int)blockDim.x) HS[t] = 0;
        __syncthreads();
        const uint64_t ks = mix64(ks_cls ^ (uint64_t)it);
        for_rows<WARP>(S.n_o, S.lbeg, S.ldeg, S.ladj, S.lw, S.vec,
                       [&](int i, int u, int w, Acc2& a) {
                           if (side[u] == side[i]) a.a += w;
                           else a.b += w;
                       },
                       [&](int i, const Acc2& a) {
                           cls[i] = -1;
                           if (side[i] != s) return;
                           const int c = loss_bucket_d(a.a - a.b) * 8 + (int)hash_range(hash32(ks, (uint32_t)i), 8u);
                           cls[i] = c;
                           atomicAdd(&HS[c], (unsigned long long)S.c(i));
                       });
        __syncthreads();
        if (threadIdx.x < 32) class_thresholds(HS, excess, cap, &sh_int[0], &sh_int[1], &HS[kIpClasses]);
        __syncthreads();
        const int T = sh_int[0], full = sh_int[1];
        const unsigned long long used = HS[kIpClasses];
        unsigned long long mv[4] = {0, 0, 0, 0};  // moves, moved weight
        // whole classes, then the partial one by id prefix (in chunks of the
        // block's threads, in id order)
        if (full < T) {
            unsigned long long run = used;
            for (int base = 0; base < S.n_o; base += (int)blockDim.x) {
                const int i = base + threadIdx.x;
                const int c = i < S.n_o ? cls[i] : -1;
                if (c >= 0 && c < full) {
                    side[i] = (uint8_t)(1 - s);
                    mv[0] += 1;
                    mv[1] += S.c(i);
                }
                const bool part_cls = c == full;
                unsigned long long tot;
                const unsigned long long pre = block_scan(part_cls ? (unsigned long long)S.c(i) : 0ull, &tot, sh);
                if (part_cls && run + pre + S.c(i) <= cap) {
                    side[i] = (uint8_t)(1 - s);
                    mv[0] += 1;
                    mv[1] += S.c(i);
                }
                run += tot;
            }
        } else {
            for (int i = threadIdx.x; i < S.n_o; i += (int)blockDim.x) {
                const int c = cls[i];
                if (c >= 0 && c < full) {
                    side[i] = (uint8_t)(1 - s);
                    mv[0] += 1;
                    mv[1] += S.c(i);
                }
            }
        }
        block_sum4(mv, sh4);
        w[s] -= mv[1];
        w[1 - s] += mv[1];
        if (mv[0] == 0) break;
    }
}

// Sums of four values over the block; every thread gets them.  `sh` holds
// 4 * (kMaxBW + 1) words.
__device__ void block_sum4(unsigned long long v[4], unsigned long long* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        if (lane == 0) sh[q * (kMaxBW + 1) + wid] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[threadIdx.x * (kMaxBW + 1) + w];
        sh[threadIdx.x * (kMaxBW + 1) + kMaxBW] = t;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = sh[q * (kMaxBW + 1) + kMaxBW];
    __syncthreads();
}

// Sums of four values over the block with one barrier: warp sums go into one
// of three rotating shared accumulators; call c clears the accumulator of
// call c + 1, which every thread last read before the barrier of call c - 1.
// Every thread of the block makes the same calls in the same order.
struct Red4 {
    unsigned long long (*acc)[4];  // [3][4], zero before the first call
    int ph;
};

__device__ void red4(unsigned long long v[4], Red4& r) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    unsigned long long* b = r.acc[r.ph];
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (v[q]) atomicAdd(&b[q], v[q]);
    const int nx = r.ph == 2 ? 0 : r.ph + 1;
    if (threadIdx.x < 4) r.acc[nx][threadIdx.x] = 0;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = b[q];
    r.ph = nx;
}

// cut and side weights of the current sides, in one reduction
template <bool WARP>
__device__ void cut_and_weights(const Sub& S, const uint8_t* side, long long* cut, unsigned long long w[2],
                                unsigned long long* sh4) {
    unsigned long long v[4] = {0, 0, 0, 0};
    for_rows<WARP>(S.n_o, S.lbeg, S.ldeg, S.ladj, S.lw, S.vec,
                   [&](int i, int u, int w, Acc2& s) { if (side[u] != side[i]) s.a += w; },
                   [&](int i, const Acc2& s) {
                       v[0] += (unsigned long long)s.a;
                       v[side[i] ? 2 : 1] += S.c(i);
                   });
    block_sum4(v, sh4);
    *cut = (long long)(v[0] / 2);
    w[0] = v[1];
    w[1] = v[2];
}

// 2-way Jet on side[] (the best state is kept in best[] and left in side[]);
// returns its cut.  The cut and side weights of the state an iteration
// leaves are summed in the next iteration's candidate pass, which reads
// every row anyway; the best-state bookkeeping of iteration it - 1 runs
// there, before iteration it moves anything (the same order as evaluating
// at the end of iteration it - 1).
template <bool WARP>
__device__ long long jet2(const Sub& S, const IpArgs& a, uint8_t* side, uint8_t* best, uint8_t* dest,
                          uint8_t* keep, long long* gain, int* moved_at, int* cls, const unsigned long long mw[2],
                          int bis_level, int bis_round, unsigned long long* HS, unsigned long long* sh,
                          unsigned long long* sh4, int* sh_int) {
    __shared__ unsigned long long racc[3][4];
    const int n_o = S.n_o;
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) moved_at[i] = -2;
    if (threadIdx.x < 12) racc[threadIdx.x / 4][threadIdx.x % 4] = 0;
    __syncthreads();
    Red4 red{racc, 0};
    // the sides alternate between two buffers: the afterburner reads the
    // current one and writes the moved state into the other (keep[])
    uint8_t* const side0 = side;
    uint8_t* nside = keep;
    unsigned long long best_ov = 0, moved_prev = 0;
    long long best_cut = 0;
    const long long c4 = a.jet_c;
    int since = 0;
    bool done = false;
    // one state evaluation: best tracking, then the stopping rule (each
    // thread copies its own nodes, which no other thread writes before the
    // copy is read at the end)
    auto evaluate = [&](long long cut, const unsigned long long w[2], bool first) -> bool {
        const unsigned long long ov = overload2(w, mw);
        if (first || ov < best_ov || (ov == best_ov && cut < best_cut)) {
            best_ov = ov;
            best_cut = cut;
            for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) best[i] = side[i];
            since = 0;
        } else {
            ++since;
        }
        return !first && (moved_prev == 0 || since >= a.jet_patience);
    };
    int it = 0;
    for (; it < a.jet_iters; ++it) {
        // candidates, and the cut and weights of the current state
        unsigned long long v[4] = {0, 0, 0, 0};
        for_rows<WARP>(n_o, S.lbeg, S.ldeg, S.ladj, S.lw, S.vec,
                       [&](int i, int u, int w, Acc2& s) {
                           if (side[u] == side[i]) s.a += w;
                           else s.b += w;
                       },
                       [&](int i, const Acc2& s) {
                           v[0] += (unsigned long long)s.b;
                           v[side[i] ? 2 : 1] += S.c(i);
                           dest[i] = 0;
                           if (moved_at[i] == it - 1 || s.b == 0) return;
                           const long long gv = s.b - s.a;
                           if (4 * gv >= -c4 * s.a) {
                               dest[i] = 1;
                               gain[i] = gv;
                           }
                       });
        red4(v, red);
        unsigned long long w[2] = {v[1], v[2]};
        if (evaluate((long long)(v[0] / 2), w, it == 0)) {
            done = true;
            break;
        }
        // afterburner (gain with every higher-priority candidate neighbour
        // moved) and the moves it keeps, into the other side buffer; the side
        // weights follow from the moved weight
        unsigned long long m[4] = {0, 0, 0, 0};  // moves, weight 0 -> 1, weight 1 -> 0
        for_rows<WARP>(n_o, S.lbeg, S.ldeg, S.ladj, S.lw, S.vec,
                       [&](int i, int u, int w, Acc2& s) {
                           int su = side[u];
                           if (dest[u] && (gain[u] > gain[i] || (gain[u] == gain[i] && u < i))) su = 1 - su;
                           s.a += su != side[i] ? w : -(long long)w;
                       },
                       [&](int i, const Acc2& s) {
                           const uint8_t si = side[i];
                           if (dest[i] && s.a >= 0) {
                               m[0] += 1;
                               m[si ? 2 : 1] += S.c(i);
                               nside[i] = (uint8_t)(si ^ 1);
                               moved_at[i] = it;
                           } else {
                               nside[i] = si;
                           }
                       },
                       [&](int i) { return dest[i] != 0; });
        red4(m, red);
        {
            uint8_t* tsd = side;
            side = nside;
            nside = tsd;
        }
        moved_prev = m[0];
        w[0] = w[0] - m[1] + m[2];
        w[1] = w[1] - m[2] + m[1];
        if (w[0] > mw[0] || w[1] > mw[1]) {
            const uint64_t ks_cls = stream_key(a.seed, TAG_BCLS, bis_level, bis_round * 64 + it);
            const bool over[2] = {w[0] > mw[0], w[1] > mw[1]};
            for (int s2 = 0; s2 < 2; ++s2)
                if (over[s2]) balance2<WARP>(S, side, cls, s2, mw, w, ks_cls, a.bal_iters, HS, sh, sh4, sh_int);
        }
    }
    if (!done) {
        // the state the last iteration left (or the start, without iterations)
        long long cut;
        unsigned long long w[2];
        cut_and_weights<WARP>(S, side, &cut, w, sh4);
        evaluate(cut, w, it == 0);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) side0[i] = best[i];
    __syncthreads();
    return best_cut;
}

// ---------------------------------------------------------------- kernels

// members and their degrees per (repetition, splitting block)
__global__ void ip_count(IpArgs a) {
    const long long total = (long long)a.reps * a.n;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < total;
         x += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(x / a.n), v = (int)(x % a.n);
        const int j = a.sidx[a.part[(long long)r * a.n + v]];
        if (j < 0) continue;
        atomicAdd(&a.cnt[r * a.nsplit + j], 1u);
        atomicAdd(&a.deg[r * a.nsplit + j], (unsigned)(a.xadj[v + 1] - a.xadj[v]));
    }
}

// node and edge slot bases per (repetition, split): one thread block
__global__ void ip_bases(IpArgs a) {
    __shared__ unsigned long long sh[kMaxBW + 1];
    for (int r = 0; r < a.reps; ++r) {
        unsigned long long nrun = 0, erun = 0;
        for (int base = 0; base < a.nsplit; base += (int)blockDim.x) {
            const int j = base + threadIdx.x;
            const bool ok = j < a.nsplit;
            unsigned long long nt, et;
            const unsigned long long np = block_scan(ok ? a.cnt[r * a.nsplit + j] + 2ull : 0ull, &nt, sh);
            const unsigned long long ep = block_scan(ok ? (unsigned long long)a.deg[r * a.nsplit + j] : 0ull, &et, sh);
            if (ok) {
                a.nbase[r * a.nsplit + j] = (unsigned)(nrun + np);
                a.ebase[r * a.nsplit + j] = (unsigned)(erun + ep);
            }
            nrun += nt;
            erun += et;
        }
    }
}

// One thread block per (repetition, split): the split block's subgraph,
// members in id order, rows restricted to the block, local ids.
__global__ void __launch_bounds__(kTryMaxBT) ip_extract(IpArgs a) {
    __shared__ unsigned long long sh[kMaxBW + 1];
    const int j = blockIdx.x % a.nsplit, r = blockIdx.x / a.nsplit;
    const int o = a.split_o[j];
    const int* part = a.part + (long long)r * a.n;
    int* lid = a.lid + (long long)r * a.n;
    const long long nb = (long long)r * a.NS + a.nbase[r * a.nsplit + j];
    const long long eb = (long long)r * a.ES + a.ebase[r * a.nsplit + j];
    int* orig = a.orig + nb;
    int* lbeg = a.lbeg + nb;
    int* ldeg = a.ldeg + nb;
    int* ladj = a.ladj + eb;
    int* lw = a.lw + eb;
    // members in id order: every warp counts the members of its own range
    // of ids, then writes them behind the ranges before it
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nwarps = (int)(blockDim.x >> 5);
    const int seg = (a.n + nwarps - 1) / nwarps;
    const int lo = wid * seg, hi = min(a.n, lo + seg);
    unsigned mine = 0;
    for (int base = lo; base < hi; base += 32) {
        const int v = base + lane;
        mine += __popc(__ballot_sync(0xffffffffu, v < hi && part[v] == o));
    }
    if (lane == 0) sh[wid] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long run = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            const unsigned long long t = sh[w];
            sh[w] = run;
            run += t;
        }
        sh[kMaxBW] = run;
    }
    __syncthreads();
    unsigned long long cnt = sh[wid];
    for (int base = lo; base < hi; base += 32) {
        const int v = base + lane;
        const bool mem = v < hi && part[v] == o;
        const unsigned m = __ballot_sync(0xffffffffu, mem);
        if (mem) {
            const unsigned long long idx = cnt + __popc(m & ((1u << lane) - 1u));
            lid[v] = (int)idx;
            orig[idx] = v;
            a.lcw[nb + idx] = a.vwgt[v];
        }
        cnt += __popc(m);
    }
    const int n_o = (int)sh[kMaxBW];
    __syncthreads();
    if (threadIdx.x == 0) a.nsub[r * a.nsplit + j] = n_o;
    // rows of up to 32 entries by their own thread, longer rows by a warp
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) {
        const int v = orig[i];
        const int e0 = a.xadj[v], e1 = a.xadj[v + 1];
        if (e1 - e0 > 32) continue;
        int d = 0, e = e0;
        for (; e + 4 <= e1; e += 4) {  // four independent gathers in flight
            const int u0 = a.adjncy[e], u1 = a.adjncy[e + 1], u2 = a.adjncy[e + 2], u3 = a.adjncy[e + 3];
            d += (part[u0] == o) + (part[u1] == o) + (part[u2] == o) + (part[u3] == o);
        }
        for (; e < e1; ++e) d += part[a.adjncy[e]] == o;
        ldeg[i] = d;
    }
    for (int i = wid; i < n_o; i += (int)(blockDim.x >> 5)) {
        const int v = orig[i];
        if (a.xadj[v + 1] - a.xadj[v] <= 32) continue;
        const int e1 = a.xadj[v + 1];
        int d = 0, e = a.xadj[v] + lane;
        for (; e + 96 < e1; e += 128) {  // four gathers per lane in flight
            const int u0 = a.adjncy[e], u1 = a.adjncy[e + 32], u2 = a.adjncy[e + 64], u3 = a.adjncy[e + 96];
            d += (part[u0] == o) + (part[u1] == o) + (part[u2] == o) + (part[u3] == o);
        }
        for (; e < e1; e += 32) d += part[a.adjncy[e]] == o;
        d = __reduce_add_sync(0xffffffffu, d);
        if (lane == 0) ldeg[i] = d;
    }
    __syncthreads();
    unsigned long long erun = 0;
    for (int base = 0; base < n_o; base += (int)blockDim.x) {
        const int i = base + threadIdx.x;
        unsigned long long tot;
        const unsigned long long pre = block_scan(i < n_o ? (unsigned long long)ldeg[i] : 0ull, &tot, sh);
        if (i < n_o) lbeg[i] = (int)(erun + pre);
        erun += tot;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) {
        const int v = orig[i];
        const int e0 = a.xadj[v], e1 = a.xadj[v + 1];
        if (e1 - e0 > 32) continue;
        int w = lbeg[i], e = e0;
        for (; e + 4 <= e1; e += 4) {  // four independent gathers in flight
            int u[4], pu[4], wt[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) u[q] = a.adjncy[e + q];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                pu[q] = part[u[q]];
                wt[q] = a.adjwgt[e + q];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (pu[q] == o) {
                    ladj[w] = lid[u[q]];
                    lw[w] = wt[q];
                    ++w;
                }
        }
        for (; e < e1; ++e) {
            const int u = a.adjncy[e];
            if (part[u] != o) continue;
            ladj[w] = lid[u];
            lw[w] = a.adjwgt[e];
            ++w;
        }
    }
    for (int i = wid; i < n_o; i += (int)(blockDim.x >> 5)) {
        const int v = orig[i];
        if (a.xadj[v + 1] - a.xadj[v] <= 32) continue;
        int w = lbeg[i];
        const int e1 = a.xadj[v + 1];
        // four 32-entry chunks loaded together, then written in order
        for (int c0 = a.xadj[v]; c0 < e1; c0 += 128) {
            int u[4], pu[4], wt[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int e = c0 + 32 * q + lane;
                u[q] = e < e1 ? a.adjncy[e] : -1;
                wt[q] = e < e1 ? a.adjwgt[e] : 0;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) pu[q] = u[q] >= 0 ? part[u[q]] : -1;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const bool in = u[q] >= 0 && pu[q] == o;
                const unsigned m = __ballot_sync(0xffffffffu, in);
                if (in) {
                    const int p = w + __popc(m & ((1u << lane) - 1u));
                    ladj[p] = lid[u[q]];
                    lw[p] = wt[q];
                }
                w += __popc(m);
            }
        }
    }
}

// One thread block per (repetition, split, try): start node, growing and
// 2-way Jet; the try's sides stay in its side[] slots, its (overload, cut)
// in try_ov / try_cut.
template <int MAXBT>
__global__ void __launch_bounds__(MAXBT) ip_try(IpArgs a) {
    __shared__ unsigned long long sh[kMaxBW + 1];
    __shared__ unsigned long long sh4[4 * (kMaxBW + 1)];
    __shared__ unsigned long long HS[kIpClasses + 1];
    __shared__ unsigned sh_cnt[3];
    __shared__ int sh_int[4];
    extern __shared__ __align__(16) unsigned char dyn[];
    const int t = blockIdx.x % a.tries;
    const int j = (blockIdx.x / a.tries) % a.nsplit;
    const int r = blockIdx.x / (a.tries * a.nsplit);
    const int kk = a.split_k[j], kl = (kk + 1) / 2;
    const int n_o = a.nsub[r * a.nsplit + j];
    const long long nb = (long long)r * a.NS + a.nbase[r * a.nsplit + j];
    const long long eb = (long long)r * a.ES + a.ebase[r * a.nsplit + j];
    const long long res = ((long long)r * a.nsplit + j) * a.tries + t;
    if (n_o == 0) {
        if (threadIdx.x == 0) { a.try_ov[res] = 0; a.try_cut[res] = 0; }
        return;
    }
    // working state of this try, by what fits in shared memory:
    //   full  kIpSmemPerNode bytes per node (buffers whose lives do not
    //         overlap share storage), the subgraph's entries too when they
    //         also fit;
    //   lean  the same without the row starts, lengths and node weights
    //         (read from global memory);
    //   bfs   only the breadth-first distances and queues;
    //   none  everything in the try's global slots.
    const long long ns = ((long long)r * a.tries + t) * a.NS + a.nbase[r * a.nsplit + j];
    uint8_t* gside = a.side + ns;
    const long long E_o = (long long)a.lbeg[nb + n_o - 1] + a.ldeg[nb + n_o - 1];
    const long long N2 = (long long)n_o + 2;
    const long long need_full = N2 * kIpSmemPerNode + 256;
    const bool full = need_full <= (long long)a.smem_bytes;
    const bool lean = !full && N2 * kIpSmemLean + 256 <= (long long)a.smem_bytes;
    const bool bfs_smem = !full && !lean && N2 * kIpSmemBfs + 256 <= (long long)a.smem_bytes;
    const bool in_smem = full || lean;  // side[] lives in shared memory
    const bool csr_smem = full && need_full + 8 * E_o + 64 <= (long long)a.smem_bytes;
    long long* gain = a.gain + ns;
    unsigned long long* layer = a.layer + ns;
    int* dist = a.dist + ns;
    int* qa = a.qa + ns;
    int* qb = a.qb + ns;
    int* moved_at = a.moved_at + ns;
    int* cls = a.cls + ns;
    const int* lbeg = a.lbeg + nb;
    const int* ldeg = a.ldeg + nb;
    const int* cw = a.lcw + nb;
    const int* ladj = a.ladj + eb;
    const int* lw = a.lw + eb;
    uint8_t* side = gside;
    uint8_t* best = a.best + ns;
    uint8_t* dest = a.dest + ns;
    uint8_t* keep = a.keep + ns;
    if (in_smem) {
        const size_t N = (size_t)N2;
        unsigned char* p = dyn;
        gain = reinterpret_cast<long long*>(p);  // growing's layer weights, then Jet's gains
        layer = reinterpret_cast<unsigned long long*>(p);
        p += 8 * N;
        dist = reinterpret_cast<int*>(p);  // distances, then Jet's best / dest / keep bytes
        best = p;
        dest = p + N;
        keep = p + 2 * N;
        p += 4 * N;
        qa = reinterpret_cast<int*>(p);  // a BFS queue, then Jet's move iterations
        moved_at = qa;
        p += 4 * N;
        qb = reinterpret_cast<int*>(p);  // the other BFS queue, then balance classes
        cls = qb;
        p += 4 * N;
        side = p;
        p += (N + 15) & ~(size_t)15;
        if (full) {
            int* sbeg = reinterpret_cast<int*>(p); p += 4 * N;
            int* sdeg = reinterpret_cast<int*>(p); p += 4 * N;
            int* scw = reinterpret_cast<int*>(p); p += 4 * N;
            for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) {
                sbeg[i] = a.lbeg[nb + i];
                sdeg[i] = a.ldeg[nb + i];
                scw[i] = a.lcw[nb + i];
            }
            lbeg = sbeg;
            ldeg = sdeg;
            cw = scw;
        }
        if (csr_smem) {
            int* sa = reinterpret_cast<int*>(p);
            int* sw = sa + E_o;
            for (long long e = threadIdx.x; e < E_o; e += blockDim.x) {
                sa[e] = a.ladj[eb + e];
                sw[e] = a.lw[eb + e];
            }
            ladj = sa;
            lw = sw;
        }
        __syncthreads();
    } else if (bfs_smem) {
        const size_t N = (size_t)N2;
        dist = reinterpret_cast<int*>(dyn);
        qa = dist + N;
        qb = qa + N;
    }
    const bool vec = !csr_smem && (((uintptr_t)a.ladj | (uintptr_t)a.lw) & 15) == 0;
    const Sub S{n_o, lbeg, ldeg, ladj, lw, cw, vec};
    // targets and bounds
    unsigned long long Wm = 0;
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) Wm += S.c(i);
    const unsigned long long W = block_sum(Wm, sh);
    const unsigned long long t0 = W * (unsigned long long)kl / (unsigned long long)kk, t1 = W - t0;
    const double eb2 = a.split_eb[j];
    const unsigned long long mw[2] = {(unsigned long long)((1.0 + eb2) * (double)t0),
                                      (unsigned long long)((1.0 + eb2) * (double)t1)};
    const bool warp_rows = E_o >= (long long)kDenseRows * n_o;
    const int bis_level = a.split_o[j], bis_round = (r * 32 + a.depth) * 64 + t;
    // 1. start: farthest from the node of smallest (hash, id)
    const uint64_t ks = stream_key(a.seed, TAG_IP, bis_level, bis_round);
    unsigned long long m0 = ~0ull;
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x)
        m0 = min(m0, ((unsigned long long)hash32(ks, (uint32_t)i) << 32) | (unsigned)i);
    const int s0 = (int)(block_min(m0, sh) & 0xffffffffu);
    if (warp_rows) bfs<true>(n_o, s0, dist, qa, qb, S.lbeg, S.ldeg, S.ladj, sh_cnt);
    else bfs<false>(n_o, s0, dist, qa, qb, S.lbeg, S.ldeg, S.ladj, sh_cnt);
    const int st = farthest(n_o, dist, sh);
    if (warp_rows) bfs<true>(n_o, st, dist, qa, qb, S.lbeg, S.ldeg, S.ladj, sh_cnt);
    else bfs<false>(n_o, st, dist, qa, qb, S.lbeg, S.ldeg, S.ladj, sh_cnt);
    // 2. growing by (distance, id): layer weights, the crossing layer, and
    // the crossing layer's id-order prefix
    unsigned long long md = 0;
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x)
        if (dist[i] != INT_MAX) md = max(md, (unsigned long long)dist[i]);
    const int maxd = (int)block_max(md, sh);
    const int nl = maxd + 2;
    for (int l = threadIdx.x; l < nl; l += (int)blockDim.x) layer[l] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x)
        atomicAdd(&layer[dist[i] == INT_MAX ? maxd + 1 : dist[i]], (unsigned long long)S.c(i));
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long cum = 0;
        int lc = 0;
        while (lc < nl && cum + layer[lc] < t0) cum += layer[lc++];
        sh_int[2] = lc;
        HS[kIpClasses] = cum;
    }
    __syncthreads();
    const int lc = sh_int[2];
    unsigned long long run = HS[kIpClasses];
    __syncthreads();
    for (int base = 0; base < n_o; base += (int)blockDim.x) {
        const int i = base + threadIdx.x;
        int l = INT_MAX;
        if (i < n_o) {
            l = dist[i] == INT_MAX ? maxd + 1 : dist[i];
            side[i] = l < lc ? 0 : 1;
        }
        const bool cross = i < n_o && l == lc;
        unsigned long long tot;
        const unsigned long long pre = block_scan(cross ? (unsigned long long)S.c(i) : 0ull, &tot, sh);
        if (cross) {
            const unsigned long long p = run + pre + S.c(i);
            if (run + pre < t0 && p <= mw[0]) side[i] = 0;
        }
        run += tot;
    }
    __syncthreads();
    // 3. 2-way Jet
    const long long c = warp_rows ? jet2<true>(S, a, side, best, dest, keep, gain, moved_at, cls, mw, bis_level,
                                               bis_round, HS, sh, sh4, sh_int)
                                  : jet2<false>(S, a, side, best, dest, keep, gain, moved_at, cls, mw, bis_level,
                                                bis_round, HS, sh, sh4, sh_int);
    unsigned long long w[2];
    side_weights(S, side, w, sh);
    if (threadIdx.x == 0) {
        a.try_ov[res] = overload2(w, mw);
        a.try_cut[res] = c;
    }
    if (in_smem)
        for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x) gside[i] = side[i];
}

// One thread block per (repetition, split): the try of smallest (overload,
// cut), the first on ties; its side 1 becomes block o + kl.
__global__ void __launch_bounds__(kBT) ip_select(IpArgs a) {
    const int j = blockIdx.x % a.nsplit, r = blockIdx.x / a.nsplit;
    const int o = a.split_o[j], kl = (a.split_k[j] + 1) / 2;
    const int n_o = a.nsub[r * a.nsplit + j];
    const long long res = ((long long)r * a.nsplit + j) * a.tries;
    int b = 0;
    for (int t = 1; t < a.tries; ++t)
        if (a.try_ov[res + t] < a.try_ov[res + b] ||
            (a.try_ov[res + t] == a.try_ov[res + b] && a.try_cut[res + t] < a.try_cut[res + b]))
            b = t;
    const long long nb = (long long)r * a.NS + a.nbase[r * a.nsplit + j];
    const uint8_t* side = a.side + ((long long)r * a.tries + b) * a.NS + a.nbase[r * a.nsplit + j];
    int* part = a.part + (long long)r * a.n;
    for (int i = threadIdx.x; i < n_o; i += (int)blockDim.x)
        if (side[i]) part[a.orig[nb + i]] = o + kl;
}

}  // namespace

void initial_partition_device(Ctx& ctx, const DevGraph& c, const Knobs& kn, int* part) {
    cudaStream_t st = ctx.stream;
    const int n = c.n, k = kn.k;
    if (n == 0) return;
    const int reps = std::max(kn.ip_reps, 1);
    int tries = std::max(kn.ip_tries, 1);
    if (c.m > 64LL * n) tries = std::min(tries, 1);  // dense coarsest graphs: one try
    // the recursion's shape depends only on k: per depth the (offset, count)
    // of every block that splits
    std::vector<std::vector<int>> so, sk;
    {
        std::vector<int> kb((size_t)k, 0);
        kb[0] = k;
        for (int d = 0; d < 32; ++d) {
            std::vector<int> o, kk;
            for (int b = 0; b < k; ++b)
                if (kb[b] > 1) { o.push_back(b); kk.push_back(kb[b]); }
            if (o.empty()) break;
            for (size_t i = 0; i < o.size(); ++i) {
                const int kl = (kk[i] + 1) / 2;
                kb[(size_t)o[i]] = kl;
                kb[(size_t)(o[i] + kl)] = kk[i] - kl;
            }
            so.push_back(o);
            sk.push_back(kk);
        }
    }
    const size_t mk = ctx.scratch.mark();
    int maxs = 1;
    for (auto& v : so) maxs = std::max(maxs, (int)v.size());
    // tables for all depths in one upload: [o | k | sidx] per depth
    std::vector<int> tab;
    std::vector<size_t> toff;
    for (size_t d = 0; d < so.size(); ++d) {
        toff.push_back(tab.size());
        tab.insert(tab.end(), so[d].begin(), so[d].end());
        tab.insert(tab.end(), sk[d].begin(), sk[d].end());
        std::vector<int> sidx((size_t)k, -1);
        for (size_t i = 0; i < so[d].size(); ++i) sidx[(size_t)so[d][i]] = (int)i;
        tab.insert(tab.end(), sidx.begin(), sidx.end());
    }
    // per split: the per-side slack max((1+eps)^(1/ceil log2 kk) - 1, min(eps, 1%))
    const double eps = kn.imbalance > 0 ? kn.imbalance : 0.0;
    std::vector<double> ebs;
    for (size_t d = 0; d < so.size(); ++d)
        for (int kk : sk[d]) {
            int lg = 0;
            while ((1 << lg) < kk) ++lg;
            double eb = std::pow(1.0 + eps, 1.0 / lg) - 1.0;
            eb = std::max(eb, std::min(eps, 0.01));
            ebs.push_back(eb);
        }
    int* dtab = ctx.scratch.alloc<int>(std::max<size_t>(tab.size(), 1));
    double* deb = ctx.scratch.alloc<double>(std::max<size_t>(ebs.size(), 1));
    if (!tab.empty()) KB_CUDA(cudaMemcpyAsync(dtab, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, st));
    if (!ebs.empty()) KB_CUDA(cudaMemcpyAsync(deb, ebs.data(), sizeof(double) * ebs.size(), cudaMemcpyHostToDevice, st));
    IpArgs a{};
    a.n = n;
    a.xadj = c.xadj;
    a.adjncy = c.adjncy;
    a.adjwgt = c.adjwgt;
    a.vwgt = c.vwgt;
    a.reps = reps;
    a.NS = (long long)n + 2LL * maxs;
    a.ES = std::max<long long>(c.m, 1);
    a.part = ctx.scratch.alloc<int>((size_t)reps * n);
    a.cnt = ctx.scratch.alloc<unsigned>((size_t)reps * maxs);
    a.deg = ctx.scratch.alloc<unsigned>((size_t)reps * maxs);
    a.nbase = ctx.scratch.alloc<unsigned>((size_t)reps * maxs);
    a.ebase = ctx.scratch.alloc<unsigned>((size_t)reps * maxs);
    a.lid = ctx.scratch.alloc<int>((size_t)reps * n);
    const size_t NSr = (size_t)reps * (size_t)a.NS, ESr = (size_t)reps * (size_t)a.ES;
    const size_t NSt = NSr * (size_t)tries;
    a.nsub = ctx.scratch.alloc<int>((size_t)reps * maxs);
    a.orig = ctx.scratch.alloc<int>(NSr);
    a.lbeg = ctx.scratch.alloc<int>(NSr);
    a.ldeg = ctx.scratch.alloc<int>(NSr);
    a.lcw = ctx.scratch.alloc<int>(NSr);
    a.ladj = ctx.scratch.alloc<int>(ESr);
    a.lw = ctx.scratch.alloc<int>(ESr);
    a.dist = ctx.scratch.alloc<int>(NSt);
    a.qa = ctx.scratch.alloc<int>(NSt);
    a.qb = ctx.scratch.alloc<int>(NSt);
    a.moved_at = ctx.scratch.alloc<int>(NSt);
    a.cls = ctx.scratch.alloc<int>(NSt);
    a.side = ctx.scratch.alloc<uint8_t>(NSt);
    a.best = ctx.scratch.alloc<uint8_t>(NSt);
    a.dest = ctx.scratch.alloc<uint8_t>(NSt);
    a.keep = ctx.scratch.alloc<uint8_t>(NSt);
    a.gain = ctx.scratch.alloc<long long>(NSt);
    a.layer = ctx.scratch.alloc<unsigned long long>(NSt);
    a.try_ov = ctx.scratch.alloc<unsigned long long>((size_t)reps * maxs * tries);
    a.try_cut = ctx.scratch.alloc<long long>((size_t)reps * maxs * tries);
    a.seed = kn.seed;
    a.tries = tries;
    a.jet_iters = kn.ip_jet_iters;
    a.jet_patience = kn.ip_jet_patience;
    a.jet_c = kn.jet_c;
    a.bal_iters = kn.bal_iters;
    a.eps = eps;
    a.smem_bytes = kIpSmem;
    static bool smem_set[64] = {};
    if (!smem_set[ctx.device & 63]) {
        KB_CUDA(cudaFuncSetAttribute(ip_try<kTryMaxBT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kIpSmem));
        KB_CUDA(cudaFuncSetAttribute(ip_try<1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, kIpSmem));
        smem_set[ctx.device & 63] = true;
    }
    a.err = ctx.dscalars + 60;
    KB_CUDA(cudaMemsetAsync(a.part, 0, sizeof(int) * (size_t)reps * n, st));
    {
        PhaseScope ps(ctx, "initial_device", 0);
        size_t eoff = 0;
        for (size_t d = 0; d < so.size(); ++d) {
            a.depth = (int)d;
            a.nsplit = (int)so[d].size();
            a.split_eb = deb + eoff;
            eoff += (size_t)a.nsplit;
            a.split_o = dtab + toff[d];
            a.split_k = a.split_o + a.nsplit;
            a.sidx = a.split_k + a.nsplit;
            KB_CUDA(cudaMemsetAsync(a.cnt, 0, sizeof(unsigned) * (size_t)reps * a.nsplit, st));
            KB_CUDA(cudaMemsetAsync(a.deg, 0, sizeof(unsigned) * (size_t)reps * a.nsplit, st));
            const long long tot = (long long)reps * n;
            ip_count<<<(int)std::max<long long>(1, std::min<long long>(div_up(tot, 256), (long long)kNumSMs * 8)), 256, 0,
                       st>>>(a);
            KB_LAUNCH();
            ip_bases<<<1, kBT, 0, st>>>(a);
            KB_LAUNCH();
            ip_extract<<<a.nsplit * reps, kTryMaxBT, 0, st>>>(a);
            KB_LAUNCH();
            // threads and shared memory per try from the expected subgraph
            // size at this depth (a larger subgraph falls back to global
            // memory for what does not fit)
            const double share = 1.1 / (double)(1LL << std::min<size_t>(d, 40));
            const long long n_est = (long long)(share * n) + 2, m_est = (long long)(share * (double)c.m);
            // (fewer threads on small subgraphs measured slower: a try's
            // passes run longer per thread than its barriers cost)
            // (the rows only when they fit beside the working state)
            const long long state = n_est * kIpSmemPerNode + 512;
            const long long want = state + 8 * m_est <= kIpSmem ? state + 8 * m_est : state;
            a.smem_bytes = (int)std::min<long long>(kIpSmem, (want + 1023) & ~1023LL);
            // large or dense subgraphs: a whole SM's threads per try
            if (n_est > 8192 || (m_est >= 65536 && m_est >= (long long)kDenseRows * n_est)) {
                ip_try<1024><<<a.nsplit * reps * tries, 1024, a.smem_bytes, st>>>(a);
            } else {
                const int bt = n_est > 2048 ? kTryMaxBT : 256;
                ip_try<kTryMaxBT><<<a.nsplit * reps * tries, bt, a.smem_bytes, st>>>(a);
            }
            KB_LAUNCH();
            ip_select<<<a.nsplit * reps, kBT, 0, st>>>(a);
            KB_LAUNCH();
        }
    }
    // the repetition of the smallest cut (the first on ties)
    int win = 0;
    if (reps > 1) {
        uint32_t* bw = ctx.scratch.alloc<uint32_t>((size_t)k);
        unsigned long long* c2 = reinterpret_cast<unsigned long long*>(ctx.dscalars + 32);
        long long bestc = LLONG_MAX;
        for (int r = 0; r < reps; ++r) {
            block_weights_and_cut(ctx, c, a.part + (size_t)r * n, k, bw, c2);
            unsigned long long h = 0;
            KB_CUDA(cudaMemcpyAsync(&h, c2, sizeof(h), cudaMemcpyDeviceToHost, st));
            KB_CUDA(cudaStreamSynchronize(st));
            if ((long long)(h / 2) < bestc) { bestc = (long long)(h / 2); win = r; }
        }
    }
    KB_CUDA(cudaMemcpyAsync(part, a.part + (size_t)win * n, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    KB_CUDA(cudaStreamSynchronize(st));
    ctx.scratch.release(mk);
}

}  // namespace kb
