// match.cu -- heavy-edge matching coarsening on the device.
//
// The reference's fast/eco presets coarsen by matching on the expansion*^2
// rating (random_matching.cpp:20-116 for the first levels, GPA,
// gpa_matching.cpp:25-129, afterwards).  Both are sequential; here the
// matching is the locally-dominant one under a strict total order on edges,
// computed in synchronous rounds:
//   propose: every unmatched vertex v points at the eligible neighbour u
//            whose entry has the largest key (primary = rating, secondary =
//            hash of the unordered pair, then ~(v+u));
//   commit:  mutual pointers match; a vertex with no eligible neighbour is
//            retired (no neighbour can pick it either: eligibility is
//            symmetric).
// The heaviest remaining edge is always mutual, so every round with an
// eligible edge left adds a pair; the result depends only on the graph, the
// ratings and the stream key.
//
// Layout: state[v] >= 0 is v's weight while unmatched, -1 matched, -2
// retired; best[v] the proposal of this round; mate[v] the partner or -1;
// cnt[r] the pairs formed in round r (a round after one with no new pair
// exits at once, so the host never waits between rounds).
#include "match.cuh"

#include "common.cuh"

namespace kb {

namespace {

constexpr int kThreads = 256;
constexpr int kLaneDeg = 32;  // rows longer than this are scanned by the whole warp

struct MatchArgs {
    int n;
    const int* xadj;
    const int* adjncy;
    const int* adjwgt;
    const uint32_t* rq;  // optional per-entry rating
    int* state;
    int* best;
    int* mate;
    unsigned* cnt;
    uint64_t ks;
    uint32_t maxvw;
};

// Primary key: IEEE bits of 1.0*w*w / (uint32)(c(u)*c(v)) (order-preserving
// for non-negative doubles; 0/0 counts as 0), or the supplied rating.
template <bool UNIT, bool ARRAY>
__device__ __forceinline__ uint64_t primary(const MatchArgs& A, int e, uint32_t cv, uint32_t cu) {
    if (ARRAY) return (uint64_t)__ldg(A.rq + e);
    const int w = UNIT ? 1 : __ldg(A.adjwgt + e);
    double r = 1.0 * w * w / (double)(uint32_t)(cu * cv);
    if (r != r) r = 0.0;
    return (uint64_t)__double_as_longlong(r);
}

__device__ __forceinline__ uint64_t secondary(uint64_t ks, uint32_t a, uint32_t b) {
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    const uint32_t h = hash32(ks, hash32(ks, lo) ^ hi);
    return ((uint64_t)h << 32) | (uint32_t)~(lo + hi);
}

struct Best {
    int u = -1;
    uint64_t k1 = 0, k2 = 0;
    __device__ __forceinline__ void offer(int cu, uint64_t a, uint64_t b) {
        if (u < 0 || a > k1 || (a == k1 && b > k2)) {
            u = cu;
            k1 = a;
            k2 = b;
        }
    }
};

template <bool UNIT, bool ARRAY>
__device__ __forceinline__ void consider(const MatchArgs& A, int v, uint32_t cv, int e, int u, int su, Best& b) {
    if (u == v || su < 0) return;
    if ((uint64_t)cv + (uint32_t)su > A.maxvw) return;
    b.offer(u, primary<UNIT, ARRAY>(A, e, cv, (uint32_t)su), secondary(A.ks, (uint32_t)v, (uint32_t)u));
}

template <bool UNIT, bool ARRAY>
__global__ void __launch_bounds__(kThreads) match_propose(MatchArgs A, int r) {
    if (r > 0 && A.cnt[r - 1] == 0) return;
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (kThreads / 32);
    for (long long base = ((long long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)) * 32; base < A.n;
         base += nwarps * 32) {
        const int v = (int)base + lane;
        int sv = -1, beg = 0, end = 0;
        if (v < A.n) {
            sv = A.state[v];
            if (sv >= 0) {
                beg = __ldg(A.xadj + v);
                end = __ldg(A.xadj + v + 1);
            }
        }
        const bool heavy = sv >= 0 && end - beg > kLaneDeg;
        Best b;
        if (sv >= 0 && !heavy) {
            // four entries per step, their loads issued together
            int e = beg;
            for (; e + 4 <= end; e += 4) {
                int u[4], su[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) u[j] = __ldg(A.adjncy + e + j);
#pragma unroll
                for (int j = 0; j < 4; ++j) su[j] = A.state[u[j]];
#pragma unroll
                for (int j = 0; j < 4; ++j) consider<UNIT, ARRAY>(A, v, (uint32_t)sv, e + j, u[j], su[j], b);
            }
            for (; e < end; ++e) {
                const int u = __ldg(A.adjncy + e);
                consider<UNIT, ARRAY>(A, v, (uint32_t)sv, e, u, A.state[u], b);
            }
        }
        unsigned hm = __ballot_sync(0xffffffffu, heavy);
        while (hm) {
            const int src = __ffs(hm) - 1;
            hm &= hm - 1;
            const int hv = __shfl_sync(0xffffffffu, v, src);
            const int hb = __shfl_sync(0xffffffffu, beg, src);
            const int he = __shfl_sync(0xffffffffu, end, src);
            const uint32_t hs = (uint32_t)__shfl_sync(0xffffffffu, sv, src);
            Best c;
            for (int e = hb + lane; e < he; e += 32) {
                const int u = __ldg(A.adjncy + e);
                consider<UNIT, ARRAY>(A, hv, hs, e, u, A.state[u], c);
            }
            // warp arg-max; keys of distinct neighbours differ, so the
            // winner does not depend on the reduction order
#pragma unroll
            for (int off = 16; off; off >>= 1) {
                const int ou = __shfl_xor_sync(0xffffffffu, c.u, off);
                const uint64_t o1 = __shfl_xor_sync(0xffffffffu, c.k1, off);
                const uint64_t o2 = __shfl_xor_sync(0xffffffffu, c.k2, off);
                if (ou >= 0) c.offer(ou, o1, o2);
            }
            if (lane == src) b = c;
        }
        if (sv >= 0) A.best[v] = b.u;
    }
}

__global__ void __launch_bounds__(kThreads) match_commit(MatchArgs A, int r) {
    if (r > 0 && A.cnt[r - 1] == 0) return;
    unsigned pairs = 0;
    for (long long v = (long long)blockIdx.x * kThreads + threadIdx.x; v < A.n; v += (long long)gridDim.x * kThreads) {
        if (A.state[v] < 0) continue;
        const int b = A.best[v];
        if (b >= 0 && A.best[b] == (int)v) {
            A.mate[v] = b;
            A.state[v] = -1;
            pairs += (int)v < b;
        } else if (b < 0) {
            A.state[v] = -2;
        }
    }
    // warp-aggregated count of the pairs formed
#pragma unroll
    for (int off = 16; off; off >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, off);
    if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(A.cnt + r, pairs);
}

__global__ void match_init(int n, const int* vwgt, int* state, int* mate) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        state[v] = vwgt[v];
        mate[v] = -1;
    }
}

__global__ void match_label(int n, const int* mate, int* label) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const int m = mate[v];
        label[v] = (m >= 0 && m < (int)v) ? m : (int)v;
    }
}

int grid_for(long long items) {
    return (int)std::max<long long>(1, std::min<long long>(div_up(items, kThreads), (long long)kNumSMs * 8));
}

template <bool UNIT, bool ARRAY>
void launch_propose(const MatchArgs& A, int r, int grid, cudaStream_t s) {
    match_propose<UNIT, ARRAY><<<grid, kThreads, 0, s>>>(A, r);
}

}  // namespace

void hem_match(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, const uint32_t* rating_q, int* label) {
    if (g.n == 0) return;
    const size_t mk = ctx.scratch.mark();
    cudaStream_t s = ctx.stream;
    const int R = std::max(kn.match_rounds, 0);
    MatchArgs A{};
    A.n = g.n;
    A.xadj = g.xadj;
    A.adjncy = g.adjncy;
    A.adjwgt = g.adjwgt;
    A.rq = rating_q;
    A.state = ctx.scratch.alloc<int>((size_t)g.n);
    A.best = ctx.scratch.alloc<int>((size_t)g.n);
    A.mate = ctx.scratch.alloc<int>((size_t)g.n);
    A.cnt = ctx.scratch.alloc<unsigned>((size_t)std::max(R, 1));
    A.ks = stream_key(kn.seed, TAG_MATCH, level, 0);
    A.maxvw = kn.max_vertex_weight;
    const int grid = grid_for(g.n);
    KB_CUDA(cudaMemsetAsync(A.cnt, 0, sizeof(unsigned) * (size_t)std::max(R, 1), s));
    match_init<<<grid, kThreads, 0, s>>>(g.n, g.vwgt, A.state, A.mate);
    KB_LAUNCH();
    // round 0 scans every row: its algorithmic bytes are exact (per vertex
    // state, xadj, proposal write; per entry adjncy, state gather, plus the
    // weight or supplied rating); later rounds scan only unmatched rows
    const double row_bytes = 4.0 * ((g.unit_weights && !rating_q) ? 2 : 3) * (double)g.m;
    const double round0_bytes = row_bytes + 12.0 * (double)g.n;
    for (int r = 0; r < R; ++r) {
        {
            PhaseScope ps(ctx, r == 0 ? "match_sweep0" : "match_sweep", r == 0 ? round0_bytes : 0.0);
            if (rating_q) launch_propose<false, true>(A, r, grid, s);
            else if (g.unit_weights) launch_propose<true, false>(A, r, grid, s);
            else launch_propose<false, false>(A, r, grid, s);
            KB_LAUNCH();
        }
        PhaseScope ps(ctx, "match_commit", 0);
        match_commit<<<grid, kThreads, 0, s>>>(A, r);
        KB_LAUNCH();
    }
    match_label<<<grid, kThreads, 0, s>>>(g.n, A.mate, label);
    KB_LAUNCH();
    ctx.scratch.release(mk);
}

}  // namespace kb
