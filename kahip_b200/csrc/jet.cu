// jet.cu -- Jet refinement on the device (Gilbert, Madduri, Boman,
// Rajamanickam, "Jet: Multilevel Graph Partitioning on GPUs", 2023), the
// synchronous form restated by the oracle (or_jet_refine); it stands in for
// the reference's k-way FM (kway_graph_refinement_core.cpp:47-171).
//
// One iteration:
//   jet_choose   every vertex not moved in the previous iteration finds its
//                most connected other block d (register slots, lane per
//                vertex; rows with more than kSlots distinct blocks or more
//                than kLaneRow entries go to jet_choose_wide, a block per
//                vertex with a dense per-block counter array); it is a
//                candidate when 4 (conn(d) - conn(own)) >= -c4 conn(own);
//   jet_afterburn the candidate's gain recomputed with its higher-priority
//                neighbours (larger gain, then smaller id) already moved;
//                kept when >= 0;
//   jet_apply    moves, block weights (integer atomics: order-free).
// Then the host repairs the balance if needed (balance()).  The partition
// an iteration leaves is judged at the start of the next one: jet_choose
// scans every row anyway, so it also sums the cut of the partition it reads
// (locked rows included), and the block weights are kept current by
// jet_apply and balance(); the best partition by (overload, cut) is kept.
// Only an iteration cap that ends the loop needs a separate cut pass.
#include "jet.cuh"

#include <vector>

#include "common.cuh"
#include "prims.cuh"

namespace kb {

namespace {

constexpr int kThreads = 256;
constexpr int kSlots = 8;
constexpr int kLaneRow = 256;
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kLocked = 0x40000000;  // wide-list flag: the row only adds to the cut (n < 2^30)

struct JetArgs {
    int n, k;
    const int* xadj;
    const int* adjncy;
    const int* adjwgt;
    const int* part;
    const int* moved_at;
    int it;
    int c4;
    uint64_t ks_tie;
    int* dest;
    long long* gain;
    int* wide;           // vertices left to jet_choose_wide (| kLocked for locked rows)
    unsigned* nwide;
    unsigned long long* cut2;  // twice the cut of part, summed by the choose kernels
};

__device__ __forceinline__ void add_cut(const JetArgs& A, unsigned long long c) {
#pragma unroll
    for (int off = 16; off; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(A.cut2, c);
}

// (conn desc, hash asc, id asc)
__device__ __forceinline__ bool beats(uint32_t cb, uint32_t b, uint32_t ca, uint32_t a, uint64_t ks) {
    if (cb != ca) return cb > ca;
    const uint32_t hb = hash32(ks, b), ha = hash32(ks, a);
    if (hb != ha) return hb < ha;
    return b < a;
}

__device__ __forceinline__ void candidate(const JetArgs& A, int v, int own, long long co, uint32_t d, uint32_t dc) {
    if (d == kNone) return;
    const long long gv = (long long)dc - co;
    if (4 * gv >= -(long long)A.c4 * co) {
        A.dest[v] = (int)d;
        A.gain[v] = gv;
    }
}

__global__ void __launch_bounds__(kThreads) jet_choose(JetArgs A) {
    unsigned long long cut = 0;
    for (long long v0 = (long long)blockIdx.x * kThreads + threadIdx.x; v0 < A.n; v0 += (long long)gridDim.x * kThreads) {
        const int v = (int)v0;
        A.dest[v] = -1;
        const bool locked = A.moved_at[v] == A.it - 1;
        const int beg = A.xadj[v], end = A.xadj[v + 1];
        if (end - beg > kLaneRow) {
            A.wide[atomicAdd(A.nwide, 1u)] = locked ? (v | kLocked) : v;
            continue;
        }
        const int own = A.part[v];
        if (locked) {
            for (int e = beg; e < end; ++e)
                if (A.part[A.adjncy[e]] != own) cut += (uint32_t)A.adjwgt[e];
            continue;
        }
        uint32_t sl[kSlots], sc[kSlots];
#pragma unroll
        for (int i = 0; i < kSlots; ++i) { sl[i] = kNone; sc[i] = 0; }
        long long co = 0;
        unsigned long long other = 0;
        bool overflow = false;
        for (int e = beg; e < end && !overflow; ++e) {
            const uint32_t b = (uint32_t)A.part[A.adjncy[e]];
            const uint32_t w = (uint32_t)A.adjwgt[e];
            if ((int)b == own) { co += w; continue; }
            other += w;
            bool hit = false;
#pragma unroll
            for (int i = 0; i < kSlots; ++i) {
                const bool m = sl[i] == b;
                sc[i] += m ? w : 0u;
                hit |= m;
            }
            if (!hit) {
                overflow |= sl[kSlots - 1] != kNone;
#pragma unroll
                for (int i = kSlots - 1; i > 0; --i) { sl[i] = sl[i - 1]; sc[i] = sc[i - 1]; }
                sl[0] = b;
                sc[0] = w;
            }
        }
        if (overflow) {
            // the row is scanned again, and its cut summed, by jet_choose_wide
            A.wide[atomicAdd(A.nwide, 1u)] = v;
            continue;
        }
        cut += other;
        uint32_t d = kNone, dc = 0;
#pragma unroll
        for (int i = 0; i < kSlots; ++i)
            if (sl[i] != kNone && sc[i] > 0 && (d == kNone || beats(sc[i], sl[i], dc, d, A.ks_tie))) {
                d = sl[i];
                dc = sc[i];
            }
        candidate(A, v, own, co, d, dc);
    }
    add_cut(A, cut);
}

// Block per listed vertex; cnt = this block's k counters (zero between
// vertices: every touched counter is read and cleared).
__global__ void __launch_bounds__(kThreads) jet_choose_wide(JetArgs A, uint32_t* counters) {
    __shared__ uint64_t sk[kThreads / 32];
    __shared__ uint32_t sb[kThreads / 32];
    uint32_t* cnt = counters + (size_t)blockIdx.x * A.k;
    const unsigned count = *A.nwide;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long cut = 0;
    for (unsigned i = blockIdx.x; i < count; i += gridDim.x) {
        const int raw = A.wide[i];
        const int v = raw & ~kLocked;
        const int beg = A.xadj[v], end = A.xadj[v + 1];
        const int own = A.part[v];
        if (raw & kLocked) {
            // block-uniform branch: a locked row only adds to the cut
            for (int e = beg + threadIdx.x; e < end; e += kThreads)
                if (A.part[A.adjncy[e]] != own) cut += (uint32_t)A.adjwgt[e];
            continue;
        }
        for (int e = beg + threadIdx.x; e < end; e += kThreads) {
            const int b = A.part[A.adjncy[e]];
            const uint32_t x = (uint32_t)A.adjwgt[e];
            atomicAdd(&cnt[b], x);
            if (b != own) cut += x;
        }
        __syncthreads();
        const long long co = cnt[own];
        __syncthreads();
        // best other block: each thread scans the targets of its entries
        // (a block can be seen many times; the key is the same each time)
        uint32_t d = kNone, dc = 0;
        for (int e = beg + threadIdx.x; e < end; e += kThreads) {
            const uint32_t b = (uint32_t)A.part[A.adjncy[e]];
            if ((int)b == own) continue;
            const uint32_t c = cnt[b];
            if (c > 0 && (d == kNone || beats(c, b, dc, d, A.ks_tie))) { d = b; dc = c; }
        }
        // block arg-max: pack (conn, ~hash, ~id) so that larger = better
        uint64_t key = d == kNone ? 0ull : (((uint64_t)dc << 32) | (uint32_t)~hash32(A.ks_tie, d));
        uint32_t id = d;
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            const uint64_t ok = __shfl_xor_sync(0xffffffffu, key, off);
            const uint32_t oi = __shfl_xor_sync(0xffffffffu, id, off);
            if (ok > key || (ok == key && oi < id)) { key = ok; id = oi; }
        }
        if (lane == 0) { sk[w] = key; sb[w] = id; }
        __syncthreads();
        // clear the counters this vertex touched
        for (int e = beg + threadIdx.x; e < end; e += kThreads) cnt[A.part[A.adjncy[e]]] = 0;
        if (threadIdx.x == 0) {
            uint64_t bk = sk[0];
            uint32_t bi = sb[0];
            for (int j = 1; j < kThreads / 32; ++j)
                if (sk[j] > bk || (sk[j] == bk && sb[j] < bi)) { bk = sk[j]; bi = sb[j]; }
            if (bk != 0ull) candidate(A, v, own, co, bi, (uint32_t)(bk >> 32));
        }
        __syncthreads();
    }
    add_cut(A, cut);
}

__device__ __forceinline__ long long afterburn_sum(const JetArgs& A, int v, int beg, int end, int step, int first) {
    const int dv = A.dest[v], pv = A.part[v];
    const long long gv = A.gain[v];
    long long adj = 0;
    for (int e = beg + first; e < end; e += step) {
        const int u = A.adjncy[e];
        int bu = A.part[u];
        const int du = A.dest[u];
        if (du >= 0) {
            const long long gu = A.gain[u];
            if (gu > gv || (gu == gv && u < v)) bu = du;
        }
        if (bu == dv) adj += A.adjwgt[e];
        else if (bu == pv) adj -= A.adjwgt[e];
    }
    return adj;
}

__global__ void __launch_bounds__(kThreads) jet_afterburn(JetArgs A, uint8_t* keep, const int* stop) {
    if (*stop) return;  // the loop ended at this iteration's evaluation
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * kThreads; base < A.n; base += (long long)gridDim.x * kThreads) {
        const int v = (int)(base + threadIdx.x);
        const bool cand = v < A.n && A.dest[v] >= 0;
        int beg = 0, end = 0;
        if (cand) { beg = A.xadj[v]; end = A.xadj[v + 1]; }
        const bool wide = cand && end - beg > kLaneRow;
        if (v < A.n) keep[v] = 0;
        unsigned wm = __ballot_sync(0xffffffffu, wide);
        while (wm) {
            const int s = __ffs(wm) - 1;
            wm &= wm - 1;
            const int hv = __shfl_sync(0xffffffffu, v, s);
            const int hb = __shfl_sync(0xffffffffu, beg, s), he = __shfl_sync(0xffffffffu, end, s);
            long long adj = afterburn_sum(A, hv, hb, he, 32, lane);
#pragma unroll
            for (int off = 16; off; off >>= 1) adj += __shfl_xor_sync(0xffffffffu, adj, off);
            if (lane == s) keep[hv] = adj >= 0 ? 1 : 0;
        }
        if (cand && !wide) keep[v] = afterburn_sum(A, v, beg, end, 1, 0) >= 0 ? 1 : 0;
    }
}

__global__ void jet_apply(int n, int it, const uint8_t* keep, const int* dest, const int* vwgt, int* part,
                          int* moved_at, uint32_t* bw, unsigned* moved, const int* stop) {
    if (*stop) return;
    unsigned c = 0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        if (!keep[v]) continue;
        const uint32_t w = (uint32_t)vwgt[v];
        atomicSub(&bw[part[v]], w);
        atomicAdd(&bw[dest[v]], w);
        part[v] = dest[v];
        moved_at[v] = it;
        ++c;
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(moved, c);
}

// The loop's state on the device, so that the host reads it once per
// iteration: the best (overload, cut) so far, iterations since it improved,
// whether the current partition is the best one, and whether the loop ended.
struct JetCtl {
    unsigned long long best_ov;
    long long best_cut;
    int since, stop, part_is_best, pad;
};

// Judges the partition the previous iteration left (cut2 summed by this
// iteration's choose kernels, bw current): best tracking, then the stopping
// rule (a move-less iteration, jet_patience iterations without a better
// partition, or the iteration cap).  One block.
__global__ void jet_track(JetCtl* c, const uint32_t* bw, int k, uint32_t bound, const unsigned long long* cut2,
                          const unsigned* moved, int it, int iters, int patience) {
    __shared__ unsigned long long red[32];
    if (c->stop) return;
    unsigned long long ov = 0;
    for (int b = threadIdx.x; b < k; b += blockDim.x)
        if (bw[b] > bound) ov += bw[b] - bound;
#pragma unroll
    for (int off = 16; off; off >>= 1) ov += __shfl_xor_sync(0xffffffffu, ov, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ov;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) ov += red[w];
        const long long cut = (long long)(*cut2 / 2);
        if (it == 0 || ov < c->best_ov || (ov == c->best_ov && cut < c->best_cut)) {
            c->best_ov = ov;
            c->best_cut = cut;
            c->part_is_best = 1;
            c->since = 0;
        } else {
            c->part_is_best = 0;
            ++c->since;
        }
        c->stop = ((it > 0 && (*moved == 0 || c->since >= patience)) || it == iters) ? 1 : 0;
    }
}

// best <- part (and the block weights) when the loop goes on from a new best
__global__ void jet_save(const JetCtl* c, int n, int k, const int* part, const uint32_t* bw, int* best,
                         uint32_t* best_bw) {
    if (c->stop || !c->part_is_best) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        best[i] = part[i];
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < k; b += gridDim.x * blockDim.x) best_bw[b] = bw[b];
}

// part <- best when the loop ended away from its best partition
__global__ void jet_restore(const JetCtl* c, int n, int k, int* part, uint32_t* bw, const int* best,
                            const uint32_t* best_bw) {
    if (c->part_is_best) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        part[i] = best[i];
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < k; b += gridDim.x * blockDim.x) bw[b] = best_bw[b];
}

__global__ void fill_i32_kernel(int n, int v, int* p) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

int grid_for(long long items) {
    return (int)std::max<long long>(1, std::min<long long>(div_up(items, kThreads), (long long)kNumSMs * 16));
}

}  // namespace

void jet_refine(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, uint32_t bound, int* part, uint32_t* bw) {
    if (g.n == 0 || kn.jet_iters <= 0) return;
    cudaStream_t s = ctx.stream;
    const size_t mk = ctx.scratch.mark();
    const int n = g.n, k = kn.k;
    int* best = ctx.scratch.alloc<int>((size_t)n);
    uint32_t* best_bw = ctx.scratch.alloc<uint32_t>((size_t)k);
    int* dest = ctx.scratch.alloc<int>((size_t)n);
    long long* gain = ctx.scratch.alloc<long long>((size_t)n);
    int* moved_at = ctx.scratch.alloc<int>((size_t)n);
    int* wide = ctx.scratch.alloc<int>((size_t)n);
    uint8_t* keep = ctx.scratch.alloc<uint8_t>((size_t)n);
    const int wblocks = 2 * kNumSMs;
    uint32_t* counters = ctx.scratch.alloc<uint32_t>((size_t)wblocks * k);
    unsigned* ctr = reinterpret_cast<unsigned*>(ctx.dscalars + 24);  // [24] wide count, [25] moved
    unsigned long long* cut2 = reinterpret_cast<unsigned long long*>(ctx.dscalars + 32);
    KB_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t) * (size_t)wblocks * k, s));
    fill_i32_kernel<<<grid_for(n), kThreads, 0, s>>>(n, -2, moved_at);
    KB_LAUNCH();
    JetArgs A{};
    A.n = n;
    A.k = k;
    A.xadj = g.xadj;
    A.adjncy = g.adjncy;
    A.adjwgt = g.adjwgt;
    A.part = part;
    A.moved_at = moved_at;
    A.c4 = level == 0 ? kn.jet_c0 : kn.jet_c;
    A.dest = dest;
    A.gain = gain;
    A.wide = wide;
    A.nwide = ctr;
    A.cut2 = cut2;
    // bw holds the block weights of part on entry (the callers keep it
    // current) and stays current: jet_apply and balance() update it.  The
    // best-state bookkeeping and the stopping rule run on the device
    // (jet_track); the host reads the stop flag once per iteration, in the
    // synchronisation that balance() needs anyway.
    JetCtl* ctl = reinterpret_cast<JetCtl*>(ctx.scratch.alloc<unsigned long long>(4));
    KB_CUDA(cudaMemsetAsync(ctl, 0, sizeof(JetCtl), s));
    const int* stop = &ctl->stop;
    for (int it = 0;; ++it) {
        // cut of the partition left by the previous iteration (the input at it = 0)
        KB_CUDA(cudaMemsetAsync(cut2, 0, sizeof(unsigned long long), s));
        if (it < kn.jet_iters) {
            A.it = it;
            A.ks_tie = stream_key(kn.seed, TAG_JTIE, level, it);
            PhaseScope ps(ctx, "jet_choose", 12.0 * (double)g.m + 16.0 * n);
            KB_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned), s));
            jet_choose<<<grid_for(n), kThreads, 0, s>>>(A);
            KB_LAUNCH();
            jet_choose_wide<<<wblocks, kThreads, 0, s>>>(A, counters);
            KB_LAUNCH();
        } else {
            block_weights_and_cut(ctx, g, part, k, bw, cut2);
        }
        {
            PhaseScope ps(ctx, "jet_afterburn", 0);
            jet_track<<<1, 256, 0, s>>>(ctl, bw, k, bound, cut2, ctr + 1, it, kn.jet_iters, kn.jet_patience);
            KB_LAUNCH();
            jet_save<<<grid_for(n), kThreads, 0, s>>>(ctl, n, k, part, bw, best, best_bw);
            KB_LAUNCH();
            jet_afterburn<<<grid_for(n), kThreads, 0, s>>>(A, keep, stop);
            KB_LAUNCH();
            KB_CUDA(cudaMemsetAsync(ctr + 1, 0, sizeof(unsigned), s));
            jet_apply<<<grid_for(n), kThreads, 0, s>>>(n, it, keep, dest, g.vwgt, part, moved_at, bw, ctr + 1, stop);
            KB_LAUNCH();
        }
        KB_CUDA(cudaMemcpyAsync(ctx.pinned + 50, stop, sizeof(int), cudaMemcpyDeviceToHost, s));
        // repairs an overloaded partition (nothing once the loop has ended);
        // synchronises, so the stop flag is on the host afterwards
        balance(ctx, g, kn, level, bound, part, bw, stop);
        if (ctx.pinned[50]) break;
    }
    jet_restore<<<grid_for(n), kThreads, 0, s>>>(ctl, n, k, part, bw, best, best_bw);
    KB_LAUNCH();
    ctx.scratch.release(mk);
}

}  // namespace kb
