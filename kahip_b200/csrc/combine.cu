// combine.cu -- device parts of the KaFFPaE combine operator
// (population.cpp:189-250): two parent partitions constrain the coarsening
// (size_constraint_label_propagation.cpp:175-178 with graph_allready_
// partitioned and combine set: a node only joins clusters of neighbours in
// its own block of both parents).  Here the constraint is applied once per
// level by filtering the edges the clusterings see; contraction still runs
// on the whole level graph, so every cut edge of either parent survives to
// the coarsest graph, where the better parent is the initial partition.
#include "combine.cuh"

#include "common.cuh"
#include "prims.cuh"

namespace kb {

namespace {

constexpr int kThreads = 256;

int grid_for(long long items) {
    return (int)std::max<long long>(1, std::min<long long>(div_up(items, kThreads), (long long)kNumSMs * 16));
}

// warp per vertex: rows of any length stay balanced across lanes
__global__ void filter_count(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                             const int* __restrict__ p1, const int* __restrict__ p2, uint32_t* cnt) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    for (long long v0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; v0 < n; v0 += warps) {
        const int v = (int)v0;
        const int a = p1[v], b = p2[v];
        uint32_t c = 0;
        for (int e = xadj[v] + lane; e < xadj[v + 1]; e += 32) {
            const int u = adjncy[e];
            c += (p1[u] == a && p2[u] == b) ? 1u : 0u;
        }
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) cnt[v] = c;
    }
}

// warp per vertex; kept entries are written in row order (ballot ranks)
__global__ void filter_write(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                             const int* __restrict__ adjwgt, const int* __restrict__ p1, const int* __restrict__ p2,
                             const uint32_t* __restrict__ fx, int* fa, int* fw) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    for (long long v0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; v0 < n; v0 += warps) {
        const int v = (int)v0;
        const int a = p1[v], b = p2[v];
        uint32_t out = fx[v];
        const int beg = xadj[v], end = xadj[v + 1];
        for (int e0 = beg; e0 < end; e0 += 32) {
            const int e = e0 + lane;
            int u = 0;
            bool keep = false;
            if (e < end) {
                u = adjncy[e];
                keep = p1[u] == a && p2[u] == b;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const uint32_t at = out + __popc(m & ((1u << lane) - 1u));
                fa[at] = u;
                fw[at] = adjwgt[e];
            }
            out += __popc(m);
        }
    }
}

__global__ void parents_check(int n, int k, const int* __restrict__ pa, const int* __restrict__ pb, int* bad) {
    int f = 0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        f |= (pa[v] < 0 || pa[v] >= k || pb[v] < 0 || pb[v] >= k) ? 1 : 0;
    f = __reduce_or_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && f) atomicOr(bad, 1);
}

__global__ void parents_down(int n, const int* __restrict__ cmap, const int* __restrict__ p1,
                             const int* __restrict__ p2, int* p1c, int* p2c) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const int c = cmap[v];
        p1c[c] = p1[v];
        p2c[c] = p2[v];
    }
}

}  // namespace

void filter_by_parents(Ctx& ctx, const DevGraph& f, const int* p1, const int* p2, DevGraph& out) {
    cudaStream_t s = ctx.stream;
    out = DevGraph{};
    out.n = f.n;
    out.vwgt = f.vwgt;
    out.unit_weights = f.unit_weights;
    out.rows_sorted = f.rows_sorted;
    uint32_t* fx = ctx.scratch.alloc<uint32_t>((size_t)f.n + 1);
    if (f.n == 0) {
        KB_CUDA(cudaMemsetAsync(fx, 0, sizeof(uint32_t), s));
        out.xadj = reinterpret_cast<const int*>(fx);
        return;
    }
    PhaseScope ps(ctx, "combine_filter", 2.0 * (8.0 * (double)f.m + 16.0 * f.n));
    filter_count<<<grid_for(32LL * f.n), kThreads, 0, s>>>(f.n, f.xadj, f.adjncy, p1, p2, fx);
    KB_LAUNCH();
    exclusive_scan_u32(fx, fx, f.n, fx + f.n, s, ctx.scratch);
    uint32_t m = 0;
    KB_CUDA(cudaMemcpyAsync(&m, fx + f.n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    KB_CUDA(cudaStreamSynchronize(s));
    int* fa = ctx.scratch.alloc<int>((size_t)std::max<uint32_t>(m, 1));
    int* fw = ctx.scratch.alloc<int>((size_t)std::max<uint32_t>(m, 1));
    filter_write<<<grid_for(32LL * f.n), kThreads, 0, s>>>(f.n, f.xadj, f.adjncy, f.adjwgt, p1, p2, fx, fa, fw);
    KB_LAUNCH();
    out.m = m;
    out.xadj = reinterpret_cast<const int*>(fx);
    out.adjncy = fa;
    out.adjwgt = fw;
    degree_stats(ctx, out);
}

bool parents_in_range(Ctx& ctx, int n, int k, const int* pa, const int* pb) {
    int* bad = ctx.dscalars + 44;  // [44] out-of-range flag
    KB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), ctx.stream));
    if (n > 0) {
        parents_check<<<grid_for(n), kThreads, 0, ctx.stream>>>(n, k, pa, pb, bad);
        KB_LAUNCH();
    }
    KB_CUDA(cudaMemcpyAsync(ctx.pinned + 44, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    return ctx.pinned[44] == 0;
}

void parents_to_coarse(Ctx& ctx, int n, const int* cmap, const int* p1, const int* p2, int* p1c, int* p2c) {
    if (n == 0) return;
    parents_down<<<grid_for(n), kThreads, 0, ctx.stream>>>(n, cmap, p1, p2, p1c, p2c);
    KB_LAUNCH();
}

}  // namespace kb
