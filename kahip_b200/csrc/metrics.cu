// metrics.cu -- edge cut and block weights (quality_metrics.cpp:23-37),
// projection (graph_hierarchy.cpp:54-58), max degree, label initialisation.
#include "lp.cuh"
#include "prims.cuh"

namespace kb {

namespace {

// One thread per vertex, block-local histogram of block weights when k fits
// into shared memory, warp-then-block reduction of the cut.  The row is read
// four entries at a time (all loads issued before the block ids are
// compared); UNIT: every edge weight is 1 (adjwgt is not read).
template <bool UNIT>
__global__ void cut_bw_kernel(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                              const int* __restrict__ adjwgt, const int* __restrict__ vwgt,
                              const int* __restrict__ part, int k, uint32_t* bw,
                              unsigned long long* cut2, int use_smem) {
    extern __shared__ uint32_t hist[];
    if (use_smem)
        for (int b = threadIdx.x; b < k; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    unsigned long long c = 0;
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(base + threadIdx.x);
        const bool ok = v < n;
        const int p = ok ? part[v] : -1;
        // neighbouring vertices mostly share a block: one atomic per block
        // id present in the warp
        const unsigned peers = __match_any_sync(0xffffffffu, p);
        const uint32_t wsum = __reduce_add_sync(peers, ok ? (uint32_t)vwgt[v] : 0u);
        if (ok && lane == __ffs(peers) - 1) {
            if (use_smem) atomicAdd(&hist[p], wsum);
            else atomicAdd(&bw[p], wsum);
        }
        if (!ok) continue;
        if (cut2) {
            const int beg = xadj[v], end = xadj[v + 1];
            int e = beg;
            for (; e + 4 <= end; e += 4) {
                int u[4];
                long long w[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    u[t] = adjncy[e + t];
                    w[t] = UNIT ? 1 : (long long)adjwgt[e + t];
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) u[t] = part[u[t]];
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (u[t] != p) c += (unsigned long long)w[t];
            }
            for (; e < end; ++e)
                if (part[adjncy[e]] != p) c += UNIT ? 1ull : (unsigned long long)(long long)adjwgt[e];
        }
    }
    __syncthreads();
    if (use_smem)
        for (int b = threadIdx.x; b < k; b += blockDim.x)
            if (hist[b]) atomicAdd(&bw[b], hist[b]);
    if (cut2) {
        for (int o = 16; o >= 1; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0 && c) atomicAdd(cut2, c);
    }
}

__global__ void project_kernel(int n, const int* __restrict__ cmap, const int* __restrict__ pc,
                               int* __restrict__ pf, const uint8_t* __restrict__ cb, uint8_t* __restrict__ fb) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int c = cmap[v];
        pf[v] = pc[c];
        if (fb) fb[v] = cb[c];
    }
}

// out[v] = 1 when a neighbour of v lies in another block (rows read four
// entries at a time, stopping at the first such neighbour)
__global__ void boundary_kernel(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                                const int* __restrict__ part, uint8_t* __restrict__ out) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int p = part[v], e1 = xadj[v + 1];
        int e = xadj[v];
        bool b = false;
        for (; !b && e + 4 <= e1; e += 4) {
            const int u0 = adjncy[e], u1 = adjncy[e + 1], u2 = adjncy[e + 2], u3 = adjncy[e + 3];
            b = (part[u0] != p) | (part[u1] != p) | (part[u2] != p) | (part[u3] != p);
        }
        for (; !b && e < e1; ++e) b = part[adjncy[e]] != p;
        out[v] = b ? 1 : 0;
    }
}

// out[0] = max degree, out[1] = isolated vertices, out[2] = their largest weight
__global__ void maxdeg_kernel(int n, const int* __restrict__ xadj, const int* __restrict__ vwgt, int* out) {
    int m = 0;
    unsigned iso = 0, w = 0, wall = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int d = xadj[v + 1] - xadj[v];
        const unsigned wv = (unsigned)vwgt[v];
        m = max(m, d);
        wall = max(wall, wv);
        if (d == 0) {
            ++iso;
            w = max(w, wv);
        }
    }
    for (int o = 16; o >= 1; o >>= 1) {
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        iso += __shfl_xor_sync(0xffffffffu, iso, o);
        w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
        wall = max(wall, __shfl_xor_sync(0xffffffffu, wall, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, m);
        if (iso) atomicAdd(reinterpret_cast<unsigned*>(out + 1), iso);
        if (w) atomicMax(reinterpret_cast<unsigned*>(out + 2), w);
        if (wall) atomicMax(reinterpret_cast<unsigned*>(out + 3), wall);
    }
}

// flag[v] = 1 for isolated vertices
__global__ void iso_flags(int n, const int* __restrict__ xadj, uint32_t* flag) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        flag[v] = xadj[v + 1] == xadj[v] ? 1u : 0u;
}

// ids[rank] = v for isolated v (rank = exclusive prefix count)
__global__ void iso_ids(int n, const int* __restrict__ xadj, const uint32_t* __restrict__ rank, int* ids) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        if (xadj[v + 1] == xadj[v]) ids[rank[v]] = v;
}

__global__ void iso_label(int n, const int* __restrict__ xadj, const uint32_t* __restrict__ rank,
                          const int* __restrict__ ids, uint32_t group, int* label) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        if (xadj[v + 1] == xadj[v]) label[v] = ids[(rank[v] / group) * group];
}

__global__ void leaders_kernel(int n, const int* __restrict__ label, unsigned* out) {
    unsigned c = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) c += label[v] == v;
    for (int o = 16; o >= 1; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void init_labels_kernel(int n, const int* __restrict__ vwgt, int* label, uint32_t* cw) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        label[v] = v;
        cw[v] = (uint32_t)vwgt[v];
    }
}

// One pass over the graph, a warp per 32 consecutive vertices: the warp
// walks the entry range of its vertices in coalesced 32-entry chunks.
// Flags: 1 target out of range, 2 negative edge weight, 4 negative node
// weight, 8 xadj not starting at 0 or not monotone (or outside [0, m]), 16
// some edge weight other than 1, 32 some row not listing its targets in
// strictly increasing order (not an error; lets the first clustering round
// skip aggregation).  *wsum = the node weights' sum (32-bit, wrapping as the
// reference's NodeWeight does).
__global__ void check_graph_kernel(int n, long long m, const int* __restrict__ xadj,
                                   const int* __restrict__ adjncy, const int* __restrict__ adjwgt,
                                   const int* __restrict__ vwgt, int* flags, unsigned* wsum, int v_lo, int v_hi,
                                   unsigned* ds) {
    int f = 0;
    unsigned w = 0;
    // degree statistics (what degree_stats computes): [0] max degree,
    // [1] isolated nodes, [2] their largest weight, [3] largest node weight
    unsigned md = 0, iso = 0, wi = 0, wa = 0;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    for (long long g0 = v_lo + ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32 * 32; g0 < v_hi;
         g0 += warps * 32) {
        const long long v = g0 + lane;
        const bool in = v < v_hi;
        long long x0 = 0, x1 = 0;
        if (in) {
            x0 = xadj[v];
            x1 = xadj[v + 1];
            const int vw = vwgt[v];
            if (vw < 0) f |= 4;
            w += (unsigned)vw;
            const unsigned d = x0 >= 0 && x1 >= x0 ? (unsigned)min(x1 - x0, (long long)INT_MAX) : 0u;
            md = max(md, d);
            wa = max(wa, (unsigned)vw);
            if (d == 0) {
                ++iso;
                wi = max(wi, (unsigned)vw);
            }
        }
        const bool sane = !in || (x0 >= 0 && x0 <= x1 && x1 <= m);
        if (!__all_sync(0xffffffffu, sane)) {
            f |= 8;
            continue;
        }
        const int last = (int)min(31LL, (long long)v_hi - 1 - g0);
        const long long lo = __shfl_sync(0xffffffffu, x0, 0), hi = __shfl_sync(0xffffffffu, x1, last);
        int carry = 0;
        // four chunks of 32 entries in flight per step (latency-bound otherwise)
        for (long long base0 = lo; base0 < hi; base0 += 128) {
            int tt[4], ww[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const long long e = base0 + 32 * c + lane;
                tt[c] = 0;
                ww[c] = 1;
                if (e < hi) {
                    tt[c] = adjncy[e];
                    if (adjwgt) ww[c] = adjwgt[e];  // null: unit weights, known on the host
                }
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const long long base = base0 + 32 * c;
                if (base >= hi) break;  // warp-uniform
                const bool ein = base + lane < hi;
                const int t = tt[c];
                if (ein) {
                    if (t < 0 || t >= n) f |= 1;
                    if (ww[c] < 0) f |= 2;
                    if (ww[c] != 1) f |= 16;
                }
                // the row starts that fall into this chunk
                const unsigned bit = (in && x0 >= base && x0 < base + 32) ? 1u << (int)(x0 - base) : 0u;
                const unsigned starts = __reduce_or_sync(0xffffffffu, bit);
                const int up = __shfl_up_sync(0xffffffffu, t, 1);
                const int prev = lane == 0 ? carry : up;
                if (ein && !((starts >> lane) & 1u) && t <= prev) f |= 32;
                carry = __shfl_sync(0xffffffffu, t, 31);
            }
        }
    }
    if (v_lo == 0 && blockIdx.x == 0 && threadIdx.x == 0 && xadj[0] != 0) f |= 8;
    f = __reduce_or_sync(0xffffffffu, f);
    w = __reduce_add_sync(0xffffffffu, w);
    md = __reduce_max_sync(0xffffffffu, md);
    iso = __reduce_add_sync(0xffffffffu, iso);
    wi = __reduce_max_sync(0xffffffffu, wi);
    wa = __reduce_max_sync(0xffffffffu, wa);
    if ((threadIdx.x & 31) == 0) {
        if (f) atomicOr(flags, f);
        if (w) atomicAdd(wsum, w);
        if (md) atomicMax(ds, md);
        if (iso) atomicAdd(ds + 1, iso);
        if (wi) atomicMax(ds + 2, wi);
        if (wa) atomicMax(ds + 3, wa);
    }
}

__global__ void rows_sorted_kernel(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                                   int* bad) {
    int f = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        for (int e = xadj[v] + 1; e < xadj[v + 1]; ++e)
            if (adjncy[e] <= adjncy[e - 1]) f = 1;
    f = __reduce_or_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && f) atomicOr(bad, 1);
}

int grid_for(long long n, int threads) {
    return (int)std::max<long long>(1, std::min<long long>(div_up(n, threads), (long long)kNumSMs * 16));
}

}  // namespace

void block_weights_and_cut(Ctx& ctx, const DevGraph& g, const int* part, int k, uint32_t* bw,
                           unsigned long long* cut2) {
    cudaStream_t st = ctx.stream;
    KB_CUDA(cudaMemsetAsync(bw, 0, sizeof(uint32_t) * (size_t)k, st));
    if (cut2) KB_CUDA(cudaMemsetAsync(cut2, 0, sizeof(unsigned long long), st));
    if (g.n == 0) return;
    int use_smem = k <= 12288;
    size_t smem = use_smem ? sizeof(uint32_t) * (size_t)k : 0;
    PhaseScope ps(ctx, cut2 ? "cut_and_weights" : "block_weights",
                  cut2 ? (g.unit_weights ? 8.0 : 12.0) * g.m + 12.0 * g.n : 8.0 * g.n);
    if (g.unit_weights)
        cut_bw_kernel<true><<<grid_for(g.n, 256), 256, smem, st>>>(g.n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, part, k,
                                                                   bw, cut2, use_smem);
    else
        cut_bw_kernel<false><<<grid_for(g.n, 256), 256, smem, st>>>(g.n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, part,
                                                                    k, bw, cut2, use_smem);
    KB_LAUNCH();
}

void project(Ctx& ctx, int n, const int* cmap, const int* part_coarse, int* part_fine, const uint8_t* cb,
             uint8_t* fb) {
    if (n == 0) return;
    PhaseScope ps(ctx, "project", 12.0 * n);
    project_kernel<<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, cmap, part_coarse, part_fine, cb, fb);
    KB_LAUNCH();
}

void boundary_flags(Ctx& ctx, const DevGraph& g, const int* part, uint8_t* out) {
    if (g.n == 0) return;
    PhaseScope ps(ctx, "boundary", 8.0 * g.m + 9.0 * g.n);
    boundary_kernel<<<grid_for(g.n, 256), 256, 0, ctx.stream>>>(g.n, g.xadj, g.adjncy, part, out);
    KB_LAUNCH();
}

void degree_stats(Ctx& ctx, DevGraph& g) {
    g.maxdeg = 0;
    g.iso_count = g.iso_wmax = g.maxvw = 0;
    if (g.n == 0) return;
    // [8] max degree, [9] isolated count, [10] their max weight, [11] max node weight
    int* d = ctx.dscalars + 8;
    KB_CUDA(cudaMemsetAsync(d, 0, 4 * sizeof(int), ctx.stream));
    maxdeg_kernel<<<grid_for(g.n, 256), 256, 0, ctx.stream>>>(g.n, g.xadj, g.vwgt, d);
    KB_LAUNCH();
    KB_CUDA(cudaMemcpyAsync(ctx.pinned + 8, d, 4 * sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    g.maxdeg = (int)ctx.pinned[8];
    g.iso_count = ctx.pinned[9];
    g.iso_wmax = ctx.pinned[10];
    g.maxvw = ctx.pinned[11];
}

int max_degree(Ctx& ctx, const DevGraph& g) {
    DevGraph h = g;
    degree_stats(ctx, h);
    return h.maxdeg;
}

void check_graph_begin(Ctx& ctx) {
    KB_CUDA(cudaMemsetAsync(ctx.dscalars + 2, 0, 2 * sizeof(int), ctx.stream));  // [2] flags, [3] weight sum
    KB_CUDA(cudaMemsetAsync(ctx.dscalars + 8, 0, 4 * sizeof(int), ctx.stream));  // [8..11] degree statistics
}

void check_graph_range(Ctx& ctx, const DevGraph& g, int v_lo, int v_hi, bool unit_known) {
    if (v_hi <= v_lo && !(v_lo == 0 && g.n == 0)) return;
    int* d = ctx.dscalars + 2;
    check_graph_kernel<<<grid_for((long long)std::max(v_hi - v_lo, 1), 256), 256, 0, ctx.stream>>>(
        g.n, g.m, g.xadj, g.adjncy, unit_known ? nullptr : g.adjwgt, g.vwgt, d, reinterpret_cast<unsigned*>(d + 1),
        v_lo, v_hi, reinterpret_cast<unsigned*>(ctx.dscalars + 8));
    KB_LAUNCH();
}

int check_graph_end(Ctx& ctx, uint32_t* total_weight, DevGraph* stats) {
    KB_CUDA(cudaMemcpyAsync(ctx.pinned + 2, ctx.dscalars + 2, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaMemcpyAsync(ctx.pinned + 8, ctx.dscalars + 8, 4 * sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    if (total_weight) *total_weight = ctx.pinned[3];
    if (stats) {
        stats->maxdeg = (int)ctx.pinned[8];
        stats->iso_count = ctx.pinned[9];
        stats->iso_wmax = ctx.pinned[10];
        stats->maxvw = ctx.pinned[11];
        stats->stats_known = true;
    }
    return (int)ctx.pinned[2];
}

int check_graph(Ctx& ctx, const DevGraph& g, uint32_t* total_weight, DevGraph* stats) {
    check_graph_begin(ctx);
    if (g.m > 0 || g.n > 0) check_graph_range(ctx, g, 0, g.n, false);
    return check_graph_end(ctx, total_weight, stats);
}

bool rows_strictly_increasing(Ctx& ctx, const DevGraph& g) {
    if (g.n == 0) return true;
    int* d = ctx.dscalars + 4;
    KB_CUDA(cudaMemsetAsync(d, 0, sizeof(int), ctx.stream));
    rows_sorted_kernel<<<grid_for(g.n, 256), 256, 0, ctx.stream>>>(g.n, g.xadj, g.adjncy, d);
    KB_LAUNCH();
    KB_CUDA(cudaMemcpyAsync(ctx.pinned + 4, d, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    return ctx.pinned[4] == 0;
}

void bundle_isolated(Ctx& ctx, const DevGraph& g, uint32_t bound, int* label) {
    const uint32_t count = g.iso_count, wmax = g.iso_wmax;
    if (g.n < 2 || bound < 2 || count < 2) return;
    const uint32_t group = wmax == 0 ? count : (bound - 1) / wmax;
    if (group < 2) return;
    cudaStream_t s = ctx.stream;
    const size_t mk = ctx.scratch.mark();
    uint32_t* rank = ctx.scratch.alloc<uint32_t>((size_t)g.n);
    int* ids = ctx.scratch.alloc<int>((size_t)g.n);
    PhaseScope ps(ctx, "isolated_bundles", 16.0 * g.n);
    iso_flags<<<grid_for(g.n, 256), 256, 0, s>>>(g.n, g.xadj, rank);
    KB_LAUNCH();
    exclusive_scan_u32(rank, rank, g.n, nullptr, s, ctx.scratch);
    iso_ids<<<grid_for(g.n, 256), 256, 0, s>>>(g.n, g.xadj, rank, ids);
    KB_LAUNCH();
    iso_label<<<grid_for(g.n, 256), 256, 0, s>>>(g.n, g.xadj, rank, ids, group, label);
    KB_LAUNCH();
    ctx.scratch.release(mk);
}

long long count_leaders(Ctx& ctx, int n, const int* label) {
    if (n == 0) return 0;
    unsigned* d = reinterpret_cast<unsigned*>(ctx.dscalars + 12);
    KB_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned), ctx.stream));
    leaders_kernel<<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, label, d);
    KB_LAUNCH();
    KB_CUDA(cudaMemcpyAsync(ctx.pinned + 12, d, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    return (long long)ctx.pinned[12];
}

void init_labels(Ctx& ctx, const DevGraph& g, int* label, uint32_t* cw) {
    if (g.n == 0) return;
    init_labels_kernel<<<grid_for(g.n, 256), 256, 0, ctx.stream>>>(g.n, g.vwgt, label, cw);
    KB_LAUNCH();
}

}  // namespace kb
