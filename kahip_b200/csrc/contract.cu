// contract.cu -- contraction of a clustering into the next coarser graph.
//
// Reference semantics: contraction.cpp:94-133 -> complete_boundary.h:511-562
// (clusters) and contraction.cpp:21-92 + contraction.h:60-82 (matchings):
// coarse node weight = sum of member weights; edges inside a coarse node are
// dropped; parallel coarse edges are merged with summed weights.  Coarse ids
// follow the order of each cluster's smallest member, which is the
// first-appearance order of remap_cluster_ids (size_constraint_label_
// propagation.cpp:207-232).  Rows come out sorted by target.
//
// Pipeline (all on the device):
//   1. leader[c] = min member (atomicMin); prefix sum over leader flags
//      gives coarse ids; cmap gather; coarse node weights (atomicAdd).
//   2. every fine node merges its neighbours by coarse target in register
//      slots and writes (cu<<tb|cv, w) entries into its own CSR range of an
//      m-sized buffer.
//   3. compaction (prefix sum of the per-vertex entry counts).
//   4. stable LSD radix sort on the 2*tb key bits.
//   5. reduce-by-key -> coarse adjncy/adjwgt, row counts -> prefix sum -> xadj.
#include "contract.cuh"
#include "prims.cuh"

#include <climits>

namespace kb {

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kThreads = 256;

int grid_for(long long n, int threads) {
    return (int)std::max<long long>(1, std::min<long long>(div_up(n, threads), (long long)kNumSMs * 16));
}

__global__ void leader_min(int n, const int* __restrict__ label, int* mm) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        atomicMin(&mm[label[v]], v);
}

__global__ void leader_flags(int n, const int* __restrict__ label, const int* __restrict__ mm,
                             uint32_t* flag) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        flag[v] = mm[label[v]] == v ? 1u : 0u;
}

__global__ void make_cmap(int n, const int* __restrict__ label, const int* __restrict__ mm,
                          const uint32_t* __restrict__ pos, const int* __restrict__ vwgt, int* cmap,
                          uint32_t* cvw) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        int c = (int)pos[mm[label[v]]];
        cmap[v] = c;
        atomicAdd(&cvw[c], (uint32_t)vwgt[v]);
    }
}

// One thread per fine vertex: merges its neighbours by coarse target in
// kEmitSlots register slots (edges inside its own coarse node are dropped)
// and writes the (cu<<tb | cv, w) entries into its own CSR range, flushing
// the slots whenever a new target finds them full -- repeated targets that
// this leaves are merged by the sort + reduce that follows.
constexpr int kEmitSlots = 8;

__global__ void __launch_bounds__(kThreads) emit_kernel(int n, const int* __restrict__ xadj,
                                                        const int* __restrict__ adjncy,
                                                        const int* __restrict__ adjwgt,
                                                        const int* __restrict__ cmap, uint64_t* ekey,
                                                        uint32_t* eval, uint32_t* vcount, int tb) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int beg = xadj[v], end = xadj[v + 1];
        const uint32_t own = (uint32_t)cmap[v];
        const uint64_t hi = (uint64_t)own << tb;
        uint32_t st[kEmitSlots], sw[kEmitSlots];
        int used = 0;
        int pos = beg;
        for (int e = beg; e < end; e += 4) {
            int u[4];
            uint32_t w[4], t[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                u[j] = -1;
                w[j] = 0;
                if (e + j < end) {
                    u[j] = adjncy[e + j];
                    w[j] = (uint32_t)adjwgt[e + j];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) t[j] = u[j] >= 0 ? (uint32_t)cmap[u[j]] : kEmpty;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (u[j] < 0 || t[j] == own) continue;
                bool hit = false;
#pragma unroll
                for (int i = 0; i < kEmitSlots; ++i)
                    if (i < used && st[i] == t[j]) { sw[i] += w[j]; hit = true; }
                if (hit) continue;
                if (used == kEmitSlots) {
#pragma unroll
                    for (int i = 0; i < kEmitSlots; ++i) {
                        ekey[pos] = hi | st[i];
                        eval[pos] = sw[i];
                        ++pos;
                    }
                    used = 0;
                }
#pragma unroll
                for (int i = 0; i < kEmitSlots; ++i)
                    if (i == used) { st[i] = t[j]; sw[i] = w[j]; }
                ++used;
            }
        }
#pragma unroll
        for (int i = 0; i < kEmitSlots; ++i)
            if (i < used) {
                ekey[pos] = hi | st[i];
                eval[pos] = sw[i];
                ++pos;
            }
        vcount[v] = (uint32_t)(pos - beg);
    }
}

// entries of vertex v move from its CSR range to voff[v] in the sort input
// (one thread per vertex; a vertex has at most a few entries)
__global__ void compact_vertices(int n, const int* __restrict__ xadj, const uint32_t* __restrict__ vcount,
                                 const uint32_t* __restrict__ voff, const uint64_t* __restrict__ ekey,
                                 const uint32_t* __restrict__ eval, uint64_t* K, uint32_t* V) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t cnt = vcount[v];
        const long long src = xadj[v];
        const long long dst = voff[v];
        for (uint32_t i = 0; i < cnt; ++i) {
            K[dst + i] = ekey[src + i];
            V[dst + i] = eval[src + i];
        }
    }
}

__global__ void head_flags(long long E, const uint64_t* __restrict__ K, uint32_t* h) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < E;
         i += (long long)gridDim.x * blockDim.x)
        h[i] = (i == 0 || K[i] != K[i - 1]) ? 1u : 0u;
}

__global__ void reduce_runs(long long E, const uint64_t* __restrict__ K, const uint32_t* __restrict__ V,
                            const uint32_t* __restrict__ uidx, int tb, int* cadj, int* cw,
                            uint32_t* rowcnt) {
    const uint64_t mask = (1ull << tb) - 1ull;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < E;
         i += (long long)gridDim.x * blockDim.x) {
        uint64_t k = K[i];
        if (i > 0 && K[i - 1] == k) continue;
        uint32_t s = V[i];
        for (long long j = i + 1; j < E && K[j] == k; ++j) s += V[j];
        uint32_t u = uidx[i];
        cadj[u] = (int)(k & mask);
        cw[u] = (int)s;
        atomicAdd(&rowcnt[k >> tb], 1u);
    }
}


}  // namespace

void contract(Ctx& ctx, const DevGraph& g, const int* label, int* cmap, DevGraph& out,
              int** out_xadj, int** out_adjncy, int** out_adjwgt, int** out_vwgt) {
    cudaStream_t st = ctx.stream;
    const size_t mk = ctx.scratch.mark();
    const int n = g.n;
    if (n == 0) {
        int* cx = ctx.hier.alloc<int>(1);
        KB_CUDA(cudaMemsetAsync(cx, 0, sizeof(int), st));
        out = DevGraph{};
        out.xadj = cx;
        *out_xadj = cx;
        *out_adjncy = *out_adjwgt = *out_vwgt = nullptr;
        return;
    }
    // 1. coarse ids
    int* mm = ctx.scratch.alloc<int>((size_t)n);
    uint32_t* pos = ctx.scratch.alloc<uint32_t>((size_t)n + 1);
    uint32_t* tot = reinterpret_cast<uint32_t*>(ctx.dscalars);
    {
        PhaseScope ps(ctx, "contract_ids", 20.0 * n);
        fill_i32(mm, n, INT_MAX, st);
        leader_min<<<grid_for(n, 256), 256, 0, st>>>(n, label, mm);
        KB_LAUNCH();
        leader_flags<<<grid_for(n, 256), 256, 0, st>>>(n, label, mm, pos);
        KB_LAUNCH();
        exclusive_scan_u32(pos, pos, n, tot, st, ctx.scratch);
    }
    KB_CUDA(cudaMemcpyAsync(ctx.pinned, tot, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    const int nc = (int)ctx.pinned[0];
    int* cvw = ctx.hier.alloc<int>((size_t)nc);
    int* cxadj = ctx.hier.alloc<int>((size_t)nc + 1);
    KB_CUDA(cudaMemsetAsync(cvw, 0, sizeof(int) * (size_t)nc, st));
    make_cmap<<<grid_for(n, 256), 256, 0, st>>>(n, label, mm, pos, g.vwgt, cmap,
                                                reinterpret_cast<uint32_t*>(cvw));
    KB_LAUNCH();
    int tb = 1;
    while ((1LL << tb) < (long long)nc) ++tb;
    // 2. emission into each vertex's CSR range
    const long long m = g.m;
    uint64_t* ekey = ctx.scratch.alloc<uint64_t>((size_t)std::max<long long>(m, 1));
    uint32_t* eval = ctx.scratch.alloc<uint32_t>((size_t)std::max<long long>(m, 1));
    uint32_t* vcount = ctx.scratch.alloc<uint32_t>((size_t)n + 1);
    uint32_t* voff = ctx.scratch.alloc<uint32_t>((size_t)n + 1);
    {
        PhaseScope ps(ctx, "contract_emit", 12.0 * m + 8.0 * n);
        emit_kernel<<<grid_for(n, kThreads), kThreads, 0, st>>>(n, g.xadj, g.adjncy, g.adjwgt, cmap, ekey, eval,
                                                                vcount, tb);
        KB_LAUNCH();
        exclusive_scan_u32(vcount, voff, n, tot, st, ctx.scratch);
    }
    KB_CUDA(cudaMemcpyAsync(ctx.pinned, tot, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    const long long E = ctx.pinned[0];
    // 3. compaction
    uint64_t* K0 = ctx.scratch.alloc<uint64_t>((size_t)std::max<long long>(E, 1));
    uint32_t* V0 = ctx.scratch.alloc<uint32_t>((size_t)std::max<long long>(E, 1));
    uint64_t* K1 = ctx.scratch.alloc<uint64_t>((size_t)std::max<long long>(E, 1));
    uint32_t* V1 = ctx.scratch.alloc<uint32_t>((size_t)std::max<long long>(E, 1));
    {
        PhaseScope ps(ctx, "contract_compact", 24.0 * E);
        compact_vertices<<<grid_for(n, kThreads), kThreads, 0, st>>>(n, g.xadj, vcount, voff, ekey, eval, K0, V0);
        KB_LAUNCH();
    }
    // 4. sort by (cu, cv)
    int which;
    {
        int bits = 2 * tb;
        PhaseScope ps(ctx, "contract_sort", 32.0 * E * ((bits + 7) / 8));
        which = radix_sort_pairs(K0, V0, K1, V1, E, bits, st, ctx.scratch);
    }
    uint64_t* K = which ? K1 : K0;
    uint32_t* V = which ? V1 : V0;
    // 5. reduce runs
    uint32_t* uidx = ctx.scratch.alloc<uint32_t>((size_t)std::max<long long>(E, 1));
    uint32_t* rowcnt = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
    {
        PhaseScope ps(ctx, "contract_reduce", 28.0 * E);
        head_flags<<<grid_for(E, 256), 256, 0, st>>>(E, K, uidx);
        KB_LAUNCH();
        exclusive_scan_u32(uidx, uidx, E, tot, st, ctx.scratch);
    }
    KB_CUDA(cudaMemcpyAsync(ctx.pinned, tot, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    const long long mc = E > 0 ? (long long)ctx.pinned[0] : 0;
    int* cadj = ctx.hier.alloc<int>((size_t)std::max<long long>(mc, 1));
    int* cwgt = ctx.hier.alloc<int>((size_t)std::max<long long>(mc, 1));
    KB_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(uint32_t) * ((size_t)nc + 1), st));
    {
        PhaseScope ps(ctx, "contract_reduce", 12.0 * E);
        if (E > 0) {
            reduce_runs<<<grid_for(E, 256), 256, 0, st>>>(E, K, V, uidx, tb, cadj, cwgt, rowcnt);
            KB_LAUNCH();
        }
        exclusive_scan_u32(rowcnt, reinterpret_cast<uint32_t*>(cxadj), (long long)nc + 1, nullptr, st,
                           ctx.scratch);
    }
    out = DevGraph{};
    out.n = nc;
    out.m = mc;
    out.xadj = cxadj;
    out.adjncy = cadj;
    out.adjwgt = cwgt;
    out.vwgt = cvw;
    *out_xadj = cxadj;
    *out_adjncy = cadj;
    *out_adjwgt = cwgt;
    *out_vwgt = cvw;
    ctx.scratch.release(mk);
}

}  // namespace kb
