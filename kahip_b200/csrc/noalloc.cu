// noalloc.cu -- edge cut and block weights of a device-resident partition
// without allocating any memory.
//
// Who needs this: code that must not call cudaMalloc while it runs -- for
// example a caller that evaluates partitions from inside a region where the
// device allocator may not be touched (a section that holds a custom memory
// pool or a fixed memory budget, a real-time loop that forbids allocator
// calls and the implicit synchronisation cudaMalloc/cudaFree can cause), or
// a host program whose device memory is owned by another runtime.  Every
// other entry point of this library takes its working memory from a
// per-call context (cudaMalloc on first use).
//
// The kernel's working memory (the 64-bit cut accumulator and one 32-bit
// accumulator per block) is a file-scope __device__ array, so every GPU that
// loads this library holds kNoAllocScratchBytes of it until the process
// exits.  Consequences for callers:
//   * k is limited to kNoAllocMaxBlocks; larger k is rejected.
//   * All calls on a device share the one array and it keeps the last
//     call's contents; each call clears what it needs before use.  Calls
//     whose work overlaps on the GPU (different streams, or host threads
//     issuing concurrently) race on it and give wrong results.
//   * The first call in a CUDA context looks up the array's device address
//     with cudaGetSymbolAddress (with that context current) and caches it
//     under the context's handle; make that first call before any stream
//     capture is started.  After cudaDeviceReset the cached address is
//     stale if the driver hands out the same context handle again, so a
//     process that resets a device must not call this entry point again.
//   * The graph is trusted as a CSR offset array: xadj[0] = 0, monotone,
//     and xadj[n] no larger than the length of adjncy.  Rows that run
//     backwards, block ids outside [0, k), targets outside [0, n) and
//     negative weights make *d_cut = -1 (the other entry points reject the
//     same inputs); the kernel cannot see the length of adjncy.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <mutex>

#include "common.cuh"

extern "C" {
#include "../../include/kahip_b200.h"
}

namespace kb {
namespace {

constexpr int kNoAllocMaxBlocks = 65536;
// [0] cut accumulator (uint64), [1] count of out-of-range ids, then
// kNoAllocMaxBlocks uint32 block weights: 256 KiB + 16 bytes
constexpr size_t kNoAllocScratchWords = 2 + kNoAllocMaxBlocks / 2;
constexpr size_t kNoAllocScratchBytes = kNoAllocScratchWords * sizeof(unsigned long long);

static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocScratchWords];

// Cached device address of the scratch array per CUDA context.
constexpr int kMaxContexts = 64;
std::mutex g_addr_mu;
CUcontext g_addr_ctx[kMaxContexts] = {};
void* g_addr[kMaxContexts] = {};
int g_addr_used = 0;

// One warp per vertex: the lanes stride over the row (coalesced reads, hub
// rows spread over 32 lanes).  Accumulates twice the cut, the block
// weights, and a count of inputs it refuses (bad block id, row running
// backwards, target out of range, negative weight).
__global__ void noalloc_cut_kernel(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                                   const int* __restrict__ adjwgt, const int* __restrict__ vwgt,
                                   const int* __restrict__ part, int k, unsigned long long* scratch) {
    unsigned long long* cut2 = scratch;
    unsigned long long* bad = scratch + 1;
    uint32_t* bw = reinterpret_cast<uint32_t*>(scratch + 2);
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    unsigned long long c = 0, b = 0;
    for (long long v = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const int p = part[v];
        const int r0 = xadj[v], r1 = xadj[v + 1];
        if (p < 0 || p >= k || r0 < 0 || r1 < r0) {
            if (lane == 0) ++b;
            continue;
        }
        if (lane == 0) {
            const int w = vwgt ? vwgt[v] : 1;
            if (w < 0) ++b;
            else atomicAdd(&bw[p], (uint32_t)w);
        }
        for (int e = r0 + lane; e < r1; e += 32) {
            const int t = adjncy[e];
            const int w = adjwgt ? adjwgt[e] : 1;
            if (t < 0 || t >= n || w < 0) { ++b; continue; }
            if (part[t] != p) c += (unsigned long long)w;
        }
    }
    for (int o = 16; o >= 1; o >>= 1) {
        c += __shfl_xor_sync(0xffffffffu, c, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
        if (c) atomicAdd(cut2, c);
        if (b) atomicAdd(bad, b);
    }
}

// cut (directed sum / 2, or -1 when an id was out of range) and block
// weights out of the scratch array
__global__ void noalloc_finish_kernel(int k, const unsigned long long* scratch, long long* d_cut,
                                      uint32_t* d_bw) {
    const uint32_t* bw = reinterpret_cast<const uint32_t*>(scratch + 2);
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < k; b += gridDim.x * blockDim.x) d_bw[b] = bw[b];
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_cut = scratch[1] ? -1LL : (long long)(scratch[0] / 2);
}

using CtxGetCurrentFn = CUresult (*)(CUcontext*);

// The current CUDA context's handle (nullptr when it cannot be read).
CUcontext current_context() {
    static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// Device address of the scratch array in the current context, looked up
// once per context with that context current.
int scratch_address(unsigned long long** out) {
    CUcontext ctx = current_context();
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (ctx)
        for (int i = 0; i < g_addr_used; ++i)
            if (g_addr_ctx[i] == ctx) {
                *out = static_cast<unsigned long long*>(g_addr[i]);
                return KB200_OK;
            }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
        (void)cudaGetLastError();
        return report_error(KB200_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    }
    if (!ctx) ctx = current_context();  // the lookup made the runtime's context current
    if (ctx && g_addr_used < kMaxContexts) {
        g_addr_ctx[g_addr_used] = ctx;
        g_addr[g_addr_used] = p;
        ++g_addr_used;
    }
    *out = static_cast<unsigned long long*>(p);
    return KB200_OK;
}

}  // namespace
}  // namespace kb

#pragma GCC visibility push(default)
extern "C" {

// Edge cut and block weights of part[] on the current device, all arrays
// device-resident (adjwgt / vwgt may be NULL = unit weights).  Writes
// *d_cut (one long long; -1 if a block id, row, target or weight was
// refused) and d_bw[k] asynchronously on `stream`.  Allocates nothing;
// k <= 65536; see the file comment for the shared scratch array and its
// limits.
int kb200_edge_cut_noalloc(int n, const int* d_xadj, const int* d_adjncy, const int* d_adjwgt,
                           const int* d_vwgt, const int* d_part, int k, long long* d_cut, uint32_t* d_bw,
                           void* stream) {
    kb::clear_error();
    if (n < 0 || !d_xadj || (n > 0 && (!d_adjncy || !d_part)) || !d_cut || !d_bw)
        return kb::report_error(KB200_ERR_INVALID_INPUT, "invalid arguments (n < 0 or a NULL array)");
    if (k < 1 || k > kb::kNoAllocMaxBlocks)
        return kb::report_error(KB200_ERR_INVALID_INPUT, "k must be in [1, 65536]");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        return kb::report_error(KB200_ERR_NO_DEVICE, "no CUDA device available (this library has no CPU path)");
    }
    unsigned long long* scratch = nullptr;
    if (int rc = kb::scratch_address(&scratch)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // clear the two counters and the k block-weight slots this call uses
    if (cudaMemsetAsync(scratch, 0, 2 * sizeof(unsigned long long) + sizeof(uint32_t) * (size_t)k, s) !=
        cudaSuccess) {
        (void)cudaGetLastError();
        return kb::report_error(KB200_ERR_CUDA, "cudaMemsetAsync of the scratch array failed");
    }
    if (n > 0) {
        int blocks = (int)std::min<long long>(((long long)n + 7) / 8, (long long)kb::kNumSMs * 8);
        kb::noalloc_cut_kernel<<<blocks, 256, 0, s>>>(n, d_xadj, d_adjncy, d_adjwgt, d_vwgt, d_part, k, scratch);
        kb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    }
    kb::noalloc_finish_kernel<<<(k + 255) / 256, 256, 0, s>>>(k, scratch, d_cut, d_bw);
    kb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return kb::report_error(KB200_ERR_CUDA, "kernel launch failed");
    return KB200_OK;
}

}  // extern "C"
#pragma GCC visibility pop
