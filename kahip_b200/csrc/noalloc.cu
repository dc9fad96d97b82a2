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
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make
//     that first call before any stream capture is started.
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

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

__global__ void noalloc_cut_kernel(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                                   const int* __restrict__ adjwgt, const int* __restrict__ vwgt,
                                   const int* __restrict__ part, int k, unsigned long long* scratch) {
    unsigned long long* cut2 = scratch;
    unsigned long long* bad = scratch + 1;
    uint32_t* bw = reinterpret_cast<uint32_t*>(scratch + 2);
    unsigned long long c = 0, b = 0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const int p = part[v];
        if (p < 0 || p >= k) { ++b; continue; }  // out-of-range block id: counted, skipped
        atomicAdd(&bw[p], (uint32_t)(vwgt ? vwgt[v] : 1));
        for (int e = xadj[v]; e < xadj[v + 1]; ++e) {
            const int t = adjncy[e];
            if (t < 0 || t >= n) { ++b; continue; }
            if (part[t] != p) c += (unsigned long long)(long long)(adjwgt ? adjwgt[e] : 1);
        }
    }
    for (int o = 16; o >= 1; o >>= 1) {
        c += __shfl_xor_sync(0xffffffffu, c, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
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

// Device address of the scratch array on `dev` (looked up once per device).
int scratch_address(int dev, unsigned long long** out) {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            (void)cudaGetLastError();
            return KB200_ERR_CUDA;
        }
        g_addr[dev] = p;
    }
    *out = static_cast<unsigned long long*>(g_addr[dev]);
    return KB200_OK;
}

}  // namespace
}  // namespace kb

#pragma GCC visibility push(default)
extern "C" {

// Edge cut and block weights of part[] on the current device, all arrays
// device-resident (adjwgt / vwgt may be NULL = unit weights).  Writes
// *d_cut (one long long; -1 if a block id or target was out of range) and
// d_bw[k] asynchronously on `stream`.  Allocates nothing; k <= 65536; see
// the file comment for the shared scratch array and its limits.
int kb200_edge_cut_noalloc(int n, const int* d_xadj, const int* d_adjncy, const int* d_adjwgt,
                           const int* d_vwgt, const int* d_part, int k, long long* d_cut, uint32_t* d_bw,
                           void* stream) {
    if (n < 0 || !d_xadj || (n > 0 && (!d_adjncy || !d_part)) || !d_cut || !d_bw) return KB200_ERR_INVALID_INPUT;
    if (k < 1 || k > kb::kNoAllocMaxBlocks) return KB200_ERR_INVALID_INPUT;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kb::kMaxDevices) {
        (void)cudaGetLastError();
        return KB200_ERR_NO_DEVICE;
    }
    unsigned long long* scratch = nullptr;
    if (int rc = kb::scratch_address(dev, &scratch)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // clear the two counters and the k block-weight slots this call uses
    if (cudaMemsetAsync(scratch, 0, 2 * sizeof(unsigned long long) + sizeof(uint32_t) * (size_t)k, s) !=
        cudaSuccess) {
        (void)cudaGetLastError();
        return KB200_ERR_CUDA;
    }
    if (n > 0) {
        int blocks = (int)std::min<long long>(((long long)n + 255) / 256, (long long)kb::kNumSMs * 16);
        kb::noalloc_cut_kernel<<<blocks, 256, 0, s>>>(n, d_xadj, d_adjncy, d_adjwgt, d_vwgt, d_part, k, scratch);
        kb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    }
    kb::noalloc_finish_kernel<<<(k + 255) / 256, 256, 0, s>>>(k, scratch, d_cut, d_bw);
    kb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return KB200_ERR_CUDA;
    return KB200_OK;
}

}  // extern "C"
#pragma GCC visibility pop
