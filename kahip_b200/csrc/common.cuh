// common.cuh -- shared definitions of the B200 KaFFPa path: status codes,
// CUDA error handling, the counter-based hash used for every tie-break and
// sub-round assignment, and small warp helpers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "hash.h"

namespace kb {

// Status codes returned by the extended C ABI (0 = success).
enum Status : int {
    KB_OK = 0,
    KB_ERR_INVALID_INPUT = -1,
    KB_ERR_CUDA = -2,
    KB_ERR_NO_DEVICE = -3,
    KB_ERR_OUT_OF_MEMORY = -4,
    KB_ERR_INTERNAL = -5,
    KB_WARN_IMBALANCED = 1,  // partition returned, but max block > bound
};

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* what) : std::runtime_error(what), code(c) {}
};

inline void check(cudaError_t e, const char* file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "CUDA error %d (%s) at %s:%d", (int)e,
                      cudaGetErrorString(e), file, line);
        throw CudaError(e, buf);
    }
}
// Number of kernels this library has launched (all threads, all devices).
extern std::atomic<long long> g_kernel_launches;

// The calling thread's error message (kb200_last_error): report_error sets
// it and returns `code`; clear_error empties it at the start of a call.
int report_error(int code, const char* msg);
void clear_error();

#define KB_CUDA(x) ::kb::check((x), __FILE__, __LINE__)
#define KB_LAUNCH()                                                          \
    do {                                                                     \
        ::kb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);     \
        ::kb::check(cudaGetLastError(), __FILE__, __LINE__);                 \
    } while (0)

constexpr int kWarp = 32;
constexpr int kNumSMs = 148;

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace kb
