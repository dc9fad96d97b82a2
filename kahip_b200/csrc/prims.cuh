// prims.cuh -- device-wide scan, radix sort and fills (prims.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "context.h"

namespace kb {

// out[i] = sum(in[0..i)); in-place allowed.  *total (device) = sum(in) if non-null.
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, long long n, uint32_t* total,
                        cudaStream_t s, Arena& arena);

// Stable LSD radix sort of (key, val) pairs on key bits [0, bits), 8 bits per
// pass.  Returns 0 if the result is in (keys, vals), 1 if in (keys_alt, vals_alt).
int radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                     long long n, int bits, cudaStream_t s, Arena& arena);

void fill_u32(uint32_t* p, long long n, uint32_t v, cudaStream_t s);
void fill_i32(int32_t* p, long long n, int32_t v, cudaStream_t s);
void fill_u8(uint8_t* p, long long n, uint8_t v, cudaStream_t s);

}  // namespace kb
