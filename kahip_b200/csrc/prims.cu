// prims.cu -- device-wide building blocks written for this library:
// exclusive scan of uint32, stable LSD radix sort of (uint64 key, uint32
// value) pairs, fills and gathers.  All are deterministic.
#include "prims.cuh"

namespace kb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if ((int)lane_id() >= o) x += y;
    }
    return x;
}

// block-wide exclusive scan of one value per thread; returns the block total
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t x, uint32_t& excl) {
    __shared__ uint32_t wsum[33];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    uint32_t inc = warp_incl_scan(x);
    if (l == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t t = l < nw ? wsum[l] : 0;
        uint32_t ti = warp_incl_scan(t);
        if (l < nw) wsum[l] = ti - t;
        if (l == 31) wsum[32] = ti;  // block total
    }
    __syncthreads();
    excl = inc - x + wsum[w];
    uint32_t total = wsum[32];
    __syncthreads();
    return total;
}

__global__ void scan_reduce(const uint32_t* __restrict__ in, long long n, uint32_t* partial) {
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        long long i = base + j;
        if (i < n) s += in[i];
    }
    uint32_t excl;
    uint32_t tot = block_excl_scan(s, excl);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// single block: exclusive scan of the partials in place, total to *total
__global__ void scan_partials(uint32_t* partial, int nb, uint32_t* total) {
    uint32_t carry = 0;
    for (int base = 0; base < nb; base += blockDim.x) {
        int i = base + threadIdx.x;
        uint32_t x = i < nb ? partial[i] : 0;
        uint32_t excl;
        uint32_t tot = block_excl_scan(x, excl);
        if (i < nb) partial[i] = excl + carry;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void scan_down(const uint32_t* in, uint32_t* out, long long n, const uint32_t* partial) {
    long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        long long i = base + j;
        v[j] = i < n ? in[i] : 0;
        s += v[j];
    }
    uint32_t excl;
    block_excl_scan(s, excl);
    uint32_t run = excl + partial[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        long long i = base + j;
        if (i < n) out[i] = run;
        run += v[j];
    }
}

// ------------------------------------------------------------- radix sort

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;                       // per lane
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kWarpTile = 32 * kSortItems;            // 512

__global__ void radix_upsweep(const uint64_t* __restrict__ keys, long long n, int shift,
                              uint32_t* __restrict__ hist, int ntiles) {
    __shared__ uint32_t h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * kSortTile;
    for (int j = 0; j < kSortItems; ++j) {
        long long i = base + (long long)j * kSortThreads + threadIdx.x;
        bool valid = i < n;
        unsigned act = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            uint32_t d = (uint32_t)(keys[i] >> shift) & 255u;
            unsigned peers = __match_any_sync(act, d);
            if ((int)lane_id() == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[(long long)d * ntiles + blockIdx.x] = h[d];
}

__global__ void radix_downsweep(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                long long n, int shift, const uint32_t* __restrict__ offs,
                                int ntiles) {
    __shared__ uint32_t wh[kSortWarps][256];
    __shared__ uint32_t toff[256];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kSortWarps * 256; i += blockDim.x) (&wh[0][0])[i] = 0;
    for (int d = threadIdx.x; d < 256; d += blockDim.x) toff[d] = offs[(long long)d * ntiles + blockIdx.x];
    __syncthreads();
    const long long wbase = (long long)blockIdx.x * kSortTile + (long long)warp * kWarpTile;
    uint64_t k[kSortItems];
    uint32_t v[kSortItems];
    uint32_t rk[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        long long i = wbase + (long long)j * 32 + lane;
        bool valid = i < n;
        k[j] = valid ? kin[i] : 0;
        v[j] = valid ? vin[i] : 0;
        rk[j] = 0;
        unsigned act = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            uint32_t d = (uint32_t)(k[j] >> shift) & 255u;
            unsigned peers = __match_any_sync(act, d);
            int leader = __ffs(peers) - 1;
            uint32_t before = 0;
            if (lane == leader) {
                before = wh[warp][d];
                wh[warp][d] = before + (uint32_t)__popc(peers);
            }
            before = __shfl_sync(peers, before, leader);
            rk[j] = before + (uint32_t)__popc(peers & lanemask_lt());
        }
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t t = wh[w][d];
            wh[w][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        long long i = wbase + (long long)j * 32 + lane;
        if (i < n) {
            uint32_t d = (uint32_t)(k[j] >> shift) & 255u;
            uint32_t pos = toff[d] + wh[warp][d] + rk[j];
            kout[pos] = k[j];
            vout[pos] = v[j];
        }
    }
}

template <class T>
__global__ void fill_kernel(T* p, long long n, T val) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        p[i] = val;
}

}  // namespace

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, long long n, uint32_t* total,
                        cudaStream_t s, Arena& arena) {
    if (n <= 0) {
        if (total) KB_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), s));
        return;
    }
    size_t mk = arena.mark();
    int nb = div_up(n, kScanTile);
    uint32_t* partial = arena.alloc<uint32_t>((size_t)nb);
    scan_reduce<<<nb, kScanThreads, 0, s>>>(in, n, partial);
    KB_LAUNCH();
    scan_partials<<<1, 1024, 0, s>>>(partial, nb, total);
    KB_LAUNCH();
    scan_down<<<nb, kScanThreads, 0, s>>>(in, out, n, partial);
    KB_LAUNCH();
    arena.release(mk);
}

int radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt,
                     long long n, int bits, cudaStream_t s, Arena& arena) {
    if (n <= 1 || bits <= 0) return 0;
    size_t mk = arena.mark();
    int ntiles = div_up(n, kSortTile);
    long long hn = 256LL * ntiles;
    uint32_t* hist = arena.alloc<uint32_t>((size_t)hn);
    uint64_t* kin = keys;
    uint32_t* vin = vals;
    uint64_t* kout = keys_alt;
    uint32_t* vout = vals_alt;
    int passes = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        radix_upsweep<<<ntiles, kSortThreads, 0, s>>>(kin, n, shift, hist, ntiles);
        KB_LAUNCH();
        exclusive_scan_u32(hist, hist, hn, nullptr, s, arena);
        radix_downsweep<<<ntiles, kSortThreads, 0, s>>>(kin, vin, kout, vout, n, shift, hist, ntiles);
        KB_LAUNCH();
        std::swap(kin, kout);
        std::swap(vin, vout);
        ++passes;
    }
    arena.release(mk);
    return passes & 1;  // 1: result is in (keys_alt, vals_alt)
}

void fill_u32(uint32_t* p, long long n, uint32_t v, cudaStream_t s) {
    if (n <= 0) return;
    int blocks = (int)std::min<long long>(div_up(n, 256), 148LL * 16);
    fill_kernel<uint32_t><<<blocks, 256, 0, s>>>(p, n, v);
    KB_LAUNCH();
}

void fill_i32(int32_t* p, long long n, int32_t v, cudaStream_t s) {
    fill_u32(reinterpret_cast<uint32_t*>(p), n, (uint32_t)v, s);
}

void fill_u8(uint8_t* p, long long n, uint8_t v, cudaStream_t s) {
    if (n <= 0) return;
    KB_CUDA(cudaMemsetAsync(p, v, (size_t)n, s));
}

}  // namespace kb
