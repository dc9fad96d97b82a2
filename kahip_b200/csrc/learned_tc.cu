// learned_tc.cu -- inference of the learned edge rating with the layer GEMMs
// on the 5th-generation tensor cores (tcgen05), fused with the neighbour
// gather that feeds them.
//
// One CTA = two warpgroups (8 warps) holding NOUT columns of TMEM (the
// 128 x NOUT FP32 accumulator of one tile).  Per tile of 128 nodes:
//   1. the warps gather the tile's A operand into shared memory: row r =
//      [h(v) | weighted mean of h over N(v)] (BF16; sums in FP32), written
//      in the no-swizzle K-major core-matrix layout (8 rows x 16 bytes per
//      core matrix, contiguous);
//   2. one thread issues K/16 tcgen05.mma (M=128, N=NOUT, K=16, BF16 in,
//      FP32 accumulate in TMEM) reading A and the layer's weights (B, loaded
//      once per CTA in the same layout) from shared memory, then
//      tcgen05.commit to an mbarrier;
//   3. every warp waits on the mbarrier (bounded), reads 32 TMEM lanes
//      (= 32 rows; warp w accesses lanes 32 (w % 4) ..) and half of the
//      columns with tcgen05.ld, adds the bias, applies ReLU, rounds to BF16
//      and stores its part of the rows.
// The gather (HBM/L2-bound) dominates; the MMAs take a few hundred cycles
// per tile.  Descriptor bit layouts follow the PTX ISA's tcgen05 matrix and
// instruction descriptors (as spelled out in CUTLASS's
// cute/arch/mma_sm100_desc.hpp).
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "learned.cuh"

namespace kb {

void launch_layer0_bf16(Ctx& ctx, const DevGraph& g, const float* P, float* wdeg, __nv_bfloat16* h0);
void launch_head_bf16(Ctx& ctx, const DevGraph& g, const float* P, const __nv_bfloat16* z, float* prob,
                      uint32_t* rating);

namespace {

constexpr int kTile = 128;               // nodes per tile = MMA M
constexpr int kTcThreads = 256;          // two warpgroups: all gather, both read TMEM
constexpr int kGatherRows = kTile / (kTcThreads / 32);  // rows gathered per warp
constexpr long long kWaitLimit = 1 << 24;  // mbarrier polls before giving up

// byte offset of element (r, c) of a K-major operand with `rows` rows in the
// no-swizzle core-matrix layout: core matrices of 8 rows x 8 BF16 (128 B,
// row-major inside); consecutive row groups 128 B apart (SBO), consecutive
// K groups rows*16 B apart (LBO)
__host__ __device__ constexpr uint32_t core_off(int r, int c, int rows) {
    return (uint32_t)((c >> 3) * (rows * 16) + (r >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// shared-memory matrix descriptor: start >> 4 [0,14), LBO >> 4 [16,30),
// SBO >> 4 [32,46), version 1 [46,48), base offset 0, no swizzle [61,64) = 0
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

// instruction descriptor, kind::f16: D FP32 [4,6)=1, A BF16 [7,10)=1,
// B BF16 [10,13)=1, both K-major, N >> 3 at [17,23), M >> 4 at [24,29)
template <int N>
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTile >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Weights of one layer, BF16, in the B-operand layout (NOUT rows x K).
template <int K, int NOUT>
__global__ void pack_weights(const float* P, int woff, __nv_bfloat16* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NOUT * K; i += gridDim.x * blockDim.x) {
        const int j = i / K, c = i % K;
        out[core_off(j, c, NOUT) / 2] = __float2bfloat16(P[woff + i]);
    }
}

// Rows longer than kLongRow (hubs of skewed graphs) would stall a whole
// tile on one group of eight lanes; their weighted neighbour sums are formed
// first, one block per row, in a fixed order (deterministic).
constexpr int kLongRow = 1024;
constexpr int kLongThreads = 1024;

__device__ __forceinline__ int end_of(const int* xadj, long long v) { return xadj[v + 1]; }

// hrank[v] = index of v among the long rows (or -1); list[] = the long rows.
__global__ void long_rows(int n, const int* xadj, int* hrank, int* list, unsigned* count) {
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        if (xadj[v + 1] - xadj[v] > kLongRow) {
            const unsigned i = atomicAdd(count, 1u);
            list[i] = (int)v;
            hrank[v] = (int)i;
        } else {
            hrank[v] = -1;
        }
    }
}

// hagg[rank][f] = sum_u w_vu h[u][f] over a long row; warp w of the block
// sums the entries e = beg + w + 32 k (lane l owns features 2l, 2l+1), then
// the 32 warp sums are added in warp order.
__global__ void __launch_bounds__(kLongThreads) long_row_sums(const int* xadj, const int* adjncy, const int* adjwgt,
                                                              const __nv_bfloat16* h, const int* list,
                                                              const unsigned* count, float* hagg) {
    __shared__ float part[kLongThreads / 32][rm::H];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const unsigned cnt = *count;
    for (unsigned i = blockIdx.x; i < cnt; i += gridDim.x) {
        const int v = list[i];
        const int beg = xadj[v], end = xadj[v + 1];
        float a0 = 0.f, a1 = 0.f;
        for (int e = beg + wp; e < end; e += kLongThreads / 32) {
            const __nv_bfloat162 hu = reinterpret_cast<const __nv_bfloat162*>(h + (long long)adjncy[e] * rm::H)[lane];
            const float w = (float)adjwgt[e];
            a0 += w * __low2float(hu);
            a1 += w * __high2float(hu);
        }
        part[wp][2 * lane] = a0;
        part[wp][2 * lane + 1] = a1;
        __syncthreads();
        if (threadIdx.x < rm::H) {
            float s = 0.f;
            for (int k = 0; k < kLongThreads / 32; ++k) s += part[k][threadIdx.x];
            hagg[(size_t)i * rm::H + threadIdx.x] = s;
        }
        __syncthreads();
    }
}

template <bool AGG, int NOUT, bool RELU>
__global__ void __launch_bounds__(kTcThreads) fused_layer_tc(int n, const int* xadj, const int* adjncy,
                                                             const int* adjwgt, const float* wdeg,
                                                             const __nv_bfloat16* h, const __nv_bfloat16* wpk,
                                                             const float* P, int boff, __nv_bfloat16* out,
                                                             const int* hrank, const float* hagg, int* err) {
    constexpr int K = AGG ? 128 : 64;
    constexpr uint32_t A_BYTES = kTile * K * 2, B_BYTES = NOUT * K * 2;
    constexpr uint32_t LBO_A = kTile * 16, LBO_B = NOUT * 16, SBO = 128;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sa = smem;
    unsigned char* sb = smem + A_BYTES;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + A_BYTES + B_BYTES);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    float* bias = reinterpret_cast<float*>(tslot + 4);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // B operand and bias, once per CTA
    for (uint32_t i = tid * 16; i < B_BYTES; i += kTcThreads * 16)
        *reinterpret_cast<uint4*>(sb + i) = *reinterpret_cast<const uint4*>(reinterpret_cast<const unsigned char*>(wpk) + i);
    for (int j = tid; j < NOUT; j += kTcThreads) bias[j] = __bfloat162float(__float2bfloat16(P[boff + j]));
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"((uint32_t)NOUT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint32_t sa_addr = smem_u32(sa), sb_addr = smem_u32(sb), mbar_addr = smem_u32(mbar);

    uint32_t phase = 0;
    bool ok = true;
    const long long tiles = ((long long)n + kTile - 1) / kTile;
    for (long long t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        // 1. gather the A tile: warp w fills kGatherRows rows, four rows at
        // a time (one per group of 8 lanes); lane j of a group owns features
        // 8j .. 8j+7 (16 bytes of a row) and keeps four neighbour rows in
        // flight
        {
            const int grp = lane >> 3, j = lane & 7;
            for (int r = warp * kGatherRows + grp; r < (warp + 1) * kGatherRows; r += 4) {
                const long long v = t * kTile + r;
                float x[8], acc[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) { x[q] = 0.f; acc[q] = 0.f; }
                if (v < n) {
                    const uint4 hv = reinterpret_cast<const uint4*>(h + v * rm::H)[j];
                    const __nv_bfloat162* hp = reinterpret_cast<const __nv_bfloat162*>(&hv);
#pragma unroll
                    for (int q = 0; q < 4; ++q) { x[2 * q] = __low2float(hp[q]); x[2 * q + 1] = __high2float(hp[q]); }
                    if (AGG && end_of(xadj, v) - xadj[v] > kLongRow) {
                        // long row: its weighted sum was formed by long_row_sums
                        const float* src = hagg + (size_t)hrank[v] * rm::H + 8 * j;
                        const float d = wdeg[v];
                        const float inv = d > 0.f ? 1.0f / d : 0.f;
#pragma unroll
                        for (int q = 0; q < 8; ++q) acc[q] = src[q] * inv;
                    } else if (AGG) {
                        const int beg = xadj[v], end = xadj[v + 1];
                        int e = beg;
                        for (; e + 4 <= end; e += 4) {
                            int u[4];
                            float w[4];
                            uint4 hu[4];
#pragma unroll
                            for (int k = 0; k < 4; ++k) { u[k] = adjncy[e + k]; w[k] = (float)adjwgt[e + k]; }
#pragma unroll
                            for (int k = 0; k < 4; ++k) hu[k] = reinterpret_cast<const uint4*>(h + (long long)u[k] * rm::H)[j];
#pragma unroll
                            for (int k = 0; k < 4; ++k) {
                                const __nv_bfloat162* p2 = reinterpret_cast<const __nv_bfloat162*>(&hu[k]);
#pragma unroll
                                for (int q = 0; q < 4; ++q) {
                                    acc[2 * q] += w[k] * __low2float(p2[q]);
                                    acc[2 * q + 1] += w[k] * __high2float(p2[q]);
                                }
                            }
                        }
                        for (; e < end; ++e) {
                            const float w = (float)adjwgt[e];
                            const uint4 hu = reinterpret_cast<const uint4*>(h + (long long)adjncy[e] * rm::H)[j];
                            const __nv_bfloat162* p2 = reinterpret_cast<const __nv_bfloat162*>(&hu);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                acc[2 * q] += w * __low2float(p2[q]);
                                acc[2 * q + 1] += w * __high2float(p2[q]);
                            }
                        }
                        const float d = wdeg[v];
                        const float inv = d > 0.f ? 1.0f / d : 0.f;
#pragma unroll
                        for (int q = 0; q < 8; ++q) acc[q] *= inv;
                    }
                }
                uint4 ox, oa;
                __nv_bfloat162* px = reinterpret_cast<__nv_bfloat162*>(&ox);
                __nv_bfloat162* pa = reinterpret_cast<__nv_bfloat162*>(&oa);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    px[q] = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
                    pa[q] = __floats2bfloat162_rn(acc[2 * q], acc[2 * q + 1]);
                }
                *reinterpret_cast<uint4*>(sa + core_off(r, 8 * j, kTile)) = ox;
                if (AGG) *reinterpret_cast<uint4*>(sa + core_off(r, 64 + 8 * j, kTile)) = oa;
            }
        }
        // generic-proxy smem writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        // 2. one thread issues the MMAs and commits them to the mbarrier
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t idesc = instr_desc<NOUT>();
#pragma unroll
            for (int kk = 0; kk < K / 16; ++kk) {
                const uint64_t da = smem_desc(sa_addr + (uint32_t)kk * 2u * LBO_A, LBO_A, SBO);
                const uint64_t db = smem_desc(sb_addr + (uint32_t)kk * 2u * LBO_B, LBO_B, SBO);
                const uint32_t acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                mbar_addr)
                         : "memory");
        }
        // 3. wait for the accumulator (bounded)
        {
            uint32_t done = 0;
            for (long long it = 0; it < kWaitLimit && !done; ++it) {
                asm volatile(
                    "{\n\t.reg .pred P;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, P;\n\t}\n"
                    : "=r"(done)
                    : "r"(mbar_addr), "r"(phase)
                    : "memory");
            }
            if (!done) {
                ok = false;
                if (lane == 0) atomicExch(err, 1);
            }
        }
        phase ^= 1u;
        if (!__all_sync(0xffffffffu, ok)) ok = false;
        if (ok) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows) and the
            // (w / 4)-th half of the columns
            const int lanes = (warp & 3) * 32;
            const long long v = t * kTile + lanes + lane;
#pragma unroll
            for (int c0 = (warp >> 2) * (NOUT / 2); c0 < (warp >> 2) * (NOUT / 2) + NOUT / 2; c0 += 16) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((uint32_t)lanes << 16) + (uint32_t)c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15}, [%16];\n"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                      "=r"(r[14]), "=r"(r[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (v < n) {
                    __nv_bfloat162 o[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        float y0 = __uint_as_float(r[2 * q]) + bias[c0 + 2 * q];
                        float y1 = __uint_as_float(r[2 * q + 1]) + bias[c0 + 2 * q + 1];
                        if (RELU) {
                            y0 = fmaxf(y0, 0.f);
                            y1 = fmaxf(y1, 0.f);
                        }
                        o[q] = __floats2bfloat162_rn(y0, y1);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(out + v * NOUT + c0);
                    dst[0] = *reinterpret_cast<uint4*>(&o[0]);
                    dst[1] = *reinterpret_cast<uint4*>(&o[4]);
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        ok = ok && !(*reinterpret_cast<volatile int*>(err));
    }
    // a timed-out MMA may still be in flight: give it one more bounded wait
    if (!ok) {
        uint32_t done = 0;
        for (long long it = 0; it < kWaitLimit && !done; ++it) {
            asm volatile(
                "{\n\t.reg .pred P;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, P;\n\t}\n"
                : "=r"(done)
                : "r"(mbar_addr), "r"(phase ^ 1u)
                : "memory");
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)NOUT));
}

template <bool AGG, int NOUT, bool RELU>
void launch_fused(Ctx& ctx, const DevGraph& g, const float* wdeg, const __nv_bfloat16* h,
                  const __nv_bfloat16* wpk, const float* P, int boff, __nv_bfloat16* out, const int* hrank,
                  const float* hagg, int* err) {
    constexpr int K = AGG ? 128 : 64;
    const size_t smem = (size_t)kTile * K * 2 + (size_t)NOUT * K * 2 + 64 + NOUT * sizeof(float);
    KB_CUDA(cudaFuncSetAttribute(fused_layer_tc<AGG, NOUT, RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    const long long tiles = ((long long)g.n + kTile - 1) / kTile;
    // ~48 KB of shared memory per CTA: four CTAs per SM
    const int grid = (int)std::max<long long>(1, std::min<long long>(tiles, 4LL * kNumSMs));
    fused_layer_tc<AGG, NOUT, RELU><<<grid, kTcThreads, smem, ctx.stream>>>(g.n, g.xadj, g.adjncy, g.adjwgt, wdeg,
                                                                             h, wpk, P, boff, out, hrank, hagg,
                                                                             err);
    KB_LAUNCH();
}

}  // namespace

void rating_infer_tc(Ctx& ctx, const DevGraph& g, const float* P, float* prob, uint32_t* rating) {
    cudaStream_t s = ctx.stream;
    const size_t mk = ctx.scratch.mark();
    const size_t nn = (size_t)std::max(g.n, 1);
    float* wdeg = ctx.scratch.alloc<float>(nn);
    __nv_bfloat16* ha = ctx.scratch.alloc<__nv_bfloat16>(nn * rm::H);
    __nv_bfloat16* hb = ctx.scratch.alloc<__nv_bfloat16>(nn * rm::H);
    __nv_bfloat16* z = ctx.scratch.alloc<__nv_bfloat16>(nn * rm::Z);
    __nv_bfloat16* wl[3];
    for (auto& p : wl) p = ctx.scratch.alloc<__nv_bfloat16>((size_t)rm::H * 2 * rm::H);
    __nv_bfloat16* wz = ctx.scratch.alloc<__nv_bfloat16>((size_t)rm::Z * rm::H);
    int* err = ctx.dscalars + 60;
    // long rows (more than kLongRow entries): at most m / (kLongRow + 1) of them
    const long long lmax = g.m / (kLongRow + 1) + 1;
    const bool has_long = g.maxdeg > kLongRow;
    int* hrank = ctx.scratch.alloc<int>(nn);
    int* hlist = ctx.scratch.alloc<int>((size_t)lmax);
    float* hagg = ctx.scratch.alloc<float>((size_t)lmax * rm::H);
    unsigned* hcount = reinterpret_cast<unsigned*>(ctx.dscalars + 20);
    {
        PhaseScope ps(ctx, "rating_layers", 0);
        if (has_long) {
            KB_CUDA(cudaMemsetAsync(hcount, 0, sizeof(unsigned), s));
            long_rows<<<(int)std::min<long long>(div_up(g.n, 256), 16LL * kNumSMs), 256, 0, s>>>(g.n, g.xadj, hrank,
                                                                                             hlist, hcount);
            KB_LAUNCH();
        }
        for (int l = 1; l <= 3; ++l) {
            pack_weights<128, 64><<<32, 256, 0, s>>>(P, rm::layer_w(l), wl[l - 1]);
            KB_LAUNCH();
        }
        pack_weights<64, 32><<<8, 256, 0, s>>>(P, rm::WZ, wz);
        KB_LAUNCH();
        launch_layer0_bf16(ctx, g, P, wdeg, ha);
        __nv_bfloat16* cur = ha;
        __nv_bfloat16* nxt = hb;
        for (int l = 1; l <= 3; ++l) {
            if (has_long) {
                long_row_sums<<<(int)std::min<long long>(lmax, 2LL * kNumSMs), kLongThreads, 0, s>>>(
                    g.xadj, g.adjncy, g.adjwgt, cur, hlist, hcount, hagg);
                KB_LAUNCH();
            }
            launch_fused<true, 64, true>(ctx, g, wdeg, cur, wl[l - 1], P, rm::layer_b(l), nxt, hrank, hagg, err);
            std::swap(cur, nxt);
        }
        launch_fused<false, 32, false>(ctx, g, wdeg, cur, wz, P, rm::BZ, z, hrank, hagg, err);
    }
    PhaseScope ps(ctx, "rating_head", 0);
    launch_head_bf16(ctx, g, P, z, prob, rating);
    ctx.scratch.release(mk);
}

}  // namespace kb
