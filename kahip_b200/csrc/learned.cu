// learned.cu -- the learned edge rating on the CUDA cores: inference (the
// reference forward of the tensor-core path in learned_tc.cu) and training
// (hand-written forward and backward kernels, Adam).
//
// Numerics: weights are rounded to BF16 before every forward (the FP32
// master copy is what Adam updates), every stored activation is rounded to
// BF16, all sums accumulate in FP32.  Backward treats the roundings as
// identities.
#include "learned.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace kb {

namespace {

constexpr int kT = 256;          // threads per block
constexpr int kWarps = kT / 32;

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16(x)); }

__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void st(float* p, float v) { *p = v; }
__device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16(v); }

int grid_nodes(long long n) {
    return (int)std::max<long long>(1, std::min<long long>(div_up(n, kWarps), (long long)kNumSMs * 16));
}

// Edge features of entry (w, c(u), c(v)).
__device__ __forceinline__ void edge_feat(int w, uint32_t cu, uint32_t cv, float& f0, float& f1) {
    double r = 1.0 * w * w / (double)(uint32_t)(cu * cv);
    if (!(r < 1e30)) r = 1e30;  // division by a wrapped-to-zero denominator, or 0/0
    f0 = log2f((float)max(w, 1)) * 0.125f;
    f1 = log2f(1.0f + (float)r) * 0.125f;
}

// x_v, weighted degree, and h0 = bf16(relu(W0 x + b0)).
template <class T>
__global__ void __launch_bounds__(kT) layer0_fwd(int n, const int* xadj, const int* adjwgt, const int* vwgt,
                                                 const float* P, float2* xout, float* wdeg, T* h0) {
    __shared__ float w0[rm::H * 2], b0[rm::H];
    for (int i = threadIdx.x; i < rm::H * 2; i += kT) w0[i] = bf16r(P[rm::W0 + i]);
    for (int i = threadIdx.x; i < rm::H; i += kT) b0[i] = bf16r(P[rm::B0 + i]);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (long long v = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5); v < n; v += (long long)gridDim.x * kWarps) {
        const int beg = xadj[v], end = xadj[v + 1];
        float sw = 0.f;
        for (int e = beg + lane; e < end; e += 32) sw += (float)adjwgt[e];
#pragma unroll
        for (int o = 16; o; o >>= 1) sw += __shfl_xor_sync(0xffffffffu, sw, o);
        const float x0 = log2f(1.0f + (float)(end - beg)) * 0.125f;
        const float x1 = log2f((float)max(vwgt[v], 1)) * 0.125f;
        if (lane == 0) {
            if (xout) xout[v] = make_float2(x0, x1);
            wdeg[v] = sw;
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = lane + 32 * q;
            const float a = w0[2 * j] * x0 + w0[2 * j + 1] * x1 + b0[j];
            st(h0 + v * rm::H + j, bf16r(fmaxf(a, 0.f)));
        }
    }
}

// agg[v] = bf16(sum_u w_vu h[u] / wdeg[v]); lane owns features 2l, 2l+1.
template <class T>
__global__ void __launch_bounds__(kT) agg_fwd(int n, const int* xadj, const int* adjncy, const int* adjwgt,
                                              const float* wdeg, const T* h, T* agg) {
    const int lane = threadIdx.x & 31;
    for (long long v = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5); v < n; v += (long long)gridDim.x * kWarps) {
        float a0 = 0.f, a1 = 0.f;
        const int beg = xadj[v], end = xadj[v + 1];
        for (int e = beg; e < end; ++e) {
            const int u = adjncy[e];
            const float w = (float)adjwgt[e];
            a0 += w * ld(h + (long long)u * rm::H + 2 * lane);
            a1 += w * ld(h + (long long)u * rm::H + 2 * lane + 1);
        }
        const float d = wdeg[v];
        const float inv = d > 0.f ? 1.0f / d : 0.f;
        st(agg + v * rm::H + 2 * lane, bf16r(a0 * inv));
        st(agg + v * rm::H + 2 * lane + 1, bf16r(a1 * inv));
    }
}

// out[v] = act(W [in0[v] | in1[v]] + b) with in1 optional (K = 64 or 128),
// N outputs (64 or 32); W row-major [N][K] in P at woff, bias at boff.
template <class T, int K, int N, bool RELU>
__global__ void __launch_bounds__(kT) dense_fwd(int n, const float* P, int woff, int boff, const T* in0,
                                                const T* in1, T* out) {
    __shared__ float wt[K * N];  // transposed: wt[k*N + j]
    __shared__ float bs[N];
    __shared__ float row[kWarps][K];
    for (int i = threadIdx.x; i < K * N; i += kT) {
        const int j = i / K, k = i % K;
        wt[k * N + j] = bf16r(P[woff + i]);
    }
    for (int i = threadIdx.x; i < N; i += kT) bs[i] = bf16r(P[boff + i]);
    __syncthreads();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    for (long long v = (long long)blockIdx.x * kWarps + wp; v < n; v += (long long)gridDim.x * kWarps) {
        for (int k = lane; k < K; k += 32)
            row[wp][k] = k < rm::H ? ld(in0 + v * rm::H + k) : ld(in1 + v * rm::H + (k - rm::H));
        __syncwarp();
#pragma unroll
        for (int q = 0; q < N / 32; ++q) {
            const int j = lane + 32 * q;
            float a = bs[j];
#pragma unroll 8
            for (int k = 0; k < K; ++k) a += wt[k * N + j] * row[wp][k];
            if (RELU) a = fmaxf(a, 0.f);
            st(out + v * N + j, bf16r(a));
        }
        __syncwarp();
    }
}

// Eight consecutive z values (q-th group of a row) with one or two 16-byte loads.
__device__ __forceinline__ void load_z8(const float* z, long long u, int q, float* out) {
    const float4* p = reinterpret_cast<const float4*>(z + u * rm::Z) + 2 * q;
    const float4 a = p[0], b = p[1];
    out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
    out[4] = b.x; out[5] = b.y; out[6] = b.z; out[7] = b.w;
}
__device__ __forceinline__ void load_z8(const __nv_bfloat16* z, long long u, int q, float* out) {
    const uint4 b = reinterpret_cast<const uint4*>(z + u * rm::Z)[q];
    const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&b);
#pragma unroll
    for (int k = 0; k < 4; ++k) { out[2 * k] = __low2float(h2[k]); out[2 * k + 1] = __high2float(h2[k]); }
}

// Per-entry score; lane per entry, warp per row.  prob/rating outputs.
template <class T>
__global__ void __launch_bounds__(kT) head_fwd(int n, const int* xadj, const int* adjncy, const int* adjwgt,
                                               const int* vwgt, const float* P, const T* z, float* prob,
                                               uint32_t* rating) {
    __shared__ float wf[rm::Z * 2], wo[rm::Z];
    __shared__ float bo;
    __shared__ float zv[kWarps][rm::Z];
    for (int i = threadIdx.x; i < rm::Z * 2; i += kT) wf[i] = bf16r(P[rm::WF + i]);
    for (int i = threadIdx.x; i < rm::Z; i += kT) wo[i] = bf16r(P[rm::WO + i]);
    if (threadIdx.x == 0) bo = bf16r(P[rm::BO]);
    __syncthreads();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    for (long long v = (long long)blockIdx.x * kWarps + wp; v < n; v += (long long)gridDim.x * kWarps) {
        zv[wp][lane] = ld(z + v * rm::Z + lane);
        __syncwarp();
        const int beg = xadj[v], end = xadj[v + 1];
        const uint32_t cv = (uint32_t)vwgt[v];
        for (int e = beg + lane; e < end; e += 32) {
            const int u = adjncy[e];
            float f0, f1;
            edge_feat(adjwgt[e], (uint32_t)vwgt[u], cv, f0, f1);
            float s = bo;
#pragma unroll 1
            for (int q = 0; q < rm::Z / 8; ++q) {
                float zu[8];
                load_z8(z, u, q, zu);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int j = 8 * q + k;
                    // IEEE addition commutes exactly: both directions of the
                    // edge get the same sum
                    const float a = zu[k] + zv[wp][j];
                    const float t = a + (wf[2 * j] * f0 + wf[2 * j + 1] * f1);
                    s += wo[j] * fmaxf(t, 0.f);
                }
            }
            const float p = 1.0f / (1.0f + expf(-s));
            if (prob) prob[e] = p;
            if (rating) {
                float q = floorf((1.0f - p) * 16777216.0f);
                q = fminf(fmaxf(q, 0.f), 16777215.f);
                rating[e] = (uint32_t)q;
            }
        }
        __syncwarp();
    }
}

// ----------------------------------------------------------------- training

struct LossArgs {
    const uint8_t* label;
    float pos_w;     // weight of a cut entry
    float inv_norm;  // 1 / sum of entry weights
};

// Head forward + backward.  dz[v] = 2 * sum over row v of dL/dt (the edge's
// other direction contributes the same to z_v by symmetry).  Parameter
// gradients (wo, Wf, bo) accumulate in block shared memory, then globally.
__global__ void __launch_bounds__(kT) head_train(int n, const int* xadj, const int* adjncy, const int* adjwgt,
                                                 const int* vwgt, const float* P, const float* z, LossArgs L,
                                                 float* dz, float* G, float* loss) {
    __shared__ float wf[rm::Z * 2], wo[rm::Z];
    __shared__ float bo;
    __shared__ float zv[kWarps][rm::Z];
    __shared__ float gwf[rm::Z * 2], gwo[rm::Z];
    __shared__ float gbo, sloss;
    for (int i = threadIdx.x; i < rm::Z * 2; i += kT) { wf[i] = bf16r(P[rm::WF + i]); gwf[i] = 0.f; }
    for (int i = threadIdx.x; i < rm::Z; i += kT) { wo[i] = bf16r(P[rm::WO + i]); gwo[i] = 0.f; }
    if (threadIdx.x == 0) { bo = bf16r(P[rm::BO]); gbo = 0.f; sloss = 0.f; }
    __syncthreads();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    float my_loss = 0.f;
    for (long long v = (long long)blockIdx.x * kWarps + wp; v < n; v += (long long)gridDim.x * kWarps) {
        zv[wp][lane] = z[v * rm::Z + lane];
        __syncwarp();
        float dzl[rm::Z];
#pragma unroll
        for (int j = 0; j < rm::Z; ++j) dzl[j] = 0.f;
        const int beg = xadj[v], end = xadj[v + 1];
        const uint32_t cv = (uint32_t)vwgt[v];
        for (int e = beg + lane; e < end; e += 32) {
            const int u = adjncy[e];
            float f0, f1;
            edge_feat(adjwgt[e], (uint32_t)vwgt[u], cv, f0, f1);
            float t[rm::Z];
            float s = bo;
#pragma unroll
            for (int j = 0; j < rm::Z; ++j) {
                const float a = z[(long long)u * rm::Z + j] + zv[wp][j];
                t[j] = a + (wf[2 * j] * f0 + wf[2 * j + 1] * f1);
                s += wo[j] * fmaxf(t[j], 0.f);
            }
            const float y = L.label[e] ? 1.f : 0.f;
            const float om = (L.label[e] ? L.pos_w : 1.f) * L.inv_norm;
            const float p = 1.0f / (1.0f + expf(-s));
            // weighted BCE from the logit: softplus(-s) for y = 1, softplus(s) for y = 0
            const float xs = y > 0.f ? -s : s;
            my_loss += om * (fmaxf(xs, 0.f) + log1pf(expf(-fabsf(xs))));
            const float g = om * (p - y);
            atomicAdd(&gbo, g);
#pragma unroll
            for (int j = 0; j < rm::Z; ++j) {
                const float r = fmaxf(t[j], 0.f);
                atomicAdd(&gwo[j], g * r);
                const float dt = t[j] > 0.f ? g * wo[j] : 0.f;
                atomicAdd(&gwf[2 * j], dt * f0);
                atomicAdd(&gwf[2 * j + 1], dt * f1);
                dzl[j] += dt;
            }
        }
        // reduce dz over the warp's entries
#pragma unroll
        for (int j = 0; j < rm::Z; ++j) {
            float x = dzl[j];
#pragma unroll
            for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == j) dz[v * rm::Z + j] = 2.f * x;
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o);
    if (lane == 0) atomicAdd(&sloss, my_loss);
    __syncthreads();
    for (int i = threadIdx.x; i < rm::Z * 2; i += kT) atomicAdd(G + rm::WF + i, gwf[i]);
    for (int i = threadIdx.x; i < rm::Z; i += kT) atomicAdd(G + rm::WO + i, gwo[i]);
    if (threadIdx.x == 0) {
        atomicAdd(G + rm::BO, gbo);
        atomicAdd(loss, sloss);
    }
}

// Backward of out = act(W [in0 | in1] + b):  dA = dOut * act'(out);
// dIn = W^T dA (dIn0, dIn1 optional halves, accumulated with +=);
// dW += dA in^T; db += dA.  Warp per node, block shared gradient buffers.
template <int K, int N, bool RELU>
__global__ void __launch_bounds__(kT) dense_bwd(int n, const float* P, int woff, const float* in0,
                                                const float* in1, const float* out, const float* dout,
                                                float* din0, float* din1, float* G, int goff_w, int goff_b) {
    extern __shared__ float sm[];
    float* w = sm;             // [N][K] (bf16-rounded)
    float* gw = w + N * K;     // [N][K]
    float* gb = gw + N * K;    // [N]
    float* rows = gb + N;      // [kWarps][K + N]
    for (int i = threadIdx.x; i < N * K; i += kT) {
        w[i] = bf16r(P[woff + i]);
        gw[i] = 0.f;
    }
    for (int i = threadIdx.x; i < N; i += kT) gb[i] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    float* xr = rows + wp * (K + N);
    float* da = xr + K;
    for (long long v = (long long)blockIdx.x * kWarps + wp; v < n; v += (long long)gridDim.x * kWarps) {
        for (int k = lane; k < K; k += 32) xr[k] = k < rm::H ? in0[v * rm::H + k] : in1[v * rm::H + (k - rm::H)];
        for (int j = lane; j < N; j += 32) {
            float d = dout[v * N + j];
            if (RELU && !(out[v * N + j] > 0.f)) d = 0.f;
            da[j] = d;
            atomicAdd(&gb[j], d);
        }
        __syncwarp();
        for (int k = lane; k < K; k += 32) {
            float acc = 0.f;
            const float x = xr[k];
            for (int j = 0; j < N; ++j) {
                acc += da[j] * w[j * K + k];
                atomicAdd(&gw[j * K + k], da[j] * x);
            }
            if (k < rm::H) {
                if (din0) din0[v * rm::H + k] += acc;
            } else if (din1) {
                din1[v * rm::H + (k - rm::H)] += acc;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < N * K; i += kT) atomicAdd(G + goff_w + i, gw[i]);
    for (int i = threadIdx.x; i < N; i += kT) atomicAdd(G + goff_b + i, gb[i]);
}

// dh[u] += sum_{v in N(u)} (w_uv / wdeg[v]) dagg[v]  (gather form; the graph
// is symmetric).
__global__ void __launch_bounds__(kT) agg_bwd(int n, const int* xadj, const int* adjncy, const int* adjwgt,
                                              const float* wdeg, const float* dagg, float* dh) {
    const int lane = threadIdx.x & 31;
    for (long long u = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5); u < n; u += (long long)gridDim.x * kWarps) {
        float a0 = 0.f, a1 = 0.f;
        for (int e = xadj[u]; e < xadj[u + 1]; ++e) {
            const int v = adjncy[e];
            const float d = wdeg[v];
            if (!(d > 0.f)) continue;
            const float c = (float)adjwgt[e] / d;
            a0 += c * dagg[(long long)v * rm::H + 2 * lane];
            a1 += c * dagg[(long long)v * rm::H + 2 * lane + 1];
        }
        dh[u * rm::H + 2 * lane] += a0;
        dh[u * rm::H + 2 * lane + 1] += a1;
    }
}

__global__ void __launch_bounds__(kT) layer0_bwd(int n, const float2* x, const float* h0, const float* dh0,
                                                 float* G) {
    __shared__ float g[rm::H * 3];
    for (int i = threadIdx.x; i < rm::H * 3; i += kT) g[i] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (long long v = (long long)blockIdx.x * kWarps + (threadIdx.x >> 5); v < n; v += (long long)gridDim.x * kWarps) {
        const float2 xv = x[v];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = lane + 32 * q;
            const float d = h0[v * rm::H + j] > 0.f ? dh0[v * rm::H + j] : 0.f;
            atomicAdd(&g[2 * j], d * xv.x);
            atomicAdd(&g[2 * j + 1], d * xv.y);
            atomicAdd(&g[2 * rm::H + j], d);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < rm::H * 2; i += kT) atomicAdd(G + rm::W0 + i, g[i]);
    for (int i = threadIdx.x; i < rm::H; i += kT) atomicAdd(G + rm::B0 + i, g[2 * rm::H + i]);
}

__global__ void adam_step(int np, float* P, const float* G, float* M, float* V, float lr, float b1t, float b2t) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const float g = G[i];
        const float m = b1 * M[i] + (1.f - b1) * g;
        const float v = b2 * V[i] + (1.f - b2) * g * g;
        M[i] = m;
        V[i] = v;
        P[i] -= lr * (m / (1.f - b1t)) / (sqrtf(v / (1.f - b2t)) + eps);
    }
}

__global__ void count_labels(long long m, const uint8_t* label, unsigned long long* pos) {
    unsigned long long c = 0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (long long)gridDim.x * blockDim.x)
        c += label[e] ? 1 : 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(pos, c);
}

template <int K, int N, bool RELU>
void launch_dense_bwd(int n, const float* P, int woff, const float* in0, const float* in1, const float* out,
                      const float* dout, float* din0, float* din1, float* G, int gw, int gb, cudaStream_t s) {
    const size_t smem = sizeof(float) * (2 * (size_t)N * K + N + (size_t)kWarps * (K + N));
    KB_CUDA(cudaFuncSetAttribute(dense_bwd<K, N, RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dense_bwd<K, N, RELU><<<grid_nodes(n), kT, smem, s>>>(n, P, woff, in0, in1, out, dout, din0, din1, G, gw, gb);
    KB_LAUNCH();
}

}  // namespace

// Launch wrappers shared with the tensor-core path (learned_tc.cu).
void launch_layer0_bf16(Ctx& ctx, const DevGraph& g, const float* P, float* wdeg, __nv_bfloat16* h0) {
    layer0_fwd<__nv_bfloat16><<<grid_nodes(g.n), kT, 0, ctx.stream>>>(g.n, g.xadj, g.adjwgt, g.vwgt, P, nullptr,
                                                                        wdeg, h0);
    KB_LAUNCH();
}

void launch_head_bf16(Ctx& ctx, const DevGraph& g, const float* P, const __nv_bfloat16* z, float* prob,
                      uint32_t* rating) {
    head_fwd<__nv_bfloat16><<<grid_nodes(g.n), kT, 0, ctx.stream>>>(g.n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, P, z,
                                                                      prob, rating);
    KB_LAUNCH();
}

// Forward of the whole network on the CUDA cores with FP32 storage of
// BF16-rounded activations.  Buffers: x[n] (float2), wdeg[n], h[4][n*64],
// agg[3][n*64], z[n*32].
struct Fwd {
    float2* x;
    float* wdeg;
    float* h[4];
    float* agg[3];
    float* z;
};

static Fwd alloc_fwd(Arena& A, int n) {
    Fwd f;
    const size_t nn = (size_t)std::max(n, 1);
    f.x = A.alloc<float2>(nn);
    f.wdeg = A.alloc<float>(nn);
    for (auto& p : f.h) p = A.alloc<float>(nn * rm::H);
    for (auto& p : f.agg) p = A.alloc<float>(nn * rm::H);
    f.z = A.alloc<float>(nn * rm::Z);
    return f;
}

static void forward_cuda_cores(Ctx& ctx, const DevGraph& g, const float* P, const Fwd& f) {
    cudaStream_t s = ctx.stream;
    const int n = g.n, gr = grid_nodes(n);
    layer0_fwd<float><<<gr, kT, 0, s>>>(n, g.xadj, g.adjwgt, g.vwgt, P, f.x, f.wdeg, f.h[0]);
    KB_LAUNCH();
    for (int l = 1; l <= 3; ++l) {
        agg_fwd<float><<<gr, kT, 0, s>>>(n, g.xadj, g.adjncy, g.adjwgt, f.wdeg, f.h[l - 1], f.agg[l - 1]);
        KB_LAUNCH();
        dense_fwd<float, 128, 64, true><<<gr, kT, 0, s>>>(n, P, rm::layer_w(l), rm::layer_b(l), f.h[l - 1],
                                                           f.agg[l - 1], f.h[l]);
        KB_LAUNCH();
    }
    dense_fwd<float, 64, 32, false><<<gr, kT, 0, s>>>(n, P, rm::WZ, rm::BZ, f.h[3], nullptr, f.z);
    KB_LAUNCH();
}

void rating_infer_tc(Ctx& ctx, const DevGraph& g, const float* params, float* prob, uint32_t* rating);

void rating_infer(Ctx& ctx, const DevGraph& g, const float* params, float* prob, uint32_t* rating, bool use_tc) {
    if (g.n == 0) return;
    if (use_tc) {
        rating_infer_tc(ctx, g, params, prob, rating);
        return;
    }
    const size_t mk = ctx.scratch.mark();
    Fwd f = alloc_fwd(ctx.scratch, g.n);
    {
        PhaseScope ps(ctx, "rating_layers", 0);
        forward_cuda_cores(ctx, g, params, f);
    }
    PhaseScope ps(ctx, "rating_head", 0);
    head_fwd<float><<<grid_nodes(g.n), kT, 0, ctx.stream>>>(g.n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, params, f.z,
                                                              prob, rating);
    KB_LAUNCH();
    ctx.scratch.release(mk);
}

void rating_train(Ctx& ctx, const TrainGraph* graphs, int count, int steps, float lr, float* params,
                  float* loss_out) {
    if (count <= 0 || steps <= 0) return;
    cudaStream_t s = ctx.stream;
    int nmax = 1;
    for (int i = 0; i < count; ++i) nmax = std::max(nmax, graphs[i].g.n);
    const size_t mk = ctx.scratch.mark();
    Fwd f = alloc_fwd(ctx.scratch, nmax);
    const size_t nn = (size_t)nmax;
    float* dz = ctx.scratch.alloc<float>(nn * rm::Z);
    float* dh[4];
    for (auto& p : dh) p = ctx.scratch.alloc<float>(nn * rm::H);
    float* dagg = ctx.scratch.alloc<float>(nn * rm::H);
    float* G = ctx.scratch.alloc<float>(rm::kParams);
    float* M = ctx.scratch.alloc<float>(rm::kParams);
    float* V = ctx.scratch.alloc<float>(rm::kParams);
    float* dloss = ctx.scratch.alloc<float>(std::max(steps, 1));
    unsigned long long* pos = ctx.scratch.alloc<unsigned long long>((size_t)count);
    KB_CUDA(cudaMemsetAsync(M, 0, sizeof(float) * rm::kParams, s));
    KB_CUDA(cudaMemsetAsync(V, 0, sizeof(float) * rm::kParams, s));
    KB_CUDA(cudaMemsetAsync(dloss, 0, sizeof(float) * (size_t)steps, s));
    KB_CUDA(cudaMemsetAsync(pos, 0, sizeof(unsigned long long) * (size_t)count, s));
    for (int i = 0; i < count; ++i) {
        count_labels<<<256, 256, 0, s>>>(graphs[i].g.m, graphs[i].label, pos + i);
        KB_LAUNCH();
    }
    std::vector<unsigned long long> hpos((size_t)count);
    KB_CUDA(cudaMemcpyAsync(hpos.data(), pos, sizeof(unsigned long long) * (size_t)count, cudaMemcpyDeviceToHost, s));
    KB_CUDA(cudaStreamSynchronize(s));
    float b1t = 1.f, b2t = 1.f;
    for (int step = 0; step < steps; ++step) {
        const TrainGraph& tg = graphs[step % count];
        const DevGraph& g = tg.g;
        const int n = g.n, gr = grid_nodes(n);
        const double P1 = (double)hpos[(size_t)(step % count)], N0 = (double)g.m - P1;
        LossArgs L;
        L.label = tg.label;
        L.pos_w = P1 > 0 ? (float)std::min(50.0, std::max(1.0, N0 / P1)) : 1.f;
        L.inv_norm = (float)(1.0 / std::max(1.0, L.pos_w * P1 + N0));
        KB_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * rm::kParams, s));
        for (auto p : dh) KB_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * (size_t)n * rm::H, s));
        forward_cuda_cores(ctx, g, params, f);
        head_train<<<gr, kT, 0, s>>>(n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, params, f.z, L, dz, G, dloss + step);
        KB_LAUNCH();
        launch_dense_bwd<64, 32, false>(n, params, rm::WZ, f.h[3], nullptr, f.z, dz, dh[3], nullptr, G, rm::WZ, rm::BZ,
                                        s);
        for (int l = 3; l >= 1; --l) {
            KB_CUDA(cudaMemsetAsync(dagg, 0, sizeof(float) * (size_t)n * rm::H, s));
            launch_dense_bwd<128, 64, true>(n, params, rm::layer_w(l), f.h[l - 1], f.agg[l - 1], f.h[l], dh[l],
                                            dh[l - 1], dagg, G, rm::layer_w(l), rm::layer_b(l), s);
            agg_bwd<<<gr, kT, 0, s>>>(n, g.xadj, g.adjncy, g.adjwgt, f.wdeg, dagg, dh[l - 1]);
            KB_LAUNCH();
        }
        layer0_bwd<<<gr, kT, 0, s>>>(n, f.x, f.h[0], dh[0], G);
        KB_LAUNCH();
        b1t *= 0.9f;
        b2t *= 0.999f;
        adam_step<<<div_up(rm::kParams, 256), 256, 0, s>>>(rm::kParams, params, G, M, V, lr, b1t, b2t);
        KB_LAUNCH();
    }
    if (loss_out) KB_CUDA(cudaMemcpyAsync(loss_out, dloss, sizeof(float) * (size_t)steps, cudaMemcpyDeviceToHost, s));
    KB_CUDA(cudaStreamSynchronize(s));
    ctx.scratch.release(mk);
}

// ------------------------------------------------ gradient of one step (tests)

// Gradient of the loss of one graph at `params` (no update): G[kParams]
// (device, out) and the loss (host, out).
void rating_grad(Ctx& ctx, const TrainGraph& tg, const float* params, float* G, float* loss) {
    cudaStream_t s = ctx.stream;
    const DevGraph& g = tg.g;
    const int n = g.n, gr = grid_nodes(n);
    const size_t mk = ctx.scratch.mark();
    Fwd f = alloc_fwd(ctx.scratch, n);
    const size_t nn = (size_t)std::max(n, 1);
    float* dz = ctx.scratch.alloc<float>(nn * rm::Z);
    float* dh[4];
    for (auto& p : dh) p = ctx.scratch.alloc<float>(nn * rm::H);
    float* dagg = ctx.scratch.alloc<float>(nn * rm::H);
    float* dloss = ctx.scratch.alloc<float>(1);
    unsigned long long* pos = ctx.scratch.alloc<unsigned long long>(1);
    KB_CUDA(cudaMemsetAsync(pos, 0, sizeof(unsigned long long), s));
    KB_CUDA(cudaMemsetAsync(dloss, 0, sizeof(float), s));
    count_labels<<<256, 256, 0, s>>>(g.m, tg.label, pos);
    KB_LAUNCH();
    unsigned long long hp = 0;
    KB_CUDA(cudaMemcpyAsync(&hp, pos, sizeof(hp), cudaMemcpyDeviceToHost, s));
    KB_CUDA(cudaStreamSynchronize(s));
    const double P1 = (double)hp, N0 = (double)g.m - P1;
    LossArgs L;
    L.label = tg.label;
    L.pos_w = P1 > 0 ? (float)std::min(50.0, std::max(1.0, N0 / P1)) : 1.f;
    L.inv_norm = (float)(1.0 / std::max(1.0, L.pos_w * P1 + N0));
    KB_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * rm::kParams, s));
    for (auto p : dh) KB_CUDA(cudaMemsetAsync(p, 0, sizeof(float) * nn * rm::H, s));
    forward_cuda_cores(ctx, g, params, f);
    head_train<<<gr, kT, 0, s>>>(n, g.xadj, g.adjncy, g.adjwgt, g.vwgt, params, f.z, L, dz, G, dloss);
    KB_LAUNCH();
    launch_dense_bwd<64, 32, false>(n, params, rm::WZ, f.h[3], nullptr, f.z, dz, dh[3], nullptr, G, rm::WZ, rm::BZ, s);
    for (int l = 3; l >= 1; --l) {
        KB_CUDA(cudaMemsetAsync(dagg, 0, sizeof(float) * nn * rm::H, s));
        launch_dense_bwd<128, 64, true>(n, params, rm::layer_w(l), f.h[l - 1], f.agg[l - 1], f.h[l], dh[l], dh[l - 1],
                                        dagg, G, rm::layer_w(l), rm::layer_b(l), s);
        agg_bwd<<<gr, kT, 0, s>>>(n, g.xadj, g.adjncy, g.adjwgt, f.wdeg, dagg, dh[l - 1]);
        KB_LAUNCH();
    }
    layer0_bwd<<<gr, kT, 0, s>>>(n, f.x, f.h[0], dh[0], G);
    KB_LAUNCH();
    KB_CUDA(cudaMemcpyAsync(loss, dloss, sizeof(float), cudaMemcpyDeviceToHost, s));
    KB_CUDA(cudaStreamSynchronize(s));
    ctx.scratch.release(mk);
}

}  // namespace kb
