// evolve.cu -- KaFFPaE-style evolutionary partitioning on one device.
//
// The reference's kaffpaE (parallel_mh_async.cpp:49-…) keeps a population of
// partitions per MPI rank, picks parents by tournament
// (population.cpp:358-369), combines them (population.cpp:189-250, here
// combine() of the multilevel driver) and inserts the offspring: dropped
// when worse than the worst member, otherwise it replaces the member with
// the fewest differing cut edges among those not better than it
// (population.cpp:120-173).  Here the schedule is deterministic: rounds of
// `per_generation` offspring, each round's selections reading the
// population at the round's start (hash-drawn tournaments), insertions in
// offspring order; members and offspring stay in device memory and the cut
// difference is one pass over the edges.
#include "evolve.cuh"

#include <atomic>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "hash.h"
#include "partitioner.cuh"

namespace kb {

namespace {

constexpr int kThreads = 256;

struct Obj {
    uint64_t ov;
    long long cut;
};

bool obj_less(Obj a, Obj b) { return a.ov < b.ov || (a.ov == b.ov && a.cut < b.cut); }

int fitter(const std::vector<Obj>& obj, int a, int b) {
    if (obj_less(obj[a], obj[b])) return a;
    if (obj_less(obj[b], obj[a])) return b;
    return a < b ? a : b;
}

// directed entries whose cut status differs between partitions a and b
__global__ void cut_difference_kernel(int n, const int* __restrict__ xadj, const int* __restrict__ adjncy,
                                      const int* __restrict__ a, const int* __restrict__ b, unsigned long long* out) {
    unsigned long long d = 0;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x / 32);
    for (long long v0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; v0 < n; v0 += warps) {
        const int v = (int)v0;
        const int av = a[v], bv = b[v];
        for (int e = xadj[v] + lane; e < xadj[v + 1]; e += 32) {
            const int u = adjncy[e];
            d += (av != a[u]) != (bv != b[u]);
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if (lane == 0 && d) atomicAdd(out, d);
}

long long cut_difference(Ctx& ctx, const DevGraph& g, const int* a, const int* b) {
    unsigned long long* d = reinterpret_cast<unsigned long long*>(ctx.dscalars + 32);
    KB_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), ctx.stream));
    if (g.n) {
        PhaseScope ps(ctx, "cut_difference", 8.0 * (double)g.m + 12.0 * g.n);
        const long long blocks = std::min<long long>(div_up(32LL * g.n, kThreads), (long long)kNumSMs * 16);
        cut_difference_kernel<<<(int)std::max<long long>(blocks, 1), kThreads, 0, ctx.stream>>>(g.n, g.xadj, g.adjncy,
                                                                                                  a, b, d);
        KB_LAUNCH();
    }
    unsigned long long h = 0;
    KB_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    return (long long)h;
}

// device buffer outside the arenas (the population outlives every call's arena use)
struct DevBuf {
    int* p = nullptr;
    explicit DevBuf(size_t count) { KB_CUDA(cudaMalloc(&p, sizeof(int) * std::max<size_t>(count, 1))); }
    ~DevBuf() { if (p) cudaFree(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

// f(c, i) for i in [0, count) on the worker contexts, one host thread per
// context; each task gets freshly reserved arenas (grown when exhausted).
// The first exception is rethrown after every thread has joined.
template <class F>
void run_tasks(const std::vector<Ctx*>& workers, const DevGraph& g0, int count, F f) {
    const int T = std::max(1, std::min((int)workers.size(), count));
    std::atomic<int> next{0};
    std::exception_ptr err;
    std::mutex mu;
    auto body = [&](int t) {
        Ctx& c = *workers[(size_t)t];
        cudaSetDevice(c.device);
        for (int i; (i = next.fetch_add(1)) < count;) {
            try {
                for (int attempt = 0;; ++attempt) {
                    try {
                        reserve_for(c, g0.n, g0.m, false, (attempt == 0 ? 1.0 : 2.0 * attempt) * 1.5);
                        c.timing = 0;
                        c.reset_stats();
                        f(c, i);
                        break;
                    } catch (const CudaError& e) {
                        if (e.code == cudaErrorMemoryAllocation && attempt < 2 &&
                            std::string(e.what()).find("arena exhausted") != std::string::npos) {
                            (void)cudaGetLastError();
                            continue;
                        }
                        throw;
                    }
                }
            } catch (...) {
                std::lock_guard<std::mutex> lk(mu);
                if (!err) err = std::current_exception();
                next.store(count);
            }
        }
    };
    std::vector<std::thread> threads;
    for (int t = 1; t < T; ++t) threads.emplace_back(body, t);
    body(0);
    for (auto& th : threads) th.join();
    if (err) std::rethrow_exception(err);
}

}  // namespace

int kaffpae(Ctx& ctx, const std::vector<Ctx*>& workers, const DevGraph& g0, const Knobs& kn, int population,
            int generations, int per_generation, int* d_best, long long* edgecut, long long* history) {
    const int P = population, W = per_generation, n = g0.n;
    const size_t nn = (size_t)std::max(n, 1);
    DevBuf pop(nn * (size_t)P), off(nn * (size_t)W);
    std::vector<Obj> obj((size_t)P), oobj((size_t)W);
    // members: the plain partitioner with seeds seed + i
    run_tasks(workers, g0, P, [&](Ctx& c, int i) {
        Knobs k = kn;
        k.seed = kn.seed + i;
        long long cut = 0;
        partition(c, g0, k, pop.p + (size_t)i * nn, &cut, nullptr);
        partition_quality(c, g0, pop.p + (size_t)i * nn, kn.k, kn.final_bound, &obj[(size_t)i].ov,
                          &obj[(size_t)i].cut);
    });
    int best = 0;
    for (int i = 1; i < P; ++i) best = fitter(obj, best, i);
    if (history) history[0] = obj[best].cut;
    std::vector<int> pa((size_t)W), pb((size_t)W);
    for (int t = 0; t < generations; ++t) {
        if (P >= 2) {
            // selections read the population at the round's start
            for (int j = 0; j < W; ++j) {
                const uint64_t ks = stream_key(kn.seed, TAG_EVO, t, j);
                const int x0 = (int)hash_range(hash32(ks, 0u), (uint32_t)P);
                const int x1 = (int)hash_range(hash32(ks, 1u), (uint32_t)P);
                const int x2 = (int)hash_range(hash32(ks, 2u), (uint32_t)P);
                const int x3 = (int)hash_range(hash32(ks, 3u), (uint32_t)P);
                const int a = fitter(obj, x0, x1);
                int b = fitter(obj, x2, x3);
                if (b == a) b = b == x2 ? x3 : x2;
                if (b == a) b = (a + 1) % P;
                pa[(size_t)j] = a;
                pb[(size_t)j] = b;
            }
            run_tasks(workers, g0, W, [&](Ctx& c, int j) {
                Knobs k = kn;
                k.seed = kn.seed + P + t * W + j;
                long long cut = 0;
                combine(c, g0, k, pop.p + (size_t)pa[(size_t)j] * nn, pop.p + (size_t)pb[(size_t)j] * nn,
                        off.p + (size_t)j * nn, &cut, nullptr);
                partition_quality(c, g0, off.p + (size_t)j * nn, kn.k, kn.final_bound, &oobj[(size_t)j].ov,
                                  &oobj[(size_t)j].cut);
            });
            // insertion in offspring order
            for (int j = 0; j < W; ++j) {
                int worst = 0;
                for (int i = 1; i < P; ++i)
                    if (obj_less(obj[worst], obj[i])) worst = i;
                if (obj_less(obj[worst], oobj[j])) continue;
                int pick = -1;
                long long pd = 0;
                for (int i = 0; i < P; ++i) {
                    if (obj_less(obj[i], oobj[j])) continue;
                    const long long d = cut_difference(ctx, g0, pop.p + (size_t)i * nn, off.p + (size_t)j * nn);
                    if (pick < 0 || d < pd) { pick = i; pd = d; }
                }
                if (n)
                    KB_CUDA(cudaMemcpyAsync(pop.p + (size_t)pick * nn, off.p + (size_t)j * nn, sizeof(int) * (size_t)n,
                                            cudaMemcpyDeviceToDevice, ctx.stream));
                obj[pick] = oobj[j];
            }
            KB_CUDA(cudaStreamSynchronize(ctx.stream));
        }
        best = 0;
        for (int i = 1; i < P; ++i) best = fitter(obj, best, i);
        if (history) history[t + 1] = obj[best].cut;
    }
    if (n)
        KB_CUDA(cudaMemcpyAsync(d_best, pop.p + (size_t)best * nn, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice,
                                ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    *edgecut = obj[best].cut;
    return obj[best].ov == 0 ? KB_OK : KB_WARN_IMBALANCED;
}

}  // namespace kb
