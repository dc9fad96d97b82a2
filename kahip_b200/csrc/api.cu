// api.cu -- the C ABI of libkahip_b200.so.
//
// kaffpa() keeps the reference signature (interface/kaHIP_interface.h:30-33)
// and semantics (interface/kaHIP_interface.cpp:146-166): Metis-style CSR in,
// edge cut and part[] out, caller owns every array, imbalance is a fraction.
// Unlike the reference it validates its input on the host; on failure it
// sets *edgecut = -1 and leaves part[] untouched (the reference has no
// error channel).  There is no CPU fallback: without a CUDA device the call
// fails.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "contract.cuh"
#include "ip_device.cuh"
#include "host/initial_partitioning.h"
#include "jet.cuh"
#include "knobs.h"
#include "learned.cuh"
#include "match.cuh"
#include "combine.cuh"
#include "evolve.cuh"
#include "partitioner.cuh"
#include "prims.cuh"

extern "C" {
#include "../../include/kaHIP_interface.h"
}

namespace kb {

std::atomic<long long> g_kernel_launches{0};

namespace {

thread_local std::string g_last_error;

// Contexts are cached per device and reused across calls (streams, pinned
// buffers and the device arenas survive); one call owns a context at a time.
std::mutex g_pool_mu;
std::vector<std::unique_ptr<Ctx>> g_pool[64];

struct Lease {
    std::unique_ptr<Ctx> ctx;
    int dev;
    explicit Lease(int d) : dev(d) {
        {
            std::lock_guard<std::mutex> lk(g_pool_mu);
            if (!g_pool[d].empty()) {
                ctx = std::move(g_pool[d].back());
                g_pool[d].pop_back();
            }
        }
        if (!ctx) ctx.reset(new Ctx());
        ctx->init(d, nullptr);
    }
    ~Lease() {
        if (!ctx) return;
        std::lock_guard<std::mutex> lk(g_pool_mu);
        g_pool[dev].push_back(std::move(ctx));
    }
};

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int current_device(int* dev) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        return fail(KB_ERR_NO_DEVICE, "no CUDA device available (this library has no CPU path)");
    }
    e = cudaGetDevice(dev);
    if (e != cudaSuccess || *dev < 0 || *dev >= 64) return fail(KB_ERR_NO_DEVICE, "cudaGetDevice failed");
    return KB_OK;
}

// Host-side validation of the O(n) part of a CSR graph (xadj starts at 0
// and is monotone).  Targets in range and non-negative weights are checked
// on the device right after the upload (check_uploaded), before any kernel
// reads through adjncy.
// Host checks that size the upload: O(1).  Monotonicity of xadj, targets in
// range and weight signs are checked on the device right after the upload
// (check_uploaded), before any kernel reads through xadj; a host-side scan of
// xadj would cost ~10 ms per 2^24 nodes on every call.
int validate(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt) {
    (void)adjwgt;
    (void)vwgt;
    if (n < 0) return fail(KB_ERR_INVALID_INPUT, "n < 0");
    if (!xadj) return fail(KB_ERR_INVALID_INPUT, "xadj is NULL");
    if (xadj[0] != 0) return fail(KB_ERR_INVALID_INPUT, "xadj[0] != 0");
    const long long m = xadj[n];
    if (m < 0) return fail(KB_ERR_INVALID_INPUT, "xadj[n] < 0");
    if (m > 0 && !adjncy) return fail(KB_ERR_INVALID_INPUT, "adjncy is NULL");
    return KB_OK;
}

// Full host check for entry points that read the graph on the host.
int validate_host_graph(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt) {
    int rc = validate(n, xadj, adjncy, adjwgt, vwgt);
    if (rc) return rc;
    for (int v = 0; v < n; ++v)
        if (xadj[v + 1] < xadj[v]) return fail(KB_ERR_INVALID_INPUT, "xadj is not monotone");
    for (long long e = 0; e < xadj[n]; ++e)
        if (adjncy[e] < 0 || adjncy[e] >= n) return fail(KB_ERR_INVALID_INPUT, "adjncy entry out of range");
    return KB_OK;
}

// Device-side checks of an uploaded graph; throws InvalidInput.
struct InvalidInput : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check_uploaded(Ctx& ctx, DevGraph& g, uint32_t* total_weight = nullptr) {
    int flags = check_graph(ctx, g, total_weight, &g);
    g.unit_weights = (flags & 16) == 0;
    g.rows_sorted = (flags & 32) ? 0 : 1;
    if (flags & 1) throw InvalidInput("adjncy entry out of range");
    if (flags & 2) throw InvalidInput("negative edge weight");
    if (flags & 4) throw InvalidInput("negative node weight");
    if (flags & 8) throw InvalidInput("xadj does not start at 0 or is not monotone");
}

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const InvalidInput& e) {
        return fail(KB_ERR_INVALID_INPUT, e.what());
    } catch (const CudaError& e) {
        (void)cudaGetLastError();
        return fail(e.code == cudaErrorMemoryAllocation ? KB_ERR_OUT_OF_MEMORY : KB_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(KB_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(KB_ERR_INTERNAL, e.what());
    }
}

// Device copies of a host graph (unit weights expanded on the device).
struct Upload {
    DevGraph g;
    int* part = nullptr;
};

Upload upload(Ctx& ctx, int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt) {
    Upload u;
    const long long m = xadj[n];
    cudaStream_t s = ctx.stream;
    int* dx = ctx.hier.alloc<int>((size_t)n + 1);
    int* da = ctx.hier.alloc<int>((size_t)std::max<long long>(m, 1));
    int* dw = ctx.hier.alloc<int>((size_t)std::max<long long>(m, 1));
    int* dv = ctx.hier.alloc<int>((size_t)std::max(n, 1));
    u.part = ctx.hier.alloc<int>((size_t)std::max(n, 1));
    KB_CUDA(cudaMemcpyAsync(dx, xadj, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, s));
    if (m) KB_CUDA(cudaMemcpyAsync(da, adjncy, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice, s));
    if (adjwgt) {
        if (m) KB_CUDA(cudaMemcpyAsync(dw, adjwgt, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice, s));
    } else {
        fill_i32(dw, m, 1, s);
    }
    if (vwgt) {
        if (n) KB_CUDA(cudaMemcpyAsync(dv, vwgt, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
    } else {
        fill_i32(dv, n, 1, s);
    }
    u.g.n = n;
    u.g.m = m;
    u.g.xadj = dx;
    u.g.adjncy = da;
    u.g.adjwgt = dw;
    u.g.vwgt = dv;
    return u;
}

// upload + the device check, overlapped: the copy stream brings xadj, the
// node weights and then adjncy (and adjwgt) in kUploadChunks pieces of equal
// entry counts; the work stream fills unit weights meanwhile and checks every
// vertex range as soon as the pieces holding its rows have landed.  Throws
// InvalidInput like check_uploaded.
// Whether host memory p is page-locked (registered or cudaHostAlloc'd).
bool is_pinned(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

constexpr int kUploadChunks = 8;

Upload upload_checked(Ctx& ctx, int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                      uint32_t* total_weight) {
    Upload u;
    const long long m = xadj[n];
    cudaStream_t s = ctx.stream, cs = ctx.copies();
    int* dx = ctx.hier.alloc<int>((size_t)n + 1);
    int* da = ctx.hier.alloc<int>((size_t)std::max<long long>(m, 1));
    int* dw = ctx.hier.alloc<int>((size_t)std::max<long long>(m, 1));
    int* dv = ctx.hier.alloc<int>((size_t)std::max(n, 1));
    u.part = ctx.hier.alloc<int>((size_t)std::max(n, 1));
    u.g.n = n;
    u.g.m = m;
    u.g.xadj = dx;
    u.g.adjncy = da;
    u.g.adjwgt = dw;
    u.g.vwgt = dv;
    std::vector<cudaEvent_t> evs;
    auto mark = [&](cudaStream_t st) {
        cudaEvent_t e;
        KB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        KB_CUDA(cudaEventRecord(e, st));
        evs.push_back(e);
        return e;
    };
    struct Free {
        std::vector<cudaEvent_t>& e;
        ~Free() { for (auto x : e) cudaEventDestroy(x); }
    } free_evs{evs};
    // the copy stream starts after everything queued on the work stream
    KB_CUDA(cudaStreamWaitEvent(cs, mark(s), 0));
    KB_CUDA(cudaMemcpyAsync(dx, xadj, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, cs));
    if (vwgt && n) KB_CUDA(cudaMemcpyAsync(dv, vwgt, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, cs));
    const cudaEvent_t e_rows = mark(cs);
    const int C = m > 0 ? kUploadChunks : 0;
    std::vector<cudaEvent_t> e_chunk((size_t)C);
    auto chunk_lo = [&](int c) { return m * c / std::max(C, 1); };
    for (int c = 0; c < C; ++c) {
        const long long lo = chunk_lo(c), hi = chunk_lo(c + 1);
        if (hi > lo) {
            KB_CUDA(cudaMemcpyAsync(da + lo, adjncy + lo, sizeof(int) * (size_t)(hi - lo), cudaMemcpyHostToDevice, cs));
            if (adjwgt)
                KB_CUDA(cudaMemcpyAsync(dw + lo, adjwgt + lo, sizeof(int) * (size_t)(hi - lo), cudaMemcpyHostToDevice,
                                        cs));
        }
        e_chunk[(size_t)c] = mark(cs);
    }
    // work stream: unit weights, then the checks behind the pieces
    if (!adjwgt) fill_i32(dw, m, 1, s);
    if (!vwgt) fill_i32(dv, n, 1, s);
    check_graph_begin(ctx);
    KB_CUDA(cudaStreamWaitEvent(s, e_rows, 0));
    if (C == 0) {
        if (n > 0) check_graph_range(ctx, u.g, 0, n, !adjwgt);
    } else {
        // vertex ranges of about m / C entries each (host xadj; a broken xadj
        // is caught by the check itself, and then every piece has landed)
        int v0 = 0;
        for (int c = 0; c < C; ++c) {
            int v1 = n;
            if (c + 1 < C) {
                const long long target = chunk_lo(c + 1);
                v1 = (int)(std::lower_bound(xadj, xadj + n + 1, (int)std::min<long long>(target, INT_MAX)) - xadj);
                v1 = std::max(v0, std::min(v1, n));
            }
            // the pieces that hold entries [xadj[v0], xadj[v1]) (all of them
            // if those values are out of order or range)
            const long long e1 = xadj[v1];
            int need = C - 1;
            if (e1 >= 0 && e1 <= m && xadj[v0] <= e1) {
                need = 0;
                while (need + 1 < C && chunk_lo(need + 1) < e1) ++need;
            }
            KB_CUDA(cudaStreamWaitEvent(s, e_chunk[(size_t)need], 0));
            if (v1 > v0 || (c == 0 && n == 0)) check_graph_range(ctx, u.g, v0, v1, !adjwgt);
            v0 = v1;
        }
    }
    KB_CUDA(cudaStreamWaitEvent(s, mark(cs), 0));
    const int flags = check_graph_end(ctx, total_weight, &u.g);
    u.g.unit_weights = (flags & 16) == 0;
    u.g.rows_sorted = (flags & 32) ? 0 : 1;
    if (flags & 1) throw InvalidInput("adjncy entry out of range");
    if (flags & 2) throw InvalidInput("negative edge weight");
    if (flags & 4) throw InvalidInput("negative node weight");
    if (flags & 8) throw InvalidInput("xadj does not start at 0 or is not monotone");
    return u;
}

void fill_stats_families(Ctx& ctx, kb200_stats* st) {
    if (!st) return;
    ctx.collect();
    st->nfamilies = (int)std::min<size_t>(ctx.phases.size(), 32);
    for (int i = 0; i < st->nfamilies; ++i) {
        std::strncpy(st->family_name[i], ctx.phases[i].name.c_str(), 23);
        st->family_name[i][23] = 0;
        st->family_ms[i] = ctx.phases[i].ms;
        st->family_bytes[i] = ctx.phases[i].bytes;
        st->family_launches[i] = ctx.phases[i].launches;
    }
    unsigned long long w[3] = {0, 0, 0};
    KB_CUDA(cudaMemcpy(w, ctx.work, sizeof(w), cudaMemcpyDeviceToHost));
    st->sweep_vertices = (long long)w[0];
    st->sweep_edges = (long long)w[1];
    st->sweep_overflow_vertices = (long long)w[2];
    st->device_bytes_peak = ctx.hier.peak() + ctx.scratch.peak();
}

void begin_stats(Ctx& ctx, kb200_stats* st) {
    ctx.timing = st ? std::max(0, std::min(2, st->timing)) : 0;
    ctx.reset_stats();
}

using clk = std::chrono::steady_clock;
double ms_since(clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); }

int check_knobs(const kb200_knobs* kn) {
    if (!kn) return fail(KB_ERR_INVALID_INPUT, "knobs is NULL");
    if (kn->k < 1 || kn->lpc_subrounds < 1 || kn->ref_subrounds < 1 || kn->ref_classes < 1 ||
        kn->coarsening < 0 || kn->coarsening > 2 || kn->max_levels < 1 || kn->max_levels > 64 ||
        kn->refinement < 0 || kn->refinement > 1 || kn->jet_iters < 0 || kn->jet_patience < 1 ||
        kn->ip_mode < 0 || kn->ip_mode > 1 || kn->ip_jet_iters < 0 || kn->ip_jet_patience < 1)
        return fail(KB_ERR_INVALID_INPUT, "invalid knobs");
    return KB_OK;
}

int run_host_in(Ctx& ctx, int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                const Knobs& kn, long long* edgecut, int* part, kb200_stats* st, clk::time_point t0,
                const int* parent_a = nullptr, const int* parent_b = nullptr, bool derive_on_device = false);

// derive_on_device: kn carries k, imbalance, seed and mode only; the other
// knobs come from the node-weight sum the device check computes (saves a
// host pass over vwgt).
int run_host(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy, const Knobs& kn,
             long long* edgecut, int* part, kb200_stats* st, bool derive_on_device = false) {
    auto t0 = clk::now();
    int rc = validate(n, xadj, adjncy, adjcwgt, vwgt);
    if (rc || (rc = check_knobs(&kn))) return rc;
    if (!edgecut || (n > 0 && !part)) return fail(KB_ERR_INVALID_INPUT, "edgecut/part is NULL");
    int dev;
    if ((rc = current_device(&dev))) return rc;
    Lease lease(dev);
    return run_host_in(*lease.ctx, n, vwgt, xadj, adjcwgt, adjncy, kn, edgecut, part, st, t0, nullptr, nullptr,
                       derive_on_device);
}

// The body of a host-buffer call on a leased context (input already
// validated).  With parent_a / parent_b (host, n each) it is a combine.
int run_host_in(Ctx& ctx, int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                const Knobs& kn_in, long long* edgecut, int* part, kb200_stats* st, clk::time_point t0,
                const int* parent_a, const int* parent_b, bool derive_on_device) {
    Knobs kn = kn_in;
    const long long m = xadj[n];
    const bool comb = parent_a != nullptr;
    for (int attempt = 0;; ++attempt) {
        try {
            // a combine also holds both parents per level and one filtered level graph
            reserve_for(ctx, n, m, true, (attempt == 0 ? 1.0 : 2.0 * attempt) * (comb ? 1.5 : 1.0));
            begin_stats(ctx, st);
            auto th = clk::now();
            uint32_t W = 0;
            Upload up = upload_checked(ctx, n, xadj, adjncy, adjcwgt, vwgt, &W);
            if (derive_on_device) derive_knobs_total(n, W, kn_in.k, kn_in.imbalance, kn_in.seed, kn_in.mode, kn);
            int* dpar = nullptr;
            if (comb) {
                dpar = ctx.hier.alloc<int>(2 * (size_t)std::max(n, 1));
                if (n) {
                    KB_CUDA(cudaMemcpyAsync(dpar, parent_a, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, ctx.stream));
                    KB_CUDA(cudaMemcpyAsync(dpar + n, parent_b, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice,
                                            ctx.stream));
                }
                if (!parents_in_range(ctx, n, kn.k, dpar, dpar + n))
                    throw InvalidInput("parent block id out of range");
            }
            double ms_h2d = ms_since(th);
            long long cut = 0;
            // the result straight from the last refinement into a page-locked
            // caller buffer (overlapped with the final cut); else copied here
            bool host_done = false;
            int* early = (!comb && is_pinned(part)) ? part : nullptr;
            int r = comb ? combine(ctx, up.g, kn, dpar, dpar + n, up.part, &cut, st)
                         : partition(ctx, up.g, kn, up.part, &cut, st, early, &host_done);
            auto td = clk::now();
            if (n && !host_done)
                KB_CUDA(cudaMemcpyAsync(part, up.part, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, ctx.stream));
            KB_CUDA(cudaStreamSynchronize(ctx.stream));
            *edgecut = cut;
            if (st) {
                st->ms_h2d = ms_h2d;
                st->ms_d2h = ms_since(td);
                fill_stats_families(ctx, st);
                st->ms_total = ms_since(t0);
            }
            return r;
        } catch (const CudaError& e) {
            if (e.code == cudaErrorMemoryAllocation && attempt < 2 &&
                std::string(e.what()).find("arena exhausted") != std::string::npos) {
                (void)cudaGetLastError();
                continue;
            }
            throw;
        }
    }
}

// Phase helpers: host graph -> device, run f, copy results back.
struct PhaseRun {
    Lease lease;
    Ctx& ctx;
    Upload up;
    PhaseRun(int dev, int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt)
        : lease(dev), ctx(*lease.ctx) {
        reserve_for(ctx, n, xadj[n], true, 1.0);
        ctx.timing = 0;
        ctx.reset_stats();
        up = upload(ctx, n, xadj, adjncy, adjwgt, vwgt);
        check_uploaded(ctx, up.g);
        degree_stats(ctx, up.g);
    }
};

}  // namespace

// Error reporting shared with the entry points defined in other files.
int report_error(int code, const char* msg) { return fail(code, msg); }
void clear_error() { g_last_error.clear(); }
}  // namespace kb

using namespace kb;

#pragma GCC visibility push(default)
extern "C" {

int kb200_derive_knobs(int n, const int* vwgt, int k, double imbalance, int seed, int mode, kb200_knobs* out) {
    if (!out || k < 1 || n < 0) return fail(KB_ERR_INVALID_INPUT, "invalid arguments");
    derive_knobs(n, vwgt, k, imbalance, seed, mode, *out);
    return KB_OK;
}

int kb200_kaffpa(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy, int nparts,
                 double imbalance, int seed, int mode, long long* edgecut, int* part, kb200_stats* stats) {
    g_last_error.clear();
    return guarded([&]() -> int {
        if (n < 0 || !xadj) return fail(KB_ERR_INVALID_INPUT, "invalid graph");
        if (nparts < 1) return fail(KB_ERR_INVALID_INPUT, "nparts < 1");
        if (!(imbalance >= 0)) return fail(KB_ERR_INVALID_INPUT, "imbalance must be >= 0");
        Knobs kn;
        // unit weights: W = n now; explicit weights: W from the device check
        derive_knobs(n, nullptr, nparts, imbalance, seed, mode, kn);
        return run_host(n, vwgt, xadj, adjcwgt, adjncy, kn, edgecut, part, stats, vwgt != nullptr);
    });
}

int kb200_kaffpa_combine(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                         const kb200_knobs* kn, const int* part_a, const int* part_b, long long* edgecut, int* part,
                         kb200_stats* stats) {
    g_last_error.clear();
    return guarded([&]() -> int {
        auto t0 = clk::now();
        int rc = validate(n, xadj, adjncy, adjcwgt, vwgt);
        if (rc || (rc = check_knobs(kn))) return rc;
        if (kn->coarsening < 0 || kn->coarsening > 2) return fail(KB_ERR_INVALID_INPUT, "unknown coarsening");
        if (!edgecut || (n > 0 && (!part || !part_a || !part_b)))
            return fail(KB_ERR_INVALID_INPUT, "edgecut/part/parents is NULL");
        // parent block ids are range-checked on the device after the upload
        int dev;
        if ((rc = current_device(&dev))) return rc;
        Lease lease(dev);
        return run_host_in(*lease.ctx, n, vwgt, xadj, adjcwgt, adjncy, *kn, edgecut, part, stats, t0, part_a,
                           part_b);
    });
}

int kb200_kaffpae(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                  const kb200_knobs* kn, int population, int generations, int per_generation, int workers,
                  long long* edgecut, int* part, long long* history) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc = validate(n, xadj, adjncy, adjcwgt, vwgt);
        if (rc || (rc = check_knobs(kn))) return rc;
        if (population < 1 || generations < 0 || per_generation < 1)
            return fail(KB_ERR_INVALID_INPUT, "population >= 1, generations >= 0, per_generation >= 1 required");
        if (!edgecut || (n > 0 && !part)) return fail(KB_ERR_INVALID_INPUT, "edgecut/part is NULL");
        if (workers < 0) return fail(KB_ERR_INVALID_INPUT, "workers must be >= 0");
        int dev;
        if ((rc = current_device(&dev))) return rc;
        Lease lease(dev);
        Ctx& ctx = *lease.ctx;
        // worker contexts: 0 = as many as a round has offspring, at most 4
        const int Wk = workers > 0 ? workers : std::max(1, std::min(4, std::max(per_generation, 1)));
        std::vector<std::unique_ptr<Lease>> leases;
        std::vector<Ctx*> wctx;
        for (int w = 0; w < Wk; ++w) {
            leases.emplace_back(new Lease(dev));
            wctx.push_back(leases.back()->ctx.get());
        }
        const long long m = xadj[n];
        for (int attempt = 0;; ++attempt) {
            try {
                // the main context holds the graph; the workers reserve their own arenas
                reserve_for(ctx, n, m, true, attempt == 0 ? 1.0 : 2.0 * attempt);
                ctx.timing = 0;
                ctx.reset_stats();
                Upload up = upload(ctx, n, xadj, adjncy, adjcwgt, vwgt);
                check_uploaded(ctx, up.g);
                long long cut = 0;
                int r = kaffpae(ctx, wctx, up.g, *kn, population, generations, per_generation, up.part, &cut,
                                history);
                if (n) KB_CUDA(cudaMemcpyAsync(part, up.part, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, ctx.stream));
                KB_CUDA(cudaStreamSynchronize(ctx.stream));
                *edgecut = cut;
                return r;
            } catch (const CudaError& e) {
                if (e.code == cudaErrorMemoryAllocation && attempt < 2 &&
                    std::string(e.what()).find("arena exhausted") != std::string::npos) {
                    (void)cudaGetLastError();
                    continue;
                }
                throw;
            }
        }
    });
}

int kb200_kaffpa_knobs(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                       const kb200_knobs* kn, long long* edgecut, int* part, kb200_stats* stats) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc;
        if ((rc = check_knobs(kn))) return rc;
        return run_host(n, vwgt, xadj, adjcwgt, adjncy, *kn, edgecut, part, stats);
    });
}

static int run_device(int n, const int* d_vwgt, const int* d_xadj, const int* d_adjcwgt, const int* d_adjncy,
                      const kb200_knobs* kn_in, int nparts, double imbalance, int seed, int mode, long long* edgecut,
                      int* d_part, void* stream, kb200_stats* st) {
    g_last_error.clear();
    return guarded([&]() -> int {
        if (kn_in) {
            int rc = check_knobs(kn_in);
            if (rc) return rc;
            nparts = kn_in->k;
            imbalance = kn_in->imbalance;
        }
        if (n < 0 || nparts < 1 || !(imbalance >= 0) || !d_xadj || !d_vwgt || !d_adjcwgt || !edgecut)
            return fail(KB_ERR_INVALID_INPUT, "invalid arguments (device entry point needs explicit weights)");
        int dev, rc;
        if ((rc = current_device(&dev))) return rc;
        Lease lease(dev);
        Ctx& ctx = *lease.ctx;
        cudaStream_t user = (cudaStream_t)stream;
        cudaStream_t saved = ctx.stream;
        if (user) ctx.stream = user;
        struct Restore {
            Ctx& c;
            cudaStream_t s;
            ~Restore() { c.stream = s; }
        } restore{ctx, saved};
        auto t0 = clk::now();
        int m32 = 0;
        KB_CUDA(cudaMemcpyAsync(&m32, d_xadj + n, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
        KB_CUDA(cudaStreamSynchronize(ctx.stream));
        if (m32 < 0) return fail(KB_ERR_INVALID_INPUT, "xadj[n] < 0");
        DevGraph g;
        g.n = n;
        g.m = m32;
        g.xadj = d_xadj;
        g.adjncy = d_adjncy;
        g.adjwgt = d_adjcwgt;
        g.vwgt = d_vwgt;
        uint32_t W = 0;
        check_uploaded(ctx, g, &W);
        Knobs kn;
        if (kn_in) kn = *kn_in;
        else derive_knobs_total(n, W, nparts, imbalance, seed, mode, kn);
        for (int attempt = 0;; ++attempt) {
            try {
                reserve_for(ctx, n, m32, false, attempt == 0 ? 1.0 : 2.0 * attempt);
                begin_stats(ctx, st);
                long long cut = 0;
                int r = partition(ctx, g, kn, d_part, &cut, st);
                *edgecut = cut;
                if (st) {
                    fill_stats_families(ctx, st);
                    st->ms_total = ms_since(t0);
                }
                return r;
            } catch (const CudaError& e) {
                if (e.code == cudaErrorMemoryAllocation && attempt < 2 &&
                    std::string(e.what()).find("arena exhausted") != std::string::npos) {
                    (void)cudaGetLastError();
                    continue;
                }
                throw;
            }
        }
    });
}

int kb200_kaffpa_device(int n, const int* d_vwgt, const int* d_xadj, const int* d_adjcwgt, const int* d_adjncy,
                        int nparts, double imbalance, int seed, int mode, long long* edgecut, int* d_part,
                        void* stream, kb200_stats* st) {
    return run_device(n, d_vwgt, d_xadj, d_adjcwgt, d_adjncy, nullptr, nparts, imbalance, seed, mode, edgecut, d_part,
                      stream, st);
}

int kb200_kaffpa_device_knobs(int n, const int* d_vwgt, const int* d_xadj, const int* d_adjcwgt,
                              const int* d_adjncy, const kb200_knobs* kn, long long* edgecut, int* d_part,
                              void* stream, kb200_stats* st) {
    if (!kn) {
        g_last_error = "knobs is NULL";
        return KB_ERR_INVALID_INPUT;
    }
    return run_device(n, d_vwgt, d_xadj, d_adjcwgt, d_adjncy, kn, kn->k, kn->imbalance, kn->seed, kn->mode, edgecut,
                      d_part, stream, st);
}

int kb200_hem_match(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                    const kb200_knobs* kn, int level, const uint32_t* rating, int* label) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if ((rc = validate(n, xadj, adjncy, adjwgt, vwgt)) || (rc = check_knobs(kn))) return rc;
        if ((rc = current_device(&dev))) return rc;
        PhaseRun pr(dev, n, xadj, adjncy, adjwgt, vwgt);
        cudaStream_t s = pr.ctx.stream;
        int* d = pr.ctx.hier.alloc<int>((size_t)std::max(n, 1));
        uint32_t* dr = nullptr;
        const long long m = xadj[n];
        if (rating) {
            dr = pr.ctx.hier.alloc<uint32_t>((size_t)std::max<long long>(m, 1));
            if (m) KB_CUDA(cudaMemcpyAsync(dr, rating, sizeof(uint32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
        }
        hem_match(pr.ctx, pr.up.g, *kn, level, dr, d);
        if (n) KB_CUDA(cudaMemcpyAsync(label, d, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaStreamSynchronize(s));
        return KB_OK;
    });
}

int kb200_rating_infer(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                       const float* params, int use_tc, float* prob, uint32_t* rating) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if ((rc = validate(n, xadj, adjncy, adjwgt, vwgt))) return rc;
        if (!params) return fail(KB_ERR_INVALID_INPUT, "params is NULL");
        if ((rc = current_device(&dev))) return rc;
        PhaseRun pr(dev, n, xadj, adjncy, adjwgt, vwgt);
        cudaStream_t s = pr.ctx.stream;
        const long long m = xadj[n];
        const size_t mm = (size_t)std::max<long long>(m, 1);
        float* dp = pr.ctx.hier.alloc<float>(rm::kParams);
        float* dprob = prob ? pr.ctx.hier.alloc<float>(mm) : nullptr;
        uint32_t* drat = rating ? pr.ctx.hier.alloc<uint32_t>(mm) : nullptr;
        KB_CUDA(cudaMemcpyAsync(dp, params, sizeof(float) * rm::kParams, cudaMemcpyHostToDevice, s));
        rating_infer(pr.ctx, pr.up.g, dp, dprob, drat, use_tc != 0);
        int err = 0;
        KB_CUDA(cudaMemcpyAsync(&err, pr.ctx.dscalars + 60, sizeof(int), cudaMemcpyDeviceToHost, s));
        if (m && prob) KB_CUDA(cudaMemcpyAsync(prob, dprob, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost, s));
        if (m && rating)
            KB_CUDA(cudaMemcpyAsync(rating, drat, sizeof(uint32_t) * (size_t)m, cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaStreamSynchronize(s));
        if (err) return fail(KB_ERR_INTERNAL, "tensor-core layer kernel gave up waiting for its MMAs");
        return KB_OK;
    });
}

// Device copies of training graphs (explicit weights) and their labels.
struct TrainUpload {
    std::vector<TrainGraph> tg;
};

static int upload_train(Ctx& ctx, const kb200_train_graph* graphs, int count, TrainUpload& out) {
    cudaStream_t s = ctx.stream;
    for (int i = 0; i < count; ++i) {
        const kb200_train_graph& t = graphs[i];
        int rc = validate(t.n, t.xadj, t.adjncy, t.adjwgt, t.vwgt);
        if (rc) return rc;
        if (!t.adjwgt || !t.vwgt || (t.xadj[t.n] > 0 && !t.label))
            return fail(KB_ERR_INVALID_INPUT, "training graphs need explicit weights and labels");
        Upload u = upload(ctx, t.n, t.xadj, t.adjncy, t.adjwgt, t.vwgt);
        check_uploaded(ctx, u.g);
        degree_stats(ctx, u.g);
        const long long m = t.xadj[t.n];
        uint8_t* dl = ctx.hier.alloc<uint8_t>((size_t)std::max<long long>(m, 1));
        if (m) KB_CUDA(cudaMemcpyAsync(dl, t.label, (size_t)m, cudaMemcpyHostToDevice, s));
        out.tg.push_back(TrainGraph{u.g, dl});
    }
    return KB_OK;
}

static void reserve_train(Ctx& ctx, const kb200_train_graph* graphs, int count) {
    double hier = (double)rm::kParams * 4 + (1 << 20), scr = (1 << 24);
    long long nmax = 1;
    for (int i = 0; i < count; ++i) {
        const long long n = graphs[i].n, m = graphs[i].xadj[graphs[i].n];
        hier += 4.0 * (n + 1) + 13.0 * m + 8.0 * n + 2048;
        nmax = std::max(nmax, n);
    }
    scr += (double)nmax * 4 * (2 + 1 + 4 * 64 + 3 * 64 + 32 + 32 + 5 * 64) + 4.0 * rm::kParams * 4 + (1 << 20);
    ctx.hier.reserve((size_t)hier);
    ctx.scratch.reserve((size_t)scr);
}

int kb200_rating_train(const kb200_train_graph* graphs, int count, int steps, float lr, float* params, float* loss) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if (count < 1 || !graphs || steps < 0 || !params) return fail(KB_ERR_INVALID_INPUT, "invalid arguments");
        if ((rc = current_device(&dev))) return rc;
        Lease lease(dev);
        Ctx& ctx = *lease.ctx;
        reserve_train(ctx, graphs, count);
        ctx.timing = 0;
        ctx.reset_stats();
        TrainUpload tu;
        if ((rc = upload_train(ctx, graphs, count, tu))) return rc;
        float* dp = ctx.hier.alloc<float>(rm::kParams);
        KB_CUDA(cudaMemcpyAsync(dp, params, sizeof(float) * rm::kParams, cudaMemcpyHostToDevice, ctx.stream));
        rating_train(ctx, tu.tg.data(), count, steps, lr, dp, loss);
        KB_CUDA(cudaMemcpyAsync(params, dp, sizeof(float) * rm::kParams, cudaMemcpyDeviceToHost, ctx.stream));
        KB_CUDA(cudaStreamSynchronize(ctx.stream));
        return KB_OK;
    });
}

int kb200_rating_grad(const kb200_train_graph* graph, const float* params, float* grad, float* loss) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if (!graph || !params || !grad || !loss) return fail(KB_ERR_INVALID_INPUT, "invalid arguments");
        if ((rc = current_device(&dev))) return rc;
        Lease lease(dev);
        Ctx& ctx = *lease.ctx;
        reserve_train(ctx, graph, 1);
        ctx.timing = 0;
        ctx.reset_stats();
        TrainUpload tu;
        if ((rc = upload_train(ctx, graph, 1, tu))) return rc;
        float* dp = ctx.hier.alloc<float>(rm::kParams);
        float* dg = ctx.hier.alloc<float>(rm::kParams);
        KB_CUDA(cudaMemcpyAsync(dp, params, sizeof(float) * rm::kParams, cudaMemcpyHostToDevice, ctx.stream));
        rating_grad(ctx, tu.tg[0], dp, dg, loss);
        KB_CUDA(cudaMemcpyAsync(grad, dg, sizeof(float) * rm::kParams, cudaMemcpyDeviceToHost, ctx.stream));
        KB_CUDA(cudaStreamSynchronize(ctx.stream));
        return KB_OK;
    });
}

int kb200_lp_cluster(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                     const kb200_knobs* kn, int level, int* label) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if ((rc = validate(n, xadj, adjncy, adjwgt, vwgt)) || (rc = check_knobs(kn))) return rc;
        if ((rc = current_device(&dev))) return rc;
        PhaseRun pr(dev, n, xadj, adjncy, adjwgt, vwgt);
        int* d = pr.ctx.hier.alloc<int>((size_t)std::max(n, 1));
        lp_cluster(pr.ctx, pr.up.g, *kn, level, d);
        if (n) KB_CUDA(cudaMemcpyAsync(label, d, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, pr.ctx.stream));
        KB_CUDA(cudaStreamSynchronize(pr.ctx.stream));
        return KB_OK;
    });
}

int kb200_contract(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt, const int* label,
                   int* nc, long long* mc, int* cmap, int* cxadj, int* cadjncy, int* cadjwgt, int* cvwgt) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if ((rc = validate(n, xadj, adjncy, adjwgt, vwgt))) return rc;
        for (int v = 0; v < n; ++v)
            if (label[v] < 0 || label[v] >= n) return fail(KB_ERR_INVALID_INPUT, "label out of range");
        if ((rc = current_device(&dev))) return rc;
        PhaseRun pr(dev, n, xadj, adjncy, adjwgt, vwgt);
        cudaStream_t s = pr.ctx.stream;
        int* dl = pr.ctx.hier.alloc<int>((size_t)std::max(n, 1));
        int* dm = pr.ctx.hier.alloc<int>((size_t)std::max(n, 1));
        if (n) KB_CUDA(cudaMemcpyAsync(dl, label, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
        DevGraph c;
        int *cx, *ca, *cw, *cv;
        contract(pr.ctx, pr.up.g, dl, dm, c, &cx, &ca, &cw, &cv);
        *nc = c.n;
        *mc = c.m;
        if (n) KB_CUDA(cudaMemcpyAsync(cmap, dm, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaMemcpyAsync(cxadj, cx, sizeof(int) * ((size_t)c.n + 1), cudaMemcpyDeviceToHost, s));
        if (c.m) {
            KB_CUDA(cudaMemcpyAsync(cadjncy, ca, sizeof(int) * (size_t)c.m, cudaMemcpyDeviceToHost, s));
            KB_CUDA(cudaMemcpyAsync(cadjwgt, cw, sizeof(int) * (size_t)c.m, cudaMemcpyDeviceToHost, s));
        }
        if (c.n) KB_CUDA(cudaMemcpyAsync(cvwgt, cv, sizeof(int) * (size_t)c.n, cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaStreamSynchronize(s));
        return KB_OK;
    });
}

static int part_phase(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                      const kb200_knobs* kn, int level, uint32_t bound, int* part, int* balanced, int what) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if ((rc = validate(n, xadj, adjncy, adjwgt, vwgt)) || (rc = check_knobs(kn))) return rc;
        for (int v = 0; v < n; ++v)
            if (part[v] < 0 || part[v] >= kn->k) return fail(KB_ERR_INVALID_INPUT, "block id out of range");
        if ((rc = current_device(&dev))) return rc;
        PhaseRun pr(dev, n, xadj, adjncy, adjwgt, vwgt);
        cudaStream_t s = pr.ctx.stream;
        uint32_t* bw = pr.ctx.hier.alloc<uint32_t>((size_t)kn->k);
        if (n) KB_CUDA(cudaMemcpyAsync(pr.up.part, part, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
        block_weights_and_cut(pr.ctx, pr.up.g, pr.up.part, kn->k, bw, nullptr);
        if (what == 1) {
            bool ok = balance(pr.ctx, pr.up.g, *kn, level, bound, pr.up.part, bw);
            if (balanced) *balanced = ok ? 1 : 0;
        } else if (what == 2) {
            jet_refine(pr.ctx, pr.up.g, *kn, level, bound, pr.up.part, bw);
        } else {
            lp_refine(pr.ctx, pr.up.g, *kn, level, bound, pr.up.part, bw);
        }
        if (n) KB_CUDA(cudaMemcpyAsync(part, pr.up.part, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaStreamSynchronize(s));
        return KB_OK;
    });
}

int kb200_lp_refine(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                    const kb200_knobs* kn, int level, uint32_t bound, int* part) {
    return part_phase(n, xadj, adjncy, adjwgt, vwgt, kn, level, bound, part, nullptr, 0);
}

int kb200_jet_refine(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                     const kb200_knobs* kn, int level, uint32_t bound, int* part) {
    return part_phase(n, xadj, adjncy, adjwgt, vwgt, kn, level, bound, part, nullptr, 2);
}

int kb200_balance(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                  const kb200_knobs* kn, int level, uint32_t bound, int* part, int* balanced) {
    return part_phase(n, xadj, adjncy, adjwgt, vwgt, kn, level, bound, part, balanced, 1);
}

int kb200_edge_cut(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt, const int* part,
                   int k, long long* cut, uint32_t* bw) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if ((rc = validate(n, xadj, adjncy, adjwgt, vwgt))) return rc;
        if (k < 1 || !cut || (n > 0 && !part)) return fail(KB_ERR_INVALID_INPUT, "invalid arguments");
        for (int v = 0; v < n; ++v)
            if (part[v] < 0 || part[v] >= k) return fail(KB_ERR_INVALID_INPUT, "block id out of range");
        if ((rc = current_device(&dev))) return rc;
        PhaseRun pr(dev, n, xadj, adjncy, adjwgt, vwgt);
        cudaStream_t s = pr.ctx.stream;
        uint32_t* dbw = pr.ctx.hier.alloc<uint32_t>((size_t)k);
        if (n) KB_CUDA(cudaMemcpyAsync(pr.up.part, part, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
        unsigned long long* c2 = reinterpret_cast<unsigned long long*>(pr.ctx.dscalars + 32);
        block_weights_and_cut(pr.ctx, pr.up.g, pr.up.part, k, dbw, c2);
        unsigned long long h = 0;
        KB_CUDA(cudaMemcpyAsync(&h, c2, sizeof(h), cudaMemcpyDeviceToHost, s));
        if (bw) KB_CUDA(cudaMemcpyAsync(bw, dbw, sizeof(uint32_t) * (size_t)k, cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaStreamSynchronize(s));
        *cut = (long long)h / 2;
        return KB_OK;
    });
}

int kb200_project(int n, const int* cmap, int nc, const int* part_coarse, int* part_fine) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if (n < 0 || nc < 0) return fail(KB_ERR_INVALID_INPUT, "invalid sizes");
        for (int v = 0; v < n; ++v)
            if (cmap[v] < 0 || cmap[v] >= nc) return fail(KB_ERR_INVALID_INPUT, "cmap out of range");
        if ((rc = current_device(&dev))) return rc;
        Lease lease(dev);
        Ctx& ctx = *lease.ctx;
        ctx.hier.reserve(((size_t)n * 8 + (size_t)nc * 4) + (1 << 20));
        cudaStream_t s = ctx.stream;
        int* dm = ctx.hier.alloc<int>((size_t)std::max(n, 1));
        int* dc = ctx.hier.alloc<int>((size_t)std::max(nc, 1));
        int* df = ctx.hier.alloc<int>((size_t)std::max(n, 1));
        if (n) KB_CUDA(cudaMemcpyAsync(dm, cmap, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
        if (nc) KB_CUDA(cudaMemcpyAsync(dc, part_coarse, sizeof(int) * (size_t)nc, cudaMemcpyHostToDevice, s));
        project(ctx, n, dm, dc, df);
        if (n) KB_CUDA(cudaMemcpyAsync(part_fine, df, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaStreamSynchronize(s));
        return KB_OK;
    });
}

int kb200_initial_partition_device(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                                   const kb200_knobs* kn, int* part) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc, dev;
        if ((rc = validate(n, xadj, adjncy, adjwgt, vwgt)) || (rc = check_knobs(kn))) return rc;
        if (n > 0 && !part) return fail(KB_ERR_INVALID_INPUT, "part is NULL");
        if ((rc = current_device(&dev))) return rc;
        PhaseRun pr(dev, n, xadj, adjncy, adjwgt, vwgt);
        initial_partition_device(pr.ctx, pr.up.g, *kn, pr.up.part);
        if (n) KB_CUDA(cudaMemcpyAsync(part, pr.up.part, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, pr.ctx.stream));
        KB_CUDA(cudaStreamSynchronize(pr.ctx.stream));
        return KB_OK;
    });
}

int kb200_initial_partition(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                            const kb200_knobs* kn, int* part) {
    g_last_error.clear();
    return guarded([&]() -> int {
        int rc;
        if ((rc = validate_host_graph(n, xadj, adjncy, adjwgt, vwgt)) || (rc = check_knobs(kn))) return rc;
        if (!adjwgt || !vwgt) return fail(KB_ERR_INVALID_INPUT, "explicit weights required");
        initial_partition(n, xadj, adjncy, adjwgt, vwgt, *kn, part);
        return KB_OK;
    });
}

// ------------------------------------------------------------- batches
//
// Many independent partitioning calls on the current device.  Each worker
// thread leases its own context (arenas, stream) and takes items from a
// shared counter, largest first; host initial partitioning runs on the
// worker's thread (no nested threads), so the host cores are shared among
// graphs instead.  Every item's result is the one a single call with the same
// arguments returns.

// Default worker count: 8 (at most the host's cores).  With the initial
// partitioning on the device a worker spends its time queueing kernels; on
// a 512-graph batch (16-core host) 8 workers gave 296-308 partitions/s,
// 4 / 6 / 12 / 16 / 24 gave 151-194 / 205-266 / 192-194 / 125-168 / 158-170.
static int batch_workers(int requested, int count) {
    if (requested > 0) return std::min(requested, std::max(count, 1));
    unsigned hc = std::thread::hardware_concurrency();
    int w = (int)std::min(8u, hc ? hc : 8u);
    return std::max(1, std::min(w, std::max(count, 1)));
}

int kb200_kaffpa_batch(kb200_batch_item* items, int count, int workers, kb200_batch_report* report) {
    g_last_error.clear();
    return guarded([&]() -> int {
        if (count < 0 || (count > 0 && !items)) return fail(KB_ERR_INVALID_INPUT, "invalid batch");
        int dev, rc;
        if ((rc = current_device(&dev))) return rc;
        auto t0 = clk::now();
        std::vector<int> order((size_t)count);
        for (int i = 0; i < count; ++i) order[(size_t)i] = i;
        auto size_of = [&](int i) {
            const kb200_batch_item& it = items[i];
            return (it.n >= 0 && it.xadj) ? (long long)it.xadj[it.n] + it.n : 0LL;
        };
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return size_of(a) > size_of(b); });
        const int W = batch_workers(workers, count);
        std::atomic<int> next{0};
        auto work = [&]() {
            cudaSetDevice(dev);
            set_ip_thread_limit(W > 1 ? 0 : -1);
            std::unique_ptr<Lease> lease;
            for (int j; (j = next.fetch_add(1)) < count;) {
                kb200_batch_item& it = items[order[(size_t)j]];
                it.edgecut = -1;
                it.status = guarded([&]() -> int {
                    int r = validate(it.n, it.xadj, it.adjncy, it.adjwgt, it.vwgt);
                    if (r) return r;
                    if (it.nparts < 1 || !(it.imbalance >= 0) || (it.n > 0 && !it.part))
                        return fail(KB_ERR_INVALID_INPUT, "invalid batch item");
                    Knobs kn;
                    derive_knobs(it.n, it.vwgt, it.nparts, it.imbalance, it.seed, it.mode, kn);
                    if (!lease) lease.reset(new Lease(dev));
                    return run_host_in(*lease->ctx, it.n, it.vwgt, it.xadj, it.adjwgt, it.adjncy, kn, &it.edgecut,
                                       it.part, nullptr, clk::now());
                });
            }
            set_ip_thread_limit(-1);
        };
        std::vector<std::thread> pool;
        for (int w = 1; w < W; ++w) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        int failed = 0, first = KB_OK;
        for (int i = 0; i < count; ++i)
            if (items[i].status < 0) {
                if (!failed) first = items[i].status;
                ++failed;
            }
        if (report) {
            report->workers = W;
            report->failed = failed;
            report->ms_total = ms_since(t0);
        }
        if (failed) return fail(first, "some batch items failed (see their status)");
        return KB_OK;
    });
}

int kb200_kaffpa_population(int n, const int* d_vwgt, const int* d_xadj, const int* d_adjcwgt, const int* d_adjncy,
                            int nparts, double imbalance, int mode, const int* seeds, int count, long long* cuts,
                            int* d_parts, int workers, kb200_batch_report* report) {
    g_last_error.clear();
    return guarded([&]() -> int {
        if (n < 0 || nparts < 1 || !(imbalance >= 0) || !d_xadj || !d_vwgt || !d_adjcwgt || count < 0 ||
            (count > 0 && (!seeds || !cuts || !d_parts)))
            return fail(KB_ERR_INVALID_INPUT, "invalid arguments");
        int dev, rc;
        if ((rc = current_device(&dev))) return rc;
        auto t0 = clk::now();
        DevGraph g;
        uint32_t W = 0;
        {
            Lease lease(dev);
            Ctx& ctx = *lease.ctx;
            int m32 = 0;
            KB_CUDA(cudaMemcpyAsync(&m32, d_xadj + n, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
            KB_CUDA(cudaStreamSynchronize(ctx.stream));
            if (m32 < 0) return fail(KB_ERR_INVALID_INPUT, "xadj[n] < 0");
            g.n = n;
            g.m = m32;
            g.xadj = d_xadj;
            g.adjncy = d_adjncy;
            g.adjwgt = d_adjcwgt;
            g.vwgt = d_vwgt;
            check_uploaded(ctx, g, &W);
        }
        const int Wk = batch_workers(workers, count);
        std::atomic<int> next{0};
        std::vector<int> status((size_t)count, KB_OK);
        auto work = [&]() {
            cudaSetDevice(dev);
            set_ip_thread_limit(Wk > 1 ? 0 : -1);
            std::unique_ptr<Lease> lease;
            for (int i; (i = next.fetch_add(1)) < count;) {
                cuts[i] = -1;
                status[(size_t)i] = guarded([&]() -> int {
                    if (!lease) lease.reset(new Lease(dev));
                    Ctx& ctx = *lease->ctx;
                    Knobs kn;
                    derive_knobs_total(n, W, nparts, imbalance, seeds[i], mode, kn);
                    for (int attempt = 0;; ++attempt) {
                        try {
                            reserve_for(ctx, n, g.m, false, attempt == 0 ? 1.0 : 2.0 * attempt);
                            begin_stats(ctx, nullptr);
                            long long cut = 0;
                            int r = partition(ctx, g, kn, d_parts + (size_t)i * (size_t)n, &cut, nullptr);
                            KB_CUDA(cudaStreamSynchronize(ctx.stream));
                            cuts[i] = cut;
                            return r;
                        } catch (const CudaError& e) {
                            if (e.code == cudaErrorMemoryAllocation && attempt < 2 &&
                                std::string(e.what()).find("arena exhausted") != std::string::npos) {
                                (void)cudaGetLastError();
                                continue;
                            }
                            throw;
                        }
                    }
                });
            }
            set_ip_thread_limit(-1);
        };
        std::vector<std::thread> pool;
        for (int w = 1; w < Wk; ++w) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        int failed = 0, first = KB_OK;
        for (int i = 0; i < count; ++i)
            if (status[(size_t)i] < 0) {
                if (!failed) first = status[(size_t)i];
                ++failed;
            }
        if (report) {
            report->workers = Wk;
            report->failed = failed;
            report->ms_total = ms_since(t0);
        }
        if (failed) return fail(first, "some population members failed");
        return KB_OK;
    });
}

const char* kb200_last_error(void) { return g_last_error.c_str(); }

long long kb200_kernel_launches(void) { return g_kernel_launches.load(); }

int kb200_device_count(void) {
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return c;
}

// ------------------------------------------------ reference-compatible ABI

void kaffpa(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
            bool suppress_output, int seed, int mode, int* edgecut, int* part) {
    (void)suppress_output;  // the reference ignores it on this path too (kaHIP_interface.cpp:108-113)
    long long cut = -1;
    int rc = (n && nparts && imbalance)
                 ? kb200_kaffpa(*n, vwgt, xadj, adjcwgt, adjncy, *nparts, *imbalance, seed, mode, &cut, part, nullptr)
                 : KB_ERR_INVALID_INPUT;
    if (edgecut) *edgecut = rc < 0 ? -1 : (int)cut;
}

void kaffpa_balance(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                    bool perfectly_balance, bool suppress_output, int seed, int mode, int* edgecut, int* part) {
    // With perfectly_balance the reference partitions with the caller's
    // epsilon and then runs cycle refinement until every block weighs at
    // most (1+eps)*ceil(W/k) (kaHIP_interface.cpp:115-129).  That is the
    // bound U that kaffpa here already meets exactly (the balance repair of
    // every level guarantees max block <= U), so both values of the flag
    // partition with the caller's imbalance unchanged.
    (void)perfectly_balance;
    kaffpa(n, vwgt, xadj, adjcwgt, adjncy, nparts, imbalance, suppress_output, seed, mode, edgecut, part);
}

void kaffpa_balance_NE(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                       bool suppress_output, int seed, int mode, int* edgecut, int* part) {
    (void)n; (void)vwgt; (void)xadj; (void)adjcwgt; (void)adjncy; (void)nparts; (void)imbalance;
    (void)suppress_output; (void)seed; (void)mode; (void)part;
    g_last_error = "kaffpa_balance_NE is not provided by the B200 library";
    if (edgecut) *edgecut = -1;
}

void process_mapping(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* hierarchy_parameter,
                     int* distance_parameter, int hierarchy_depth, int mode_partitioning, int mode_mapping,
                     double* imbalance, bool suppress_output, int seed, int* edgecut, int* qap, int* part) {
    (void)n; (void)vwgt; (void)xadj; (void)adjcwgt; (void)adjncy; (void)hierarchy_parameter;
    (void)distance_parameter; (void)hierarchy_depth; (void)mode_partitioning; (void)mode_mapping;
    (void)imbalance; (void)suppress_output; (void)seed; (void)part;
    g_last_error = "process_mapping is not provided by the B200 library";
    if (edgecut) *edgecut = -1;
    if (qap) *qap = -1;
}

void node_separator(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                    bool suppress_output, int seed, int mode, int* num_separator_vertices, int** separator) {
    (void)n; (void)vwgt; (void)xadj; (void)adjcwgt; (void)adjncy; (void)nparts; (void)imbalance;
    (void)suppress_output; (void)seed; (void)mode;
    g_last_error = "node_separator is not provided by the B200 library";
    if (num_separator_vertices) *num_separator_vertices = -1;
    if (separator) *separator = nullptr;
}

void reduced_nd(int* n, int* xadj, int* adjncy, bool suppress_output, int seed, int mode, int* ordering) {
    (void)n; (void)xadj; (void)adjncy; (void)suppress_output; (void)seed; (void)mode; (void)ordering;
    g_last_error = "reduced_nd is not provided by the B200 library";
}

void edge_partitioning(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                       bool suppress_output, int seed, int mode, int* vertexcut, int* part,
                       int infinity_edge_weight) {
    (void)n; (void)vwgt; (void)xadj; (void)adjcwgt; (void)adjncy; (void)nparts; (void)imbalance;
    (void)suppress_output; (void)seed; (void)mode; (void)part; (void)infinity_edge_weight;
    g_last_error = "edge_partitioning is not provided by the B200 library";
    if (vertexcut) *vertexcut = -1;
}

}  // extern "C"
#pragma GCC visibility pop
