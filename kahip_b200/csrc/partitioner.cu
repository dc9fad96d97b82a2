// partitioner.cu -- the multilevel driver (graph_partitioner.cpp:240-273,
// coarsening.cpp:30-97, uncoarsening.cpp:43-121 restated for the device):
// coarsen by LP clustering + contraction until the simple stop rule says
// stop, partition the coarsest graph on the host, then project, repair
// balance and refine level by level.  Also holds the Ctx implementation.
#include "partitioner.cuh"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include "combine.cuh"
#include "contract.cuh"
#include "host/initial_partitioning.h"
#include "ip_device.cuh"
#include "jet.cuh"
#include "learned.cuh"
#include "match.cuh"
#include "prims.cuh"

namespace kb {

// ------------------------------------------------------------------- Ctx

Ctx::~Ctx() {
    if (device >= 0) cudaSetDevice(device);
    for (auto& p : pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : ev_free) cudaEventDestroy(e);
    if (origin) cudaEventDestroy(origin);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (pinned) cudaFreeHost(pinned);
    if (dscalars) cudaFree(dscalars);
    hier.free_all();
    scratch.free_all();
    if (own_stream && stream) cudaStreamDestroy(stream);
}

void Ctx::init(int dev, cudaStream_t s) {
    device = dev;
    KB_CUDA(cudaSetDevice(dev));
    if (!stream) {
        KB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        own_stream = true;
    }
    if (!pinned) KB_CUDA(cudaMallocHost(&pinned, 64 * sizeof(uint32_t)));
    if (!dscalars) {
        KB_CUDA(cudaMalloc(&dscalars, 64 * sizeof(int) + 4 * sizeof(unsigned long long)));
        work = reinterpret_cast<unsigned long long*>(dscalars + 64);
    }
    (void)s;
}

int Ctx::phase_id(const char* name) {
    for (size_t i = 0; i < phases.size(); ++i)
        if (phases[i].name == name) return (int)i;
    phases.push_back(PhaseTimer{name, 0, 0, 0});
    return (int)phases.size() - 1;
}

cudaEvent_t Ctx::ev() {
    if (!ev_free.empty()) {
        cudaEvent_t e = ev_free.back();
        ev_free.pop_back();
        return e;
    }
    cudaEvent_t e;
    KB_CUDA(cudaEventCreate(&e));
    return e;
}

cudaStream_t Ctx::copies() {
    if (!copy_stream) KB_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    return copy_stream;
}

void Ctx::begin(int phase, cudaEvent_t& a) {
    (void)phase;
    a = ev();
    KB_CUDA(cudaEventRecord(a, stream));
}

void Ctx::end(int phase, cudaEvent_t a, double bytes) {
    cudaEvent_t b = ev();
    KB_CUDA(cudaEventRecord(b, stream));
    pending.push_back(Pending{phase, a, b, bytes});
    if (pending.size() > 4096) {
        KB_CUDA(cudaStreamSynchronize(stream));
        collect();
    }
}

void Ctx::collect() {
    FILE* tf = (trace_path && origin && !pending.empty()) ? std::fopen(trace_path, "a") : nullptr;
    for (auto& p : pending) {
        float ms = 0;
        KB_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
        if (tf) {
            float t0 = 0, t1 = 0;
            KB_CUDA(cudaEventElapsedTime(&t0, origin, p.a));
            KB_CUDA(cudaEventElapsedTime(&t1, origin, p.b));
            std::fprintf(tf, "%s %.4f %.4f\n", phases[p.phase].name.c_str(), t0, t1);
        }
        phases[p.phase].ms += ms;
        phases[p.phase].bytes += p.bytes;
        phases[p.phase].launches += 1;
        ev_free.push_back(p.a);
        ev_free.push_back(p.b);
    }
    pending.clear();
    if (tf) std::fclose(tf);
}

void Ctx::reset_stats() {
    phases.clear();
    if (timing) {
        trace_path = std::getenv("KB200_TRACE");
        if (trace_path) {
            if (!origin) KB_CUDA(cudaEventCreate(&origin));
            KB_CUDA(cudaEventRecord(origin, stream));
            if (FILE* tf = std::fopen(trace_path, "a")) {
                std::fprintf(tf, "# call\n");
                std::fclose(tf);
            }
        }
    }
    if (work) KB_CUDA(cudaMemsetAsync(work, 0, 4 * sizeof(unsigned long long), stream));
    if (dscalars) KB_CUDA(cudaMemsetAsync(dscalars + 60, 0, sizeof(int), stream));
}

// ------------------------------------------------------------ the driver

namespace {

using clk = std::chrono::steady_clock;
double ms_since(clk::time_point t) {
    return std::chrono::duration<double, std::milli>(clk::now() - t).count();
}

struct Level {
    DevGraph g;
    int* cmap = nullptr;  // fine -> coarse (null at the coarsest level)
    int* part = nullptr;
};

uint32_t read_max_bw(Ctx& ctx, const uint32_t* bw, int k, std::vector<uint32_t>& host) {
    host.resize((size_t)k);
    KB_CUDA(cudaMemcpyAsync(host.data(), bw, sizeof(uint32_t) * (size_t)k, cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    uint32_t mx = 0;
    for (uint32_t x : host) mx = std::max(mx, x);
    return mx;
}

long long read_cut(Ctx& ctx, const DevGraph& g, const int* part, int k, uint32_t* bw) {
    unsigned long long* c = reinterpret_cast<unsigned long long*>(ctx.dscalars + 32);
    block_weights_and_cut(ctx, g, part, k, bw, c);
    unsigned long long h = 0;
    KB_CUDA(cudaMemcpyAsync(&h, c, sizeof(h), cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    return (long long)h / 2;
}

}  // namespace

void reserve_for(Ctx& ctx, int n, long long m, bool copy_input, double factor) {
    double hier = (copy_input ? 4.0 * (n + 1) + 8.0 * m + 4.0 * n : 0.0) + 12.0 * m + 40.0 * n + (64 << 20);
    // heavy-vertex hash tables are capped at min(1 GiB, 8 B per directed entry)
    double heavy = std::min(1.0 * (1 << 30), 8.0 * m) + (1 << 20);
    double scr = 40.0 * m + 48.0 * n + heavy + (64 << 20);
    ctx.hier.reserve((size_t)(hier * factor));
    ctx.scratch.reserve((size_t)(scr * factor));
}

// p1/p2 (device, n each, optional): the parents of a combine, p1 the better
// one; the coarsening then runs on the edges inside both parents' blocks and
// the coarsest graph takes p1 instead of an initial partitioning.
static int partition_once(Ctx& ctx, const DevGraph& g0, const Knobs& kn, int* d_part, long long* edgecut,
                          kb200_stats* st, const int* p1 = nullptr, const int* p2 = nullptr,
                          int* host_part = nullptr) {
    const int k = kn.k;
    const bool collect = st && st->collect_level_cuts;
    const bool combine = p1 != nullptr;
    cudaStream_t s = ctx.stream;
    std::vector<Level> lv;
    std::vector<const int*> P1{p1}, P2{p2};
    lv.push_back(Level{g0, nullptr, d_part});
    if (!lv[0].g.stats_known) degree_stats(ctx, lv[0].g);
    // learned rating: the model's parameters, once per call
    float* d_model = nullptr;
    if (kn.coarsening == 2 && kn.rating_model) {
        d_model = ctx.hier.alloc<float>(rm::kParams);
        KB_CUDA(cudaMemcpyAsync(d_model, kn.rating_model, sizeof(float) * rm::kParams, cudaMemcpyHostToDevice, s));
    }

    // ---------------------------------------------------------- coarsening
    auto t0 = clk::now();
    {
        int L = 0;
        while (L + 1 < kn.max_levels && lv[L].g.n > 0) {
            const DevGraph& f = lv[L].g;
            lv[L].cmap = ctx.hier.alloc<int>((size_t)f.n);
            const size_t mk = ctx.scratch.mark();
            int* label = ctx.scratch.alloc<int>((size_t)f.n);
            // a combine clusters on the edges inside both parents' blocks and
            // bundles no isolated nodes (they may lie in different blocks)
            DevGraph filtered;
            if (combine) filter_by_parents(ctx, f, P1[L], P2[L], filtered);
            const DevGraph& cg = combine ? filtered : f;
            bool lp = kn.coarsening == 0;
            if (!lp) {
                if (kn.coarsening == 2 && d_model && (kn.rating_levels <= 0 || L < kn.rating_levels)) {
                    uint32_t* rating = ctx.scratch.alloc<uint32_t>((size_t)std::max<long long>(cg.m, 1));
                    rating_infer(ctx, cg, d_model, nullptr, rating, true);
                    hem_match(ctx, cg, kn, L, rating, label);
                } else {
                    hem_match(ctx, cg, kn, L, nullptr, label);
                }
                if (!combine) bundle_isolated(ctx, cg, kn.max_vertex_weight + 1u, label);
                // a matching that removes less than 40 % of the nodes
                // (stars, skewed degrees) gives way to LP clustering
                const long long nc = count_leaders(ctx, f.n, label);
                lp = 5 * nc > 3 * (long long)f.n;
            }
            if (lp) {
                lp_cluster(ctx, cg, kn, L, label);
                if (!combine) bundle_isolated(ctx, cg, kn.cluster_bound, label);
            }
            Level c;
            int *cx, *ca, *cw, *cv;
            // contraction also fills the coarse graph's degree statistics
            contract(ctx, f, label, lv[L].cmap, c.g, &cx, &ca, &cw, &cv);
            ctx.scratch.release(mk);
            if (combine) {
                int* q1 = ctx.hier.alloc<int>((size_t)std::max(c.g.n, 1));
                int* q2 = ctx.hier.alloc<int>((size_t)std::max(c.g.n, 1));
                parents_to_coarse(ctx, f.n, lv[L].cmap, P1[L], P2[L], q1, q2);
                P1.push_back(q1);
                P2.push_back(q2);
            }
            const int nf = f.n, nc = c.g.n;
            lv.push_back(c);
            ++L;
            bool cont = (1.0 * nf / (double)nc >= 1.1) && (uint32_t)nc >= kn.num_stop;
            if (!cont) break;
        }
    }
    KB_CUDA(cudaStreamSynchronize(s));
    double ms_coarsen = ms_since(t0);
    const int L = (int)lv.size() - 1;

    // ------------------------------------------------ initial partitioning
    auto t1 = clk::now();
    for (int l = 1; l <= L; ++l) lv[l].part = ctx.hier.alloc<int>((size_t)std::max(lv[l].g.n, 1));
    long long initial_cut = 0;
    if (combine) {
        // the better parent, carried down the hierarchy
        const DevGraph& c = lv[L].g;
        if (c.n)
            KB_CUDA(cudaMemcpyAsync(lv[L].part, P1[L], sizeof(int) * (size_t)c.n, cudaMemcpyDeviceToDevice, s));
        const size_t mk = ctx.scratch.mark();
        uint32_t* tbw = ctx.scratch.alloc<uint32_t>((size_t)k);
        initial_cut = read_cut(ctx, c, lv[L].part, k, tbw);
        ctx.scratch.release(mk);
    } else if (kn.ip_mode == 1) {
        // on the device: every bisection of a recursion depth in one launch
        const DevGraph& c = lv[L].g;
        initial_partition_device(ctx, c, kn, lv[L].part);
        const size_t mk = ctx.scratch.mark();
        uint32_t* tbw = ctx.scratch.alloc<uint32_t>((size_t)k);
        initial_cut = read_cut(ctx, c, lv[L].part, k, tbw);
        ctx.scratch.release(mk);
    } else {
        const DevGraph& c = lv[L].g;
        std::vector<int> hx((size_t)c.n + 1), ha((size_t)c.m), hw((size_t)c.m), hv((size_t)c.n), hp((size_t)c.n);
        KB_CUDA(cudaMemcpyAsync(hx.data(), c.xadj, sizeof(int) * hx.size(), cudaMemcpyDeviceToHost, s));
        if (c.m) {
            KB_CUDA(cudaMemcpyAsync(ha.data(), c.adjncy, sizeof(int) * ha.size(), cudaMemcpyDeviceToHost, s));
            KB_CUDA(cudaMemcpyAsync(hw.data(), c.adjwgt, sizeof(int) * hw.size(), cudaMemcpyDeviceToHost, s));
        }
        if (c.n) KB_CUDA(cudaMemcpyAsync(hv.data(), c.vwgt, sizeof(int) * hv.size(), cudaMemcpyDeviceToHost, s));
        KB_CUDA(cudaStreamSynchronize(s));
        initial_partition(c.n, hx.data(), ha.data(), hw.data(), hv.data(), kn, hp.data());
        for (int v = 0; v < c.n; ++v)
            for (int e = hx[v]; e < hx[v + 1]; ++e)
                if (hp[v] != hp[ha[e]]) initial_cut += hw[e];
        initial_cut /= 2;
        if (c.n) KB_CUDA(cudaMemcpyAsync(lv[L].part, hp.data(), sizeof(int) * hp.size(), cudaMemcpyHostToDevice, s));
        KB_CUDA(cudaStreamSynchronize(s));
    }
    double ms_initial = ms_since(t1);

    // -------------------------------------------------------- uncoarsening
    auto t2 = clk::now();
    uint32_t* bw = ctx.hier.alloc<uint32_t>((size_t)k);
    std::vector<uint32_t> hbw;
    bool balanced = true;
    long long final_cut = 0;
    // LP refinement: a vertex can only move if it has a neighbour in another
    // block, and then so does its coarse node one level up -- the first
    // round sweeps only vertices whose coarse node was on the boundary after
    // that level's refinement (all of them again when the balance repair ran)
    const size_t mkb = ctx.scratch.mark();
    uint8_t* bflag[2] = {nullptr, nullptr};
    if (kn.refinement == 0 && L > 0) {
        bflag[0] = ctx.scratch.alloc<uint8_t>((size_t)std::max(lv[0].g.n, 1));
        bflag[1] = ctx.scratch.alloc<uint8_t>((size_t)std::max(lv[0].g.n, 1));
    }
    const uint8_t* cb = nullptr;  // boundary flags of level l + 1
    // LP refinement never lets a block exceed the bound it refines under, and
    // projection keeps block weights: after a level that ended within its
    // bound, the next level under the same bound needs no balance check
    bool within = false;
    uint32_t within_bound = 0;
    for (int l = L; l >= 0; --l) {
        const DevGraph& g = lv[l].g;
        uint8_t* act0 = cb ? bflag[l & 1] : nullptr;
        if (l < L) project(ctx, g.n, lv[l].cmap, lv[l + 1].part, lv[l].part, cb, act0);
        const uint32_t bound = l == 0 ? kn.final_bound : kn.upper_bound;
        block_weights_and_cut(ctx, g, lv[l].part, k, bw, nullptr);
        bool repaired = false;
        const bool ok = (within && bound == within_bound) ? true
                                                         : balance(ctx, g, kn, l, bound, lv[l].part, bw, nullptr, &repaired);
        within = ok && kn.refinement == 0;
        within_bound = bound;
        if (kn.refinement == 1) jet_refine(ctx, g, kn, l, bound, lv[l].part, bw);
        else lp_refine(ctx, g, kn, l, bound, lv[l].part, bw, repaired ? nullptr : act0);
        // (level l's own flags replace its first-round set, which is no
        // longer needed; level l - 1 projects them into the other buffer)
        cb = nullptr;
        if (bflag[0] && l > 0) {
            boundary_flags(ctx, g, lv[l].part, bflag[l & 1]);
            cb = bflag[l & 1];
        }
        if (l == 0 && host_part && g.n) {
            // the final partition goes to the host on the copy stream while the
            // cut and block weights are computed
            cudaEvent_t done = ctx.ev();
            KB_CUDA(cudaEventRecord(done, s));
            KB_CUDA(cudaStreamWaitEvent(ctx.copies(), done, 0));
            KB_CUDA(cudaMemcpyAsync(host_part, lv[0].part, sizeof(int) * (size_t)g.n, cudaMemcpyDeviceToHost,
                                    ctx.copies()));
            ctx.ev_free.push_back(done);
        }
        if (l == 0) balanced = ok;
        if (collect || l == 0) {
            long long c = read_cut(ctx, g, lv[l].part, k, bw);
            uint32_t mx = read_max_bw(ctx, bw, k, hbw);
            if (l == 0) { final_cut = c; balanced = mx <= bound; }
            if (st && l < 64) { st->level_cut[l] = c; st->level_maxbw[l] = mx; }
        }
    }
    ctx.scratch.release(mkb);
    KB_CUDA(cudaStreamSynchronize(s));
    if (host_part) KB_CUDA(cudaStreamSynchronize(ctx.copies()));
    double ms_uncoarsen = ms_since(t2);

    {
        int err = 0;
        KB_CUDA(cudaMemcpy(&err, ctx.dscalars + 60, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) throw std::runtime_error("device hash table overflow (internal invariant broken)");
    }
    *edgecut = final_cut;
    if (st) {
        st->levels = L + 1;
        for (int l = 0; l <= L && l < 64; ++l) {
            st->level_n[l] = lv[l].g.n;
            st->level_m[l] = lv[l].g.m;
        }
        st->initial_cut = initial_cut;
        st->balanced = balanced ? 1 : 0;
        st->ms_coarsen = ms_coarsen;
        st->ms_initial = ms_initial;
        st->ms_uncoarsen = ms_uncoarsen;
    }
    return balanced ? KB_OK : KB_WARN_IMBALANCED;
}

void partition_quality(Ctx& ctx, const DevGraph& g, const int* part, int k, uint32_t bound, uint64_t* ov,
                       long long* cut) {
    const size_t mk = ctx.scratch.mark();
    uint32_t* bw = ctx.scratch.alloc<uint32_t>((size_t)k);
    *cut = read_cut(ctx, g, part, k, bw);
    std::vector<uint32_t> h((size_t)k);
    KB_CUDA(cudaMemcpyAsync(h.data(), bw, sizeof(uint32_t) * (size_t)k, cudaMemcpyDeviceToHost, ctx.stream));
    KB_CUDA(cudaStreamSynchronize(ctx.stream));
    ctx.scratch.release(mk);
    *ov = 0;
    for (uint32_t x : h) if (x > bound) *ov += x - bound;
}

int combine(Ctx& ctx, const DevGraph& g0, const Knobs& kn, const int* pa, const int* pb, int* d_part,
            long long* edgecut, kb200_stats* st) {
    if (st) st->rating_fallback_used = 0;
    uint64_t ova, ovb;
    long long ca, cb;
    partition_quality(ctx, g0, pa, kn.k, kn.final_bound, &ova, &ca);
    partition_quality(ctx, g0, pb, kn.k, kn.final_bound, &ovb, &cb);
    const bool b_first = ovb < ova || (ovb == ova && cb < ca);
    const int* p1 = b_first ? pb : pa;
    const int* p2 = b_first ? pa : pb;
    const uint64_t ov1 = b_first ? ovb : ova;
    const long long c1 = b_first ? cb : ca;
    int r = partition_once(ctx, g0, kn, d_part, edgecut, st, p1, p2);
    uint64_t ovr;
    long long cr;
    partition_quality(ctx, g0, d_part, kn.k, kn.final_bound, &ovr, &cr);
    if (ov1 < ovr || (ov1 == ovr && c1 < cr)) {
        // never worse than the better parent
        if (g0.n) KB_CUDA(cudaMemcpyAsync(d_part, p1, sizeof(int) * (size_t)g0.n, cudaMemcpyDeviceToDevice, ctx.stream));
        KB_CUDA(cudaStreamSynchronize(ctx.stream));
        *edgecut = c1;
        r = ov1 == 0 ? KB_OK : KB_WARN_IMBALANCED;
        if (st) st->balanced = ov1 == 0 ? 1 : 0;
    }
    return r;
}

int partition(Ctx& ctx, const DevGraph& g0, const Knobs& kn, int* d_part, long long* edgecut,
              kb200_stats* st, int* host_part, bool* host_done) {
    if (st) st->rating_fallback_used = 0;
    if (host_done) *host_done = false;
    if (!(kn.coarsening == 2 && kn.rating_model && kn.rating_fallback > 0)) {
        const int r = partition_once(ctx, g0, kn, d_part, edgecut, st, nullptr, nullptr, host_part);
        if (host_done) *host_done = host_part != nullptr;
        return r;
    }
    // learned rating with a guard: the expansion*^2 matching runs too, and
    // its partition is kept when the learned one cuts more than
    // rating_fallback times as much
    int* plain = ctx.hier.alloc<int>((size_t)std::max(g0.n, 1));
    const size_t mk = ctx.hier.mark();
    Knobs kp = kn;
    kp.coarsening = 1;
    long long cut_plain = 0;
    const int rp = partition_once(ctx, g0, kp, plain, &cut_plain, nullptr);
    ctx.hier.release(mk);
    long long cut_learned = 0;
    const int rl = partition_once(ctx, g0, kn, d_part, &cut_learned, st);
    if ((double)cut_learned > kn.rating_fallback * (double)cut_plain) {
        if (g0.n)
            KB_CUDA(cudaMemcpyAsync(d_part, plain, sizeof(int) * (size_t)g0.n, cudaMemcpyDeviceToDevice, ctx.stream));
        KB_CUDA(cudaStreamSynchronize(ctx.stream));
        *edgecut = cut_plain;
        if (st) st->rating_fallback_used = 1;
        return rp;
    }
    *edgecut = cut_learned;
    return rl;
}

}  // namespace kb
