// initial_partitioning.cpp -- host initial partitioner for the coarsest graph.
//
// Recursive multilevel bisection, as the reference's initial partitioning
// (initial_partitioning.cpp:39-134 -> graph_partitioner.cpp:110-238 ->
// bipartition.cpp:24-222) is built, made deterministic:
//   * k blocks split as ceil(k/2) | floor(k/2), target weights in proportion;
//     each side may exceed its target by max((1+eps)^(1/ceil log2 k) - 1,
//     min(eps, 1%));
//   * a bisection coarsens by sequential heavy-edge matching on the
//     expansion*^2 rating while the graph has > 200 nodes and shrinks by at
//     least 1.1 (node weight bound 1.5 W / 200), runs `tries` greedy growings
//     from a pseudo-peripheral node (BFS twice from a hashed start), each
//     with 2-way FM, keeps the best by (overload, cut), and refines with FM
//     on every level on the way up;
//   * `reps` repetitions of the whole recursion keep the smallest cut.
// The graph is small (a few thousand nodes), so this stays on the host.
// Repetitions, the two halves of a bisection and the tries of a bisection
// are independent (their hash streams are keyed by position, not by order
// of execution) and run as tasks of one process-wide thread pool; results
// are reduced in index order, so they do not depend on the thread count.
#include "initial_partitioning.h"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../hash.h"

namespace kb {

namespace {

// Fork-join pool: run(count, f) calls f(0..count-1) on the caller and on
// idle workers and returns when all calls are done; a waiting caller runs
// queued work meanwhile, so nested run() calls cannot deadlock.
class TaskPool {
public:
    static TaskPool& get() {
        static TaskPool* pool = new TaskPool();  // never destroyed: workers may outlive static teardown
        return *pool;
    }

    void run(int count, const std::function<void(int)>& f) {
        if (count <= 0) return;
        if (count == 1 || workers_ == 0) {
            for (int i = 0; i < count; ++i) f(i);
            return;
        }
        auto job = std::make_shared<Job>();
        job->f = &f;
        job->count = count;
        int posted = 0;
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int i = 1; i < count && i <= workers_; ++i, ++posted) queue_.push_back(job);
            queued_.store((int)queue_.size(), std::memory_order_release);
        }
        for (int i = 0; i < posted; ++i) cv_.notify_one();
        work_on(*job);
        while (job->done.load(std::memory_order_acquire) < count) {
            if (!run_one()) std::this_thread::yield();
        }
    }

private:
    struct Job {
        const std::function<void(int)>* f = nullptr;
        int count = 0;
        std::atomic<int> next{0}, done{0};
    };

    TaskPool() {
        unsigned hw = std::thread::hardware_concurrency();
        workers_ = (int)std::min(15u, hw > 1 ? hw - 1 : 0u);
        for (int i = 0; i < workers_; ++i) std::thread([this] { loop(); }).detach();
    }

    static void work_on(Job& j) {
        for (int i; (i = j.next.fetch_add(1, std::memory_order_relaxed)) < j.count;) {
            (*j.f)(i);
            j.done.fetch_add(1, std::memory_order_release);
        }
    }

    bool run_one() {
        if (queued_.load(std::memory_order_acquire) == 0) return false;
        std::shared_ptr<Job> j;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (queue_.empty()) return false;
            j = std::move(queue_.front());
            queue_.pop_front();
            queued_.store((int)queue_.size(), std::memory_order_release);
        }
        work_on(*j);
        return true;
    }

    void loop() {
        for (;;) {
            // a short spin before sleeping: fork-join waves come in quick succession
            for (int spin = 0; spin < 20000; ++spin) {
                if (run_one()) spin = 0;
                else std::this_thread::yield();
            }
            std::shared_ptr<Job> j;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return !queue_.empty(); });
                j = std::move(queue_.front());
                queue_.pop_front();
                queued_.store((int)queue_.size(), std::memory_order_release);
            }
            work_on(*j);
        }
    }

    int workers_ = 0;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::shared_ptr<Job>> queue_;
    std::atomic<int> queued_{0};
};

// f(0..count-1), on the pool when par is set
void for_each_index(int count, bool par, const std::function<void(int)>& f) {
    if (par) {
        TaskPool::get().run(count, f);
    } else {
        for (int i = 0; i < count; ++i) f(i);
    }
}

struct HostGraph {
    int n = 0;
    std::vector<int> xadj, adjncy, adjwgt, vwgt;
    long long weight() const {
        long long w = 0;
        for (int x : vwgt) w += x;
        return w;
    }
};

// Indexed binary max-heap over node ids, priority (key desc, id asc).
class GainHeap {
public:
    explicit GainHeap(int n) : pos_(n, -1) { heap_.reserve(n); }
    bool empty() const { return heap_.empty(); }
    bool contains(int v) const { return pos_[v] >= 0; }
    void push(int v, const std::vector<long long>& key) {
        pos_[v] = (int)heap_.size();
        heap_.push_back(v);
        sift_up(pos_[v], key);
    }
    int pop(const std::vector<long long>& key) {
        int top = heap_[0];
        pos_[top] = -1;
        int last = heap_.back();
        heap_.pop_back();
        if (!heap_.empty()) {
            heap_[0] = last;
            pos_[last] = 0;
            sift_down(0, key);
        }
        return top;
    }
    void changed(int v, const std::vector<long long>& key) {
        sift_up(pos_[v], key);
        sift_down(pos_[v], key);
    }
    // after key[v] grew / shrank: one direction suffices
    void increased(int v, const std::vector<long long>& key) { sift_up(pos_[v], key); }
    void decreased(int v, const std::vector<long long>& key) { sift_down(pos_[v], key); }
    // heap of the given nodes (none of them queued), built bottom-up
    void build(const std::vector<int>& nodes, const std::vector<long long>& key) {
        for (int v : nodes) {
            pos_[v] = (int)heap_.size();
            heap_.push_back(v);
        }
        for (int i = (int)heap_.size() / 2 - 1; i >= 0; --i) sift_down(i, key);
    }
    void clear() {
        for (int v : heap_) pos_[v] = -1;
        heap_.clear();
    }

private:
    static bool below(int a, int b, const std::vector<long long>& key) {  // a ranks below b
        return key[a] != key[b] ? key[a] < key[b] : a > b;
    }
    void put(int i, int v) { heap_[i] = v; pos_[v] = i; }
    void sift_up(int i, const std::vector<long long>& key) {
        int v = heap_[i];
        while (i > 0) {
            int p = (i - 1) >> 1;
            if (!below(heap_[p], v, key)) break;
            put(i, heap_[p]);
            i = p;
        }
        put(i, v);
    }
    void sift_down(int i, const std::vector<long long>& key) {
        int v = heap_[i];
        const int sz = (int)heap_.size();
        for (;;) {
            int l = 2 * i + 1, r = l + 1, best = i;
            int bv = v;
            if (l < sz && below(bv, heap_[l], key)) { best = l; bv = heap_[l]; }
            if (r < sz && below(bv, heap_[r], key)) { best = r; bv = heap_[r]; }
            if (best == i) break;
            put(i, heap_[best]);
            i = best;
        }
        put(i, v);
    }
    std::vector<int> heap_;
    std::vector<int> pos_;
};

struct Limits {
    uint64_t maxw[2];
    uint64_t overload(const uint64_t w[2]) const {
        uint64_t o = 0;
        for (int s = 0; s < 2; ++s) o += w[s] > maxw[s] ? w[s] - maxw[s] : 0;
        return o;
    }
};

long long cut_of(const HostGraph& g, const std::vector<char>& side) {
    long long c = 0;
    for (int v = 0; v < g.n; ++v)
        for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e)
            if (side[v] != side[g.adjncy[e]]) c += g.adjwgt[e];
    return c / 2;
}

// Last node dequeued by a breadth-first search from s.
int farthest(const HostGraph& g, int s) {
    thread_local std::vector<char> seen;
    thread_local std::vector<int> q;
    seen.assign(g.n, 0);
    q.clear();
    q.push_back(s);
    seen[s] = 1;
    for (size_t h = 0; h < q.size(); ++h) {
        int v = q[h];
        for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
            int u = g.adjncy[e];
            if (!seen[u]) { seen[u] = 1; q.push_back(u); }
        }
    }
    return q.back();
}

// Greedy growing of side 0 from `start` towards `target0` without
// exceeding max0.  Gain of a side-1 node = w(to side 0) - w(to side 1).
void grow_region(const HostGraph& g, int start, uint64_t target0, uint64_t max0,
                 std::vector<char>& side, std::vector<long long>& key, GainHeap& heap) {
    side.assign(g.n, 1);
    thread_local std::vector<char> skipped;
    skipped.assign(g.n, 0);
    for (int v = 0; v < g.n; ++v) {
        long long d = 0;
        for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e) d += g.adjwgt[e];
        key[v] = -d;
    }
    uint64_t w0 = 0;
    int scan = 0;
    int pending = start;
    while (w0 < target0) {
        int v;
        if (pending >= 0) {
            v = pending;
            pending = -1;
        } else if (!heap.empty()) {
            v = heap.pop(key);
        } else {
            while (scan < g.n && (side[scan] == 0 || skipped[scan])) ++scan;
            if (scan == g.n) break;
            v = scan;
        }
        if (side[v] == 0 || skipped[v]) continue;
        if (w0 + (uint64_t)g.vwgt[v] > max0) { skipped[v] = 1; continue; }
        side[v] = 0;
        w0 += (uint64_t)g.vwgt[v];
        for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
            int u = g.adjncy[e];
            if (side[u] == 0 || skipped[u]) continue;
            key[u] += 2LL * g.adjwgt[e];
            if (heap.contains(u)) heap.increased(u, key);
            else heap.push(u, key);
        }
    }
    heap.clear();
}

// 2-way FM with rollback to the best prefix by (overload, cut).
long long fm_refine(const HostGraph& g, std::vector<char>& side, const Limits& lim, int passes,
                    int stall_limit, std::vector<long long>& key, GainHeap& heap) {
    uint64_t w[2] = {0, 0};
    for (int v = 0; v < g.n; ++v) w[(int)side[v]] += (uint64_t)g.vwgt[v];
    thread_local std::vector<char> locked;
    thread_local std::vector<int> log, boundary;
    locked.assign(g.n, 0);
    log.clear();
    long long cut = cut_of(g, side);
    for (int pass = 0; pass < passes; ++pass) {
        boundary.clear();
        for (int v = 0; v < g.n; ++v) {
            long long inside = 0, outside = 0;
            for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e)
                (side[g.adjncy[e]] == side[v] ? inside : outside) += g.adjwgt[e];
            key[v] = outside - inside;
            if (outside > 0) boundary.push_back(v);
        }
        heap.build(boundary, key);
        log.clear();
        size_t best_len = 0;
        int stall = 0;
        long long cur = cut, best_cut = cut;
        uint64_t best_ov = lim.overload(w);
        while (!heap.empty() && stall < stall_limit) {
            int v = heap.pop(key);
            int from = side[v], to = 1 - from;
            if (w[to] + (uint64_t)g.vwgt[v] > lim.maxw[to]) continue;
            side[v] = (char)to;
            w[from] -= (uint64_t)g.vwgt[v];
            w[to] += (uint64_t)g.vwgt[v];
            cur -= key[v];
            locked[v] = 1;
            log.push_back(v);
            for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
                int u = g.adjncy[e];
                if (locked[u]) continue;
                const long long d = 2LL * g.adjwgt[e];
                const bool drop = side[u] == to;
                key[u] += drop ? -d : d;
                if (!heap.contains(u)) heap.push(u, key);
                else if (drop) heap.decreased(u, key);
                else heap.increased(u, key);
            }
            uint64_t ov = lim.overload(w);
            if (ov < best_ov || (ov == best_ov && cur < best_cut)) {
                best_ov = ov;
                best_cut = cur;
                best_len = log.size();
                stall = 0;
            } else {
                ++stall;
            }
        }
        heap.clear();
        while (log.size() > best_len) {
            int v = log.back();
            log.pop_back();
            int from = side[v], to = 1 - from;
            side[v] = (char)to;
            w[from] -= (uint64_t)g.vwgt[v];
            w[to] += (uint64_t)g.vwgt[v];
        }
        for (int v : log) locked[v] = 0;
        // moves that were undone are unlocked too
        std::fill(locked.begin(), locked.end(), 0);
        cut = best_cut;
        if (best_len == 0) break;
    }
    return cut;
}

// Matching-based coarsening step: nodes visited in hash order, each
// unmatched node takes the unmatched neighbour of best expansion*^2 rating
// (edge_ratings.cpp:171-183), ties to the smaller id.  Leader = min id.
std::vector<int> heavy_edge_labels(const HostGraph& g, uint64_t ks, uint64_t maxnode) {
    // (hash, id) order by a stable LSD radix sort on the hash (ids start
    // ascending): the same order as sorting the pairs
    thread_local std::vector<std::pair<uint32_t, int>> tmp;
    std::vector<std::pair<uint32_t, int>> order(g.n);
    tmp.resize(g.n);
    for (int v = 0; v < g.n; ++v) order[v] = {hash32(ks, (uint32_t)v), v};
    for (int sh = 0; sh < 32; sh += 8) {
        int cnt[257] = {0};
        for (int i = 0; i < g.n; ++i) ++cnt[((order[i].first >> sh) & 255u) + 1];
        for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
        for (int i = 0; i < g.n; ++i) tmp[cnt[(order[i].first >> sh) & 255u]++] = order[i];
        order.swap(tmp);
    }
    std::vector<int> mate(g.n, -1);
    for (const auto& hv : order) {
        int u = hv.second;
        if (mate[u] >= 0) continue;
        const uint32_t cu = (uint32_t)g.vwgt[u];
        int pick = -1;
        double pr = 0;
        for (int e = g.xadj[u]; e < g.xadj[u + 1]; ++e) {
            int v = g.adjncy[e];
            if (v == u || mate[v] >= 0) continue;
            const uint32_t cv = (uint32_t)g.vwgt[v];
            if ((uint64_t)cu + cv > maxnode) continue;
            const int w = g.adjwgt[e];
            double r = 1.0 * w * w / (uint32_t)(cu * cv);
            if (pick < 0 || r > pr || (r == pr && v < pick)) { pick = v; pr = r; }
        }
        if (pick < 0) {
            mate[u] = u;
        } else {
            mate[u] = pick;
            mate[pick] = u;
        }
    }
    std::vector<int> label(g.n);
    for (int v = 0; v < g.n; ++v) label[v] = std::min(v, mate[v]);
    return label;
}

// Contraction on the host (coarse ids by smallest member, rows sorted).
HostGraph contract_host(const HostGraph& g, const std::vector<int>& label, std::vector<int>& cmap) {
    std::vector<int> id(g.n, -1);
    cmap.assign(g.n, 0);
    int nc = 0;
    for (int v = 0; v < g.n; ++v) {
        if (id[label[v]] < 0) id[label[v]] = nc++;
        cmap[v] = id[label[v]];
    }
    HostGraph c;
    c.n = nc;
    c.vwgt.assign(nc, 0);
    for (int v = 0; v < g.n; ++v) c.vwgt[cmap[v]] += g.vwgt[v];
    // members of every coarse node by counting sort
    std::vector<int> start(nc + 1, 0), mem(g.n);
    for (int v = 0; v < g.n; ++v) start[cmap[v] + 1]++;
    for (int i = 0; i < nc; ++i) start[i + 1] += start[i];
    {
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (int v = 0; v < g.n; ++v) mem[fill[cmap[v]]++] = v;
    }
    std::vector<uint32_t> acc(nc, 0);
    std::vector<char> hit(nc, 0);
    std::vector<int> targets;
    c.xadj.assign(nc + 1, 0);
    c.adjncy.reserve(g.xadj[g.n]);
    c.adjwgt.reserve(g.xadj[g.n]);
    for (int cu = 0; cu < nc; ++cu) {
        targets.clear();
        for (int i = start[cu]; i < start[cu + 1]; ++i) {
            const int v = mem[i];
            for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
                int t = cmap[g.adjncy[e]];
                if (t == cu) continue;
                if (!hit[t]) { hit[t] = 1; targets.push_back(t); }
                acc[t] += (uint32_t)g.adjwgt[e];
            }
        }
        if (targets.size() <= 24) {
            for (size_t i = 1; i < targets.size(); ++i) {
                const int x = targets[i];
                size_t j = i;
                for (; j > 0 && targets[j - 1] > x; --j) targets[j] = targets[j - 1];
                targets[j] = x;
            }
        } else {
            std::sort(targets.begin(), targets.end());
        }
        for (int t : targets) {
            c.adjncy.push_back(t);
            c.adjwgt.push_back((int)acc[t]);
            acc[t] = 0;
            hit[t] = 0;
        }
        c.xadj[cu + 1] = (int)c.adjncy.size();
    }
    return c;
}

struct Bisector {
    const Knobs& kn;

    // tries on the coarsest graph of one bisection
    std::vector<char> coarsest(const HostGraph& g, uint64_t t0, const Limits& lim, int bis_key, bool par) const {
        struct Try {
            std::vector<char> side;
            uint64_t ov = 0;
            long long cut = 0;
        };
        std::vector<Try> tries((size_t)std::max(kn.ip_tries, 0));
        for_each_index(kn.ip_tries, par && g.n > 32, [&](int t) {
            const uint64_t ks = stream_key(kn.seed, TAG_IP, bis_key, t);
            int s0 = 0;
            uint32_t hmin = UINT32_MAX;
            for (int v = 0; v < g.n; ++v) {
                uint32_t h = hash32(ks, (uint32_t)v);
                if (h < hmin) { hmin = h; s0 = v; }
            }
            std::vector<long long> key(g.n, 0);
            GainHeap heap(g.n);
            Try& r = tries[t];
            int start = farthest(g, farthest(g, s0));
            grow_region(g, start, t0, lim.maxw[0], r.side, key, heap);
            r.cut = fm_refine(g, r.side, lim, kn.ip_fm_passes, kn.ip_fm_stall, key, heap);
            uint64_t w[2] = {0, 0};
            for (int v = 0; v < g.n; ++v) w[(int)r.side[v]] += (uint64_t)g.vwgt[v];
            r.ov = lim.overload(w);
        });
        // the first try of the smallest (overload, cut)
        int b = -1;
        for (int t = 0; t < kn.ip_tries; ++t)
            if (b < 0 || tries[t].ov < tries[b].ov || (tries[t].ov == tries[b].ov && tries[t].cut < tries[b].cut))
                b = t;
        return b < 0 ? std::vector<char>(g.n, 1) : std::move(tries[b].side);
    }

    std::vector<char> multilevel(const HostGraph& g, uint64_t t0, const Limits& lim, int bis_key, bool par) const {
        std::vector<HostGraph> levels;
        std::vector<std::vector<int>> maps;
        const uint64_t maxnode = (uint64_t)(1.5 * (double)g.weight() / 200.0);
        const HostGraph* cur = &g;
        while ((int)levels.size() < 32 && cur->n > 200) {
            std::vector<int> lab =
                heavy_edge_labels(*cur, stream_key(kn.seed, TAG_IPM, bis_key, (int)levels.size()), maxnode);
            std::vector<int> cmap;
            HostGraph c = contract_host(*cur, lab, cmap);
            if (1.0 * cur->n / (double)c.n < 1.1) break;
            maps.push_back(std::move(cmap));
            levels.push_back(std::move(c));
            cur = &levels.back();
        }
        std::vector<char> side = coarsest(*cur, t0, lim, bis_key, par);
        for (int l = (int)levels.size() - 1; l >= 0; --l) {
            const HostGraph& fine = l == 0 ? g : levels[l - 1];
            std::vector<char> fs(fine.n);
            for (int v = 0; v < fine.n; ++v) fs[v] = side[maps[l][v]];
            side.swap(fs);
            std::vector<long long> key(fine.n, 0);
            GainHeap heap(fine.n);
            fm_refine(fine, side, lim, kn.ip_fm_passes, kn.ip_fm_stall, key, heap);
        }
        return side;
    }
};

HostGraph induced(const HostGraph& g, const std::vector<int>& orig, const std::vector<char>& side, int which,
                  std::vector<int>& sub_orig) {
    std::vector<int> nid(g.n, -1);
    HostGraph s;
    sub_orig.clear();
    for (int v = 0; v < g.n; ++v)
        if (side[v] == which) {
            nid[v] = s.n++;
            sub_orig.push_back(orig[v]);
        }
    s.xadj.assign(s.n + 1, 0);
    s.vwgt.resize(s.n);
    for (int v = 0; v < g.n; ++v) {
        if (side[v] != which) continue;
        int u = nid[v];
        s.vwgt[u] = g.vwgt[v];
        for (int e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
            int t = g.adjncy[e];
            if (side[t] != which) continue;
            s.adjncy.push_back(nid[t]);
            s.adjwgt.push_back(g.adjwgt[e]);
        }
        s.xadj[u + 1] = (int)s.adjncy.size();
    }
    return s;
}

int levels_needed(int k) {
    int l = 0;
    while ((1 << l) < k) ++l;
    return l;
}

// Recursion over the bisection tree.  A bisection's hash streams depend only
// on its position in the tree (root 1, children 2i and 2i+1) and the
// repetition, so the two halves are independent and run as pool tasks when
// par is set, with results identical to a sequential recursion.
void recurse(const Knobs& kn, const HostGraph& g, const std::vector<int>& orig, int k, int offset, int rep,
             uint32_t node, std::vector<int>& out, bool par) {
    if (k == 1 || g.n == 0) {
        for (int v = 0; v < g.n; ++v) out[orig[v]] = offset;
        return;
    }
    const int kl = (k + 1) / 2, kr = k - kl;
    const uint64_t W = (uint64_t)g.weight();
    const uint64_t t0 = W * (uint64_t)kl / (uint64_t)k;
    const uint64_t t1 = W - t0;
    const double eps = kn.imbalance > 0 ? kn.imbalance : 0.0;
    double eb = std::pow(1.0 + eps, 1.0 / levels_needed(k)) - 1.0;
    eb = std::max(eb, std::min(eps, 0.01));
    Limits lim{{(uint64_t)((1.0 + eb) * (double)t0), (uint64_t)((1.0 + eb) * (double)t1)}};
    Bisector bis{kn};
    std::vector<char> side = bis.multilevel(g, t0, lim, (int)(node * 64u + (uint32_t)rep), par);
    std::vector<int> lo, ro;
    HostGraph L, R;
    for_each_index(2, par && g.n > 1024, [&](int h) {
        if (h == 0) L = induced(g, orig, side, 0, lo);
        else R = induced(g, orig, side, 1, ro);
    });
    side.clear();
    side.shrink_to_fit();
    // out[] entries written by the two halves are disjoint
    const bool fork = par && kl > 1 && kr > 1 && L.n > 64 && R.n > 64;
    for_each_index(2, fork, [&](int h) {
        if (h == 0) recurse(kn, L, lo, kl, offset, rep, 2u * node, out, par);
        else recurse(kn, R, ro, kr, offset + kl, rep, 2u * node + 1u, out, par);
    });
}

thread_local int t_spawn_limit = -1;

}  // namespace

void set_ip_thread_limit(int depth) { t_spawn_limit = depth; }

void initial_partition(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                       const Knobs& knobs, int* part) {
    // a dense coarsest graph (average degree > 64: skewed-degree inputs whose
    // coarsening stalls) gets one growing try and one FM pass per bisection;
    // its cut hardly depends on them and the FM's cost grows with the degree
    Knobs kn = knobs;
    if ((long long)xadj[n] > 64LL * n) {
        kn.ip_tries = std::min(kn.ip_tries, 1);
        kn.ip_fm_passes = std::min(kn.ip_fm_passes, 1);
    }
    HostGraph g;
    g.n = n;
    g.xadj.assign(xadj, xadj + n + 1);
    g.adjncy.assign(adjncy, adjncy + xadj[n]);
    g.adjwgt.assign(adjwgt, adjwgt + xadj[n]);
    g.vwgt.assign(vwgt, vwgt + n);
    std::vector<int> orig(n);
    for (int v = 0; v < n; ++v) orig[v] = v;
    const bool par = t_spawn_limit != 0 && std::thread::hardware_concurrency() > 1;
    const int reps = std::max(kn.ip_reps, 0);
    std::vector<std::vector<int>> cand((size_t)reps);
    std::vector<long long> cut((size_t)reps, 0);
    for_each_index(reps, par, [&](int rep) {
        cand[rep].assign(n, 0);
        recurse(kn, g, orig, kn.k, 0, rep, 1u, cand[rep], par);
        const std::vector<int>& c = cand[rep];
        long long x = 0;
        for (int v = 0; v < n; ++v)
            for (int e = xadj[v]; e < xadj[v + 1]; ++e)
                if (c[v] != c[adjncy[e]]) x += adjwgt[e];
        cut[rep] = x / 2;
    });
    // the first repetition of the smallest cut
    int b = -1;
    for (int rep = 0; rep < reps; ++rep)
        if (b < 0 || cut[rep] < cut[b]) b = rep;
    if (b >= 0) std::copy(cand[b].begin(), cand[b].end(), part);
}

}  // namespace kb
