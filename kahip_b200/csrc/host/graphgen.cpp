// graphgen.cpp -- seeded synthetic graph generators (int32 METIS-style CSR).
//
// These produce the workloads the partitioner is measured and tested on:
//   * 2D / 3D random geometric graphs (points uniform in the unit square /
//     cube, edge iff Euclidean distance < r), node ids in grid-cell order so
//     that ids are spatially sorted, every row sorted by target;
//   * R-MAT graphs (recursive quadrant sampling with probabilities a,b,c,d),
//     symmetrised, self loops dropped, duplicate multiplicity folded into the
//     edge weight;
//   * 2D grids with the 5-point stencil.
// All randomness is counter based (splitmix64 finaliser over (seed, index)),
// so the output is a pure function of the arguments and independent of the
// number of host threads used.
//
// C ABI: a generator returns an opaque kbgen_graph*; the caller reads n and m,
// copies the arrays out, and frees the handle.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z) {
    // splitmix64 output function (Steele, Lea, Flood 2014; Vigna's constants)
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline double unit(uint64_t key) {  // uniform in [0,1) with 53 random bits
    return (double)(mix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

int num_threads() {
    unsigned t = std::thread::hardware_concurrency();
    if (const char* s = std::getenv("KBGEN_THREADS")) t = (unsigned)std::atoi(s);
    return t == 0 ? 1 : (int)std::min(t, 64u);
}

template <class F>
void parallel_for(int64_t n, F f) {
    int T = num_threads();
    if (n < 4096 || T == 1) { f(0, n, 0); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
        int64_t lo = n * t / T, hi = n * (t + 1) / T;
        th.emplace_back([=] { f(lo, hi, t); });
    }
    for (auto& x : th) x.join();
}

}  // namespace

struct kbgen_graph {
    int64_t n = 0, m = 0;
    std::vector<int32_t> xadj, adjncy, adjwgt, vwgt;  // adjwgt/vwgt empty = unit
    std::vector<double> coords;                       // dim * n, optional
    int dim = 0;
};

namespace {

// Random geometric graph in `dim` dimensions (2 or 3).
kbgen_graph* rgg(int64_t n, int dim, double radius, uint64_t seed) {
    auto* g = new kbgen_graph();
    g->n = n;
    g->dim = dim;
    const uint64_t base = mix64(seed ^ (0x52474700ull + (uint64_t)dim));
    std::vector<double> pts((size_t)(n * dim));
    parallel_for(n, [&](int64_t lo, int64_t hi, int) {
        for (int64_t i = lo; i < hi; ++i)
            for (int d = 0; d < dim; ++d) pts[(size_t)(i * dim + d)] = unit(base + (uint64_t)(i * dim + d));
    });
    int64_t cells1 = std::max<int64_t>(1, (int64_t)std::floor(1.0 / radius));
    int64_t ncell = 1;
    for (int d = 0; d < dim; ++d) ncell *= cells1;
    auto cell_of = [&](const double* p) {
        int64_t c = 0;
        for (int d = dim - 1; d >= 0; --d) {
            int64_t x = std::min<int64_t>(cells1 - 1, (int64_t)(p[d] * (double)cells1));
            c = c * cells1 + x;
        }
        return c;  // x fastest
    };
    // counting sort of points by cell, stable in the original index
    std::vector<int64_t> cell((size_t)n);
    parallel_for(n, [&](int64_t lo, int64_t hi, int) {
        for (int64_t i = lo; i < hi; ++i) cell[(size_t)i] = cell_of(&pts[(size_t)(i * dim)]);
    });
    std::vector<int64_t> cstart((size_t)ncell + 1, 0);
    for (int64_t i = 0; i < n; ++i) cstart[(size_t)cell[(size_t)i] + 1]++;
    for (int64_t c = 0; c < ncell; ++c) cstart[(size_t)c + 1] += cstart[(size_t)c];
    std::vector<double> sp((size_t)(n * dim));
    {
        std::vector<int64_t> fill(cstart.begin(), cstart.end() - 1);
        for (int64_t i = 0; i < n; ++i) {
            int64_t pos = fill[(size_t)cell[(size_t)i]]++;
            for (int d = 0; d < dim; ++d) sp[(size_t)(pos * dim + d)] = pts[(size_t)(i * dim + d)];
        }
    }
    pts.clear(); pts.shrink_to_fit();
    cell.clear(); cell.shrink_to_fit();
    const double r2 = radius * radius;
    // For node p, visit neighbouring cells in increasing cell index; since node
    // ids follow cell order, every row comes out sorted by target.
    auto visit = [&](int64_t p, auto&& emit) {
        const double* P = &sp[(size_t)(p * dim)];
        int64_t cx[3];
        for (int d = 0; d < dim; ++d) cx[d] = std::min<int64_t>(cells1 - 1, (int64_t)(P[d] * (double)cells1));
        int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) { lo[d] = cx[d] > 0 ? -1 : 0; hi[d] = cx[d] < cells1 - 1 ? 1 : 0; }
        for (int dz = (dim == 3 ? lo[2] : 0); dz <= (dim == 3 ? hi[2] : 0); ++dz)
            for (int dy = lo[1]; dy <= hi[1]; ++dy)
                for (int dx = lo[0]; dx <= hi[0]; ++dx) {
                    int64_t c = cx[0] + dx + cells1 * (cx[1] + dy + (dim == 3 ? cells1 * (cx[2] + dz) : 0));
                    for (int64_t q = cstart[(size_t)c]; q < cstart[(size_t)c + 1]; ++q) {
                        if (q == p) continue;
                        const double* Q = &sp[(size_t)(q * dim)];
                        double s = 0;
                        for (int d = 0; d < dim; ++d) { double t = P[d] - Q[d]; s += t * t; }
                        if (s < r2) emit(q);
                    }
                }
    };
    std::vector<int64_t> deg((size_t)n + 1, 0);
    parallel_for(n, [&](int64_t lo, int64_t hi, int) {
        for (int64_t p = lo; p < hi; ++p) {
            int64_t c = 0;
            visit(p, [&](int64_t) { ++c; });
            deg[(size_t)p + 1] = c;
        }
    });
    for (int64_t p = 0; p < n; ++p) deg[(size_t)p + 1] += deg[(size_t)p];
    g->m = deg[(size_t)n];
    if (g->m > INT32_MAX) { delete g; return nullptr; }
    g->xadj.resize((size_t)n + 1);
    for (int64_t p = 0; p <= n; ++p) g->xadj[(size_t)p] = (int32_t)deg[(size_t)p];
    g->adjncy.resize((size_t)g->m);
    parallel_for(n, [&](int64_t lo, int64_t hi, int) {
        for (int64_t p = lo; p < hi; ++p) {
            int64_t pos = deg[(size_t)p];
            visit(p, [&](int64_t q) { g->adjncy[(size_t)pos++] = (int32_t)q; });
        }
    });
    g->coords = std::move(sp);
    return g;
}

// LSD radix sort of 64-bit keys (used by the R-MAT builder).
void radix_sort_u64(std::vector<uint64_t>& a, int bits) {
    std::vector<uint64_t> tmp(a.size());
    for (int shift = 0; shift < bits; shift += 16) {
        const int T = num_threads();
        const int64_t N = (int64_t)a.size();
        std::vector<std::vector<int64_t>> cnt(T, std::vector<int64_t>(65536, 0));
        parallel_for(N, [&](int64_t lo, int64_t hi, int t) {
            auto& c = cnt[(size_t)t];
            for (int64_t i = lo; i < hi; ++i) c[(a[(size_t)i] >> shift) & 0xFFFF]++;
        });
        // exclusive offsets per (digit, thread) in digit-major, thread-minor order
        int64_t run = 0;
        for (int d = 0; d < 65536; ++d)
            for (int t = 0; t < T; ++t) { int64_t x = cnt[(size_t)t][(size_t)d]; cnt[(size_t)t][(size_t)d] = run; run += x; }
        parallel_for(N, [&](int64_t lo, int64_t hi, int t) {
            auto& c = cnt[(size_t)t];
            for (int64_t i = lo; i < hi; ++i) tmp[(size_t)c[(a[(size_t)i] >> shift) & 0xFFFF]++] = a[(size_t)i];
        });
        a.swap(tmp);
    }
}

kbgen_graph* rmat(int scale, int64_t samples, double a, double b, double c, uint64_t seed) {
    auto* g = new kbgen_graph();
    const int64_t n = (int64_t)1 << scale;
    g->n = n;
    const uint64_t base = mix64(seed ^ 0x524D4154ull);
    const double ab = a + b, abc = a + b + c;
    std::vector<uint64_t> keys((size_t)samples);
    std::atomic<int64_t> dropped{0};
    parallel_for(samples, [&](int64_t lo, int64_t hi, int) {
        int64_t drop = 0;
        for (int64_t s = lo; s < hi; ++s) {
            uint64_t u = 0, v = 0;
            for (int l = 0; l < scale; ++l) {
                double x = unit(base + (uint64_t)s * 64u + (uint64_t)l);
                int q = x < a ? 0 : x < ab ? 1 : x < abc ? 2 : 3;
                u = (u << 1) | (uint64_t)(q >> 1);
                v = (v << 1) | (uint64_t)(q & 1);
            }
            if (u == v) { keys[(size_t)s] = ~0ull; ++drop; continue; }
            uint64_t lo_ = std::min(u, v), hi_ = std::max(u, v);
            keys[(size_t)s] = (lo_ << 32) | hi_;
        }
        dropped += drop;
    });
    radix_sort_u64(keys, 64);
    keys.resize((size_t)(samples - dropped.load()));
    // unique undirected edges with multiplicity
    std::vector<uint64_t> uk;
    std::vector<int32_t> mult;
    uk.reserve(keys.size());
    mult.reserve(keys.size());
    for (size_t i = 0; i < keys.size();) {
        size_t j = i;
        while (j < keys.size() && keys[j] == keys[i]) ++j;
        uk.push_back(keys[i]);
        mult.push_back((int32_t)(j - i));
        i = j;
    }
    keys.clear(); keys.shrink_to_fit();
    std::vector<int64_t> deg((size_t)n + 1, 0);
    for (uint64_t k : uk) { deg[(size_t)(k >> 32) + 1]++; deg[(size_t)(k & 0xFFFFFFFFu) + 1]++; }
    for (int64_t v = 0; v < n; ++v) deg[(size_t)v + 1] += deg[(size_t)v];
    g->m = deg[(size_t)n];
    if (g->m > INT32_MAX) { delete g; return nullptr; }
    g->xadj.assign(deg.begin(), deg.end());
    g->adjncy.resize((size_t)g->m);
    g->adjwgt.resize((size_t)g->m);
    std::vector<int64_t> fill(deg.begin(), deg.end() - 1);
    // uk is sorted by (lo, hi): appending (lo -> hi) in that order and
    // (hi -> lo) in that order keeps every row sorted only if we place both
    // directions by a second pass; do it with a per-row sort afterwards.
    for (size_t i = 0; i < uk.size(); ++i) {
        int64_t u = (int64_t)(uk[i] >> 32), v = (int64_t)(uk[i] & 0xFFFFFFFFu);
        g->adjncy[(size_t)fill[(size_t)u]] = (int32_t)v; g->adjwgt[(size_t)fill[(size_t)u]++] = mult[i];
        g->adjncy[(size_t)fill[(size_t)v]] = (int32_t)u; g->adjwgt[(size_t)fill[(size_t)v]++] = mult[i];
    }
    parallel_for(n, [&](int64_t lo, int64_t hi, int) {
        std::vector<std::pair<int32_t, int32_t>> row;
        for (int64_t v = lo; v < hi; ++v) {
            int64_t s = deg[(size_t)v], e = deg[(size_t)v + 1];
            row.clear();
            for (int64_t i = s; i < e; ++i) row.emplace_back(g->adjncy[(size_t)i], g->adjwgt[(size_t)i]);
            std::sort(row.begin(), row.end());
            for (int64_t i = s; i < e; ++i) { g->adjncy[(size_t)i] = row[(size_t)(i - s)].first; g->adjwgt[(size_t)i] = row[(size_t)(i - s)].second; }
        }
    });
    return g;
}

kbgen_graph* grid2d(int64_t nx, int64_t ny) {
    auto* g = new kbgen_graph();
    const int64_t n = nx * ny;
    g->n = n;
    g->xadj.resize((size_t)n + 1);
    g->xadj[0] = 0;
    for (int64_t y = 0; y < ny; ++y)
        for (int64_t x = 0; x < nx; ++x) {
            int64_t v = y * nx + x;
            int d = (x > 0) + (x < nx - 1) + (y > 0) + (y < ny - 1);
            g->xadj[(size_t)v + 1] = g->xadj[(size_t)v] + d;
        }
    g->m = g->xadj[(size_t)n];
    g->adjncy.resize((size_t)g->m);
    for (int64_t y = 0; y < ny; ++y)
        for (int64_t x = 0; x < nx; ++x) {
            int64_t v = y * nx + x;
            int64_t p = g->xadj[(size_t)v];
            if (y > 0) g->adjncy[(size_t)p++] = (int32_t)(v - nx);
            if (x > 0) g->adjncy[(size_t)p++] = (int32_t)(v - 1);
            if (x < nx - 1) g->adjncy[(size_t)p++] = (int32_t)(v + 1);
            if (y < ny - 1) g->adjncy[(size_t)p++] = (int32_t)(v + nx);
        }
    return g;
}

}  // namespace

extern "C" {

// 2D random geometric graph: n points, radius = r_factor * sqrt(ln n / n).
kbgen_graph* kbgen_rgg2d(long long n, double r_factor, unsigned long long seed) {
    if (n <= 0) return nullptr;
    double r = r_factor * std::sqrt(std::log((double)n) / (double)n);
    if (n == 1) r = 1.0;
    return rgg(n, 2, r, seed);
}

// 3D random geometric graph: radius = r_factor * cbrt(ln n / n).
kbgen_graph* kbgen_rgg3d(long long n, double r_factor, unsigned long long seed) {
    if (n <= 0) return nullptr;
    double r = r_factor * std::cbrt(std::log((double)n) / (double)n);
    if (n == 1) r = 1.0;
    return rgg(n, 3, r, seed);
}

// R-MAT with 2^scale nodes and `samples` edge samples.
kbgen_graph* kbgen_rmat(int scale, long long samples, double a, double b, double c,
                        unsigned long long seed) {
    if (scale <= 0 || scale > 30 || samples < 0) return nullptr;
    return rmat(scale, samples, a, b, c, seed);
}

kbgen_graph* kbgen_grid2d(long long nx, long long ny) {
    if (nx <= 0 || ny <= 0) return nullptr;
    return grid2d(nx, ny);
}

long long kbgen_n(const kbgen_graph* g) { return g ? g->n : -1; }
long long kbgen_m(const kbgen_graph* g) { return g ? g->m : -1; }
int kbgen_has_adjwgt(const kbgen_graph* g) { return g && !g->adjwgt.empty(); }

// Copies the CSR out; adjwgt may be NULL (or is filled with 1 when the graph
// is unweighted), vwgt may be NULL (filled with 1 otherwise).
void kbgen_copy(const kbgen_graph* g, int* xadj, int* adjncy, int* adjwgt, int* vwgt) {
    if (!g) return;
    if (xadj) std::memcpy(xadj, g->xadj.data(), sizeof(int32_t) * (size_t)(g->n + 1));
    if (adjncy) std::memcpy(adjncy, g->adjncy.data(), sizeof(int32_t) * (size_t)g->m);
    if (adjwgt) {
        if (g->adjwgt.empty()) std::fill(adjwgt, adjwgt + g->m, 1);
        else std::memcpy(adjwgt, g->adjwgt.data(), sizeof(int32_t) * (size_t)g->m);
    }
    if (vwgt) std::fill(vwgt, vwgt + g->n, 1);
}

void kbgen_free(kbgen_graph* g) { delete g; }

}  // extern "C"
