// graph_io.cpp -- graph and partition files on the host (the formats of
// lib/io/graph_io.cpp:82-191 and parallel_graph_io.cpp:474-594), read in
// parallel: the file is mapped, split at line starts into one chunk per
// thread, each thread counts its vertex lines and entries, prefix sums give
// every chunk its first vertex and entry, and a second pass parses the
// numbers straight into the CSR arrays.
//
// METIS text: first non-comment line "n m [fmt]" (m undirected edges;
// fmt 1 = edge weights, 10 = node weights, 11 = both); then one line per
// vertex: [node weight] targets (1-based) [edge weight after each target];
// lines starting with '%' are comments.  Binary (.bgf): uint64 words
// version (3), n, m (directed entries), n + 1 byte offsets of the rows, then
// m uint64 targets (0-based); unit weights.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "graph_io.h"

namespace kb {

namespace {

struct Mapped {
    const char* p = nullptr;
    size_t size = 0;
    int fd = -1;
    ~Mapped() {
        if (p && size) munmap(const_cast<char*>(p), size);
        if (fd >= 0) close(fd);
    }
    bool open_file(const char* path) {
        fd = ::open(path, O_RDONLY);
        if (fd < 0) return false;
        struct stat st;
        if (fstat(fd, &st) != 0) return false;
        size = (size_t)st.st_size;
        if (size == 0) return true;
        void* m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (m == MAP_FAILED) { size = 0; return false; }
        p = static_cast<const char*>(m);
        return true;
    }
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Parses an unsigned decimal at s (after blanks); returns false at end of line.
inline bool next_uint(const char*& s, const char* end, unsigned long long& out) {
    while (s < end && is_space(*s)) ++s;
    if (s >= end || *s == '\n') return false;
    if (*s < '0' || *s > '9') {
        out = ~0ull;  // not a number: reported by the caller
        ++s;
        return true;
    }
    unsigned long long v = 0;
    while (s < end && *s >= '0' && *s <= '9') v = v * 10 + (unsigned long long)(*s++ - '0');
    out = v;
    return true;
}

int threads_for(size_t bytes) {
    unsigned hc = std::thread::hardware_concurrency();
    size_t t = std::max<size_t>(1, std::min<size_t>(hc ? hc : 4, bytes / (1 << 20) + 1));
    return (int)std::min<size_t>(t, 64);
}

}  // namespace

int read_metis(const char* path, HostCSR& g, std::string& err) {
    Mapped f;
    if (!f.open_file(path)) { err = std::string("cannot open ") + path; return -1; }
    const char* b = f.p;
    const char* e = f.p + f.size;
    // header: first line that is not a comment
    const char* s = b;
    while (s < e && *s == '%') {
        while (s < e && *s != '\n') ++s;
        if (s < e) ++s;
    }
    unsigned long long hn = 0, hm = 0, fmt = 0;
    const char* h = s;
    if (!next_uint(h, e, hn) || !next_uint(h, e, hm)) { err = "bad header line"; return -1; }
    if (!next_uint(h, e, fmt)) fmt = 0;
    if (hn > 0x7fffffffull || 2 * hm > 0x7fffffffull) { err = "graph too large for 32-bit CSR"; return -1; }
    const bool ew = fmt == 1 || fmt == 11, nw = fmt == 10 || fmt == 11;
    if (fmt != 0 && fmt != 1 && fmt != 10 && fmt != 11) { err = "unsupported format flag"; return -1; }
    while (h < e && *h != '\n') ++h;
    const char* body = h < e ? h + 1 : e;
    // chunks starting at line starts
    const int T = threads_for((size_t)(e - body));
    std::vector<const char*> cs(T + 1);
    cs[0] = body;
    cs[T] = e;
    for (int t = 1; t < T; ++t) {
        const char* q = body + (size_t)(e - body) * t / T;
        if (q < cs[t - 1]) q = cs[t - 1];
        while (q < e && q > body && q[-1] != '\n') ++q;
        cs[t] = q;
    }
    // pass 1: vertex lines and numbers per chunk
    std::vector<long long> lines(T, 0), nums(T, 0);
    auto count = [&](int t) {
        long long ln = 0, nu = 0;
        const char* q = cs[t];
        while (q < cs[t + 1]) {
            if (*q == '%') {
                while (q < cs[t + 1] && *q != '\n') ++q;
                if (q < cs[t + 1]) ++q;
                continue;
            }
            ++ln;
            unsigned long long x;
            while (next_uint(q, cs[t + 1], x)) ++nu;
            if (q < cs[t + 1]) ++q;  // the newline
        }
        lines[t] = ln;
        nums[t] = nu;
    };
    {
        std::vector<std::thread> th;
        for (int t = 1; t < T; ++t) th.emplace_back(count, t);
        count(0);
        for (auto& x : th) x.join();
    }
    long long L = 0, NU = 0;
    for (int t = 0; t < T; ++t) { L += lines[t]; NU += nums[t]; }
    if (L < (long long)hn) { err = "number of specified nodes mismatch"; return -1; }
    const long long per_edge = ew ? 2 : 1;
    const long long entries = (NU - (nw ? (long long)hn : 0)) / per_edge;
    if (entries != 2 * (long long)hm || (NU - (nw ? (long long)hn : 0)) % per_edge) {
        err = "number of specified edges mismatch";
        return -1;
    }
    g.n = (int)hn;
    g.m = entries;
    g.xadj.assign((size_t)hn + 1, 0);
    g.adjncy.assign((size_t)entries, 0);
    g.adjwgt.assign((size_t)entries, 1);
    g.vwgt.assign((size_t)hn, 1);
    // pass 2: vertex offsets from the line counts, entry offsets from the numbers
    std::vector<long long> v0(T + 1, 0), e0(T + 1, 0);
    for (int t = 0; t < T; ++t) {
        v0[t + 1] = v0[t] + lines[t];
        const long long own = nums[t] - (nw ? lines[t] : 0);
        e0[t + 1] = e0[t] + own / per_edge;
    }
    std::vector<int> bad(T, 0);
    auto fill = [&](int t) {
        long long v = v0[t], p = e0[t];
        const char* q = cs[t];
        while (q < cs[t + 1] && v < (long long)hn) {
            if (*q == '%') {
                while (q < cs[t + 1] && *q != '\n') ++q;
                if (q < cs[t + 1]) ++q;
                continue;
            }
            g.xadj[(size_t)v] = (int)p;
            unsigned long long x;
            if (nw) {
                if (!next_uint(q, cs[t + 1], x) || x > 0x7fffffffull) { bad[t] = 1; return; }
                g.vwgt[(size_t)v] = (int)x;
            }
            while (next_uint(q, cs[t + 1], x)) {
                if (x == 0 || x > hn || x == ~0ull) { bad[t] = 2; return; }
                if ((long long)x - 1 == v) { bad[t] = 3; return; }
                if (p >= entries) { bad[t] = 4; return; }
                g.adjncy[(size_t)p] = (int)(x - 1);
                if (ew) {
                    if (!next_uint(q, cs[t + 1], x) || x > 0x7fffffffull) { bad[t] = 1; return; }
                    g.adjwgt[(size_t)p] = (int)x;
                }
                ++p;
            }
            if (q < cs[t + 1]) ++q;
            ++v;
        }
    };
    {
        std::vector<std::thread> th;
        for (int t = 1; t < T; ++t) th.emplace_back(fill, t);
        fill(0);
        for (auto& x : th) x.join();
    }
    for (int t = 0; t < T; ++t) {
        if (bad[t] == 1) { err = "bad weight"; return -1; }
        if (bad[t] == 2) { err = "target out of range"; return -1; }
        if (bad[t] == 3) { err = "the graph file contains self-loops"; return -1; }
        if (bad[t] == 4) { err = "malformed line"; return -1; }
    }
    g.xadj[(size_t)hn] = (int)entries;
    return 0;
}

int read_bgf(const char* path, HostCSR& g, std::string& err) {
    Mapped f;
    if (!f.open_file(path)) { err = std::string("cannot open ") + path; return -1; }
    if (f.size < 24) { err = "file too short"; return -1; }
    const uint64_t* w = reinterpret_cast<const uint64_t*>(f.p);
    const uint64_t version = w[0], n = w[1], m = w[2];
    if (version != 3) { err = "unsupported binary graph version"; return -1; }
    if (n > 0x7fffffffull || m > 0x7fffffffull) { err = "graph too large for 32-bit CSR"; return -1; }
    const uint64_t need = (3 + n + 1 + m) * 8;
    if (f.size < need) { err = "file too short"; return -1; }
    const uint64_t base = (3 + n + 1) * 8;
    g.n = (int)n;
    g.m = (long long)m;
    g.xadj.assign((size_t)n + 1, 0);
    g.adjncy.assign((size_t)m, 0);
    g.adjwgt.assign((size_t)m, 1);
    g.vwgt.assign((size_t)n, 1);
    const uint64_t* off = w + 3;
    for (uint64_t v = 0; v <= n; ++v) {
        const uint64_t o = off[v];
        if (o < base || (o - base) % 8 || (o - base) / 8 > m || (v > 0 && o < off[v - 1])) {
            err = "bad row offset";
            return -1;
        }
        g.xadj[(size_t)v] = (int)((o - base) / 8);
    }
    if (g.xadj[(size_t)n] != (int)m) { err = "row offsets do not cover the edges"; return -1; }
    const uint64_t* tg = w + 3 + n + 1;
    for (uint64_t i = 0; i < m; ++i) {
        if (tg[i] >= n) { err = "target out of range"; return -1; }
        g.adjncy[(size_t)i] = (int)tg[i];
    }
    return 0;
}

int write_partition(const char* path, int n, const int* part, std::string& err) {
    FILE* fp = std::fopen(path, "wb");
    if (!fp) { err = std::string("cannot create ") + path; return -1; }
    std::vector<char> buf;
    buf.reserve(1 << 20);
    char tmp[16];
    for (int v = 0; v < n; ++v) {
        int x = part[v], len = 0;
        if (x < 0) { err = "negative block id"; std::fclose(fp); return -1; }
        do { tmp[len++] = (char)('0' + x % 10); x /= 10; } while (x);
        while (len) buf.push_back(tmp[--len]);
        buf.push_back('\n');
        if (buf.size() > (1 << 20) - 16) {
            if (std::fwrite(buf.data(), 1, buf.size(), fp) != buf.size()) { err = "write failed"; std::fclose(fp); return -1; }
            buf.clear();
        }
    }
    if (!buf.empty() && std::fwrite(buf.data(), 1, buf.size(), fp) != buf.size()) {
        err = "write failed";
        std::fclose(fp);
        return -1;
    }
    if (std::fclose(fp) != 0) { err = "write failed"; return -1; }
    return 0;
}

}  // namespace kb

// ------------------------------------------------------------------ C ABI

namespace {
thread_local std::string g_io_error;

int export_csr(kb::HostCSR& g, int* n, long long* m, int** xadj, int** adjncy, int** adjwgt, int** vwgt) {
    auto dup = [](const std::vector<int>& v) {
        int* p = static_cast<int*>(std::malloc(sizeof(int) * std::max<size_t>(v.size(), 1)));
        if (p && !v.empty()) std::memcpy(p, v.data(), sizeof(int) * v.size());
        return p;
    };
    int* a = dup(g.xadj);
    int* b = dup(g.adjncy);
    int* c = dup(g.adjwgt);
    int* d = dup(g.vwgt);
    if (!a || !b || !c || !d) {
        std::free(a); std::free(b); std::free(c); std::free(d);
        g_io_error = "host allocation failed";
        return -4;
    }
    *n = g.n;
    *m = g.m;
    *xadj = a;
    *adjncy = b;
    *adjwgt = c;
    *vwgt = d;
    return 0;
}
}  // namespace

extern "C" {

__attribute__((visibility("default"))) int kb200_read_metis(const char* path, int* n, long long* m, int** xadj,
                                                            int** adjncy, int** adjwgt, int** vwgt) {
    if (!path || !n || !m || !xadj || !adjncy || !adjwgt || !vwgt) { g_io_error = "NULL argument"; return -1; }
    kb::HostCSR g;
    std::string err;
    if (kb::read_metis(path, g, err)) { g_io_error = err; return -1; }
    return export_csr(g, n, m, xadj, adjncy, adjwgt, vwgt);
}

__attribute__((visibility("default"))) int kb200_read_bgf(const char* path, int* n, long long* m, int** xadj,
                                                          int** adjncy, int** adjwgt, int** vwgt) {
    if (!path || !n || !m || !xadj || !adjncy || !adjwgt || !vwgt) { g_io_error = "NULL argument"; return -1; }
    kb::HostCSR g;
    std::string err;
    if (kb::read_bgf(path, g, err)) { g_io_error = err; return -1; }
    return export_csr(g, n, m, xadj, adjncy, adjwgt, vwgt);
}

__attribute__((visibility("default"))) int kb200_write_partition(const char* path, int n, const int* part) {
    if (!path || n < 0 || (n > 0 && !part)) { g_io_error = "invalid arguments"; return -1; }
    std::string err;
    if (kb::write_partition(path, n, part, err)) { g_io_error = err; return -1; }
    return 0;
}

__attribute__((visibility("default"))) void kb200_free(void* p) { std::free(p); }

__attribute__((visibility("default"))) const char* kb200_io_error(void) { return g_io_error.c_str(); }

}  // extern "C"
