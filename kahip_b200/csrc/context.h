// context.h -- per-call GPU context: device, stream, device-memory arena,
// pinned staging buffers and per-phase event timers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace kb {

// Bump allocator over one device allocation.  Allocations are 256-byte
// aligned; mark()/release() give stack discipline for per-phase scratch.
class Arena {
public:
    Arena() = default;
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;
    ~Arena() { free_all(); }

    // Ensures capacity >= bytes; drops all current allocations.
    void reserve(size_t bytes) {
        if (bytes <= cap_) { top_ = 0; return; }
        free_all();
        cudaError_t e = cudaMalloc(&base_, bytes);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            base_ = nullptr;
            throw CudaError(e, "device arena allocation failed");
        }
        cap_ = bytes;
        top_ = 0;
    }
    void free_all() {
        if (base_) cudaFree(base_);
        base_ = nullptr;
        cap_ = top_ = 0;
    }
    template <class T>
    T* alloc(size_t count) {
        size_t bytes = ((count * sizeof(T)) + 255) & ~(size_t)255;
        if (bytes == 0) bytes = 256;
        if (top_ + bytes > cap_) throw CudaError(cudaErrorMemoryAllocation, "device arena exhausted");
        T* p = reinterpret_cast<T*>(base_ + top_);
        top_ += bytes;
        if (top_ > peak_) peak_ = top_;
        return p;
    }
    size_t mark() const { return top_; }
    void release(size_t m) { top_ = m; }
    size_t capacity() const { return cap_; }
    size_t peak() const { return peak_; }

private:
    char* base_ = nullptr;
    size_t cap_ = 0, top_ = 0, peak_ = 0;
};

// Accumulated device time and algorithmic bytes per kernel family.
struct PhaseTimer {
    std::string name;
    double ms = 0;
    double bytes = 0;
    long long launches = 0;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t copy_stream = nullptr;  // host <-> device copies beside the work (created on first use)
    cudaStream_t copies();
    Arena hier;     // graph hierarchy (lives for the whole call)
    Arena scratch;  // per-phase scratch (mark/release)
    // small device scalars (counters, flags) and their pinned host mirror
    int* dscalars = nullptr;               // 64 ints
    unsigned long long* work = nullptr;    // [0] swept vertices, [1] swept edges
    uint32_t* pinned = nullptr;            // 64 words, page-locked
    // timing: 0 off, 1 every kernel family, 2 only the LP clustering sweep
    int timing = 0;
    std::vector<PhaseTimer> phases;
    struct Pending { int phase; cudaEvent_t a, b; double bytes; };
    std::vector<cudaEvent_t> ev_free;
    std::vector<Pending> pending;
    // trace: with KB200_TRACE=<file> set, every timed span is appended to the
    // file as "family start_ms end_ms" relative to the call's first event
    const char* trace_path = nullptr;
    cudaEvent_t origin = nullptr;

    ~Ctx();
    void init(int dev, cudaStream_t s);
    int phase_id(const char* name);
    cudaEvent_t ev();
    void begin(int phase, cudaEvent_t& a);
    void end(int phase, cudaEvent_t a, double bytes);
    void collect();  // resolves pending events (after a stream sync)
    void reset_stats();
};

// RAII bracket: KB_PHASE(ctx, "lp_sweep", bytes) around launches.
struct PhaseScope {
    Ctx& c;
    int id;
    cudaEvent_t a = nullptr;
    double bytes;
    PhaseScope(Ctx& c_, const char* name, double b) : c(c_), id(-1), bytes(b) {
        if (c.timing == 1 || (c.timing == 2 && std::strcmp(name, "lp_cluster_sweep") == 0)) {
            id = c.phase_id(name);
            c.begin(id, a);
        }
    }
    ~PhaseScope() {
        if (id >= 0) c.end(id, a, bytes);
    }
};

}  // namespace kb
