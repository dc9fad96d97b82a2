// hash.h -- the counter-based hash behind every tie-break, sub-round
// assignment and priority class (host and device).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define KB_HD __host__ __device__ __forceinline__
#else
#define KB_HD inline
#endif

namespace kb {

// Hash tags: one independent stream per decision kind.
enum HashTag : int {
    TAG_CSUB = 1,   // clustering sub-round membership
    TAG_CTIE = 2,   // clustering tie-break between clusters
    TAG_RSUB = 3,   // refinement sub-round membership
    TAG_RTIE = 4,   // refinement tie-break between blocks
    TAG_RPRIO = 5,  // refinement admission priority class
    TAG_BTIE = 6,   // balance: target tie-break
    TAG_BCLS = 7,   // balance: release class refinement
    TAG_BPRIO = 8,  // balance: admission priority class
    TAG_IP = 9,     // initial partitioning: start nodes
    TAG_IPM = 10,   // initial partitioning: matching order
    TAG_MATCH = 11, // heavy-edge matching: pair hash
    TAG_JTIE = 12,  // Jet refinement: destination tie-break
    TAG_EVO = 13,   // evolutionary partitioning: tournament draws
};

// splitmix64 output function (Steele, Lea & Flood, OOPSLA 2014).
KB_HD uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// A stream key per (seed, decision kind, level, round); computed on the host
// once and passed to kernels by value.
KB_HD uint64_t stream_key(int seed, int tag, int level, int round) {
    uint64_t s = mix64((uint64_t)(uint32_t)seed ^ ((uint64_t)(uint32_t)tag << 40));
    s = mix64(s ^ (uint64_t)(uint32_t)level);
    return mix64(s ^ (uint64_t)(uint32_t)round);
}

// Per-item hash: a murmur3-style 32-bit finaliser (MurmurHash3 fmix32,
// Appleby) keyed by both halves of the stream key.
KB_HD uint32_t hash32(uint64_t ks, uint32_t x) {
    uint32_t h = (x * 0x9E3779B1u) ^ (uint32_t)ks;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= (uint32_t)(ks >> 32) | 1u;
    h ^= h >> 16;
    return h;
}

// Maps a uniform 32-bit hash onto [0, n) (multiply-shift range reduction).
KB_HD uint32_t hash_range(uint32_t h, uint32_t n) {
    return (uint32_t)(((uint64_t)h * n) >> 32);
}

}  // namespace kb
