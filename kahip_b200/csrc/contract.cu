// contract.cu -- contraction of a clustering into the next coarser graph.
//
// Reference semantics: contraction.cpp:94-133 -> complete_boundary.h:511-562
// (clusters) and contraction.cpp:21-92 + contraction.h:60-82 (matchings):
// coarse node weight = sum of member weights; edges inside a coarse node are
// dropped; parallel coarse edges are merged with summed weights.  Coarse ids
// follow the order of each cluster's smallest member, which is the
// first-appearance order of remap_cluster_ids (size_constraint_label_
// propagation.cpp:207-232).  Rows come out sorted by target.
//
// Pipeline (all on the device):
//   1. leader[c] = min member (atomicMin); prefix sum over leader flags
//      gives coarse ids; cmap gather; coarse node weights (atomicAdd).
//   2. every coarse row gets a bucket as large as its members' degrees
//      together (prefix sum); every fine node merges its neighbours by
//      coarse target in register slots and appends (cv << 32 | w) entries
//      to its coarse row's bucket, one atomic reservation per slot flush
//      (long rows: the whole warp).
//   3. (no separate pass: the buckets are filled by the emission)
//   4. a warp per coarse row sorts its bucket in shared memory (bitonic),
//      sums the weights of equal targets and keeps the distinct entries;
//      rows longer than kSegMax go through a stable LSD radix sort on the
//      2*tb key bits and a reduce-by-key instead.
//   5. distinct counts -> prefix sum -> xadj; rows copied into place.
#include "contract.cuh"
#include "prims.cuh"

#include <climits>

namespace kb {

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kThreads = 256;

int grid_for(long long n, int threads) {
    return (int)std::max<long long>(1, std::min<long long>(div_up(n, threads), (long long)kNumSMs * 16));
}

// mm[c] = the smallest member of cluster c.  Lanes of a warp with the same
// label take one atomic: the lowest of them holds the group's smallest id.
__global__ void leader_min(int n, const int* __restrict__ label, int* mm) {
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(base + threadIdx.x);
        const bool ok = v < n;
        const int l = ok ? label[v] : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, l);
        if (ok && lane == __ffs(peers) - 1) atomicMin(&mm[l], v);
    }
}

__global__ void leader_flags(int n, const int* __restrict__ label, const int* __restrict__ mm,
                             uint32_t* flag) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        flag[v] = mm[label[v]] == v ? 1u : 0u;
}

// cmap, coarse node weights, each coarse row's bucket capacity (the degrees
// of its members) and, when msize is given, each coarse node's member count.
// Consecutive fine nodes often share a coarse node: the lanes of a warp with
// equal coarse ids add their shares together and one of them does the atomics.
__global__ void make_cmap(int n, const int* __restrict__ label, const int* __restrict__ mm,
                          const uint32_t* __restrict__ pos, const int* __restrict__ vwgt,
                          const int* __restrict__ xadj, int* cmap, uint32_t* cvw, uint32_t* rowcap,
                          uint32_t* msize) {
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(base + threadIdx.x);
        const bool ok = v < n;
        int c = -1;
        uint32_t w = 0, d = 0;
        if (ok) {
            c = (int)pos[mm[label[v]]];
            cmap[v] = c;
            w = (uint32_t)vwgt[v];
            d = (uint32_t)(xadj[v + 1] - xadj[v]);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const uint32_t sw = __reduce_add_sync(peers, w);
        const uint32_t sd = __reduce_add_sync(peers, d);
        if (ok && lane == __ffs(peers) - 1) {
            atomicAdd(&cvw[c], sw);
            if (sd) atomicAdd(&rowcap[c], sd);
            if (msize) atomicAdd(&msize[c], (uint32_t)__popc(peers));
        }
    }
}

// Member rows: the rows (xadj[v], degree) of the fine nodes bucketed by
// coarse id; mrow[mbeg[c] .. mbeg[c + 1]) are the rows of c's members, in
// no particular order.
__global__ void scatter_members(int n, const int* __restrict__ cmap, const int* __restrict__ xadj,
                                const uint32_t* __restrict__ mbeg, uint32_t* mfill, int2* mrow) {
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(base + threadIdx.x);
        const bool ok = v < n;
        const int c = ok ? cmap[v] : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const int leader = __ffs(peers) - 1;
        uint32_t at = 0;
        if (ok && lane == leader) at = atomicAdd(&mfill[c], (uint32_t)__popc(peers));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (ok) {
            const int b = xadj[v];
            mrow[mbeg[c] + at + __popc(peers & lanemask_lt())] = make_int2(b, xadj[v + 1] - b);
        }
    }
}

// ---- gather contraction: a warp per coarse node walks the rows of all its
// members back to back (32 entries per batch, kGatherWin batches loaded
// together), drops the entries inside the node, adds the others into the
// warp's shared-memory table (shared-memory atomics; a key is inserted by
// compare-and-swap once), then sorts the distinct targets and writes them to
// the node's bucket.  Nodes with more than kGatherMaxDistinct distinct targets, or more
// than kGatherMaxEntries member entries, are flagged (sel) for the emission
// path below.
constexpr int kGatherWarps = 8;
constexpr int kGatherTab = 256;                  // table slots per warp
constexpr int kGatherMaxDistinct = kGatherTab / 2;
constexpr int kGatherList = kGatherMaxDistinct + 32;  // a batch may add 32 past the limit
constexpr int kGatherSort = 256;                 // sort buffer (power of two >= kGatherList)
constexpr int kGatherWin = 4;
constexpr int kGatherBlocksPerSM = 6;
constexpr long long kGatherMaxEntries = 8192;

__device__ __forceinline__ uint32_t gather_slot(uint32_t key) {
    return (key * 0x9E3779B1u) >> 24;  // kGatherTab == 256
}

template <bool UNIT>
__global__ void __launch_bounds__(kGatherWarps * 32, kGatherBlocksPerSM) gather_rows(
    int nc, const uint32_t* __restrict__ mbeg, const int2* __restrict__ mrow, const int* __restrict__ adjncy,
    const int* __restrict__ adjwgt, const int* __restrict__ cmap, const uint32_t* __restrict__ rowoff,
    uint64_t* bucket, uint32_t* ucnt, uint8_t* sel, unsigned* nsel) {
    static_assert(kGatherTab == 256 && kGatherSort >= kGatherList, "table layout");
    __shared__ uint32_t tk[kGatherWarps][kGatherTab];
    __shared__ uint32_t tv[kGatherWarps][kGatherTab];
    __shared__ uint64_t sb[kGatherWarps][kGatherSort];  // used slots, then the sorted entries
    __shared__ unsigned tcount[kGatherWarps];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    volatile uint32_t* K = tk[wp];
    uint32_t* V = tv[wp];
    uint64_t* B = sb[wp];
    for (int i = lane; i < kGatherTab; i += 32) {
        K[i] = kEmpty;
        V[i] = 0;
    }
    if (lane == 0) tcount[wp] = 0;
    __syncwarp();
    const long long nwarps = (long long)gridDim.x * kGatherWarps;
    long long cc = (long long)blockIdx.x * kGatherWarps + wp;
    // the next node's member range and row capacity are loaded one node ahead
    uint32_t nm0 = 0, nm1 = 0, nr0 = 0, nr1 = 0;
    if (cc < nc) {
        nm0 = mbeg[cc];
        nm1 = mbeg[cc + 1];
        nr0 = rowoff[cc];
        nr1 = rowoff[cc + 1];
    }
    for (; cc < nc; cc += nwarps) {
        const int c = (int)cc;
        const uint32_t m0 = nm0, m1 = nm1, r0 = nr0, r1 = nr1;
        if (cc + nwarps < nc) {
            nm0 = mbeg[cc + nwarps];
            nm1 = mbeg[cc + nwarps + 1];
            nr0 = rowoff[cc + nwarps];
            nr1 = rowoff[cc + nwarps + 1];
        }
        if ((long long)r1 - r0 > kGatherMaxEntries) {
            if (lane == 0) {
                sel[c] = 1;
                atomicAdd(nsel, 1u);
            }
            continue;
        }
        bool over = false;
        for (uint32_t mb = m0; mb < m1 && !over; mb += 32) {
            int beg = 0, deg = 0;
            if (mb + lane < m1) {
                const int2 r = mrow[mb + lane];
                beg = r.x;
                deg = r.y;
            }
            int incl = deg;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int off = incl - deg;
            const int E = __shfl_sync(0xffffffffu, incl, 31);
            for (int q0 = 0; q0 < E && !over; q0 += 32 * kGatherWin) {
                int tg[kGatherWin];
                uint32_t wg[kGatherWin];
#pragma unroll
                for (int b = 0; b < kGatherWin; ++b) {
                    const int q = q0 + b * 32 + lane;
                    // owner: the largest lane o with off[o] <= q (its degree is > 0)
                    int o = 0;
#pragma unroll
                    for (int step = 16; step >= 1; step >>= 1) {
                        const int oc = __shfl_sync(0xffffffffu, off, o + step);
                        if (oc <= q) o += step;
                    }
                    const int ob = __shfl_sync(0xffffffffu, beg, o);
                    const int oo = __shfl_sync(0xffffffffu, off, o);
                    tg[b] = -1;
                    wg[b] = 0;
                    if (q < E) {
                        const int e = ob + (q - oo);
                        tg[b] = adjncy[e];
                        wg[b] = UNIT ? 1u : (uint32_t)adjwgt[e];
                    }
                }
#pragma unroll
                for (int b = 0; b < kGatherWin; ++b)
                    if (tg[b] >= 0) tg[b] = cmap[tg[b]];
                bool full = false;
#pragma unroll
                for (int b = 0; b < kGatherWin; ++b) {
                    if (tg[b] < 0 || tg[b] == c) continue;
                    // a new key goes in only while fewer than kGatherMaxDistinct are
                    // (at most 31 other lanes pass that test together), so the table
                    // never holds kGatherList keys and the probe ends
                    const uint32_t key = (uint32_t)tg[b];
                    uint32_t sl = gather_slot(key);
                    for (int probe = 0; probe < kGatherTab; ++probe) {
                        const uint32_t cur = K[sl];
                        if (cur == key) {
                            atomicAdd(&V[sl], wg[b]);
                            break;
                        }
                        if (cur == kEmpty) {
                            if (*(volatile unsigned*)&tcount[wp] >= (unsigned)kGatherMaxDistinct) {
                                full = true;
                                break;
                            }
                            const uint32_t prev = atomicCAS(const_cast<uint32_t*>(&K[sl]), kEmpty, key);
                            if (prev == kEmpty) {
                                B[atomicAdd(&tcount[wp], 1u)] = sl;
                                atomicAdd(&V[sl], wg[b]);
                                break;
                            }
                            if (prev == key) {
                                atomicAdd(&V[sl], wg[b]);
                                break;
                            }
                        }
                        sl = (sl + 1) & (kGatherTab - 1);
                    }
                }
                if (__any_sync(0xffffffffu, full)) over = true;
            }
        }
        __syncwarp();
        const int d = (int)tcount[wp];
        if (over) {
            for (int i = lane; i < d; i += 32) {
                const uint32_t sl = (uint32_t)B[i];
                K[sl] = kEmpty;
                V[sl] = 0;
            }
            if (lane == 0) {
                sel[c] = 1;
                atomicAdd(nsel, 1u);
                tcount[wp] = 0;
            }
            __syncwarp();
            continue;
        }
        // entries (target << 32 | weight); the table is cleared behind them
        if (d <= 32) {
            uint64_t x = ~0ull;
            if (lane < d) {
                const uint32_t sl = (uint32_t)B[lane];
                x = ((uint64_t)K[sl] << 32) | V[sl];
                K[sl] = kEmpty;
                V[sl] = 0;
            }
            for (int k = 2; k <= 32; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const uint64_t y = __shfl_xor_sync(0xffffffffu, x, j);
                    const bool lower = (lane & j) == 0, up = (lane & k) == 0;
                    x = (lower == up) ? (x < y ? x : y) : (x > y ? x : y);
                }
            if (lane < d) bucket[(long long)r0 + lane] = x;
        } else {
            int P = 64;
            while (P < d) P <<= 1;
            for (int i = lane; i < d; i += 32) {
                const uint32_t sl = (uint32_t)B[i];
                B[i] = ((uint64_t)K[sl] << 32) | V[sl];
                K[sl] = kEmpty;
                V[sl] = 0;
            }
            for (int i = d + lane; i < P; i += 32) B[i] = ~0ull;
            __syncwarp();
            for (int k = 2; k <= P; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < P; i += 32) {
                        const int l = i ^ j;
                        if (l > i) {
                            const uint64_t x = B[i], y = B[l];
                            const bool up = (i & k) == 0;
                            if ((x > y) == up) {
                                B[i] = y;
                                B[l] = x;
                            }
                        }
                    }
                    __syncwarp();
                }
            for (int i = lane; i < d; i += 32) bucket[(long long)r0 + i] = B[i];
        }
        if (lane == 0) {
            ucnt[c] = (uint32_t)d;
            tcount[wp] = 0;
        }
        __syncwarp();
    }
}

// One thread per fine vertex: merges its neighbours by coarse target in
// kEmitSlots register slots (edges inside its own coarse node are dropped)
// and appends the (cv << 32 | w) entries to its coarse row's bucket,
// flushing the slots whenever a new target finds them full -- repeated
// targets that this leaves are merged by the per-row sort that follows.
constexpr int kEmitSlots = 8;
constexpr int kEmitLaneDeg = 256;  // longer rows are emitted by the whole warp

__device__ __forceinline__ void flush_slots(int cnt, const uint32_t* st, const uint32_t* sw, uint64_t* dst) {
#pragma unroll
    for (int i = 0; i < kEmitSlots; ++i)
        if (i < cnt) dst[i] = ((uint64_t)st[i] << 32) | sw[i];
}

// Merges the entries [e0, e1) with stride `step` of a row whose coarse node
// is `own` into kEmitSlots register slots and appends them to the bucket
// at rowoff[own] through the row's fill counter.
__device__ __forceinline__ void emit_range(int e0, int e1, int step, uint32_t own, const int* __restrict__ adjncy,
                                           const int* __restrict__ adjwgt, const int* __restrict__ cmap,
                                           const uint32_t* __restrict__ rowoff, uint32_t* fill, uint64_t* bucket) {
    uint32_t st[kEmitSlots], sw[kEmitSlots];
    int used = 0;
    for (int e = e0; e < e1; e += step) {
        const uint32_t t = (uint32_t)cmap[adjncy[e]];
        const uint32_t w = (uint32_t)adjwgt[e];
        if (t == own) continue;
        bool hit = false;
#pragma unroll
        for (int i = 0; i < kEmitSlots; ++i)
            if (i < used && st[i] == t) { sw[i] += w; hit = true; }
        if (hit) continue;
        if (used == kEmitSlots) {
            flush_slots(kEmitSlots, st, sw, bucket + rowoff[own] + atomicAdd(&fill[own], (uint32_t)kEmitSlots));
            used = 0;
        }
#pragma unroll
        for (int i = 0; i < kEmitSlots; ++i)
            if (i == used) { st[i] = t; sw[i] = w; }
        ++used;
    }
    if (used) flush_slots(used, st, sw, bucket + rowoff[own] + atomicAdd(&fill[own], (uint32_t)used));
}

// Rows longer than kEmitLaneDeg are left to emit_wide.  UNIT: every edge
// weight is 1 (adjwgt is not read).  The row entries of the next group of
// four are loaded while the coarse ids of the current group are gathered.
// With sel, only the fine nodes of flagged coarse nodes are emitted, and
// nothing at all when *nsel is 0.
template <bool UNIT>
__global__ void __launch_bounds__(kThreads) emit_kernel(int n, const int* __restrict__ xadj,
                                                        const int* __restrict__ adjncy,
                                                        const int* __restrict__ adjwgt,
                                                        const int* __restrict__ cmap,
                                                        const uint32_t* __restrict__ rowoff, uint32_t* fill,
                                                        uint64_t* bucket, const uint8_t* __restrict__ sel,
                                                        const unsigned* __restrict__ nsel) {
    if (nsel && *nsel == 0u) return;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        const int v = (int)(base + threadIdx.x);
        if (v >= n) continue;
        const uint32_t own = (uint32_t)cmap[v];
        if (sel && !sel[own]) continue;
        const int beg = xadj[v], end = xadj[v + 1];
        if (end - beg > kEmitLaneDeg) continue;
        uint32_t st[kEmitSlots], sw[kEmitSlots];
        int used = 0;
        int un[4];
        uint32_t wn[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            un[j] = -1;
            wn[j] = 0;
            if (beg + j < end) {
                un[j] = adjncy[beg + j];
                wn[j] = UNIT ? 1u : (uint32_t)adjwgt[beg + j];
            }
        }
        for (int e = beg; e < end; e += 4) {
            int u[4];
            uint32_t w[4], t[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                u[j] = un[j];
                w[j] = wn[j];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) t[j] = u[j] >= 0 ? (uint32_t)cmap[u[j]] : kEmpty;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                un[j] = -1;
                wn[j] = 0;
                if (e + 4 + j < end) {
                    un[j] = adjncy[e + 4 + j];
                    wn[j] = UNIT ? 1u : (uint32_t)adjwgt[e + 4 + j];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (u[j] < 0 || t[j] == own) continue;
                bool hit = false;
#pragma unroll
                for (int i = 0; i < kEmitSlots; ++i)
                    if (i < used && st[i] == t[j]) { sw[i] += w[j]; hit = true; }
                if (hit) continue;
                if (used == kEmitSlots) {
                    flush_slots(kEmitSlots, st, sw,
                                bucket + rowoff[own] + atomicAdd(&fill[own], (uint32_t)kEmitSlots));
                    used = 0;
                }
#pragma unroll
                for (int i = 0; i < kEmitSlots; ++i)
                    if (i == used) { st[i] = t[j]; sw[i] = w[j]; }
                ++used;
            }
        }
        if (used) flush_slots(used, st, sw, bucket + rowoff[own] + atomicAdd(&fill[own], (uint32_t)used));
    }
}

// Long rows, spread over warps: the entry space is cut into chunks of
// kEmitChunk entries; the warp of a chunk emits the part of every long row
// that falls into it (light rows are emit_kernel's), taking write positions
// from the row's cursor by atomics.  Chunks of one row are not merged with
// each other here; the per-row merge later is.
constexpr int kEmitChunk = 2048;

__global__ void __launch_bounds__(kThreads) emit_wide(int n, long long m, const int* __restrict__ xadj,
                                                      const int* __restrict__ adjncy, const int* __restrict__ adjwgt,
                                                      const int* __restrict__ cmap, const uint32_t* __restrict__ rowoff,
                                                      uint32_t* fill, uint64_t* bucket, const uint8_t* __restrict__ sel,
                                                      const unsigned* __restrict__ nsel) {
    if (nsel && *nsel == 0u) return;
    const int lane = threadIdx.x & 31;
    const long long chunks = (m + kEmitChunk - 1) / kEmitChunk;
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; c < chunks;
         c += (long long)gridDim.x * blockDim.x / 32) {
        const long long lo = c * kEmitChunk, hi = std::min<long long>(lo + kEmitChunk, m);
        // v = the row holding entry lo: largest v with xadj[v] <= lo
        int a = 0, b = n;
        while (b - a > 1) {
            const int mid = (a + b) >> 1;
            if (xadj[mid] <= lo) a = mid;
            else b = mid;
        }
        for (int v = a; v < n && xadj[v] < hi; ++v) {
            const int beg = xadj[v], end = xadj[v + 1];
            if (end - beg <= kEmitLaneDeg) continue;
            const uint32_t own = (uint32_t)cmap[v];
            if (sel && !sel[own]) continue;
            const int s = (int)std::max<long long>(lo, beg), e = (int)std::min<long long>(hi, end);
            emit_range(s + lane, e, 32, own, adjncy, adjwgt, cmap, rowoff, fill, bucket);
        }
    }
}


__global__ void head_flags(long long E, const uint64_t* __restrict__ K, uint32_t* h) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < E;
         i += (long long)gridDim.x * blockDim.x)
        h[i] = (i == 0 || K[i] != K[i - 1]) ? 1u : 0u;
}

// ---- segmented merge: entries bucketed by coarse source row, each row
// sorted and merged on its own

constexpr int kSegMax = 1024;       // rows up to this many entries merge in shared memory
constexpr int kSegSmall = 64;       // rows up to this many entries sort in registers
constexpr int kMergeWarps = 4;      // warps per block of the shared-memory merge
constexpr int kMergeWarpsSmall = 8; // warps per block of the register merge

// Warp per coarse row: sorts the row's bucket (bitonic), sums the weights of
// equal targets and writes the distinct entries back to the start of the
// bucket; ucnt[row] = their number.  LARGE = false takes the rows of at
// most kSegSmall entries (sorted in registers, a 512-byte staging buffer
// per warp, so many warps fit on an SM); LARGE = true the rows of up to
// kSegMax entries (sorted in an 8 KiB shared buffer per warp) and marks the
// longer ones for the global path (bigsz[row] = their size).  With sel, only
// the flagged rows (none when *nsel is 0).
template <bool LARGE>
__global__ void __launch_bounds__((LARGE ? kMergeWarps : kMergeWarpsSmall) * 32)
    merge_rows(int nc, const uint32_t* __restrict__ rowoff, const uint32_t* __restrict__ fill, uint64_t* bucket,
               uint32_t* ucnt, uint32_t* bigsz, const uint8_t* __restrict__ sel, const unsigned* __restrict__ nsel) {
    constexpr int W = LARGE ? kMergeWarps : kMergeWarpsSmall;
    constexpr int CAP = LARGE ? kSegMax : kSegSmall;
    __shared__ uint64_t buf[W][CAP];
    if (nsel && *nsel == 0u) return;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    uint64_t* b = buf[wp];
    for (long long r = (long long)blockIdx.x * W + wp; r < nc; r += (long long)gridDim.x * W) {
        if (sel && !sel[r]) continue;  // a row of the gather path
        const long long beg = rowoff[r];
        const int s = (int)fill[r];
        if (LARGE && s > kSegMax) {
            if (lane == 0) { bigsz[r] = (uint32_t)s; ucnt[r] = 0; }
            continue;
        }
        if ((s <= kSegSmall) == LARGE) continue;  // the other kernel's row
        int P = 1;
        while (P < s) P <<= 1;
        if (P <= 32) {
            // bitonic sort in registers, one element per lane
            uint64_t x = lane < s ? bucket[beg + lane] : ~0ull;
            for (int k = 2; k <= 32; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const uint64_t y = __shfl_xor_sync(0xffffffffu, x, j);
                    const bool lower = (lane & j) == 0, up = (lane & k) == 0;
                    x = (lower == up) ? (x < y ? x : y) : (x > y ? x : y);
                }
            b[lane] = x;
            __syncwarp();
        } else if (P <= 64) {
            // bitonic sort in registers: element i = lane + 32 r, r = 0, 1
            uint64_t x0 = lane < s ? bucket[beg + lane] : ~0ull;
            uint64_t x1 = lane + 32 < s ? bucket[beg + lane + 32] : ~0ull;
            for (int k = 2; k <= 64; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    if (j == 32) {
                        // partner in the same lane: elements lane and lane + 32
                        const bool up = (lane & k) == 0;
                        if ((x0 > x1) == up) { const uint64_t t = x0; x0 = x1; x1 = t; }
                    } else {
                        const uint64_t y0 = __shfl_xor_sync(0xffffffffu, x0, j);
                        const uint64_t y1 = __shfl_xor_sync(0xffffffffu, x1, j);
                        const bool lower = (lane & j) == 0;
                        const bool up0 = (lane & k) == 0, up1 = ((lane + 32) & k) == 0;
                        x0 = (lower == up0) ? (x0 < y0 ? x0 : y0) : (x0 > y0 ? x0 : y0);
                        x1 = (lower == up1) ? (x1 < y1 ? x1 : y1) : (x1 > y1 ? x1 : y1);
                    }
                }
            b[lane] = x0;
            b[lane + 32] = x1;
            __syncwarp();
        } else if (LARGE) {
            for (int i = lane; i < P; i += 32) b[i] = i < s ? bucket[beg + i] : ~0ull;
            __syncwarp();
            for (int k = 2; k <= P; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < P; i += 32) {
                        const int l = i ^ j;
                        if (l > i) {
                            const uint64_t x = b[i], y = b[l];
                            const bool up = (i & k) == 0;
                            if ((x > y) == up) { b[i] = y; b[l] = x; }
                        }
                    }
                    __syncwarp();
                }
        }
        // distinct targets, weights summed over each run
        uint32_t written = 0;
        for (int i0 = 0; i0 < s; i0 += 32) {
            const int i = i0 + lane;
            bool head = false;
            uint64_t outv = 0;
            if (i < s) {
                const uint32_t t = (uint32_t)(b[i] >> 32);
                head = i == 0 || (uint32_t)(b[i - 1] >> 32) != t;
                if (head) {
                    uint32_t sum = (uint32_t)b[i];
                    for (int j = i + 1; j < s && (uint32_t)(b[j] >> 32) == t; ++j) sum += (uint32_t)b[j];
                    outv = ((uint64_t)t << 32) | sum;
                }
            }
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if (head) bucket[beg + written + __popc(hm & ((1u << lane) - 1u))] = outv;
            written += __popc(hm);
        }
        if (lane == 0) ucnt[r] = written;
        __syncwarp();
    }
}

// Entries of the long rows, gathered for the global sort: key cu << tb | cv.
__global__ void gather_big(int nc, const uint32_t* __restrict__ rowoff, const uint32_t* __restrict__ bigsz,
                           const uint32_t* __restrict__ bigoff, const uint64_t* __restrict__ bucket, int tb,
                           uint64_t* K, uint32_t* V) {
    for (int r = blockIdx.x; r < nc; r += gridDim.x) {
        const uint32_t s = bigsz[r];
        if (!s) continue;
        const long long src = rowoff[r], dst = bigoff[r];
        for (uint32_t i = threadIdx.x; i < s; i += blockDim.x) {
            const uint64_t x = bucket[src + i];
            K[dst + i] = ((uint64_t)r << tb) | (x >> 32);
            V[dst + i] = (uint32_t)x;
        }
    }
}

// The distinct keys of the sorted long-row entries go back to the start of
// their row's bucket, in order: position = global distinct index minus the
// row's first distinct index (ufirst, an atomicMin).
__global__ void first_unique(long long E, const uint64_t* __restrict__ K, const uint32_t* __restrict__ uidx, int tb,
                             uint32_t* ufirst) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (long long)gridDim.x * blockDim.x)
        if (i == 0 || (K[i - 1] >> tb) != (K[i] >> tb)) ufirst[K[i] >> tb] = uidx[i];
}

__global__ void reduce_big(long long E, const uint64_t* __restrict__ K, const uint32_t* __restrict__ V,
                           const uint32_t* __restrict__ uidx, const uint32_t* __restrict__ ufirst,
                           const uint32_t* __restrict__ rowoff, int tb, uint64_t* bucket, uint32_t* ucnt) {
    const uint64_t mask = (1ull << tb) - 1ull;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (long long)gridDim.x * blockDim.x) {
        const uint64_t k = K[i];
        if (i > 0 && K[i - 1] == k) continue;
        uint32_t s = V[i];
        for (long long j = i + 1; j < E && K[j] == k; ++j) s += V[j];
        const uint32_t r = (uint32_t)(k >> tb);
        bucket[(long long)rowoff[r] + (uidx[i] - ufirst[r])] = ((k & mask) << 32) | s;
        atomicAdd(&ucnt[r], 1u);
    }
}

// Degree statistics of the coarse graph from its row lengths, before the
// rows are copied: [0] max degree, [1] isolated nodes, [2] their largest
// weight, [3] largest node weight (what degree_stats computes).
__global__ void coarse_stats(int nc, const uint32_t* __restrict__ ucnt, const int* __restrict__ cvw, unsigned* out) {
    unsigned md = 0, iso = 0, wi = 0, wa = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nc; r += gridDim.x * blockDim.x) {
        const unsigned d = ucnt[r], w = (unsigned)cvw[r];
        md = max(md, d);
        wa = max(wa, w);
        if (d == 0) {
            ++iso;
            wi = max(wi, w);
        }
    }
    for (int o = 16; o >= 1; o >>= 1) {
        md = max(md, __shfl_xor_sync(0xffffffffu, md, o));
        iso += __shfl_xor_sync(0xffffffffu, iso, o);
        wi = max(wi, __shfl_xor_sync(0xffffffffu, wi, o));
        wa = max(wa, __shfl_xor_sync(0xffffffffu, wa, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (md) atomicMax(out, md);
        if (iso) atomicAdd(out + 1, iso);
        if (wi) atomicMax(out + 2, wi);
        if (wa) atomicMax(out + 3, wa);
    }
}

// Warp per row: the distinct entries move from the bucket to the coarse CSR.
__global__ void copy_rows(int nc, const uint32_t* __restrict__ rowoff, const uint32_t* __restrict__ ucnt,
                          const int* __restrict__ cxadj, const uint64_t* __restrict__ bucket, int* cadj, int* cw) {
    const int lane = threadIdx.x & 31;
    for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; r < nc;
         r += (long long)gridDim.x * blockDim.x / 32) {
        const long long src = rowoff[r], dst = cxadj[r];
        const uint32_t u = ucnt[r];
        for (uint32_t i = lane; i < u; i += 32) {
            const uint64_t x = bucket[src + i];
            cadj[dst + i] = (int)(x >> 32);
            cw[dst + i] = (int)(uint32_t)x;
        }
    }
}

}  // namespace

void contract(Ctx& ctx, const DevGraph& g, const int* label, int* cmap, DevGraph& out,
              int** out_xadj, int** out_adjncy, int** out_adjwgt, int** out_vwgt) {
    cudaStream_t st = ctx.stream;
    const size_t mk = ctx.scratch.mark();
    const int n = g.n;
    if (n == 0) {
        int* cx = ctx.hier.alloc<int>(1);
        KB_CUDA(cudaMemsetAsync(cx, 0, sizeof(int), st));
        out = DevGraph{};
        out.maxvw = 0;
        out.xadj = cx;
        *out_xadj = cx;
        *out_adjncy = *out_adjwgt = *out_vwgt = nullptr;
        return;
    }
    // 1. coarse ids
    int* mm = ctx.scratch.alloc<int>((size_t)n);
    uint32_t* pos = ctx.scratch.alloc<uint32_t>((size_t)n + 1);
    uint32_t* tot = reinterpret_cast<uint32_t*>(ctx.dscalars);
    {
        PhaseScope ps(ctx, "contract_ids", 20.0 * n);
        fill_i32(mm, n, INT_MAX, st);
        leader_min<<<grid_for(n, 256), 256, 0, st>>>(n, label, mm);
        KB_LAUNCH();
        leader_flags<<<grid_for(n, 256), 256, 0, st>>>(n, label, mm, pos);
        KB_LAUNCH();
        exclusive_scan_u32(pos, pos, n, tot, st, ctx.scratch);
    }
    KB_CUDA(cudaMemcpyAsync(ctx.pinned, tot, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    KB_CUDA(cudaStreamSynchronize(st));
    const int nc = (int)ctx.pinned[0];
    int* cvw = ctx.hier.alloc<int>((size_t)nc);
    int* cxadj = ctx.hier.alloc<int>((size_t)nc + 1);
    const long long m = g.m;
    uint32_t* rowcap = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
    uint32_t* rowoff = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
    uint32_t* fill = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
    KB_CUDA(cudaMemsetAsync(cvw, 0, sizeof(int) * (size_t)nc, st));
    KB_CUDA(cudaMemsetAsync(rowcap, 0, sizeof(uint32_t) * ((size_t)nc + 1), st));
    KB_CUDA(cudaMemsetAsync(fill, 0, sizeof(uint32_t) * ((size_t)nc + 1), st));
    // clusterings (several members per coarse node on average) take the
    // gather path; matchings (at most two) the emission path
    const bool gather = (long long)n * 2 >= (long long)nc * 5;
    uint32_t* msize = nullptr;
    if (gather) {
        msize = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
        KB_CUDA(cudaMemsetAsync(msize, 0, sizeof(uint32_t) * ((size_t)nc + 1), st));
    }
    {
        PhaseScope ps(ctx, "contract_ids", 16.0 * n);
        make_cmap<<<grid_for(n, 256), 256, 0, st>>>(n, label, mm, pos, g.vwgt, g.xadj, cmap,
                                                    reinterpret_cast<uint32_t*>(cvw), rowcap, msize);
        KB_LAUNCH();
        // bucket of coarse row c: [rowoff[c], rowoff[c] + its members' degrees)
        exclusive_scan_u32(rowcap, rowoff, (long long)nc + 1, nullptr, st, ctx.scratch);
    }
    int tb = 1;
    while ((1LL << tb) < (long long)nc) ++tb;
    uint64_t* bucket = ctx.scratch.alloc<uint64_t>((size_t)std::max<long long>(m, 1));
    uint32_t* ucnt = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
    uint32_t* bigsz = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
    uint32_t* bigoff = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
    uint32_t* big = reinterpret_cast<uint32_t*>(ctx.dscalars + 16);  // [16] long-row entries
    // ucnt / bigsz have nc + 1 entries (the scans read the last one)
    KB_CUDA(cudaMemsetAsync(ucnt, 0, sizeof(uint32_t) * ((size_t)nc + 1), st));
    KB_CUDA(cudaMemsetAsync(bigsz, 0, sizeof(uint32_t) * ((size_t)nc + 1), st));
    // 2a. gather path: member lists, then a warp per coarse node; the nodes it
    // flags go through the emission path, which then skips all others
    uint8_t* sel = nullptr;
    unsigned* nsel = nullptr;
    if (gather) {
        uint32_t* mbeg = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
        uint32_t* mfill = ctx.scratch.alloc<uint32_t>((size_t)nc);
        int2* mrow = ctx.scratch.alloc<int2>((size_t)n);
        sel = ctx.scratch.alloc<uint8_t>((size_t)nc);
        nsel = reinterpret_cast<unsigned*>(ctx.dscalars + 18);  // [18] flagged nodes
        KB_CUDA(cudaMemsetAsync(mfill, 0, sizeof(uint32_t) * (size_t)nc, st));
        KB_CUDA(cudaMemsetAsync(sel, 0, (size_t)nc, st));
        KB_CUDA(cudaMemsetAsync(nsel, 0, sizeof(unsigned), st));
        {
            PhaseScope ps(ctx, "contract_ids", 12.0 * n);
            exclusive_scan_u32(msize, mbeg, (long long)nc + 1, nullptr, st, ctx.scratch);
            scatter_members<<<grid_for(n, 256), 256, 0, st>>>(n, cmap, g.xadj, mbeg, mfill, mrow);
            KB_LAUNCH();
        }
        PhaseScope ps(ctx, "contract_gather", (g.unit_weights ? 8.0 : 12.0) * m + 16.0 * n);
        const int gg = (int)std::max<long long>(1, std::min<long long>(div_up(nc, kGatherWarps), (long long)kNumSMs * kGatherBlocksPerSM));
        if (g.unit_weights)
            gather_rows<true><<<gg, kGatherWarps * 32, 0, st>>>(nc, mbeg, mrow, g.adjncy, g.adjwgt, cmap, rowoff,
                                                                bucket, ucnt, sel, nsel);
        else
            gather_rows<false><<<gg, kGatherWarps * 32, 0, st>>>(nc, mbeg, mrow, g.adjncy, g.adjwgt, cmap, rowoff,
                                                                 bucket, ucnt, sel, nsel);
        KB_LAUNCH();
    }
    // 2b. emission straight into the coarse rows' buckets (at most m entries)
    {
        PhaseScope ps(ctx, "contract_emit", gather ? 0.0 : (g.unit_weights ? 8.0 : 12.0) * m + 8.0 * n);
        if (g.unit_weights)
            emit_kernel<true><<<grid_for(n, kThreads), kThreads, 0, st>>>(n, g.xadj, g.adjncy, g.adjwgt, cmap, rowoff,
                                                                          fill, bucket, sel, nsel);
        else
            emit_kernel<false><<<grid_for(n, kThreads), kThreads, 0, st>>>(n, g.xadj, g.adjncy, g.adjwgt, cmap, rowoff,
                                                                           fill, bucket, sel, nsel);
        KB_LAUNCH();
        if (g.maxdeg > kEmitLaneDeg) {
            const long long chunks = (m + kEmitChunk - 1) / kEmitChunk;
            emit_wide<<<grid_for(32LL * chunks, kThreads), kThreads, 0, st>>>(n, m, g.xadj, g.adjncy, g.adjwgt, cmap,
                                                                           rowoff, fill, bucket, sel, nsel);
            KB_LAUNCH();
        }
    }
    // 4. merge each row: shared-memory sort for rows up to kSegMax entries
    {
        PhaseScope ps(ctx, "contract_merge", gather ? 0.0 : 16.0 * m);
        const int gs = (int)std::max<long long>(1, std::min<long long>(div_up(nc, kMergeWarpsSmall), (long long)kNumSMs * 16));
        merge_rows<false><<<gs, kMergeWarpsSmall * 32, 0, st>>>(nc, rowoff, fill, bucket, ucnt, bigsz, sel, nsel);
        KB_LAUNCH();
        if (g.maxdeg > 0) {
            const int gb = (int)std::max<long long>(1, std::min<long long>(div_up(nc, kMergeWarps), (long long)kNumSMs * 7));
            merge_rows<true><<<gb, kMergeWarps * 32, 0, st>>>(nc, rowoff, fill, bucket, ucnt, bigsz, sel, nsel);
            KB_LAUNCH();
        }
        exclusive_scan_u32(bigsz, bigoff, (long long)nc + 1, big, st, ctx.scratch);
    }
    // row lengths -> coarse xadj and the coarse degree statistics, read back
    // with the long-row count in one synchronisation (redone below in the
    // rare case of long rows, whose lengths the global path still has to add)
    unsigned* stats = reinterpret_cast<unsigned*>(ctx.dscalars + 40);  // [40..43]
    uint32_t* mct = reinterpret_cast<uint32_t*>(ctx.dscalars + 17);    // [17] coarse entries
    auto rows_and_stats = [&]() {
        PhaseScope ps(ctx, "contract_rows", 8.0 * nc);
        exclusive_scan_u32(ucnt, reinterpret_cast<uint32_t*>(cxadj), (long long)nc + 1, mct, st, ctx.scratch);
        KB_CUDA(cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned), st));
        coarse_stats<<<grid_for(nc, 256), 256, 0, st>>>(nc, ucnt, cvw, stats);
        KB_LAUNCH();
        // pinned[0] long-row entries, [1] coarse entries, [2..5] statistics
        KB_CUDA(cudaMemcpyAsync(ctx.pinned, big, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaMemcpyAsync(ctx.pinned + 1, mct, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaMemcpyAsync(ctx.pinned + 2, stats, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        KB_CUDA(cudaStreamSynchronize(st));
    };
    rows_and_stats();
    const long long EB = ctx.pinned[0];
    if (EB > 0) {
        // longer rows: global LSD radix sort of their entries, then reduce
        const size_t mk2 = ctx.scratch.mark();
        uint64_t* K0 = ctx.scratch.alloc<uint64_t>((size_t)EB);
        uint32_t* V0 = ctx.scratch.alloc<uint32_t>((size_t)EB);
        uint64_t* K1 = ctx.scratch.alloc<uint64_t>((size_t)EB);
        uint32_t* V1 = ctx.scratch.alloc<uint32_t>((size_t)EB);
        uint32_t* uidx = ctx.scratch.alloc<uint32_t>((size_t)EB);
        uint32_t* ufirst = ctx.scratch.alloc<uint32_t>((size_t)nc + 1);
        PhaseScope ps(ctx, "contract_sort", 32.0 * EB * ((2 * tb + 7) / 8));
        gather_big<<<grid_for(nc, 256), 256, 0, st>>>(nc, rowoff, bigsz, bigoff, bucket, tb, K0, V0);
        KB_LAUNCH();
        const int which = radix_sort_pairs(K0, V0, K1, V1, EB, 2 * tb, st, ctx.scratch);
        uint64_t* K = which ? K1 : K0;
        uint32_t* V = which ? V1 : V0;
        head_flags<<<grid_for(EB, 256), 256, 0, st>>>(EB, K, uidx);
        KB_LAUNCH();
        exclusive_scan_u32(uidx, uidx, EB, nullptr, st, ctx.scratch);
        first_unique<<<grid_for(EB, 256), 256, 0, st>>>(EB, K, uidx, tb, ufirst);
        KB_LAUNCH();
        reduce_big<<<grid_for(EB, 256), 256, 0, st>>>(EB, K, V, uidx, ufirst, rowoff, tb, bucket, ucnt);
        KB_LAUNCH();
        ctx.scratch.release(mk2);
        rows_and_stats();
    }
    // 5. the rows themselves
    const long long mc = (long long)ctx.pinned[1];
    const int c_maxdeg = (int)ctx.pinned[2];
    const unsigned c_iso = ctx.pinned[3], c_isow = ctx.pinned[4], c_maxvw = ctx.pinned[5];
    int* cadj = ctx.hier.alloc<int>((size_t)std::max<long long>(mc, 1));
    int* cwgt = ctx.hier.alloc<int>((size_t)std::max<long long>(mc, 1));
    {
        PhaseScope ps(ctx, "contract_rows", 16.0 * mc + 12.0 * nc);
        copy_rows<<<grid_for(32LL * nc, 256), 256, 0, st>>>(nc, rowoff, ucnt, cxadj, bucket, cadj, cwgt);
        KB_LAUNCH();
    }
    out = DevGraph{};
    out.n = nc;
    out.m = mc;
    out.maxdeg = c_maxdeg;
    out.iso_count = c_iso;
    out.iso_wmax = c_isow;
    out.maxvw = c_maxvw;
    out.rows_sorted = 1;  // rows come out sorted by target, without repeats
    out.xadj = cxadj;
    out.adjncy = cadj;
    out.adjwgt = cwgt;
    out.vwgt = cvw;
    *out_xadj = cxadj;
    *out_adjncy = cadj;
    *out_adjwgt = cwgt;
    *out_vwgt = cvw;
    ctx.scratch.release(mk);
}

}  // namespace kb
