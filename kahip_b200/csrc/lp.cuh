// lp.cuh -- device graph view and the label-propagation phases
// (clustering, refinement, balance repair) of the multilevel scheme.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "context.h"
#include "knobs.h"

namespace kb {

// A graph level resident in device memory (int32 CSR).
struct DevGraph {
    int n = 0;
    long long m = 0;
    int maxdeg = 0;
    unsigned iso_count = 0, iso_wmax = 0;  // isolated vertices and their largest weight (max_degree fills them)
    unsigned maxvw = 0xFFFFFFFFu;          // largest node weight (degree_stats fills it; all ones: unknown)
    bool unit_weights = false;  // every edge weight is 1 (lets sweeps skip adjwgt)
    int rows_sorted = -1;       // 1 / 0: rows do / do not list targets strictly increasing; -1 unknown
    bool stats_known = false;   // maxdeg, iso_count, iso_wmax and maxvw are filled (the input check did it)
    const int* xadj = nullptr;
    const int* adjncy = nullptr;
    const int* adjwgt = nullptr;
    const int* vwgt = nullptr;
};

// Work counters of the sweep kernels (vertices and edges actually scanned).
struct SweepWork {
    unsigned long long vertices = 0, edges = 0;
};

// LP clustering of one coarsening level; label[n] (device) out.
void lp_cluster(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, int* label);

// LP refinement at one level; part[n] in/out, bw[k] in/out (device).
// active0 (device, optional): the vertices the first round sweeps (flags);
// it must hold every vertex with a neighbour in another block -- the others
// cannot propose a move, so leaving them out changes nothing.  Null: all.
void lp_refine(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, uint32_t bound, int* part,
               uint32_t* bw, const uint8_t* active0 = nullptr);

// Exact balance repair; returns true if every block ends <= bound.  skip
// (device, optional): when *skip != 0 the call does nothing (a caller whose
// own loop already ended on the device).  *moved (optional) tells whether
// the repair ran (and may have moved vertices).
bool balance(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, uint32_t bound, int* part,
             uint32_t* bw, const int* skip = nullptr, bool* moved = nullptr);

// Block weights (bw[k] zeroed and filled) and, when cut != nullptr, the edge
// cut (device uint64, sum over directed entries / 2 applied by the caller).
void block_weights_and_cut(Ctx& ctx, const DevGraph& g, const int* part, int k, uint32_t* bw,
                           unsigned long long* cut2);

// part_fine[v] = part_coarse[cmap[v]]; with cb and fb also fb[v] = cb[cmap[v]]
void project(Ctx& ctx, int n, const int* cmap, const int* part_coarse, int* part_fine,
             const uint8_t* cb = nullptr, uint8_t* fb = nullptr);

// out[v] = 1 when v has a neighbour in another block of part (device)
void boundary_flags(Ctx& ctx, const DevGraph& g, const int* part, uint8_t* out);

// max degree of g (device reduction + readback)
int max_degree(Ctx& ctx, const DevGraph& g);

// Same, and fills g.maxdeg, g.iso_count and g.iso_wmax in one readback.
void degree_stats(Ctx& ctx, DevGraph& g);

// Device-side input checks: bit 1 = target out of range, 2 = negative edge
// weight, 4 = negative node weight, 8 = xadj not starting at 0 / not
// monotone, 16 = some edge weight differs from 1 (not an error), 32 = some
// row does not list its targets in strictly increasing order (not an error).  Also returns the node weight sum (32-bit, as the reference's
// NodeWeight accumulates it).  Synchronises the stream.
// stats (optional): receives the degree statistics of degree_stats as well.
int check_graph(Ctx& ctx, const DevGraph& g, uint32_t* total_weight = nullptr, DevGraph* stats = nullptr);
// The same check in parts: begin (clears the flags), any number of vertex
// ranges (unit_known: every edge weight is 1, adjwgt is not read), end
// (synchronises and returns the flags).
void check_graph_begin(Ctx& ctx);
void check_graph_range(Ctx& ctx, const DevGraph& g, int v_lo, int v_hi, bool unit_known);
int check_graph_end(Ctx& ctx, uint32_t* total_weight, DevGraph* stats = nullptr);

// true if every row lists its targets in strictly increasing order
// (synchronises the stream)
bool rows_strictly_increasing(Ctx& ctx, const DevGraph& g);

// Bundles the isolated vertices (degree 0) of a level, which no clustering
// or matching can merge: in increasing id order, consecutive groups of
// G = (bound - 1) / (largest isolated node weight) vertices (all of them when
// that weight is 0) share the label of their first member, so every bundle
// weighs less than `bound`.  Nothing changes when G < 2 or fewer than two
// vertices are isolated.  label[] of non-isolated vertices is left as is.
// Uses g.iso_count / g.iso_wmax (degree_stats) and does not synchronise.
void bundle_isolated(Ctx& ctx, const DevGraph& g, uint32_t bound, int* label);

// Number of v with label[v] == v (synchronises the stream).
long long count_leaders(Ctx& ctx, int n, const int* label);

// label[v] = v, cw[v] = vwgt[v]
void init_labels(Ctx& ctx, const DevGraph& g, int* label, uint32_t* cw);

}  // namespace kb
