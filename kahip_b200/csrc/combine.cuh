// combine.cuh -- device parts of the KaFFPaE combine operator (combine.cu).
#pragma once

#include "lp.cuh"

namespace kb {

// out = the edges of f whose two ends lie in the same block of p1 and of p2
// (rows keep their order; arrays in ctx.scratch).  Degree statistics are
// filled; unit_weights and rows_sorted are inherited from f.
void filter_by_parents(Ctx& ctx, const DevGraph& f, const int* p1, const int* p2, DevGraph& out);

// Whether every entry of pa and pb (n each, device) lies in [0, k); synchronises.
bool parents_in_range(Ctx& ctx, int n, int k, const int* pa, const int* pb);

// p1c[cmap[v]] = p1[v], p2c[cmap[v]] = p2[v] (every coarse node lies inside
// one block of each parent, so all writers of a coarse node agree).
void parents_to_coarse(Ctx& ctx, int n, const int* cmap, const int* p1, const int* p2, int* p1c, int* p2c);

}  // namespace kb
