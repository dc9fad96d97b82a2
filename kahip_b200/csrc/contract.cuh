// contract.cuh -- contraction of a clustering (contract.cu).
#pragma once

#include "lp.cuh"

namespace kb {

// Builds the coarse graph of clustering `label` (arbitrary ids < n).  cmap[n]
// (device, caller-allocated) receives fine -> coarse ids.  The coarse arrays
// are allocated in ctx.hier and returned both as `out` and as writable
// pointers.  Synchronises the stream three times (n', entry count, m').
void contract(Ctx& ctx, const DevGraph& g, const int* label, int* cmap, DevGraph& out,
              int** out_xadj, int** out_adjncy, int** out_adjwgt, int** out_vwgt);

}  // namespace kb
