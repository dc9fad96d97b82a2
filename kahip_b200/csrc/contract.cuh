// contract.cuh -- contraction of a clustering (contract.cu).
#pragma once

#include "lp.cuh"

namespace kb {

// Builds the coarse graph of clustering `label` (arbitrary ids < n).  cmap[n]
// (device, caller-allocated) receives fine -> coarse ids.  The coarse arrays
// are allocated in ctx.hier and returned both as `out` and as writable
// pointers; `out` carries its degree statistics (what degree_stats fills).
// Synchronises the stream twice (n'; then long-row entries, m' and the
// statistics together), a third time only when some coarse row gathers more
// than 1024 entries.
void contract(Ctx& ctx, const DevGraph& g, const int* label, int* cmap, DevGraph& out,
              int** out_xadj, int** out_adjncy, int** out_adjwgt, int** out_vwgt);

}  // namespace kb
