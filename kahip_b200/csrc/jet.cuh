// jet.cuh -- Jet refinement (jet.cu).
#pragma once

#include "lp.cuh"

namespace kb {

// Jet refinement of one level (synchronous form of Gilbert et al. 2023,
// restated by the oracle's or_jet_refine): part[n] in/out, bw[k] in/out
// (device).  The best partition by (overload, cut) over the iterations is
// kept; blocks above `bound` are repaired by balance() after each move step.
void jet_refine(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, uint32_t bound, int* part, uint32_t* bw);

}  // namespace kb
