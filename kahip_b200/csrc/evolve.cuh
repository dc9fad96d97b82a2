// evolve.cuh -- KaFFPaE-style evolutionary partitioning on one device (evolve.cu).
#pragma once

#include <vector>

#include "lp.cuh"

namespace kb {

// population members from the plain partitioner (seed + i), then
// `generations` rounds of `per_generation` combines of tournament-selected
// pairs, offspring inserted by the reference's rule; d_best (n, device) and
// *edgecut: the best member; history[generations + 1] (host, optional): the
// best cut after the initial population and after every round.
// Returns KB_OK or KB_WARN_IMBALANCED (for the best member).
// The members and each round's combines run concurrently, one host thread
// per worker context (same device as ctx, which holds g0); results do not
// depend on the number of workers.
int kaffpae(Ctx& ctx, const std::vector<Ctx*>& workers, const DevGraph& g0, const Knobs& kn, int population,
            int generations, int per_generation, int* d_best, long long* edgecut, long long* history);

}  // namespace kb
