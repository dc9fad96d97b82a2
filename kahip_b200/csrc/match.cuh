// match.cuh -- heavy-edge matching coarsening (match.cu).
#pragma once

#include "lp.cuh"

namespace kb {

// Heavy-edge matching of one coarsening level by synchronous
// locally-dominant rounds: every unmatched vertex points at its best
// eligible neighbour under a strict edge order (rating, pair hash, endpoint
// sum); mutual pointers match.  Eligible: both unmatched, v != u and
// c(v) + c(u) <= max_vertex_weight (random_matching.cpp:85-112).  The rating
// is expansion*^2 (edge_ratings.cpp:171-183), or rating_q[e] (one 32-bit
// value per directed entry, symmetric) when rating_q != nullptr.  Stops after
// a round without a new pair or after kn.match_rounds rounds.
// label[v] (device, out) = min(v, mate(v)), or v when unmatched.
void hem_match(Ctx& ctx, const DevGraph& g, const Knobs& kn, int level, const uint32_t* rating_q, int* label);

}  // namespace kb
