// knobs.h -- the parameters of one partitioning call, derived from
// (n, node weights, k, imbalance, seed, mode) exactly as the reference's
// presets and balance configuration derive theirs.
#pragma once

#include <cstdint>

extern "C" {
#include "../../include/kahip_b200.h"
}

namespace kb {

using Knobs = kb200_knobs;

// Fills kn; see knobs.cpp for the reference lines each value follows.
void derive_knobs(int n, const int* vwgt, int k, double imbalance, int seed, int mode, Knobs& kn);

// Same, from the node weight sum W (accumulated as a 32-bit unsigned).
void derive_knobs_total(int n, uint32_t W, int k, double imbalance, int seed, int mode, Knobs& kn);

}  // namespace kb
