// knobs.cpp -- parameter derivation for one partitioning call.
#include "knobs.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace kb {

void derive_knobs(int n, const int* vwgt, int k, double imbalance, int seed, int mode, Knobs& kn) {
    // Total node weight as the reference accumulates it (NodeWeight is a
    // 32-bit unsigned, app/balance_configuration.h:20-23).
    uint32_t W = 0;
    if (vwgt) {
        for (int v = 0; v < n; ++v) W += (uint32_t)vwgt[v];
    } else {
        W = (uint32_t)n;
    }
    derive_knobs_total(n, W, k, imbalance, seed, mode, kn);
}

void derive_knobs_total(int n, uint32_t W, int k, double imbalance, int seed, int mode, Knobs& kn) {
    std::memset(&kn, 0, sizeof(kn));
    kn.k = k;
    kn.imbalance = imbalance;
    kn.seed = seed;
    kn.mode = mode;
    kn.total_weight = W;

    // kaffpa() turns the fraction into percent (interface/kaHIP_interface.cpp:115);
    // configurate_balance turns it back and truncates U to NodeWeight
    // (app/balance_configuration.h:40-47).  With imbalance 0 the reference
    // switches to "perfectly balanced" mode: U gets +1% slack for the
    // multilevel phases and the final result must fit ceil(W/k).
    const double pct = 100 * imbalance;
    const double eps = pct / 100.0;
    const double avg = std::ceil(W / (double)k);
    if (pct == 0) {
        kn.upper_bound = (uint32_t)((1 + eps + 0.01) * avg);
        kn.final_bound = (uint32_t)avg;
    } else {
        kn.upper_bound = (uint32_t)((1 + eps) * avg);
        kn.final_bound = kn.upper_bound;
    }

    // simple_stop_rule (stop_rules.h:46-56): coarsen while the graph keeps
    // at least max(n / (2*60*k), 60*k) nodes; coarse nodes stay below
    // 1.5 * W / num_stop.
    const double x = 60;
    kn.num_stop = (uint32_t)std::max(n / (2.0 * x * k), 60.0 * k);
    kn.max_vertex_weight = (uint32_t)(1.5 * W / kn.num_stop);

    // Cluster bound of size-constrained LP clustering, ceil(U / 18)
    // (size_constraint_label_propagation.cpp:57, cluster_coarsening_factor
    // app/configuration.h:422), tightened so coarse nodes respect the
    // max_vertex_weight of the fast/eco presets.  The test is strict (:175).
    uint32_t cb = (uint32_t)std::ceil(kn.upper_bound / 18.0);
    cb = std::min<uint32_t>(cb, kn.max_vertex_weight + 1u);
    kn.cluster_bound = cb;

    // Schedule knobs.  FAST/FASTSOCIAL use the cheap preset; everything else
    // (ECO, STRONG*, unknown modes -- which the reference maps to eco,
    // kaHIP_interface.cpp:60-61) the thorough one.
    const bool fast = mode == 0 || mode == 3;
    kn.lpc_rounds = fast ? 5 : 10;       // label_iterations = 10 (configuration.h:424)
    kn.lpc_subrounds = 2;                // later rounds: two sub-rounds (round 0 is one)
    kn.ref_rounds = fast ? 10 : 25;      // label_iterations_refinement = 25 (:425)
    kn.ref_subrounds = 2;
    kn.ref_classes = 16;
    kn.bal_iters = 64;
    kn.ip_reps = fast ? 1 : 2;
    kn.ip_tries = fast ? 4 : 16;         // bipartition_tries = 4 (fast/eco) at every level of
                                         // the reference's multilevel bisection; more growing
                                         // tries on one level here
    kn.ip_fm_passes = fast ? 3 : 6;
    kn.ip_fm_stall = 100;
    kn.max_levels = 48;
    kn.coarsening = 0;                   // LP clustering; 1 selects heavy-edge matching
    kn.match_rounds = 16;                // matching converges in < 10 rounds on meshes
    kn.rating_model = nullptr;
    kn.rating_fallback = 0.0;
    kn.rating_levels = 0;
    // Jet (this library's FM counterpart) wherever the reference runs FM-based
    // pair refinement: every mode but fast, and fast with k <= 8
    // (app/configuration.h:108-118 disables quotient-graph refinement above 8)
    kn.refinement = (fast && k > 8) ? 0 : 1;
    kn.jet_iters = 32;                   // Jet (Gilbert et al. 2023): patience 12, tolerance
    kn.jet_patience = 12;                // 0.25 of the own connection on the finest level,
    kn.jet_c0 = 1;                       // 0.75 on coarser ones
    kn.jet_c = 3;
    // initial partitioning on the device: every bisection of a recursion
    // depth in one launch (breadth-first growing, 2-way Jet refinement)
    kn.ip_mode = 1;
    // the bisection tries' 2-way Jet: 20 iterations, patience 8 (against 32 /
    // 12, on the oracle: final cut +0.04 % in geometric mean over RGG2D 2^15 /
    // 2^17, RGG3D 2^16, R-MAT 2^15 at k = 16 / 64 / 256, seeds 0-3, and
    // +0.00 % over RGG2D 2^21, RGG3D 2^20, k = 16 / 64 / 256, seeds 0-4;
    // 16 / 6 gave +0.09 % and +0.31 %)
    kn.ip_jet_iters = 20;
    kn.ip_jet_patience = 8;
}

}  // namespace kb
