// partitioner.cuh -- the multilevel driver (partitioner.cu).
#pragma once

#include "lp.cuh"

namespace kb {

// Reserves both arenas for a graph of n nodes and m directed entries
// (copy_input: the level-0 graph is copied into the hierarchy arena).
void reserve_for(Ctx& ctx, int n, long long m, bool copy_input, double factor);

// Partitions the device graph g0 (level 0) into kn.k blocks; d_part[n] out.
// Returns KB_OK or KB_WARN_IMBALANCED.  Throws CudaError on CUDA failures
// (including an exhausted arena, which the caller answers with a larger
// reservation).  With host_part (page-locked, n ints), the final partition
// may also be copied there on the copy stream, overlapped with the last cut
// computation; *host_done tells whether it was (complete on return).
int partition(Ctx& ctx, const DevGraph& g0, const Knobs& kn, int* d_part, long long* edgecut,
              kb200_stats* st, int* host_part = nullptr, bool* host_done = nullptr);

// (overload against bound, cut) of the device partition part of g.
void partition_quality(Ctx& ctx, const DevGraph& g, const int* part, int k, uint32_t bound, uint64_t* ov,
                       long long* cut);

// KaFFPaE combine of the device partitions pa and pb of g0 (population.cpp:
// 189-250): the better parent by (overload, cut) (pa on ties) is the initial
// partition of a coarsening that keeps both parents' blocks apart; the
// result (d_part) is never worse than that parent.  Same returns as partition.
int combine(Ctx& ctx, const DevGraph& g0, const Knobs& kn, const int* pa, const int* pb, int* d_part,
            long long* edgecut, kb200_stats* st);

}  // namespace kb
