// initial_partitioning.h -- host initial partitioner of the coarsest graph.
#pragma once

#include "../knobs.h"

namespace kb {

// Partitions the (small) graph into kn.k blocks; part[n] out.  All arrays
// are host memory; adjwgt and vwgt must be non-null.
void initial_partition(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                       const Knobs& kn, int* part);

// For calls made by the calling thread: 0 runs the partitioner on that
// thread alone; any other value (default -1) lets repetitions, bisection
// halves and tries run on the process-wide host thread pool.  Results do not
// depend on it.
void set_ip_thread_limit(int depth);

}  // namespace kb
