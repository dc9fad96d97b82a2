// initial_partitioning.h -- host initial partitioner of the coarsest graph.
#pragma once

#include "../knobs.h"

namespace kb {

// Partitions the (small) graph into kn.k blocks; part[n] out.  All arrays
// are host memory; adjwgt and vwgt must be non-null.
void initial_partition(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                       const Knobs& kn, int* part);

// Caps, for calls made by the calling thread, the depth of the bisection
// tree down to which the two halves run on separate host threads (0 = no
// extra threads; -1 = derived from the host's core count).  Results do not
// depend on it.
void set_ip_thread_limit(int depth);

}  // namespace kb
