// ip_device.cuh -- initial partitioning of the coarsest graph on the device
// (ip_device.cu).
#pragma once

#include "lp.cuh"

namespace kb {

// Recursive bisection of the device graph c into kn.k blocks, every
// bisection of a recursion depth in one launch; part[c.n] (device) out.
// kn.ip_reps repetitions, the one of the smallest cut kept (the first on
// ties).  Synchronises the context's stream before returning.
void initial_partition_device(Ctx& ctx, const DevGraph& c, const Knobs& kn, int* part);

}  // namespace kb
