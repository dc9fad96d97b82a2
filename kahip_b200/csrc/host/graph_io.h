// graph_io.h -- graph and partition files on the host (graph_io.cpp).
#pragma once

#include <string>
#include <vector>

namespace kb {

// Host CSR with explicit weights (unit weights filled in).
struct HostCSR {
    int n = 0;
    long long m = 0;
    std::vector<int> xadj, adjncy, adjwgt, vwgt;
};

// METIS text format (lib/io/graph_io.cpp:82-191); 0 on success, else -1
// with err set.
int read_metis(const char* path, HostCSR& g, std::string& err);

// ParHIP binary format, version 3 (parallel_graph_io.cpp:474-594).
int read_bgf(const char* path, HostCSR& g, std::string& err);

// One block id per line (graph_io::writePartition).
int write_partition(const char* path, int n, const int* part, std::string& err);

}  // namespace kb
