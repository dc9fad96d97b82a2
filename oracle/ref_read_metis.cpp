// ref_read_metis.cpp -- test infrastructure, not product code.
//
// Reads a METIS graph file with the reference's own reader
// (graph_io::readGraphWeighted, through ref_harness.cpp) and writes the CSR
// to a binary file: int32 n, int64 m, then xadj[n+1], adjncy[m], adjwgt[m],
// vwgt[n] as int32.  A separate program so that the reference's iostreams
// run with the C++ runtime it was built against.
//
//     ref_read_metis <graph file> <output file>
#include <cstdio>
#include <vector>

extern "C" int ref_read_metis(const char* path, int* n, long long* m, int* xadj, int* adjncy, int* adjwgt,
                              int* vwgt);

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    int n = 0;
    long long m = 0;
    if (ref_read_metis(argv[1], &n, &m, nullptr, nullptr, nullptr, nullptr) != 0) return 1;
    std::vector<int> x(n + 1), a(m), w(m), v(n);
    if (ref_read_metis(argv[1], &n, &m, x.data(), a.data(), w.data(), v.data()) != 0) return 1;
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 1;
    std::fwrite(&n, sizeof n, 1, f);
    std::fwrite(&m, sizeof m, 1, f);
    std::fwrite(x.data(), sizeof(int), x.size(), f);
    std::fwrite(a.data(), sizeof(int), a.size(), f);
    std::fwrite(w.data(), sizeof(int), w.size(), f);
    std::fwrite(v.data(), sizeof(int), v.size(), f);
    return std::fclose(f) == 0 ? 0 : 1;
}
