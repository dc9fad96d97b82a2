/* kaHIP_interface.h -- drop-in declarations of the KaHIP C interface as
 * exported by libkahip_b200.so.
 *
 * Each declaration has the signature of its counterpart in the reference's
 * interface/kaHIP_interface.h so that existing callers (C/C++, the pybind11
 * module misc/pymodule/kahip.cpp, the JNI wrapper misc/java_jni_wrapper)
 * link against this library unchanged:
 *   kaffpa             interface/kaHIP_interface.h:30-33  (GPU multilevel path)
 *   kaffpa_balance     interface/kaHIP_interface.h:36-41  (both flag values: max block <= (1+eps)*ceil(W/k))
 *   kaffpa_balance_NE  interface/kaHIP_interface.h:44-47  (not provided: edgecut = -1)
 *   process_mapping    interface/kaHIP_interface.h:52-58  (not provided: edgecut = qap = -1)
 *   node_separator     interface/kaHIP_interface.h:61-64  (not provided)
 *   reduced_nd         interface/kaHIP_interface.h:68-70  (not provided)
 *   edge_partitioning  interface/kaHIP_interface.h:72-75  (not provided)
 * Mode constants keep the reference's values (interface/kaHIP_interface.h:17-22).
 */
#ifndef KAHIP_B200_INTERFACE_H
#define KAHIP_B200_INTERFACE_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

static const int FAST = 0;
static const int ECO = 1;
static const int STRONG = 2;
static const int FASTSOCIAL = 3;
static const int ECOSOCIAL = 4;
static const int STRONGSOCIAL = 5;

static const int MAPMODE_MULTISECTION = 0;
static const int MAPMODE_BISECTION = 1;

/* Metis-style CSR in; *edgecut and part[n] (caller-allocated) out.
 * vwgt / adjcwgt may be NULL (unit weights); imbalance is a fraction. */
void kaffpa(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
            bool suppress_output, int seed, int mode, int* edgecut, int* part);

void kaffpa_balance(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                    bool perfectly_balance, bool suppress_output, int seed, int mode, int* edgecut, int* part);

void kaffpa_balance_NE(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                       bool suppress_output, int seed, int mode, int* edgecut, int* part);

void process_mapping(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* hierarchy_parameter,
                     int* distance_parameter, int hierarchy_depth, int mode_partitioning, int mode_mapping,
                     double* imbalance, bool suppress_output, int seed, int* edgecut, int* qap, int* part);

void node_separator(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                    bool suppress_output, int seed, int mode, int* num_separator_vertices, int** separator);

void reduced_nd(int* n, int* xadj, int* adjncy, bool suppress_output, int seed, int mode, int* ordering);

#ifdef __cplusplus
void edge_partitioning(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                       bool suppress_output, int seed, int mode, int* vertexcut, int* part,
                       int infinity_edge_weight = 1000);
#else
void edge_partitioning(int* n, int* vwgt, int* xadj, int* adjcwgt, int* adjncy, int* nparts, double* imbalance,
                       bool suppress_output, int seed, int mode, int* vertexcut, int* part,
                       int infinity_edge_weight);
#endif

#ifdef __cplusplus
}
#endif

#endif
