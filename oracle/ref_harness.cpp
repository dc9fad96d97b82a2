// ref_harness.cpp -- test infrastructure, not product code.
//
// Exposes single functions of the reference KaHIP library (compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libkahip_ref.so) as
// plain extern "C" entry points, so the tests can pin the C oracle against
// the reference's own arithmetic: block upper bound, stop rule, edge rating,
// edge cut, balance, contraction, projection, and the sequential label
// propagation clustering / refinement on tie-free inputs.
//
// Every function copies the caller's CSR into a reference graph_access, calls
// the reference routine, and copies the result back out.  Nothing here is
// used by the product library.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "data_structure/graph_access.h"
#include "partition/partition_config.h"
#include "partition/coarsening/contraction.h"
#include "partition/coarsening/edge_rating/edge_ratings.h"
#include "partition/coarsening/clustering/size_constraint_label_propagation.h"
#include "partition/coarsening/clustering/node_ordering.h"
#include "partition/coarsening/stop_rules/stop_rules.h"
#include "partition/uncoarsening/refinement/label_propagation_refinement/label_propagation_refinement.h"
#include "partition/uncoarsening/refinement/quotient_graph_refinement/complete_boundary.h"
#include "io/graph_io.h"
#include "tools/quality_metrics.h"
#include "tools/random_functions.h"
#include "configuration.h"
#include "balance_configuration.h"

namespace {

void build(graph_access& G, int n, const int* xadj, const int* adjncy,
           const int* vwgt, const int* adjwgt) {
    G.build_from_metis(n, const_cast<int*>(xadj), const_cast<int*>(adjncy));
    if (vwgt) {
        for (int v = 0; v < n; ++v) G.setNodeWeight(v, vwgt[v]);
    }
    if (adjwgt) {
        for (int e = 0; e < xadj[n]; ++e) G.setEdgeWeight(e, adjwgt[e]);
    }
}

void set_mode(PartitionConfig& pc, int k, int mode) {
    configuration cfg;
    pc.k = k;
    switch (mode) {
        case 0: cfg.fast(pc); break;
        case 1: cfg.eco(pc); break;
        case 2: cfg.strong(pc); break;
        case 3: cfg.fastsocial(pc); break;
        case 4: cfg.ecosocial(pc); break;
        case 5: cfg.strongsocial(pc); break;
        default: cfg.eco(pc); break;
    }
}

void export_graph(graph_access& C, int* out_n, int* cxadj, int* cadjncy,
                  int* cadjwgt, int* cvwgt) {
    int nc = C.number_of_nodes();
    *out_n = nc;
    int pos = 0;
    for (int u = 0; u < nc; ++u) {
        cxadj[u] = pos;
        cvwgt[u] = (int)C.getNodeWeight(u);
        for (EdgeID e = C.get_first_edge(u); e < C.get_first_invalid_edge(u); ++e) {
            cadjncy[pos] = (int)C.getEdgeTarget(e);
            cadjwgt[pos] = C.getEdgeWeight(e);
            ++pos;
        }
    }
    cxadj[nc] = pos;
}

}  // namespace

extern "C" {

// interface/kaHIP_interface.cpp:146-166 (kaffpa) + app/balance_configuration.h:19-56
// + lib/partition/coarsening/stop_rules/stop_rules.h:46-66.
// Returns U, the simple stop rule's num_stop and max_vertex_weight for a graph
// with node weights vwgt (NULL = unit) partitioned into k blocks.
void ref_balance_config(int n, const int* vwgt, int k, double imbalance, int mode,
                        unsigned* upper_bound, unsigned* num_stop_out,
                        unsigned* max_vertex_weight) {
    std::vector<int> xadj(n + 1, 0);
    graph_access G;
    build(G, n, xadj.data(), nullptr, vwgt, nullptr);
    PartitionConfig pc;
    set_mode(pc, k, mode);
    pc.imbalance = 100 * imbalance;
    G.set_partition_count(k);
    balance_configuration bc;
    bc.configurate_balance(pc, G);
    *upper_bound = pc.upper_bound_partition;
    PartitionConfig copy = pc;
    simple_stop_rule rule(copy, n);
    // num_stop is private; recompute it with the same expression (stop_rules.h:49-50).
    double x = 60;
    *num_stop_out = (NodeID)std::max(n / (2.0 * x * pc.k), 60.0 * pc.k);
    *max_vertex_weight = copy.max_vertex_weight;
}

// stop_rules.h:64-66: does the coarsening loop continue after a level that
// went from nf to nc nodes?
int ref_stop_rule_continue(unsigned nf, unsigned nc, int n0, int k, unsigned work_load) {
    PartitionConfig pc;
    set_mode(pc, k, 0);
    pc.work_load = work_load;
    simple_stop_rule rule(pc, n0);
    return rule.stop(nf, nc) ? 1 : 0;
}

// lib/tools/quality_metrics.cpp:23-37
int ref_edge_cut(int n, const int* xadj, const int* adjncy, const int* adjwgt,
                 const int* part, int k) {
    graph_access G;
    build(G, n, xadj, adjncy, nullptr, adjwgt);
    G.set_partition_count(k);
    for (int v = 0; v < n; ++v) G.setPartitionIndex(v, part[v]);
    quality_metrics qm;
    return qm.edge_cut(G);
}

// lib/tools/quality_metrics.cpp:265-288
double ref_balance(int n, const int* xadj, const int* adjncy, const int* vwgt,
                   const int* part, int k) {
    graph_access G;
    build(G, n, xadj, adjncy, vwgt, nullptr);
    G.set_partition_count(k);
    for (int v = 0; v < n; ++v) G.setPartitionIndex(v, part[v]);
    quality_metrics qm;
    return qm.balance(G);
}

// lib/partition/coarsening/edge_rating/edge_ratings.cpp:171-183
void ref_rate_expansion_star_2(int n, const int* xadj, const int* adjncy,
                               const int* vwgt, const int* adjwgt, double* rating) {
    graph_access G;
    build(G, n, xadj, adjncy, vwgt, adjwgt);
    PartitionConfig pc;
    set_mode(pc, 2, 0);
    pc.edge_rating = EXPANSIONSTAR2;
    edge_ratings er(pc);
    er.rate(G, 10);  // level >= aggressive_random_levels so the rating is computed
    for (int e = 0; e < xadj[n]; ++e) rating[e] = G.getEdgeRating(e);
}

// size_constraint_label_propagation.cpp:207-232 (first-appearance relabel) +
// contraction.cpp:94-133 -> complete_boundary.h:511-562.
// cluster[] holds arbitrary cluster ids < n.  Outputs the coarse graph in the
// reference's own row order, and the fine->coarse map.
void ref_contract_clustering(int n, const int* xadj, const int* adjncy,
                             const int* vwgt, const int* adjwgt, const int* cluster,
                             int* out_nc, int* cxadj, int* cadjncy, int* cadjwgt,
                             int* cvwgt, int* cmap) {
    graph_access G;
    build(G, n, xadj, adjncy, vwgt, adjwgt);
    G.set_partition_count(2);
    PartitionConfig pc;
    set_mode(pc, 2, 3);
    pc.matching_type = CLUSTER_COARSENING;
    pc.combine = false;
    std::vector<NodeWeight> cid(cluster, cluster + n);
    NodeID nc = 0;
    size_constraint_label_propagation lp;
    lp.remap_cluster_ids(pc, G, cid, nc, false);
    CoarseMapping mapping(cid.begin(), cid.end());
    Matching matching(n);
    NodePermutationMap perm(n);
    for (int v = 0; v < n; ++v) { matching[v] = v; perm[v] = v; }
    graph_access C;
    contraction con;
    con.contract(pc, G, C, matching, mapping, nc, perm);
    export_graph(C, out_nc, cxadj, cadjncy, cadjwgt, cvwgt);
    for (int v = 0; v < n; ++v) cmap[v] = (int)mapping[v];
}

// contraction.cpp:21-92 with a matching; coarse ids in leader (first
// appearance) order as random_matching.cpp:104-110 assigns them.
// match[v] = partner (or v itself when unmatched); must be symmetric.
void ref_contract_matching(int n, const int* xadj, const int* adjncy,
                           const int* vwgt, const int* adjwgt, const int* match,
                           int* out_nc, int* cxadj, int* cadjncy, int* cadjwgt,
                           int* cvwgt, int* cmap) {
    graph_access G;
    build(G, n, xadj, adjncy, vwgt, adjwgt);
    G.set_partition_count(2);
    PartitionConfig pc;
    set_mode(pc, 2, 0);
    pc.matching_type = MATCHING_RANDOM;
    pc.combine = false;
    pc.graph_allready_partitioned = false;
    Matching matching(match, match + n);
    CoarseMapping mapping(n, 0);
    std::vector<char> seen(n, 0);
    NodeID nc = 0;
    for (int v = 0; v < n; ++v) {
        if (seen[v]) continue;
        seen[v] = 1;
        mapping[v] = nc;
        if (match[v] != v) { seen[match[v]] = 1; mapping[match[v]] = nc; }
        ++nc;
    }
    NodePermutationMap perm(n);
    for (int v = 0; v < n; ++v) perm[v] = v;
    graph_access C;
    contraction con;
    con.contract(pc, G, C, matching, mapping, nc, perm);
    export_graph(C, out_nc, cxadj, cadjncy, cadjwgt, cvwgt);
    for (int v = 0; v < n; ++v) cmap[v] = (int)mapping[v];
}

// node_ordering.h:43-48 -- the degree order the reference's label
// propagation visits nodes in (std::sort by degree; libstdc++ here).
void ref_degree_order(int n, const int* xadj, const int* adjncy, int* order) {
    graph_access G;
    build(G, n, xadj, adjncy, nullptr, nullptr);
    PartitionConfig pc;
    set_mode(pc, 2, 3);
    pc.node_ordering = DEGREE_NODEORDERING;
    std::vector<NodeID> perm(n);
    node_ordering no;
    no.order_nodes(pc, G, perm);
    for (int v = 0; v < n; ++v) order[v] = (int)perm[v];
}

// size_constraint_label_propagation.cpp:134-194 (+ remap :207-232).
// Deterministic only when no two candidate clusters of a node ever tie
// (the reference breaks ties with a global coin flip).
void ref_lp_cluster(int n, const int* xadj, const int* adjncy, const int* vwgt,
                    const int* adjwgt, unsigned block_upperbound, int iterations,
                    int* cluster_out, int* num_clusters) {
    graph_access G;
    build(G, n, xadj, adjncy, vwgt, adjwgt);
    PartitionConfig pc;
    set_mode(pc, 2, 3);
    pc.label_iterations = iterations;
    pc.node_ordering = DEGREE_NODEORDERING;
    pc.graph_allready_partitioned = false;
    pc.combine = false;
    random_functions::setSeed(0);
    std::vector<NodeWeight> cid(n);
    NodeID nb = 0;
    size_constraint_label_propagation lp;
    lp.label_propagation(pc, G, block_upperbound, cid, nb);
    for (int v = 0; v < n; ++v) cluster_out[v] = (int)cid[v];
    *num_clusters = (int)nb;
}

// label_propagation_refinement.cpp:21-98.  part[] is updated in place.
// Deterministic only on tie-free inputs (see ref_lp_cluster).
void ref_lp_refine(int n, const int* xadj, const int* adjncy, const int* vwgt,
                   const int* adjwgt, int k, unsigned upper_bound, int iterations,
                   int* part) {
    graph_access G;
    build(G, n, xadj, adjncy, vwgt, adjwgt);
    G.set_partition_count(k);
    for (int v = 0; v < n; ++v) G.setPartitionIndex(v, part[v]);
    PartitionConfig pc;
    set_mode(pc, k, 3);
    pc.k = k;
    pc.upper_bound_partition = upper_bound;
    pc.label_iterations_refinement = iterations;
    pc.node_ordering = DEGREE_NODEORDERING;
    random_functions::setSeed(0);
    complete_boundary boundary(&G);
    label_propagation_refinement lpr;
    lpr.perform_refinement(pc, G, boundary);
    for (int v = 0; v < n; ++v) part[v] = (int)G.getPartitionIndex(v);
}

// graph_io::readGraphWeighted (lib/io/graph_io.cpp:82-191).  First call with
// null arrays returns n and the entry count; the second call fills them.
int ref_read_metis(const char* path, int* n, long long* m, int* xadj, int* adjncy, int* adjwgt, int* vwgt) {
    graph_access G;
    if (graph_io::readGraphWeighted(G, path) != 0) return -1;
    *n = (int)G.number_of_nodes();
    *m = (long long)G.number_of_edges();
    if (!xadj) return 0;
    int e = 0;
    for (int v = 0; v < *n; ++v) {
        xadj[v] = e;
        vwgt[v] = (int)G.getNodeWeight(v);
        for (EdgeID x = G.get_first_edge(v); x < G.get_first_invalid_edge(v); ++x) {
            adjncy[e] = (int)G.getEdgeTarget(x);
            adjwgt[e] = (int)G.getEdgeWeight(x);
            ++e;
        }
    }
    xadj[*n] = e;
    return 0;
}

}  // extern "C"
