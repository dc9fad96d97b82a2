/* kahip_b200.h -- extended C ABI of the B200 KaFFPa library (libkahip_b200.so).
 *
 * The drop-in entry point kaffpa() and its siblings are declared in
 * kaHIP_interface.h with the reference's exact signatures.  This header adds
 * status-returning variants, a device-pointer variant, and one entry point
 * per phase of the multilevel scheme so that each phase can be checked
 * against the CPU oracle.  Plain pointers and sizes only.
 *
 * Conventions: graphs are METIS-style int32 CSR (xadj[n+1], adjncy[xadj[n]],
 * optional adjwgt[xadj[n]] and vwgt[n]; NULL = unit weights), symmetric,
 * 0-based, no self loops.  Host-pointer entry points copy to the current CUDA
 * device and back.  Every int-returning call returns 0 on success, a negative
 * kb200 status on failure (kb200_last_error() describes it), or
 * KB200_WARN_IMBALANCED when a partition was produced but a block exceeds the
 * bound.
 */
#ifndef KAHIP_B200_H
#define KAHIP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KB200_OK 0
#define KB200_ERR_INVALID_INPUT (-1)
#define KB200_ERR_CUDA (-2)
#define KB200_ERR_NO_DEVICE (-3)
#define KB200_ERR_OUT_OF_MEMORY (-4)
#define KB200_ERR_INTERNAL (-5)
#define KB200_WARN_IMBALANCED 1

/* Parameters of one call.  kb200_derive_knobs() fills them from
 * (n, vwgt, k, imbalance, seed, mode) following
 *   app/balance_configuration.h:19-56   (upper_bound, total_weight),
 *   lib/partition/coarsening/stop_rules/stop_rules.h:46-66 (num_stop,
 *                                         max_vertex_weight),
 *   size_constraint_label_propagation.cpp:57 (cluster_bound),
 *   app/configuration.h:83-134          (fast / eco presets). */
typedef struct kb200_knobs {
    int k;
    double imbalance;          /* fraction, as kaffpa() takes it */
    int seed;
    int mode;                  /* FAST=0 ECO=1 STRONG=2 FASTSOCIAL=3 ECOSOCIAL=4 STRONGSOCIAL=5 */
    uint32_t total_weight;
    uint32_t upper_bound;      /* U = (1+eps)*ceil(W/k), truncated */
    uint32_t final_bound;      /* U, or ceil(W/k) when imbalance == 0 */
    uint32_t num_stop;
    uint32_t max_vertex_weight;
    uint32_t cluster_bound;    /* strict bound on cluster weight during coarsening */
    int lpc_rounds, lpc_subrounds;                 /* clustering */
    int ref_rounds, ref_subrounds, ref_classes;    /* refinement */
    int bal_iters;                                 /* balance repair */
    int ip_reps, ip_tries, ip_fm_passes, ip_fm_stall; /* initial partitioning */
    int max_levels;
    int coarsening;            /* 0 = LP clustering (default), 1 = heavy-edge matching on
                                  expansion*^2, 2 = heavy-edge matching on the learned rating */
    int match_rounds;          /* cap on locally-dominant matching rounds per level */
    const float* rating_model; /* coarsening 2: host array of KB200_RATING_PARAMS floats
                                  (NULL = fall back to expansion*^2) */
    double rating_fallback;    /* coarsening 2: > 0 also runs the expansion*^2 matching and
                                  keeps it when learned cut > rating_fallback * its cut */
    int rating_levels;         /* coarsening 2: levels 0 .. rating_levels-1 use the learned
                                  rating, deeper ones expansion*^2 (<= 0: every level) */
    int refinement;            /* 0 = LP refinement (default), 1 = Jet refinement */
    int jet_iters, jet_patience;  /* Jet: iteration cap, iterations without a better cut */
    int jet_c0, jet_c;         /* Jet: negative-gain tolerance in quarters of the own
                                  connection, finest level / coarser levels */
    int ip_mode;               /* initial partitioning of the coarsest graph: 1 = on the
                                  device, every bisection of a recursion depth in one launch
                                  (default); 0 = the host's multilevel bisection with FM */
    int ip_jet_iters, ip_jet_patience;  /* ip_mode 1: the 2-way Jet of every bisection try:
                                  iteration cap, iterations without a better state */
} kb200_knobs;

/* Parameter count of the learned edge rating (kahip_b200/csrc/learned.cuh). */
#define KB200_RATING_PARAMS 27137

/* Per-call report.  level 0 is the input graph. */
typedef struct kb200_stats {
    int levels;
    int level_n[64];
    long long level_m[64];
    long long level_cut[64];       /* cut after refinement (filled when collect_level_cuts) */
    uint32_t level_maxbw[64];
    long long initial_cut;         /* cut of the initial partition of the coarsest graph */
    int balanced;                  /* final max block weight <= final_bound */
    /* inputs to the report */
    int collect_level_cuts;        /* in: 1 = compute the cut at every level */
    int timing;                    /* in: 1 = time every kernel family with CUDA events,
                                      2 = only the LP clustering sweep (lp_cluster_sweep) */
    /* timings (milliseconds) */
    double ms_total;               /* wall time of the call on the host */
    double ms_h2d, ms_coarsen, ms_initial, ms_uncoarsen, ms_d2h;
    /* kernel families (timing 1 or 2): device ms, algorithmic bytes, launches */
    int nfamilies;
    char family_name[32][24];
    double family_ms[32];
    double family_bytes[32];
    long long family_launches[32];
    /* LP sweep work actually performed */
    long long sweep_vertices, sweep_edges;
    long long sweep_overflow_vertices;   /* of which needed the shared-table path */
    size_t device_bytes_peak;
    int rating_fallback_used;  /* coarsening 2 with rating_fallback: 1 = the expansion*^2
                                  partition was returned */
} kb200_stats;

int kb200_derive_knobs(int n, const int* vwgt, int k, double imbalance, int seed, int mode,
                       kb200_knobs* out);

/* Whole multilevel partitioning with host buffers (kaffpa() semantics,
 * interface/kaHIP_interface.h:30-33) plus status and report. */
int kb200_kaffpa(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                 int nparts, double imbalance, int seed, int mode, long long* edgecut, int* part,
                 kb200_stats* stats);

/* Same with device buffers on the current device; part is a device array.
 * stream: a cudaStream_t (NULL = a stream owned by the library). */
int kb200_kaffpa_device(int n, const int* d_vwgt, const int* d_xadj, const int* d_adjcwgt,
                        const int* d_adjncy, int nparts, double imbalance, int seed, int mode,
                        long long* edgecut, int* d_part, void* stream, kb200_stats* stats);

/* Whole partitioning with explicit knobs (kb200_derive_knobs() output,
 * possibly edited: coarsening, round counts ...); kn->k blocks. */
int kb200_kaffpa_knobs(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                       const kb200_knobs* kn, long long* edgecut, int* part, kb200_stats* stats);

/* KaFFPaE combine operator (replaces population::combine,
 * lib/parallel_mh/population.cpp:189-250, which has no C entry point in the
 * reference): part_a and part_b are two partitions of the graph into kn->k
 * blocks.  The better one by (overload against the final bound, cut; part_a
 * on ties) becomes the initial partition of a multilevel run whose
 * coarsening never joins nodes that either parent separates; part[] out is
 * never worse than that parent. */
int kb200_kaffpa_combine(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                         const kb200_knobs* kn, const int* part_a, const int* part_b, long long* edgecut, int* part,
                         kb200_stats* stats);

/* KaFFPaE-style evolutionary partitioning on one device (replaces the
 * kaffpaE program's loop, lib/parallel_mh/parallel_mh_async.cpp:49-…, with
 * population.cpp:120-173 insertion and :358-369 tournament selection; the
 * reference has no C entry point for it).  `population` members come from
 * the plain partitioner with seeds kn->seed + i; each of `generations`
 * rounds combines `per_generation` tournament-selected pairs (deterministic
 * hash draws; every selection of a round reads the population at the
 * round's start) with kb200_kaffpa_combine's operator and inserts the
 * offspring in order.  part[]/edgecut: the best member by (overload, cut);
 * history[generations + 1] (optional): the best cut after the initial
 * population and after every round.  workers: concurrent partitionings on
 * the device (0 = min(per_generation, 4)); results do not depend on it. */
int kb200_kaffpae(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                  const kb200_knobs* kn, int population, int generations, int per_generation, int workers,
                  long long* edgecut, int* part, long long* history);

/* Same with device buffers (explicit weights), like kb200_kaffpa_device. */
int kb200_kaffpa_device_knobs(int n, const int* d_vwgt, const int* d_xadj, const int* d_adjcwgt,
                              const int* d_adjncy, const kb200_knobs* kn, long long* edgecut, int* d_part,
                              void* stream, kb200_stats* stats);

/* ---- batches: many independent calls on one device ----
 * Each worker thread leases its own context and stream; items are taken
 * largest first.  Every item's result equals a single call with the same
 * arguments.  workers <= 0 picks min(count, 8, host threads) (8 measured
 * fastest on a 512-graph batch; results do not depend on it). */
typedef struct kb200_batch_item {
    int n;                     /* in: host CSR graph (NULL weights = unit) */
    const int* xadj;
    const int* adjncy;
    const int* adjwgt;
    const int* vwgt;
    int nparts;                /* in: kaffpa() parameters of this item */
    double imbalance;
    int seed;
    int mode;
    int* part;                 /* out: caller-allocated n ints */
    long long edgecut;         /* out: -1 when the item failed */
    int status;                /* out: kb200 status of this item */
} kb200_batch_item;

typedef struct kb200_batch_report {
    int workers;               /* concurrent workers used */
    int failed;                /* items with a negative status */
    double ms_total;           /* wall time of the batch on the host */
} kb200_batch_report;

/* Independent graphs, host buffers (KaFFPaE-style populations of several
 * graphs, parameter sweeps).  Returns 0 when every item succeeded, else the
 * first failing item's status. */
int kb200_kaffpa_batch(kb200_batch_item* items, int count, int workers, kb200_batch_report* report);

/* One device-resident graph, `count` seeds (a KaFFPaE-style population;
 * lib/parallel_mh/parallel_mh_async.cpp:49-54 gives each member its own
 * seed).  d_parts: count * n device ints, member i at d_parts + i*n;
 * cuts[count] host out. */
int kb200_kaffpa_population(int n, const int* d_vwgt, const int* d_xadj, const int* d_adjcwgt,
                            const int* d_adjncy, int nparts, double imbalance, int mode, const int* seeds,
                            int count, long long* cuts, int* d_parts, int workers,
                            kb200_batch_report* report);

/* ---- learned edge rating (no counterpart in the reference) ----
 * A 3-layer message-passing network (hidden 64, BF16 weights and
 * activations, FP32 accumulation) predicting per directed entry the
 * probability p that a partition cuts the edge; the matching rating is
 * floor((1 - p) * 2^24).  params: KB200_RATING_PARAMS host floats. */

/* prob[m] / rating[m] out (either may be NULL); use_tc = 1 runs the layer
 * GEMMs on the tensor cores (tcgen05), 0 on the CUDA cores. */
int kb200_rating_infer(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                       const float* params, int use_tc, float* prob, uint32_t* rating);

/* One training graph: host CSR (explicit weights) and one 0/1 label per
 * directed entry (1 = cut). */
typedef struct kb200_train_graph {
    int n;
    const int* xadj;
    const int* adjncy;
    const int* adjwgt;
    const int* vwgt;
    const uint8_t* label;
} kb200_train_graph;

/* Adam on the weighted BCE of the labels, one graph per step (round robin):
 * params in/out (host), loss[steps] out (host, may be NULL). */
int kb200_rating_train(const kb200_train_graph* graphs, int count, int steps, float lr, float* params,
                       float* loss);

/* Loss and gradient of one graph at params (host out: grad[KB200_RATING_PARAMS], *loss). */
int kb200_rating_grad(const kb200_train_graph* graph, const float* params, float* grad, float* loss);

/* ---- phases (host buffers), for parity checks against the CPU oracle ---- */

/* Heavy-edge matching of one coarsening level (replaces random_matching.cpp:
 * 20-116 / gpa_matching.cpp:25-129): label[n] out = min(v, mate(v)) or v.
 * rating: NULL = expansion*^2 (edge_ratings.cpp:171-183); else one 32-bit
 * rating per directed entry (must be symmetric), larger = match first. */
int kb200_hem_match(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                    const kb200_knobs* kn, int level, const uint32_t* rating, int* label);

/* LP clustering of one coarsening level: label[n] out. */
int kb200_lp_cluster(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                     const kb200_knobs* kn, int level, int* label);

/* Contraction of a clustering.  Outputs: nc, mc, cmap[n], cxadj[nc+1],
 * cadjncy/cadjwgt[mc] (capacity xadj[n]), cvwgt[nc] (capacity n). */
int kb200_contract(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                   const int* label, int* nc, long long* mc, int* cmap, int* cxadj, int* cadjncy,
                   int* cadjwgt, int* cvwgt);

/* LP refinement at one level: part[n] in/out. */
int kb200_lp_refine(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                    const kb200_knobs* kn, int level, uint32_t bound, int* part);

/* Jet refinement at one level (stands in for the reference's k-way FM,
 * kway_graph_refinement_core.cpp:47-171): part[n] in/out. */
int kb200_jet_refine(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                     const kb200_knobs* kn, int level, uint32_t bound, int* part);

/* Balance repair: part[n] in/out; *balanced = 1 if every block <= bound. */
int kb200_balance(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                  const kb200_knobs* kn, int level, uint32_t bound, int* part, int* balanced);

/* Edge cut and block weights (bw[k], may be NULL) of a partition. */
int kb200_edge_cut(int n, const int* xadj, const int* adjncy, const int* adjwgt, const int* vwgt,
                   const int* part, int k, long long* cut, uint32_t* bw);

/* Projection part_fine[v] = part_coarse[cmap[v]]. */
int kb200_project(int n, const int* cmap, int nc, const int* part_coarse, int* part_fine);

/* Host initial partitioner (recursive multilevel bisection) of a small graph. */
int kb200_initial_partition(int n, const int* xadj, const int* adjncy, const int* adjwgt,
                            const int* vwgt, const kb200_knobs* kn, int* part);

/* The device initial partitioner (every bisection of a recursion depth in one
 * launch; initial_partitioning.cpp:39-134 -> graph_partitioner.cpp:110-238 is
 * the reference's counterpart) on a host graph: uploads it, partitions it
 * into kn->k blocks and downloads part[n].  kn->ip_mode is ignored. */
int kb200_initial_partition_device(int n, const int* xadj, const int* adjncy, const int* adjwgt,
                                   const int* vwgt, const kb200_knobs* kn, int* part);

/* Edge cut and block weights of a device-resident partition, computed
 * without allocating anything.  No counterpart in the reference (which has no
 * device code); it exists for callers that must not call cudaMalloc while
 * they run (fixed device-memory budgets, allocator-free sections, device
 * memory owned by another runtime).  All arrays are device pointers on the
 * current device (adjwgt / vwgt may be NULL = unit weights); *d_cut and
 * d_bw[k] are written asynchronously on `stream` (a cudaStream_t, NULL = the
 * default stream).  xadj must be a valid CSR offset array (xadj[0] = 0,
 * monotone, xadj[n] <= the length of adjncy): the device cannot see the
 * length of adjncy.  *d_cut = -1 if a block id is outside [0, k), a row
 * runs backwards, a target is outside [0, n) or a weight is negative (the
 * inputs the other entry points reject).
 * Limits: k <= 65536 (larger k returns KB200_ERR_INVALID_INPUT).  Its working
 * memory is one 256 KiB __device__ array held by every GPU that loads the
 * library until exit and shared by all calls: calls that overlap on the GPU
 * race and give wrong results.  The first call in a CUDA context looks up
 * that array's address, so make it before any stream capture begins; after
 * cudaDeviceReset the looked-up address may be stale, so do not call it
 * again in a process that reset its device. */
int kb200_edge_cut_noalloc(int n, const int* d_xadj, const int* d_adjncy, const int* d_adjwgt,
                           const int* d_vwgt, const int* d_part, int k, long long* d_cut, uint32_t* d_bw,
                           void* stream);

/* ---- graph and partition files (host; no counterpart needed on the device) ----
 * kb200_read_metis: METIS text format as the reference reads it
 * (lib/io/graph_io.cpp:82-191: header "n m [fmt]", fmt 1/10/11 = edge /
 * node / both weights, 1-based targets, '%' comments); parsed in parallel.
 * kb200_read_bgf: ParHIP binary graph, version 3 (parallel_graph_io.cpp:
 * 474-594).  Both return 0 and library-allocated arrays (unit weights
 * filled in; release each with kb200_free), or -1 (kb200_io_error() says
 * why; self-loops and miscounted nodes/edges are errors).
 * kb200_write_partition: one block id per line (graph_io::writePartition). */
int kb200_read_metis(const char* path, int* n, long long* m, int** xadj, int** adjncy, int** adjwgt, int** vwgt);
int kb200_read_bgf(const char* path, int* n, long long* m, int** xadj, int** adjncy, int** adjwgt, int** vwgt);
int kb200_write_partition(const char* path, int n, const int* part);
void kb200_free(void* p);
const char* kb200_io_error(void);

/* Last error message of the calling thread ("" if none). */
const char* kb200_last_error(void);

/* Number of kernels this library has launched so far (process-wide). */
long long kb200_kernel_launches(void);

/* Number of CUDA devices visible (0 when none). */
int kb200_device_count(void);

#ifdef __cplusplus
}
#endif
#endif
