/* oracle.h -- CPU restatement of the deterministic synchronous multilevel
 * schedule.  TEST INFRASTRUCTURE ONLY: the product library never links,
 * loads or calls anything in oracle/; only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg use it, as the checker.
 *
 * Every rule cites the reference function it restates (paths relative to the
 * KaHIP source tree).  The schedule (synchronous sub-rounds, hash tie-breaks,
 * sort-free admission) is this project's; the rules inside it are the
 * reference's.  Parity is pinned against the reference's own routines by the
 * tests through oracle/ref_harness.cpp (see tests/test_oracle_pins.py).
 */
#ifndef KB_ORACLE_H
#define KB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int n;
    const int* xadj;
    const int* adjncy;
    const int* adjwgt; /* never NULL here: callers expand unit weights */
    const int* vwgt;   /* never NULL here */
} or_graph;

/* Knobs of one partitioning call; or_derive_knobs fills them exactly as the
 * product's host code does (same field meanings). */
typedef struct {
    int k;
    double imbalance; /* fraction, as the kaffpa() ABI takes it */
    int seed;
    int mode;
    uint32_t total_weight;
    uint32_t upper_bound;   /* U, app/balance_configuration.h:40-47 */
    uint32_t final_bound;   /* U, or ceil(W/k) when imbalance == 0 */
    uint32_t num_stop;      /* stop_rules.h:49-50 */
    uint32_t max_vertex_weight; /* stop_rules.h:51-55 */
    uint32_t cluster_bound; /* strict bound of LP clustering */
    int lpc_rounds, lpc_subrounds;
    int ref_rounds, ref_subrounds, ref_classes;
    int bal_iters;
    int ip_reps, ip_tries, ip_fm_passes, ip_fm_stall;
    int max_levels;
    int coarsening;         /* 0 = LP clustering, 1 = heavy-edge matching (2, the learned
                               rating, is not restated here) */
    int match_rounds;       /* cap on locally-dominant matching rounds */
    const float* rating_model; /* unused by the oracle (same layout as the product's knobs) */
    double rating_fallback;    /* unused by the oracle */
    int rating_levels;         /* unused by the oracle */
    int refinement;            /* 0 = LP refinement, 1 = Jet refinement */
    int jet_iters, jet_patience, jet_c0, jet_c;
    int ip_mode;               /* 0 = multilevel recursive bisection with FM (host form),
                                  1 = batched recursive bisection (the device's form) */
    int ip_jet_iters, ip_jet_patience;  /* ip_mode 1: 2-way Jet per bisection try */
} or_knobs;

typedef struct {
    int levels;           /* number of graphs in the hierarchy (>= 1) */
    int level_n[64];
    long long level_m[64];
    long long level_cut[64];     /* cut after refinement at that level */
    uint32_t level_maxbw[64];
    long long initial_cut;       /* cut of the initial partition of the coarsest graph */
    int balanced;                /* 1 if max block weight <= final_bound */
} or_stats;

/* hashing (splitmix64 finaliser) -- identical on the device */
uint64_t or_mix64(uint64_t z);
uint64_t or_stream(int seed, int tag, int level, int round);
uint32_t or_hash(uint64_t stream, uint32_t x);

void or_derive_knobs(int n, const int* vwgt, int k, double imbalance, int seed, int mode,
                     or_knobs* out);

/* stop_rules.h:64-66 */
int or_stop_continue(const or_knobs* kn, int nf, int nc);

/* quality_metrics.cpp:23-37 and :265-288 */
long long or_edge_cut(const or_graph* g, const int* part);
void or_block_weights(const or_graph* g, const int* part, int k, uint32_t* bw);
double or_balance_ratio(const or_graph* g, const int* part, int k);

/* edge_ratings.cpp:171-183 */
void or_rate_expansion_star_2(const or_graph* g, double* rating);

/* Heavy-edge matching of one coarsening level: synchronous locally-dominant
 * rounds on a strict edge order (rating, edge hash, endpoints).  rating_q:
 * NULL = expansion*^2 (edge_ratings.cpp:171-183) computed per entry, else one
 * 32-bit rating per directed entry (symmetric).  Pairs obey
 * c(u)+c(v) <= max_vertex_weight (random_matching.cpp:85-112).
 * label[v] = min(v, mate(v)), or v when unmatched. */
void or_hem_match(const or_graph* g, const or_knobs* kn, int level, const uint32_t* rating_q, int* label);

/* Isolated vertices (degree 0) in increasing id order, in consecutive groups
 * of G = (bound-1) / (largest isolated node weight) (all of them when that
 * weight is 0), take the label of the group's first member; nothing happens
 * when G < 2 or fewer than two vertices are isolated.  label[] in/out. */
void or_bundle_isolated(const or_graph* g, uint32_t bound, int* label);

/* Jet refinement of one level (Gilbert et al. 2023, synchronous form; see
 * oracle.c): part[n] in/out, blocks kept at or below `bound`. */
void or_jet_refine(const or_graph* g, const or_knobs* kn, int level, uint32_t bound, int* part);

/* LP clustering, synchronous schedule (one coarsening level). label[n] out. */
void or_lp_cluster(const or_graph* g, const or_knobs* kn, int level, int* label);
/* LP clustering, sequential schedule in a given node order (pin mode):
 * size_constraint_label_propagation.cpp:134-194 then :207-232 (remap). */
int or_lp_cluster_seq(const or_graph* g, uint32_t bound, int rounds, const int* order, int* label);

/* contraction (leader = min member, rows sorted by target).
 * cxadj[n'+1], cadjncy/cadjwgt[m] capacity, cvwgt[n'], cmap[n].  Returns n'. */
int or_contract(const or_graph* g, const int* label, int* cmap, int* cxadj, int* cadjncy,
                int* cadjwgt, int* cvwgt);

/* LP refinement, synchronous schedule. part in/out. */
void or_lp_refine(const or_graph* g, const or_knobs* kn, int level, uint32_t bound, int* part);
/* label_propagation_refinement.cpp:21-98 in the reference's queue order (pin mode). */
void or_lp_refine_seq(const or_graph* g, int k, uint32_t bound, int rounds, const int* order,
                      int* part);

/* exact balance repair; returns 1 if every block ends <= bound */
int or_balance(const or_graph* g, const or_knobs* kn, int level, uint32_t bound, int* part);

/* initial partitioning of a (coarsest) graph into kn->k blocks */
/* batched recursive bisection: every bisection of a depth together (the
 * device's initial partitioner) */
void or_initial_partition_batched(const or_graph* g, const or_knobs* kn, int* part);
void or_initial_partition(const or_graph* g, const or_knobs* kn, int* part);

/* whole multilevel call, kaffpa() semantics (interface/kaHIP_interface.h:30-33).
 * vwgt/adjcwgt may be NULL (unit).  Returns 0 on success, <0 on invalid input. */
int or_kaffpa(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
              int nparts, double imbalance, int seed, int mode, long long* edgecut, int* part,
              or_stats* stats);
/* Same with explicit knobs (kn->k blocks). */
int or_kaffpa_knobs(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                    const or_knobs* kn, long long* edgecut, int* part, or_stats* stats);

/* KaFFPaE combine of two partitions of the same graph (population.cpp:189-250):
 * coarsening keeps every node pair that some parent separates apart, the
 * coarsest graph takes the better parent (by overload, then cut; part_a on
 * ties), and the result is never worse than that parent. */
int or_kaffpa_combine(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
                      const or_knobs* kn, const int* part_a, const int* part_b, long long* edgecut, int* part,
                      or_stats* stats);

/* KaFFPaE-style evolution on one process (parallel_mh_async.cpp:49-…,
 * population.cpp:120-173,358-369): `population` members from the plain
 * partitioner (seed + i), then `generations` rounds of `per_generation`
 * combines of tournament-selected pairs (all reading the population at the
 * round's start), each offspring inserted in order by the reference's rule.
 * part/edgecut: the best member; history[generations + 1] (optional): the
 * best cut after the initial population and after every round. */
int or_kaffpae(int n, const int* vwgt, const int* xadj, const int* adjcwgt, const int* adjncy,
               const or_knobs* kn, int population, int generations, int per_generation, long long* edgecut,
               int* part, long long* history);

#ifdef __cplusplus
}
#endif
#endif
