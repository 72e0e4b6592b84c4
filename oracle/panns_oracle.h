/* CPU oracle for the PANNS search path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's query-time search, used by tests/,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline leg, to check results.
 * The product never links, loads or calls it.
 *
 * Parity is pinned against the reference itself: the binaries built by
 * oracle/Makefile from the reference sources (oracle/_ref/) and the committed
 * fixtures under tests/golden/ (see tests/golden/make_golden.py).
 *
 * Graph: CSR, offsets[N+1] (u64) into nbrs (u32). Data: N x d float32 rows.
 * Every search returns K ids per query (row-major nq x K) and the number of
 * distance computations (the reference's count_distance_computation_).
 */
#ifndef PANNS_ORACLE_H
#define PANNS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { PO_DIST_IP_NORM = 0, PO_DIST_L2 = 1 };

/* ||v||^2 in the reference's 8-lane order. */
float po_norm(const float *v, int d, int fused);
/* ||v||^2 - 2<v,q> (norm trick) or sum (v-q)^2, reference lane order. */
float po_distance(const float *v, const float *q, float norm, int d, int kind, int fused);

/* Selects whether multiply+add pairs in the lane accumulators are fused (FMA),
 * Default 1: the reference built with its own flags (-O3 -march=native)
 * fuses every lane step into one FMA (one rounding); a generically tuned
 * build keeps them separate (fused = 0). */
void po_set_fused(int fused);

/* PANNS prepare_init_ids: entry's neighbours (deduplicated), then entry+1,
 * entry+2, ... with wrap-around, until L ids. */
int po_prepare_init_ids(const uint64_t *offsets, const uint32_t *nbrs, uint32_t n,
                        uint32_t entry, uint32_t L, uint32_t *out);

/* glibc rand() (TYPE_3 additive feedback generator), self-contained. */
typedef struct { int32_t tbl[31]; int32_t *fptr; int32_t *rptr; } po_rand_state;
uint32_t po_rand_state_size(void);
void po_srand(po_rand_state *s, uint32_t seed);
int32_t po_rand(po_rand_state *s);

/* efanna2e init ids for nq consecutive queries: entry's first min(L, deg)
 * neighbours, then rand() % n until L distinct; the rand() stream continues
 * across queries. out: nq x L. */
int po_efanna_init_ids(const uint64_t *offsets, const uint32_t *nbrs, uint32_t n,
                       uint32_t entry, uint32_t L, uint32_t nq, po_rand_state *s,
                       uint32_t *out);

/* PANNS top-M search at one thread (M = 1 is seq_search_simple_search and
 * PSS_v5 at T = 1). init_ids: L ids shared by all queries, or nq x L when
 * init_per_query != 0. */
int po_search_top_m(const float *data, const float *norms, uint32_t n, uint32_t d,
                    const uint64_t *offsets, const uint32_t *nbrs,
                    const float *queries, uint32_t nq, const uint32_t *init_ids,
                    int init_per_query, uint32_t K, uint32_t L, uint32_t M, int kind,
                    uint32_t *out_ids, uint64_t *out_ndist, int threads);

/* PSS_v5 with T queues (T-1 workers + master), L_local, X sub-iterations, in
 * the deterministic round-robin schedule (one expansion per worker per round,
 * workers in id order, master last). T = 1 equals po_search_top_m with M = 1. */
/* Top-M search from per-query init lists of any length (<= list_stride),
 * queue length Lq[i] per query; repeated init ids enter once. */
int po_search_top_m_lists(const float *data, const float *norms, uint32_t n, uint32_t d,
                          const uint64_t *offsets, const uint32_t *nbrs, const float *queries,
                          uint32_t nq, const uint32_t *init_lists, uint32_t list_stride,
                          const uint32_t *init_counts, const uint32_t *Lq, uint32_t K, uint32_t M,
                          int kind, uint32_t *out_ids, uint64_t *out_ndist, int threads);
int po_search_pss(const float *data, const float *norms, uint32_t n, uint32_t d,
                  const uint64_t *offsets, const uint32_t *nbrs,
                  const float *queries, uint32_t nq, const uint32_t *init_ids,
                  uint32_t K, uint32_t L, uint32_t L_local, uint32_t X, uint32_t T,
                  int kind, uint32_t *out_ids, uint64_t *out_ndist, int threads);

/* efanna2e IndexNSG::Search (kind L2) / SearchWithOptGraph (kind IP_NORM):
 * distance-only order, `dist >= last` rejected; init ids nq x L. */
int po_search_efanna(const float *data, const float *norms, uint32_t n, uint32_t d,
                     const uint64_t *offsets, const uint32_t *nbrs,
                     const float *queries, uint32_t nq, const uint32_t *init_ids,
                     uint32_t K, uint32_t L, int kind,
                     uint32_t *out_ids, uint64_t *out_ndist, int threads);

/* Top-k by float64 squared L2, ties by id. */
int po_ground_truth_fp64(const float *data, uint32_t n, uint32_t d,
                         const float *queries, uint32_t nq, uint32_t k,
                         uint32_t *out_ids, double *out_dist, int threads);

/* NSG-style graph: exact k-NN by float64 (one FMA chain per distance), MRNG
 * prune to R, medoid entry, reachability repair (parallel_anns_b200/csrc/graph_build.cu). */
int po_build_nsg(const float *x, uint32_t n, uint32_t d, uint32_t k, uint32_t R, uint32_t *knn_out,
                 uint32_t *entry_out, uint64_t *off_out, uint32_t *nbrs_out, uint64_t nbrs_cap,
                 uint32_t *width_out, int threads);

/* The same graph as po_build_nsg and the same top-k as a float64 brute force
 * (d64 by one FMA chain, ties by id), computed with cluster lower bounds so a
 * 1M-vertex workload takes seconds (oracle/host_build.c). queries == NULL:
 * the k-NN of every base row, the row itself excluded. */
int po_host_knn(const float *x, uint32_t n, uint32_t d, const float *queries, uint32_t nq, uint32_t k,
                uint32_t *out_ids, double *out_dist, int threads);
int po_host_build_nsg(const float *x, uint32_t n, uint32_t d, uint32_t k, uint32_t R, uint32_t *knn_out,
                      uint32_t *entry_out, uint64_t *off_out, uint32_t *nbrs_out, uint64_t nbrs_cap,
                      uint32_t *width_out, int threads);

#ifdef __cplusplus
}
#endif
#endif
