/* panns_build — C ABI of the GPU graph construction of panns_b200.
 *
 * Builds the NSG-style proximity graph the search runs on: exact k-NN lists,
 * relative-neighbourhood (MRNG) pruning to at most R neighbours, the medoid as
 * entry vertex, and a reachability repair so that every vertex is reachable
 * from the entry. It plays the part of efanna2e's IndexNSG::Build
 * (include/efanna2e/index_nsg.cpp:638-718, whose pruning rule is
 * sync_prune :233-283) on exact k-NN lists instead of search-based candidate
 * pools, and IndexNSG::Save (:20-32) for the .nsg file.
 *
 * Semantics: d64(x, y) = one float64 FMA chain over the dimensions in order;
 * knn(a) = the k vertices b != a with the smallest (d64(a, b), b); b in knn(a)
 * is kept, in that order, unless a kept c has d64(c, b) < d64(a, b), up to R;
 * entry = argmin over v of (d64(v, mean), v) with mean = the float64 mean of
 * the rows; repair: every vertex not reachable from the entry, in id order,
 * gets an in-edge from the first reachable vertex of its k-NN list (else from
 * the entry). The k-NN lists come from a float32 screen of all pairs keeping
 * k + 8 candidates per row, ranked exactly in float64.
 */
#ifndef PANNS_BUILD_H
#define PANNS_BUILD_H

#include "panns_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct panns_graph panns_graph;

/* k-NN screen of the build: all pairs in float32 on CUDA cores keeping k + 8
 * candidates per row; by TF32 tensor-core GEMMs (cuBLAS) keeping k + 32; or
 * by the library's own tcgen05 kernel (TF32 MMAs into tensor memory, TMA-fed,
 * the per-row selection in the epilogue, no distance tile written; d a
 * multiple of 32 up to 128) keeping k + 32. Either way the candidates are
 * ranked exactly in float64. AUTO: the tcgen05 kernel from 100,000 vectors on
 * where it applies, else TF32 from 100,000 vectors on, else float32. */
#define PANNS_SCREEN_AUTO 0u
#define PANNS_SCREEN_FP32 1u
#define PANNS_SCREEN_TF32 2u
#define PANNS_SCREEN_TC 3u

/* Build the graph of n row-major float32 vectors of width d (host pointer) on
 * GPU `device`; knn_k <= 128, 0 < R <= knn_k. *out is released with
 * panns_graph_free. */
int panns_build_nsg(int device, const float *base, uint32_t n, uint32_t d, uint32_t knn_k, uint32_t R,
                    panns_graph **out);
/* The same with the k-NN screen chosen (PANNS_SCREEN_*). */
int panns_build_nsg_ex(int device, const float *base, uint32_t n, uint32_t d, uint32_t knn_k, uint32_t R,
                       uint32_t screen, panns_graph **out);

/* The construction of the large-graph configuration (100M vectors on one GPU,
 * where all pairs are out of reach): the vertices are partitioned into
 * `cells` k-means cells (Lloyd, `iters` rounds from a farthest-point start
 * seeded by `seed`, on `sample` rows taken at a fixed stride; then every
 * vertex goes to its nearest centroid), and the k-NN list of vertex a holds
 * the knn_k vertices b != a with the smallest (d64(a, b), b) among the
 * members of a's cell and of the `probe` cells whose centroids are nearest to
 * it (by float64 squared distance, then index). The candidates come from a
 * float32 screen keeping k + 8 per row, ranked exactly in float64; prune,
 * entry and repair are those of panns_build_nsg. probe <= 8; a list with
 * fewer than knn_k candidates is shorter. With `reverse` set, before the
 * repair every pruned edge a -> b (a ascending, then list order) also gives
 * b -> a while b has fewer than R neighbours and not a already (the part
 * efanna2e's InterInsert plays), which keeps tight, far-apart clusters
 * navigable from inside. panns_graph_cells returns the partition. This
 * plays the part of the reference's k-NN graph input
 * (IndexNSG::Load_nn_graph) for sizes its all-pairs tools cannot build. */
int panns_build_nsg_cells(int device, const float *base, uint32_t n, uint32_t d, uint32_t knn_k, uint32_t R,
                          uint32_t cells, uint32_t probe, uint32_t sample, uint32_t iters, uint32_t seed,
                          uint32_t reverse, panns_graph **out);
/* The partition of a graph built by panns_build_nsg_cells (each pointer
 * optional): number of cells, probe, the cell of every vertex (n), and each
 * cell's probe nearest cells (cells x probe; ~0 where there are fewer). */
int panns_graph_cells(const panns_graph *g, uint32_t *cells, uint32_t *probe, uint32_t *cell, uint32_t *near);
/* Sizes of a built graph (each pointer optional): vertices, largest degree,
 * entry vertex, total adjacency entries, in-edges added by the repair. */
int panns_graph_info(const panns_graph *g, uint32_t *n, uint32_t *width, uint32_t *entry, uint64_t *n_edges,
                     uint32_t *repaired);

/* Copy out (each optional): offsets n + 1 (CSR), nbrs n_edges, knn n x knn_k. */
int panns_graph_copy(const panns_graph *g, uint64_t *offsets, uint32_t *nbrs, uint32_t *knn);

/* Write the graph as a .nsg file (uint32 width, uint32 entry, then per vertex
 * uint32 degree and the ids), the layout IndexNSG::Save writes and
 * panns_load_nsg / Searching::load_nsg_graph read. */
int panns_graph_save_nsg(const panns_graph *g, const char *path);

int panns_graph_free(panns_graph *g);

/* efanna2e's own NSG construction, IndexNSG::Build
 * (include/efanna2e/index_nsg.cpp:403-450; get_neighbors :141-207,
 * sync_prune :226-276, InterInsert :278-354, tree_grow / DFS / findroot
 * :638-718), with the reference's parameters L (search pool), R (degree) and
 * C (candidates considered by the prune), from a k-NN graph given as
 * n x knn_k ids (what IndexNSG::Load_nn_graph reads from an EFANNA file) and
 * n row-major float32 vectors of width d (a multiple of 8), host pointers.
 * The result equals the reference's Build run with one OpenMP thread from a
 * glibc rand() stream seeded with rand_seed (1 = a process that never called
 * srand): every vertex's search and prune runs on GPU `device`, one warp per
 * vertex, the reverse-edge insertion and the reachability repair on the host
 * in the reference's order. Exactly equal distances (duplicate rows) are the
 * one input whose order the reference leaves unspecified. *out is released
 * with panns_graph_free; panns_graph_save_nsg writes it as IndexNSG::Save. */
int panns_efanna_build(int device, const float *base, uint32_t n, uint32_t d, const uint32_t *knn,
                       uint32_t knn_k, uint32_t L, uint32_t R, uint32_t C, uint32_t rand_seed,
                       panns_graph **out);

#ifdef __cplusplus
}
#endif

#endif
