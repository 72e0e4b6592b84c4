/* panns_b200 — C ABI of the B200-native best-first search over NSG graphs.
 *
 * This is the drop-in boundary for the query-time search path of PANNS
 * (johnpzh/parallel_ANNS). Every entry point takes plain pointers and sizes,
 * returns an int status (PANNS_OK = 0, negative on error) and never exits
 * the process; panns_last_error() gives a message for the last failure on
 * the calling thread. One handle owns one GPU's copy of the base vectors and
 * the graph plus one CUDA stream; calls on one handle must not overlap
 * (the reference engine is single-caller too), different handles are
 * independent. Host pointers are read or written synchronously unless a
 * function says otherwise.
 *
 * Reference interfaces each entry point replaces (paths relative to the
 * parallel_ANNS project root; PSS = core/Searching.202102022027.PSS_v5.dist_thresh.profiling,
 * LG = core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling,
 * TOPM = core/Searching.202011241533.top_m_pure, NSG = include/efanna2e/index_nsg):
 */
#ifndef PANNS_B200_H
#define PANNS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PANNS_OK 0
#define PANNS_EINVAL (-1)     /* bad argument or size */
#define PANNS_EIO (-2)        /* file missing, truncated or malformed */
#define PANNS_ENOMEM (-3)     /* host or device allocation failed */
#define PANNS_ECUDA (-4)      /* CUDA runtime error, or no usable GPU */
#define PANNS_ESTATE (-5)     /* handle not ready (no base / graph loaded) */
#define PANNS_EDEVICE (-6)    /* the kernel flagged a bad input (e.g. a neighbour id >= N) */

/* Search semantics. All return the K best ids of the final queue.
 * NSG_SEQ   PANNS sequential best-first search (Searching::seq_search_simple_search,
 *           TOPM.cpp:1486-1605; identical to PSS_v5 at one thread).
 * TOP_M     PANNS top-M search at one thread: the M best unchecked candidates
 *           are expanded per step (TOPM.cpp:1881-1965, para_search_with_top_m_pure
 *           with num_threads_ = 1; seq_search_with_top_m_pure :1382-1484).
 * PSS_V5    PANNS PSS_v5 (PSS.cpp:1218-1515, LG.cpp:1376-1726) with T queues
 *           (T-1 workers + master), L_local and X; its parallel expand phase is
 *           run in a fixed round-robin order (one expansion per worker per
 *           round, master last). T = 1 is NSG_SEQ.
 * EFANNA    efanna2e IndexNSG::Search / SearchWithOptGraph (NSG.cpp:452-611):
 *           distance-only order, `dist >= L-th` rejected, per-query init ids. */
typedef enum {
    PANNS_MODE_NSG_SEQ = 0,
    PANNS_MODE_TOP_M = 1,
    PANNS_MODE_PSS_V5 = 2,
    PANNS_MODE_EFANNA = 3
} panns_mode;

/* Distance. NORM_IP: ||v||^2 - 2<v,q> with the stored norm (PSS.cpp:294-391,
 * the "opt graph" of load_nsg_graph and efanna2e SearchWithOptGraph);
 * L2: sum (v-q)^2 (LG.cpp:525-563, efanna2e Search). Both accumulate in the
 * reference's 8-lane order with one FMA per lane step, bit-identical to the
 * reference built with -O3 -march=native. */
typedef enum { PANNS_DIST_NORM_IP = 0, PANNS_DIST_L2 = 1 } panns_distance;

/* Storage of the base vectors on the GPU. FP32 is exact. BF16 and FP8 (E4M3
 * with a per-dimension absmax scale) cut gathered bytes 2x / 4x; the final L
 * candidates are then re-ranked in exact FP32 from the float32 originals. */
typedef enum { PANNS_STORE_FP32 = 0, PANNS_STORE_BF16 = 1, PANNS_STORE_FP8 = 2 } panns_storage;

typedef struct {
    uint32_t mode;        /* panns_mode */
    uint32_t distance;    /* panns_distance */
    uint32_t K;           /* ids returned per query, K <= L */
    uint32_t L;           /* queue length (L_master of PSS_v5, L_search of efanna2e) */
    uint32_t M;           /* TOP_M: candidates expanded per step (>= 1) */
    uint32_t T;           /* PSS_V5: number of queues (workers + master, >= 1) */
    uint32_t L_local;     /* PSS_V5: worker queue capacity (0 = L) */
    uint32_t X;           /* PSS_V5: expansions per worker per stage (>= 1) */
    uint32_t warps_per_block; /* warps (queries in flight) per block, <= 4; 0 = 4, fewer when four
                                 queues of L do not fit one block's shared memory */
    uint32_t storage;     /* panns_storage the search distances use: FP32 (exact), or
                             the reduced copy built by panns_set_base (NSG_SEQ / TOP_M
                             only; the final L are re-ranked in exact FP32) */
    uint32_t flags;       /* PANNS_FLAG_* bits, 0 for none */
    const uint32_t *L_query; /* optional host array, one queue length per query of the call
                                (K <= L_query[i] <= L; not for PSS_V5 with T > 1). NSG_SEQ,
                                TOP_M, PSS_V5: query i searches exactly as with L = L_query[i];
                                EFANNA: with the first L_query[i] of its L init ids. NULL = L
                                for every query. No counterpart in the reference (one L per
                                call, PSS.cpp:1218). */
    uint32_t blocks_per_sm;  /* resident blocks per SM; fewer leave more of the SM's L1 / shared
                                array to L1, which caches gathered rows. 0 = as many as fit,
                                but no more than fit in 196 KB of shared memory */
    uint32_t warps_per_query; /* 1: one warp per query (warps_per_block queries per block);
                                 2, 4 or 8: that many warps share each query's steps (one query per
                                 block; NSG_SEQ, TOP_M, PSS_V5 at T = 1, any storage, with or
                                 without PANNS_FLAG_LEARNED), for small batches and long queues; same
                                 ids and counts.
                                 0: chosen from nq and L (8 up to one query per SM or for L >= 2048,
                                 2 up to ten per SM, else 1) when the mode allows it and
                                 warps_per_block and blocks_per_sm are 0, else 1 */
} panns_search_params;

/* Enqueue the launch (per-call memsets, query layout and the search kernel)
 * as a CUDA graph, captured once per launch shape and replayed while the
 * shape and buffers stay the same: small batches then pay one graph launch
 * instead of several API calls. Results are identical. */
#define PANNS_FLAG_CUDA_GRAPH 1u

typedef struct {
    uint64_t n_dist;      /* distance computations (count_distance_computation_) */
    uint64_t n_expand;    /* expanded candidates */
    uint64_t n_edges;     /* adjacency words read: sum over expansions of 1 + degree */
    uint64_t n_iter;      /* search steps (picks) */
    double kernel_ms;     /* device time of the search kernel(s), CUDA events */
    double total_ms;      /* wall time of the call including copies */
} panns_stats;

typedef struct panns_index panns_index;

/* Last error message of the calling thread ("" if none). */
const char *panns_last_error(void);
/* ABI version, (major << 16) | minor. */
uint32_t panns_version(void);

/* Open a handle on CUDA device `device`. Replaces constructing
 * PANNS::Searching (PSS.h:30-226) / efanna2e::IndexNSG (NSG.h:17-43). */
int panns_open(panns_index **out, int device);
/* Release all host and device memory of the handle (Searching::~Searching,
 * PSS.h:213-226). */
int panns_close(panns_index *h);

/* Base vectors, n x d float32 row-major (host pointer, copied).
 * Replaces Searching::load_data_load (PSS.cpp:14-28) with the file already
 * read; d must be a multiple of 8 (the reference's 8-lane kernels read
 * past the row otherwise). `storage` BF16 or FP8 also builds that reduced
 * copy (the float32 rows are always kept, for exact searches and re-ranks). */
int panns_set_base(panns_index *h, const float *data, uint32_t n, uint32_t d, uint32_t storage);
/* Read an fvecs file (include/utils.h:95-138 DiskIO::load_data) and call
 * panns_set_base. */
int panns_load_fvecs_base(panns_index *h, const char *path, uint32_t storage);
/* Queries, nq x d float32 (host, copied and kept on the GPU). Replaces
 * Searching::load_queries_load (PSS.cpp:34-49). */
int panns_set_queries(panns_index *h, const float *queries, uint32_t nq, uint32_t d);
int panns_load_fvecs_queries(panns_index *h, const char *path);

/* Graph in CSR form: offsets[n+1] (u64) into nbrs (u32). Replaces
 * load_nsg_graph (PSS.cpp:57-133) / load_common_nsg_graph (LG.cpp:138-258) /
 * IndexNSG::Load (NSG.cpp:34-51). `width` and `entry` are the .nsg header. */
int panns_set_graph(panns_index *h, uint32_t width, uint32_t entry, const uint64_t *offsets,
                    const uint32_t *nbrs, uint32_t n);
/* Read a .nsg file (u32 width, u32 entry, then per vertex u32 deg + deg ids). */
int panns_load_nsg(panns_index *h, const char *path);

/* Sizes of what is loaded (any pointer may be NULL). */
int panns_info(const panns_index *h, uint32_t *n, uint32_t *d, uint32_t *nq, uint32_t *width,
               uint32_t *entry);

/* PANNS init ids: the entry's neighbours (deduplicated), then entry+1, entry+2,
 * ... with wrap-around, until L (Searching::prepare_init_ids, PSS.cpp:238-291). */
int panns_prepare_init_ids(const panns_index *h, uint32_t L, uint32_t *out);
/* efanna2e init ids for nq consecutive queries: the entry's first min(L, deg)
 * neighbours, then rand() % N until L distinct (NSG.cpp:462-474). The rand()
 * stream is glibc's, held in *rand_state (an opaque 40-int32 buffer set up by
 * panns_rand_seed, seed 1 = a never-seeded process) and continued across calls.
 * out: nq x L. */
int panns_rand_seed(int32_t *rand_state, uint32_t seed);
int panns_efanna_init_ids(const panns_index *h, uint32_t L, uint32_t nq, int32_t *rand_state,
                          uint32_t *out);

/* Batched search of the loaded queries [q_begin, q_begin + nq).
 * init_ids: L ids shared by all queries (NSG_SEQ, TOP_M, PSS_V5; NULL = the
 * panns_prepare_init_ids list) or nq x L per query (EFANNA; NULL = replay
 * of a fresh seed-1 rand() stream). out_ids: nq x K row-major, query i's K ids
 * at out_ids + i*K (the set_K_list order of the reference apps). Replaces the
 * per-query loops over para_search_PSS_v5_dist_thresh_profiling
 * (app/PSS_v5_distance_threshold_profiling.cpp:132-152), seq_search_simple_search,
 * para_search_with_top_m_pure and IndexNSG::Search / SearchWithOptGraph. */
int panns_search(panns_index *h, const panns_search_params *p, const uint32_t *init_ids,
                 uint32_t q_begin, uint32_t nq, uint32_t *out_ids, panns_stats *stats);

/* Same, for nq queries given as a host pointer (nq x d float32). */
int panns_search_host(panns_index *h, const panns_search_params *p, const float *queries,
                      uint32_t nq, const uint32_t *init_ids, uint32_t *out_ids, panns_stats *stats);

/* Same, with device pointers (queries nq x d float32 and out_ids nq x K on the
 * handle's device) enqueued on `stream` (a cudaStream_t; NULL = the handle's
 * stream). Asynchronous: returns after enqueueing; `stats` (if not NULL) is
 * filled only with what is known on the host (no counts, no times). */
int panns_search_device(panns_index *h, const panns_search_params *p, const float *d_queries,
                        uint32_t nq, const uint32_t *init_ids, uint32_t *d_out_ids, void *stream,
                        panns_stats *stats);

/* The batched search without any memory allocation, for callers that cannot
 * allocate GPU memory once they are running (a serving process whose memory
 * is all reserved by a framework's pool, a latency-bound loop, a plug-in in a
 * host that forbids allocations after start-up). No counterpart in the
 * reference, which allocates its scratch (set_L, is_visited) in the caller.
 * d_queries: nq x d float32 and d_out_ids: nq x K u32 (original ids), both
 * device pointers owned by the caller; `stream` is a cudaStream_t (NULL = the
 * handle's stream). Modes NSG_SEQ, TOP_M and PSS_V5 with T = 1 (the PANNS init
 * list), L <= 1024. All scratch comes from one fixed 32 MiB array in the
 * library's device image: N, nq and the warp count must fit it, otherwise
 * PANNS_EINVAL says so. One warp per query with as many blocks per SM as
 * fit: warps_per_query > 1 or blocks_per_sm != 0 give PANNS_EINVAL. The index
 * must already be laid out on the GPU (one panns_search or panns_search_host
 * call before). The first call on a device looks up the array's address. Do
 * not call it while a stream is being captured: every call copies the init
 * list from host memory, reads the error word back and synchronises. Calls
 * share the array: calls that overlap on the GPU race. Returns after the
 * search has finished. */
int panns_search_static(panns_index *h, const panns_search_params *p, const float *d_queries,
                        uint32_t nq, uint32_t *d_out_ids, void *stream);

/* Recall@k (k in {1, 5, 10, 20, 50, 100}) of result ids against a true-NN
 * list, with the reference's definition (PSS.cpp:191-230): a true top-k id
 * counts if it appears in result[0 : min(L, 100, k)]. true_ids: nq x true_k. */
int panns_recall(const uint32_t *result_ids, uint32_t nq, uint32_t K, const uint32_t *true_ids,
                 uint32_t true_k, uint32_t L, uint32_t at, double *out);

/* Float64 brute-force ground truth on the GPU: the top-k ids (original ids)
 * by exact squared L2 in float64, ties by id, for nq host queries (nq x d
 * float32); out_dist (optional) gets the float64 distances. Needs the base
 * and the graph: a search gives each query a distance bound, one float64
 * pass over all N collects the vertices within it, and an exact sort of those
 * gives the answer. Plays the role of tools/save_true_nearest_neighbors.cpp:16-64
 * (which scans in float32). */
int panns_ground_truth(panns_index *h, const float *queries, uint32_t nq, uint32_t k, uint32_t *out_ids,
                       double *out_dist);

/* Read a true-NN file (u32 nq, u32 K, then nq x K x (u32 id, f32 dist)):
 * Searching::load_true_NN (PSS.cpp:141-189). Call with ids == NULL to get
 * the sizes first; ids is nq x K, dists (optional) likewise. */
int panns_load_true_nn(const char *path, uint32_t *nq, uint32_t *K, uint32_t *ids, float *dists);

#ifdef __cplusplus
}
#endif
#endif
