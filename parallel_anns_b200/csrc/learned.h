// Host-side launchers of the learned-entry part (learned.cu), used by the
// index code in panns_abi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "mlp_infer.cuh"

namespace panns {

// Records `msg` as the calling thread's last error (panns_last_error) and
// returns `code`.
int set_error(int code, const std::string &msg);

// Lloyd's k-means on n row-major float32 rows of width d (device), k
// centroids initialised by farthest-point seeding (the first centre chosen
// by `seed`) on up to 32 k rows at a fixed stride. On return
// (enqueued on `stream`, synchronised): centroids (k x d, device), assign[i]
// = cell of row i (device), rep[c] = the row of cell c nearest to its
// centroid (device; cells left empty get a row no other cell uses).
// Returns a PANNS_* status.
int kmeans_run(const float *rows, uint32_t n, uint32_t d, uint32_t k, uint32_t iters, uint32_t seed,
               float *centroids, uint32_t *assign, uint32_t *rep, cudaStream_t stream);

// cell[i] = the nearest (squared L2, via ||c||^2 - 2 x.c; ties to the lower
// index) of the k rows center_rows[0..k) (device) for each of the n rows
// (device, row-major, width d). Enqueued on `stream`, synchronised.
int nearest_center(const float *rows, uint32_t n, uint32_t d, const uint32_t *center_rows, uint32_t k,
                   uint32_t *cell, cudaStream_t stream);

// The same with the k centres given as rows of width d (device, k x d).
int nearest_centroid(const float *rows, uint32_t n, uint32_t d, const float *centroids, uint32_t k, uint32_t *cell,
                     cudaStream_t stream);

// Packs the float32 training parameters (layout of panns_mlp_param_count)
// into the inference layout read by mlp_decide: BF16 w1 (d x 256),
// w2 (256 x 256), w3 (256 x R) into `wbf` (device, 256 (d + 256 + R)
// elements) and float32 b1, b2, b3, wl, bl into `fb` (device, 256 * 3 + R + 1).
int mlp_pack_inference(const float *params_dev, uint32_t d, uint32_t R, void *wbf, float *fb,
                       cudaStream_t stream);

// Device scratch of mlp_decide for a chunk of `rows` queries: X (rows x d),
// H1 and H2 (rows x 256), Z (rows x R).
struct MlpScratch {
    float *X, *H1, *H2, *Z;
    uint32_t rows;
};

// Batched inference of the network `m` (device pointers) for nq queries,
// chain-major rows of width dpad at q_cm (device): per chunk of scratch.rows
// queries, the three layers as tensor-core GEMMs, then each query's decision
// record (kMlpRecWords words: L_q | fallback << 31, E, E entry vertices as
// device ids) into `record`. The call's queue length is L, or Lq[q] when Lq
// (device) is given. Only enqueues on `stream` (graph-capturable); returns the
// first launch error.
cudaError_t mlp_decide(const MlpDev &m, const float *q_cm, uint32_t dpad, uint32_t nq, uint32_t L, const uint32_t *Lq,
               uint32_t K, const MlpScratch &scratch, uint32_t *record, cudaStream_t stream);

}  // namespace panns
