/* panns_learned — C ABI of the learned entry / L-budget part of panns_b200.
 *
 * No counterpart in the reference, whose searches always start from the
 * graph's entry vertex (the init list of Searching::prepare_init_ids,
 * PSS.cpp:1162-1216) with one fixed L per call. Here a small network maps each
 * query to entry vertices among k-means representatives of the base and to a
 * queue length; the plain search (PANNS init list, the call's L) stays both
 * the fallback for queries the network is not confident about and the
 * yardstick of its recall.
 *
 * Network: x (d) -> relu(256) -> relu(256) -> R entry logits + 1 L-budget
 * output. Parameters are one float32 array in this order (row-major, the
 * weight matrices input-major, i.e. [inputs][outputs]):
 *   W1 d x 256, b1 256, W2 256 x 256, b2 256, W3 256 x (R + 1), b3 R + 1
 * (column R of W3 / entry R of b3 = the L-budget output). The forward pass
 * computes with the weight matrices rounded to BF16 and float32 everything
 * else; training keeps float32 master weights (Adam).
 *
 * Loss per query: softmax cross-entropy of the R logits against the
 * query's label histogram (T cell labels, each worth 1/T) plus
 * lambda_L / 2 * (z_R - y)^2 for the L-budget target y; averaged over the batch.
 */
#ifndef PANNS_LEARNED_H
#define PANNS_LEARNED_H

#include "panns_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Searches with this flag run the attached network over the whole batch just
 * before the search kernel (tensor-core GEMMs), and each query's search
 * starts from that query's decision (NSG_SEQ, TOP_M and PSS_V5 at T = 1;
 * any storage). */
#define PANNS_FLAG_LEARNED 2u

/* Number of float32 parameters of the network for input width d and R classes. */
uint64_t panns_mlp_param_count(uint32_t d, uint32_t R);

/* Loss and gradient of one batch (B queries) on GPU `device`, by the same
 * kernels training uses. X: B x d float32, cells: B x T uint16 labels (< R),
 * y: B float32 targets; grad: param_count float32 (host); loss: the mean. */
int panns_mlp_loss_grad(int device, uint32_t d, uint32_t R, uint32_t T, const float *params, const float *X,
                        const uint16_t *cells, const float *y, uint32_t B, float lambda_L, float *grad,
                        double *loss);

/* Forward pass of n queries (training layout, BF16 weights): Z n x (R + 1). */
int panns_mlp_forward(int device, uint32_t d, uint32_t R, const float *params, const float *X, uint32_t n,
                      float *Z);

typedef struct {
    uint32_t d, R, T;      /* input width, classes, labels per query */
    uint32_t batch;        /* minibatch size */
    uint32_t epochs;
    uint32_t seed;         /* order of the samples in each epoch */
    float lr, beta1, beta2, eps, weight_decay;
    float lambda_L;        /* weight of the L-budget loss */
} panns_mlp_train_params;

/* Adam training on GPU `device` over n samples, minibatches in a seeded
 * shuffled order per epoch. params: initial values in, trained values out.
 * epoch_loss (optional, `epochs` doubles): mean training loss of each epoch. */
int panns_mlp_train(int device, const panns_mlp_train_params *tp, const float *X, const uint16_t *cells,
                    const float *y, uint32_t n, float *params, double *epoch_loss);

/* k-means over the handle's base vectors (Lloyd, `iters` rounds from a
 * farthest-point start, its first centre chosen by `seed`). Outputs (host, each optional): rep_ids k original
 * ids, the base vertex of each cell nearest its centroid; assign n cells per
 * original id; centroids k x d. */
int panns_kmeans(panns_index *h, uint32_t k, uint32_t iters, uint32_t seed, uint32_t *rep_ids,
                 uint32_t *assign, float *centroids);

typedef struct {
    uint32_t E;           /* learned entries placed first in the queue (<= 64; 0 = none) */
    uint32_t L_init;      /* plain init ids after them (at most L_q - E; >= L fills the queue) */
    uint32_t L_min;       /* lower bound of the predicted queue length */
    uint32_t use_L;       /* 1: queue length L_q = clamp(ceil(L_scale * exp(L_exp * z_R)), max(K, L_min), L) */
    float L_scale;
    float L_exp;          /* 1 = the regressor's L; < 1 narrows the spread of the budgets */
    float min_conf;       /* softmax confidence below which the query runs the plain search */
} panns_learned_params;

/* Attach the network (float32 parameters for the handle's d and R classes)
 * and its R representative vertices (original ids) to the handle, for
 * searches with PANNS_FLAG_LEARNED. Replaces any previous network. */
int panns_set_learned(panns_index *h, const float *params, uint32_t R, const uint32_t *rep_ids,
                      const panns_learned_params *lp);

/* After a PANNS_FLAG_LEARNED search: per query of that call, 66 words: the
 * queue length used (bit 31 set when the query fell back to the plain
 * search), the number E' of learned entries, then those E' entries
 * (original ids, best first). */
int panns_learned_record(panns_index *h, uint32_t nq, uint32_t *out);

#ifdef __cplusplus
}
#endif

#endif
