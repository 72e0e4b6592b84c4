// The entry / L-budget network as the search sees it.
//
// The network maps a query (d floats) through two ReLU layers of 256 to R
// entry logits (one per k-means representative vertex) and one L-budget
// regressor output:
//     h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2),
//     z  = W3 h2 + b3 (R logits),  r = wl . h2 + bl.
// Weights are BF16, everything else (inputs, accumulators, biases) float32.
//
// Inference runs batched, before the search kernel of the same launch
// sequence (mlp_decide in learned.cu): the three layers as tensor-core GEMMs
// over the whole batch (each weight tile read once per 64 queries, not once
// per query), then one warp per query turns its logits and regressor output
// into a decision record, which the search kernel's prologue reads.
//
// Decision (per query): confidence = the largest softmax probability of the
// logits. Below `min_conf` the query falls back to the plain method (the
// PANNS init list and the call's L, exactly the search without the network).
// Otherwise the E representatives with the largest logits enter the queue
// first, followed by at most L_init ids of the plain init list, and the
// queue length is L_q = clamp(ceil(L_scale * exp(L_exp * r)), max(K, L_min), L).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace panns {

constexpr int kMlpH = 256;      // hidden width
constexpr int kMlpMaxR = 4096;  // entry classes (multiple of 256)
constexpr int kMlpMaxE = 64;    // learned entries per query (WarpMem::cand holds them)
constexpr int kMlpRecWords = 2 + kMlpMaxE;  // per-query record: L_q | fallback << 31, E, entries
#define PANNS_NEG_INF __int_as_float(0xff800000u)

// The network in its inference layout (device pointers) and the decision rule.
struct MlpDev {
    const __nv_bfloat16 *w1;  // d x 256, input-major: row i holds the weights of input i
    const __nv_bfloat16 *w2;  // 256 x 256
    const __nv_bfloat16 *w3;  // 256 x R (entry logits)
    const float *b1, *b2, *b3;  // 256, 256, R
    const float *wl;          // 256, L-budget regressor
    float bl;
    const uint32_t *rep;      // R representative vertices (device ids)
    uint32_t d, R, E, L_init, L_min, use_entry, use_L;
    float min_conf;
    float L_scale, L_exp;     // L_q = L_scale * exp(L_exp * regressor)
};

// Float index of query element e in a chain-major row (the padded layout
// whose term k of lane chain c is element c + 8k, or, when d % 16 == 8,
// element d - 8 + c for k = 0 and c + 8(k - 1) after it).
__host__ __device__ __forceinline__ uint32_t chain_major_index(uint32_t d, uint32_t e) {
    const uint32_t DR = d % 16, DD = d - DR;
    uint32_t c, k;
    if (DR && e >= DD) {
        c = e - DD;
        k = 0;
    } else {
        c = e & 7;
        k = (e >> 3) + (DR ? 1u : 0u);
    }
    return (8 * (k >> 2) + c) * 4 + (k & 3);
}

// The search prologue's view of query q's decision record: writes the
// learned entries (device ids) to cand[0..E) and returns {E | n_plain << 8,
// L_q}, where n_plain is how many ids of the plain init list follow them.
__device__ __forceinline__ uint2 mlp_read_decision(const uint32_t *__restrict__ rec_all, uint32_t L_init, uint32_t q,
                                                   uint32_t *cand, int lane) {
    const uint32_t *rec = rec_all + (size_t) q * kMlpRecWords;
    const uint32_t Lq = __ldg(rec) & 0x7fffffffu;
    const uint32_t E = min(__ldg(rec + 1), (uint32_t) kMlpMaxE);
    for (uint32_t i = lane; i < E; i += 32) cand[i] = __ldg(rec + 2 + i);
    __syncwarp();
    uint32_t n_plain = Lq - E;
    if (E) n_plain = min(n_plain, L_init);
    return make_uint2(E | (n_plain << 8), Lq);
}

}  // namespace panns
