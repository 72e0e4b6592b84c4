// Inference of the entry / L-budget MLP in the search kernel's prologue.
//
// The network maps a query (d floats) through two ReLU layers of 256 to R
// entry logits (one per k-means representative vertex) and one L-budget
// regressor output:
//     h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2),
//     z  = W3 h2 + b3 (R logits),  r = wl . h2 + bl.
// Weights are BF16, everything else (inputs, accumulators, biases) float32.
// One warp evaluates one query: lane t owns the 8 consecutive outputs
// 8t..8t+7 of each 256-wide slice, reads their 8 BF16 weights of input i as
// one 16-byte load (input-major layout, so a warp reads 512 contiguous bytes
// per input), and gets input i of the next layer from lane i / 8 by a
// shuffle. The weights (about 0.7 MB at d = 96, R = 1024) stay in L2.
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
constexpr int kMlpMaxR = 1024;  // entry classes (multiple of 256)
constexpr int kMlpMaxE = 64;    // learned entries per query (WarpMem::cand holds them)
constexpr int kMlpRecWords = 2 + kMlpMaxE;  // per-query record: L_q | fallback << 31, E, entries
#define PANNS_NEG_INF __int_as_float(0xff800000u)

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
    float *logits;            // warp slots x R scratch
    uint32_t *record;         // per query kMlpRecWords words (or null)
};

// Float index of query element e in a chain-major row (the padded layout
// whose term k of lane chain c is element c + 8k, or, when d % 16 == 8,
// element d - 8 + c for k = 0 and c + 8(k - 1) after it).
__device__ __forceinline__ uint32_t chain_major_index(uint32_t d, uint32_t e) {
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

__device__ __forceinline__ void fma8(float *acc, float x, uint4 w) {
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float lo = __uint_as_float(ws[j] << 16);
        const float hi = __uint_as_float(ws[j] & 0xffff0000u);
        acc[2 * j] = fmaf(x, lo, acc[2 * j]);
        acc[2 * j + 1] = fmaf(x, hi, acc[2 * j + 1]);
    }
}

// acc[0..8) += sum over the 256 inputs held 8 per lane in h[] of
// x_i * W[i][col0 + 8 lane .. + 8], W input-major with row stride `ld`.
__device__ __forceinline__ void layer_from_lanes(float *acc, const float *h, const __nv_bfloat16 *W,
                                                 uint32_t ld, uint32_t col0, int lane) {
    const uint4 *base = reinterpret_cast<const uint4 *>(W + col0) + lane;
    const uint32_t ld4 = ld / 8;
#pragma unroll 2
    for (int s = 0; s < 32; ++s) {
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const float x = __shfl_sync(0xffffffffu, h[e], s);
            fma8(acc, x, __ldg(base + (size_t) (s * 8 + e) * ld4));
        }
    }
}

// Runs the network for query row `qrow` (chain-major) and decides the
// query's entries and queue length. Writes the entry vertices (device ids)
// to cand[0..E'). Returns {E' | n_plain << 8, L_q}.
static __device__ __noinline__ uint2 mlp_prologue(const MlpDev *__restrict__ mp, const float *__restrict__ qrow,
                                                  uint32_t L, uint32_t K, uint32_t slot, uint32_t q,
                                                  uint32_t *cand, int lane) {
    const uint32_t d = mp->d, R = mp->R;
    float acc[8], h[8];
    // Layer 1: inputs straight from the query row.
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = __ldg(mp->b1 + lane * 8 + j);
    {
        const uint4 *w1 = reinterpret_cast<const uint4 *>(mp->w1) + lane;
        for (uint32_t i = 0; i < d; ++i) {
            const float x = __ldg(qrow + chain_major_index(d, i));
            fma8(acc, x, __ldg(w1 + (size_t) i * (kMlpH / 8)));
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) h[j] = fmaxf(acc[j], 0.f);
    // Layer 2.
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = __ldg(mp->b2 + lane * 8 + j);
    layer_from_lanes(acc, h, mp->w2, kMlpH, 0, lane);
#pragma unroll
    for (int j = 0; j < 8; ++j) h[j] = fmaxf(acc[j], 0.f);
    // L-budget regressor.
    float r = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) r = fmaf(__ldg(mp->wl + lane * 8 + j), h[j], r);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    r += mp->bl;
    // Entry logits, 256 at a time, with running softmax statistics.
    float *lg = mp->logits + (size_t) slot * R;
    float mx = PANNS_NEG_INF, se = 0.f;
    for (uint32_t c0 = 0; c0 < R; c0 += kMlpH) {
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = __ldg(mp->b3 + c0 + lane * 8 + j);
        layer_from_lanes(acc, h, mp->w3, R, c0, lane);
        float4 *dst = reinterpret_cast<float4 *>(lg + c0 + lane * 8);
        dst[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
        dst[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
        float cm = acc[0];
#pragma unroll
        for (int j = 1; j < 8; ++j) cm = fmaxf(cm, acc[j]);
        const float nm = fmaxf(mx, cm);
        float s = se * expf(mx - nm);
#pragma unroll
        for (int j = 0; j < 8; ++j) s += expf(acc[j] - nm);
        mx = nm;
        se = s;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float m2 = __shfl_xor_sync(0xffffffffu, mx, o);
        const float s2 = __shfl_xor_sync(0xffffffffu, se, o);
        const float nm = fmaxf(mx, m2);
        se = se * expf(mx - nm) + s2 * expf(m2 - nm);
        mx = nm;
    }
    const float conf = 1.f / se;  // softmax probability of the largest logit
    const bool fallback = !(conf >= mp->min_conf);
    uint32_t Lq = L;
    if (!fallback && mp->use_L) {
        const float v = mp->L_scale * expf(mp->L_exp * r);
        const uint32_t lo = max(K, min(mp->L_min, L));
        if (v < (float) L) Lq = max(lo, (uint32_t) ceilf(fmaxf(v, 0.f)));
    }
    uint32_t E = 0;
    if (!fallback && mp->use_entry) {
        const uint32_t want = min(min(mp->E, (uint32_t) kMlpMaxE), Lq);
        __syncwarp();
        for (; E < want; ++E) {
            float best = PANNS_NEG_INF;
            uint32_t bi = 0xffffffffu;
            for (uint32_t j = lane; j < R; j += 32) {
                const float v = lg[j];
                if (v > best) {
                    best = v;
                    bi = j;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float b2 = __shfl_xor_sync(0xffffffffu, best, o);
                const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, o);
                if (b2 > best || (b2 == best && i2 < bi)) {
                    best = b2;
                    bi = i2;
                }
            }
            if (bi >= R) break;  // only -inf or NaN left
            if (lane == 0) {
                const uint32_t v = __ldg(mp->rep + bi);
                cand[E] = v;
                if (mp->record) mp->record[(size_t) q * kMlpRecWords + 2 + E] = v;
            }
            if (lane == (int) (bi & 31)) lg[bi] = PANNS_NEG_INF;
            __syncwarp();
        }
        __syncwarp();
    }
    uint32_t n_plain = Lq - E;
    if (E) n_plain = min(n_plain, mp->L_init);
    if (lane == 0 && mp->record) {
        mp->record[(size_t) q * kMlpRecWords] = Lq | (fallback ? 0x80000000u : 0u);
        mp->record[(size_t) q * kMlpRecWords + 1] = E;
    }
    return make_uint2(E | (n_plain << 8), Lq);
}

}  // namespace panns
