// Float64 brute-force ground truth.
//
// The k results of any search are k distinct vertices, so the largest of their
// exact distances, tau, is an upper bound of the true k-th smallest distance.
// One tiled pass over the base therefore only has to collect the vertices
// whose float64 distance is <= tau (about k of them for a good search) into a
// per-query list; an exact (distance, id) sort of that list gives the top k.
// Distances are sum over dimensions, in order, of fma(t, t, acc) with
// t = (double) x - (double) q, in both kernels, so the search's own results
// meet their own bound bit for bit. Plays the role of
// tools/save_true_nearest_neighbors.cpp:16-35 (which scans in float32).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace panns {

constexpr int kGtQ = 64;    // queries per block tile
constexpr int kGtV = 128;   // vertices per block tile
constexpr int kGtK = 8;     // dimensions per shared-memory step

// tau[q] = max over the k ids of query q of its float64 distance.
__global__ void gt_tau_kernel(const float *__restrict__ base, int d, const float *__restrict__ queries,
                              uint32_t nq, const uint32_t *__restrict__ ids, uint32_t k,
                              double *__restrict__ tau) {
    const int lane = threadIdx.x & 31;
    const uint32_t q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= nq) return;
    const float *qr = queries + (size_t) q * d;
    double mx = 0.0;
    for (uint32_t i = lane; i < k; i += 32) {
        const float *x = base + (size_t) ids[(size_t) q * k + i] * d;
        double acc = 0.0;
        for (int j = 0; j < d; ++j) {
            const double t = (double) x[j] - (double) qr[j];
            acc = fma(t, t, acc);
        }
        mx = fmax(mx, acc);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) tau[q] = mx;
}

// Grid: x = query tiles (fastest, so the tiles of one vertex range run
// together and share it through L2), y = vertex tiles v_tile0 + blockIdx.y
// (launched in slices of at most 65,535 tiles, the grid's y limit). 256 threads; thread
// (ty, tx) owns queries 4*ty..4*ty+3 and vertices tx + 16*j, j < 8.
__global__ void __launch_bounds__(256) gt_collect_kernel(const float *__restrict__ base, uint32_t n, int d,
                                                         const float *__restrict__ queries, uint32_t nq,
                                                         const double *__restrict__ tau, uint32_t cap,
                                                         uint32_t *__restrict__ cnt, double *__restrict__ cand_d,
                                                         uint32_t *__restrict__ cand_i, uint32_t v_tile0) {
    __shared__ double sq[kGtK][kGtQ];
    __shared__ double sv[kGtK][kGtV];
    const uint32_t q0 = blockIdx.x * kGtQ, v0 = (blockIdx.y + v_tile0) * kGtV;
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    double acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    for (int k0 = 0; k0 < d; k0 += kGtK) {
        for (int e = tid; e < kGtQ * kGtK; e += 256) {
            const int qq = e / kGtK, kk = e % kGtK;
            const uint32_t q = q0 + qq;
            sq[kk][qq] = (q < nq && k0 + kk < d) ? (double) queries[(size_t) q * d + k0 + kk] : 0.0;
        }
        for (int e = tid; e < kGtV * kGtK; e += 256) {
            const int vv = e / kGtK, kk = e % kGtK;
            const uint32_t v = v0 + vv;
            sv[kk][vv] = (v < n && k0 + kk < d) ? (double) base[(size_t) v * d + k0 + kk] : 0.0;
        }
        __syncthreads();
        const int kmax = min(kGtK, d - k0);
        for (int kk = 0; kk < kmax; ++kk) {
            double a[4], b[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sq[kk][4 * ty + i];
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = sv[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const double t = b[j] - a[i];
                    acc[i][j] = fma(t, t, acc[i][j]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t q = q0 + 4 * ty + i;
        if (q >= nq) continue;
        const double tq = tau[q];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t v = v0 + tx + 16 * j;
            if (v < n && acc[i][j] <= tq) {
                const uint32_t pos = atomicAdd(cnt + q, 1u);
                if (pos < cap) {
                    cand_d[(size_t) q * cap + pos] = acc[i][j];
                    cand_i[(size_t) q * cap + pos] = v;
                }
            }
        }
    }
}

}  // namespace panns
