// NSG-style graph construction on the GPU: exact k-NN lists, relative-
// neighbourhood (MRNG) pruning to R, medoid entry, reachability repair.
//
// Semantics (restated by po_build_nsg in oracle/panns_oracle.c):
//   * d64(x, y) = sum over j = 0..d-1, in order, of fma(t, t, acc) with
//     t = (double) x_j - (double) y_j (one float64 chain).
//   * knn(a) = the k vertices b != a with the smallest (d64(a, b), b).
//   * prune(a): walk knn(a) in order; b is kept unless some already kept c has
//     d64(c, b) < d64(a, b); at most R are kept (the NSG rule of
//     include/efanna2e/index_nsg.cpp:233-283 applied to exact k-NN lists).
//   * entry = the vertex with the smallest (d64(v, mean), v), mean = the float64
//     mean of the rows summed in id order.
//   * repair: from the entry, every vertex not reached (in id order) gets an
//     in-edge from the first reached vertex of its k-NN list (else the entry),
//     then everything it reaches is marked (index_nsg.cpp:638-718 plays this
//     part with a DFS tree).
// The k-NN search screens all pairs (||y||^2 - 2 x.y) either in float32 on CUDA
// cores (tiled here, C = k + 8 candidates kept per row) or with TF32
// tensor-core GEMMs (cuBLAS) folded tile by tile into the rows' lists (C = k +
// 32), and ranks the C survivors by d64; the result equals the exact k-NN
// unless a true neighbour falls outside the screen's top C, which needs the
// screen's rounding to move it past 8 (float32) or 32 (TF32) others.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include "../../include/panns_build.h"
#include "graph_types.h"
#include "learned.h"
#include "tc_screen.h"

namespace panns {
namespace {

#define GCU(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return set_error(PANNS_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
struct Buf {
    T *p = nullptr;
    ~Buf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

constexpr int kBQ = 64;    // rows (queries) per block
constexpr int kBV = 128;   // candidate rows per tile
constexpr int kBK = 16;    // dimensions per shared-memory step
constexpr int kMaxC = 136; // screen list length (k + 8 <= 136)

__global__ void sqnorm32_kernel(const float *__restrict__ x, uint32_t n, uint32_t d, float *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float s = 0.f;
    for (uint32_t j = 0; j < d; ++j) s = fmaf(x[(size_t) r * d + j], x[(size_t) r * d + j], s);
    out[r] = s;
}

// Insert this warp's 32 candidates (dv, iv) (one per lane; +inf = none) into
// the sorted list (rd, ri)[0..c) of capacity C, by (distance, id): each one
// that beats the C-th in turn goes to its rank, the list shifting up by one.
__device__ __forceinline__ void list_insert(float *rd, uint32_t *ri, uint32_t &c, uint32_t C, float dv, uint32_t iv,
                                            int lane) {
    const float thr_d = c == C ? rd[C - 1] : __int_as_float(0x7f800000);
    const uint32_t thr_i = c == C ? ri[C - 1] : 0xffffffffu;
    bool want = dv < thr_d || (dv == thr_d && iv < thr_i);
    want = want && !(dv == __int_as_float(0x7f800000));
    uint32_t bm = __ballot_sync(0xffffffffu, want);
    while (bm) {
        const int src = __ffs(bm) - 1;
        bm &= bm - 1;
        const float sd = __shfl_sync(0xffffffffu, dv, src);
        const uint32_t si = __shfl_sync(0xffffffffu, iv, src);
        // still better than the C-th after earlier inserts?
        if (c == C && !(sd < rd[C - 1] || (sd == rd[C - 1] && si < ri[C - 1]))) continue;
        // position = number of entries smaller than (sd, si)
        uint32_t pos = 0;
        for (uint32_t e0 = 0; e0 < c; e0 += 32) {
            const uint32_t e = e0 + lane;
            const bool less = e < c && (rd[e] < sd || (rd[e] == sd && ri[e] < si));
            pos += __popc(__ballot_sync(0xffffffffu, less));
        }
        const uint32_t end = c < C ? c : C - 1;  // last index that moves
        // shift [pos, end) up by one, from the top down in chunks of 32
        for (int e0 = (int) end - 1; e0 >= (int) pos; e0 -= 32) {
            const int e = e0 - lane;
            float td = 0.f;
            uint32_t ti = 0;
            const bool mv = e >= (int) pos;
            if (mv) {
                td = rd[e];
                ti = ri[e];
            }
            __syncwarp();
            if (mv) {
                rd[e + 1] = td;
                ri[e + 1] = ti;
            }
            __syncwarp();
        }
        if (lane == 0) {
            rd[pos] = sd;
            ri[pos] = si;
        }
        __syncwarp();
        if (c < C) ++c;
    }
}

// Tensor-core screen, second half: G (nr x nc, row-major) holds -2 x_r . y_c
// for rows r0.. and candidates c0..; one warp per row merges ||y_c||^2 + G
// into the row's list (global ld / li / cnt, staged in shared memory).
__global__ void __launch_bounds__(256) topk_tile_kernel(const float *__restrict__ G, uint32_t nr, uint32_t nc,
                                                        uint32_t r0, uint32_t c0, const float *__restrict__ yn,
                                                        uint32_t n, uint32_t C, float *__restrict__ gld,
                                                        uint32_t *__restrict__ gli, uint32_t *__restrict__ gcnt) {
    __shared__ float sd[8][kMaxC];
    __shared__ uint32_t si[8][kMaxC];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t rr = blockIdx.x * 8 + w;
    if (rr >= nr) return;
    const uint32_t row = r0 + rr;
    uint32_t c = gcnt[row];
    for (uint32_t e = lane; e < c; e += 32) {
        sd[w][e] = gld[(size_t) row * C + e];
        si[w][e] = gli[(size_t) row * C + e];
    }
    __syncwarp();
    const float *g = G + (size_t) rr * nc;
    for (uint32_t j0 = 0; j0 < nc; j0 += 32) {
        const uint32_t j = j0 + lane, col = c0 + j;
        const bool ok = j < nc && col < n && col != row;
        const float dv = ok ? g[j] + yn[col] : __int_as_float(0x7f800000);
        list_insert(sd[w], si[w], c, C, dv, col, lane);
    }
    for (uint32_t e = lane; e < c; e += 32) {
        gld[(size_t) row * C + e] = sd[w][e];
        gli[(size_t) row * C + e] = si[w][e];
    }
    if (lane == 0) gcnt[row] = c;
}

// Float32 screen: for each of the kBQ rows of this block, the C candidates
// (all rows but itself) with the smallest (||y||^2 - 2 x.y, id), over tiles of
// kBV candidates. 256 threads: thread (ty, tx) computes a 4 x 8 block of the
// 64 x 128 tile; then warp w inserts the tile into the lists of rows 8w..8w+7.
__global__ void __launch_bounds__(256) screen_kernel(const float *__restrict__ x, uint32_t n, uint32_t d,
                                                     const float *__restrict__ xn, uint32_t C,
                                                     uint32_t *__restrict__ out_ids) {
    extern __shared__ __align__(16) uint8_t sm[];
    float *Qs = reinterpret_cast<float *>(sm);                 // [kBK][kBQ]
    float *Vs = Qs + kBK * kBQ;                                // [kBK][kBV]
    float *D = Vs + kBK * kBV;                                 // [kBQ][kBV + 1]
    float *ld = D + kBQ * (kBV + 1);                           // [kBQ][C]
    uint32_t *li = reinterpret_cast<uint32_t *>(ld + kBQ * C); // [kBQ][C]
    uint32_t *cnt = li + kBQ * C;                              // [kBQ]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t q0 = blockIdx.x * kBQ;
    for (int i = tid; i < kBQ; i += 256) cnt[i] = 0;
    const int ty = tid / 16, tx = tid % 16;  // rows ty*4.., cols tx*8..
    __syncthreads();
    for (uint32_t v0 = 0; v0 < n; v0 += kBV) {
        float acc[4][8];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
        for (uint32_t k0 = 0; k0 < d; k0 += kBK) {
            for (int t = tid; t < kBK * kBQ; t += 256) {
                const int kk = t % kBK, qq = t / kBK;
                const uint32_t gq = q0 + qq, gk = k0 + kk;
                Qs[kk * kBQ + qq] = (gq < n && gk < d) ? x[(size_t) gq * d + gk] : 0.f;
            }
            for (int t = tid; t < kBK * kBV; t += 256) {
                const int kk = t % kBK, vv = t / kBK;
                const uint32_t gv = v0 + vv, gk = k0 + kk;
                Vs[kk * kBV + vv] = (gv < n && gk < d) ? x[(size_t) gv * d + gk] : 0.f;
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < kBK; ++kk) {
                const float4 a4 = *reinterpret_cast<const float4 *>(Qs + kk * kBQ + ty * 4);
                const float4 b4 = *reinterpret_cast<const float4 *>(Vs + kk * kBV + tx * 8);
                const float4 b5 = *reinterpret_cast<const float4 *>(Vs + kk * kBV + tx * 8 + 4);
                const float a[4] = {a4.x, a4.y, a4.z, a4.w};
                const float b[8] = {b4.x, b4.y, b4.z, b4.w, b5.x, b5.y, b5.z, b5.w};
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t gq = q0 + ty * 4 + i;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t gv = v0 + tx * 8 + j;
                const bool ok = gv < n && gv != gq;
                D[(ty * 4 + i) * (kBV + 1) + tx * 8 + j] =
                    ok ? fmaf(-2.f, acc[i][j], xn[gv]) : __int_as_float(0x7f800000);
            }
        }
        __syncthreads();
        // Insert: rows 8w..8w+7 of this warp, each candidate that beats the
        // row's current C-th (distance, id).
        for (int r = warp * 8; r < warp * 8 + 8; ++r) {
            uint32_t c = cnt[r];
            for (int j0 = 0; j0 < kBV; j0 += 32)
                list_insert(ld + r * C, li + r * C, c, C, D[r * (kBV + 1) + j0 + lane], v0 + j0 + lane, lane);
            if (lane == 0) cnt[r] = c;
            __syncwarp();
        }
        __syncthreads();
    }
    for (int r = warp; r < kBQ; r += 8) {
        const uint32_t gq = q0 + r;
        if (gq >= n) continue;
        for (uint32_t e = lane; e < C; e += 32)
            out_ids[(size_t) gq * C + e] = e < cnt[r] ? li[r * C + e] : 0xffffffffu;
    }
}

// Float32 screen restricted to cells: block b screens up to kBQ rows of cell
// blk_cell[b] (members[blk_row0[b] ..], within the cell) against the members
// of the cell itself and of its P nearest cells (near[c * P ..]), keeping per
// row the C candidates with the smallest (||y||^2 - 2 x.y, id). The same
// tiling and list insertion as screen_kernel; rows and candidates are read
// through the members list (cell by cell, ids ascending within a cell).
__global__ void __launch_bounds__(256) screen_cells_kernel(
    const float *__restrict__ x, uint32_t n, uint32_t d, const float *__restrict__ xn, uint32_t C,
    const uint32_t *__restrict__ members, const uint32_t *__restrict__ cstart, const uint32_t *__restrict__ near,
    uint32_t P, const uint32_t *__restrict__ blk_cell, const uint32_t *__restrict__ blk_row0,
    uint32_t *__restrict__ out_ids) {
    extern __shared__ __align__(16) uint8_t sm[];
    float *Qs = reinterpret_cast<float *>(sm);                 // [kBK][kBQ]
    float *Vs = Qs + kBK * kBQ;                                // [kBK][kBV]
    float *D = Vs + kBK * kBV;                                 // [kBQ][kBV + 1]
    float *ld = D + kBQ * (kBV + 1);                           // [kBQ][C]
    uint32_t *li = reinterpret_cast<uint32_t *>(ld + kBQ * C); // [kBQ][C]
    uint32_t *cnt = li + kBQ * C;                              // [kBQ]
    uint32_t *qid = cnt + kBQ;                                 // [kBQ] row ids (~0: none)
    uint32_t *vid = qid + kBQ;                                 // [kBV] candidate ids of the tile (~0: none)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t cell = blk_cell[blockIdx.x];
    const uint32_t p0 = blk_row0[blockIdx.x], pend = cstart[cell + 1];
    for (int i = tid; i < kBQ; i += 256) {
        cnt[i] = 0;
        qid[i] = p0 + i < pend ? members[p0 + i] : 0xffffffffu;
    }
    const int ty = tid / 16, tx = tid % 16;  // rows ty*4.., cols tx*8..
    __syncthreads();
    for (uint32_t sgi = 0; sgi <= P; ++sgi) {
        const uint32_t sc = sgi == 0 ? cell : near[(size_t) cell * P + sgi - 1];
        if (sc == 0xffffffffu) continue;
        const uint32_t s0 = cstart[sc], s1 = cstart[sc + 1];
        for (uint32_t v0 = s0; v0 < s1; v0 += kBV) {
            for (int i = tid; i < kBV; i += 256) vid[i] = v0 + i < s1 ? members[v0 + i] : 0xffffffffu;
            __syncthreads();
            float acc[4][8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
            for (uint32_t k0 = 0; k0 < d; k0 += kBK) {
                for (int t = tid; t < kBK * kBQ; t += 256) {
                    const int kk = t % kBK, qq = t / kBK;
                    const uint32_t gq = qid[qq], gk = k0 + kk;
                    Qs[kk * kBQ + qq] = (gq < n && gk < d) ? x[(size_t) gq * d + gk] : 0.f;
                }
                for (int t = tid; t < kBK * kBV; t += 256) {
                    const int kk = t % kBK, vv = t / kBK;
                    const uint32_t gv = vid[vv], gk = k0 + kk;
                    Vs[kk * kBV + vv] = (gv < n && gk < d) ? x[(size_t) gv * d + gk] : 0.f;
                }
                __syncthreads();
#pragma unroll
                for (int kk = 0; kk < kBK; ++kk) {
                    const float4 a4 = *reinterpret_cast<const float4 *>(Qs + kk * kBQ + ty * 4);
                    const float4 b4 = *reinterpret_cast<const float4 *>(Vs + kk * kBV + tx * 8);
                    const float4 b5 = *reinterpret_cast<const float4 *>(Vs + kk * kBV + tx * 8 + 4);
                    const float a[4] = {a4.x, a4.y, a4.z, a4.w};
                    const float b[8] = {b4.x, b4.y, b4.z, b4.w, b5.x, b5.y, b5.z, b5.w};
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
                }
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint32_t gq = qid[ty * 4 + i];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t gv = vid[tx * 8 + j];
                    const bool ok = gv < n && gv != gq;
                    D[(ty * 4 + i) * (kBV + 1) + tx * 8 + j] =
                        ok ? fmaf(-2.f, acc[i][j], xn[gv]) : __int_as_float(0x7f800000);
                }
            }
            __syncthreads();
            for (int r = warp * 8; r < warp * 8 + 8; ++r) {
                uint32_t c = cnt[r];
                for (int j0 = 0; j0 < kBV; j0 += 32)
                    list_insert(ld + r * C, li + r * C, c, C, D[r * (kBV + 1) + j0 + lane], vid[j0 + lane], lane);
                if (lane == 0) cnt[r] = c;
                __syncwarp();
            }
            __syncthreads();
        }
    }
    for (int r = warp; r < kBQ; r += 8) {
        const uint32_t gq = qid[r];
        if (gq >= n) continue;
        for (uint32_t e = lane; e < C; e += 32)
            out_ids[(size_t) gq * C + e] = e < cnt[r] ? li[r * C + e] : 0xffffffffu;
    }
}

// For every cell c (one block each), the P other cells whose centroids are
// nearest by (float64 squared distance, index); ~0 where there are fewer.
__global__ void __launch_bounds__(256) near_cells_kernel(const float *__restrict__ cent, uint32_t cells, uint32_t d,
                                                         uint32_t P, uint32_t *__restrict__ near) {
    constexpr int kMaxP = 8;
    __shared__ double bd[256 * kMaxP];
    __shared__ uint32_t bi[256 * kMaxP];
    const uint32_t c = blockIdx.x;
    double md[kMaxP];
    uint32_t mi[kMaxP];
    for (int t = 0; t < kMaxP; ++t) {
        md[t] = __longlong_as_double(0x7ff0000000000000ll);
        mi[t] = 0xffffffffu;
    }
    for (uint32_t j = threadIdx.x; j < cells; j += blockDim.x) {
        if (j == c) continue;
        double acc = 0.0;
        for (uint32_t e = 0; e < d; ++e) {
            const double t = (double) cent[(size_t) c * d + e] - (double) cent[(size_t) j * d + e];
            acc = fma(t, t, acc);
        }
        // insert (acc, j) into this thread's sorted best P
        if (acc < md[P - 1] || (acc == md[P - 1] && j < mi[P - 1])) {
            int pos = (int) P - 1;
            while (pos > 0 && (acc < md[pos - 1] || (acc == md[pos - 1] && j < mi[pos - 1]))) {
                md[pos] = md[pos - 1];
                mi[pos] = mi[pos - 1];
                --pos;
            }
            md[pos] = acc;
            mi[pos] = j;
        }
    }
    for (uint32_t t = 0; t < P; ++t) {
        bd[threadIdx.x * P + t] = md[t];
        bi[threadIdx.x * P + t] = mi[t];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t tot = blockDim.x * P;
        for (uint32_t t = 0; t < P; ++t) {  // P smallest of the block's lists
            uint32_t best = 0;
            for (uint32_t e = 1; e < tot; ++e)
                if (bd[e] < bd[best] || (bd[e] == bd[best] && bi[e] < bi[best])) best = e;
            near[(size_t) c * P + t] = bi[best];
            bd[best] = __longlong_as_double(0x7ff0000000000000ll);
            bi[best] = 0xffffffffu;
        }
    }
}

// Rows idx[0..m) of x gathered into out (m x d).
__global__ void gather_rows_f32_kernel(const float *__restrict__ x, uint32_t d, const uint32_t *__restrict__ idx,
                                       uint32_t m, float *__restrict__ out) {
    const size_t total = (size_t) m * d;
    for (size_t t = blockIdx.x * (size_t) blockDim.x + threadIdx.x; t < total; t += (size_t) gridDim.x * blockDim.x)
        out[t] = x[(size_t) idx[t / d] * d + t % d];
}

__device__ __forceinline__ double d64(const float *__restrict__ a, const float *__restrict__ b, uint32_t d) {
    double acc = 0.0;
    for (uint32_t j = 0; j < d; ++j) {
        const double t = (double) a[j] - (double) b[j];
        acc = fma(t, t, acc);
    }
    return acc;
}

// One warp per row a0 + r (r < na): float64 distances of its C screened
// candidates, ranked by (d64, id); the k best go out (ids and distances, row r
// of the chunk's knn / knn_d; a list short of k valid candidates ends in
// invalid ids, which the caller pre-sets).
__global__ void rerank_kernel(const float *__restrict__ x, uint32_t n, uint32_t d, const uint32_t *__restrict__ cand,
                              uint32_t C, uint32_t k, uint32_t a0, uint32_t na, uint32_t *__restrict__ knn,
                              double *__restrict__ knn_d) {
    __shared__ double sd[8][kMaxC];
    __shared__ uint32_t si[8][kMaxC];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t r = blockIdx.x * 8 + w;
    if (r >= na) return;
    const uint32_t a = a0 + r;
    const float *xa = x + (size_t) a * d;
    for (uint32_t e = lane; e < C; e += 32) {
        const uint32_t b = cand[(size_t) a * C + e];
        si[w][e] = b;
        sd[w][e] = b < n ? d64(xa, x + (size_t) b * d, d) : __longlong_as_double(0x7ff0000000000000ll);
    }
    __syncwarp();
    for (uint32_t e = lane; e < C; e += 32) {
        const double de = sd[w][e];
        const uint32_t ie = si[w][e];
        uint32_t rank = 0;
        for (uint32_t f = 0; f < C; ++f) {
            const double df = sd[w][f];
            const uint32_t jf = si[w][f];
            rank += (df < de || (df == de && jf < ie)) ? 1u : 0u;
        }
        if (rank < k && ie < n) {
            knn[(size_t) r * k + rank] = ie;
            knn_d[(size_t) r * k + rank] = de;
        }
    }
}

// One warp per row a0 + r (r < na): MRNG pruning of its k-NN list (row r of
// the chunk's knn / knn_d) to at most R (row r of out, deg).
__global__ void prune_kernel(const float *__restrict__ x, uint32_t n, uint32_t d, const uint32_t *__restrict__ knn,
                             const double *__restrict__ knn_d, uint32_t k, uint32_t R, uint32_t na,
                             uint32_t *__restrict__ out, uint32_t *__restrict__ deg) {
    extern __shared__ uint32_t kept_all[];  // [8][R]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t r = blockIdx.x * 8 + w;
    if (r >= na) return;
    uint32_t *kept = kept_all + w * R;
    uint32_t nk = 0;
    for (uint32_t i = 0; i < k && nk < R; ++i) {
        const uint32_t b = knn[(size_t) r * k + i];
        if (b >= n) break;
        const double dab = knn_d[(size_t) r * k + i];
        const float *xb = x + (size_t) b * d;
        bool occl = false;
        for (uint32_t c0 = 0; c0 < nk && !occl; c0 += 32) {
            const uint32_t c = c0 + lane;
            const bool o = c < nk && d64(x + (size_t) kept[c] * d, xb, d) < dab;
            occl = __any_sync(0xffffffffu, o);
        }
        if (!occl) {
            if (lane == 0) kept[nk] = b;
            __syncwarp();
            ++nk;
        }
    }
    for (uint32_t e = lane; e < nk; e += 32) out[(size_t) r * R + e] = kept[e];
    if (lane == 0) deg[r] = nk;
}

// d64 of every row to one float64 point (the mean).
__global__ void dist_to_point_kernel(const float *__restrict__ x, uint32_t n, uint32_t d,
                                     const double *__restrict__ p, double *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    double acc = 0.0;
    for (uint32_t j = 0; j < d; ++j) {
        const double t = (double) x[(size_t) r * d + j] - p[j];
        acc = fma(t, t, acc);
    }
    out[r] = acc;
}

}  // namespace

// The steps after the k-NN screen, shared by every construction: the C
// screened candidates of each row (cand, device, n x C; ~0 = none) ranked
// exactly by (d64, id) into k-NN lists, the MRNG prune to R, the entry (the
// row nearest the float64 mean of base, summed in id order) and the
// reachability repair. The rows go through the rerank and the prune in
// chunks, so the per-row float64 lists never exist for all n at once.
static int finish_graph(const float *base, const float *x, uint32_t n, uint32_t d, uint32_t k, uint32_t R,
                        const uint32_t *cand, uint32_t C, cudaStream_t s, std::unique_ptr<panns_graph> &g,
                        bool reverse = false) {
    const uint32_t chunk = std::min<uint32_t>(n, 1u << 23);
    Buf<uint32_t> knn, pr, deg;
    Buf<double> knn_d, mean, dm;
    GCU(knn.alloc((size_t) chunk * k));
    GCU(knn_d.alloc((size_t) chunk * k));
    GCU(pr.alloc((size_t) chunk * R));
    GCU(deg.alloc(chunk));
    GCU(mean.alloc(d));
    GCU(dm.alloc(n));
    g.reset(new panns_graph());
    g->n = n;
    g->k = k;
    std::vector<uint32_t> prh((size_t) n * R), degh(n);
    g->knn.resize((size_t) n * k);
    for (uint32_t a0 = 0; a0 < n; a0 += chunk) {
        const uint32_t na = std::min(chunk, n - a0);
        GCU(cudaMemsetAsync(knn.p, 0xff, (size_t) na * k * 4, s));
        rerank_kernel<<<(na + 7) / 8, 256, 0, s>>>(x, n, d, cand, C, k, a0, na, knn.p, knn_d.p);
        GCU(cudaGetLastError());
        prune_kernel<<<(na + 7) / 8, 256, 8 * R * 4, s>>>(x, n, d, knn.p, knn_d.p, k, R, na, pr.p, deg.p);
        GCU(cudaGetLastError());
        GCU(cudaMemcpyAsync(prh.data() + (size_t) a0 * R, pr.p, (size_t) na * R * 4, cudaMemcpyDeviceToHost, s));
        GCU(cudaMemcpyAsync(degh.data() + a0, deg.p, na * 4ull, cudaMemcpyDeviceToHost, s));
        GCU(cudaMemcpyAsync(g->knn.data() + (size_t) a0 * k, knn.p, (size_t) na * k * 4, cudaMemcpyDeviceToHost, s));
        GCU(cudaStreamSynchronize(s));
    }
    // Entry: float64 mean of the rows in id order (host), then the nearest row.
    std::vector<double> mh(d, 0.0);
    for (uint32_t r = 0; r < n; ++r)
        for (uint32_t j = 0; j < d; ++j) mh[j] += (double) base[(size_t) r * d + j];
    for (uint32_t j = 0; j < d; ++j) mh[j] /= (double) n;
    GCU(cudaMemcpyAsync(mean.p, mh.data(), d * 8ull, cudaMemcpyHostToDevice, s));
    dist_to_point_kernel<<<(n + 255) / 256, 256, 0, s>>>(x, n, d, mean.p, dm.p);
    GCU(cudaGetLastError());
    std::vector<double> dmh(n);
    GCU(cudaMemcpyAsync(dmh.data(), dm.p, n * 8ull, cudaMemcpyDeviceToHost, s));
    GCU(cudaStreamSynchronize(s));
    uint32_t entry = 0;
    for (uint32_t r = 1; r < n; ++r)
        if (dmh[r] < dmh[entry]) entry = r;
    g->entry = entry;
    if (reverse) {
        // Reverse edges: for every pruned edge a -> b (a ascending, then list
        // order), b -> a is appended to b's list while it holds fewer than R
        // and does not contain a already (efanna2e's InterInsert plays this
        // part, with a re-prune on overflow instead of the cap).
        const std::vector<uint32_t> deg0(degh);
        for (uint32_t a = 0; a < n; ++a) {
            const uint32_t *la = prh.data() + (size_t) a * R;
            for (uint32_t e = 0; e < deg0[a]; ++e) {
                const uint32_t b = la[e];
                uint32_t *lb = prh.data() + (size_t) b * R;
                if (degh[b] >= R || std::find(lb, lb + degh[b], a) != lb + degh[b]) continue;
                lb[degh[b]++] = a;
            }
        }
    }
    // Reachability repair from the entry over the pruned lists. A repair edge
    // parent -> u is followed at once by a walk from u, so walks never need
    // the repair edges themselves; they are appended to their parents' lists
    // (in the order they were made) when the CSR is built.
    std::vector<uint8_t> reached(n, 0);
    std::vector<uint32_t> stack;
    auto walk = [&](uint32_t src) {  // breadth-first from src over the pruned lists
        reached[src] = 1;
        stack.assign(1, src);
        for (size_t h = 0; h < stack.size(); ++h) {
            const uint32_t v = stack[h];
            const uint32_t *lv = prh.data() + (size_t) v * R;
            for (uint32_t e = 0; e < degh[v]; ++e)
                if (!reached[lv[e]]) {
                    reached[lv[e]] = 1;
                    stack.push_back(lv[e]);
                }
        }
    };
    walk(entry);
    std::vector<std::pair<uint32_t, uint32_t>> extra;  // (parent, u)
    std::vector<uint32_t> nextra(n, 0);
    for (uint32_t u = 0; u < n; ++u) {
        if (reached[u]) continue;
        uint32_t parent = entry;
        for (uint32_t i = 0; i < k; ++i) {
            const uint32_t c = g->knn[(size_t) u * k + i];
            if (c < n && reached[c]) {
                parent = c;
                break;
            }
        }
        extra.emplace_back(parent, u);
        ++nextra[parent];
        ++g->repaired;
        walk(u);
    }
    g->off.assign((size_t) n + 1, 0);
    for (uint32_t a = 0; a < n; ++a) {
        const uint32_t da = degh[a] + nextra[a];
        g->off[a + 1] = g->off[a] + da;
        g->width = std::max(g->width, da);
    }
    g->nbrs.resize(g->off[n]);
    std::vector<uint64_t> fill(n);
    for (uint32_t a = 0; a < n; ++a) {
        std::copy(prh.begin() + (size_t) a * R, prh.begin() + (size_t) a * R + degh[a], g->nbrs.begin() + g->off[a]);
        fill[a] = g->off[a] + degh[a];
    }
    for (const auto &pe : extra) g->nbrs[fill[pe.first]++] = pe.second;
    return PANNS_OK;
}

}  // namespace panns

using namespace panns;

extern "C" {

int panns_build_nsg(int device, const float *base, uint32_t n, uint32_t d, uint32_t knn_k, uint32_t R,
                    panns_graph **out) {
    return panns_build_nsg_ex(device, base, n, d, knn_k, R, PANNS_SCREEN_AUTO, out);
}

int panns_build_nsg_ex(int device, const float *base, uint32_t n, uint32_t d, uint32_t knn_k, uint32_t R,
                       uint32_t screen, panns_graph **out) {
    if (!out || !base) return set_error(PANNS_EINVAL, "panns_build_nsg: NULL argument");
    *out = nullptr;
    if (n < 2 || d == 0) return set_error(PANNS_EINVAL, "panns_build_nsg: need n >= 2, d > 0");
    if (knn_k == 0 || knn_k >= n) return set_error(PANNS_EINVAL, "panns_build_nsg: need 0 < knn_k < n");
    if (knn_k + 8 > (uint32_t) kMaxC) return set_error(PANNS_EINVAL, "panns_build_nsg: knn_k > 128 is not supported");
    if (R == 0 || R > knn_k) return set_error(PANNS_EINVAL, "panns_build_nsg: need 0 < R <= knn_k");
    if (screen > PANNS_SCREEN_TC) return set_error(PANNS_EINVAL, "panns_build_nsg: unknown screen");
    const uint32_t k = knn_k;
    const uint32_t C_tc = std::min(std::min(knn_k + 32u, (uint32_t) kMaxC), n - 1);
    if (screen == PANNS_SCREEN_AUTO)
        screen = n < 100000 ? PANNS_SCREEN_FP32
                            : tc_screen_supported(n, d, C_tc) ? PANNS_SCREEN_TC : PANNS_SCREEN_TF32;
    if (screen == PANNS_SCREEN_TC && !tc_screen_supported(n, d, C_tc))
        return set_error(PANNS_EINVAL, "panns_build_nsg: the tcgen05 screen needs d a multiple of 32 up to 128 "
                                       "and n >= 128");
    const bool tc = screen == PANNS_SCREEN_TF32;
    const bool tcg = screen == PANNS_SCREEN_TC;
    const uint32_t C = (tc || tcg) ? C_tc : std::min(std::min(knn_k + 8u, (uint32_t) kMaxC), n - 1);
    GCU(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    GCU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct SG {
        cudaStream_t s;
        ~SG() { cudaStreamDestroy(s); }
    } sg{s};
    Buf<float> x, xn;
    Buf<uint32_t> cand;
    GCU(x.alloc((size_t) n * d));
    GCU(xn.alloc(n));
    GCU(cand.alloc((size_t) n * C));
    GCU(cudaMemcpyAsync(x.p, base, (size_t) n * d * 4, cudaMemcpyHostToDevice, s));
    sqnorm32_kernel<<<(n + 255) / 256, 256, 0, s>>>(x.p, n, d, xn.p);
    if (tcg) {
        int num_sms = 0;
        GCU(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
        const int rc = tc_screen(x.p, xn.p, n, d, C, cand.p, num_sms, s);
        if (rc) return rc;
    } else if (!tc) {
        const size_t smem = (size_t) (kBK * kBQ + kBK * kBV + kBQ * (kBV + 1)) * 4 + (size_t) kBQ * C * 8 + kBQ * 4;
        GCU(cudaFuncSetAttribute(screen_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        screen_kernel<<<(n + kBQ - 1) / kBQ, 256, smem, s>>>(x.p, n, d, xn.p, C, cand.p);
        GCU(cudaGetLastError());
    } else {
        // -2 x.y for tiles of TR rows x TC candidates by TF32 tensor-core GEMMs
        // (cuBLAS, a plain library GEMM), each folded into the rows' lists.
        const uint32_t TR = std::min(n, 8192u), TC = std::min(n, 32768u);
        Buf<float> G, gld;
        Buf<uint32_t> gcnt;
        GCU(G.alloc((size_t) TR * TC));
        GCU(gld.alloc((size_t) n * C));
        GCU(gcnt.alloc(n));
        GCU(cudaMemsetAsync(gcnt.p, 0, n * 4ull, s));
        cublasHandle_t hb = nullptr;
        if (cublasCreate(&hb) != CUBLAS_STATUS_SUCCESS) return set_error(PANNS_ECUDA, "panns_build_nsg: cublasCreate failed");
        struct HB {
            cublasHandle_t h;
            ~HB() { cublasDestroy(h); }
        } hbg{hb};
        if (cublasSetStream(hb, s) != CUBLAS_STATUS_SUCCESS)
            return set_error(PANNS_ECUDA, "panns_build_nsg: cublasSetStream failed");
        const float alpha = -2.f, beta = 0.f;
        for (uint32_t r0 = 0; r0 < n; r0 += TR) {
            const uint32_t nr = std::min(TR, n - r0);
            for (uint32_t c0 = 0; c0 < n; c0 += TC) {
                const uint32_t nc = std::min(TC, n - c0);
                const cublasStatus_t st = cublasGemmEx(
                    hb, CUBLAS_OP_T, CUBLAS_OP_N, (int) nc, (int) nr, (int) d, &alpha, x.p + (size_t) c0 * d, CUDA_R_32F,
                    (int) d, x.p + (size_t) r0 * d, CUDA_R_32F, (int) d, &beta, G.p, CUDA_R_32F, (int) nc,
                    CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT);
                if (st != CUBLAS_STATUS_SUCCESS)
                    return set_error(PANNS_ECUDA, "panns_build_nsg: cublasGemmEx failed (" + std::to_string((int) st) + ")");
                topk_tile_kernel<<<(nr + 7) / 8, 256, 0, s>>>(G.p, nr, nc, r0, c0, xn.p, n, C, gld.p, cand.p, gcnt.p);
                GCU(cudaGetLastError());
            }
        }
        GCU(cudaStreamSynchronize(s));
    }
    std::unique_ptr<panns_graph> g;
    const int rc = finish_graph(base, x.p, n, d, k, R, cand.p, C, s, g);
    if (rc) return rc;
    *out = g.release();
    return PANNS_OK;
}

int panns_build_nsg_cells(int device, const float *base, uint32_t n, uint32_t d, uint32_t knn_k, uint32_t R,
                          uint32_t cells, uint32_t probe, uint32_t sample, uint32_t iters, uint32_t seed,
                          uint32_t reverse, panns_graph **out) {
    if (!out || !base) return set_error(PANNS_EINVAL, "panns_build_nsg_cells: NULL argument");
    *out = nullptr;
    if (n < 2 || d == 0) return set_error(PANNS_EINVAL, "panns_build_nsg_cells: need n >= 2, d > 0");
    if (knn_k == 0 || knn_k >= n) return set_error(PANNS_EINVAL, "panns_build_nsg_cells: need 0 < knn_k < n");
    if (knn_k + 8 > (uint32_t) kMaxC) return set_error(PANNS_EINVAL, "panns_build_nsg_cells: knn_k > 128 is not supported");
    if (R == 0 || R > knn_k) return set_error(PANNS_EINVAL, "panns_build_nsg_cells: need 0 < R <= knn_k");
    const uint32_t S = std::min(n, std::max(sample, cells));
    if (cells < 1 || cells > S) return set_error(PANNS_EINVAL, "panns_build_nsg_cells: need 1 <= cells <= sample, n");
    if (probe > 8 || (probe >= cells && cells > 1)) return set_error(PANNS_EINVAL, "panns_build_nsg_cells: need probe <= 8 and probe < cells");
    const uint32_t k = knn_k, P = cells > 1 ? probe : 0u;
    const uint32_t C = std::min(knn_k + 8u, (uint32_t) kMaxC);
    GCU(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    GCU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct SG {
        cudaStream_t s;
        ~SG() { cudaStreamDestroy(s); }
    } sg{s};
    Buf<float> x, xn;
    GCU(x.alloc((size_t) n * d));
    GCU(xn.alloc(n));
    GCU(cudaMemcpyAsync(x.p, base, (size_t) n * d * 4, cudaMemcpyHostToDevice, s));
    sqnorm32_kernel<<<(n + 255) / 256, 256, 0, s>>>(x.p, n, d, xn.p);
    GCU(cudaGetLastError());
    // Cells: Lloyd k-means on S rows at a fixed stride, then every row to its
    // nearest centroid; each cell's P nearest cells by centroid distance.
    std::vector<uint32_t> cellh(n), nearh((size_t) cells * std::max(P, 1u), 0xffffffffu);
    {
        Buf<uint32_t> sidx, sas, srep, dcell, dnear;
        Buf<float> xs, cent;
        std::vector<uint32_t> idx(S);
        for (uint32_t i = 0; i < S; ++i) idx[i] = (uint32_t) ((uint64_t) i * n / S);
        GCU(sidx.alloc(S));
        GCU(xs.alloc((size_t) S * d));
        GCU(sas.alloc(S));
        GCU(srep.alloc(cells));
        GCU(cent.alloc((size_t) cells * d));
        GCU(dcell.alloc(n));
        GCU(cudaMemcpyAsync(sidx.p, idx.data(), S * 4ull, cudaMemcpyHostToDevice, s));
        gather_rows_f32_kernel<<<1024, 256, 0, s>>>(x.p, d, sidx.p, S, xs.p);
        GCU(cudaGetLastError());
        int rc = kmeans_run(xs.p, S, d, cells, iters, seed, cent.p, sas.p, srep.p, s);
        if (rc) return rc;
        rc = nearest_centroid(x.p, n, d, cent.p, cells, dcell.p, s);
        if (rc) return rc;
        GCU(cudaMemcpyAsync(cellh.data(), dcell.p, n * 4ull, cudaMemcpyDeviceToHost, s));
        if (P) {
            GCU(dnear.alloc((size_t) cells * P));
            near_cells_kernel<<<cells, 256, 0, s>>>(cent.p, cells, d, P, dnear.p);
            GCU(cudaGetLastError());
            GCU(cudaMemcpyAsync(nearh.data(), dnear.p, (size_t) cells * P * 4, cudaMemcpyDeviceToHost, s));
        }
        GCU(cudaStreamSynchronize(s));
    }
    // Members of each cell in id order, and the screen's blocks of up to kBQ
    // rows of one cell.
    std::vector<uint32_t> cstart(cells + 1, 0), members(n), blk_cell, blk_row0;
    for (uint32_t i = 0; i < n; ++i) ++cstart[cellh[i] + 1];
    for (uint32_t c = 0; c < cells; ++c) cstart[c + 1] += cstart[c];
    {
        std::vector<uint32_t> pos(cstart.begin(), cstart.end() - 1);
        for (uint32_t i = 0; i < n; ++i) members[pos[cellh[i]]++] = i;
    }
    for (uint32_t c = 0; c < cells; ++c)
        for (uint32_t r = cstart[c]; r < cstart[c + 1]; r += kBQ) {
            blk_cell.push_back(c);
            blk_row0.push_back(r);
        }
    Buf<uint32_t> cand;
    GCU(cand.alloc((size_t) n * C));
    GCU(cudaMemsetAsync(cand.p, 0xff, (size_t) n * C * 4, s));
    {
        Buf<uint32_t> dmem, dstart, dnear, dbc, dbr;
        GCU(dmem.alloc(n));
        GCU(dstart.alloc(cells + 1));
        GCU(dnear.alloc(nearh.size()));
        GCU(dbc.alloc(blk_cell.size()));
        GCU(dbr.alloc(blk_row0.size()));
        GCU(cudaMemcpyAsync(dmem.p, members.data(), n * 4ull, cudaMemcpyHostToDevice, s));
        GCU(cudaMemcpyAsync(dstart.p, cstart.data(), (cells + 1) * 4ull, cudaMemcpyHostToDevice, s));
        GCU(cudaMemcpyAsync(dnear.p, nearh.data(), nearh.size() * 4, cudaMemcpyHostToDevice, s));
        GCU(cudaMemcpyAsync(dbc.p, blk_cell.data(), blk_cell.size() * 4, cudaMemcpyHostToDevice, s));
        GCU(cudaMemcpyAsync(dbr.p, blk_row0.data(), blk_row0.size() * 4, cudaMemcpyHostToDevice, s));
        const size_t smem = (size_t) (kBK * kBQ + kBK * kBV + kBQ * (kBV + 1)) * 4 + (size_t) kBQ * C * 8 +
                            (size_t) kBQ * 8 + (size_t) kBV * 4;
        GCU(cudaFuncSetAttribute(screen_cells_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        screen_cells_kernel<<<(unsigned) blk_cell.size(), 256, smem, s>>>(x.p, n, d, xn.p, C, dmem.p, dstart.p,
                                                                           dnear.p, P, dbc.p, dbr.p, cand.p);
        GCU(cudaGetLastError());
        GCU(cudaStreamSynchronize(s));
    }
    std::unique_ptr<panns_graph> g;
    const int rc = finish_graph(base, x.p, n, d, k, R, cand.p, C, s, g, reverse != 0);
    if (rc) return rc;
    g->cells = cells;
    g->probe = P;
    g->cell.swap(cellh);
    g->near.swap(nearh);
    *out = g.release();
    return PANNS_OK;
}

int panns_graph_cells(const panns_graph *g, uint32_t *cells, uint32_t *probe, uint32_t *cell, uint32_t *near) {
    if (!g) return set_error(PANNS_EINVAL, "panns_graph_cells: NULL graph");
    if (cells) *cells = g->cells;
    if (probe) *probe = g->probe;
    if (cell && !g->cell.empty()) memcpy(cell, g->cell.data(), g->cell.size() * 4);
    if (near && g->probe) memcpy(near, g->near.data(), (size_t) g->cells * g->probe * 4);
    return PANNS_OK;
}

int panns_graph_info(const panns_graph *g, uint32_t *n, uint32_t *width, uint32_t *entry, uint64_t *n_edges,
                     uint32_t *repaired) {
    if (!g) return set_error(PANNS_EINVAL, "panns_graph_info: NULL graph");
    if (n) *n = g->n;
    if (width) *width = g->width;
    if (entry) *entry = g->entry;
    if (n_edges) *n_edges = g->off.empty() ? 0 : g->off.back();
    if (repaired) *repaired = g->repaired;
    return PANNS_OK;
}

int panns_graph_copy(const panns_graph *g, uint64_t *offsets, uint32_t *nbrs, uint32_t *knn) {
    if (!g) return set_error(PANNS_EINVAL, "panns_graph_copy: NULL graph");
    if (offsets) memcpy(offsets, g->off.data(), g->off.size() * 8);
    if (nbrs && !g->nbrs.empty()) memcpy(nbrs, g->nbrs.data(), g->nbrs.size() * 4);
    if (knn) memcpy(knn, g->knn.data(), g->knn.size() * 4);
    return PANNS_OK;
}

int panns_graph_save_nsg(const panns_graph *g, const char *path) {
    if (!g || !path) return set_error(PANNS_EINVAL, "panns_graph_save_nsg: NULL argument");
    FILE *f = fopen(path, "wb");
    if (!f) return set_error(PANNS_EIO, std::string("panns_graph_save_nsg: cannot open ") + path);
    bool ok = fwrite(&g->width, 4, 1, f) == 1 && fwrite(&g->entry, 4, 1, f) == 1;
    for (uint32_t a = 0; ok && a < g->n; ++a) {
        const uint32_t k = (uint32_t) (g->off[a + 1] - g->off[a]);
        ok = fwrite(&k, 4, 1, f) == 1 && (k == 0 || fwrite(g->nbrs.data() + g->off[a], 4, k, f) == k);
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? PANNS_OK : set_error(PANNS_EIO, std::string("panns_graph_save_nsg: write failed: ") + path);
}

int panns_graph_free(panns_graph *g) {
    delete g;
    return PANNS_OK;
}

}  // extern "C"
