// The learned part: k-means representatives of the base and the entry /
// L-budget network's training (forward, backward, Adam) on the GPU.
//
// Training shapes are small (batch x {d, 256, R + 1}), so one generic tiled
// GEMM (tensor cores, float32 accuracy) serves every product of the forward
// and backward passes, reading the weight matrices as BF16 (the precision
// inference uses: the same GEMMs run the batched forward pass of mlp_decide).
// Everything is deterministic: fixed reduction orders, no floating-point
// atomics, a seeded sample order.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/panns_learned.h"
#include "learned.h"
#include "mlp_infer.cuh"

namespace panns {
namespace {

#define LCU(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return set_error(PANNS_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
struct Dev {
    T *p = nullptr;
    size_t n = 0;
    ~Dev() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
};

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }

// TF32 split of x: hi = x rounded to TF32, lo = the remainder rounded to TF32.
__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
    const float r = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

// c += a * b for one m16n8k8 tile (A row-major, B column-major, TF32, float32 accumulate).
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M x N] = A(M x K) * B(K x N) (+ bias[n]) (relu) (or C += when accumulate).
// A(m, k) = AT ? A[k * lda + m] : A[m * lda + k]; B(k, n) = BT ? B[n * ldb + k]
// : B[k * ldb + n]. 64 x 64 tiles staged through shared memory 32 deep, the
// next slice's loads in flight (registers) while the tensor cores work on the
// current one (split TF32, float32 accumulation); the order of every sum is
// fixed (k ascending in steps of 8), so results are deterministic.
template <typename TA, typename TB, bool AT, bool BT>
__global__ void __launch_bounds__(256) gemm_kernel(const TA *__restrict__ A, int lda, const TB *__restrict__ B,
                                                   int ldb, float *__restrict__ C, int ldc, int M, int N, int K,
                                                   const float *__restrict__ bias, int relu, int accumulate) {
    constexpr int BK = 32;
    constexpr bool kBExact = std::is_same<TB, __nv_bfloat16>::value;  // BF16 is exact in TF32
    __shared__ float As[2][BK][64 + 4];
    __shared__ float Bs[2][BK][64 + 4];
    const int tid = threadIdx.x;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    // 8 warps: warp w computes rows wm..wm+15 and columns wn..wn+31 of the tile.
    const int warp = tid >> 5, lane = tid & 31;
    const int wm = (warp & 3) * 16, wn = (warp >> 2) * 32;
    const int g = lane >> 2, tq = lane & 3;  // MMA fragment coordinates
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    // Element e = tid + 256 i of a slice: A as (m, k), B as (k, n), each in
    // the order that keeps a warp's global loads contiguous.
    float ra[8], rb[8];
    auto load = [&](int k0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = tid + 256 * i;
            const int mm = AT ? e % 64 : e / BK, kk = AT ? e / 64 : e % BK;
            const int gm = m0 + mm, gk = k0 + kk;
            ra[i] = (gm < M && gk < K) ? to_f(AT ? A[(size_t) gk * lda + gm] : A[(size_t) gm * lda + gk]) : 0.f;
            const int nn = BT ? e / BK : e % 64, kb = BT ? e % BK : e / 64;
            const int gn = n0 + nn, gkb = k0 + kb;
            rb[i] = (gn < N && gkb < K) ? to_f(BT ? B[(size_t) gn * ldb + gkb] : B[(size_t) gkb * ldb + gn]) : 0.f;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = tid + 256 * i;
            As[buf][AT ? e / 64 : e % BK][AT ? e % 64 : e / BK] = ra[i];
            Bs[buf][BT ? e % BK : e / 64][BT ? e / BK : e % 64] = rb[i];
        }
    };
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < K; k0 += BK) {
        const bool more = k0 + BK < K;
        if (more) load(k0 + BK);  // in flight during the MMAs below
        // Tensor cores: per 8-deep k step, the warp's 16 x 32 block of C as
        // four m16n8k8 TF32 MMAs. A float32 operand is split into a TF32 high
        // part and the TF32 rounding of its remainder, and the products
        // hi*hi + hi*lo + lo*hi accumulate in float32, which keeps float32
        // accuracy; a BF16 operand is exact in TF32 (no low part, one MMA less).
#pragma unroll
        for (int kk = 0; kk < BK; kk += 8) {
            uint32_t ah[4], al[4];
            {
                const float av[4] = {As[buf][kk + tq][wm + g], As[buf][kk + tq][wm + g + 8],
                                     As[buf][kk + tq + 4][wm + g], As[buf][kk + tq + 4][wm + g + 8]};
#pragma unroll
                for (int i = 0; i < 4; ++i) split_tf32(av[i], ah[i], al[i]);
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int nb = wn + nt * 8;
                uint32_t bh[2], bl[2];
                if (kBExact) {
                    bh[0] = __float_as_uint(Bs[buf][kk + tq][nb + g]);
                    bh[1] = __float_as_uint(Bs[buf][kk + tq + 4][nb + g]);
                    mma_tf32(acc[nt], ah, bh);
                    mma_tf32(acc[nt], al, bh);
                } else {
                    split_tf32(Bs[buf][kk + tq][nb + g], bh[0], bl[0]);
                    split_tf32(Bs[buf][kk + tq + 4][nb + g], bh[1], bl[1]);
                    mma_tf32(acc[nt], ah, bh);
                    mma_tf32(acc[nt], ah, bl);
                    mma_tf32(acc[nt], al, bh);
                }
            }
        }
        if (more) store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int gm = m0 + wm + g + (h >= 2 ? 8 : 0);
            const int gn = n0 + wn + nt * 8 + 2 * tq + (h & 1);
            if (gm >= M || gn >= N) continue;
            float v = acc[nt][h];
            if (bias) v += bias[gn];
            if (relu) v = fmaxf(v, 0.f);
            float *c = C + (size_t) gm * ldc + gn;
            *c = accumulate ? *c + v : v;
        }
    }
}

template <typename TA, typename TB, bool AT, bool BT>
cudaError_t gemm(const TA *A, int lda, const TB *B, int ldb, float *C, int ldc, int M, int N, int K,
                 const float *bias, int relu, cudaStream_t s) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    gemm_kernel<TA, TB, AT, BT><<<grid, 256, 0, s>>>(A, lda, B, ldb, C, ldc, M, N, K, bias, relu, 0);
    return cudaGetLastError();
}

// Block-wide reductions (blockDim.x a multiple of 32, <= 1024).
__device__ float block_max(float v, float *red) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    v = l < nw ? red[l] : PANNS_NEG_INF;
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ float block_sum(float v, float *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    v = l < nw ? red[l] : 0.f;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One block per query row: softmax cross-entropy of the R logits against the
// label histogram (T labels, 1/T each) and the L-budget squared error.
// dZ = gradient of the batch-mean loss; loss[b] = this row's loss.
__global__ void __launch_bounds__(256) loss_kernel(const float *__restrict__ Z, int R,
                                                   const uint16_t *__restrict__ cells, int T,
                                                   const float *__restrict__ y, float lam, float inv_B,
                                                   float *__restrict__ dZ, float *__restrict__ loss) {
    extern __shared__ float cnt[];  // R
    __shared__ float red[32];
    const int b = blockIdx.x;
    const float *z = Z + (size_t) b * (R + 1);
    float *g = dZ + (size_t) b * (R + 1);
    for (int j = threadIdx.x; j < R; j += blockDim.x) cnt[j] = 0.f;
    __syncthreads();
    if (threadIdx.x == 0)  // one thread: the counts are then exact and ordered
        for (int t = 0; t < T; ++t) cnt[cells[(size_t) b * T + t]] += 1.f;
    __syncthreads();
    float mx = PANNS_NEG_INF;
    for (int j = threadIdx.x; j < R; j += blockDim.x) mx = fmaxf(mx, z[j]);
    mx = block_max(mx, red);
    float se = 0.f, pz = 0.f;
    for (int j = threadIdx.x; j < R; j += blockDim.x) {
        se += expf(z[j] - mx);
        pz += cnt[j] * z[j];
    }
    se = block_sum(se, red);
    pz = block_sum(pz, red);
    const float lse = mx + logf(se);
    const float invT = 1.f / (float) T;
    for (int j = threadIdx.x; j < R; j += blockDim.x) g[j] = (expf(z[j] - lse) - cnt[j] * invT) * inv_B;
    if (threadIdx.x == 0) {
        const float e = z[R] - y[b];
        g[R] = lam * e * inv_B;
        loss[b] = lse - pz * invT + 0.5f * lam * e * e;
    }
}

__global__ void relu_bwd_kernel(float *__restrict__ dH, const float *__restrict__ H, size_t n) {
    for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
        if (!(H[i] > 0.f)) dH[i] = 0.f;
}

// db[n] = sum over the B rows of dY[., n], rows in order.
__global__ void colsum_kernel(const float *__restrict__ dY, int B, int N, float *__restrict__ db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += dY[(size_t) b * N + n];
    db[n] = s;
}

// Mean of the per-row losses, summed in row order by one thread.
__global__ void loss_mean_kernel(const float *__restrict__ loss, int B, double *__restrict__ acc) {
    if (threadIdx.x || blockIdx.x) return;
    double s = 0.0;
    for (int b = 0; b < B; ++b) s += loss[b];
    *acc += s / B;
}

__global__ void to_bf16_kernel(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, size_t n) {
    for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

// Adam with decoupled weight decay; refreshes the BF16 copy.
__global__ void adam_kernel(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ g, size_t n, float lr, float b1, float b2, float eps,
                            float wd, float c1, float c2, __nv_bfloat16 *__restrict__ wb) {
    for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n;
         i += (size_t) gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float upd = (mi / c1) / (sqrtf(vi / c2) + eps);
        const float wi = w[i] - lr * (upd + wd * w[i]);
        w[i] = wi;
        wb[i] = __float2bfloat16_rn(wi);
    }
}

// Rows idx[0..B) of X (width d), cells (width T) and y into contiguous batches.
__global__ void gather_batch_kernel(const float *__restrict__ X, int d, const uint16_t *__restrict__ cells, int T,
                                    const float *__restrict__ y, const uint32_t *__restrict__ idx, int B,
                                    float *__restrict__ Xb, uint16_t *__restrict__ cb, float *__restrict__ yb) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const size_t r = idx[b];
    for (int j = threadIdx.x; j < d; j += blockDim.x) Xb[(size_t) b * d + j] = X[r * d + j];
    for (int j = threadIdx.x; j < T; j += blockDim.x) cb[(size_t) b * T + j] = cells[r * T + j];
    if (threadIdx.x == 0) yb[b] = y[r];
}

struct Layout {
    size_t w1, b1, w2, b2, w3, b3, total;
    __host__ __device__ Layout(uint32_t d, uint32_t R) {
        w1 = 0;
        b1 = w1 + (size_t) d * kMlpH;
        w2 = b1 + kMlpH;
        b2 = w2 + (size_t) kMlpH * kMlpH;
        w3 = b2 + kMlpH;
        b3 = w3 + (size_t) kMlpH * (R + 1);
        total = b3 + R + 1;
    }
};

// Device state of one training / gradient computation at batch size B.
struct Trainer {
    uint32_t d, R, T, B;
    Layout lay;
    Dev<float> w, g, m, v, H1, H2, Z, dZ, dH2, dH1, Xb, yb, loss;
    Dev<__nv_bfloat16> wb;
    Dev<uint16_t> cb;
    Dev<double> acc;
    Trainer(uint32_t d_, uint32_t R_, uint32_t T_, uint32_t B_) : d(d_), R(R_), T(T_), B(B_), lay(d_, R_) {}

    cudaError_t alloc(bool adam) {
        cudaError_t e = cudaSuccess;
        const size_t P = lay.total;
        auto A = [&e](auto &buf, size_t n) {
            if (e == cudaSuccess) e = buf.alloc(n);
        };
        A(w, P);
        A(g, P);
        A(wb, P);
        if (adam) {
            A(m, P);
            A(v, P);
        }
        A(H1, (size_t) B * kMlpH);
        A(H2, (size_t) B * kMlpH);
        A(Z, (size_t) B * (R + 1));
        A(dZ, (size_t) B * (R + 1));
        A(dH2, (size_t) B * kMlpH);
        A(dH1, (size_t) B * kMlpH);
        A(Xb, (size_t) B * d);
        A(yb, B);
        A(loss, B);
        A(cb, (size_t) B * T);
        A(acc, 1);
        return e;
    }

    cudaError_t forward(const float *X, int rows, float *H1o, float *H2o, float *Zo, cudaStream_t s) {
        const int H = kMlpH;
        cudaError_t e = gemm<float, __nv_bfloat16, false, false>(X, d, wb.p + lay.w1, H, H1o, H, rows, H, d,
                                                                 w.p + lay.b1, 1, s);
        if (e == cudaSuccess)
            e = gemm<float, __nv_bfloat16, false, false>(H1o, H, wb.p + lay.w2, H, H2o, H, rows, H, H,
                                                         w.p + lay.b2, 1, s);
        if (e == cudaSuccess)
            e = gemm<float, __nv_bfloat16, false, false>(H2o, H, wb.p + lay.w3, R + 1, Zo, R + 1, rows, R + 1, H,
                                                         w.p + lay.b3, 0, s);
        return e;
    }

    // Loss (mean over the batch, added to acc) and gradient g of the batch in Xb, cb, yb.
    cudaError_t loss_grad(float lam, cudaStream_t s) {
        const int H = kMlpH;
        cudaError_t e = forward(Xb.p, B, H1.p, H2.p, Z.p, s);
        if (e != cudaSuccess) return e;
        loss_kernel<<<B, 256, R * sizeof(float), s>>>(Z.p, R, cb.p, T, yb.p, lam, 1.f / B, dZ.p, loss.p);
        loss_mean_kernel<<<1, 32, 0, s>>>(loss.p, B, acc.p);
        const int rb = (int) std::min<size_t>(((size_t) B * H + 255) / 256, 4096);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = gemm<float, float, true, false>(H2.p, H, dZ.p, R + 1, g.p + lay.w3, R + 1, H, R + 1, B, nullptr, 0, s);
        if (e == cudaSuccess) {
            colsum_kernel<<<(R + 1 + 255) / 256, 256, 0, s>>>(dZ.p, B, R + 1, g.p + lay.b3);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = gemm<float, __nv_bfloat16, false, true>(dZ.p, R + 1, wb.p + lay.w3, R + 1, dH2.p, H, B, H, R + 1,
                                                        nullptr, 0, s);
        if (e == cudaSuccess) {
            relu_bwd_kernel<<<rb, 256, 0, s>>>(dH2.p, H2.p, (size_t) B * H);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = gemm<float, float, true, false>(H1.p, H, dH2.p, H, g.p + lay.w2, H, H, H, B, nullptr, 0, s);
        if (e == cudaSuccess) {
            colsum_kernel<<<1, 256, 0, s>>>(dH2.p, B, H, g.p + lay.b2);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = gemm<float, __nv_bfloat16, false, true>(dH2.p, H, wb.p + lay.w2, H, dH1.p, H, B, H, H, nullptr, 0, s);
        if (e == cudaSuccess) {
            relu_bwd_kernel<<<rb, 256, 0, s>>>(dH1.p, H1.p, (size_t) B * H);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = gemm<float, float, true, false>(Xb.p, d, dH1.p, H, g.p + lay.w1, H, d, H, B, nullptr, 0, s);
        if (e == cudaSuccess) {
            colsum_kernel<<<1, 256, 0, s>>>(dH1.p, B, H, g.p + lay.b1);
            e = cudaGetLastError();
        }
        return e;
    }
};

int check_shape(uint32_t d, uint32_t R) {
    if (d == 0 || d > 256 || d % 8) return set_error(PANNS_EINVAL, "mlp: need d a multiple of 8, 8 <= d <= 256");
    if (R == 0 || R > (uint32_t) kMlpMaxR || R % kMlpH)
        return set_error(PANNS_EINVAL, "mlp: need R a multiple of 256, R <= 4096");
    return PANNS_OK;
}

int check_cells(const uint16_t *cells, size_t count, uint32_t R) {
    for (size_t i = 0; i < count; ++i)
        if (cells[i] >= R) return set_error(PANNS_EINVAL, "mlp: a cell label is >= R");
    return PANNS_OK;
}

// ---- k-means ---------------------------------------------------------------

__global__ void gather_rows_kernel(const float *__restrict__ rows, uint32_t d, const uint32_t *__restrict__ idx,
                                   uint32_t k, float *__restrict__ out) {
    const uint32_t c = blockIdx.x;
    if (c >= k) return;
    for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) out[(size_t) c * d + j] = rows[(size_t) idx[c] * d + j];
}

// Farthest-point seeding, all on the GPU. mind[s] = the squared distance of
// sample row sidx[s] to the nearest centre chosen so far; kpp_update folds
// in the newest centre (sample slot *slot).
__global__ void kpp_update_kernel(const float *__restrict__ rows, uint32_t d, const uint32_t *__restrict__ sidx,
                                  uint32_t S, const uint32_t *__restrict__ slot, float *__restrict__ mind) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= S) return;
    const float *x = rows + (size_t) sidx[t] * d;
    const float *c = rows + (size_t) sidx[*slot] * d;
    float acc = 0.f;
    for (uint32_t j = 0; j < d; ++j) {
        const float u = x[j] - c[j];
        acc = fmaf(u, u, acc);
    }
    mind[t] = fminf(mind[t], acc);
}

// One block of 1024 threads: the next centre, the sample slot with the
// largest mind (ties to the lower slot).
__global__ void __launch_bounds__(1024) kpp_pick_kernel(const float *__restrict__ mind, uint32_t S,
                                                        uint32_t *__restrict__ slot) {
    __shared__ float bv[32];
    __shared__ uint32_t bi[32];
    float best = -1.f;
    uint32_t bidx = 0xffffffffu;
    for (uint32_t i = threadIdx.x; i < S; i += blockDim.x)
        if (mind[i] > best) {  // ascending i: the lower slot wins ties
            best = mind[i];
            bidx = i;
        }
    for (int o = 16; o > 0; o >>= 1) {
        const float v2 = __shfl_xor_sync(0xffffffffu, best, o);
        const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bidx, o);
        if (v2 > best || (v2 == best && i2 < bidx)) {
            best = v2;
            bidx = i2;
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        bv[w] = best;
        bi[w] = bidx;
    }
    __syncthreads();
    if (w == 0) {
        best = bv[l];
        bidx = bi[l];
        for (int o = 16; o > 0; o >>= 1) {
            const float v2 = __shfl_xor_sync(0xffffffffu, best, o);
            const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (v2 > best || (v2 == best && i2 < bidx)) {
                best = v2;
                bidx = i2;
            }
        }
        if (l == 0) *slot = bidx < S ? bidx : 0u;
    }
}

__global__ void sqnorm_kernel(const float *__restrict__ rows, uint32_t n, uint32_t d, float *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float s = 0.f;
    for (uint32_t j = 0; j < d; ++j) s = fmaf(rows[(size_t) r * d + j], rows[(size_t) r * d + j], s);
    out[r] = s;
}

// assign[r0 + i] = argmin_c (||c||^2 - 2 G[i][c]), ties to the lower cell.
__global__ void argmin_kernel(const float *__restrict__ G, uint32_t rows, uint32_t k,
                              const float *__restrict__ cn, uint32_t *__restrict__ assign) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= rows) return;
    float best = __int_as_float(0x7f800000);
    uint32_t bi = 0xffffffffu;
    for (uint32_t c = lane; c < k; c += 32) {
        const float v = cn[c] - 2.f * G[(size_t) w * k + c];
        if (v < best) {
            best = v;
            bi = c;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float b2 = __shfl_xor_sync(0xffffffffu, best, o);
        const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        if (b2 < best || (b2 == best && i2 < bi)) {
            best = b2;
            bi = i2;
        }
    }
    if (lane == 0) assign[w] = bi < k ? bi : 0u;
}

// One block per cell: the centroid = mean of its rows (listed in id order in
// members[off[c]..off[c+1])), kept when the cell is empty; with rep != null,
// the member nearest to the centroid (exact float32 squared distance, ties to
// the lower id) instead.
__global__ void cell_kernel(const float *__restrict__ rows, uint32_t d, const uint32_t *__restrict__ members,
                            const uint32_t *__restrict__ off, float *__restrict__ cent, uint32_t *__restrict__ rep) {
    const uint32_t c = blockIdx.x;
    const uint32_t b = off[c], e = off[c + 1];
    if (!rep) {
        if (b == e) return;
        for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) {
            double s = 0.0;
            for (uint32_t i = b; i < e; ++i) s += rows[(size_t) members[i] * d + j];
            cent[(size_t) c * d + j] = (float) (s / (double) (e - b));
        }
        return;
    }
    __shared__ float bd[32];
    __shared__ uint32_t bi[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float best = __int_as_float(0x7f800000);
    uint32_t bid = 0xffffffffu;
    for (uint32_t i = b + w; i < e; i += nw) {
        const uint32_t r = members[i];
        float s = 0.f;
        for (uint32_t j = lane; j < d; j += 32) {
            const float t = rows[(size_t) r * d + j] - cent[(size_t) c * d + j];
            s = fmaf(t, t, s);
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (s < best || (s == best && r < bid)) {
            best = s;
            bid = r;
        }
    }
    if (lane == 0) {
        bd[w] = best;
        bi[w] = bid;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int t = 1; t < nw; ++t)
            if (bd[t] < bd[0] || (bd[t] == bd[0] && bi[t] < bi[0])) {
                bd[0] = bd[t];
                bi[0] = bi[t];
            }
        rep[c] = bi[0];
    }
}

}  // namespace

int kmeans_run(const float *rows, uint32_t n, uint32_t d, uint32_t k, uint32_t iters, uint32_t seed,
               float *cent, uint32_t *assign, uint32_t *rep, cudaStream_t s) {
    if (k == 0 || k > n) return set_error(PANNS_EINVAL, "kmeans: need 0 < k <= N");
    // Start: farthest-point seeding (Gonzalez, 1985) on S rows at a fixed
    // stride: a seeded first centre, then each next one the sample row
    // farthest from the centres so far (on the GPU). Far-apart clusters then
    // each get a centre before any is split, which random starts (and D^2
    // sampling, with as many centres as clusters) miss.
    std::vector<uint32_t> start(k);
    {
        const uint32_t S = (uint32_t) std::min<uint64_t>(n, std::max<uint64_t>(k, 32ull * k));
        std::vector<uint32_t> sidx(S), slots(k);
        for (uint32_t i = 0; i < S; ++i) sidx[i] = (uint32_t) ((uint64_t) i * n / S);
        std::mt19937_64 rng(seed);
        Dev<uint32_t> dsidx, dslot;
        Dev<float> mind;
        LCU(dsidx.alloc(S));
        LCU(dslot.alloc(k));
        LCU(mind.alloc(S));
        LCU(cudaMemcpyAsync(dsidx.p, sidx.data(), S * 4ull, cudaMemcpyHostToDevice, s));
        LCU(cudaMemsetAsync(mind.p, 0x7f, S * 4ull, s));  // 3.4e38: larger than any distance
        const uint32_t first = (uint32_t) (rng() % S);
        LCU(cudaMemcpyAsync(dslot.p, &first, 4, cudaMemcpyHostToDevice, s));
        for (uint32_t c = 0; c < k; ++c) {
            kpp_update_kernel<<<(S + 255) / 256, 256, 0, s>>>(rows, d, dsidx.p, S, dslot.p + c, mind.p);
            if (c + 1 < k) kpp_pick_kernel<<<1, 1024, 0, s>>>(mind.p, S, dslot.p + c + 1);
        }
        LCU(cudaGetLastError());
        LCU(cudaMemcpyAsync(slots.data(), dslot.p, k * 4ull, cudaMemcpyDeviceToHost, s));
        LCU(cudaStreamSynchronize(s));
        for (uint32_t c = 0; c < k; ++c) start[c] = sidx[slots[c]];
    }
    Dev<uint32_t> didx, doff, dmem;
    Dev<float> cn, G;
    const uint32_t chunk = std::min<uint32_t>(n, 65536);
    LCU(didx.alloc(k));
    LCU(doff.alloc(k + 1));
    LCU(dmem.alloc(n));
    LCU(cn.alloc(k));
    LCU(G.alloc((size_t) chunk * k));
    LCU(cudaMemcpyAsync(didx.p, start.data(), k * 4ull, cudaMemcpyHostToDevice, s));
    gather_rows_kernel<<<k, 128, 0, s>>>(rows, d, didx.p, k, cent);
    LCU(cudaGetLastError());
    std::vector<uint32_t> h_assign(n), off(k + 1), members(n);
    for (uint32_t it = 0; it <= iters; ++it) {
        sqnorm_kernel<<<(k + 255) / 256, 256, 0, s>>>(cent, k, d, cn.p);
        LCU(cudaGetLastError());
        for (uint32_t r0 = 0; r0 < n; r0 += chunk) {
            const uint32_t rows_c = std::min(chunk, n - r0);
            LCU((gemm<float, float, false, true>(rows + (size_t) r0 * d, d, cent, d, G.p, k, rows_c, k, d, nullptr,
                                                 0, s)));
            argmin_kernel<<<(rows_c * 32 + 255) / 256, 256, 0, s>>>(G.p, rows_c, k, cn.p, assign + r0);
            LCU(cudaGetLastError());
        }
        // Members of each cell in id order (counting sort on the host).
        LCU(cudaMemcpyAsync(h_assign.data(), assign, n * 4ull, cudaMemcpyDeviceToHost, s));
        LCU(cudaStreamSynchronize(s));
        std::fill(off.begin(), off.end(), 0u);
        for (uint32_t i = 0; i < n; ++i) ++off[h_assign[i] + 1];
        for (uint32_t c = 0; c < k; ++c) off[c + 1] += off[c];
        {
            std::vector<uint32_t> pos(off.begin(), off.end() - 1);
            for (uint32_t i = 0; i < n; ++i) members[pos[h_assign[i]]++] = i;
        }
        LCU(cudaMemcpyAsync(doff.p, off.data(), (k + 1) * 4ull, cudaMemcpyHostToDevice, s));
        LCU(cudaMemcpyAsync(dmem.p, members.data(), n * 4ull, cudaMemcpyHostToDevice, s));
        // Last round: representatives of the final cells; otherwise new centroids.
        cell_kernel<<<k, 256, 0, s>>>(rows, d, dmem.p, doff.p, cent, it == iters ? rep : nullptr);
        LCU(cudaGetLastError());
        LCU(cudaStreamSynchronize(s));  // the host vectors are rewritten next iteration
    }
    // Empty cells: give each a row that no other cell uses.
    std::vector<uint32_t> h_rep(k);
    LCU(cudaMemcpyAsync(h_rep.data(), rep, k * 4ull, cudaMemcpyDeviceToHost, s));
    LCU(cudaStreamSynchronize(s));
    std::vector<uint8_t> used(n, 0);
    bool fix = false;
    for (uint32_t c = 0; c < k; ++c)
        if (off[c + 1] > off[c]) used[h_rep[c]] = 1;
    uint32_t next = 0;
    for (uint32_t c = 0; c < k; ++c) {
        if (off[c + 1] > off[c]) continue;
        while (used[next]) ++next;
        used[next] = 1;
        h_rep[c] = next;
        fix = true;
    }
    if (fix) {
        LCU(cudaMemcpyAsync(rep, h_rep.data(), k * 4ull, cudaMemcpyHostToDevice, s));
        LCU(cudaStreamSynchronize(s));
    }
    return PANNS_OK;
}

int nearest_centroid(const float *rows, uint32_t n, uint32_t d, const float *cent, uint32_t k, uint32_t *cell,
                     cudaStream_t s) {
    Dev<float> cn, G;
    const uint32_t chunk = std::min<uint32_t>(n, std::max<uint32_t>(1024u, (uint32_t) std::min<uint64_t>(65536, (1ull << 29) / k)));
    LCU(cn.alloc(k));
    LCU(G.alloc((size_t) chunk * k));
    sqnorm_kernel<<<(k + 255) / 256, 256, 0, s>>>(cent, k, d, cn.p);
    LCU(cudaGetLastError());
    for (uint32_t r0 = 0; r0 < n; r0 += chunk) {
        const uint32_t rows_c = std::min(chunk, n - r0);
        LCU((gemm<float, float, false, true>(rows + (size_t) r0 * d, d, cent, d, G.p, k, rows_c, k, d, nullptr, 0,
                                             s)));
        argmin_kernel<<<(rows_c * 32 + 255) / 256, 256, 0, s>>>(G.p, rows_c, k, cn.p, cell + r0);
        LCU(cudaGetLastError());
    }
    LCU(cudaStreamSynchronize(s));
    return PANNS_OK;
}

int nearest_center(const float *rows, uint32_t n, uint32_t d, const uint32_t *center_rows, uint32_t k,
                   uint32_t *cell, cudaStream_t s) {
    Dev<float> cent;
    LCU(cent.alloc((size_t) k * d));
    gather_rows_kernel<<<k, 128, 0, s>>>(rows, d, center_rows, k, cent.p);
    LCU(cudaGetLastError());
    return nearest_centroid(rows, n, d, cent.p, k, cell, s);
}

namespace {
__global__ void pack_kernel(const float *__restrict__ w, uint32_t d, uint32_t R, __nv_bfloat16 *__restrict__ wbf,
                            float *__restrict__ fb) {
    const Layout lay(d, R);
    const size_t n1 = (size_t) d * kMlpH, n2 = (size_t) kMlpH * kMlpH, n3 = (size_t) kMlpH * R;
    const size_t stride = (size_t) gridDim.x * blockDim.x;
    for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n1 + n2 + n3; i += stride) {
        float v;
        if (i < n1) v = w[lay.w1 + i];
        else if (i < n1 + n2) v = w[lay.w2 + (i - n1)];
        else {
            const size_t t = i - n1 - n2, row = t / R, col = t % R;
            v = w[lay.w3 + row * (R + 1) + col];
        }
        wbf[i] = __float2bfloat16_rn(v);
    }
    // fb: b1 (256), b2 (256), b3 (R), wl (256), bl (1)
    for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < 3u * kMlpH + R + 1; i += stride) {
        float v;
        if (i < kMlpH) v = w[lay.b1 + i];
        else if (i < 2u * kMlpH) v = w[lay.b2 + (i - kMlpH)];
        else if (i < 2u * kMlpH + R) v = w[lay.b3 + (i - 2u * kMlpH)];
        else if (i < 3u * kMlpH + R) v = w[lay.w3 + (i - 2u * kMlpH - R) * (R + 1) + R];
        else v = w[lay.b3 + R];
        fb[i] = v;
    }
}
}  // namespace

int mlp_pack_inference(const float *params_dev, uint32_t d, uint32_t R, void *wbf, float *fb, cudaStream_t s) {
    pack_kernel<<<256, 256, 0, s>>>(params_dev, d, R, reinterpret_cast<__nv_bfloat16 *>(wbf), fb);
    LCU(cudaGetLastError());
    return PANNS_OK;
}

namespace {
// X[q][i] = query q's element i, from the chain-major rows (width dpad).
__global__ void rows_from_chain_major_kernel(const float *__restrict__ q_cm, uint32_t dpad, uint32_t d, uint32_t nq,
                                             float *__restrict__ X) {
    const size_t total = (size_t) nq * d;
    for (size_t t = blockIdx.x * (size_t) blockDim.x + threadIdx.x; t < total; t += (size_t) gridDim.x * blockDim.x) {
        const size_t q = t / d;
        const uint32_t i = (uint32_t) (t - q * d);
        X[t] = q_cm[q * dpad + chain_major_index(d, i)];
    }
}

// The regressor output r = wl . h2 + bl of one query (lane t holds hidden
// units 8t..8t+7), reduced over the warp.
__device__ __forceinline__ float regressor(const MlpDev &m, const float *__restrict__ h2, int lane) {
    const float *h = h2 + lane * 8;
    float r = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) r = fmaf(m.wl[lane * 8 + j], h[j], r);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    return r + m.bl;
}

// Queue length and fallback of one query from its confidence and regressor.
__device__ __forceinline__ uint32_t decide_L(const MlpDev &m, float conf, float r, uint32_t Lc, uint32_t K,
                                             bool &fallback) {
    fallback = !(conf >= m.min_conf);
    uint32_t Lq = Lc;
    if (!fallback && m.use_L) {
        const float x = m.L_scale * expf(m.L_exp * r);
        const uint32_t lo = max(K, min(m.L_min, Lc));
        if (x < (float) Lc) Lq = max(lo, (uint32_t) ceilf(fmaxf(x, 0.f)));
    }
    return Lq;
}

// Warp argmax of (best, bi) pairs, ties to the lower index.
__device__ __forceinline__ void warp_argmax(float &best, uint32_t &bi) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float b2 = __shfl_xor_sync(0xffffffffu, best, o);
        const uint32_t i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        if (b2 > best || (b2 == best && i2 < bi)) {
            best = b2;
            bi = i2;
        }
    }
}

// One warp per query: the decision from its logits Z[q] (R) and its second
// hidden layer H2[q] (256). Up to 1,024 classes the logits sit in registers
// (lane t owns logits t, t + 32, ...); beyond, they are read from Z (scratch)
// once per pass, and chosen ones are overwritten with -inf there.
template <bool REGS>
__global__ void __launch_bounds__(256) decide_kernel(MlpDev m, const float *__restrict__ H2, float *__restrict__ Z,
                                                     uint32_t nq, uint32_t L, const uint32_t *__restrict__ Lq_in,
                                                     uint32_t K, uint32_t *__restrict__ record) {
    constexpr int NC = REGS ? 32 : 1;  // logits per lane held in registers
    const int lane = threadIdx.x & 31;
    const uint32_t q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= nq) return;
    const uint32_t R = m.R, nc = R / 32;
    const float r = regressor(m, H2 + (size_t) q * kMlpH, lane);
    float *z = Z + (size_t) q * R;
    float v[NC];
    float mx = PANNS_NEG_INF;
    if (REGS) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            v[c] = (uint32_t) c < nc ? z[c * 32 + lane] : PANNS_NEG_INF;
            mx = fmaxf(mx, v[c]);
        }
    } else {
        for (uint32_t c = 0; c < nc; ++c) mx = fmaxf(mx, z[c * 32 + lane]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float se = 0.f;
    if (REGS) {
#pragma unroll
        for (int c = 0; c < NC; ++c)
            if ((uint32_t) c < nc) se += expf(v[c] - mx);
    } else {
        for (uint32_t c = 0; c < nc; ++c) se += expf(z[c * 32 + lane] - mx);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    const float conf = 1.f / se;  // softmax probability of the largest logit
    bool fallback;
    const uint32_t Lq = decide_L(m, conf, r, Lq_in ? Lq_in[q] : L, K, fallback);
    uint32_t *rec = record + (size_t) q * kMlpRecWords;
    uint32_t E = 0;
    if (!fallback && m.use_entry) {
        // The E largest logits, one warp argmax each (ties to the lower index).
        const uint32_t want = min(min(m.E, (uint32_t) kMlpMaxE), Lq);
        for (; E < want; ++E) {
            float best = PANNS_NEG_INF;
            uint32_t bi = 0xffffffffu;
            if (REGS) {
#pragma unroll
                for (int c = 0; c < NC; ++c)
                    if (v[c] > best) {
                        best = v[c];
                        bi = c * 32 + lane;
                    }
            } else {
                for (uint32_t c = 0; c < nc; ++c) {
                    const float x = z[c * 32 + lane];
                    if (x > best) {
                        best = x;
                        bi = c * 32 + lane;
                    }
                }
            }
            warp_argmax(best, bi);
            if (bi >= R) break;  // only -inf or NaN left
            if (lane == 0) rec[2 + E] = __ldg(m.rep + bi);
            if (lane == (int) (bi & 31)) {
                if (REGS) {
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        if ((uint32_t) c == (bi >> 5)) v[c] = PANNS_NEG_INF;
                } else {
                    z[bi] = PANNS_NEG_INF;
                }
            }
            __syncwarp();
        }
    }
    if (lane == 0) {
        rec[0] = Lq | (fallback ? 0x80000000u : 0u);
        rec[1] = E;
    }
}
}  // namespace

cudaError_t mlp_decide(const MlpDev &m, const float *q_cm, uint32_t dpad, uint32_t nq, uint32_t L, const uint32_t *Lq,
                       uint32_t K, const MlpScratch &w, uint32_t *record, cudaStream_t s) {
    const int H = kMlpH, d = (int) m.d, R = (int) m.R;
    cudaError_t e = cudaSuccess;
    for (uint32_t r0 = 0; r0 < nq && e == cudaSuccess; r0 += w.rows) {
        const uint32_t rows = std::min(w.rows, nq - r0);
        const size_t total = (size_t) rows * m.d;
        rows_from_chain_major_kernel<<<(unsigned) std::min<size_t>((total + 255) / 256, 4096), 256, 0, s>>>(
            q_cm + (size_t) r0 * dpad, dpad, m.d, rows, w.X);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = gemm<float, __nv_bfloat16, false, false>(w.X, d, m.w1, H, w.H1, H, (int) rows, H, d, m.b1, 1, s);
        if (e == cudaSuccess)
            e = gemm<float, __nv_bfloat16, false, false>(w.H1, H, m.w2, H, w.H2, H, (int) rows, H, H, m.b2, 1, s);
        if (e == cudaSuccess)
            e = gemm<float, __nv_bfloat16, false, false>(w.H2, H, m.w3, R, w.Z, R, (int) rows, R, H, m.b3, 0, s);
        if (e == cudaSuccess) {
            if (m.R <= 1024)
                decide_kernel<true><<<(rows + 7) / 8, 256, 0, s>>>(m, w.H2, w.Z, rows, L, Lq ? Lq + r0 : nullptr, K,
                                                                   record + (size_t) r0 * kMlpRecWords);
            else
                decide_kernel<false><<<(rows + 7) / 8, 256, 0, s>>>(m, w.H2, w.Z, rows, L, Lq ? Lq + r0 : nullptr, K,
                                                                    record + (size_t) r0 * kMlpRecWords);
            e = cudaGetLastError();
        }
    }
    return e;
}

}  // namespace panns

using namespace panns;

extern "C" {

uint64_t panns_mlp_param_count(uint32_t d, uint32_t R) { return Layout(d, R).total; }

int panns_mlp_loss_grad(int device, uint32_t d, uint32_t R, uint32_t T, const float *params, const float *X,
                        const uint16_t *cells, const float *y, uint32_t B, float lambda_L, float *grad,
                        double *loss) {
    int rc = check_shape(d, R);
    if (rc) return rc;
    if (!params || !X || !cells || !y || !grad || !loss || B == 0 || T == 0)
        return set_error(PANNS_EINVAL, "panns_mlp_loss_grad: NULL argument or empty batch");
    rc = check_cells(cells, (size_t) B * T, R);
    if (rc) return rc;
    LCU(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    LCU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{s};
    Trainer t(d, R, T, B);
    LCU(t.alloc(false));
    const size_t P = t.lay.total;
    LCU(cudaMemcpyAsync(t.w.p, params, P * 4, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpyAsync(t.Xb.p, X, (size_t) B * d * 4, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpyAsync(t.cb.p, cells, (size_t) B * T * 2, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpyAsync(t.yb.p, y, (size_t) B * 4, cudaMemcpyHostToDevice, s));
    LCU(cudaMemsetAsync(t.acc.p, 0, 8, s));
    to_bf16_kernel<<<256, 256, 0, s>>>(t.w.p, t.wb.p, P);
    LCU(cudaGetLastError());
    LCU(t.loss_grad(lambda_L, s));
    LCU(cudaMemcpyAsync(grad, t.g.p, P * 4, cudaMemcpyDeviceToHost, s));
    LCU(cudaMemcpyAsync(loss, t.acc.p, 8, cudaMemcpyDeviceToHost, s));
    LCU(cudaStreamSynchronize(s));
    return PANNS_OK;
}

int panns_mlp_forward(int device, uint32_t d, uint32_t R, const float *params, const float *X, uint32_t n,
                      float *Z) {
    int rc = check_shape(d, R);
    if (rc) return rc;
    if (!params || (n && (!X || !Z))) return set_error(PANNS_EINVAL, "panns_mlp_forward: NULL argument");
    if (n == 0) return PANNS_OK;
    LCU(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    LCU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{s};
    const uint32_t B = std::min<uint32_t>(n, 8192);
    Trainer t(d, R, 1, B);
    LCU(t.alloc(false));
    const size_t P = t.lay.total;
    LCU(cudaMemcpyAsync(t.w.p, params, P * 4, cudaMemcpyHostToDevice, s));
    to_bf16_kernel<<<256, 256, 0, s>>>(t.w.p, t.wb.p, P);
    LCU(cudaGetLastError());
    for (uint32_t r0 = 0; r0 < n; r0 += B) {
        const uint32_t rows = std::min(B, n - r0);
        LCU(cudaMemcpyAsync(t.Xb.p, X + (size_t) r0 * d, (size_t) rows * d * 4, cudaMemcpyHostToDevice, s));
        LCU(t.forward(t.Xb.p, (int) rows, t.H1.p, t.H2.p, t.Z.p, s));
        LCU(cudaMemcpyAsync(Z + (size_t) r0 * (R + 1), t.Z.p, (size_t) rows * (R + 1) * 4, cudaMemcpyDeviceToHost,
                            s));
        LCU(cudaStreamSynchronize(s));
    }
    return PANNS_OK;
}

int panns_mlp_train(int device, const panns_mlp_train_params *tp, const float *X, const uint16_t *cells,
                    const float *y, uint32_t n, float *params, double *epoch_loss) {
    if (!tp) return set_error(PANNS_EINVAL, "panns_mlp_train: NULL params");
    int rc = check_shape(tp->d, tp->R);
    if (rc) return rc;
    if (!X || !cells || !y || !params) return set_error(PANNS_EINVAL, "panns_mlp_train: NULL argument");
    if (tp->batch == 0 || tp->batch > n || tp->T == 0)
        return set_error(PANNS_EINVAL, "panns_mlp_train: need 0 < batch <= n and T > 0");
    rc = check_cells(cells, (size_t) n * tp->T, tp->R);
    if (rc) return rc;
    const uint32_t d = tp->d, R = tp->R, T = tp->T, B = tp->batch;
    LCU(cudaSetDevice(device));
    cudaStream_t s = nullptr;
    LCU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{s};
    Trainer t(d, R, T, B);
    LCU(t.alloc(true));
    const size_t P = t.lay.total;
    Dev<float> dX, dy;
    Dev<uint16_t> dc;
    Dev<uint32_t> didx;
    LCU(dX.alloc((size_t) n * d));
    LCU(dy.alloc(n));
    LCU(dc.alloc((size_t) n * T));
    LCU(didx.alloc(n));
    LCU(cudaMemcpyAsync(dX.p, X, (size_t) n * d * 4, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpyAsync(dy.p, y, (size_t) n * 4, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpyAsync(dc.p, cells, (size_t) n * T * 2, cudaMemcpyHostToDevice, s));
    LCU(cudaMemcpyAsync(t.w.p, params, P * 4, cudaMemcpyHostToDevice, s));
    LCU(cudaMemsetAsync(t.m.p, 0, P * 4, s));
    LCU(cudaMemsetAsync(t.v.p, 0, P * 4, s));
    to_bf16_kernel<<<256, 256, 0, s>>>(t.w.p, t.wb.p, P);
    LCU(cudaGetLastError());
    std::vector<uint32_t> order(n);
    std::mt19937_64 rng(tp->seed);
    const uint32_t nb = n / B;
    uint64_t step = 0;
    double c1p = 1.0, c2p = 1.0;
    for (uint32_t ep = 0; ep < tp->epochs; ++ep) {
        std::iota(order.begin(), order.end(), 0u);
        for (uint32_t i = n - 1; i > 0; --i) std::swap(order[i], order[rng() % (i + 1)]);
        LCU(cudaMemcpyAsync(didx.p, order.data(), (size_t) n * 4, cudaMemcpyHostToDevice, s));
        LCU(cudaMemsetAsync(t.acc.p, 0, 8, s));
        for (uint32_t b = 0; b < nb; ++b) {
            gather_batch_kernel<<<B, 128, 0, s>>>(dX.p, d, dc.p, T, dy.p, didx.p + (size_t) b * B, B, t.Xb.p, t.cb.p,
                                                  t.yb.p);
            LCU(cudaGetLastError());
            LCU(t.loss_grad(tp->lambda_L, s));
            ++step;
            c1p *= tp->beta1;
            c2p *= tp->beta2;
            adam_kernel<<<512, 256, 0, s>>>(t.w.p, t.m.p, t.v.p, t.g.p, P, tp->lr, tp->beta1, tp->beta2, tp->eps,
                                            tp->weight_decay, (float) (1.0 - c1p), (float) (1.0 - c2p), t.wb.p);
            LCU(cudaGetLastError());
        }
        // The order vector is rewritten next epoch: wait for its copy.
        double l = 0.0;
        LCU(cudaMemcpyAsync(&l, t.acc.p, 8, cudaMemcpyDeviceToHost, s));
        LCU(cudaStreamSynchronize(s));
        if (epoch_loss) epoch_loss[ep] = nb ? l / nb : 0.0;
    }
    LCU(cudaMemcpyAsync(params, t.w.p, P * 4, cudaMemcpyDeviceToHost, s));
    LCU(cudaStreamSynchronize(s));
    (void) step;
    return PANNS_OK;
}

}  // extern "C"
