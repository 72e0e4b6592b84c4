// k-NN screen of the graph construction on the 5th-generation tensor cores.
//
// For every row x of the base it keeps the C candidates y != x with the
// smallest screen distance ||y||^2 - 2 x.y (||x||^2 is the same for the whole
// row and left out); graph_build.cu then ranks the C candidates exactly in
// float64, as for its other screens. The contraction x.y runs as TF32
// tcgen05.mma with float32 accumulation in tensor memory, and the selection
// runs in the epilogue, so no tile of distances is ever written to memory
// (the cuBLAS screen writes and reads every one, O(n^2) bytes).
//
// One persistent CTA per SM owns blocks of 128 rows, one at a time, and
// sweeps every column for them in tiles of 64 rows of the base (the "B" tiles):
//   warp 4   TMA producer: the row block's 128 x d operand once ("A"), then
//            the B tiles through a ring of S shared-memory stages;
//   warp 5   one elected thread issues the MMAs (M = 128, N = 64, K = 8
//            each, d / 8 per tile) into one of two TMEM accumulators of 64
//            columns, and commits them to the stage's and the accumulator's
//            mbarriers;
//   warps 0-3 epilogue: thread t of warp w owns row 32 w + t (TMEM lane), reads
//            its 64 accumulators with one tcgen05.ld, frees the accumulator and
//            keeps the C best (distance, id) in a max-heap in shared memory.
// Operands are K-major with the 128-byte swizzle: each 32-float slice of d is
// one TMA box, 128 rows (A) or 64 rows (B) of 128 bytes, and an MMA's K step
// advances the descriptor's start address by 32 bytes inside the slice.
// Every wait on an mbarrier is bounded: on expiry the kernel records an error,
// every role stops, and the CTA still releases its tensor memory.
//
// No multicast anywhere: every TMA load reads this GPU's own base copy.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "../../include/panns_b200.h"
#include "learned.h"
#include "tc_screen.h"

namespace panns {
namespace {

constexpr uint32_t kTcM = 128;        // rows per block (TMEM lanes)
constexpr uint32_t kTcN = 64;         // columns per tile
constexpr uint32_t kTcSlice = 32;     // floats per TMA box row (128 bytes)
constexpr uint32_t kTcThreads = 192;  // 4 epilogue warps, producer, MMA issuer
constexpr uint32_t kTcTmemCols = 128; // two accumulators of 64 columns
constexpr uint32_t kTcMaxWait = 1u << 24;

enum : uint32_t { TC_ERR_TIMEOUT = 1u };

struct TcArgs {
    const float *yn;   // ||y||^2 of every row of the base
    uint32_t n, d, C, slices, stages;
    uint32_t *cand;    // n x C candidate ids
    uint32_t *error;
};

struct TcSmem {  // offsets into the dynamic shared memory (bytes)
    uint32_t a, b, heap_d, heap_i, bar, total;
};

__host__ __device__ inline TcSmem tc_layout(uint32_t slices, uint32_t stages, uint32_t C) {
    TcSmem s;
    s.a = 0;                                              // slices x 16 KB
    s.b = s.a + slices * kTcM * 128;                      // stages x slices x 8 KB
    s.heap_d = s.b + stages * slices * kTcN * 128;        // C x 128 floats
    s.heap_i = s.heap_d + C * kTcM * 4;                   // C x 128 ids
    s.bar = (s.heap_i + C * kTcM * 4 + 7) & ~7u;          // mbarriers + TMEM address
    s.total = s.bar + 8 * (2 + 2 * 8 + 4) + 16;
    return s;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Wait for the phase of parity `parity` to complete; false after kTcMaxWait
// tries (the caller records the error and stops).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < kTcMaxWait; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"((uint64_t) map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart, Blackwell descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t desc = 0;
    desc |= (uint64_t) ((saddr & 0x3FFFFu) >> 4);   // start address
    desc |= (uint64_t) 1 << 16;                     // leading byte offset (unused with this swizzle)
    desc |= (uint64_t) (1024 >> 4) << 32;           // stride byte offset
    desc |= (uint64_t) 1 << 46;                     // version
    desc |= (uint64_t) 2 << 61;                     // SWIZZLE_128B
    return desc;
}

// Instruction descriptor: D float32, A and B TF32, both K-major, N = 64, M = 128.
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((kTcN >> 3) << 17) | ((kTcM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %4, p;\n\t}"
        ::"r"(tmem), "l"(da), "l"(db), "r"(accumulate), "r"(kTcIdesc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&v)[64]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
        "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
        "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]),
          "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]),
          "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]),
          "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]),
          "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Max-heap of the row's best C (distance, id), stored column-major (entry e
// of thread r at e * 128 + r) so that the threads of a warp hit distinct banks.
__device__ __forceinline__ bool key_gt(float ad, uint32_t ai, float bd, uint32_t bi) {
    return ad > bd || (ad == bd && ai > bi);
}

__device__ __forceinline__ void heap_replace_top(float *hd, uint32_t *hi, uint32_t C, uint32_t r, float dv,
                                                 uint32_t iv) {
    uint32_t i = 0;
    for (;;) {
        const uint32_t l = 2 * i + 1;
        if (l >= C) break;
        uint32_t m = l;
        float md = hd[l * kTcM + r];
        uint32_t mi = hi[l * kTcM + r];
        if (l + 1 < C) {
            const float rd = hd[(l + 1) * kTcM + r];
            const uint32_t ri = hi[(l + 1) * kTcM + r];
            if (key_gt(rd, ri, md, mi)) {
                m = l + 1;
                md = rd;
                mi = ri;
            }
        }
        if (!key_gt(md, mi, dv, iv)) break;
        hd[i * kTcM + r] = md;
        hi[i * kTcM + r] = mi;
        i = m;
    }
    hd[i * kTcM + r] = dv;
    hi[i * kTcM + r] = iv;
}

template <bool FUSED>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_screen_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     TcArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t) 1023);
    const TcSmem L = tc_layout(a.slices, a.stages, a.C);
    uint8_t *sa = smem + L.a;
    uint8_t *sb = smem + L.b;
    float *hd = reinterpret_cast<float *>(smem + L.heap_d);
    uint32_t *hi = reinterpret_cast<uint32_t *>(smem + L.heap_i);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L.bar);
    uint64_t *a_full = bars, *a_empty = bars + 1;
    uint64_t *b_full = bars + 2, *b_empty = bars + 2 + 8;
    uint64_t *t_full = bars + 18, *t_empty = bars + 20;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 22);
    volatile uint32_t *abort_flag = tmem_slot + 1;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row_blocks = (a.n + kTcM - 1) / kTcM;
    const uint32_t col_tiles = (a.n + kTcN - 1) / kTcN;
    const uint32_t a_bytes = a.slices * kTcM * 128, b_bytes = a.slices * kTcN * 128;

    if (threadIdx.x == 0) {
        mbar_init(a_full, 1);
        mbar_init(a_empty, 1);
        for (uint32_t s = 0; s < a.stages; ++s) {
            mbar_init(b_full + s, 1);
            mbar_init(b_empty + s, 1);
        }
        for (int t = 0; t < 2; ++t) {
            mbar_init(t_full + t, 1);
            mbar_init(t_empty + t, 4);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    auto fail = [&]() {
        atomicOr(a.error, TC_ERR_TIMEOUT);
        *abort_flag = 1;
    };

    if (warp == 4) {
        // ---- TMA producer ----
        if (lane == 0) {
            uint32_t g = 0, rbi = 0;
            for (uint32_t rb = blockIdx.x; rb < row_blocks && !*abort_flag; rb += gridDim.x, ++rbi) {
                if (!mbar_wait(a_empty, (rbi & 1) ^ 1)) { fail(); break; }
                mbar_expect_tx(a_full, a_bytes);
                for (uint32_t sl = 0; sl < a.slices; ++sl)
                    tma_load_2d(sa + sl * kTcM * 128, &map_a, a_full, (int32_t) (sl * kTcSlice), (int32_t) (rb * kTcM));
                for (uint32_t ct = 0; ct < col_tiles; ++ct, ++g) {
                    const uint32_t s = g % a.stages, ph = (g / a.stages) & 1;
                    if (!mbar_wait(b_empty + s, ph ^ 1)) { fail(); break; }
                    if (*abort_flag) break;
                    mbar_expect_tx(b_full + s, b_bytes);
                    uint8_t *dst = sb + s * b_bytes;
                    for (uint32_t sl = 0; sl < a.slices; ++sl)
                        tma_load_2d(dst + sl * kTcN * 128, &map_b, b_full + s, (int32_t) (sl * kTcSlice),
                                    (int32_t) (ct * kTcN));
                }
            }
        }
    } else if (warp == 5) {
        // ---- MMA issuer ----
        if (lane == 0) {
            uint32_t g = 0, rbi = 0;
            for (uint32_t rb = blockIdx.x; rb < row_blocks && !*abort_flag; rb += gridDim.x, ++rbi) {
                if (!mbar_wait(a_full, rbi & 1)) { fail(); break; }
                for (uint32_t ct = 0; ct < col_tiles; ++ct, ++g) {
                    const uint32_t s = g % a.stages, ph = (g / a.stages) & 1;
                    const uint32_t t = g & 1, tph = (g >> 1) & 1;
                    if (!mbar_wait(t_empty + t, tph ^ 1)) { fail(); break; }
                    if (!mbar_wait(b_full + s, ph)) { fail(); break; }
                    if (*abort_flag) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t abase = smem_u32(sa), bbase = smem_u32(sb + s * b_bytes);
                    for (uint32_t sl = 0; sl < a.slices; ++sl)
                        for (uint32_t ks = 0; ks < 4; ++ks)
                            umma_tf32(tmem + t * kTcN, umma_desc(abase + sl * kTcM * 128 + ks * 32),
                                      umma_desc(bbase + sl * kTcN * 128 + ks * 32), (sl | ks) != 0);
                    umma_commit(b_empty + s);
                    umma_commit(t_full + t);
                }
                umma_commit(a_empty);
            }
        }
    } else {
        // ---- epilogue: warps 0-3, thread r = 32 w + lane owns row r of the block ----
        const uint32_t r = warp * 32 + lane;
        uint32_t g = 0;
        for (uint32_t rb = blockIdx.x; rb < row_blocks && !*abort_flag; rb += gridDim.x) {
            const uint32_t row = rb * kTcM + r;
            for (uint32_t e = 0; e < a.C; ++e) {
                hd[e * kTcM + r] = __int_as_float(0x7f800000);
                hi[e * kTcM + r] = 0xffffffffu;
            }
            for (uint32_t ct = 0; ct < col_tiles; ++ct, ++g) {
                const uint32_t t = g & 1, tph = (g >> 1) & 1;
                const uint32_t c0 = ct * kTcN;
                // the 64 columns' norms, two per lane (already in the accumulators when FUSED)
                const float y0 = !FUSED && c0 + lane < a.n ? __ldg(a.yn + c0 + lane) : 0.f;
                const float y1 = !FUSED && c0 + 32 + lane < a.n ? __ldg(a.yn + c0 + 32 + lane) : 0.f;
                bool ok = mbar_wait(t_full + t, tph);
                ok = __all_sync(0xffffffffu, ok);
                if (!ok) {
                    if (lane == 0) fail();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                uint32_t v[64];
                tmem_ld64(tmem + ((warp * 32) << 16) + t * kTcN, v);
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(t_empty + t);
                // Screen distances, and a bit per column that beats the
                // heap's top (the current C-th best) before this tile.
                const float top_d = hd[r];
                uint64_t beat;
                if constexpr (FUSED) {
                    // the accumulators hold ||y||^2 - 2 x.y; a distance equal to
                    // the top's is decided by id in the insertion loop
                    uint32_t lo = 0, hi32 = 0;
#pragma unroll
                    for (int j = 0; j < 32; ++j) lo |= (uint32_t) (__uint_as_float(v[j]) <= top_d) << j;
#pragma unroll
                    for (int j = 0; j < 32; ++j) hi32 |= (uint32_t) (__uint_as_float(v[32 + j]) <= top_d) << j;
                    beat = ((uint64_t) hi32 << 32) | lo;
                } else {
                    const uint32_t top_i = hi[r];
                    beat = 0;
#pragma unroll
                    for (int j = 0; j < 64; ++j) {
                        const float yj = __shfl_sync(0xffffffffu, j < 32 ? y0 : y1, j & 31);
                        const float sd = fmaf(-2.f, __uint_as_float(v[j]), yj);
                        v[j] = __float_as_uint(sd);
                        beat |= (uint64_t) key_gt(top_d, top_i, sd, c0 + j) << j;
                    }
                }
                if (row >= a.n) beat = 0;
                const uint32_t self = row - c0;  // the row's own column, if in this tile
                if (self < 64) beat &= ~(1ull << self);
                if (c0 + 64 > a.n) beat &= a.n - c0 >= 64 ? ~0ull : ((1ull << (a.n - c0)) - 1);
                // Insertions, in column order (each rechecked against the top).
                while (beat) {
                    const int j = __ffsll((long long) beat) - 1;
                    beat &= beat - 1;
                    float sd = 0.f;
#pragma unroll
                    for (int t = 0; t < 64; ++t)
                        if (t == j) sd = __uint_as_float(v[t]);
                    if (key_gt(hd[r], hi[r], sd, c0 + j)) heap_replace_top(hd, hi, a.C, r, sd, c0 + j);
                }
            }
            if (*abort_flag) break;
            if (row < a.n)
                for (uint32_t e = 0; e < a.C; ++e) a.cand[(size_t) row * a.C + e] = hi[e * kTcM + r];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
    }
}

// Rows with the norm folded into the contraction: xa = [x, 1, 1, 0...] and
// xb = [-2x, hi, lo, 0...] (width w), hi = ||x||^2 cut to TF32 (exact in the
// MMA), lo = the rest, so that xa_i . xb_j = ||x_j||^2 - 2 x_i . x_j.
__global__ void augment_kernel(const float *__restrict__ x, const float *__restrict__ xn, uint32_t n, uint32_t d,
                               uint32_t w, float *__restrict__ xa, float *__restrict__ xb) {
    const uint64_t total = (uint64_t) n * w;
    for (uint64_t t = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; t < total;
         t += (uint64_t) gridDim.x * blockDim.x) {
        const uint64_t r = t / w;
        const uint32_t c = (uint32_t) (t % w);
        float va = 0.f, vb = 0.f;
        if (c < d) {
            va = x[r * d + c];
            vb = -2.f * va;
        } else if (c == d || c == d + 1) {
            va = 1.f;
            const float y2 = xn[r];
            const float hi = __uint_as_float(__float_as_uint(y2) & 0xffffe000u);
            vb = c == d ? hi : y2 - hi;
        }
        xa[t] = va;
        xb[t] = vb;
    }
}

int make_map(CUtensorMap *map, const float *x, uint32_t n, uint32_t d, uint32_t box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return set_error(PANNS_ECUDA, "tc screen: cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[2] = {d, n};
    const cuuint64_t strides[1] = {(cuuint64_t) d * 4};
    const cuuint32_t box[2] = {kTcSlice, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(x), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(PANNS_ECUDA, "tc screen: cuTensorMapEncodeTiled failed (" + std::to_string((int) r) + ")");
    return PANNS_OK;
}

}  // namespace

bool tc_screen_supported(uint32_t n, uint32_t d, uint32_t C) {
    return d % kTcSlice == 0 && d >= kTcSlice && d <= 128 && C >= 1 && C <= 128 && C < n && n >= kTcM;
}

int tc_screen(const float *x, const float *xn, uint32_t n, uint32_t d, uint32_t C, uint32_t *cand, int num_sms,
              cudaStream_t s) {
    if (!tc_screen_supported(n, d, C)) return set_error(PANNS_EINVAL, "tc screen: unsupported shape");
    if (reinterpret_cast<uintptr_t>(x) % 16) return set_error(PANNS_EINVAL, "tc screen: base not 16-byte aligned");
    // The norm rides in an extra 32-wide slice when that still fits (d <= 96).
    const bool fused = d + kTcSlice <= 128;
    const uint32_t w = fused ? d + kTcSlice : d;
    const uint32_t slices = w / kTcSlice;
    uint32_t stages = 4;
    while (stages > 2 && tc_layout(slices, stages, C).total + 1024 > 227u * 1024u) --stages;
    const TcSmem L = tc_layout(slices, stages, C);
    const size_t smem = L.total + 1024;
    if (smem > 227u * 1024u) return set_error(PANNS_EINVAL, "tc screen: C too large for shared memory");
    float *xa = nullptr, *xb = nullptr;
    uint32_t *err = nullptr;
    cudaError_t e = cudaMallocAsync(&err, 4, s);
    if (e == cudaSuccess && fused) e = cudaMallocAsync(&xa, (size_t) n * w * 4, s);
    if (e == cudaSuccess && fused) e = cudaMallocAsync(&xb, (size_t) n * w * 4, s);
    if (e != cudaSuccess) {
        cudaFreeAsync(err, s);
        if (xa) cudaFreeAsync(xa, s);
        return set_error(PANNS_ECUDA, std::string("tc screen: ") + cudaGetErrorString(e));
    }
    cudaMemsetAsync(err, 0, 4, s);
    if (fused) {
        const uint64_t total = (uint64_t) n * w;
        const int blocks = (int) std::min<uint64_t>((total + 255) / 256, (uint64_t) num_sms * 32);
        augment_kernel<<<blocks, 256, 0, s>>>(x, xn, n, d, w, xa, xb);
    }
    CUtensorMap ma, mb;
    int rc = make_map(&ma, fused ? xa : x, n, w, kTcM);
    if (!rc) rc = make_map(&mb, fused ? xb : x, n, w, kTcN);
    if (rc) {
        cudaFreeAsync(err, s);
        if (xa) cudaFreeAsync(xa, s);
        if (xb) cudaFreeAsync(xb, s);
        return rc;
    }
    TcArgs a;
    a.yn = xn;
    a.n = n;
    a.d = w;
    a.C = C;
    a.slices = slices;
    a.stages = stages;
    a.cand = cand;
    a.error = err;
    const void *kern = fused ? (const void *) tc_screen_kernel<true> : (const void *) tc_screen_kernel<false>;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e == cudaSuccess) {
        const uint32_t row_blocks = (n + kTcM - 1) / kTcM;
        const uint32_t grid = std::min<uint32_t>(row_blocks, (uint32_t) num_sms);
        if (fused) tc_screen_kernel<true><<<grid, kTcThreads, smem, s>>>(ma, mb, a);
        else tc_screen_kernel<false><<<grid, kTcThreads, smem, s>>>(ma, mb, a);
        e = cudaGetLastError();
    }
    uint32_t herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(err, s);
    if (xa) cudaFreeAsync(xa, s);
    if (xb) cudaFreeAsync(xb, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_error(PANNS_ECUDA, std::string("tc screen: ") + cudaGetErrorString(e));
    if (herr) return set_error(PANNS_EDEVICE, "tc screen: an mbarrier wait expired");
    return PANNS_OK;
}

}  // namespace panns
