// Persistent best-first search over an NSG graph, one warp per query.
//
// Semantics (exact, ID-identical to the reference's deterministic forms):
//   * PANNS top-M at one thread (M = 1: sequential search, PSS_v5 at T = 1):
//     core/Searching.202011241533.top_m_pure.cpp:1881-1965,
//     core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:1218-1515.
//     Queue order (dist, id) (include/Candidate.h:11-28); a neighbour is
//     rejected when dist > the L-th distance; k = nk <= last_k ? nk : last_k + 1.
//   * efanna2e IndexNSG::Search / SearchWithOptGraph
//     (include/efanna2e/index_nsg.cpp:452-611): order by distance only, a new
//     element after existing equal distances (InsertIntoPool,
//     include/efanna2e/neighbor.h:103-131), rejected when dist >= the L-th.
//
// Why a step can be done in parallel: inside one step the reference inserts
// the freshly computed neighbours one by one into a full, sorted queue of L,
// each against the live L-th element. That sequence always leaves the queue
// equal to the L best of (old queue + all fresh neighbours), and the lowest
// insert position it reports equals the final position of the best fresh
// element when that element survives (and L otherwise). So the warp computes
// all fresh distances of the step at once, sorts the survivors and merges
// them in one rank-based pass; chunked merges give the same result.
//
// Vertex numbering on the device: vertices are stored in a locality order
// (see panns_abi.cu), so a query's visited bits and gathers cluster. The
// kernel works on these device ids; `orig` maps them back. Original ids are
// used wherever the reference's semantics depend on ids: the (dist, id)
// tie-break (looked up only when two distances are exactly equal) and the
// output.
//
// HBM layout (built in panns_abi.cu):
//   vec   n x (CL*8) float4, "chain-major": float4 number 8*i + c of a row holds
//         terms 4i..4i+3 of lane accumulator c of the reference's 8-lane
//         distance loop, so the 8 threads of a vertex read one 128-byte line
//         per load and each thread runs its lane's FMA chain in the reference
//         order. Padding terms are zero (an FMA with 0*0 leaves a lane as is).
//   norm  n float32, ||v||^2 in the same lane order (norm-trick distance).
//   head  n x 32 u32: degree, then the first 31 neighbour ids (one 128-byte
//         read per expansion); ovf_off/ovf: the rest of longer rows (CSR).
//
// Per warp (shared memory): the queue (L x (dist f32, id u32 with bit 31 =
// checked)), a buffer of fresh candidates, the picked candidates. Per warp slot in
// global memory: a visited bitset of n bits plus the list of its words that
// went from zero to non-zero, so only those are cleared after the query.
#pragma once

#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mlp_infer.cuh"

namespace panns {

constexpr uint32_t kChecked = 0x80000000u;
constexpr uint32_t kIdMask = 0x7fffffffu;
constexpr uint32_t kFull = 0xffffffffu;
constexpr int kHeadWords = 32;   // degree + 31 neighbours
constexpr int kHeadNbrs = kHeadWords - 1;
#ifndef PANNS_KBUF
#define PANNS_KBUF 256
#endif
#ifndef PANNS_WIDE_DIST
#define PANNS_WIDE_DIST 0  // 1: 16 rows in flight per warp pass in the one-warp kernel too
#endif
#ifndef PANNS_FP8_MIXED
#define PANNS_FP8_MIXED 1  // FP8 rows times a half-precision query by mixed-precision FMAs
#endif
#ifndef PANNS_SEARCH_MIN_BLOCKS
#define PANNS_SEARCH_MIN_BLOCKS 6
#endif
constexpr int kBuf = PANNS_KBUF;  // fresh-candidate buffer per warp
// warp_sort pads a chunk to the next power of two >= its size inside the buffer.
static_assert(kBuf >= 64 && (kBuf & (kBuf - 1)) == 0, "kBuf must be a power of two >= 64");
constexpr int kCandGroup = 8;    // candidates whose head rows are loaded at once
constexpr int kGroupChunks = (kCandGroup * kHeadNbrs + 31) / 32;
// A group's head-row neighbours go into the fresh buffer without a flush in between.
static_assert(kCandGroup * kHeadNbrs <= kBuf, "kBuf must hold a group's head-row neighbours");
constexpr int kOvfChunks = 2;    // overflow neighbours per batch of loads: kOvfChunks * 32
constexpr int kMaxM = 64;

enum { ORDER_PANNS = 0, ORDER_EFANNA = 1 };
enum { KIND_IP = 0, KIND_L2 = 1 };
// Storage the search distances are computed from: the exact float32 rows, or
// a reduced copy (BF16, or FP8 E4M3 with per-dimension scales) whose final L
// candidates are re-ranked with the exact float32 distance.
enum { STORE_FP32 = 0, STORE_BF16 = 1, STORE_FP8 = 2 };

// Error bits written to SearchArgs::error.
enum : uint32_t { ERR_BAD_ID = 1u, ERR_BAD_INIT = 2u };

struct SearchArgs {
    const float4 *vec;        // n x (CL*8) float4
    const float *norms;       // n (KIND_IP)
    const uint32_t *head;     // n x 32
    const uint64_t *ovf_off;  // n
    const uint32_t *ovf;      // overflow neighbours
    const uint32_t *orig;     // device id -> original id
    uint32_t n;
    const float4 *queries;    // nq x (CL*8) float4, chain-major
    uint32_t nq;
    const uint32_t *init_ids; // L device ids, or nq x L when init_stride == L
    uint32_t init_stride;
    uint32_t K, L, M;
    uint32_t *out_ids;        // nq x K original ids
    uint4 *out_stats;         // nq x {n_dist, n_expand, n_edges, n_iter}
    uint32_t *visited;        // slots x vis_words
    uint32_t vis_words;
    uint32_t *dirty;          // slots x dirty_cap
    uint32_t dirty_cap;
    uint32_t *counter;        // work-stealing query counter
    uint32_t *error;          // ERR_* bits
    uint32_t queue_cap;       // shared-memory queue entries per warp (>= L, a multiple of 32)
    const void *vec_lo;       // reduced rows, natural element order: n x dpad (BF16 or FP8)
    const float *norms_lo;    // ||v||^2 of the dequantised rows
    const float *scales;      // FP8: per-dimension scale (dpad)
    uint32_t d;               // dimension
    const uint32_t *Lq;       // per-query queue length (K <= Lq[q] <= L), or null: L for all
    const uint32_t *decisions;  // per-query records of the entry / L-budget network (mlp_decide), or null
    uint32_t dec_L_init;      // plain init ids kept after learned entries
    uint32_t block_round;     // search_block_kernel: candidates per warp and merge round
};

// Bytes of shared memory one warp needs.
__host__ __device__ inline uint32_t warp_smem_bytes(uint32_t queue_cap) {
    return queue_cap * 8u                 // queue dist + id
           + kBuf * 12u                   // buffer dist + id + key
           + kMaxM * 4u;                  // picked candidate ids / learned entries
}

struct WarpMem {
    float *qd;
    uint32_t *qi;
    float *bd;
    uint32_t *bi;
    uint32_t *bk;
    uint32_t *cand;
};

static __device__ __forceinline__ WarpMem carve(uint8_t *base, uint32_t queue_cap) {
    WarpMem m;
    m.qd = reinterpret_cast<float *>(base);
    m.qi = reinterpret_cast<uint32_t *>(m.qd + queue_cap);
    m.bd = reinterpret_cast<float *>(m.qi + queue_cap);
    m.bi = reinterpret_cast<uint32_t *>(m.bd + kBuf);
    m.bk = m.bi + kBuf;
    m.cand = m.bk + kBuf;
    return m;
}

static __device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// Distances of two vertices per 8-lane group (c = lane & 7 is the lane
// accumulator this thread owns): both rows are loaded before either is used.
// Lane sum: ((u0 + u1) + u2) + ... + u7; norm trick: -2 * dot + norm, which
// is one rounding either way because -2 * dot is exact.
// ---------------------------------------------------------------------------
template <int KIND, int CL>
__device__ __forceinline__ float chain(const float4 (&x)[CL], const float4 (&qv)[CL]) {
    float acc = 0.0f;
#pragma unroll
    for (int i = 0; i < CL; ++i) {
        if (KIND == KIND_IP) {
            acc = __fmaf_rn(x[i].x, qv[i].x, acc);
            acc = __fmaf_rn(x[i].y, qv[i].y, acc);
            acc = __fmaf_rn(x[i].z, qv[i].z, acc);
            acc = __fmaf_rn(x[i].w, qv[i].w, acc);
        } else {
            float t;
            t = __fsub_rn(x[i].x, qv[i].x); acc = __fmaf_rn(t, t, acc);
            t = __fsub_rn(x[i].y, qv[i].y); acc = __fmaf_rn(t, t, acc);
            t = __fsub_rn(x[i].z, qv[i].z); acc = __fmaf_rn(t, t, acc);
            t = __fsub_rn(x[i].w, qv[i].w); acc = __fmaf_rn(t, t, acc);
        }
    }
    return acc;
}

static __device__ __forceinline__ float lane_sum8(float acc, int lane) {
    const int base = lane & ~7;
    float s = __shfl_sync(kFull, acc, base);
#pragma unroll
    for (int j = 1; j < 8; ++j) s = __fadd_rn(s, __shfl_sync(kFull, acc, base + j));
    return s;
}

template <int KIND, int CL>
__device__ __forceinline__ void group_distance2(const float4 *__restrict__ vec,
                                                const float *__restrict__ norms, uint32_t v0,
                                                bool a0, uint32_t v1, bool a1,
                                                const float4 (&qv)[CL], int lane, float &d0,
                                                float &d1) {
    const int c = lane & 7;
    float4 x0[CL], x1[CL];
    float n0 = 0.f, n1 = 0.f;
    const float4 *r0 = vec + (size_t) v0 * (CL * 8) + c;
    const float4 *r1 = vec + (size_t) v1 * (CL * 8) + c;
#pragma unroll
    for (int i = 0; i < CL; ++i) {
        x0[i] = a0 ? __ldg(r0 + 8 * i) : make_float4(0.f, 0.f, 0.f, 0.f);
        x1[i] = a1 ? __ldg(r1 + 8 * i) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (KIND == KIND_IP) {
        n0 = a0 ? __ldg(norms + v0) : 0.f;
        n1 = a1 ? __ldg(norms + v1) : 0.f;
    }
    float s0 = lane_sum8(chain<KIND, CL>(x0, qv), lane);
    float s1 = lane_sum8(chain<KIND, CL>(x1, qv), lane);
    if (KIND == KIND_IP) {
        s0 = __fmaf_rn(-2.0f, s0, n0);
        s1 = __fmaf_rn(-2.0f, s1, n1);
    }
    d0 = s0;
    d1 = s1;
}

// (dist, key) order. PANNS: key is a device id and equal distances compare
// original ids; EFANNA: key is the arrival index.
template <int ORDER>
__device__ __forceinline__ bool key_less(float ad, uint32_t ak, float bd, uint32_t bk,
                                         const uint32_t *__restrict__ orig) {
    if (ad != bd) return ad < bd;
    if (ORDER == ORDER_PANNS) {
        if (ak == bk) return false;
        if (ak == kFull || bk == kFull) return ak < bk;  // padding sorts last
        return __ldg(orig + ak) < __ldg(orig + bk);
    }
    return ak < bk;
}

// Number of queue elements that precede a fresh element (d, id).
template <int ORDER>
__device__ __forceinline__ uint32_t queue_rank(const float *qd, const uint32_t *qi, uint32_t sz,
                                               float d, uint32_t id, const uint32_t *orig) {
    uint32_t lo = 0, hi = sz;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        const float md = qd[mid];
        bool before;
        if (ORDER == ORDER_PANNS) {
            before = md < d || (md == d && __ldg(orig + (qi[mid] & kIdMask)) < __ldg(orig + id));
        } else {
            before = md <= d;  // older elements stay ahead of equal distances
        }
        if (before) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Number of sorted fresh elements that precede a queue element (d, id). Fresh
// ids may carry the checked bit (worker queues merged into the master).
template <int ORDER>
__device__ __forceinline__ uint32_t fresh_rank(const float *bd, const uint32_t *bi, uint32_t cnt,
                                               float d, uint32_t id, const uint32_t *orig) {
    uint32_t lo = 0, hi = cnt;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        const float md = bd[mid];
        bool before;
        if (ORDER == ORDER_PANNS) {
            before = md < d || (md == d && __ldg(orig + (bi[mid] & kIdMask)) < __ldg(orig + id));
        } else {
            before = md < d;
        }
        if (before) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// (dist, key) order of the fresh buffer: the key is the original vertex id
// or the device id (PANNS; then replaced by the original id when distances
// tie, see flush) or the arrival index (EFANNA), distinct within a buffer, so
// the order is total and needs no lookups.
__device__ __forceinline__ bool plain_less(float ad, uint32_t ak, float bd, uint32_t bk) {
    return ad < bd || (ad == bd && ak < bk);
}

// Sort (bd, bk, bi)[0..cnt) by (dist, key). Up to 64 elements: by rank (each
// lane counts the elements that precede its own one or two, with independent
// shuffles, then writes them to their ranks); more: a bitonic network in
// shared memory (padding up to the next power of two holds (+inf, ~0)).
template <int ORDER>
__device__ void warp_sort(float *bd, uint32_t *bi, uint32_t *bk, uint32_t cnt,
                          const uint32_t *orig, int lane) {
    (void) orig;
    if (cnt <= 1) return;
    if (cnt <= 64) {
        const uint32_t j0 = lane, j1 = lane + 32;
        const bool h0 = j0 < cnt, h1 = j1 < cnt;
        const float d0 = h0 ? bd[j0] : __int_as_float(0x7f800000);
        const float d1 = h1 ? bd[j1] : __int_as_float(0x7f800000);
        const uint32_t k0 = h0 ? bk[j0] : kFull, k1 = h1 ? bk[j1] : kFull;
        const uint32_t i0 = h0 ? bi[j0] : 0u, i1 = h1 ? bi[j1] : 0u;
        uint32_t r0 = 0, r1 = 0;
        const bool two = cnt > 32;
#pragma unroll 8
        for (int src = 0; src < 32; ++src) {
            const float sd = __shfl_sync(kFull, d0, src);
            const uint32_t sk = __shfl_sync(kFull, k0, src);
            r0 += plain_less(sd, sk, d0, k0);
            r1 += plain_less(sd, sk, d1, k1);
            if (two) {
                const float td = __shfl_sync(kFull, d1, src);
                const uint32_t tk = __shfl_sync(kFull, k1, src);
                r0 += plain_less(td, tk, d0, k0);
                r1 += plain_less(td, tk, d1, k1);
            }
        }
        __syncwarp();
        if (h0) {
            bd[r0] = d0;
            bk[r0] = k0;
            bi[r0] = i0;
        }
        if (h1) {
            bd[r1] = d1;
            bk[r1] = k1;
            bi[r1] = i1;
        }
        __syncwarp();
        return;
    }
    uint32_t n = 64;
    while (n < cnt) n <<= 1;
    for (uint32_t i = cnt + lane; i < n; i += 32) {
        bd[i] = __int_as_float(0x7f800000);
        bi[i] = kFull;
        bk[i] = kFull;
    }
    __syncwarp();
    // One compare-exchange pair per lane and pass: pair p has its lower index
    // i = p with a zero bit inserted at bit j, its upper one i | j.
    for (uint32_t k = 2; k <= n; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t p = lane; p < (n >> 1); p += 32) {
                const uint32_t i = ((p & ~(j - 1)) << 1) | (p & (j - 1));
                const uint32_t ixj = i | j;
                const float ad = bd[i], xd = bd[ixj];
                const uint32_t ak = bk[i], xk = bk[ixj];
                const bool up = (i & k) == 0;
                const bool sw = up ? plain_less(xd, xk, ad, ak) : plain_less(ad, ak, xd, xk);
                if (sw) {
                    bd[i] = xd; bd[ixj] = ad;
                    bk[i] = xk; bk[ixj] = ak;
                    const uint32_t t = bi[i]; bi[i] = bi[ixj]; bi[ixj] = t;
                }
            }
            __syncwarp();
        }
    }
}

// Merge the sorted fresh elements (bd, bi)[0..cnt) into the queue (qd, qi)
// of size *sz and capacity cap. Returns the position of the first fresh
// element if it was inserted (< cap), else cap. Uses bk as scratch.
template <int ORDER>
__device__ uint32_t merge_into(float *qd, uint32_t *qi, uint32_t *sz, uint32_t cap, const float *bd,
                               const uint32_t *bi, uint32_t *bk, uint32_t cnt, const uint32_t *orig,
                               int lane) {
    const uint32_t qsz = *sz;
    if (cnt == 0) return cap;
    // Merged position of each fresh element: its index plus its rank in the old queue.
    for (uint32_t i = lane; i < cnt; i += 32)
        bk[i] = i + queue_rank<ORDER>(qd, qi, qsz, bd[i], bi[i] & kIdMask, orig);
    __syncwarp();
    const uint32_t p0 = bk[0];
    if (p0 >= cap) return cap;
    // Move queue elements [p0, qsz) to their merged positions, top chunk first;
    // a chunk is read completely before any of it is written.
    for (int32_t top = (int32_t) qsz - 1; top >= (int32_t) p0; top -= 32) {
        const int32_t j = top - lane;
        float d = 0.f;
        uint32_t id = 0, np = cap;
        if (j >= (int32_t) p0) {
            d = qd[j];
            id = qi[j];
            np = (uint32_t) j + fresh_rank<ORDER>(bd, bi, cnt, d, id & kIdMask, orig);
        }
        __syncwarp();
        if (np < cap) {
            qd[np] = d;
            qi[np] = id;
        }
        __syncwarp();
    }
    for (uint32_t i = lane; i < cnt; i += 32) {
        const uint32_t np = bk[i];
        if (np < cap) {
            qd[np] = bd[i];
            qi[np] = bi[i];
        }
    }
    __syncwarp();
    *sz = min(cap, qsz + cnt);
    return p0;
}

template <int ORDER>
__device__ __forceinline__ uint32_t warp_merge(const WarpMem &m, uint32_t *sz, uint32_t L, uint32_t cnt,
                                               const uint32_t *orig, int lane) {
    return merge_into<ORDER>(m.qd, m.qi, sz, L, m.bd, m.bi, m.bk, cnt, orig, lane);
}

// Visited bitset: test-and-set returns the previous word.
static __device__ __forceinline__ uint32_t visit_issue(uint32_t *vis, uint32_t id, bool valid) {
    return valid ? atomicOr(vis + (id >> 5), 1u << (id & 31)) : kFull;
}

// Record the words that went from zero to non-zero (only those are cleared
// after the query).
static __device__ __forceinline__ void note_dirty(uint32_t *dirty, uint32_t dirty_cap, uint32_t &dcount,
                                           bool first, uint32_t word) {
    const uint32_t bm = __ballot_sync(kFull, first);
    if (first) {
        const uint32_t pos = dcount + __popc(bm & lanemask_lt());
        if (pos < dirty_cap) dirty[pos] = word;
    }
    dcount += __popc(bm);
}

// ---------------------------------------------------------------------------
// Distance policies. distances(a, ids, out, nb): out[b] = distance of the
// query to vertex ids[b] & kIdMask, for b < nb, computed by the whole warp.
// ---------------------------------------------------------------------------
template <int KIND, int CL, int STORE>
struct Dist;

// Exact float32, reference lane order (8 lanes per vertex, chain-major rows).
template <int KIND, int CL>
struct Dist<KIND, CL, STORE_FP32> {
    float4 qv[CL];
    __device__ __forceinline__ void load(const SearchArgs &a, uint32_t q, int lane) {
        const float4 *qrow = a.queries + (size_t) q * (CL * 8);
#pragma unroll
        for (int i = 0; i < CL; ++i) qv[i] = __ldg(qrow + 8 * i + (lane & 7));
    }
    __device__ __forceinline__ void distances(const SearchArgs &a, const uint32_t *ids, float *out,
                                              uint32_t nb, int lane) const {
        const int g = lane >> 3;
        // 8 vertices per round (2 per 8-lane group, loads issued together).
        for (uint32_t b0 = 0; b0 < nb; b0 += 8) {
            const uint32_t b = b0 + g, bb = b0 + 4 + g;
            const bool act0 = b < nb, act1 = bb < nb;
            const uint32_t v0 = act0 ? ids[b] & kIdMask : 0u, v1 = act1 ? ids[bb] & kIdMask : 0u;
            float d0, d1;
            group_distance2<KIND, CL>(a.vec, a.norms, v0, act0, v1, act1, qv, lane, d0, d1);
            if ((lane & 7) == 0) {
                if (act0) out[b] = d0;
                if (act1) out[bb] = d1;
            }
        }
        __syncwarp();
    }
};

// Four vertices per 8-lane group (16 per warp pass), all rows loaded before
// any is used: the same per-vertex arithmetic as group_distance2, with twice
// the loads in flight, for kernels with registers to spare.
template <int KIND, int CL>
__device__ __forceinline__ void distances_wide(const SearchArgs &a, const float4 (&qv)[CL], const uint32_t *ids,
                                               float *out, uint32_t nb, int lane) {
    const int g = lane >> 3, c = lane & 7;
    for (uint32_t b0 = 0; b0 < nb; b0 += 16) {
        uint32_t v[4];
        bool act[4];
        float4 x[4][CL];
        float nrm[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t b = b0 + 4 * u + g;
            act[u] = b < nb;
            v[u] = act[u] ? ids[b] & kIdMask : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 *r = a.vec + (size_t) v[u] * (CL * 8) + c;
#pragma unroll
            for (int i = 0; i < CL; ++i) x[u][i] = act[u] ? __ldg(r + 8 * i) : make_float4(0.f, 0.f, 0.f, 0.f);
            nrm[u] = (KIND == KIND_IP && act[u]) ? __ldg(a.norms + v[u]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            float s = lane_sum8(chain<KIND, CL>(x[u], qv), lane);
            if (KIND == KIND_IP) s = __fmaf_rn(-2.0f, s, nrm[u]);
            if (c == 0 && act[u]) out[b0 + 4 * u + g] = s;
        }
    }
    __syncwarp();
}

// Position of natural element e in a chain-major padded row (inverse of the
// layout's chain_term_element).
static __device__ __forceinline__ int chain_major_pos(int d, int e) {
    const int DR = d % 16, DD = d - DR;
    int c, k;
    if (DR && e >= DD) {
        c = e - DD;
        k = 0;
    } else {
        c = e & 7;
        k = (e >> 3) + (DR ? 1 : 0);
    }
    return (8 * (k >> 2) + c) * 4 + (k & 3);
}

// Reduced copy: 4 lanes per vertex, lane t of the group owns 8-element chunks
// t, t+4, ..., t+4(CL-1) of the row; accumulation in float32; the ranking
// distance is ||v^||^2 - 2 <v^, q> on the dequantised row v^ (the constant
// ||q||^2 is left out, as in the norm trick). FP8 scales are folded into the
// query once.
template <int KIND, int CL, int STORE>
struct Dist {
    // FP8 with PANNS_FP8_MIXED: the query (times the per-dimension scales and
    // 2^12, which keeps it in half precision's normal range) as half pairs,
    // multiplied with the E4M3 rows converted to half pairs by mixed-precision
    // FMAs (half x half products are exact in float32, float32 accumulation);
    // the 2^-12 is taken back in the final norm-trick FMA.
    static constexpr bool kMixed = STORE == STORE_FP8 && PANNS_FP8_MIXED;
    static constexpr float kMixedScale = 4096.0f;
    float ql[kMixed ? 1 : 8 * CL];
    uint32_t qh[kMixed ? 4 * CL : 1];
    __device__ __forceinline__ void load(const SearchArgs &a, uint32_t q, int lane) {
        const float *qrow = reinterpret_cast<const float *>(a.queries) + (size_t) q * (CL * 32);
        const int t = lane & 3;
#pragma unroll
        for (int i = 0; i < CL; ++i) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int e = 8 * (t + 4 * i) + j;
                float x = e < (int) a.d ? __ldg(qrow + chain_major_pos((int) a.d, e)) : 0.f;
                if (STORE == STORE_FP8) x *= __ldg(a.scales + e);
                if constexpr (kMixed) {
                    const __half h = __float2half_rn(x * kMixedScale);
                    const uint32_t hb = (uint32_t) __half_as_ushort(h);
                    if (j & 1) qh[4 * i + j / 2] |= hb << 16;
                    else qh[4 * i + j / 2] = hb;
                } else {
                    ql[8 * i + j] = x;
                }
            }
        }
    }
    // BF16: partial dot product of this lane's chunks of row v.
    __device__ __forceinline__ float dot_row_bf16(const void *vec_lo, uint32_t v, int t) const {
        float acc = 0.f;
        const uint4 *row = reinterpret_cast<const uint4 *>(vec_lo) + (size_t) v * (CL * 4);
        uint4 x[CL];
#pragma unroll
        for (int i = 0; i < CL; ++i) x[i] = __ldg(row + t + 4 * i);
#pragma unroll
        for (int i = 0; i < CL; ++i) {
            const uint32_t w[4] = {x[i].x, x[i].y, x[i].z, x[i].w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                acc = fmaf(__uint_as_float(w[j] << 16), ql[8 * i + 2 * j], acc);
                acc = fmaf(__uint_as_float(w[j] & 0xffff0000u), ql[8 * i + 2 * j + 1], acc);
            }
        }
        return acc;
    }
    // FP8: partial dot product of this lane's chunks of row v, component 0
    // over the even elements, component 1 over the odd ones.
    __device__ __forceinline__ float2 dot_row2(const void *vec_lo, uint32_t v, int t) const {
        float2 acc = make_float2(0.f, 0.f);
        if constexpr (kMixed) {
            const uint2 *row = reinterpret_cast<const uint2 *>(vec_lo) + (size_t) v * (CL * 4);
            uint2 x[CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) x[i] = __ldg(row + t + 4 * i);
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                const uint32_t w[2] = {x[i].x, x[i].y};
#pragma unroll
                for (int j = 0; j < 2; ++j) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const __nv_fp8x2_storage_t pair = (__nv_fp8x2_storage_t) (w[j] >> (16 * h));
                        const __half2_raw hr = __nv_cvt_fp8x2_to_halfraw2(pair, __NV_E4M3);
                        const uint32_t xv = (uint32_t) hr.x | ((uint32_t) hr.y << 16);
                        asm("{\n\t.reg .b16 a0, a1, b0, b1;\n\t"
                            "mov.b32 {a0, a1}, %2;\n\t"
                            "mov.b32 {b0, b1}, %3;\n\t"
                            "fma.rn.f32.f16 %0, a0, b0, %0;\n\t"
                            "fma.rn.f32.f16 %1, a1, b1, %1;\n\t}"
                            : "+f"(acc.x), "+f"(acc.y)
                            : "r"(xv), "r"(qh[4 * i + 2 * j + h]));
                    }
                }
            }
        } else {
            const uint2 *row = reinterpret_cast<const uint2 *>(vec_lo) + (size_t) v * (CL * 4);
            uint2 x[CL];
#pragma unroll
            for (int i = 0; i < CL; ++i) x[i] = __ldg(row + t + 4 * i);
#pragma unroll
            for (int i = 0; i < CL; ++i) {
                const uint32_t w[2] = {x[i].x, x[i].y};
#pragma unroll
                for (int j = 0; j < 2; ++j) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const __nv_fp8x2_storage_t pair = (__nv_fp8x2_storage_t) (w[j] >> (16 * h));
                        const __half2_raw hr = __nv_cvt_fp8x2_to_halfraw2(pair, __NV_E4M3);
                        const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&hr));
                        acc = __ffma2_rn(f, make_float2(ql[8 * i + 4 * j + 2 * h], ql[8 * i + 4 * j + 2 * h + 1]),
                                         acc);
                    }
                }
            }
        }
        return acc;
    }
    __device__ __forceinline__ void distances(const SearchArgs &a, const uint32_t *ids, float *out,
                                              uint32_t nb, int lane) const {
        const int g = lane >> 2, t = lane & 3;
        // 16 vertices per round (2 per 4-lane group, loads issued together).
        for (uint32_t b0 = 0; b0 < nb; b0 += 16) {
            const uint32_t b = b0 + g, bb = b0 + 8 + g;
            const bool act0 = b < nb, act1 = bb < nb;
            const uint32_t v0 = act0 ? ids[b] & kIdMask : 0u, v1 = act1 ? ids[bb] & kIdMask : 0u;
            const float n0 = act0 ? __ldg(a.norms_lo + v0) : 0.f;
            const float n1 = act1 ? __ldg(a.norms_lo + v1) : 0.f;
            if constexpr (STORE == STORE_BF16) {
                float s0 = act0 ? dot_row_bf16(a.vec_lo, v0, t) : 0.f;
                float s1 = act1 ? dot_row_bf16(a.vec_lo, v1, t) : 0.f;
                s0 += __shfl_xor_sync(kFull, s0, 1);
                s1 += __shfl_xor_sync(kFull, s1, 1);
                s0 += __shfl_xor_sync(kFull, s0, 2);
                s1 += __shfl_xor_sync(kFull, s1, 2);
                if (t == 0) {
                    if (act0) out[b] = fmaf(-2.f, s0, n0);
                    if (act1) out[bb] = fmaf(-2.f, s1, n1);
                }
                continue;
            }
            const float2 p0 = act0 ? dot_row2(a.vec_lo, v0, t) : make_float2(0.f, 0.f);
            const float2 p1 = act1 ? dot_row2(a.vec_lo, v1, t) : make_float2(0.f, 0.f);
            float2 s = __fadd2_rn(make_float2(p0.x, p1.x), make_float2(p0.y, p1.y));
            s = __fadd2_rn(s, make_float2(__shfl_xor_sync(kFull, s.x, 1), __shfl_xor_sync(kFull, s.y, 1)));
            s = __fadd2_rn(s, make_float2(__shfl_xor_sync(kFull, s.x, 2), __shfl_xor_sync(kFull, s.y, 2)));
            if (t == 0) {
                const float m2 = kMixed ? -2.f / kMixedScale : -2.f;
                const float2 r = __ffma2_rn(make_float2(m2, m2), s, make_float2(n0, n1));
                if (act0) out[b] = r.x;
                if (act1) out[bb] = r.y;
            }
        }
        __syncwarp();
    }
};

// Sort (qd, qi)[0..sz) by (dist, original id) in place; the arrays have room
// for the next power of two >= sz (padding (+inf, ~0)).
static __device__ void rank_sort(float *qd, uint32_t *qi, uint32_t sz, const uint32_t *orig, int lane) {
    uint32_t n = 1;
    while (n < sz) n <<= 1;
    for (uint32_t i = sz + lane; i < n; i += 32) {
        qd[i] = __int_as_float(0x7f800000);
        qi[i] = kFull;
    }
    __syncwarp();
    for (uint32_t k = 2; k <= n; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t p = lane; p < (n >> 1); p += 32) {  // pairs, as in warp_sort
                const uint32_t i = ((p & ~(j - 1)) << 1) | (p & (j - 1));
                const uint32_t ixj = i | j;
                const float ad = qd[i], xd = qd[ixj];
                const uint32_t ai = qi[i], xi = qi[ixj];
                const uint32_t ak = ai == kFull ? kFull : (ai & kIdMask);
                const uint32_t xk = xi == kFull ? kFull : (xi & kIdMask);
                const bool up = (i & k) == 0;
                const bool sw = up ? key_less<ORDER_PANNS>(xd, xk, ad, ak, orig)
                                   : key_less<ORDER_PANNS>(ad, ak, xd, xk, orig);
                if (sw) {
                    qd[i] = xd; qd[ixj] = ad;
                    qi[i] = xi; qi[ixj] = ai;
                }
            }
            __syncwarp();
        }
    }
}

// Order the sz entries (qd, qi) by (distance, original id) and write the
// original ids of the first K to out. The entries are cut into runs whose
// sizes are the binary digits of sz (largest first); each run is sorted in
// place by rank_sort (a power of two, so it needs no padding) and an entry's
// output position is its index in its run plus, for every other run, the
// number of that run's entries that precede it. The queue therefore needs no
// room beyond sz.
static __device__ void rerank_output(float *qd, uint32_t *qi, uint32_t sz, uint32_t K, const uint32_t *orig,
                                     uint32_t *out, int lane) {
    for (uint32_t start = 0, b = 32; b-- > 0;) {
        const uint32_t n = 1u << b;
        if (!(sz & n)) continue;
        rank_sort(qd + start, qi + start, n, orig, lane);
        start += n;
    }
    __syncwarp();
    for (uint32_t i = lane; i < sz; i += 32) {
        const float d = qd[i];
        const uint32_t key = __ldg(orig + (qi[i] & kIdMask));
        uint32_t rank = 0;
        for (uint32_t start = 0, b = 32; b-- > 0;) {
            const uint32_t n = 1u << b;
            if (!(sz & n)) continue;
            if (i >= start && i < start + n) {
                rank += i - start;
            } else {
                uint32_t lo = 0, hi = n;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    const float md = qd[start + mid];
                    const bool before = md < d || (md == d && __ldg(orig + (qi[start + mid] & kIdMask)) < key);
                    if (before) lo = mid + 1;
                    else hi = mid;
                }
                rank += lo;
            }
            start += n;
        }
        if (rank < K) out[rank] = key;
    }
}

// Compute distances of the buffered fresh vertices bi[0..nb), keep the ones
// that can still enter the queue, sort them and merge them. Returns the merge
// position of the best survivor or L.
template <int KIND, int ORDER, int CL, int STORE>
__device__ uint32_t flush(const SearchArgs &a, const WarpMem &m, uint32_t nb, uint32_t *sz, uint32_t L,
                          bool filter, const Dist<KIND, CL, STORE> &D, int lane) {
    constexpr bool kLazyKeys = ORDER == ORDER_PANNS && STORE != STORE_FP8;
#if PANNS_WIDE_DIST
    if constexpr (STORE == STORE_FP32) distances_wide<KIND, CL>(a, D.qv, m.bi, m.bd, nb, lane);
    else D.distances(a, m.bi, m.bd, nb, lane);
#else
    D.distances(a, m.bi, m.bd, nb, lane);
#endif
    // Keep the survivors, in arrival order.
    const float bound = (filter && *sz >= L) ? m.qd[L - 1] : __int_as_float(0x7f800000);
    const bool any_bound = filter && *sz >= L;
    uint32_t cnt = 0;
    for (uint32_t b0 = 0; b0 < nb; b0 += 32) {
        const uint32_t b = b0 + lane;
        float d = 0.f;
        uint32_t id = 0;
        bool keep = false;
        if (b < nb) {
            d = m.bd[b];
            id = m.bi[b];
            keep = !any_bound || (ORDER == ORDER_PANNS ? !(d > bound) : d < bound);
        }
        const uint32_t bm = __ballot_sync(kFull, keep);
        __syncwarp();
        if (keep) {
            const uint32_t pos = cnt + __popc(bm & lanemask_lt());
            m.bd[pos] = d;
            m.bi[pos] = id;
            m.bk[pos] = ORDER == ORDER_PANNS ? (kLazyKeys ? id : __ldg(a.orig + id)) : pos;
        }
        cnt += __popc(bm);
        __syncwarp();
    }
    if (cnt == 0) return L;
    // With lazy keys the survivors are sorted by (distance, device id); PANNS
    // order breaks equal distances by original id, so if the sorted
    // survivors hold equal distances (rare) they are sorted once more with
    // the original ids as keys (one inlined copy of warp_sort either way).
    // Measured (10,000 queries, L = 384, M = 8, same ids): float32 rows
    // 5.42 -> 5.31 ms, BF16 5.08 -> 5.02 ms, FP8 5.03 -> 5.08 ms, so the FP8
    // kernel keeps loading the original ids in the filter.
    for (int pass = 0;; ++pass) {
        warp_sort<ORDER>(m.bd, m.bi, m.bk, cnt, a.orig, lane);
        if (!kLazyKeys || pass) break;
        bool tie = false;
        for (uint32_t i = lane; i + 1 < cnt; i += 32) tie |= m.bd[i] == m.bd[i + 1];
        if (!__any_sync(kFull, tie)) break;
        for (uint32_t i = lane; i < cnt; i += 32) m.bk[i] = __ldg(a.orig + (m.bi[i] & kIdMask));
        __syncwarp();
    }
    return warp_merge<ORDER>(m, sz, L, cnt, a.orig, lane);
}

// Append this lane's fresh vertex (if any) to the buffer. The caller makes
// room first (one flush per group of candidates or batch of overflow
// neighbours, so the kernel holds few inlined copies of flush).
__device__ __forceinline__ void append_ids(const WarpMem &m, uint32_t &nb, bool fresh, uint32_t id, int lane) {
    const uint32_t bm = __ballot_sync(kFull, fresh);
    if (fresh) m.bi[nb + __popc(bm & lanemask_lt())] = id;
    nb += __popc(bm);
    __syncwarp();
}

// One query, run by one warp.
template <int KIND, int ORDER, int CL, int STORE>
__device__ void search_one(const SearchArgs &a, const WarpMem &m, uint32_t q, uint32_t *vis, uint32_t *dirty,
                           int lane) {
    uint32_t L = a.Lq ? __ldg(a.Lq + q) : a.L;
    // Init ids: n_lrn learned entries (m.cand) then n_plain of the init list.
    uint32_t n_lrn = 0, n_plain = L;
    if (ORDER == ORDER_PANNS && a.decisions) {
        const uint2 r = mlp_read_decision(a.decisions, a.dec_L_init, q, m.cand, lane);
        n_lrn = r.x & 0xffu;
        n_plain = r.x >> 8;
        L = r.y;
    }
    Dist<KIND, CL, STORE> D;
    D.load(a, q, lane);
    uint32_t dcount = 0;
    uint32_t n_dist = 0, n_expand = 0, n_edges = 0, n_iter = 0;
    uint32_t sz = 0;

    // Initial queue: the init ids, all marked visited, sorted (init order
    // breaks equal distances for efanna2e). A repeated id (a learned entry
    // that is also in the init list) enters once.
    const uint32_t *init = a.init_ids + (size_t) q * a.init_stride;
    const uint32_t n_init = n_lrn + n_plain;
    uint32_t nb = 0;
    for (uint32_t i0 = 0; i0 < n_init; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool valid = i < n_init;
        uint32_t id = valid ? (i < n_lrn ? m.cand[i] : __ldg(init + (i - n_lrn))) : 0u;
        const bool ok = valid && id < a.n;
        if (valid && !ok) atomicOr(a.error, ERR_BAD_INIT);
        const uint32_t old = visit_issue(vis, id, ok);
        note_dirty(dirty, a.dirty_cap, dcount, ok && old == 0, id >> 5);
        const bool fresh = ok && !(old & (1u << (id & 31)));
        const uint32_t bm = __ballot_sync(kFull, fresh);
        if (fresh) m.bi[nb + __popc(bm & lanemask_lt())] = id;
        nb += __popc(bm);
        __syncwarp();
        if (nb > kBuf - 32 || i0 + 32 >= n_init) {
            n_dist += nb;
            flush<KIND, ORDER, CL, STORE>(a, m, nb, &sz, L, false, D, lane);
            nb = 0;
        }
    }

    uint32_t k = 0;
    const uint32_t M = a.M;
    for (;;) {
        // Pick up to M unchecked candidates at positions >= k.
        uint32_t cnt = 0, last_k = L;
        for (uint32_t p0 = k; p0 < sz && cnt < M; p0 += 32) {
            const uint32_t p = p0 + lane;
            const bool un = p < sz && !(m.qi[p] & kChecked);
            const uint32_t bm = __ballot_sync(kFull, un);
            const uint32_t take = min((uint32_t) __popc(bm), M - cnt);
            const uint32_t r = __popc(bm & lanemask_lt());
            if (un && r < take) {
                const uint32_t id = m.qi[p];
                m.qi[p] = id | kChecked;
                m.cand[cnt + r] = id;
            }
            if (take) {
                // position of the take-th unchecked slot in this window
                uint32_t x = bm;
                for (uint32_t t = 1; t < take; ++t) x &= x - 1;
                last_k = p0 + (__ffs(x) - 1);
            }
            cnt += take;
            __syncwarp();
        }
        if (cnt == 0) break;
        ++n_iter;
        n_expand += cnt;
        uint32_t nk = L;
        nb = 0;
        // The step's work in units: the head rows of a group of up to
        // kCandGroup candidates, then (if any of them is longer than its head
        // row) batches of kOvfChunks * 32 overflow neighbours of the group.
        // The fresh buffer is flushed at one place: before a unit that might
        // not fit, and at the end of the step (the kernel then holds few
        // inlined copies of flush, which keeps the hot loop's code compact).
        uint32_t c0 = 0, gc = 0;              // the current group
        uint64_t my_off = 0;                  // lane j < gc: candidate j's overflow offset
        uint32_t oexcl = 0, ototal = 0, f0 = 0;
        bool ovf = false;                     // overflow batches of the group left (warp-uniform)
        for (;;) {
            const bool done = !ovf && c0 >= cnt;
            const uint32_t need = ovf ? 32u * kOvfChunks
                                      : done ? (uint32_t) kBuf + 1u : min((uint32_t) kCandGroup, cnt - c0) * kHeadNbrs;
            if (nb && nb + need > kBuf) {
                n_dist += nb;
                nk = min(nk, flush<KIND, ORDER, CL, STORE>(a, m, nb, &sz, L, true, D, lane));
                nb = 0;
            }
            if (done) break;
            if (!ovf) {
                gc = min((uint32_t) kCandGroup, cnt - c0);
                // The head rows: one warp-wide 128-byte load per candidate, all
                // issued before any is used. Lane j < gc also fetches candidate
                // j's overflow offset (used if its row is longer than the head row).
                my_off = (uint32_t) lane < gc ? __ldg(a.ovf_off + m.cand[c0 + lane]) : 0ull;
                // The head rows stay in registers: lane l holds word l of every
                // candidate's row (word 0 the degree, words 1..31 neighbours), and
                // the test-and-sets go by candidate, one row per chunk, so the
                // neighbours keep their (candidate, slot) order.
                uint32_t hv[kCandGroup], olds[kCandGroup];
#pragma unroll
                for (int j = 0; j < kCandGroup; ++j)
                    hv[j] = (uint32_t) j < gc ? __ldg(a.head + (size_t) m.cand[c0 + j] * kHeadWords + lane) : 0u;
                uint32_t deg = 0, degsum = 0;
#pragma unroll
                for (int j = 0; j < kCandGroup; ++j) {
                    const uint32_t dj = __shfl_sync(kFull, hv[j], 0);  // 0 past the group
                    degsum += dj;
                    if (lane == j) deg = dj;
                    bool valid = lane >= 1 && (uint32_t) lane <= min(dj, (uint32_t) kHeadNbrs);
                    if (valid && hv[j] >= a.n) {
                        atomicOr(a.error, ERR_BAD_ID);
                        valid = false;
                    }
                    if (!valid) hv[j] = kFull;
                    olds[j] = visit_issue(vis, hv[j], valid);
                }
                n_edges += gc + degsum;
#pragma unroll
                for (int j = 0; j < kCandGroup; ++j) {
                    if ((uint32_t) j >= gc) break;
                    const uint32_t id = hv[j];
                    const bool valid = id != kFull;
                    const bool fresh = valid && !(olds[j] & (1u << (id & 31)));
                    note_dirty(dirty, a.dirty_cap, dcount, valid && olds[j] == 0, id >> 5);
                    append_ids(m, nb, fresh, id, lane);
                }
                // Rows longer than the head row: the rest from the overflow
                // lists of all the group's long candidates, flattened in
                // (candidate, slot) order, in the batches that follow.
                if (__any_sync(kFull, deg > (uint32_t) kHeadNbrs)) {
                    const uint32_t ocount = deg > (uint32_t) kHeadNbrs ? deg - kHeadNbrs : 0u;  // 0 for lanes >= gc
                    uint32_t oincl = ocount;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t t = __shfl_up_sync(kFull, oincl, o);
                        if (lane >= o) oincl += t;
                    }
                    ototal = __shfl_sync(kFull, oincl, 31);
                    oexcl = oincl - ocount;
                    f0 = 0;
                    ovf = true;
                } else {
                    c0 += kCandGroup;
                }
            } else {
                // One overflow batch: every load is issued before any
                // test-and-set, and every test-and-set before any result is used.
                uint32_t oid[kOvfChunks], oold[kOvfChunks];
#pragma unroll
                for (int ch = 0; ch < kOvfChunks; ++ch) {
                    const uint32_t f = f0 + ch * 32 + lane;
                    // owner: the last candidate whose flattened range starts at or before f
                    uint32_t j = 0;
                    for (uint32_t t = 1; t < gc; ++t)
                        if (__shfl_sync(kFull, oexcl, t) <= f) j = t;
                    const uint32_t pj = __shfl_sync(kFull, oexcl, j);
                    const uint64_t offj = __shfl_sync(kFull, my_off, j);
                    oid[ch] = f < ototal ? __ldg(a.ovf + offj + (f - pj)) : kFull;
                }
#pragma unroll
                for (int ch = 0; ch < kOvfChunks; ++ch) {
                    bool valid = oid[ch] != kFull;
                    if (valid && oid[ch] >= a.n) {
                        atomicOr(a.error, ERR_BAD_ID);
                        valid = false;
                        oid[ch] = kFull;
                    }
                    oold[ch] = visit_issue(vis, oid[ch], valid);
                }
#pragma unroll
                for (int ch = 0; ch < kOvfChunks; ++ch) {
                    if (f0 + ch * 32 >= ototal) break;
                    const uint32_t id = oid[ch];
                    const bool valid = id != kFull;
                    const bool fresh = valid && !(oold[ch] & (1u << (id & 31)));
                    note_dirty(dirty, a.dirty_cap, dcount, valid && oold[ch] == 0, id >> 5);
                    append_ids(m, nb, fresh, id, lane);
                }
                f0 += 32 * kOvfChunks;
                if (f0 >= ototal) {
                    ovf = false;
                    c0 += kCandGroup;
                }
            }
            __syncwarp();
        }
        k = nk <= last_k ? nk : last_k + 1;
    }

    if (STORE != STORE_FP32) {
        // Re-rank the final L with the exact float32 distance (reference lane
        // order); the K best by (distance, original id) go out.
        Dist<KIND, CL, STORE_FP32> E;
        E.load(a, q, lane);
        E.distances(a, m.qi, m.qd, sz, lane);
        rerank_output(m.qd, m.qi, sz, a.K, a.orig, a.out_ids + (size_t) q * a.K, lane);
    } else {
        // Results (original ids).
        for (uint32_t i = lane; i < a.K; i += 32)
            a.out_ids[(size_t) q * a.K + i] = __ldg(a.orig + (m.qi[i] & kIdMask));
    }
    if (lane == 0 && a.out_stats) a.out_stats[q] = make_uint4(n_dist, n_expand, n_edges, n_iter);
    // Clear the visited words this query set.
    if (dcount <= a.dirty_cap) {
        for (uint32_t i = lane; i < dcount; i += 32) vis[dirty[i]] = 0u;
    } else {
        for (uint32_t i = lane; i < a.vis_words; i += 32) vis[i] = 0u;
    }
    __syncwarp();
}

template <int KIND, int ORDER, int CL, int STORE>
__global__ void __launch_bounds__(128, PANNS_SEARCH_MIN_BLOCKS) search_kernel(SearchArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const WarpMem m = carve(smem + (size_t) wid * warp_smem_bytes(a.queue_cap), a.queue_cap);
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wid;
    uint32_t *vis = a.visited + (size_t) slot * a.vis_words;
    uint32_t *dirty = a.dirty + (size_t) slot * a.dirty_cap;
    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(a.counter, 1u);
        q = __shfl_sync(kFull, q, 0);
        if (q >= a.nq) break;
        search_one<KIND, ORDER, CL, STORE>(a, m, q, vis, dirty, lane);
    }
}

}  // namespace panns
