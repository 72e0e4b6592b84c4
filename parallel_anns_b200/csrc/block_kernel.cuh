// Several warps per query: the same search as search_kernel (PANNS order; the
// float32 rows, or a BF16 / FP8 copy with the exact float32 re-rank of the
// final L), for small batches where one warp per query leaves the GPU idle and
// every query pays the whole serial latency, and for long queues.
//
// One block of W warps runs one query at a time (work-stealing counter across
// blocks). The queue lives in the block's shared memory. A search step is:
//   1. warp 0 picks the M best unchecked candidates (as in search_kernel);
//   2. in rounds, warp w expands candidates w, w + W, ... (at most G per warp
//      and round, G * width <= kBuf so its fresh buffer cannot overflow):
//      head rows, visited test-and-set on the block's bitset, distances, then
//      the filter against the queue's L-th distance at the start of the round,
//      then a sort of its survivors;
//   3. the W sorted survivor lists are placed into one sorted list by rank
//      (each element's index plus the number of smaller elements in the other
//      lists; (distance, original id) is a total order), and the whole block
//      merges that list into the queue (the rank merge of merge_into, spread
//      over W * 32 threads).
// Each round's merge leaves the queue equal to the L best of (queue + round
// survivors), and the round's first insert position is the best survivor's,
// exactly as one flush of search_kernel (see the exactness note there), so
// ids and distance counts equal search_kernel's and the reference's.
#pragma once

#include "search_kernel.cuh"

namespace panns {

constexpr int kBlockCtl = 24;  // control words in shared memory (BC_SEG + W <= 24)

// Shared memory of one block of W warps with a queue of queue_cap entries.
__host__ __device__ inline uint32_t block_smem_bytes(uint32_t queue_cap, uint32_t W) {
    return queue_cap * 8u                                             // queue (dist, id)
           + W * (kBuf * 12u + kCandGroup * kHeadWords * 4u + 64u * 4u) // per-warp lists, head rows, scratch
           + W * kBuf * 12u                                           // merged sorted survivors
           + kMaxM * 4u                                               // picked candidates
           + kBlockCtl * 4u;                                          // control words
}

enum { BC_Q = 0, BC_SZ, BC_CNT, BC_LASTK, BC_K, BC_NK, BC_DIRTY, BC_DIST, BC_EDGES, BC_LRN, BC_LQ,
       BC_SEG };  // BC_SEG + w, w < W <= 8

// Number of elements of the sorted list (d, k)[0..n) that precede (dv, kv).
__device__ __forceinline__ uint32_t list_rank(const float *d, const uint32_t *k, uint32_t n, float dv, uint32_t kv) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (plain_less(d[mid], k[mid], dv, kv)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <int KIND, int CL, int W, int STORE>
__device__ void block_search_one(const SearchArgs &a, uint32_t q, uint8_t *smem, uint32_t *vis, uint32_t *dirty) {
    constexpr int T = W * 32;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint32_t qcap = a.queue_cap;
    float *qd = reinterpret_cast<float *>(smem);
    uint32_t *qi = reinterpret_cast<uint32_t *>(qd + qcap);
    float *segD = reinterpret_cast<float *>(qi + qcap);
    uint32_t *segI = reinterpret_cast<uint32_t *>(segD + W * kBuf);
    uint32_t *segK = segI + W * kBuf;
    uint32_t *hrowAll = segK + W * kBuf;
    uint32_t *preAll = hrowAll + W * kCandGroup * kHeadWords;
    float *cD = reinterpret_cast<float *>(preAll + W * 64);
    uint32_t *cI = reinterpret_cast<uint32_t *>(cD + W * kBuf);
    uint32_t *cK = cI + W * kBuf;
    uint32_t *cand = cK + W * kBuf;
    uint32_t *ctl = cand + kMaxM;
    float *bd = segD + w * kBuf;
    uint32_t *bi = segI + w * kBuf;
    uint32_t *bk = segK + w * kBuf;
    uint32_t *hrow = hrowAll + w * kCandGroup * kHeadWords;
    uint32_t *pre = preAll + w * 64;

    uint32_t L = a.Lq ? __ldg(a.Lq + q) : a.L;
    // Init ids: n_lrn learned entries (cand) then n_plain of the init list.
    uint32_t n_lrn = 0, n_plain = L;
    if (a.decisions) {
        if (w == 0) {
            const uint2 r = mlp_read_decision(a.decisions, a.dec_L_init, q, cand, lane);
            if (lane == 0) {
                ctl[BC_LRN] = r.x;
                ctl[BC_LQ] = r.y;
            }
        }
        __syncthreads();
        n_lrn = ctl[BC_LRN] & 0xffu;
        n_plain = ctl[BC_LRN] >> 8;
        L = ctl[BC_LQ];
    }
    const uint32_t n_init = n_lrn + n_plain;
    Dist<KIND, CL, STORE> D;
    D.load(a, q, lane);
    if (tid == 0) {
        ctl[BC_SZ] = 0;
        ctl[BC_DIRTY] = 0;
        ctl[BC_DIST] = 0;
        ctl[BC_EDGES] = 0;
        ctl[BC_K] = 0;
    }
    __syncthreads();

    // Block-wide list of the visited words that went from zero to non-zero.
    auto note_dirty_block = [&](bool first, uint32_t word) {
        const uint32_t bm = __ballot_sync(kFull, first);
        uint32_t base = 0;
        if (lane == 0 && bm) base = atomicAdd(&ctl[BC_DIRTY], (uint32_t) __popc(bm));
        base = __shfl_sync(kFull, base, 0);
        if (first) {
            const uint32_t pos = base + __popc(bm & lanemask_lt());
            if (pos < a.dirty_cap) dirty[pos] = word;
        }
    };

    // Merge the W sorted lists (counts in ctl[BC_SEG + w]) into the queue.
    // Returns nothing; updates ctl[BC_SZ] and ctl[BC_NK].
    auto block_merge = [&]() {
        const uint32_t my = ctl[BC_SEG + w];
        uint32_t total = 0;
#pragma unroll
        for (int v = 0; v < W; ++v) total += ctl[BC_SEG + v];
        for (uint32_t i = lane; i < my; i += 32) {
            const float dv = bd[i];
            const uint32_t kv = bk[i];
            uint32_t r = i;
#pragma unroll
            for (int v = 0; v < W; ++v)
                if (v != w) r += list_rank(segD + v * kBuf, segK + v * kBuf, ctl[BC_SEG + v], dv, kv);
            cD[r] = dv;
            cI[r] = bi[i];
        }
        __syncthreads();
        const uint32_t qsz = ctl[BC_SZ];
        if (total == 0) return;  // uniform
        for (uint32_t i = tid; i < total; i += T)
            cK[i] = i + queue_rank<ORDER_PANNS>(qd, qi, qsz, cD[i], cI[i] & kIdMask, a.orig);
        __syncthreads();
        const uint32_t p0 = cK[0];
        if (p0 < L) {
            for (int32_t top = (int32_t) qsz - 1; top >= (int32_t) p0; top -= T) {
                const int32_t j = top - tid;
                float d = 0.f;
                uint32_t id = 0, np = L;
                if (j >= (int32_t) p0) {
                    d = qd[j];
                    id = qi[j];
                    np = (uint32_t) j + fresh_rank<ORDER_PANNS>(cD, cI, total, d, id & kIdMask, a.orig);
                }
                __syncthreads();
                if (np < L) {
                    qd[np] = d;
                    qi[np] = id;
                }
                __syncthreads();
            }
            for (uint32_t i = tid; i < total; i += T) {
                const uint32_t np = cK[i];
                if (np < L) {
                    qd[np] = cD[i];
                    qi[np] = cI[i];
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            ctl[BC_SZ] = min(L, qsz + total);
            ctl[BC_NK] = min(ctl[BC_NK], p0 < L ? p0 : L);
        }
        __syncthreads();
    };

    // Distances, filter against the queue's L-th (bound), keys, sort; leaves
    // the warp's survivor count in ctl[BC_SEG + w].
    auto finish_list = [&](uint32_t nb, bool filter) {
        if constexpr (STORE == STORE_FP32) distances_wide<KIND, CL>(a, D.qv, bi, bd, nb, lane);
        else D.distances(a, bi, bd, nb, lane);
        if (lane == 0 && nb) atomicAdd(&ctl[BC_DIST], nb);
        const uint32_t sz = ctl[BC_SZ];
        const bool any_bound = filter && sz >= L;
        const float bound = any_bound ? qd[L - 1] : __int_as_float(0x7f800000);
        uint32_t cnt = 0;
        for (uint32_t b0 = 0; b0 < nb; b0 += 32) {
            const uint32_t b = b0 + lane;
            float d = 0.f;
            uint32_t id = 0;
            bool keep = false;
            if (b < nb) {
                d = bd[b];
                id = bi[b];
                keep = !any_bound || !(d > bound);
            }
            const uint32_t bm = __ballot_sync(kFull, keep);
            __syncwarp();
            if (keep) {
                const uint32_t pos = cnt + __popc(bm & lanemask_lt());
                bd[pos] = d;
                bi[pos] = id;
                bk[pos] = __ldg(a.orig + id);
            }
            cnt += __popc(bm);
            __syncwarp();
        }
        warp_sort<ORDER_PANNS>(bd, bi, bk, cnt, a.orig, lane);
        if (lane == 0) ctl[BC_SEG + w] = cnt;
    };

    // Initial queue: the init ids (learned entries first, a repeated id
    // entering once), W * kBuf at a time.
    const uint32_t *init = a.init_ids + (size_t) q * a.init_stride;
    for (uint32_t r0 = 0; r0 < n_init; r0 += W * kBuf) {
        uint32_t nb = 0;
        const uint32_t lo = r0 + w * kBuf, hi = min(n_init, lo + kBuf);
        for (uint32_t i0 = lo; i0 < hi; i0 += 32) {
            const uint32_t i = i0 + lane;
            const bool valid = i < hi;
            const uint32_t id = valid ? (i < n_lrn ? cand[i] : __ldg(init + (i - n_lrn))) : 0u;
            const bool ok = valid && id < a.n;
            if (valid && !ok) atomicOr(a.error, ERR_BAD_INIT);
            const uint32_t old = visit_issue(vis, id, ok);
            note_dirty_block(ok && old == 0, id >> 5);
            const bool fresh = ok && !(old & (1u << (id & 31)));
            const uint32_t bm = __ballot_sync(kFull, fresh);
            if (fresh) bi[nb + __popc(bm & lanemask_lt())] = id;
            nb += __popc(bm);
            __syncwarp();
        }
        finish_list(nb, false);
        if (tid == 0) ctl[BC_NK] = L;
        __syncthreads();
        block_merge();
    }

    uint32_t n_expand = 0, n_iter = 0;
    const uint32_t M = a.M;
    const uint32_t G = a.block_round;
    for (;;) {
        // 1. Pick (warp 0), exactly as search_kernel.
        if (w == 0) {
            const uint32_t k = ctl[BC_K], sz = ctl[BC_SZ];
            uint32_t cnt = 0, last_k = L;
            for (uint32_t p0 = k; p0 < sz && cnt < M; p0 += 32) {
                const uint32_t p = p0 + lane;
                const bool un = p < sz && !(qi[p] & kChecked);
                const uint32_t bm = __ballot_sync(kFull, un);
                const uint32_t take = min((uint32_t) __popc(bm), M - cnt);
                const uint32_t r = __popc(bm & lanemask_lt());
                if (un && r < take) {
                    const uint32_t id = qi[p];
                    qi[p] = id | kChecked;
                    cand[cnt + r] = id;
                }
                if (take) {
                    uint32_t x = bm;
                    for (uint32_t t = 1; t < take; ++t) x &= x - 1;
                    last_k = p0 + (__ffs(x) - 1);
                }
                cnt += take;
                __syncwarp();
            }
            if (lane == 0) {
                ctl[BC_CNT] = cnt;
                ctl[BC_LASTK] = last_k;
                ctl[BC_NK] = L;
            }
        }
        __syncthreads();
        const uint32_t cnt = ctl[BC_CNT];
        if (cnt == 0) break;
        ++n_iter;
        n_expand += cnt;
        // 2-3. Rounds of at most G candidates per warp.
        for (uint32_t r0 = 0; r0 < cnt; r0 += W * G) {
            // this warp's candidates: r0 + w + W * t, t < G
            uint32_t gc = 0;
            for (uint32_t t = 0; t < G; ++t)
                if (r0 + w + W * t < cnt) ++gc;
            uint32_t nb = 0;
            if (gc) {
                uint32_t hv[kCandGroup];
#pragma unroll
                for (int j = 0; j < kCandGroup; ++j)
                    hv[j] = (uint32_t) j < gc ? __ldg(a.head + (size_t) cand[r0 + w + W * j] * kHeadWords + lane) : 0u;
#pragma unroll
                for (int j = 0; j < kCandGroup; ++j)
                    if ((uint32_t) j < gc) hrow[j * kHeadWords + lane] = hv[j];
            }
            __syncwarp();
            uint32_t deg = 0, hcount = 0;
            if (lane < (int) gc) {
                deg = hrow[lane * kHeadWords];
                hcount = min(deg, (uint32_t) kHeadNbrs);
            }
            uint32_t incl = hcount;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += t;
            }
            const uint32_t total = __shfl_sync(kFull, incl, 31);
            if (lane < (int) gc) pre[lane] = incl - hcount;
            uint32_t degsum = deg;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) degsum += __shfl_xor_sync(kFull, degsum, o);
            if (lane == 0 && gc) atomicAdd(&ctl[BC_EDGES], gc + degsum);
            const bool any_long = __any_sync(kFull, deg > (uint32_t) kHeadNbrs);
            __syncwarp();
            // Head-row neighbours: every visited test-and-set of the round is
            // issued before any result is used (total <= kCandGroup * 31).
            uint32_t ids[kGroupChunks], olds[kGroupChunks];
#pragma unroll
            for (int ch = 0; ch < kGroupChunks; ++ch) {
                const uint32_t f = ch * 32 + lane;
                uint32_t id = 0;
                bool valid = f < total;
                if (valid) {
                    uint32_t j = 0;
                    while (j + 1 < gc && pre[j + 1] <= f) ++j;
                    id = hrow[j * kHeadWords + 1 + (f - pre[j])];
                    if (id >= a.n) {
                        atomicOr(a.error, ERR_BAD_ID);
                        valid = false;
                    }
                }
                ids[ch] = valid ? id : kFull;
                olds[ch] = visit_issue(vis, id, valid);
            }
#pragma unroll
            for (int ch = 0; ch < kGroupChunks; ++ch) {
                if (ch * 32 >= (int) total) break;
                const uint32_t id = ids[ch];
                const bool valid = id != kFull;
                const bool fresh = valid && !(olds[ch] & (1u << (id & 31)));
                note_dirty_block(valid && olds[ch] == 0, id >> 5);
                const uint32_t bm = __ballot_sync(kFull, fresh);
                if (fresh) bi[nb + __popc(bm & lanemask_lt())] = id;
                nb += __popc(bm);
                __syncwarp();
            }
            if (any_long) {
                for (uint32_t j = 0; j < gc; ++j) {
                    const uint32_t dj = hrow[j * kHeadWords];
                    if (dj <= (uint32_t) kHeadNbrs) continue;
                    const uint64_t off = __ldg(a.ovf_off + cand[r0 + w + W * j]);
                    for (uint32_t s0 = kHeadNbrs; s0 < dj; s0 += 32) {
                        const uint32_t s = s0 + lane;
                        bool valid = s < dj;
                        const uint32_t id = valid ? __ldg(a.ovf + off + (s - kHeadNbrs)) : 0u;
                        if (valid && id >= a.n) {
                            atomicOr(a.error, ERR_BAD_ID);
                            valid = false;
                        }
                        const uint32_t old = visit_issue(vis, id, valid);
                        const bool fresh = valid && !(old & (1u << (id & 31)));
                        note_dirty_block(valid && old == 0, id >> 5);
                        const uint32_t bm = __ballot_sync(kFull, fresh);
                        if (fresh) bi[nb + __popc(bm & lanemask_lt())] = id;
                        nb += __popc(bm);
                        __syncwarp();
                    }
                }
            }
            finish_list(nb, true);
            __syncthreads();
            block_merge();
        }
        if (tid == 0) {
            const uint32_t nk = ctl[BC_NK], last_k = ctl[BC_LASTK];
            ctl[BC_K] = nk <= last_k ? nk : last_k + 1;
        }
        __syncthreads();
    }

    if constexpr (STORE != STORE_FP32) {
        // Re-rank the final L in exact float32 (warp 0), as search_kernel does.
        if (w == 0) {
            Dist<KIND, CL, STORE_FP32> E;
            E.load(a, q, lane);
            const uint32_t sz = ctl[BC_SZ];
            E.distances(a, qi, qd, sz, lane);
            rerank_output(qd, qi, sz, a.K, a.orig, a.out_ids + (size_t) q * a.K, lane);
        }
    } else {
        for (uint32_t i = tid; i < a.K; i += T) a.out_ids[(size_t) q * a.K + i] = __ldg(a.orig + (qi[i] & kIdMask));
    }
    if (tid == 0 && a.out_stats) a.out_stats[q] = make_uint4(ctl[BC_DIST], n_expand, ctl[BC_EDGES], n_iter);
    const uint32_t dcount = ctl[BC_DIRTY];
    if (dcount <= a.dirty_cap) {
        for (uint32_t i = tid; i < dcount; i += T) vis[dirty[i]] = 0u;
    } else {
        for (uint32_t i = tid; i < a.vis_words; i += T) vis[i] = 0u;
    }
    __syncthreads();
}

template <int KIND, int CL, int W, int STORE>
__global__ void __launch_bounds__(W * 32) search_block_kernel(SearchArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t slot = blockIdx.x;
    uint32_t *vis = a.visited + (size_t) slot * a.vis_words;
    uint32_t *dirty = a.dirty + (size_t) slot * a.dirty_cap;
    uint32_t *ctl = reinterpret_cast<uint32_t *>(smem + block_smem_bytes(a.queue_cap, W) - kBlockCtl * 4);
    for (;;) {
        if (threadIdx.x == 0) ctl[BC_Q] = atomicAdd(a.counter, 1u);
        __syncthreads();
        const uint32_t q = ctl[BC_Q];
        __syncthreads();
        if (q >= a.nq) break;
        block_search_one<KIND, CL, W, STORE>(a, q, smem, vis, dirty);
    }
}

}  // namespace panns
