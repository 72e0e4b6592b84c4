// PSS_v5 with T queues on the GPU: one warp per query.
//
// Reference: core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:1218-1515
// (large-graph twin :1376-1726 of core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.cpp).
// Stage structure, all in shared memory:
//   pick   pick_top_m_to_workers (:756-786): the master's unchecked candidates
//          from k_master are dealt round-robin to workers 0..T-2; every T-th is
//          skipped and stays unchecked in the master; dealing stops when a
//          worker queue reaches L_local.
//   expand each queue runs its own best-first loop for up to X expansions
//          (:1403-1456). The reference runs them in parallel threads that race
//          on the shared visited bitset; here they run in a fixed round-robin
//          order: in every round worker 0, 1, ..., T-2 and then the master each
//          expand one candidate. Every neighbour bound is the master's L-th
//          distance, as in the reference.
//   merge  merge_all_queues_to_master (:642-681) with
//          merge_two_queues_into_1st_queue_seq_fixed (:479-550): each worker
//          queue, in worker order, is merged into the master's L; a candidate
//          the worker holds unchecked re-opens the master's checked copy; the
//          lowest insert position pulls k_master back.
// One expansion's neighbours are processed by the whole warp at once (the
// visited test-and-set, the distances, one sorted merge), which gives the
// same queue as the reference's one-by-one inserts (see search_kernel.cuh).
#pragma once

#include "search_kernel.cuh"

namespace panns {

struct PssArgs {
    SearchArgs s;
    uint32_t T, L_local, X;
    uint32_t wcap;  // shared-memory entries per worker queue (>= L_local)
};

__host__ __device__ inline uint32_t pss_smem_bytes(uint32_t qcap, uint32_t T, uint32_t wcap) {
    return qcap * 8u + (T - 1) * wcap * 8u + kBuf * 12u + 4u * ((3u * T + 31u) / 32u * 32u) + 64u * 4u;
}

struct PssMem {
    float *md;       // master queue
    uint32_t *mi;
    float *wd;       // worker queues, (T-1) x wcap
    uint32_t *wi;
    float *bd;       // fresh buffer
    uint32_t *bi;
    uint32_t *bk;
    uint32_t *wsz;   // queue sizes (T; the master's is L)
    uint32_t *kuc;   // per-queue scan position
    uint32_t *iters; // per-queue expansions this stage
};

// Distances of the buffered fresh vertices, keep those not above the master's
// L-th distance, sort, merge into (qd, qi) of size *sz and capacity cap.
template <int KIND, int CL>
__device__ uint32_t pss_flush(const SearchArgs &a, const PssMem &m, uint32_t nb, float *qd, uint32_t *qi,
                              uint32_t *sz, uint32_t cap, const float4 (&qv)[CL], int lane) {
    const int g = lane >> 3;
    for (uint32_t b0 = 0; b0 < nb; b0 += 8) {
        const uint32_t b = b0 + g, bb = b0 + 4 + g;
        const bool act0 = b < nb, act1 = bb < nb;
        const uint32_t v0 = act0 ? m.bi[b] : 0u, v1 = act1 ? m.bi[bb] : 0u;
        float d0, d1;
        group_distance2<KIND, CL>(a.vec, a.norms, v0, act0, v1, act1, qv, lane, d0, d1);
        if ((lane & 7) == 0) {
            if (act0) m.bd[b] = d0;
            if (act1) m.bd[bb] = d1;
        }
    }
    __syncwarp();
    const float bound = m.md[a.L - 1];
    uint32_t cnt = 0;
    for (uint32_t b0 = 0; b0 < nb; b0 += 32) {
        const uint32_t b = b0 + lane;
        float d = 0.f;
        uint32_t id = 0;
        bool keep = false;
        if (b < nb) {
            d = m.bd[b];
            id = m.bi[b];
            keep = !(d > bound);
        }
        const uint32_t bm = __ballot_sync(kFull, keep);
        __syncwarp();
        if (keep) {
            const uint32_t pos = cnt + __popc(bm & lanemask_lt());
            m.bd[pos] = d;
            m.bi[pos] = id;
            m.bk[pos] = __ldg(a.orig + id);
        }
        cnt += __popc(bm);
        __syncwarp();
    }
    if (cnt == 0) return cap;
    warp_sort<ORDER_PANNS>(m.bd, m.bi, m.bk, cnt, a.orig, lane);
    return merge_into<ORDER_PANNS>(qd, qi, sz, cap, m.bd, m.bi, m.bk, cnt, a.orig, lane);
}

// expand_one_candidate (:824-895): visit the neighbours of device vertex v,
// insert the fresh ones into (qd, qi, *sz, cap). Returns the lowest insert
// position or cap.
template <int KIND, int CL>
__device__ uint32_t pss_expand(const SearchArgs &a, const PssMem &m, uint32_t v, float *qd, uint32_t *qi,
                               uint32_t *sz, uint32_t cap, uint32_t *vis, uint32_t *dirty,
                               uint32_t &dcount, uint32_t &n_dist, uint32_t &n_edges,
                               const float4 (&qv)[CL], int lane) {
    const uint32_t hw = __ldg(a.head + (size_t) v * kHeadWords + lane);
    const uint32_t deg = __shfl_sync(kFull, hw, 0);
    n_edges += 1 + deg;
    uint64_t off = 0;
    if (deg > (uint32_t) kHeadNbrs) off = __ldg(a.ovf_off + v);
    uint32_t nk = cap, nb = 0;
    for (uint32_t s0 = 0; s0 < deg; s0 += 32) {
        const uint32_t s = s0 + lane;
        bool valid = s < deg;
        // slot s: head word s + 1 for s < 31, else overflow entry s - 31
        const uint32_t from_head = __shfl_sync(kFull, hw, (lane + 1) & 31);
        uint32_t id = 0;
        if (valid) id = (s < (uint32_t) kHeadNbrs) ? from_head : __ldg(a.ovf + off + (s - kHeadNbrs));
        if (valid && id >= a.n) {
            atomicOr(a.error, ERR_BAD_ID);
            valid = false;
        }
        const uint32_t old = visit_issue(vis, id, valid);
        const bool fresh = valid && !(old & (1u << (id & 31)));
        note_dirty(dirty, a.dirty_cap, dcount, valid && old == 0, id >> 5);
        if (nb + 32 > kBuf) {
            n_dist += nb;
            nk = min(nk, pss_flush<KIND, CL>(a, m, nb, qd, qi, sz, cap, qv, lane));
            nb = 0;
        }
        const uint32_t bm = __ballot_sync(kFull, fresh);
        if (fresh) m.bi[nb + __popc(bm & lanemask_lt())] = id;
        nb += __popc(bm);
        __syncwarp();
    }
    if (nb) {
        n_dist += nb;
        nk = min(nk, pss_flush<KIND, CL>(a, m, nb, qd, qi, sz, cap, qv, lane));
    }
    return nk;
}

// merge_two_queues_into_1st_queue_seq_fixed (:479-550): merge worker queue
// (wd, wi)[0..s) into the master's L. Returns the lower bound of the worker's
// first element in the master (L if none).
static __device__ uint32_t pss_merge_fixed(const SearchArgs &a, const PssMem &m, const float *wd, const uint32_t *wi,
                                    uint32_t s, int lane) {
    const uint32_t L = a.L;
    const uint32_t pos0 = queue_rank<ORDER_PANNS>(m.md, m.mi, L, wd[0], wi[0] & kIdMask, a.orig);
    if (pos0 >= L) return L;
    if (pos0 == L - 1) {
        if (lane == 0) {
            m.md[L - 1] = wd[0];
            m.mi[L - 1] = wi[0];
        }
        __syncwarp();
        return pos0;
    }
    uint32_t msz = L;
    for (uint32_t c0 = 0; c0 < s; c0 += kBuf) {
        const uint32_t cn = min((uint32_t) kBuf, s - c0);
        uint32_t cnt = 0;
        for (uint32_t b0 = 0; b0 < cn; b0 += 32) {
            const uint32_t b = b0 + lane;
            bool keep = false;
            float d = 0.f;
            uint32_t id = 0;
            if (b < cn) {
                d = wd[c0 + b];
                id = wi[c0 + b];
                const uint32_t lb = queue_rank<ORDER_PANNS>(m.md, m.mi, msz, d, id & kIdMask, a.orig);
                const bool dup = lb < msz && (m.mi[lb] & kIdMask) == (id & kIdMask);
                if (dup) {
                    // the worker still holds it unchecked: re-open the master's copy
                    if (!(id & kChecked) && (m.mi[lb] & kChecked)) m.mi[lb] &= kIdMask;
                } else {
                    keep = true;
                }
            }
            const uint32_t bm = __ballot_sync(kFull, keep);
            __syncwarp();
            if (keep) {
                const uint32_t pos = cnt + __popc(bm & lanemask_lt());
                m.bd[pos] = d;
                m.bi[pos] = id;
            }
            cnt += __popc(bm);
            __syncwarp();
        }
        merge_into<ORDER_PANNS>(m.md, m.mi, &msz, L, m.bd, m.bi, m.bk, cnt, a.orig, lane);
    }
    return pos0;
}

// First unchecked position in [from, size) or size.
static __device__ __forceinline__ uint32_t first_unchecked(const uint32_t *qi, uint32_t from, uint32_t size, int lane) {
    for (uint32_t p0 = from; p0 < size; p0 += 32) {
        const uint32_t p = p0 + lane;
        const uint32_t bm = __ballot_sync(kFull, p < size && !(qi[p] & kChecked));
        if (bm) return p0 + __ffs(bm) - 1;
    }
    return size;
}

template <int KIND, int CL>
__device__ void pss_one(const PssArgs &pa, const PssMem &m, uint32_t q, uint32_t *vis, uint32_t *dirty,
                        int lane) {
    const SearchArgs &a = pa.s;
    const uint32_t L = a.L, T = pa.T, Ll = pa.L_local, X = pa.X, wcap = pa.wcap;
    float4 qv[CL];
    {
        const float4 *qrow = a.queries + (size_t) q * (CL * 8);
#pragma unroll
        for (int i = 0; i < CL; ++i) qv[i] = __ldg(qrow + 8 * i + (lane & 7));
    }
    uint32_t dcount = 0, n_dist = 0, n_expand = 0, n_edges = 0, n_iter = 0;
    // Initial master queue (initialize_set_L_para :897-935).
    uint32_t msz = 0;
    {
        uint32_t nb = 0;
        for (uint32_t i0 = 0; i0 < L; i0 += 32) {
            const uint32_t i = i0 + lane;
            const bool valid = i < L;
            const uint32_t id = valid ? __ldg(a.init_ids + i) : 0u;
            const bool ok = valid && id < a.n;
            if (valid && !ok) atomicOr(a.error, ERR_BAD_INIT);
            const uint32_t old = visit_issue(vis, id, ok);
            note_dirty(dirty, a.dirty_cap, dcount, ok && old == 0, id >> 5);
            const uint32_t bm = __ballot_sync(kFull, ok);
            if (ok) m.bi[nb + __popc(bm & lanemask_lt())] = id;
            nb += __popc(bm);
            __syncwarp();
            if (nb > kBuf - 32 || i0 + 32 >= L) {
                // no bound yet: distances, sort, merge
                const int g = lane >> 3;
                for (uint32_t b0 = 0; b0 < nb; b0 += 8) {
                    const uint32_t b = b0 + g, bb = b0 + 4 + g;
                    const bool act0 = b < nb, act1 = bb < nb;
                    float d0, d1;
                    group_distance2<KIND, CL>(a.vec, a.norms, act0 ? m.bi[b] : 0u, act0,
                                              act1 ? m.bi[bb] : 0u, act1, qv, lane, d0, d1);
                    if ((lane & 7) == 0) {
                        if (act0) m.bd[b] = d0;
                        if (act1) m.bd[bb] = d1;
                    }
                }
                __syncwarp();
                for (uint32_t b = lane; b < nb; b += 32) m.bk[b] = __ldg(a.orig + m.bi[b]);
                __syncwarp();
                warp_sort<ORDER_PANNS>(m.bd, m.bi, m.bk, nb, a.orig, lane);
                merge_into<ORDER_PANNS>(m.md, m.mi, &msz, L, m.bd, m.bi, m.bk, nb, a.orig, lane);
                n_dist += nb;
                nb = 0;
            }
        }
    }
    uint32_t k_master = 0;
    // One sequential expansion (seq_iter_bound = 1).
    {
        uint32_t r = L;
        if (!(m.mi[0] & kChecked)) {
            const uint32_t v = m.mi[0];
            __syncwarp();
            if (lane == 0) m.mi[0] = v | kChecked;
            __syncwarp();
            ++n_expand;
            r = pss_expand<KIND, CL>(a, m, v, m.md, m.mi, &msz, L, vis, dirty, dcount, n_dist, n_edges, qv, lane);
        }
        k_master = r <= k_master ? r : k_master + 1;
    }
    const uint32_t limit = (Ll - 1) * T + 1;  // dealt candidates when worker 0 fills
    for (;;) {
        ++n_iter;
        // pick_top_m_to_workers
        uint32_t seen = 0;
        for (uint32_t p0 = k_master; p0 < L && seen < limit; p0 += 32) {
            const uint32_t p = p0 + lane;
            const bool un = p < L && !(m.mi[p] & kChecked);
            const uint32_t bm = __ballot_sync(kFull, un);
            const uint32_t i = seen + __popc(bm & lanemask_lt());
            if (un && i < limit) {
                const uint32_t dest = i % T;
                if (dest != T - 1) {
                    const uint32_t slot = i / T;
                    m.wd[(size_t) dest * wcap + slot] = m.md[p];
                    m.wi[(size_t) dest * wcap + slot] = m.mi[p];
                    m.mi[p] |= kChecked;
                }
            }
            seen += __popc(bm);
            __syncwarp();
        }
        const uint32_t count = min(seen, limit);
        if (count == 0) break;
        for (uint32_t w = lane; w < T; w += 32) {
            m.wsz[w] = w == T - 1 ? L : (count > w ? (count - 1 - w) / T + 1 : 0u);
            m.kuc[w] = w == T - 1 ? k_master : 0u;
            m.iters[w] = 0;
        }
        __syncwarp();
        // Expand: rounds of one expansion per queue, workers first, master last.
        for (;;) {
            bool any = false;
            for (uint32_t w = 0; w < T; ++w) {
                const bool master = w == T - 1;
                float *qd = master ? m.md : m.wd + (size_t) w * wcap;
                uint32_t *qi = master ? m.mi : m.wi + (size_t) w * wcap;
                const uint32_t cap = master ? L : Ll;
                uint32_t size = master ? msz : m.wsz[w];
                uint32_t kuc = m.kuc[w];
                if (m.iters[w] >= X || kuc >= size) continue;
                const uint32_t p = first_unchecked(qi, kuc, size, lane);
                if (p >= size) {
                    if (lane == 0) m.kuc[w] = size;
                    __syncwarp();
                    continue;
                }
                const uint32_t v = qi[p];
                __syncwarp();
                if (lane == 0) {
                    qi[p] = v | kChecked;
                    m.iters[w] += 1;
                }
                __syncwarp();
                ++n_expand;
                const uint32_t r = pss_expand<KIND, CL>(a, m, v & kIdMask, qd, qi, &size, cap, vis, dirty,
                                                        dcount, n_dist, n_edges, qv, lane);
                if (master) msz = size;
                __syncwarp();
                if (lane == 0) {
                    m.kuc[w] = r <= p ? r : p + 1;
                    if (!master) m.wsz[w] = size;
                }
                __syncwarp();
                any = true;
            }
            if (!any) break;
        }
        k_master = m.kuc[T - 1];
        // Merge the workers into the master, in worker order.
        uint32_t nk = L;
        for (uint32_t w = 0; w + 1 < T; ++w) {
            const uint32_t s = m.wsz[w];
            if (!s) continue;
            const uint32_t r = pss_merge_fixed(a, m, m.wd + (size_t) w * wcap, m.wi + (size_t) w * wcap, s, lane);
            nk = min(nk, r);
        }
        if (nk <= k_master) k_master = nk;
    }
    for (uint32_t i = lane; i < a.K; i += 32)
        a.out_ids[(size_t) q * a.K + i] = __ldg(a.orig + (m.mi[i] & kIdMask));
    if (lane == 0 && a.out_stats) a.out_stats[q] = make_uint4(n_dist, n_expand, n_edges, n_iter);
    if (dcount <= a.dirty_cap) {
        for (uint32_t i = lane; i < dcount; i += 32) vis[dirty[i]] = 0u;
    } else {
        for (uint32_t i = lane; i < a.vis_words; i += 32) vis[i] = 0u;
    }
    __syncwarp();
}

template <int KIND, int CL>
__global__ void __launch_bounds__(128, 4) pss_kernel(PssArgs pa) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const SearchArgs &a = pa.s;
    const uint32_t qcap = a.queue_cap;
    uint8_t *base = smem + (size_t) wid * pss_smem_bytes(qcap, pa.T, pa.wcap);
    PssMem m;
    m.md = reinterpret_cast<float *>(base);
    m.mi = reinterpret_cast<uint32_t *>(m.md + qcap);
    m.wd = reinterpret_cast<float *>(m.mi + qcap);
    m.wi = reinterpret_cast<uint32_t *>(m.wd + (size_t) (pa.T - 1) * pa.wcap);
    m.bd = reinterpret_cast<float *>(m.wi + (size_t) (pa.T - 1) * pa.wcap);
    m.bi = reinterpret_cast<uint32_t *>(m.bd + kBuf);
    m.bk = m.bi + kBuf;
    m.wsz = m.bk + kBuf;
    m.kuc = m.wsz + pa.T;
    m.iters = m.kuc + pa.T;
    const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + wid;
    uint32_t *vis = a.visited + (size_t) slot * a.vis_words;
    uint32_t *dirty = a.dirty + (size_t) slot * a.dirty_cap;
    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(a.counter, 1u);
        q = __shfl_sync(kFull, q, 0);
        if (q >= a.nq) break;
        pss_one<KIND, CL>(pa, m, q, vis, dirty, lane);
    }
}

}  // namespace panns
