// efanna2e IndexNSG::Build on one GPU (include/efanna2e/index_nsg.cpp).
//
// The reference builds an NSG from a k-NN graph in five steps, restated here
// with the reference's arithmetic and order:
//   1. init_graph (:209-224): the float mean of the rows (summed in id
//      order), a random start vertex (rand() % n) and a search for the mean
//      from it over the k-NN graph; the best vertex found is the navigating
//      node ep.
//   2. Link, first loop (:372-395): for every vertex q, get_neighbors
//      (:141-207), an efanna2e search for q over the k-NN graph from the init
//      list (ep's k-NN list, then rand() ids) that keeps every vertex whose
//      distance it computes; then sync_prune (:226-276): that pool plus q's
//      k-NN neighbours it did not visit, sorted by distance, q itself
//      skipped, each kept unless a kept r has d(r, p) < d(q, p), at most R of
//      the first C.
//   3. Link, second loop (:397-403), InterInsert (:278-354): every vertex n,
//      in id order, offers itself to each of its kept neighbours' lists,
//      which are pruned again when they overflow R.
//   4. the lists become the graph (:419-434);
//   5. tree_grow (:702-718): depth-first from ep; the first vertex not
//      reached is attached (findroot :670-700) to the nearest reached vertex a
//      search for it finds, and the walk goes on from there.
// Step 2 is independent per vertex once its init list is known, and that list
// depends only on the position in the rand() stream, so the host replays
// glibc's rand() for every vertex in id order (the reference at one thread)
// and the GPU runs every vertex's search and prune at once, one warp per
// vertex. Steps 1 and 3-5 are sequential in the reference and run on the
// host.
//
// Distances are the reference's DistanceL2 (include/efanna2e/distance.h:24-60)
// as its -O3 -march=native build computes it: 8 lane accumulators, lane j
// summing elements j, j+8, ... (the last 8 first when d % 16 == 8), each step
// one FMA, then the lanes added 0..7 left to right.
//
// Ties: the reference sorts pools with std::sort by distance only, which
// leaves the order of exactly equal distances unspecified. The host steps call
// the same std::sort on the same sequences; the GPU step orders equal
// distances by arrival. Only inputs with exactly equal distances (duplicate
// rows, for instance) can therefore give a different graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <stack>
#include <string>
#include <vector>

#include "../../include/panns_build.h"
#include "graph_types.h"
#include "learned.h"
#include "search_kernel.cuh"

namespace panns {
namespace {

#define NCU(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return set_error(PANNS_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
struct NBuf {
    T *p = nullptr;
    ~NBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

// DistanceL2::compare of rows a and b (either order gives the same bits).
__host__ __device__ inline float l2_ref(const float *a, const float *b, uint32_t d) {
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const uint32_t DR = d % 16, DD = d - DR;
    if (DR) {
        for (int j = 0; j < 8; ++j) {
            const float t = a[DD + j] - b[DD + j];
            acc[j] = fmaf(t, t, acc[j]);
        }
    }
    for (uint32_t i = 0; i < DD; i += 8)
        for (int j = 0; j < 8; ++j) {
            const float t = a[i + j] - b[i + j];
            acc[j] = fmaf(t, t, acc[j]);
        }
    float r = acc[0];
    for (int j = 1; j < 8; ++j) r = r + acc[j];
    return r;
}

constexpr uint32_t kLinkBuf = 256;     // fresh vertices per flush
constexpr uint32_t kLinkDirty = 4096;  // cleared-word list per warp
constexpr uint32_t kLinkMaxR = 256;
constexpr uint32_t kLinkWarps = 4;

enum : uint32_t { LINK_ERR_BAD_ID = 1u, LINK_ERR_SHORT_POOL = 2u };

struct LinkArgs {
    const float *x;         // n x d rows
    uint32_t n, d;
    const uint32_t *knn;    // n x K
    uint32_t K;
    const uint32_t *init;   // n x L init ids
    uint32_t L, R, C, Lc, Cc;
    uint32_t *visited;      // slots x vis_words
    uint32_t vis_words;
    uint32_t *dirty;        // slots x kLinkDirty
    uint32_t *cut_ids;      // n x R
    float *cut_d;           // n x R
    uint32_t *cut_n;        // n
    uint32_t *counter;
    uint32_t *error;
};

__host__ __device__ inline size_t link_warp_bytes(uint32_t Lc, uint32_t Cc) {
    return (size_t) (Lc + Cc) * 8 + kLinkBuf * 12 + kLinkMaxR * 4;
}

// Distances of q to bi[0..nb), one lane per vertex, into bd; keys = arrival.
__device__ void link_distances(const LinkArgs &a, const float *qrow, const uint32_t *bi, float *bd, uint32_t *bk,
                               uint32_t nb, uint32_t key0, int lane) {
    for (uint32_t i = lane; i < nb; i += 32) {
        bd[i] = l2_ref(a.x + (size_t) bi[i] * a.d, qrow, a.d);
        bk[i] = key0 + i;
    }
    __syncwarp();
}

// Sort the buffered fresh vertices, merge them all into the pool (top C),
// then the ones under the queue's bound into the queue (top L). Returns the
// queue position of the best one inserted, or L.
__device__ uint32_t link_flush(const LinkArgs &a, const float *qrow, float *qd, uint32_t *qi, uint32_t *qsz,
                               float *pd, uint32_t *pi, uint32_t *psz, float *bd, uint32_t *bi, uint32_t *bk,
                               uint32_t nb, uint32_t &key, bool filter, int lane) {
    if (nb == 0) return a.L;
    link_distances(a, qrow, bi, bd, bk, nb, key, lane);
    key += nb;
    warp_sort<ORDER_EFANNA>(bd, bi, bk, nb, nullptr, lane);
    merge_into<ORDER_EFANNA>(pd, pi, psz, a.C, bd, bi, bk, nb, nullptr, lane);
    // survivors, in their sorted order
    const bool bounded = filter && *qsz >= a.L;
    const float bound = bounded ? qd[a.L - 1] : 0.f;
    uint32_t cnt = 0;
    for (uint32_t b0 = 0; b0 < nb; b0 += 32) {
        const uint32_t b = b0 + lane;
        float dv = 0.f;
        uint32_t id = 0;
        bool keep = false;
        if (b < nb) {
            dv = bd[b];
            id = bi[b];
            keep = !bounded || dv < bound;
        }
        const uint32_t bm = __ballot_sync(kFull, keep);
        __syncwarp();
        if (keep) {
            const uint32_t pos = cnt + __popc(bm & lanemask_lt());
            bd[pos] = dv;
            bi[pos] = id;
        }
        cnt += __popc(bm);
        __syncwarp();
    }
    if (cnt == 0) return a.L;
    return merge_into<ORDER_EFANNA>(qd, qi, qsz, a.L, bd, bi, bk, cnt, nullptr, lane);
}

// One warp per vertex: get_neighbors over the k-NN graph, then sync_prune.
__global__ void __launch_bounds__(kLinkWarps * 32) link_kernel(LinkArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint8_t *base = smem + (size_t) wid * link_warp_bytes(a.Lc, a.Cc);
    float *qd = reinterpret_cast<float *>(base);
    uint32_t *qi = reinterpret_cast<uint32_t *>(qd + a.Lc);
    float *pd = reinterpret_cast<float *>(qi + a.Lc);
    uint32_t *pi = reinterpret_cast<uint32_t *>(pd + a.Cc);
    float *bd = reinterpret_cast<float *>(pi + a.Cc);
    uint32_t *bi = reinterpret_cast<uint32_t *>(bd + kLinkBuf);
    uint32_t *bk = bi + kLinkBuf;
    uint32_t *rid = bk + kLinkBuf;
    const uint32_t slot = blockIdx.x * kLinkWarps + wid;
    uint32_t *vis = a.visited + (size_t) slot * a.vis_words;
    uint32_t *dirty = a.dirty + (size_t) slot * kLinkDirty;
    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(a.counter, 1u);
        q = __shfl_sync(kFull, q, 0);
        if (q >= a.n) break;
        const float *qrow = a.x + (size_t) q * a.d;
        uint32_t dcount = 0, qsz = 0, psz = 0, key = 0, nb = 0;
        // Init list: every id marked, distances computed, all kept (pool and queue).
        const uint32_t *init = a.init + (size_t) q * a.L;
        for (uint32_t i0 = 0; i0 < a.L; i0 += 32) {
            const uint32_t i = i0 + lane;
            const bool valid = i < a.L;
            const uint32_t id = valid ? __ldg(init + i) : 0u;
            const bool ok = valid && id < a.n;
            if (valid && !ok) atomicOr(a.error, LINK_ERR_BAD_ID);
            const uint32_t old = visit_issue(vis, id, ok);
            note_dirty(dirty, kLinkDirty, dcount, ok && old == 0, id >> 5);
            const bool fresh = ok && !(old & (1u << (id & 31)));
            const uint32_t bm = __ballot_sync(kFull, fresh);
            if (fresh) bi[nb + __popc(bm & lanemask_lt())] = id;
            nb += __popc(bm);
            __syncwarp();
            if (nb > kLinkBuf - 32 || i0 + 32 >= a.L) {
                link_flush(a, qrow, qd, qi, &qsz, pd, pi, &psz, bd, bi, bk, nb, key, false, lane);
                nb = 0;
            }
        }
        // The search: expand the first unchecked entry, k as in get_neighbors.
        uint32_t k = 0;
        while (k < qsz) {
            uint32_t nk = a.L;
            const uint32_t e = qi[k];
            __syncwarp();
            if (!(e & kChecked)) {
                if (lane == 0) qi[k] = e | kChecked;
                const uint32_t cand = e & kIdMask;
                nb = 0;
                for (uint32_t c0 = 0; c0 < a.K; c0 += 32) {
                    const uint32_t c = c0 + lane;
                    uint32_t id = c < a.K ? __ldg(a.knn + (size_t) cand * a.K + c) : 0u;
                    bool ok = c < a.K;
                    if (ok && id >= a.n) {
                        atomicOr(a.error, LINK_ERR_BAD_ID);
                        ok = false;
                    }
                    const uint32_t old = visit_issue(vis, id, ok);
                    note_dirty(dirty, kLinkDirty, dcount, ok && old == 0, id >> 5);
                    const bool fresh = ok && !(old & (1u << (id & 31)));
                    if (nb + 32 > kLinkBuf) {
                        nk = min(nk, link_flush(a, qrow, qd, qi, &qsz, pd, pi, &psz, bd, bi, bk, nb, key, true, lane));
                        nb = 0;
                    }
                    const uint32_t bm = __ballot_sync(kFull, fresh);
                    if (fresh) bi[nb + __popc(bm & lanemask_lt())] = id;
                    nb += __popc(bm);
                    __syncwarp();
                }
                nk = min(nk, link_flush(a, qrow, qd, qi, &qsz, pd, pi, &psz, bd, bi, bk, nb, key, true, lane));
            }
            k = nk <= k ? nk : k + 1;
        }
        // q's own k-NN neighbours that the search did not visit join the pool.
        nb = 0;
        for (uint32_t c0 = 0; c0 < a.K; c0 += 32) {
            const uint32_t c = c0 + lane;
            const uint32_t id = c < a.K ? __ldg(a.knn + (size_t) q * a.K + c) : 0u;
            const bool add = c < a.K && id < a.n && !(__ldcg(vis + (id >> 5)) & (1u << (id & 31)));
            const uint32_t bm = __ballot_sync(kFull, add);
            if (add) bi[nb + __popc(bm & lanemask_lt())] = id;
            nb += __popc(bm);
            __syncwarp();
            if (nb + 32 > kLinkBuf || c0 + 32 >= a.K) {
                if (nb) {
                    link_distances(a, qrow, bi, bd, bk, nb, key, lane);
                    key += nb;
                    warp_sort<ORDER_EFANNA>(bd, bi, bk, nb, nullptr, lane);
                    merge_into<ORDER_EFANNA>(pd, pi, &psz, a.C, bd, bi, bk, nb, nullptr, lane);
                }
                nb = 0;
            }
        }
        // sync_prune over the pool's first C entries.
        uint32_t start = (psz > 0 && pi[0] == q) ? 1u : 0u;
        uint32_t nres = 0;
        if (start < psz) {
            if (lane == 0) rid[0] = pi[start];
            nres = 1;
            __syncwarp();
            while (nres < a.R && ++start < psz) {
                const uint32_t p = pi[start];
                const float dp = pd[start];
                const float *prow = a.x + (size_t) p * a.d;
                bool occl = false;
                for (uint32_t t = lane; t < nres; t += 32) {
                    const uint32_t r = rid[t];
                    occl |= r == p || l2_ref(a.x + (size_t) r * a.d, prow, a.d) < dp;
                }
                if (!__any_sync(kFull, occl)) {
                    if (lane == 0) rid[nres] = p;
                    ++nres;
                }
                __syncwarp();
            }
        } else if (lane == 0) {
            atomicOr(a.error, LINK_ERR_SHORT_POOL);
        }
        __syncwarp();
        // The kept distances are d(q, r) as the pool holds them.
        for (uint32_t t = lane; t < nres; t += 32) {
            const uint32_t r = rid[t];
            a.cut_ids[(size_t) q * a.R + t] = r;
            a.cut_d[(size_t) q * a.R + t] = l2_ref(a.x + (size_t) r * a.d, qrow, a.d);
        }
        if (lane == 0) a.cut_n[q] = nres;
        // Clear the visited words this vertex set.
        if (dcount <= kLinkDirty) {
            for (uint32_t i = lane; i < dcount; i += 32) vis[dirty[i]] = 0u;
        } else {
            for (uint32_t i = lane; i < a.vis_words; i += 32) vis[i] = 0u;
        }
        __syncwarp();
    }
}

// ---- host side -------------------------------------------------------------

struct Nb {  // efanna2e Neighbor
    uint32_t id;
    float distance;
    bool flag;
    bool operator<(const Nb &o) const { return distance < o.distance; }
};
struct SNb {  // efanna2e SimpleNeighbor
    uint32_t id;
    float distance;
    bool operator<(const SNb &o) const { return distance < o.distance; }
};

// InsertIntoPool (include/efanna2e/neighbor.h:103-131).
uint32_t insert_into_pool(Nb *addr, uint32_t K, Nb nn) {
    uint32_t left = 0, right = K - 1;
    if (addr[left].distance > nn.distance) {
        memmove(&addr[left + 1], &addr[left], K * sizeof(Nb));
        addr[left] = nn;
        return left;
    }
    if (addr[right].distance < nn.distance) {
        addr[K] = nn;
        return K;
    }
    while (left < right - 1) {
        const uint32_t mid = (left + right) / 2;
        if (addr[mid].distance > nn.distance) right = mid;
        else left = mid;
    }
    while (left > 0) {
        if (addr[left].distance < nn.distance) break;
        if (addr[left].id == nn.id) return K + 1;
        left--;
    }
    if (addr[left].id == nn.id || addr[right].id == nn.id) return K + 1;
    memmove(&addr[right + 1], &addr[right], (K - right) * sizeof(Nb));
    addr[right] = nn;
    return right;
}

struct HostBuild {
    const float *x;
    uint32_t n, d, L;
    int32_t rs[40];  // glibc rand() state
    std::vector<std::vector<uint32_t>> graph;  // the graph searched (k-NN, later the NSG)
    uint32_t ep = 0;

    uint32_t rnd() { return (uint32_t) glibc_rand_next(rs); }

    // get_neighbors without a caller's flags (index_nsg.cpp:74-139): the
    // search result (retset, L + 1 entries) and the expansions' pool.
    void get_neighbors(const float *query, std::vector<Nb> &retset, std::vector<Nb> &fullset) {
        uint32_t Lp = L;
        retset.assign(Lp + 1, Nb{0, 0.f, false});
        std::vector<uint32_t> init_ids(Lp);
        std::vector<uint8_t> flags(n, 0);
        uint32_t l = 0;
        for (uint32_t i = 0; i < init_ids.size() && i < graph[ep].size(); i++) {
            init_ids[i] = graph[ep][i];
            flags[init_ids[i]] = 1;
            l++;
        }
        while (l < init_ids.size()) {
            const uint32_t id = rnd() % n;
            if (flags[id]) continue;
            init_ids[l] = id;
            l++;
            flags[id] = 1;
        }
        l = 0;
        for (uint32_t i = 0; i < init_ids.size(); i++) {
            const uint32_t id = init_ids[i];
            if (id >= n) continue;
            retset[i] = Nb{id, l2_ref(x + (size_t) d * id, query, d), true};
            l++;
        }
        std::sort(retset.begin(), retset.begin() + l);
        int k = 0;
        while (k < (int) l) {
            int nk = (int) l;
            if (retset[k].flag) {
                retset[k].flag = false;
                const uint32_t nn = retset[k].id;
                for (uint32_t m = 0; m < graph[nn].size(); ++m) {
                    const uint32_t id = graph[nn][m];
                    if (flags[id]) continue;
                    flags[id] = 1;
                    const float dist = l2_ref(query, x + (size_t) d * id, d);
                    Nb v{id, dist, true};
                    fullset.push_back(v);
                    if (dist >= retset[l - 1].distance) continue;
                    const int r = (int) insert_into_pool(retset.data(), l, v);
                    if (l + 1 < retset.size()) ++l;
                    if (r < nk) nk = r;
                }
            }
            if (nk <= k) k = nk;
            else ++k;
        }
    }
};

}  // namespace
}  // namespace panns

using namespace panns;

extern "C" int panns_efanna_build(int device, const float *base, uint32_t n, uint32_t d, const uint32_t *knn,
                                  uint32_t knn_k, uint32_t L, uint32_t R, uint32_t C, uint32_t rand_seed,
                                  panns_graph **out) {
    if (!base || !knn || !out) return set_error(PANNS_EINVAL, "panns_efanna_build: NULL argument");
    if (n < 2 || d == 0 || d % 8) return set_error(PANNS_EINVAL, "panns_efanna_build: need n >= 2 and d a multiple of 8");
    if (knn_k == 0 || L == 0 || L >= n || R == 0 || R > kLinkMaxR || C == 0)
        return set_error(PANNS_EINVAL, "panns_efanna_build: need knn_k > 0, 0 < L < n, 0 < R <= 256, C > 0");
    for (uint64_t i = 0; i < (uint64_t) n * knn_k; ++i)
        if (knn[i] >= n) return set_error(PANNS_EINVAL, "panns_efanna_build: a k-NN id >= n");
    const uint32_t Lc = (L + 31) / 32 * 32, Cc = (C + 31) / 32 * 32;
    const size_t smem = kLinkWarps * link_warp_bytes(Lc, Cc);
    if (smem > 200u * 1024u) return set_error(PANNS_EINVAL, "panns_efanna_build: L + C too large for shared memory");

    HostBuild hb;
    hb.x = base;
    hb.n = n;
    hb.d = d;
    hb.L = L;
    panns_rand_seed(hb.rs, rand_seed);
    hb.graph.resize(n);
    for (uint32_t i = 0; i < n; ++i) hb.graph[i].assign(knn + (size_t) i * knn_k, knn + (size_t) (i + 1) * knn_k);

    // 1. init_graph: the float mean, a random start, the best vertex found.
    std::vector<float> center(d, 0.f);
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t j = 0; j < d; j++) center[j] += base[(size_t) i * d + j];
    for (uint32_t j = 0; j < d; j++) center[j] /= (float) n;
    {
        std::vector<Nb> tmp, pool;
        hb.ep = hb.rnd() % n;
        hb.get_neighbors(center.data(), tmp, pool);
        hb.ep = tmp[0].id;
    }
    const uint32_t ep = hb.ep;

    // 2a. Every vertex's init list, in id order through one rand() stream.
    std::vector<uint32_t> init((size_t) n * L);
    {
        std::vector<uint8_t> mark(n, 0);
        const std::vector<uint32_t> &en = hb.graph[ep];
        const uint32_t pre = std::min<uint32_t>(L, (uint32_t) en.size());
        for (uint32_t i = 0; i < pre; ++i) mark[en[i]] = 1;
        for (uint32_t q = 0; q < n; ++q) {
            uint32_t *row = init.data() + (size_t) q * L;
            for (uint32_t i = 0; i < pre; ++i) row[i] = en[i];
            uint32_t l = pre;
            while (l < L) {
                const uint32_t id = hb.rnd() % n;
                if (mark[id]) continue;
                row[l++] = id;
                mark[id] = 1;
            }
            for (uint32_t i = pre; i < L; ++i) mark[row[i]] = 0;
        }
    }

    // 2b. get_neighbors + sync_prune of every vertex on the GPU.
    NCU(cudaSetDevice(device));
    cudaDeviceProp prop;
    NCU(cudaGetDeviceProperties(&prop, device));
    cudaStream_t s = nullptr;
    NCU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    NCU(cudaFuncSetAttribute(link_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int per_sm = 0;
    NCU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, link_kernel, kLinkWarps * 32, smem));
    if (per_sm < 1) return set_error(PANNS_EINVAL, "panns_efanna_build: L + C too large for shared memory");
    const uint32_t vis_words = (n + 31) / 32;
    uint32_t blocks = std::min<uint32_t>((uint32_t) per_sm * prop.multiProcessorCount, (n + kLinkWarps - 1) / kLinkWarps);
    while (blocks > 1 && (uint64_t) blocks * kLinkWarps * (vis_words + kLinkDirty) * 4 > (4ull << 30)) blocks /= 2;
    const uint32_t slots = blocks * kLinkWarps;
    NBuf<float> dx, dcd;
    NBuf<uint32_t> dknn, dinit, dvis, ddirty, dcid, dcn, dctl;
    NCU(dx.alloc((size_t) n * d));
    NCU(dknn.alloc((size_t) n * knn_k));
    NCU(dinit.alloc((size_t) n * L));
    NCU(dvis.alloc((size_t) slots * vis_words));
    NCU(ddirty.alloc((size_t) slots * kLinkDirty));
    NCU(dcid.alloc((size_t) n * R));
    NCU(dcd.alloc((size_t) n * R));
    NCU(dcn.alloc(n));
    NCU(dctl.alloc(2));
    NCU(cudaMemcpyAsync(dx.p, base, (size_t) n * d * 4, cudaMemcpyHostToDevice, s));
    NCU(cudaMemcpyAsync(dknn.p, knn, (size_t) n * knn_k * 4, cudaMemcpyHostToDevice, s));
    NCU(cudaMemcpyAsync(dinit.p, init.data(), init.size() * 4, cudaMemcpyHostToDevice, s));
    NCU(cudaMemsetAsync(dvis.p, 0, (size_t) slots * vis_words * 4, s));
    NCU(cudaMemsetAsync(dctl.p, 0, 8, s));
    LinkArgs la;
    memset(&la, 0, sizeof(la));
    la.x = dx.p;
    la.n = n;
    la.d = d;
    la.knn = dknn.p;
    la.K = knn_k;
    la.init = dinit.p;
    la.L = L;
    la.R = R;
    la.C = C;
    la.Lc = Lc;
    la.Cc = Cc;
    la.visited = dvis.p;
    la.vis_words = vis_words;
    la.dirty = ddirty.p;
    la.cut_ids = dcid.p;
    la.cut_d = dcd.p;
    la.cut_n = dcn.p;
    la.counter = dctl.p;
    la.error = dctl.p + 1;
    link_kernel<<<blocks, kLinkWarps * 32, smem, s>>>(la);
    NCU(cudaGetLastError());
    std::vector<uint32_t> cid((size_t) n * R), cn(n);
    std::vector<float> cd((size_t) n * R);
    uint32_t err = 0;
    NCU(cudaMemcpyAsync(cid.data(), dcid.p, cid.size() * 4, cudaMemcpyDeviceToHost, s));
    NCU(cudaMemcpyAsync(cd.data(), dcd.p, cd.size() * 4, cudaMemcpyDeviceToHost, s));
    NCU(cudaMemcpyAsync(cn.data(), dcn.p, n * 4ull, cudaMemcpyDeviceToHost, s));
    NCU(cudaMemcpyAsync(&err, dctl.p + 1, 4, cudaMemcpyDeviceToHost, s));
    NCU(cudaStreamSynchronize(s));
    if (err & LINK_ERR_BAD_ID) return set_error(PANNS_EDEVICE, "panns_efanna_build: an id >= n on the GPU");
    if (err & LINK_ERR_SHORT_POOL) return set_error(PANNS_EINVAL, "panns_efanna_build: a vertex found no neighbour");

    // The cut graph: per vertex R slots, a distance of -1 ends a list.
    std::vector<SNb> cut((size_t) n * R);
    for (uint32_t q = 0; q < n; ++q) {
        SNb *p = cut.data() + (size_t) q * R;
        for (uint32_t t = 0; t < cn[q]; ++t) p[t] = SNb{cid[(size_t) q * R + t], cd[(size_t) q * R + t]};
        if (cn[q] < R) p[cn[q]].distance = -1;
    }

    // 3. InterInsert, vertex by vertex (index_nsg.cpp:278-354).
    for (uint32_t nn = 0; nn < n; ++nn) {
        SNb *src = cut.data() + (size_t) nn * R;
        for (uint32_t i = 0; i < R; i++) {
            if (src[i].distance == -1) break;
            const SNb sn{nn, src[i].distance};
            const uint32_t des = src[i].id;
            SNb *dp = cut.data() + (size_t) des * R;
            std::vector<SNb> temp;
            bool dup = false;
            for (uint32_t j = 0; j < R; j++) {
                if (dp[j].distance == -1) break;
                if (nn == dp[j].id) {
                    dup = true;
                    break;
                }
                temp.push_back(dp[j]);
            }
            if (dup) continue;
            temp.push_back(sn);
            if (temp.size() > R) {
                std::vector<SNb> result;
                uint32_t st = 0;
                std::sort(temp.begin(), temp.end());
                result.push_back(temp[st]);
                while (result.size() < R && (++st) < temp.size()) {
                    const SNb &p = temp[st];
                    bool occl = false;
                    for (uint32_t t = 0; t < result.size(); t++) {
                        if (p.id == result[t].id) {
                            occl = true;
                            break;
                        }
                        const float djk = l2_ref(base + (size_t) d * result[t].id, base + (size_t) d * p.id, d);
                        if (djk < p.distance) {
                            occl = true;
                            break;
                        }
                    }
                    if (!occl) result.push_back(p);
                }
                for (uint32_t t = 0; t < result.size(); t++) dp[t] = result[t];
            } else {
                for (uint32_t t = 0; t < R; t++) {
                    if (dp[t].distance == -1) {
                        dp[t] = sn;
                        if (t + 1 < R) dp[t + 1].distance = -1;
                        break;
                    }
                }
            }
        }
    }

    // 4. The lists become the graph (index_nsg.cpp:419-434).
    for (uint32_t i = 0; i < n; i++) {
        const SNb *p = cut.data() + (size_t) i * R;
        uint32_t size = 0;
        for (uint32_t j = 0; j < R; j++) {
            if (p[j].distance == -1) break;
            size = j;
        }
        size++;
        hb.graph[i].resize(size);
        for (uint32_t j = 0; j < size; j++) hb.graph[i][j] = p[j].id;
    }

    // 5. tree_grow: DFS (:638-668) and findroot (:670-700).
    uint32_t width = R;
    {
        std::vector<uint8_t> flag(n, 0);
        uint32_t root = ep, cnt = 0;
        while (cnt < n) {
            {
                uint32_t tmp = root;
                std::stack<uint32_t> stk;
                stk.push(root);
                if (!flag[root]) cnt++;
                flag[root] = 1;
                while (!stk.empty()) {
                    uint32_t next = n + 1;
                    for (uint32_t i = 0; i < hb.graph[tmp].size(); i++) {
                        if (!flag[hb.graph[tmp][i]]) {
                            next = hb.graph[tmp][i];
                            break;
                        }
                    }
                    if (next == n + 1) {
                        stk.pop();
                        if (stk.empty()) break;
                        tmp = stk.top();
                        continue;
                    }
                    tmp = next;
                    flag[tmp] = 1;
                    stk.push(tmp);
                    cnt++;
                }
            }
            if (cnt >= n) break;
            uint32_t id = n;
            for (uint32_t i = 0; i < n; i++)
                if (!flag[i]) {
                    id = i;
                    break;
                }
            if (id == n) break;
            std::vector<Nb> tmp, pool;
            hb.get_neighbors(base + (size_t) d * id, tmp, pool);
            std::sort(pool.begin(), pool.end());
            bool found = false;
            for (uint32_t i = 0; i < pool.size(); i++)
                if (flag[pool[i].id]) {
                    root = pool[i].id;
                    found = true;
                    break;
                }
            if (!found) {
                for (;;) {
                    const uint32_t rid = hb.rnd() % n;
                    if (flag[rid]) {
                        root = rid;
                        break;
                    }
                }
            }
            hb.graph[root].push_back(id);
        }
        for (uint32_t i = 0; i < n; ++i) width = std::max<uint32_t>(width, (uint32_t) hb.graph[i].size());
    }

    std::unique_ptr<panns_graph> g(new panns_graph());
    g->n = n;
    g->k = knn_k;
    g->entry = ep;
    g->width = width;
    g->knn.assign(knn, knn + (size_t) n * knn_k);
    g->off.assign(n + 1, 0);
    for (uint32_t a = 0; a < n; ++a) g->off[a + 1] = g->off[a] + hb.graph[a].size();
    g->nbrs.resize(g->off[n]);
    for (uint32_t a = 0; a < n; ++a) std::copy(hb.graph[a].begin(), hb.graph[a].end(), g->nbrs.begin() + g->off[a]);
    *out = g.release();
    return PANNS_OK;
}
