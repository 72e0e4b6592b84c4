/* CPU oracle for the PANNS search path — TEST INFRASTRUCTURE ONLY.
 * See panns_oracle.h. Each function cites the reference code it restates
 * (paths relative to the parallel_ANNS project root).
 */
#include "panns_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_fused = 1;
void po_set_fused(int fused) { g_fused = fused ? 1 : 0; }

/* ---------------------------------------------------------------------------
 * Distances. core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:294-391
 * (compute_norm, compute_distance_with_norm) and
 * core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.cpp:525-563
 * (compute_distance); include/efanna2e/distance.h:24-60, 132-165, 231-324.
 * Eight lane accumulators; lane j sums elements j, j+8, j+16, ... in that
 * order, except that when d % 16 == 8 the last 8 elements are added first;
 * then lane 0 + lane 1 + ... + lane 7, left to right. The norm trick returns
 * -2 * dot + norm.
 * ------------------------------------------------------------------------- */
static inline float lane_sum(const float acc[8]) {
    float r = acc[0];
    for (int j = 1; j < 8; ++j) r = r + acc[j];
    return r;
}

float po_norm(const float *v, int d, int fused) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int DR = d % 16, DD = d - DR;
    if (DR) {
        for (int j = 0; j < 8; ++j) {
            float a = v[DD + j];
            acc[j] = fused ? fmaf(a, a, acc[j]) : acc[j] + a * a;
        }
    }
    for (int i = 0; i < DD; i += 8) {
        for (int j = 0; j < 8; ++j) {
            float a = v[i + j];
            acc[j] = fused ? fmaf(a, a, acc[j]) : acc[j] + a * a;
        }
    }
    return lane_sum(acc);
}

float po_distance(const float *v, const float *q, float norm, int d, int kind, int fused) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int DR = d % 16, DD = d - DR;
    if (kind == PO_DIST_IP_NORM) {
        if (DR) {
            for (int j = 0; j < 8; ++j)
                acc[j] = fused ? fmaf(v[DD + j], q[DD + j], acc[j]) : acc[j] + v[DD + j] * q[DD + j];
        }
        for (int i = 0; i < DD; i += 8)
            for (int j = 0; j < 8; ++j)
                acc[j] = fused ? fmaf(v[i + j], q[i + j], acc[j]) : acc[j] + v[i + j] * q[i + j];
        float dot = lane_sum(acc);
        return -2.0f * dot + norm;
    } else {
        if (DR) {
            for (int j = 0; j < 8; ++j) {
                float t = v[DD + j] - q[DD + j];
                acc[j] = fused ? fmaf(t, t, acc[j]) : acc[j] + t * t;
            }
        }
        for (int i = 0; i < DD; i += 8)
            for (int j = 0; j < 8; ++j) {
                float t = v[i + j] - q[i + j];
                acc[j] = fused ? fmaf(t, t, acc[j]) : acc[j] + t * t;
            }
        return lane_sum(acc);
    }
}

static inline float vdist(const float *data, const float *norms, uint32_t d, uint32_t id,
                          const float *q, int kind) {
    return po_distance(data + (size_t) id * d, q, norms ? norms[id] : 0.0f, (int) d, kind, g_fused);
}

/* ---------------------------------------------------------------------------
 * Init ids. prepare_init_ids:
 * core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:238-291.
 * ------------------------------------------------------------------------- */
int po_prepare_init_ids(const uint64_t *offsets, const uint32_t *nbrs, uint32_t n,
                        uint32_t entry, uint32_t L, uint32_t *out) {
    if (L > n) return -1;
    uint8_t *sel = (uint8_t *) calloc(n, 1);
    if (!sel) return -2;
    uint32_t end = 0;
    for (uint64_t e = offsets[entry]; e < offsets[entry + 1] && end < L; ++e) {
        uint32_t v = nbrs[e];
        if (sel[v]) continue;
        sel[v] = 1;
        out[end++] = v;
    }
    uint32_t t = entry + 1;
    while (end < L) {
        if (t == n) t = 0;
        uint32_t v = t++;
        if (sel[v]) continue;
        sel[v] = 1;
        out[end++] = v;
    }
    free(sel);
    return 0;
}

/* glibc's rand(): the TYPE_3 additive feedback generator (degree 31,
 * separation 3) seeded by a Park-Miller (16807, 2^31-1) sequence, with the
 * first 310 outputs discarded; each output is the 32-bit sum shifted right by
 * one. Used by include/efanna2e/index_nsg.cpp:468-474, 541-547 through the
 * never-seeded process-wide rand() (seed 1). */
void po_srand(po_rand_state *s, uint32_t seed) {
    int32_t *r = s->tbl;
    if (seed == 0) seed = 1;
    r[0] = (int32_t) seed;
    for (int i = 1; i < 31; ++i) {
        int64_t hi = r[i - 1] / 127773, lo = r[i - 1] % 127773;
        int64_t w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        r[i] = (int32_t) w;
    }
    /* front pointer starts 3 ahead of the rear pointer; discard 310 outputs */
    s->fptr = &r[3];
    s->rptr = &r[0];
    for (int i = 0; i < 310; ++i) po_rand(s);
}

uint32_t po_rand_state_size(void) { return (uint32_t) sizeof(po_rand_state); }

int32_t po_rand(po_rand_state *s) {
    int32_t *r = s->tbl;
    uint32_t val = (uint32_t) *s->fptr + (uint32_t) *s->rptr;
    *s->fptr = (int32_t) val;
    int32_t result = (int32_t) (val >> 1);
    ++s->fptr;
    if (s->fptr >= &r[31]) {
        s->fptr = r;
        ++s->rptr;
    } else {
        ++s->rptr;
        if (s->rptr >= &r[31]) s->rptr = r;
    }
    return result;
}

/* efanna2e init: include/efanna2e/index_nsg.cpp:458-474 (Search) and
 * :530-547 (SearchWithOptGraph). */
int po_efanna_init_ids(const uint64_t *offsets, const uint32_t *nbrs, uint32_t n,
                       uint32_t entry, uint32_t L, uint32_t nq, po_rand_state *s,
                       uint32_t *out) {
    if (L > n) return -1;
    uint8_t *flags = (uint8_t *) calloc(n, 1);
    if (!flags) return -2;
    const uint64_t deg = offsets[entry + 1] - offsets[entry];
    for (uint32_t q = 0; q < nq; ++q) {
        uint32_t *ids = out + (size_t) q * L;
        uint32_t t = 0;
        for (; t < L && t < deg; ++t) {
            ids[t] = nbrs[offsets[entry] + t];
            flags[ids[t]] = 1;
        }
        while (t < L) {
            uint32_t id = (uint32_t) po_rand(s) % n;
            if (flags[id]) continue;
            flags[id] = 1;
            ids[t++] = id;
        }
        for (uint32_t i = 0; i < L; ++i) flags[ids[i]] = 0;
    }
    free(flags);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Queue of Candidate{id, dist, checked}, total order (dist, id):
 * include/Candidate.h:11-28.
 * ------------------------------------------------------------------------- */
typedef struct { uint32_t id; float dist; uint8_t checked; } cand_t;

static inline int cand_less(const cand_t *a, const cand_t *b) {
    if (a->dist != b->dist) return a->dist < b->dist;
    return a->id < b->id;
}

static uint32_t lower_bound(const cand_t *q, uint32_t size, const cand_t *c) {
    uint32_t lo = 0, hi = size;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (cand_less(&q[mid], c)) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* add_into_queue: core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:396-439 */
static uint32_t add_into_queue(cand_t *q, uint32_t *size, uint32_t cap, cand_t c) {
    if (*size == 0) {
        q[(*size)++] = c;
        return 0;
    }
    uint32_t end = *size;
    uint32_t pos = lower_bound(q, end, &c);
    if (pos != end) {
        if (q[pos].id == c.id) return cap;
        if (*size >= cap) { --(*size); --end; }
    } else {
        if (*size < cap) {
            q[pos] = c;
            ++(*size);
            return *size - 1;
        }
        return cap;
    }
    memmove(q + pos + 1, q + pos, (size_t) (end - pos) * sizeof(cand_t));
    q[pos] = c;
    ++(*size);
    return pos;
}

/* insert_one_element_at: :460-473 (fixed size; the last element falls off) */
static void insert_one_at(cand_t *q, uint32_t idx, uint32_t size, cand_t c) {
    memmove(q + idx + 1, q + idx, (size_t) (size - idx - 1) * sizeof(cand_t));
    q[idx] = c;
}

/* merge_two_queues_into_1st_queue_seq_fixed: :479-550 */
static uint32_t merge_fixed(cand_t *q1, uint32_t size1, const cand_t *q2, uint32_t size2) {
    uint32_t pos = lower_bound(q1, size1, &q2[0]);
    if (pos == size1) return pos;
    if (pos == size1 - 1) {
        q1[pos] = q2[0];
        return pos;
    }
    if (q2[0].id != q1[pos].id) {
        insert_one_at(q1, pos, size1, q2[0]);
    } else if (!q2[0].checked && q1[pos].checked) {
        q1[pos].checked = 0;
    }
    if (size2 == 1) return pos;
    uint32_t i1 = pos + 1, i2 = 1;
    for (uint32_t ins = pos + 1; ins < size1; ++ins) {
        if (i1 >= size1 || i2 >= size2) break;
        if (cand_less(&q1[i1], &q2[i2])) {
            ++i1;
        } else if (cand_less(&q2[i2], &q1[i1])) {
            insert_one_at(q1, ins, size1, q2[i2++]);
            ++i1;
        } else {
            if (!q2[i2].checked && q1[i1].checked) q1[i1].checked = 0;
            ++i2;
            ++i1;
        }
    }
    return pos;
}

static int cmp_cand(const void *a, const void *b) {
    const cand_t *x = (const cand_t *) a, *y = (const cand_t *) b;
    if (cand_less(x, y)) return -1;
    if (cand_less(y, x)) return 1;
    return 0;
}

typedef struct {
    const float *data, *norms, *q;
    uint32_t d, n;
    int kind;
    const uint64_t *off;
    const uint32_t *nbrs;
    uint64_t *visited;
    uint64_t ndist;
} ctx_t;

static inline int test_and_set(uint64_t *bits, uint32_t v) {
    uint64_t m = (uint64_t) 1 << (v & 63);
    if (bits[v >> 6] & m) return 1;
    bits[v >> 6] |= m;
    return 0;
}

/* initialize_set_L_para: :897-935 (visited marks, L distances, sort by (dist, id)) */
static void init_queue(ctx_t *c, const uint32_t *init_ids, uint32_t L, cand_t *q) {
    for (uint32_t i = 0; i < L; ++i) test_and_set(c->visited, init_ids[i]);
    for (uint32_t i = 0; i < L; ++i) {
        q[i].id = init_ids[i];
        q[i].dist = vdist(c->data, c->norms, c->d, init_ids[i], c->q, c->kind);
        q[i].checked = 0;
    }
    c->ndist += L;
    qsort(q, L, sizeof(cand_t), cmp_cand);
}

/* expand_one_candidate: :824-895 (small graph), LG :984-1053. `bound_q` is
 * the queue whose last element is the live bound (the master queue). */
static uint32_t expand(ctx_t *c, uint32_t cand, const cand_t *bound_q, uint32_t bound_idx,
                       cand_t *q, uint32_t *size, uint32_t cap) {
    uint32_t nk = cap;
    for (uint64_t e = c->off[cand]; e < c->off[cand + 1]; ++e) {
        uint32_t nb = c->nbrs[e];
        if (test_and_set(c->visited, nb)) continue;
        float dist = vdist(c->data, c->norms, c->d, nb, c->q, c->kind);
        ++c->ndist;
        if (dist > bound_q[bound_idx].dist) continue;
        cand_t cc = {nb, dist, 0};
        uint32_t r = add_into_queue(q, size, cap, cc);
        if (r < nk) nk = r;
    }
    return nk;
}

static int prep_ctx(ctx_t *c, const float *data, const float *norms, uint32_t n, uint32_t d,
                    const uint64_t *off, const uint32_t *nbrs, int kind) {
    c->data = data; c->norms = norms; c->n = n; c->d = d; c->kind = kind;
    c->off = off; c->nbrs = nbrs; c->ndist = 0;
    c->visited = (uint64_t *) calloc((n + 63) / 64, sizeof(uint64_t));
    return c->visited ? 0 : -2;
}

/* Top-M at T = 1: core/Searching.202011241533.top_m_pure.cpp:1881-1965
 * (para_search_with_top_m_pure, 1 == num_threads_ branch), with
 * pick_top_m_unchecked :1038-1064 and the update k = nk <= last_k ? nk : last_k + 1. */
static void search_top_m_one(ctx_t *c, const uint32_t *init_ids, uint32_t K, uint32_t L,
                             uint32_t M, cand_t *q, uint32_t *top, uint32_t *out) {
    init_queue(c, init_ids, L, q);
    uint32_t size = L, k = 0;
    for (;;) {
        uint32_t last_k = L, cnt = 0;
        for (uint32_t i = k; i < size && cnt < M; ++i) {
            if (q[i].checked) continue;
            last_k = i;
            q[i].checked = 1;
            top[cnt++] = q[i].id;
        }
        if (!cnt) break;
        uint32_t nk = L;
        for (uint32_t j = 0; j < cnt; ++j) {
            uint32_t r = expand(c, top[j], q, L - 1, q, &size, L);
            if (r < nk) nk = r;
        }
        k = nk <= last_k ? nk : last_k + 1;
    }
    for (uint32_t i = 0; i < K; ++i) out[i] = q[i].id;
}

int po_search_top_m(const float *data, const float *norms, uint32_t n, uint32_t d,
                    const uint64_t *offsets, const uint32_t *nbrs,
                    const float *queries, uint32_t nq, const uint32_t *init_ids,
                    int init_per_query, uint32_t K, uint32_t L, uint32_t M, int kind,
                    uint32_t *out_ids, uint64_t *out_ndist, int threads) {
    if (K > L || L > n || M == 0 || d % 8) return -1;
    uint64_t total = 0;
    int err = 0;
#pragma omp parallel num_threads(threads > 0 ? threads : 1) reduction(+ : total) reduction(| : err)
    {
        ctx_t c;
        cand_t *q = (cand_t *) malloc((size_t) L * sizeof(cand_t));
        uint32_t *top = (uint32_t *) malloc((size_t) M * sizeof(uint32_t));
        if (prep_ctx(&c, data, norms, n, d, offsets, nbrs, kind) || !q || !top) {
            err |= 1;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (uint32_t i = 0; i < nq; ++i) {
                c.q = queries + (size_t) i * d;
                const uint32_t *ii = init_ids + (init_per_query ? (size_t) i * L : 0);
                search_top_m_one(&c, ii, K, L, M, q, top, out_ids + (size_t) i * K);
                memset(c.visited, 0, ((n + 63) / 64) * sizeof(uint64_t));
            }
        }
        total += c.ndist;
        free(c.visited);
        free(q);
        free(top);
    }
    if (out_ndist) *out_ndist = total;
    return err ? -2 : 0;
}

/* Top-M search started from a per-query init list of any length <= its own
 * queue length L_q (the learned-entry search of panns_b200; no reference
 * counterpart). Repeated init ids enter once; while the queue holds fewer
 * than L_q candidates nothing is rejected, afterwards a neighbour is rejected
 * when dist > the L_q-th distance, as in expand(). Otherwise the step of
 * search_top_m_one. */
static void search_top_m_list_one(ctx_t *c, const uint32_t *init, uint32_t n_init, uint32_t K,
                                  uint32_t L, uint32_t M, cand_t *q, uint32_t *top, uint32_t *out) {
    uint32_t size = 0;
    for (uint32_t i = 0; i < n_init && size < L; ++i) {
        if (test_and_set(c->visited, init[i])) continue;
        q[size].id = init[i];
        q[size].dist = vdist(c->data, c->norms, c->d, init[i], c->q, c->kind);
        q[size].checked = 0;
        ++size;
        ++c->ndist;
    }
    qsort(q, size, sizeof(cand_t), cmp_cand);
    uint32_t k = 0;
    for (;;) {
        uint32_t last_k = L, cnt = 0;
        for (uint32_t i = k; i < size && cnt < M; ++i) {
            if (q[i].checked) continue;
            last_k = i;
            q[i].checked = 1;
            top[cnt++] = q[i].id;
        }
        if (!cnt) break;
        uint32_t nk = L;
        for (uint32_t j = 0; j < cnt; ++j) {
            const uint32_t cand = top[j];
            for (uint64_t e = c->off[cand]; e < c->off[cand + 1]; ++e) {
                const uint32_t nb = c->nbrs[e];
                if (test_and_set(c->visited, nb)) continue;
                const float dist = vdist(c->data, c->norms, c->d, nb, c->q, c->kind);
                ++c->ndist;
                if (size >= L && dist > q[L - 1].dist) continue;
                cand_t cc = {nb, dist, 0};
                const uint32_t r = add_into_queue(q, &size, L, cc);
                if (r < nk) nk = r;
            }
        }
        k = nk <= last_k ? nk : last_k + 1;
    }
    for (uint32_t i = 0; i < K; ++i) out[i] = i < size ? q[i].id : 0xffffffffu;
}

int po_search_top_m_lists(const float *data, const float *norms, uint32_t n, uint32_t d,
                          const uint64_t *offsets, const uint32_t *nbrs, const float *queries,
                          uint32_t nq, const uint32_t *init_lists, uint32_t list_stride,
                          const uint32_t *init_counts, const uint32_t *Lq, uint32_t K, uint32_t M,
                          int kind, uint32_t *out_ids, uint64_t *out_ndist, int threads) {
    if (M == 0 || d % 8) return -1;
    uint32_t Lmax = 0;
    for (uint32_t i = 0; i < nq; ++i) {
        if (Lq[i] < K || Lq[i] > n || init_counts[i] > list_stride) return -1;
        if (Lq[i] > Lmax) Lmax = Lq[i];
    }
    uint64_t total = 0;
    int err = 0;
#pragma omp parallel num_threads(threads > 0 ? threads : 1) reduction(+ : total) reduction(| : err)
    {
        ctx_t c;
        cand_t *q = (cand_t *) malloc((size_t) (Lmax + 1) * sizeof(cand_t));
        uint32_t *top = (uint32_t *) malloc((size_t) M * sizeof(uint32_t));
        if (prep_ctx(&c, data, norms, n, d, offsets, nbrs, kind) || !q || !top) {
            err |= 1;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (uint32_t i = 0; i < nq; ++i) {
                c.q = queries + (size_t) i * d;
                search_top_m_list_one(&c, init_lists + (size_t) i * list_stride, init_counts[i], K, Lq[i],
                                      M, q, top, out_ids + (size_t) i * K);
                memset(c.visited, 0, ((n + 63) / 64) * sizeof(uint64_t));
            }
        }
        total += c.ndist;
        free(c.visited);
        free(q);
        free(top);
    }
    if (out_ndist) *out_ndist = total;
    return err ? -2 : 0;
}

/* PSS_v5: core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:1218-1515
 * (LG twin :1376-1726 adds a per-stage snapshot bound that is never tighter
 * than the live master bound, so it filters nothing extra). The parallel
 * expand phase (:1403-1456) is serialised round-robin: in each round every
 * worker, in id order, then the master, advances its own loop by one
 * expansion. Pick: pick_top_m_to_workers :756-786; merge:
 * merge_all_queues_to_master :642-681. */
static void search_pss_one(ctx_t *c, const uint32_t *init_ids, uint32_t K, uint32_t L,
                           uint32_t L_local, uint32_t X, uint32_t T, cand_t *set_L,
                           uint32_t *sizes, uint32_t *kuc, uint32_t *iters, uint32_t *out) {
    const uint32_t mstart = (T - 1) * L_local;
    cand_t *master = set_L + mstart;
    init_queue(c, init_ids, L, master);
    for (uint32_t w = 0; w < T; ++w) sizes[w] = 0;
    sizes[T - 1] = L;
    uint32_t k_master = 0;
    int done = 0;
    /* one sequential expansion (seq_iter_bound = 1) */
    {
        cand_t *cd = &master[k_master];
        uint32_t r;
        if (!cd->checked) {
            cd->checked = 1;
            r = expand(c, cd->id, master, L - 1, master, &sizes[T - 1], L);
        } else {
            r = L;
        }
        k_master = r <= k_master ? r : k_master + 1;
        (void) done;
    }
    for (;;) {
        /* pick_top_m_to_workers */
        uint32_t count = 0, dest = 0;
        for (uint32_t ci = k_master; ci < sizes[T - 1]; ++ci) {
            if (master[ci].checked) continue;
            ++count;
            if (T - 1 != dest) {
                set_L[dest * L_local + sizes[dest]++] = master[ci];
                master[ci].checked = 1;
                if (sizes[dest] == L_local) break;
                ++dest;
            } else {
                dest = 0;
            }
        }
        if (!count) break;
        for (uint32_t w = 0; w < T; ++w) {
            kuc[w] = (w == T - 1) ? k_master : 0;
            iters[w] = 0;
        }
        for (;;) {
            int any = 0;
            for (uint32_t w = 0; w < T; ++w) {
                cand_t *lq = (w == T - 1) ? master : set_L + (size_t) w * L_local;
                const uint32_t cap = (w == T - 1) ? L : L_local;
                while (iters[w] < X && kuc[w] < sizes[w]) {
                    cand_t *cd = &lq[kuc[w]];
                    if (!cd->checked) {
                        cd->checked = 1;
                        ++iters[w];
                        uint32_t r = expand(c, cd->id, master, L - 1, lq, &sizes[w], cap);
                        kuc[w] = r <= kuc[w] ? r : kuc[w] + 1;
                        any = 1;
                        break;
                    }
                    ++kuc[w];
                }
            }
            if (!any) break;
        }
        k_master = kuc[T - 1];
        uint32_t nk = L;
        for (uint32_t w = 0; w + 1 < T; ++w) {
            if (!sizes[w]) continue;
            uint32_t r = merge_fixed(master, L, set_L + (size_t) w * L_local, sizes[w]);
            if (r < nk) nk = r;
            sizes[w] = 0;
        }
        if (nk <= k_master) k_master = nk;
    }
    for (uint32_t i = 0; i < K; ++i) out[i] = master[i].id;
}

int po_search_pss(const float *data, const float *norms, uint32_t n, uint32_t d,
                  const uint64_t *offsets, const uint32_t *nbrs,
                  const float *queries, uint32_t nq, const uint32_t *init_ids,
                  uint32_t K, uint32_t L, uint32_t L_local, uint32_t X, uint32_t T,
                  int kind, uint32_t *out_ids, uint64_t *out_ndist, int threads) {
    if (K > L || L > n || T == 0 || X == 0 || L_local == 0 || d % 8) return -1;
    uint64_t total = 0;
    int err = 0;
#pragma omp parallel num_threads(threads > 0 ? threads : 1) reduction(+ : total) reduction(| : err)
    {
        ctx_t c;
        cand_t *set_L = (cand_t *) malloc(((size_t) (T - 1) * L_local + L) * sizeof(cand_t));
        uint32_t *sizes = (uint32_t *) malloc(T * sizeof(uint32_t) * 3);
        if (prep_ctx(&c, data, norms, n, d, offsets, nbrs, kind) || !set_L || !sizes) {
            err |= 1;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (uint32_t i = 0; i < nq; ++i) {
                c.q = queries + (size_t) i * d;
                search_pss_one(&c, init_ids, K, L, L_local, X, T, set_L, sizes, sizes + T,
                               sizes + 2 * T, out_ids + (size_t) i * K);
                memset(c.visited, 0, ((n + 63) / 64) * sizeof(uint64_t));
            }
        }
        total += c.ndist;
        free(c.visited);
        free(set_L);
        free(sizes);
    }
    if (out_ndist) *out_ndist = total;
    return err ? -2 : 0;
}

/* efanna2e: include/efanna2e/index_nsg.cpp:452-518 (Search) and :520-611
 * (SearchWithOptGraph); InsertIntoPool include/efanna2e/neighbor.h:103-131.
 * Order is by distance only; a new element goes after equal distances; a
 * neighbour is rejected when dist >= the L-th distance. The initial sort of
 * equal distances keeps init-id order (the reference's std::sort leaves that
 * order unspecified). */
typedef struct { uint32_t id; float dist; uint8_t flag; uint32_t seq; } ecand_t;

static int cmp_ecand(const void *a, const void *b) {
    const ecand_t *x = (const ecand_t *) a, *y = (const ecand_t *) b;
    if (x->dist < y->dist) return -1;
    if (x->dist > y->dist) return 1;
    return x->seq < y->seq ? -1 : (x->seq > y->seq);
}

static uint32_t insert_into_pool(ecand_t *addr, uint32_t K, ecand_t nn) {
    uint32_t left = 0, right = K - 1;
    if (addr[left].dist > nn.dist) {
        memmove(&addr[left + 1], &addr[left], (size_t) K * sizeof(ecand_t));
        addr[left] = nn;
        return left;
    }
    if (addr[right].dist < nn.dist) {
        addr[K] = nn;
        return K;
    }
    while (left < right - 1) {
        uint32_t mid = (left + right) / 2;
        if (addr[mid].dist > nn.dist) right = mid; else left = mid;
    }
    while (left > 0) {
        if (addr[left].dist < nn.dist) break;
        if (addr[left].id == nn.id) return K + 1;
        left--;
    }
    if (addr[left].id == nn.id || addr[right].id == nn.id) return K + 1;
    memmove(&addr[right + 1], &addr[right], (size_t) (K - right) * sizeof(ecand_t));
    addr[right] = nn;
    return right;
}

int po_search_efanna(const float *data, const float *norms, uint32_t n, uint32_t d,
                     const uint64_t *offsets, const uint32_t *nbrs,
                     const float *queries, uint32_t nq, const uint32_t *init_ids,
                     uint32_t K, uint32_t L, int kind,
                     uint32_t *out_ids, uint64_t *out_ndist, int threads) {
    if (K > L || L > n || d % 8 || L < 2) return -1;
    uint64_t total = 0;
    int err = 0;
#pragma omp parallel num_threads(threads > 0 ? threads : 1) reduction(+ : total) reduction(| : err)
    {
        ctx_t c;
        ecand_t *ret = (ecand_t *) malloc(((size_t) L + 1) * sizeof(ecand_t));
        if (prep_ctx(&c, data, norms, n, d, offsets, nbrs, kind) || !ret) {
            err |= 1;
        } else {
#pragma omp for schedule(dynamic, 4)
            for (uint32_t qi = 0; qi < nq; ++qi) {
                c.q = queries + (size_t) qi * d;
                const uint32_t *ii = init_ids + (size_t) qi * L;
                for (uint32_t i = 0; i < L; ++i) test_and_set(c.visited, ii[i]);
                for (uint32_t i = 0; i < L; ++i) {
                    ret[i].id = ii[i];
                    ret[i].dist = vdist(data, norms, d, ii[i], c.q, kind);
                    ret[i].flag = 1;
                    ret[i].seq = i;
                }
                c.ndist += L;
                qsort(ret, L, sizeof(ecand_t), cmp_ecand);
                uint32_t k = 0;
                while (k < L) {
                    uint32_t nk = L;
                    if (ret[k].flag) {
                        ret[k].flag = 0;
                        uint32_t v = ret[k].id;
                        for (uint64_t e = offsets[v]; e < offsets[v + 1]; ++e) {
                            uint32_t id = nbrs[e];
                            if (test_and_set(c.visited, id)) continue;
                            float dist = vdist(data, norms, d, id, c.q, kind);
                            ++c.ndist;
                            if (dist >= ret[L - 1].dist) continue;
                            ecand_t nn = {id, dist, 1, 0};
                            uint32_t r = insert_into_pool(ret, L, nn);
                            if (r < nk) nk = r;
                        }
                    }
                    if (nk <= k) k = nk; else ++k;
                }
                for (uint32_t i = 0; i < K; ++i) out_ids[(size_t) qi * K + i] = ret[i].id;
                memset(c.visited, 0, ((n + 63) / 64) * sizeof(uint64_t));
            }
        }
        total += c.ndist;
        free(c.visited);
        free(ret);
    }
    if (out_ndist) *out_ndist = total;
    return err ? -2 : 0;
}

/* ---------------------------------------------------------------------------
 * Ground truth: brute force in float64, top-k by (distance, id); the role of
 * tools/save_true_nearest_neighbors.cpp:16-35 (which scans in float32).
 * ------------------------------------------------------------------------- */
int po_ground_truth_fp64(const float *data, uint32_t n, uint32_t d,
                         const float *queries, uint32_t nq, uint32_t k,
                         uint32_t *out_ids, double *out_dist, int threads) {
    if (k > n) return -1;
    int err = 0;
#pragma omp parallel num_threads(threads > 0 ? threads : 1) reduction(| : err)
    {
        double *bd = (double *) malloc((size_t) (k + 1) * sizeof(double));
        uint32_t *bi = (uint32_t *) malloc((size_t) (k + 1) * sizeof(uint32_t));
        if (!bd || !bi) err |= 1;
        else {
#pragma omp for schedule(dynamic, 1)
            for (uint32_t qi = 0; qi < nq; ++qi) {
                const float *q = queries + (size_t) qi * d;
                uint32_t cnt = 0;
                for (uint32_t v = 0; v < n; ++v) {
                    const float *x = data + (size_t) v * d;
                    double s = 0;
                    for (uint32_t j = 0; j < d; ++j) {
                        double t = (double) x[j] - (double) q[j];
                        s += t * t;
                    }
                    if (cnt == k && !(s < bd[k - 1])) continue; /* ties keep the lower id */
                    uint32_t pos = cnt < k ? cnt : k - 1;
                    while (pos > 0 && bd[pos - 1] > s) {
                        bd[pos] = bd[pos - 1];
                        bi[pos] = bi[pos - 1];
                        --pos;
                    }
                    bd[pos] = s;
                    bi[pos] = v;
                    if (cnt < k) ++cnt;
                }
                memcpy(out_ids + (size_t) qi * k, bi, k * sizeof(uint32_t));
                if (out_dist) memcpy(out_dist + (size_t) qi * k, bd, k * sizeof(double));
            }
        }
        free(bd);
        free(bi);
    }
    return err ? -2 : 0;
}

/* ---- graph construction (restates parallel_anns_b200/csrc/graph_build.cu) ----
 * No PANNS counterpart: the graphs the benchmark workloads describe
 * (exact k-NN, MRNG prune, medoid, reachability repair); the pruning rule is
 * efanna2e's sync_prune (include/efanna2e/index_nsg.cpp:233-283) on exact k-NN
 * lists, the repair plays the part of its tree_grow (:638-718). */
static double po_d64(const float *a, const float *b, uint32_t d) {
    double acc = 0.0;
    for (uint32_t j = 0; j < d; ++j) {
        const double t = (double) a[j] - (double) b[j];
        acc = fma(t, t, acc);
    }
    return acc;
}

typedef struct { double d; uint32_t id; } po_dk;

static int po_dk_less(const po_dk *a, const po_dk *b) {
    return a->d < b->d || (a->d == b->d && a->id < b->id);
}

int po_build_nsg(const float *x, uint32_t n, uint32_t d, uint32_t k, uint32_t R, uint32_t *knn_out,
                 uint32_t *entry_out, uint64_t *off_out, uint32_t *nbrs_out, uint64_t nbrs_cap,
                 uint32_t *width_out, int threads) {
    if (n < 2 || k == 0 || k >= n || R == 0 || R > k) return -1;
    uint32_t *pr = (uint32_t *) malloc((size_t) n * R * sizeof(uint32_t));
    uint32_t *deg = (uint32_t *) calloc(n, sizeof(uint32_t));
    double *kd = (double *) malloc((size_t) n * k * sizeof(double));
    if (!pr || !deg || !kd) return -2;
    /* exact k-NN by (d64, id) */
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 16)
    for (uint32_t a = 0; a < n; ++a) {
        po_dk *best = (po_dk *) malloc((size_t) (k + 1) * sizeof(po_dk));
        uint32_t cnt = 0;
        for (uint32_t b = 0; b < n; ++b) {
            if (b == a) continue;
            po_dk c = {po_d64(x + (size_t) a * d, x + (size_t) b * d, d), b};
            if (cnt == k && !po_dk_less(&c, &best[k - 1])) continue;
            uint32_t pos = cnt < k ? cnt : k - 1;
            while (pos > 0 && po_dk_less(&c, &best[pos - 1])) {
                best[pos] = best[pos - 1];
                --pos;
            }
            best[pos] = c;
            if (cnt < k) ++cnt;
        }
        for (uint32_t i = 0; i < k; ++i) {
            knn_out[(size_t) a * k + i] = best[i].id;
            kd[(size_t) a * k + i] = best[i].d;
        }
        free(best);
        /* MRNG prune */
        uint32_t nk = 0;
        for (uint32_t i = 0; i < k && nk < R; ++i) {
            const uint32_t b = knn_out[(size_t) a * k + i];
            const double dab = kd[(size_t) a * k + i];
            int occl = 0;
            for (uint32_t c = 0; c < nk && !occl; ++c)
                occl = po_d64(x + (size_t) pr[(size_t) a * R + c] * d, x + (size_t) b * d, d) < dab;
            if (!occl) pr[(size_t) a * R + nk++] = b;
        }
        deg[a] = nk;
    }
    /* entry: nearest to the float64 mean (rows summed in id order) */
    double *mean = (double *) calloc(d, sizeof(double));
    for (uint32_t r = 0; r < n; ++r)
        for (uint32_t j = 0; j < d; ++j) mean[j] += (double) x[(size_t) r * d + j];
    for (uint32_t j = 0; j < d; ++j) mean[j] /= (double) n;
    uint32_t entry = 0;
    double be = 0.0;
    for (uint32_t r = 0; r < n; ++r) {
        double acc = 0.0;
        for (uint32_t j = 0; j < d; ++j) {
            const double t = (double) x[(size_t) r * d + j] - mean[j];
            acc = fma(t, t, acc);
        }
        if (r == 0 || acc < be) {
            be = acc;
            entry = r;
        }
    }
    free(mean);
    /* adjacency with room for repair edges: lists as (start, length) in a growable pool */
    uint32_t **lists = (uint32_t **) malloc(n * sizeof(uint32_t *));
    uint32_t *len = (uint32_t *) malloc(n * sizeof(uint32_t));
    uint32_t *cap = (uint32_t *) malloc(n * sizeof(uint32_t));
    for (uint32_t a = 0; a < n; ++a) {
        cap[a] = deg[a] + 4;
        lists[a] = (uint32_t *) malloc(cap[a] * sizeof(uint32_t));
        memcpy(lists[a], pr + (size_t) a * R, deg[a] * sizeof(uint32_t));
        len[a] = deg[a];
    }
    uint8_t *reached = (uint8_t *) calloc(n, 1);
    uint32_t *queue = (uint32_t *) malloc(n * sizeof(uint32_t));
    /* BFS from src over not-yet-reached vertices */
#define PO_WALK(src)                                                         \
    do {                                                                     \
        uint32_t qh = 0, qt = 0;                                             \
        reached[src] = 1;                                                    \
        queue[qt++] = (src);                                                 \
        while (qh < qt) {                                                    \
            const uint32_t v = queue[qh++];                                  \
            for (uint32_t e = 0; e < len[v]; ++e) {                          \
                const uint32_t w = lists[v][e];                              \
                if (!reached[w]) { reached[w] = 1; queue[qt++] = w; }        \
            }                                                                \
        }                                                                    \
    } while (0)
    PO_WALK(entry);
    for (uint32_t u = 0; u < n; ++u) {
        if (reached[u]) continue;
        uint32_t parent = entry;
        for (uint32_t i = 0; i < k; ++i) {
            const uint32_t c = knn_out[(size_t) u * k + i];
            if (reached[c]) { parent = c; break; }
        }
        if (len[parent] == cap[parent]) {
            cap[parent] *= 2;
            lists[parent] = (uint32_t *) realloc(lists[parent], cap[parent] * sizeof(uint32_t));
        }
        lists[parent][len[parent]++] = u;
        PO_WALK(u);
    }
#undef PO_WALK
    uint64_t total = 0;
    uint32_t width = 0;
    off_out[0] = 0;
    int err = 0;
    for (uint32_t a = 0; a < n; ++a) {
        if (total + len[a] > nbrs_cap) err = 1;
        if (!err) memcpy(nbrs_out + total, lists[a], len[a] * sizeof(uint32_t));
        total += len[a];
        off_out[a + 1] = total;
        if (len[a] > width) width = len[a];
        free(lists[a]);
    }
    *entry_out = entry;
    *width_out = width;
    free(lists); free(len); free(cap); free(reached); free(queue); free(pr); free(deg); free(kd);
    return err ? -3 : 0;
}
