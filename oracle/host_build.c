/* Host-side construction of the benchmark workload's inputs — TEST AND
 * BENCHMARK INFRASTRUCTURE ONLY (part of oracle/_ref/panns_oracle.so).
 *
 * The reference arm of the benchmark runs the reference's own CPU search, so
 * its inputs (the NSG-style graph and the float64 ground truth) must be made
 * without the GPU library. These functions compute exactly what
 * po_build_nsg / the GPU construction (parallel_anns_b200/csrc/graph_build.cu)
 * and the GPU ground truth (parallel_anns_b200/csrc/gt_kernel.cuh) compute:
 *
 *   d64(x, y) = sum over j = 0..d-1, in order, of fma(t, t, acc),
 *               t = (double) x[j] - (double) y[j]  (the sign of t is irrelevant);
 *   knn(a)    = the k vertices b with the smallest (d64(a, b), b), b != a for
 *               the graph, every b for the ground truth of a query;
 *   prune, entry and repair as in po_build_nsg.
 *
 * Only the order of work differs, so that a 1M-vertex workload takes seconds
 * instead of hours: the base is partitioned into clusters (farthest-point
 * seeds, two Lloyd rounds), and a point scans its own cluster first and then
 * only the clusters whose triangle-inequality lower bound
 * (|p - c| - radius(c))^2 does not exceed its current k-th distance (with a
 * safety margin far above the rounding error). Every distance that can enter a
 * list is computed by the same float64 FMA chain, so the result equals the
 * brute-force one bit for bit; tests/test_host_build.py checks it against
 * po_build_nsg and po_ground_truth_fp64.
 */
#include "panns_oracle.h"

#include <immintrin.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HB_LANES 16u             /* candidates per scan block */
#define HB_NONE 0xffffffffu

typedef struct {
    uint32_t n, d, P;
    double *center;   /* P x d */
    double *radius;   /* P */
    uint32_t *blk0;   /* P + 1: first block of each cluster */
    uint32_t *ids;    /* nblk x 16 original ids (HB_NONE = padding) */
    float *blk;       /* nblk x d x 16 coordinates, candidate-minor */
} hb_clusters;

static double hb_d64(const float *a, const double *b, uint32_t d) {
    double acc = 0.0;
    for (uint32_t j = 0; j < d; ++j) {
        const double t = (double) a[j] - b[j];
        acc = fma(t, t, acc);
    }
    return acc;
}

static int hb_threads(int t) {
#ifdef _OPENMP
    return t > 0 ? t : omp_get_max_threads();
#else
    (void) t;
    return 1;
#endif
}

static void hb_free(hb_clusters *c) {
    free(c->center);
    free(c->radius);
    free(c->blk0);
    free(c->ids);
    free(c->blk);
}

/* Partition the rows of x into P clusters; the partition only affects speed. */
static int hb_cluster(const float *x, uint32_t n, uint32_t d, int threads, hb_clusters *C) {
    memset(C, 0, sizeof(*C));
    C->n = n;
    C->d = d;
    uint32_t P = n >= 4096 ? 64u : 1u;
    C->P = P;
    C->center = (double *) calloc((size_t) P * d, sizeof(double));
    C->radius = (double *) calloc(P, sizeof(double));
    C->blk0 = (uint32_t *) calloc(P + 1, sizeof(uint32_t));
    uint32_t *asg = (uint32_t *) malloc((size_t) n * sizeof(uint32_t));
    double *mind = NULL;
    if (!C->center || !C->radius || !C->blk0 || !asg) {
        free(asg);
        return -2;
    }
    if (P > 1) {
        /* farthest-point seeds on a strided sample (ties: the lowest index) */
        const uint32_t stride = n > 65536 ? n / 65536 : 1;
        const uint32_t ns = (n + stride - 1) / stride;
        mind = (double *) malloc((size_t) ns * sizeof(double));
        if (!mind) {
            free(asg);
            return -2;
        }
        uint32_t pick = 0;
        for (uint32_t c = 0; c < P; ++c) {
            for (uint32_t j = 0; j < d; ++j) C->center[(size_t) c * d + j] = (double) x[(size_t) pick * stride * d + j];
            const double *cc = C->center + (size_t) c * d;
            uint32_t best = 0;
            double bv = -1.0;
#pragma omp parallel num_threads(hb_threads(threads))
            {
                uint32_t tb = 0;
                double tv = -1.0;
#pragma omp for schedule(static)
                for (uint32_t s = 0; s < ns; ++s) {
                    const double v = hb_d64(x + (size_t) s * stride * d, cc, d);
                    if (c == 0 || v < mind[s]) mind[s] = v;
                    if (mind[s] > tv) {
                        tv = mind[s];
                        tb = s;
                    }
                }
#pragma omp critical
                {
                    if (tv > bv || (tv == bv && tb < best)) {
                        bv = tv;
                        best = tb;
                    }
                }
            }
            pick = best;
        }
        free(mind);
        /* two Lloyd rounds: assign to the nearest seed (ties: the lowest
         * cluster), then move each centre to its members' mean (id order) */
        double *sum = (double *) malloc((size_t) P * d * sizeof(double));
        uint32_t *cnt = (uint32_t *) malloc(P * sizeof(uint32_t));
        if (!sum || !cnt) {
            free(sum);
            free(cnt);
            free(asg);
            return -2;
        }
        for (int round = 0; round < 3; ++round) {
#pragma omp parallel for num_threads(hb_threads(threads)) schedule(static)
            for (uint32_t i = 0; i < n; ++i) {
                uint32_t b = 0;
                double bv = 0.0;
                for (uint32_t c = 0; c < P; ++c) {
                    const double v = hb_d64(x + (size_t) i * d, C->center + (size_t) c * d, d);
                    if (c == 0 || v < bv) {
                        bv = v;
                        b = c;
                    }
                }
                asg[i] = b;
            }
            if (round == 2) break;
            memset(sum, 0, (size_t) P * d * sizeof(double));
            memset(cnt, 0, P * sizeof(uint32_t));
            for (uint32_t i = 0; i < n; ++i) {
                double *s = sum + (size_t) asg[i] * d;
                for (uint32_t j = 0; j < d; ++j) s[j] += (double) x[(size_t) i * d + j];
                cnt[asg[i]]++;
            }
            for (uint32_t c = 0; c < P; ++c)
                if (cnt[c])
                    for (uint32_t j = 0; j < d; ++j) C->center[(size_t) c * d + j] = sum[(size_t) c * d + j] / cnt[c];
        }
        free(sum);
        free(cnt);
    } else {
        for (uint32_t i = 0; i < n; ++i) asg[i] = 0;
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t j = 0; j < d; ++j) C->center[j] += (double) x[(size_t) i * d + j];
        for (uint32_t j = 0; j < d; ++j) C->center[j] /= (double) (n ? n : 1);
    }
    /* members in (cluster, id) order, padded to blocks of 16 */
    uint32_t *members = (uint32_t *) calloc(P + 1, sizeof(uint32_t));
    if (!members) {
        free(asg);
        return -2;
    }
    for (uint32_t i = 0; i < n; ++i) members[asg[i]]++;
    uint32_t nblk = 0;
    for (uint32_t c = 0; c < P; ++c) {
        C->blk0[c] = nblk;
        nblk += (members[c] + HB_LANES - 1) / HB_LANES;
    }
    C->blk0[P] = nblk;
    C->ids = (uint32_t *) malloc((size_t) nblk * HB_LANES * sizeof(uint32_t));
    C->blk = (float *) calloc((size_t) nblk * HB_LANES * d, sizeof(float));
    if (!C->ids || !C->blk) {
        free(members);
        free(asg);
        return -2;
    }
    for (size_t i = 0; i < (size_t) nblk * HB_LANES; ++i) C->ids[i] = HB_NONE;
    memset(members, 0, (P + 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t c = asg[i];
        const size_t slot = (size_t) C->blk0[c] * HB_LANES + members[c]++;
        C->ids[slot] = i;
        float *b = C->blk + (slot / HB_LANES) * HB_LANES * d + slot % HB_LANES;
        for (uint32_t j = 0; j < d; ++j) b[(size_t) j * HB_LANES] = x[(size_t) i * d + j];
    }
    free(members);
    /* radii: the largest member distance to the centre */
#pragma omp parallel for num_threads(hb_threads(threads)) schedule(static)
    for (uint32_t c = 0; c < P; ++c) {
        double r = 0.0;
        for (size_t s = (size_t) C->blk0[c] * HB_LANES; s < (size_t) C->blk0[c + 1] * HB_LANES; ++s) {
            if (C->ids[s] == HB_NONE) continue;
            const double v = sqrt(hb_d64(x + (size_t) C->ids[s] * d, C->center + (size_t) c * d, d));
            if (v > r) r = v;
        }
        C->radius[c] = r;
    }
    free(asg);
    return 0;
}

/* d64 of one point (as float64 q) to the 16 candidates of a block. */
static inline void hb_block16(const float *blk, const double *q, uint32_t d, double *out) {
    __m256d a0 = _mm256_setzero_pd(), a1 = _mm256_setzero_pd();
    __m256d a2 = _mm256_setzero_pd(), a3 = _mm256_setzero_pd();
    for (uint32_t j = 0; j < d; ++j) {
        const float *r = blk + (size_t) j * HB_LANES;
        const __m256d qj = _mm256_set1_pd(q[j]);
        const __m256 x0 = _mm256_loadu_ps(r), x1 = _mm256_loadu_ps(r + 8);
        const __m256d t0 = _mm256_sub_pd(_mm256_cvtps_pd(_mm256_castps256_ps128(x0)), qj);
        const __m256d t1 = _mm256_sub_pd(_mm256_cvtps_pd(_mm256_extractf128_ps(x0, 1)), qj);
        const __m256d t2 = _mm256_sub_pd(_mm256_cvtps_pd(_mm256_castps256_ps128(x1)), qj);
        const __m256d t3 = _mm256_sub_pd(_mm256_cvtps_pd(_mm256_extractf128_ps(x1, 1)), qj);
        a0 = _mm256_fmadd_pd(t0, t0, a0);
        a1 = _mm256_fmadd_pd(t1, t1, a1);
        a2 = _mm256_fmadd_pd(t2, t2, a2);
        a3 = _mm256_fmadd_pd(t3, t3, a3);
    }
    _mm256_storeu_pd(out, a0);
    _mm256_storeu_pd(out + 4, a1);
    _mm256_storeu_pd(out + 8, a2);
    _mm256_storeu_pd(out + 12, a3);
}

/* Sorted insert of (v, id) into the k best by (distance, id). */
static inline void hb_insert(double *bd, uint32_t *bi, uint32_t *cnt, uint32_t k, double v, uint32_t id) {
    if (*cnt == k && !(v < bd[k - 1] || (v == bd[k - 1] && id < bi[k - 1]))) return;
    uint32_t pos = *cnt < k ? *cnt : k - 1;
    while (pos > 0 && (v < bd[pos - 1] || (v == bd[pos - 1] && id < bi[pos - 1]))) {
        bd[pos] = bd[pos - 1];
        bi[pos] = bi[pos - 1];
        --pos;
    }
    bd[pos] = v;
    bi[pos] = id;
    if (*cnt < k) ++*cnt;
}

/* Exact top-k of each query row (queries == NULL: every base row, itself
 * excluded) by (d64, id). */
static int hb_knn(const hb_clusters *C, const float *x, const float *queries, uint32_t nq, uint32_t k,
                  uint32_t *out_ids, double *out_d, int threads) {
    const uint32_t d = C->d, P = C->P;
    const int self = queries == NULL;
    const uint32_t count = self ? C->n : nq;
    if (k == 0 || k > C->n - (self ? 1u : 0u)) return -1;
    int err = 0;
#pragma omp parallel num_threads(hb_threads(threads)) reduction(| : err)
    {
        double *q = (double *) malloc((size_t) d * sizeof(double));
        double *bd = (double *) malloc((size_t) k * sizeof(double));
        uint32_t *bi = (uint32_t *) malloc((size_t) k * sizeof(uint32_t));
        double *lb = (double *) malloc((size_t) P * sizeof(double));
        uint32_t *order = (uint32_t *) malloc((size_t) P * sizeof(uint32_t));
        double dist[HB_LANES];
        if (!q || !bd || !bi || !lb || !order) {
            err |= 1;
        } else {
#pragma omp for schedule(dynamic, 32)
            for (uint32_t r = 0; r < count; ++r) {
                const float *qr = self ? x + (size_t) r * d : queries + (size_t) r * d;
                for (uint32_t j = 0; j < d; ++j) q[j] = (double) qr[j];
                /* clusters by lower bound (own cluster first: its bound is 0) */
                for (uint32_t c = 0; c < P; ++c) {
                    const double t = sqrt(hb_d64(qr, C->center + (size_t) c * d, d)) - C->radius[c];
                    lb[c] = t > 0 ? t * t : 0.0;
                    uint32_t p = c;
                    while (p > 0 && lb[order[p - 1]] > lb[c]) {
                        order[p] = order[p - 1];
                        --p;
                    }
                    order[p] = c;
                }
                uint32_t cnt = 0;
                for (uint32_t oc = 0; oc < P; ++oc) {
                    const uint32_t c = order[oc];
                    if (cnt == k && lb[c] > bd[k - 1] * (1.0 + 1e-9) + 1e-12) break;
                    for (uint32_t b = C->blk0[c]; b < C->blk0[c + 1]; ++b) {
                        hb_block16(C->blk + (size_t) b * HB_LANES * d, q, d, dist);
                        const uint32_t *ids = C->ids + (size_t) b * HB_LANES;
                        for (uint32_t l = 0; l < HB_LANES; ++l) {
                            const uint32_t id = ids[l];
                            if (id == HB_NONE || (self && id == r)) continue;
                            hb_insert(bd, bi, &cnt, k, dist[l], id);
                        }
                    }
                }
                memcpy(out_ids + (size_t) r * k, bi, k * sizeof(uint32_t));
                if (out_d) memcpy(out_d + (size_t) r * k, bd, k * sizeof(double));
            }
        }
        free(q);
        free(bd);
        free(bi);
        free(lb);
        free(order);
    }
    return err ? -2 : 0;
}

int po_host_knn(const float *x, uint32_t n, uint32_t d, const float *queries, uint32_t nq, uint32_t k,
                uint32_t *out_ids, double *out_dist, int threads) {
    if (!x || n == 0 || d == 0 || !out_ids) return -1;
    hb_clusters C;
    int rc = hb_cluster(x, n, d, threads, &C);
    if (rc == 0) rc = hb_knn(&C, x, queries, nq, k, out_ids, out_dist, threads);
    hb_free(&C);
    return rc;
}

int po_host_build_nsg(const float *x, uint32_t n, uint32_t d, uint32_t k, uint32_t R, uint32_t *knn_out,
                      uint32_t *entry_out, uint64_t *off_out, uint32_t *nbrs_out, uint64_t nbrs_cap,
                      uint32_t *width_out, int threads) {
    if (n < 2 || k == 0 || k >= n || R == 0 || R > k) return -1;
    double *kd = (double *) malloc((size_t) n * k * sizeof(double));
    uint32_t *pr = (uint32_t *) malloc((size_t) n * R * sizeof(uint32_t));
    uint32_t *deg = (uint32_t *) calloc(n, sizeof(uint32_t));
    if (!kd || !pr || !deg) {
        free(kd); free(pr); free(deg);
        return -2;
    }
    int rc = po_host_knn(x, n, d, NULL, 0, k, knn_out, kd, threads);
    if (rc) {
        free(kd); free(pr); free(deg);
        return rc;
    }
    /* MRNG prune: b (in list order) is dropped when a kept c has
     * d64(c, b) < d64(a, b); four kept vertices per vector, each lane one
     * exact FMA chain over the dimensions in order. */
    const uint32_t R4 = (R + 3) & ~3u;
    int err = 0;
#pragma omp parallel num_threads(hb_threads(threads)) reduction(| : err)
    {
        double *S = (double *) malloc((size_t) d * k * sizeof(double));   /* candidate rows, transposed */
        double *KT = (double *) calloc((size_t) d * R4, sizeof(double));  /* kept rows, transposed */
        if (!S || !KT) {
            err |= 1;
        } else {
#pragma omp for schedule(dynamic, 64)
            for (uint32_t a = 0; a < n; ++a) {
                const uint32_t *lst = knn_out + (size_t) a * k;
                for (uint32_t i = 0; i < k; ++i)
                    for (uint32_t j = 0; j < d; ++j) S[(size_t) j * k + i] = (double) x[(size_t) lst[i] * d + j];
                uint32_t nk = 0;
                for (uint32_t i = 0; i < k && nk < R; ++i) {
                    const double dab = kd[(size_t) a * k + i];
                    const __m256d vdab = _mm256_set1_pd(dab);
                    int occl = 0;
                    for (uint32_t c0 = 0; c0 < nk && !occl; c0 += 4) {
                        __m256d acc = _mm256_setzero_pd();
                        for (uint32_t j = 0; j < d; ++j) {
                            const __m256d t = _mm256_sub_pd(_mm256_loadu_pd(KT + (size_t) j * R4 + c0),
                                                            _mm256_set1_pd(S[(size_t) j * k + i]));
                            acc = _mm256_fmadd_pd(t, t, acc);
                        }
                        const int m = _mm256_movemask_pd(_mm256_cmp_pd(acc, vdab, _CMP_LT_OQ));
                        const uint32_t live = nk - c0 >= 4 ? 0xfu : (1u << (nk - c0)) - 1u;
                        occl = (m & (int) live) != 0;
                    }
                    if (!occl) {
                        for (uint32_t j = 0; j < d; ++j) KT[(size_t) j * R4 + nk] = S[(size_t) j * k + i];
                        pr[(size_t) a * R + nk++] = lst[i];
                    }
                }
                deg[a] = nk;
            }
        }
        free(S);
        free(KT);
    }
    free(kd);
    if (err) {
        free(pr); free(deg);
        return -2;
    }
    /* entry: the smallest (d64(v, mean), v), mean summed in id order */
    double *mean = (double *) calloc(d, sizeof(double));
    for (uint32_t r = 0; r < n; ++r)
        for (uint32_t j = 0; j < d; ++j) mean[j] += (double) x[(size_t) r * d + j];
    for (uint32_t j = 0; j < d; ++j) mean[j] /= (double) n;
    uint32_t entry = 0;
    double be = 0.0;
    int have = 0;
#pragma omp parallel num_threads(hb_threads(threads))
    {
        uint32_t te = 0;
        double tv = 0.0;
        int th = 0;
#pragma omp for schedule(static)
        for (uint32_t r = 0; r < n; ++r) {
            const double v = hb_d64(x + (size_t) r * d, mean, d);
            if (!th || v < tv) {
                tv = v;
                te = r;
                th = 1;
            }
        }
#pragma omp critical
        {
            if (th && (!have || tv < be || (tv == be && te < entry))) {
                be = tv;
                entry = te;
                have = 1;
            }
        }
    }
    free(mean);
    /* reachability repair, exactly as po_build_nsg */
    uint32_t **lists = (uint32_t **) malloc(n * sizeof(uint32_t *));
    uint32_t *len = (uint32_t *) malloc(n * sizeof(uint32_t));
    uint32_t *cap = (uint32_t *) malloc(n * sizeof(uint32_t));
    uint8_t *reached = (uint8_t *) calloc(n, 1);
    uint32_t *queue = (uint32_t *) malloc(n * sizeof(uint32_t));
    if (!lists || !len || !cap || !reached || !queue) {
        free(lists); free(len); free(cap); free(reached); free(queue); free(pr); free(deg);
        return -2;
    }
    for (uint32_t a = 0; a < n; ++a) {
        cap[a] = deg[a] + 4;
        lists[a] = (uint32_t *) malloc(cap[a] * sizeof(uint32_t));
        memcpy(lists[a], pr + (size_t) a * R, deg[a] * sizeof(uint32_t));
        len[a] = deg[a];
    }
#define HB_WALK(src)                                                         \
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
    HB_WALK(entry);
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
        HB_WALK(u);
    }
#undef HB_WALK
    uint64_t total = 0;
    uint32_t width = 0;
    off_out[0] = 0;
    int over = 0;
    for (uint32_t a = 0; a < n; ++a) {
        if (total + len[a] > nbrs_cap) over = 1;
        if (!over) memcpy(nbrs_out + total, lists[a], len[a] * sizeof(uint32_t));
        total += len[a];
        off_out[a + 1] = total;
        if (len[a] > width) width = len[a];
        free(lists[a]);
    }
    *entry_out = entry;
    *width_out = width;
    free(lists); free(len); free(cap); free(reached); free(queue); free(pr); free(deg);
    return over ? -3 : 0;
}
