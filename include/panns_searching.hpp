// panns_searching.hpp — PANNS::Searching and efanna2e::IndexNSG over the C ABI.
//
// Header-only C++ facade with the names, member variables and method
// signatures the reference's search drivers use, so that a driver such as
// app/PSS_v5_distance_threshold_profiling.cpp compiles against it by swapping
// its `#include "../core/Searching....h"` for this header and linking
// libpanns_b200.so. Every search runs on the GPU through include/panns_b200.h.
//
// Replaced interfaces (paths relative to the parallel_ANNS project root):
//   PANNS::Searching   core/Searching.202102022027.PSS_v5.dist_thresh.profiling.h:30-274
//                      core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.h
//                      core/Searching.202011241533.top_m_pure.h
//   PANNS::Candidate   include/Candidate.h:11-28
//   efanna2e::IndexNSG include/efanna2e/index_nsg.h:17-86 (query path)
//
// Differences, all deliberate:
//   * Errors throw panns::Error instead of exit(EXIT_FAILURE).
//   * Scratch arguments of the per-query methods (set_L, local_queues_*,
//     is_visited, top_m_candidates) are accepted for source compatibility and
//     not used: that state lives on the GPU. Any bitset type is accepted.
//   * A per-query call is one GPU launch; the *_batch methods search a whole
//     range of loaded queries in one launch and fill set_K_list directly.
//   * num_threads_ > 1 runs PSS_v5's worker queues in a fixed round-robin
//     order (the reference's threads race), see include/panns_b200.h.
#ifndef PANNS_SEARCHING_HPP
#define PANNS_SEARCHING_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "panns_b200.h"

namespace panns {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != PANNS_OK) throw Error(rc, panns_last_error());
}

}  // namespace panns

namespace PANNS {

using dataf = float;
using distf = float;
using idi = uint32_t;
using edgei = uint64_t;

struct Candidate {
    idi id_;
    distf distance_;
    bool is_checked_;
    Candidate() = default;
    Candidate(idi id, distf dist, bool is_checked) : id_(id), distance_(dist), is_checked_(is_checked) {}
    bool operator<(const Candidate &b) const {
        if (distance_ != b.distance_) return distance_ < b.distance_;
        return id_ < b.id_;
    }
};

class Searching {
public:
    idi num_v_ = 0;
    edgei num_e_ = 0;
    idi num_queries_ = 0;
    uint64_t dimension_ = 0;
    idi width_ = 0;
    idi ep_ = 0;
    int num_threads_ = 1;
    idi index_thresh_ = 99;
    uint64_t count_distance_computation_ = 0;
    uint64_t count_merge_ = 0;
    double time_expand_ = 0.0;
    double time_merge_ = 0.0;
    double time_seq_ = 0.0;
    // Storage of the search distances (PANNS_STORE_*); FP32 is the exact engine.
    uint32_t storage_ = PANNS_STORE_FP32;

    explicit Searching(int device = 0) { panns::check(panns_open(&h_, device)); }
    ~Searching() { panns_close(h_); }
    Searching(const Searching &) = delete;
    Searching &operator=(const Searching &) = delete;

    panns_index *handle() { return h_; }

    void load_data_load(char *filename) {
        panns::check(panns_load_fvecs_base(h_, filename, storage_));
        sync();
    }
    void load_queries_load(char *filename) {
        panns::check(panns_load_fvecs_queries(h_, filename));
        sync();
    }
    // Small-graph engine: norm-trick distance.
    void load_nsg_graph(char *filename) {
        panns::check(panns_load_nsg(h_, filename));
        distance_ = PANNS_DIST_NORM_IP;
        sync();
    }
    // Large-graph engine: full L2 distance.
    void load_common_nsg_graph(char *filename) {
        panns::check(panns_load_nsg(h_, filename));
        distance_ = PANNS_DIST_L2;
        sync();
    }

    void prepare_init_ids(std::vector<unsigned> &init_ids, const unsigned L) const {
        init_ids.resize(L);
        panns::check(panns_prepare_init_ids(h_, L, init_ids.data()));
    }

    void load_true_NN(const char *filename, std::vector<std::vector<idi>> &true_nn_list) {
        uint32_t nq = 0, k = 0;
        panns::check(panns_load_true_nn(filename, &nq, &k, nullptr, nullptr));
        if (nq < num_queries_) throw panns::Error(PANNS_EIO, "t_query_num is smaller than num_queries_");
        if (k < 100) throw panns::Error(PANNS_EIO, "t_K is smaller than 100");
        std::vector<uint32_t> ids((size_t) nq * k);
        panns::check(panns_load_true_nn(filename, &nq, &k, ids.data(), nullptr));
        true_nn_list.assign(nq, std::vector<idi>(k));
        for (uint32_t q = 0; q < nq; ++q)
            for (uint32_t i = 0; i < k; ++i) true_nn_list[q][i] = ids[(size_t) q * k + i];
    }

    void get_recall_for_all_queries(const std::vector<std::vector<idi>> &true_nn_list,
                                    const std::vector<std::vector<unsigned>> &set_K_list,
                                    std::unordered_map<unsigned, double> &recalls, const idi L) const {
        if (true_nn_list.empty() || true_nn_list[0].size() < 100)
            throw panns::Error(PANNS_EINVAL, "Number of true nearest neighbors of a query is smaller than 100.");
        const uint32_t nq = num_queries_, tk = (uint32_t) true_nn_list[0].size();
        const uint32_t K = set_K_list.empty() ? 0 : (uint32_t) set_K_list[0].size();
        std::vector<uint32_t> t((size_t) nq * tk), r((size_t) nq * K);
        for (uint32_t q = 0; q < nq; ++q) {
            for (uint32_t i = 0; i < tk; ++i) t[(size_t) q * tk + i] = true_nn_list[q][i];
            for (uint32_t i = 0; i < K; ++i) r[(size_t) q * K + i] = set_K_list[q][i];
        }
        for (unsigned at : {1u, 5u, 10u, 20u, 50u, 100u}) {
            double v = 0.0;
            if (K) panns::check(panns_recall(r.data(), nq, K, t.data(), tk, L, at, &v));
            recalls[at] = v;
        }
    }

    // ---- batched searches: queries [q_begin, q_begin + nq) in one launch ----
    void para_search_PSS_v5_batch(idi K, idi L, const std::vector<idi> &init_ids, idi L_local, idi X,
                                  std::vector<std::vector<idi>> &set_K_list, idi q_begin = 0,
                                  idi nq = ~0u) {
        run(PANNS_MODE_PSS_V5, K, L, 1, L_local, X, init_ids, set_K_list, q_begin, nq);
    }
    void seq_search_simple_search_batch(idi K, idi L, const std::vector<idi> &init_ids,
                                        std::vector<std::vector<idi>> &set_K_list, idi q_begin = 0,
                                        idi nq = ~0u) {
        run(PANNS_MODE_NSG_SEQ, K, L, 1, 0, 1, init_ids, set_K_list, q_begin, nq);
    }
    void para_search_with_top_m_pure_batch(idi M, idi K, idi L, const std::vector<idi> &init_ids,
                                           std::vector<std::vector<idi>> &set_K_list, idi q_begin = 0,
                                           idi nq = ~0u) {
        run(PANNS_MODE_TOP_M, K, L, M, 0, 1, init_ids, set_K_list, q_begin, nq);
    }

    // ---- per-query forms with the reference's signatures ----
    template <class Bitset>
    void para_search_PSS_v5_dist_thresh_profiling(const idi query_id, const idi K, const idi L,
                                                  std::vector<Candidate> &, const std::vector<idi> &init_ids,
                                                  std::vector<idi> &set_K, const idi local_queue_capacity,
                                                  const std::vector<idi> &, std::vector<idi> &, Bitset &,
                                                  const idi subsearch_iterations) {
        one(PANNS_MODE_PSS_V5, K, L, 1, local_queue_capacity, subsearch_iterations, init_ids, set_K, query_id);
    }
    template <class Bitset>
    void para_search_PSS_v5_large_graph_dist_thresh_profiling(
            const idi query_id, const idi K, const idi L, std::vector<Candidate> &set_L,
            const std::vector<idi> &init_ids, std::vector<idi> &set_K, const idi local_queue_capacity,
            const std::vector<idi> &starts, std::vector<idi> &sizes, Bitset &is_visited,
            const idi subsearch_iterations) {
        para_search_PSS_v5_dist_thresh_profiling(query_id, K, L, set_L, init_ids, set_K, local_queue_capacity,
                                                 starts, sizes, is_visited, subsearch_iterations);
    }
    template <class Bitset>
    void seq_search_simple_search(const idi query_id, const idi K, const idi L, std::vector<Candidate> &,
                                  const std::vector<idi> &init_ids, std::vector<idi> &set_K, Bitset &) {
        one(PANNS_MODE_NSG_SEQ, K, L, 1, 0, 1, init_ids, set_K, query_id);
    }
    template <class Bitset>
    void seq_search_with_top_m_pure(const idi M, const idi query_id, const idi K, const idi L,
                                    std::vector<Candidate> &, const std::vector<idi> &init_ids,
                                    std::vector<idi> &set_K, std::vector<idi> &, Bitset &) {
        one(PANNS_MODE_TOP_M, K, L, M, 0, 1, init_ids, set_K, query_id);
    }
    template <class Bitset>
    void para_search_with_top_m_pure(const idi M, const idi query_id, const idi K, const idi L,
                                     std::vector<Candidate> &, const std::vector<idi> &init_ids,
                                     std::vector<idi> &set_K, const idi, const std::vector<idi> &,
                                     std::vector<idi> &, std::vector<idi> &, Bitset &) {
        one(PANNS_MODE_TOP_M, K, L, M, 0, 1, init_ids, set_K, query_id);
    }

    panns_stats last_stats{};

private:
    panns_index *h_ = nullptr;
    uint32_t distance_ = PANNS_DIST_NORM_IP;

    void sync() {
        uint32_t n = 0, d = 0, nq = 0, w = 0, e = 0;
        panns::check(panns_info(h_, &n, &d, &nq, &w, &e));
        num_v_ = n;
        dimension_ = d;
        num_queries_ = nq;
        width_ = w;
        ep_ = e;
    }

    panns_search_params params(uint32_t mode, idi K, idi L, idi M, idi L_local, idi X) const {
        panns_search_params p{};
        p.mode = mode;
        p.distance = distance_;
        p.K = K;
        p.L = L;
        p.M = M;
        p.T = mode == PANNS_MODE_PSS_V5 ? (uint32_t) num_threads_ : 1u;
        p.L_local = L_local;
        p.X = X;
        p.storage = (mode == PANNS_MODE_PSS_V5 && num_threads_ > 1) ? PANNS_STORE_FP32 : storage_;
        return p;
    }

    void run(uint32_t mode, idi K, idi L, idi M, idi L_local, idi X, const std::vector<idi> &init_ids,
             std::vector<std::vector<idi>> &set_K_list, idi q_begin, idi nq) {
        if (nq == ~0u) nq = num_queries_ - q_begin;
        const panns_search_params p = params(mode, K, L, M, L_local, X);
        std::vector<uint32_t> out((size_t) nq * K);
        panns::check(panns_search(h_, &p, init_ids.empty() ? nullptr : init_ids.data(), q_begin, nq,
                                  out.data(), &last_stats));
        if (set_K_list.size() < (size_t) q_begin + nq) set_K_list.resize((size_t) q_begin + nq);
        for (idi q = 0; q < nq; ++q)
            set_K_list[q_begin + q].assign(out.begin() + (size_t) q * K, out.begin() + (size_t) (q + 1) * K);
        count_distance_computation_ += last_stats.n_dist;
        count_merge_ += last_stats.n_iter;
    }

    void one(uint32_t mode, idi K, idi L, idi M, idi L_local, idi X, const std::vector<idi> &init_ids,
             std::vector<idi> &set_K, idi query_id) {
        const panns_search_params p = params(mode, K, L, M, L_local, X);
        set_K.resize(K);
        panns::check(panns_search(h_, &p, init_ids.empty() ? nullptr : init_ids.data(), query_id, 1,
                                  set_K.data(), &last_stats));
        count_distance_computation_ += last_stats.n_dist;
        count_merge_ += last_stats.n_iter;
    }
};

}  // namespace PANNS

namespace efanna2e {

enum Metric { L2 = 0, INNER_PRODUCT = 1, FAST_L2 = 2, PQ = 3 };

// Parameters holds the one value the query path reads ("L_search").
class Parameters {
public:
    template <class T>
    void Set(const std::string &key, T value) {
        if (key == "L_search") L_search_ = (unsigned) value;
    }
    template <class T>
    T Get(const std::string &key) const {
        if (key != "L_search") throw panns::Error(PANNS_EINVAL, "only L_search is used by the search");
        return (T) L_search_;
    }

private:
    unsigned L_search_ = 0;
};

class IndexNSG {
public:
    uint64_t count_distance_computation_ = 0;
    uint64_t count_iters_ = 0;

    IndexNSG(size_t dimension, size_t n, Metric, void *, int device = 0) : dim_(dimension), n_(n) {
        panns::check(panns_open(&h_, device));
        panns::check(panns_rand_seed(rand_state_, 1));  // the never-seeded process-wide rand()
    }
    ~IndexNSG() { panns_close(h_); }
    IndexNSG(const IndexNSG &) = delete;
    IndexNSG &operator=(const IndexNSG &) = delete;

    void Load(const char *filename) { panns::check(panns_load_nsg(h_, filename)); }
    void OptimizeGraph(float *data) {
        set_base(data);
        opt_ = true;
    }
    void Search(const float *query, const float *x, size_t K, const Parameters &parameters, unsigned *indices) {
        if (!base_set_) set_base(x);
        search(query, 1, K, parameters.Get<unsigned>("L_search"), PANNS_DIST_L2, indices);
    }
    void SearchWithOptGraph(const float *query, size_t K, const Parameters &parameters, unsigned *indices) {
        if (!opt_) throw panns::Error(PANNS_ESTATE, "OptimizeGraph must be called first");
        search(query, 1, K, parameters.Get<unsigned>("L_search"), PANNS_DIST_NORM_IP, indices);
    }
    // nq consecutive queries in one launch; the rand() stream advances as if
    // they had been searched one by one.
    void SearchBatch(const float *queries, size_t nq, size_t K, unsigned L, bool opt_graph, unsigned *indices) {
        search(queries, nq, K, L, opt_graph ? PANNS_DIST_NORM_IP : PANNS_DIST_L2, indices);
    }

private:
    panns_index *h_ = nullptr;
    size_t dim_, n_;
    bool base_set_ = false, opt_ = false;
    int32_t rand_state_[40];

    void set_base(const float *x) {
        panns::check(panns_set_base(h_, x, (uint32_t) n_, (uint32_t) dim_, PANNS_STORE_FP32));
        base_set_ = true;
    }
    void search(const float *q, size_t nq, size_t K, unsigned L, uint32_t dist, unsigned *indices) {
        std::vector<uint32_t> init((size_t) nq * L);
        panns::check(panns_efanna_init_ids(h_, L, (uint32_t) nq, rand_state_, init.data()));
        panns_search_params p{};
        p.mode = PANNS_MODE_EFANNA;
        p.distance = dist;
        p.K = (uint32_t) K;
        p.L = L;
        p.M = 1;
        p.T = 1;
        p.X = 1;
        panns_stats st{};
        panns::check(panns_search_host(h_, &p, q, (uint32_t) nq, init.data(), indices, &st));
        count_distance_computation_ += st.n_dist;
        count_iters_ += st.n_expand;
    }
};

}  // namespace efanna2e

#endif
