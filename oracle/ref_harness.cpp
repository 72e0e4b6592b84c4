// Checker harness around the reference's own search code (test infrastructure).
//
// This file is compiled together with the reference sources, unchanged and
// where they lie, into the binaries under oracle/_ref/ (see oracle/Makefile).
// It only loads the inputs, calls the reference's public methods in the same
// order as the reference apps do, and dumps the result ID lists, the distance
// computation count and the wall time. It is never part of the product.
//
// One source, four builds (one per reference engine, because every engine
// defines its own PANNS::Searching class):
//   -DREF_PSS     core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp
//                 (para_search_PSS_v5_dist_thresh_profiling, :1218-1515;
//                  call sequence of app/PSS_v5_distance_threshold_profiling.cpp:122-152)
//   -DREF_PSS_LG  core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.cpp
//                 (para_search_PSS_v5_large_graph_dist_thresh_profiling, :1376-1726)
//   -DREF_TOPM    core/Searching.202011241533.top_m_pure.cpp
//                 (seq_search_simple_search :1486-1605, seq_search_with_top_m_pure
//                  :1382-1484, para_search_with_top_m_pure :1881-2070)
//   -DREF_MULTI   core/Searching.202107292234.PSS_v5.multi_queries.LG.cpp
//                 (para_search_PSS_v5_multi_queries_LG :1379; inter-query mode: an
//                  outer OpenMP loop over queries, T / inner threads, each query
//                  searched by `inner` PSS_v5 threads, as in
//                  app/PSS_v5_multi_queries_LG.cpp:89-160)
//   -DREF_EFANNA  include/efanna2e/index_nsg.cpp (Search :452-518,
//                 SearchWithOptGraph :520-611; call sequence of
//                 app/profile_find_L_seq_single_query_simple_search.cpp:144-171)
//
// Arguments are key=value pairs:
//   data= queries= nsg= K= L= out= [truenn=] [nq=] [T=1] [L_local=L] [X=1]
//   [M=1] [mode=] [reps=1]
//   mode (REF_TOPM): simple | topm_seq | topm_para
//   mode (REF_EFANNA): search | opt
//   mode=dist (REF_PSS / REF_PSS_LG): write the distance of every query to
//       every vertex id listed in ids= (a raw u32 file) to out= as f32,
//       row-major [nq x n_ids]; REF_PSS also writes the vertex norms to
//       out=.norms.
// stdout: one JSON line with n_dist (of the last repetition), runtime_s (the
// best repetition), qps, recall100 (if truenn=), rep_times (every repetition,
// timed like app/PSS_v5_distance_threshold_profiling.cpp:129-152: a
// std::chrono bracket around prepare_init_ids and the query loop).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>
#include <omp.h>

#if defined(REF_PSS)
#include "core/Searching.202102022027.PSS_v5.dist_thresh.profiling.h"
#elif defined(REF_PSS_LG)
#include "core/Searching.202102031939.PSS_v5.large_graph.dist_thresh.profiling.h"
#elif defined(REF_TOPM)
#include "core/Searching.202011241533.top_m_pure.h"
#elif defined(REF_MULTI)
#include "core/Searching.202107292234.PSS_v5.multi_queries.LG.h"
#elif defined(REF_EFANNA)
#include "include/efanna2e/index_nsg.h"
#else
#error "define one of REF_PSS REF_PSS_LG REF_TOPM REF_MULTI REF_EFANNA"
#endif

static std::map<std::string, std::string> g_args;

static const char *arg_s(const char *k, const char *def = nullptr) {
    auto it = g_args.find(k);
    if (it == g_args.end()) {
        if (!def) {
            fprintf(stderr, "missing argument %s=\n", k);
            exit(2);
        }
        return def;
    }
    return it->second.c_str();
}
static unsigned arg_u(const char *k, const char *def = nullptr) {
    return (unsigned) strtoull(arg_s(k, def), nullptr, 0);
}

static void write_ids(const char *path, const std::vector<std::vector<unsigned>> &res) {
    FILE *f = fopen(path, "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
    for (const auto &r : res) fwrite(r.data(), sizeof(unsigned), r.size(), f);
    fclose(f);
}

// Recall@100 with the reference's definition
// (core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:191-230):
// |true top-100 ∩ result[0:min(L,100)]| / 100, averaged over queries.
static double recall100(const char *truenn, const std::vector<std::vector<unsigned>> &res, unsigned L) {
    FILE *f = fopen(truenn, "rb");
    if (!f) return -1.0;
    unsigned tq = 0, tk = 0;
    if (fread(&tq, 4, 1, f) != 1 || fread(&tk, 4, 1, f) != 1) { fclose(f); return -1.0; }
    std::vector<unsigned> ids((size_t) tq * tk);
    for (size_t i = 0; i < (size_t) tq * tk; ++i) {
        unsigned id; float d;
        if (fread(&id, 4, 1, f) != 1 || fread(&d, 4, 1, f) != 1) { fclose(f); return -1.0; }
        ids[i] = id;
    }
    fclose(f);
    const unsigned nq = (unsigned) res.size();
    if (tq < nq || tk < 100) return -1.0;
    const unsigned kk = L < 100 ? L : 100;
    double hit = 0;
    for (unsigned q = 0; q < nq; ++q) {
        for (unsigned t = 0; t < 100; ++t) {
            unsigned tid = ids[(size_t) q * tk + t];
            for (unsigned n = 0; n < kk && n < res[q].size(); ++n) {
                if (res[q][n] == tid) { hit += 1; break; }
            }
        }
    }
    return hit / (100.0 * nq);
}

static std::vector<double> g_rep_times;

static void report(double secs, unsigned long long n_dist, unsigned nq,
                   const std::vector<std::vector<unsigned>> &res, unsigned L, int threads) {
    double rec = -1.0;
    if (g_args.count("truenn")) rec = recall100(arg_s("truenn"), res, L);
    printf("{\"n_dist\": %llu, \"runtime_s\": %.9f, \"qps\": %.3f, \"recall100\": %.6f, "
           "\"threads\": %d, \"nq\": %u, \"rep_times\": [",
           n_dist, secs, nq / secs, rec, threads, nq);
    for (size_t i = 0; i < g_rep_times.size(); ++i) printf(i ? ", %.9f" : "%.9f", g_rep_times[i]);
    printf("]}\n");
}

int main(int argc, char **argv) {
    for (int i = 1; i < argc; ++i) {
        const char *eq = strchr(argv[i], '=');
        if (!eq) { fprintf(stderr, "bad argument %s\n", argv[i]); return 2; }
        g_args[std::string(argv[i], eq - argv[i])] = std::string(eq + 1);
    }
    const unsigned K = arg_u("K", "100");
    const unsigned L = arg_u("L", "100");
    const int T = (int) arg_u("T", "1");
    const unsigned reps = arg_u("reps", "1");
    const std::string mode = arg_s("mode", "");

#if defined(REF_MULTI)
    PANNS::Searching engine;
    engine.load_data_load(const_cast<char *>(arg_s("data")));
    engine.load_queries_load(const_cast<char *>(arg_s("queries")));
    engine.load_common_nsg_graph(const_cast<char *>(arg_s("nsg")));
    unsigned nq = arg_u("nq", "0");
    if (nq == 0 || nq > engine.num_queries_) nq = engine.num_queries_;
    {
        // Thread split of app/PSS_v5_multi_queries_LG.cpp:89-99 (inner = 8 when
        // T > 8), or the given inner= (1 = one thread per query).
        const unsigned inner = arg_u("inner", T > 8 ? "8" : std::to_string(T).c_str());
        const int outer = std::max(1, T / (int) inner);
        omp_set_max_active_levels(2);
        engine.num_threads_inner_ = (int) inner;
        const unsigned L_local = arg_u("L_local", std::to_string(L).c_str());
        const unsigned X = arg_u("X", "1");
        std::vector<std::vector<unsigned>> set_K_list(nq, std::vector<unsigned>(K));
        std::vector<unsigned> init_ids(L);
        std::vector<unsigned> local_queues_starts(inner);
        for (unsigned q_i = 0; q_i < inner; ++q_i) local_queues_starts[q_i] = q_i * L_local;
        double best = 1e300;
        unsigned long long n_dist = 0;
        for (unsigned rep = 0; rep < reps; ++rep) {
            uint64_t cnt = 0;
            auto s = std::chrono::high_resolution_clock::now();
            engine.prepare_init_ids(init_ids, L);
#pragma omp parallel for num_threads(outer) reduction(+ : cnt)
            for (unsigned q_i = 0; q_i < nq; ++q_i) {
                engine.para_search_PSS_v5_multi_queries_LG(q_i, K, L, init_ids, set_K_list[q_i], L_local,
                                                            local_queues_starts, X, cnt);
            }
            auto e = std::chrono::high_resolution_clock::now();
            double secs = std::chrono::duration<double>(e - s).count();
            g_rep_times.push_back(secs);
            if (secs < best) best = secs;
            n_dist = cnt;
        }
        write_ids(arg_s("out"), set_K_list);
        report(best, n_dist, nq, set_K_list, L, outer * (int) inner);
        return 0;
    }
#elif defined(REF_PSS) || defined(REF_PSS_LG) || defined(REF_TOPM)
    PANNS::Searching engine;
    engine.load_data_load(const_cast<char *>(arg_s("data")));
    engine.load_queries_load(const_cast<char *>(arg_s("queries")));
#if defined(REF_PSS_LG)
    engine.load_common_nsg_graph(const_cast<char *>(arg_s("nsg")));
#else
    engine.load_nsg_graph(const_cast<char *>(arg_s("nsg")));
#endif
    unsigned nq = arg_u("nq", "0");
    if (nq == 0 || nq > engine.num_queries_) nq = engine.num_queries_;

#if defined(REF_PSS) || defined(REF_PSS_LG)
    if (mode == "dist") {
        FILE *f = fopen(arg_s("ids"), "rb");
        if (!f) { fprintf(stderr, "cannot open ids\n"); return 2; }
        std::vector<unsigned> ids;
        unsigned v;
        while (fread(&v, 4, 1, f) == 1) ids.push_back(v);
        fclose(f);
        std::vector<float> out((size_t) nq * ids.size());
        for (unsigned q = 0; q < nq; ++q) {
            const float *qd = engine.queries_load_ + (size_t) q * engine.dimension_;
            for (size_t j = 0; j < ids.size(); ++j) {
#if defined(REF_PSS)
                const float *vd = reinterpret_cast<const float *>(
                        engine.opt_nsg_graph_ + (size_t) ids[j] * engine.vertex_bytes_);
                out[(size_t) q * ids.size() + j] = engine.compute_distance_with_norm(vd + 1, qd, vd[0]);
#else
                const float *vd = engine.data_load_ + (size_t) ids[j] * engine.dimension_;
                out[(size_t) q * ids.size() + j] = engine.compute_distance(vd, qd);
#endif
            }
        }
        f = fopen(arg_s("out"), "wb");
        fwrite(out.data(), 4, out.size(), f);
        fclose(f);
#if defined(REF_PSS)
        std::string np = std::string(arg_s("out")) + ".norms";
        f = fopen(np.c_str(), "wb");
        for (size_t j = 0; j < ids.size(); ++j) {
            const float *vd = reinterpret_cast<const float *>(
                    engine.opt_nsg_graph_ + (size_t) ids[j] * engine.vertex_bytes_);
            fwrite(vd, 4, 1, f);
        }
        fclose(f);
#endif
        return 0;
    }
#endif

    engine.num_threads_ = T;
    omp_set_num_threads(T);
    std::vector<std::vector<unsigned>> set_K_list(nq, std::vector<unsigned>(K));
    std::vector<unsigned> init_ids(L);
    boost::dynamic_bitset<> is_visited(engine.num_v_);
    double best = 1e300;
    unsigned long long n_dist = 0;

#if defined(REF_PSS) || defined(REF_PSS_LG)
    const unsigned L_local = arg_u("L_local", std::to_string(L).c_str());
    const unsigned X = arg_u("X", "1");
    std::vector<PANNS::Candidate> set_L((size_t) (T - 1) * L_local + L);
    std::vector<unsigned> local_queues_sizes(T, 0);
    std::vector<unsigned> local_queues_starts(T);
    for (int q_i = 0; q_i < T; ++q_i) local_queues_starts[q_i] = q_i * L_local;
    for (unsigned rep = 0; rep < reps; ++rep) {
        engine.count_distance_computation_ = 0;
        auto s = std::chrono::high_resolution_clock::now();
        engine.prepare_init_ids(init_ids, L);
        for (unsigned q_i = 0; q_i < nq; ++q_i) {
#if defined(REF_PSS)
            engine.para_search_PSS_v5_dist_thresh_profiling(
#else
            engine.para_search_PSS_v5_large_graph_dist_thresh_profiling(
#endif
                    q_i, K, L, set_L, init_ids, set_K_list[q_i], L_local,
                    local_queues_starts, local_queues_sizes, is_visited, X);
        }
        auto e = std::chrono::high_resolution_clock::now();
        double secs = std::chrono::duration<double>(e - s).count();
        g_rep_times.push_back(secs);
        if (secs < best) best = secs;
        n_dist = engine.count_distance_computation_;
    }
#else  // REF_TOPM
    const unsigned M = arg_u("M", "1");
    std::vector<PANNS::Candidate> set_L((size_t) (T - 1) * L + L);
    std::vector<unsigned> local_queues_sizes(T, 0);
    std::vector<unsigned> local_queues_starts(T);
    for (int q_i = 0; q_i < T; ++q_i) local_queues_starts[q_i] = q_i * L;
    std::vector<unsigned> top_m_candidates(M);
    for (unsigned rep = 0; rep < reps; ++rep) {
        engine.count_distance_computation_ = 0;
        auto s = std::chrono::high_resolution_clock::now();
        engine.prepare_init_ids(init_ids, L);
        for (unsigned q_i = 0; q_i < nq; ++q_i) {
            if (mode == "simple") {
                engine.seq_search_simple_search(q_i, K, L, set_L, init_ids, set_K_list[q_i], is_visited);
            } else if (mode == "topm_seq") {
                engine.seq_search_with_top_m_pure(M, q_i, K, L, set_L, init_ids, set_K_list[q_i],
                                                  top_m_candidates, is_visited);
            } else if (mode == "topm_para") {
                engine.para_search_with_top_m_pure(M, q_i, K, L, set_L, init_ids, set_K_list[q_i], L,
                                                   local_queues_starts, local_queues_sizes,
                                                   top_m_candidates, is_visited);
            } else {
                fprintf(stderr, "unknown mode %s\n", mode.c_str());
                return 2;
            }
        }
        auto e = std::chrono::high_resolution_clock::now();
        double secs = std::chrono::duration<double>(e - s).count();
        g_rep_times.push_back(secs);
        if (secs < best) best = secs;
        n_dist = engine.count_distance_computation_;
    }
#endif
    write_ids(arg_s("out"), set_K_list);
    report(best, n_dist, nq, set_K_list, L, T);
    return 0;

#else  // REF_EFANNA
    // Loader of app/profile_find_L_seq_single_query_simple_search.cpp:109-131,
    // restated: fvecs rows of (u32 dim, dim x f32).
    auto load = [](const char *fn, std::vector<float> &v, unsigned &num, unsigned &dim) {
        FILE *f = fopen(fn, "rb");
        if (!f) { fprintf(stderr, "cannot open %s\n", fn); exit(2); }
        if (fread(&dim, 4, 1, f) != 1) exit(2);
        fseek(f, 0, SEEK_END);
        size_t sz = (size_t) ftell(f);
        num = (unsigned) (sz / (dim + 1) / 4);
        v.resize((size_t) num * dim);
        fseek(f, 0, SEEK_SET);
        for (size_t i = 0; i < num; ++i) {
            unsigned d;
            if (fread(&d, 4, 1, f) != 1 || fread(v.data() + i * dim, 4, dim, f) != dim) exit(2);
        }
        fclose(f);
    };
    std::vector<float> data, queries;
    unsigned n, dim, nq_all, qdim;
    load(arg_s("data"), data, n, dim);
    load(arg_s("queries"), queries, nq_all, qdim);
    unsigned nq = arg_u("nq", "0");
    if (nq == 0 || nq > nq_all) nq = nq_all;
    efanna2e::IndexNSG index(dim, n, efanna2e::L2, nullptr);
    index.Load(arg_s("nsg"));
    if (mode == "opt") index.OptimizeGraph(data.data());
    efanna2e::Parameters paras;
    paras.Set<unsigned>("L_search", L);
    paras.Set<unsigned>("P_search", L);
    std::vector<std::vector<unsigned>> res(nq, std::vector<unsigned>(K));
    auto s = std::chrono::high_resolution_clock::now();
    for (unsigned i = 0; i < nq; i++) {
        if (mode == "opt")
            index.SearchWithOptGraph(queries.data() + (size_t) i * dim, K, paras, res[i].data());
        else
            index.Search(queries.data() + (size_t) i * dim, data.data(), K, paras, res[i].data());
    }
    auto e = std::chrono::high_resolution_clock::now();
    write_ids(arg_s("out"), res);
    report(std::chrono::duration<double>(e - s).count(), index.count_distance_computation_, nq, res, L, 1);
    return 0;
#endif
}
