// A driver written the way the reference's app/PSS_v5_distance_threshold_profiling.cpp
// (:48-152) drives PANNS::Searching, compiled against include/panns_searching.hpp:
// load data, queries and graph, prepare the init ids once, search every query
// with the per-query method, then the batched form, and print the ids.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "panns_searching.hpp"

int main(int argc, char **argv) {
    if (argc != 8) {
        fprintf(stderr, "usage: %s data query nsg K L T X\n", argv[0]);
        return 2;
    }
    PANNS::Searching engine;
    engine.load_data_load(argv[1]);
    engine.load_queries_load(argv[2]);
    engine.load_nsg_graph(argv[3]);
    const unsigned K = strtoul(argv[4], nullptr, 0), L = strtoul(argv[5], nullptr, 0);
    const int T = (int) strtoul(argv[6], nullptr, 0);
    const unsigned X = strtoul(argv[7], nullptr, 0);
    engine.num_threads_ = T;
    std::vector<std::vector<PANNS::idi>> set_K_list(engine.num_queries_, std::vector<PANNS::idi>(K));
    std::vector<PANNS::idi> init_ids(L);
    std::vector<bool> is_visited(engine.num_v_);
    std::vector<PANNS::Candidate> set_L((T - 1) * L + L);
    std::vector<PANNS::idi> sizes(T, 0), starts(T);
    for (int i = 0; i < T; ++i) starts[i] = i * L;
    engine.prepare_init_ids(init_ids, L);
    for (unsigned q = 0; q < engine.num_queries_; ++q)
        engine.para_search_PSS_v5_dist_thresh_profiling(q, K, L, set_L, init_ids, set_K_list[q], L, starts, sizes,
                                                        is_visited, X);
    std::vector<std::vector<PANNS::idi>> batch;
    engine.para_search_PSS_v5_batch(K, L, init_ids, L, X, batch);
    int same = batch == set_K_list;
    for (const auto &r : set_K_list) {
        for (unsigned i = 0; i < K; ++i) printf(i ? " %u" : "%u", r[i]);
        printf("\n");
    }
    fprintf(stderr, "batch_equal=%d n_dist=%llu\n", same, (unsigned long long) engine.count_distance_computation_);
    return same ? 0 : 1;
}
