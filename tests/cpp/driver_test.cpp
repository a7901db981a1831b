// Uses include/jet.h the way the reference's app/driver.cpp uses its jet.h
// (app/driver.cpp:97-146): load a METIS graph, allocate unit vertex weights
// with View("vertex weights", n) + deep_copy, run config.num_iter device-space
// partition attempts, keep the best partition and report the median cut.
//
//   driver_test <metis_graph> <k> <attempts> <best_part_out>
//
// Prints "device <min cut> <median cut> <n> <levels>", then the same for one
// host-space call ("host <cut>"), then "error <code>" for a call with k = 0.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <vector>

#include "jet.h"

using namespace jet_partitioner;

static value_t median(std::vector<value_t>& cuts) {
    std::sort(cuts.begin(), cuts.end());
    size_t c = cuts.size();
    return c % 2 == 0 ? (cuts[c / 2] + cuts[c / 2 - 1]) / 2 : cuts[c / 2];
}

int main(int argc, char** argv) {
    if (argc < 5) return 2;
    // the reference's load_metis_graph, app/io.hpp:99-217, through the library's reader
    int64_t n = 0, nnz = 0;
    void *row = nullptr, *adj = nullptr, *val = nullptr;
    int uniform = 0;
    if (jet_read_metis(argv[1], 0, 0, &n, &nnz, &row, &adj, &val, &uniform) != JET_OK) {
        std::fprintf(stderr, "%s\n", jet_last_error());
        return 3;
    }
    // host arrays -> owning device views, as io.hpp deep_copies its mirrors
    View<edge_offset_t, Space::Device> row_d("row map", (size_t)n + 1);
    View<ordinal_t, Space::Device> adj_d("entries", (size_t)nnz);
    wgt_vt val_d("values", (size_t)nnz);
    deep_copy(row_d, View<edge_offset_t, Space::Host>((edge_offset_t*)row, (size_t)n + 1));
    deep_copy(adj_d, View<ordinal_t, Space::Host>((ordinal_t*)adj, (size_t)nnz));
    deep_copy(val_d, View<value_t, Space::Host>((value_t*)val, (size_t)nnz));
    matrix_t g("input graph", (ordinal_t)n, val_d, matrix_t::Graph{row_d, adj_d});
    bool uniform_ew = uniform != 0;

    config_t config;
    config.coarsening_alg = 1;
    config.num_parts = std::atoi(argv[2]);
    config.num_iter = std::atoi(argv[3]);
    config.max_imb_ratio = 1.03;

    // app/driver.cpp:102-103
    wgt_vt vweights("vertex weights", g.numRows());
    deep_copy(vweights, 1);

    // app/driver.cpp:105-143
    part_vt best_part;
    value_t edgecut_min = std::numeric_limits<value_t>::max();
    std::vector<value_t> cuts;
    int levels = 0;
    for (int i = 0; i < config.num_iter; i++) {
        value_t edgecut = 0;
        experiment_data<value_t> experiment;
        set_seed(11 + i);
        part_vt part = partition(edgecut, config, g, vweights, uniform_ew, experiment);
        if (edgecut < edgecut_min) {
            edgecut_min = edgecut;
            best_part = part;
        }
        cuts.push_back(edgecut);
        levels = experiment.stats.num_levels;
    }
    // app/io.hpp:219-231 write_part
    part_mt best_host = create_mirror_view_and_copy(best_part);
    std::ofstream ofp(argv[4]);
    for (size_t x = 0; x < best_host.size(); x++) ofp << best_host(x) << "\n";
    ofp.close();
    value_t med = median(cuts);
    std::printf("device %d %d %zu %d\n", edgecut_min, med, best_part.size(), levels);

    // the host-space entry point on the same graph (host arrays)
    host_matrix_t gh("input graph", (ordinal_t)n, wgt_host_vt((value_t*)val, (size_t)nnz),
                     host_matrix_t::Graph{View<edge_offset_t, Space::Host>((edge_offset_t*)row, (size_t)n + 1),
                                          View<ordinal_t, Space::Host>((ordinal_t*)adj, (size_t)nnz)});
    wgt_host_vt vw_h("vertex weights", (size_t)n);
    deep_copy(vw_h, 1);
    value_t hcut = 0;
    experiment_data<value_t> hexp;
    set_seed(11);
    part_mt hp = partition_host(hcut, config, gh, vw_h, uniform_ew, hexp);
    std::printf("host %d %zu\n", hcut, hp.size());
    try {
        config_t bad = config;
        bad.num_parts = 0;
        partition_host(hcut, bad, gh, vw_h, uniform_ew, hexp);
        std::printf("error none\n");
    } catch (const jet_error& e) {
        std::printf("error %d\n", e.code);
    }
    jet_free_host(row);
    jet_free_host(adj);
    jet_free_host(val);
    return 0;
}
