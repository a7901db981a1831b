// Exercises include/jet.h the way the reference's app/driver.cpp uses
// jet.h: build a CrsMatrix, call partition_host / partition, read the cut and
// the experiment report.  Prints "host <cut> <maxpart>" and "device <cut>".
#include <cuda_runtime.h>
#include <cstdio>
#include <vector>
#include "jet.h"

using namespace jet_partitioner;

int main() {
    const int nx = 96, ny = 80, n = nx * ny;
    std::vector<edge_offset_t> row(n + 1, 0);
    std::vector<ordinal_t> adj;
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            int i = y * nx + x;
            if (y > 0) adj.push_back(i - nx);
            if (x > 0) adj.push_back(i - 1);
            if (x + 1 < nx) adj.push_back(i + 1);
            if (y + 1 < ny) adj.push_back(i + nx);
            row[i + 1] = (edge_offset_t)adj.size();
        }
    std::vector<value_t> val(adj.size(), 1), vw(n, 1);
    config_t config;
    config.coarsening_alg = 1;
    config.num_parts = 16;
    config.max_imb_ratio = 1.03;
    host_matrix_t::Graph hg{View<edge_offset_t, Space::Host>(row.data(), row.size()), View<ordinal_t, Space::Host>(adj.data(), adj.size())};
    host_matrix_t g("grid", n, View<value_t, Space::Host>(val.data(), val.size()), hg);
    value_t cut = 0;
    experiment_data<value_t> exp;
    set_seed(3);
    part_mt part = partition_host(cut, config, g, wgt_host_vt(vw.data(), vw.size()), true, exp);
    int maxp = 0;
    for (size_t i = 0; i < part.size(); i++) maxp = part(i) > maxp ? part(i) : maxp;
    printf("host %d %d %d\n", cut, maxp, exp.stats.num_levels);

    edge_offset_t* drow; ordinal_t* dadj; value_t* dval; value_t* dvw; part_t* dpart;
    cudaMalloc(&drow, sizeof(edge_offset_t) * row.size());
    cudaMalloc(&dadj, sizeof(ordinal_t) * adj.size());
    cudaMalloc(&dval, sizeof(value_t) * val.size());
    cudaMalloc(&dvw, sizeof(value_t) * vw.size());
    cudaMalloc(&dpart, sizeof(part_t) * n);
    cudaMemcpy(drow, row.data(), sizeof(edge_offset_t) * row.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(dadj, adj.data(), sizeof(ordinal_t) * adj.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(dval, val.data(), sizeof(value_t) * val.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(dvw, vw.data(), sizeof(value_t) * vw.size(), cudaMemcpyHostToDevice);
    matrix_t::Graph dg{View<edge_offset_t, Space::Device>(drow, row.size()), View<ordinal_t, Space::Device>(dadj, adj.size())};
    matrix_t gd("grid", n, View<value_t, Space::Device>(dval, val.size()), dg);
    set_device_output(dpart);
    value_t dcut = 0;
    experiment_data<value_t> dexp;
    part_vt dp = partition(dcut, config, gd, wgt_vt(dvw, vw.size()), true, dexp);
    printf("device %d %zu\n", dcut, dp.size());
    try {
        config_t bad = config;
        bad.num_parts = 0;
        partition_host(cut, bad, g, wgt_host_vt(vw.data(), vw.size()), true, exp);
        printf("no error\n");
    } catch (const jet_error& e) {
        printf("error %d\n", e.code);
    }
    return 0;
}
