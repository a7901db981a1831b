// jet.h -- C++ drop-in for the reference's public header (header/jet.h,
// header/jet_defs.h, header/jet_config.h, header/experiment_data.hpp) over
// the C ABI of libjetb200.so (include/jet_b200.h).
//
// Same namespace, type names, config fields, function names and parameter
// order as the reference.  Kokkos is not used: the matrix and view types are
// light structs over raw pointers -- device pointers for the default-space
// types (matrix_t, wgt_vt, part_vt), host pointers for the *_host / *_serial
// types -- exposing the members the reference's callers use (numRows(),
// nnz(), graph.row_map, graph.entries, values), the allocating
// View("label", n) constructor, deep_copy and create_mirror_view_and_copy.
// Device-space partition calls return an owning device view, host-space ones
// an owning host view.  All computation runs on the current CUDA device
// either way.  Errors throw jet_partitioner::jet_error
// (the reference exits on a Metis failure, src/initial_partition.hpp:106-109).
#pragma once

#include <cstdint>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "jet_b200.h"

namespace jet_partitioner {

// header/jet_defs.h:47-53
using big_ordinal_t = int64_t;
using big_offset_t = int64_t;
using big_val_t = int64_t;
using ordinal_t = int32_t;
using edge_offset_t = int32_t;
using value_t = int32_t;
using part_t = int;

// header/jet_config.h:43-52
struct config_t {
    int coarsening_alg = 0;
    int num_iter = 1;
    double max_imb_ratio = 1.03;
    int num_parts = 2;
    double refine_tolerance = 0.999;
    bool dump_coarse = false;
    bool verbose = false;
    bool ultra_settings = false;
};

struct jet_error : std::runtime_error {
    int code;
    jet_error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum class Space { Device, Host };

// A one-dimensional view: pointer + extent, optionally owning its storage.
//   View(ptr, n)        wraps caller memory (host or device, by S);
//   View("label", n)    allocates n zeroed elements and owns them, as
//                       Kokkos::View("label", n) does (app/driver.cpp:102):
//                       host memory for Space::Host, device memory of the
//                       current CUDA device for Space::Device.
// Copies share storage (reference counted), as Kokkos views do.
template <class T, Space S>
struct View {
    using value_type = T;
    using HostMirror = View<T, Space::Host>;
    T* ptr = nullptr;
    size_t n = 0;
    std::shared_ptr<void> owner;
    View() {}
    View(T* p, size_t count) : ptr(p), n(count) {}
    View(const std::string& label, size_t count) : n(count) {
        (void)label;
        if (S == Space::Host) {
            auto store = std::make_shared<std::vector<T>>(count, T());
            ptr = store->data();
            owner = store;
        } else {
            void* p = nullptr;
            int rc = jet_device_alloc((int64_t)(count * sizeof(T)), &p);
            if (rc != JET_OK) throw std::runtime_error(std::string("jet: device allocation failed: ") + jet_last_error());
            owner = std::shared_ptr<void>(p, [](void* q) { jet_device_free(q); });
            ptr = static_cast<T*>(p);
            if (count) {
                std::vector<T> zeros(count, T());
                jet_copy(ptr, zeros.data(), (int64_t)(count * sizeof(T)));
            }
        }
    }
    View(const char* label, size_t count) : View(std::string(label), count) {}
    T* data() const { return ptr; }
    size_t extent(int) const { return n; }
    size_t size() const { return n; }
    T& operator()(size_t i) const { return ptr[i]; }  // host views only
};

// Kokkos::deep_copy counterparts for these views: fill with a value, or copy
// between any two views of equal extent (host or device, either direction).
template <class T, Space S, class U>
void deep_copy(const View<T, S>& dst, const U& value) {
    if (S == Space::Host) {
        for (size_t i = 0; i < dst.n; i++) dst.ptr[i] = (T)value;
    } else if (dst.n) {
        std::vector<T> tmp(dst.n, (T)value);
        if (jet_copy(dst.ptr, tmp.data(), (int64_t)(dst.n * sizeof(T))) != JET_OK)
            throw std::runtime_error(std::string("jet: deep_copy failed: ") + jet_last_error());
    }
}
template <class T, Space S1, Space S2>
void deep_copy(const View<T, S1>& dst, const View<T, S2>& src) {
    if (dst.n != src.n) throw std::runtime_error("jet: deep_copy between views of different extents");
    if (dst.n && jet_copy(dst.ptr, src.ptr, (int64_t)(dst.n * sizeof(T))) != JET_OK)
        throw std::runtime_error(std::string("jet: deep_copy failed: ") + jet_last_error());
}
// Kokkos::create_mirror_view_and_copy: a host copy of any view.
template <class T, Space S>
View<T, Space::Host> create_mirror_view_and_copy(const View<T, S>& v) {
    View<T, Space::Host> h("mirror", v.n);
    deep_copy(h, v);
    return h;
}

// KokkosSparse::CrsMatrix shape (header/jet_defs.h:64-92).
template <class Val, class Ord, class Off, Space S>
struct CrsMatrix {
    using value_type = Val;
    using ordinal_type = Ord;
    using size_type = Off;
    struct Graph {
        View<Off, S> row_map;
        View<Ord, S> entries;
    } graph;
    View<Val, S> values;
    Ord num_rows = 0;
    CrsMatrix() {}
    CrsMatrix(const char*, Ord n, View<Val, S> vals, Graph g) : graph(g), values(vals), num_rows(n) {}
    Ord numRows() const { return num_rows; }
    Off nnz() const { return (Off)graph.entries.n; }
};

using matrix_t = CrsMatrix<value_t, ordinal_t, edge_offset_t, Space::Device>;
using host_matrix_t = CrsMatrix<value_t, ordinal_t, edge_offset_t, Space::Host>;
using serial_matrix_t = host_matrix_t;
using big_matrix_t = CrsMatrix<big_val_t, ordinal_t, big_offset_t, Space::Device>;
using big_host_matrix_t = CrsMatrix<big_val_t, ordinal_t, big_offset_t, Space::Host>;
using big_serial_matrix_t = big_host_matrix_t;
using biggest_matrix_t = CrsMatrix<big_val_t, big_ordinal_t, big_offset_t, Space::Device>;
using biggest_host_matrix_t = CrsMatrix<big_val_t, big_ordinal_t, big_offset_t, Space::Host>;
using biggest_serial_matrix_t = biggest_host_matrix_t;
using wgt_vt = View<value_t, Space::Device>;
using wgt_host_vt = View<value_t, Space::Host>;
using wgt_serial_vt = wgt_host_vt;
using big_wgt_vt = View<big_val_t, Space::Device>;
using big_wgt_host_vt = View<big_val_t, Space::Host>;
using big_wgt_serial_vt = big_wgt_host_vt;
using part_vt = View<part_t, Space::Device>;  // device partitions come back in library-allocated, owning views
using part_mt = View<part_t, Space::Host>;

// header/experiment_data.hpp:50-72
enum class Measurement : int {
    Map, Build, Count, Prefix, Bucket, Dedupe, RadixSort, RadixDedupe, WriteGraph, Permute, MapConstruct, Heavy,
    InitTransfer, HashmapAllocate, HashmapInsert, InitPartition, Coarsen, Refine, FreeGraph, Total, END
};

template <typename scalar_t>
class experiment_data {
public:
    std::vector<std::string> measurementNames{
        "coarsen-map", "coarsen-build", "coarsen-count", "coarsen-prefix-sum", "coarsen-bucket", "coarsen-dedupe",
        "coarsen-radix-sort", "coarsen-radix-dedupe", "coarsen-write-graph", "coarsen-permute", "coarsen-map-construct",
        "heavy", "initial-transfer-to-device", "hashmap-allocate", "hashmap-insert", "initial-partition", "coarsen",
        "refine", "free-graph", "total"};
    std::vector<double> measurements = std::vector<double>((int)Measurement::END, 0.0);
    jet_stats_c stats{};

    double getMeasurement(Measurement m) { return measurements[(int)m]; }
    void addMeasurement(Measurement m, double v) { measurements[(int)m] += v; }
    void fill(const jet_stats_c& s) {
        stats = s;
        for (int i = 0; i < (int)Measurement::END; i++) measurements[i] += s.measurements[i];
    }
    // header/experiment_data.hpp:177-207
    void log(const char* filename, bool first, bool last) {
        std::ofstream f(filename, std::ios::app);
        if (!f.is_open()) { std::cerr << "Could not open " << filename << std::endl; return; }
        if (first) f << "[";
        f << "{" << "\"edge-cut\":" << std::fixed << stats.edge_cut << "," << "\"max-part-cut\":" << stats.max_part_cut << ","
          << "\"objective\":" << stats.objective << "," << "\"imbalance-ratio\":" << stats.imb_ratio << ',';
        for (int i = 0; i < (int)Measurement::END; i++) f << "\"" << measurementNames[i] << "-duration-seconds\":" << measurements[i] << ",";
        f << "\"number-coarse-levels\":" << stats.num_levels << ",";
        f << "\"finest-refinement-duration-seconds\":" << (stats.num_levels ? stats.levels[stats.num_levels - 1].total_ref_time : 0.0);
        f << "}" << (last ? "]" : ",");
    }
    // header/experiment_data.hpp:230-242
    void refinementReport() {
        std::cout << std::setprecision(6) << std::left << std::setw(6) << "Level" << std::setw(16) << "Edge Cut" << std::setw(10)
                  << "Imbalance" << std::setw(13) << "Vertices" << std::setw(16) << "Edges" << std::setw(22) << "Total Refinement Time"
                  << std::setw(17) << "Total Iterations" << std::setw(14) << "LP Iterations" << std::setw(23) << "Average Iteration Time"
                  << std::endl;
        int nl = stats.num_levels < JET_MAX_LEVELS ? stats.num_levels : JET_MAX_LEVELS;
        for (int i = 0; i < nl; i++) {
            const jet_level_stats_c& cl = stats.levels[i];
            std::cout << std::fixed << std::left << std::setw(6) << (nl - 1 - i) << std::setw(16) << cl.edge_cut << std::setw(10) << cl.imb
                      << std::setw(13) << cl.num_vertices << std::setw(16) << cl.num_edges << std::setw(22) << cl.total_ref_time << std::setw(17)
                      << cl.total_iterations << std::setw(14) << cl.lp_iterations << std::setw(23)
                      << (cl.total_iterations ? cl.iterations_time / cl.total_iterations : 0.0) << std::endl;
        }
    }
    // header/experiment_data.hpp:209-228
    void verboseReport() {
        std::cout << "Final cut: " << std::fixed << stats.edge_cut << "; Max part cut: " << stats.max_part_cut << "; imb: " << stats.imb_ratio
                  << "; largest: " << stats.largest_part << "; smallest: " << stats.smallest_part << std::endl;
        std::cout << std::setprecision(5) << "Coarsening time: " << getMeasurement(Measurement::Coarsen) << std::endl
                  << "Initial partitioning time: " << getMeasurement(Measurement::InitPartition) << std::endl
                  << "Uncoarsening time: " << getMeasurement(Measurement::Refine) << std::endl
                  << "Total Partitioning Time: " << getMeasurement(Measurement::Total) << std::endl
                  << "Comm size: " << stats.objective << std::endl;
    }
};

namespace detail {
inline jet_config_c to_c(const config_t& c) {
    jet_config_c r;
    r.coarsening_alg = c.coarsening_alg; r.num_iter = c.num_iter; r.max_imb_ratio = c.max_imb_ratio; r.num_parts = c.num_parts;
    r.refine_tolerance = c.refine_tolerance; r.dump_coarse = c.dump_coarse; r.verbose = c.verbose; r.ultra_settings = c.ultra_settings;
    return r;
}
inline void check(int rc) {
    if (rc != JET_OK) throw jet_error(rc, std::string("jet: ") + jet_last_error());
}
inline uint64_t& seed() {
    static thread_local uint64_t s = 1;
    return s;
}
}  // namespace detail

// Coarsening RNG seed (the reference seeds from the clock, src/contract.hpp:503).
inline void set_seed(uint64_t s) { detail::seed() = s; }

// Device-space calls return a fresh device view the caller owns, as the
// reference returns a freshly allocated Kokkos view (header/jet.h:46-51).
template <class Mat, class WV, class Cut, class Fn>
part_vt partition_device_impl(Cut& edge_cut, const config_t& config, const Mat& g, const WV& vweights, bool uniform_ew,
                              experiment_data<Cut>& experiment, Fn fn) {
    part_vt out("part", (size_t)g.numRows());
    jet_config_c c = detail::to_c(config);
    jet_stats_c st;
    detail::check(fn(&c, g.numRows(), g.graph.row_map.data(), g.graph.entries.data(), g.values.data(), vweights.data(),
                     (int)uniform_ew, JET_MEM_DEVICE, detail::seed(), nullptr, out.data(), &edge_cut, &st));
    experiment.fill(st);
    return out;
}

template <class Mat, class WV, class Cut, class Fn>
part_mt partition_host_impl(Cut& edge_cut, const config_t& config, const Mat& g, const WV& vweights, bool uniform_ew,
                            experiment_data<Cut>& experiment, Fn fn) {
    part_mt res("part", (size_t)g.numRows());
    jet_config_c c = detail::to_c(config);
    jet_stats_c st;
    detail::check(fn(&c, g.numRows(), g.graph.row_map.data(), g.graph.entries.data(), g.values.data(), vweights.data(),
                     (int)uniform_ew, JET_MEM_HOST, detail::seed(), nullptr, res.ptr, &edge_cut, &st));
    experiment.fill(st);
    return res;
}

// header/jet.h:46-107
inline part_vt partition(value_t& edge_cut, const config_t& config, const matrix_t g, const wgt_vt vweights, bool uniform_ew,
                         experiment_data<value_t>& experiment) {
    return partition_device_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_i32);
}
inline part_mt partition_host(value_t& edge_cut, const config_t& config, const host_matrix_t g, const wgt_host_vt vweights,
                              bool uniform_ew, experiment_data<value_t>& experiment) {
    return partition_host_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_i32);
}
inline part_mt partition_serial(value_t& edge_cut, const config_t& config, const serial_matrix_t g, const wgt_serial_vt vweights,
                                bool uniform_ew, experiment_data<value_t>& experiment) {
    return partition_host_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_i32);
}
inline part_vt partition_big(big_val_t& edge_cut, const config_t& config, const big_matrix_t g, const big_wgt_vt vweights,
                             bool uniform_ew, experiment_data<big_val_t>& experiment) {
    return partition_device_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_big);
}
inline part_mt partition_host_big(big_val_t& edge_cut, const config_t& config, const big_host_matrix_t g,
                                  const big_wgt_host_vt vweights, bool uniform_ew, experiment_data<big_val_t>& experiment) {
    return partition_host_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_big);
}
inline part_mt partition_serial_big(big_val_t& edge_cut, const config_t& config, const big_serial_matrix_t g,
                                    const big_wgt_serial_vt vweights, bool uniform_ew, experiment_data<big_val_t>& experiment) {
    return partition_host_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_big);
}
inline part_vt partition_biggest(big_val_t& edge_cut, const config_t& config, const biggest_matrix_t g, const big_wgt_vt vweights,
                                 bool uniform_ew, experiment_data<big_val_t>& experiment) {
    return partition_device_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_biggest);
}
inline part_mt partition_host_biggest(big_val_t& edge_cut, const config_t& config, const biggest_host_matrix_t g,
                                      const big_wgt_host_vt vweights, bool uniform_ew, experiment_data<big_val_t>& experiment) {
    return partition_host_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_biggest);
}
inline part_mt partition_serial_biggest(big_val_t& edge_cut, const config_t& config, const biggest_serial_matrix_t g,
                                        const big_wgt_serial_vt vweights, bool uniform_ew, experiment_data<big_val_t>& experiment) {
    return partition_host_impl(edge_cut, config, g, vweights, uniform_ew, experiment, jet_partition_biggest);
}

}  // namespace jet_partitioner
