// KokkosSparse_CrsMatrix.hpp -- TEST INFRASTRUCTURE ONLY.
//
// The CrsMatrix / StaticCrsGraph shapes the Jet reference uses
// (reference header/jet_defs.h:64-92, app/io.hpp:213-214), over the host-only
// views of the Kokkos stand-in in this directory.
#pragma once
#include "Kokkos_Core.hpp"

namespace Kokkos {

struct LayoutLeft {};
struct LayoutRight {};

template <class Ordinal, class Layout, class Dev, class MemTraits = void, class SizeType = size_t>
class StaticCrsGraph {
public:
    using execution_space = typename Dev::execution_space;
    using memory_space = HostSpace;
    using device_type = Device<execution_space, memory_space>;
    using data_type = Ordinal;
    using size_type = SizeType;
    using entries_type = View<Ordinal*, device_type>;
    using row_map_type = View<const SizeType*, device_type>;

    entries_type entries;
    row_map_type row_map;

    StaticCrsGraph() = default;
    template <class E, class R>
    StaticCrsGraph(const E& e, const R& r) : entries(e), row_map(r) {}
    Ordinal numRows() const { return row_map.extent(0) > 0 ? (Ordinal)(row_map.extent(0) - 1) : 0; }
};

}  // namespace Kokkos

namespace KokkosSparse {

template <class Scalar, class Ordinal, class Dev, class MemTraits = void, class SizeType = size_t>
class CrsMatrix {
public:
    using execution_space = typename Dev::execution_space;
    using memory_space = Kokkos::HostSpace;
    using device_type = Kokkos::Device<execution_space, memory_space>;
    using value_type = Scalar;
    using scalar_type = Scalar;
    using ordinal_type = Ordinal;
    using size_type = SizeType;
    using staticcrsgraph_type = Kokkos::StaticCrsGraph<Ordinal, Kokkos::LayoutLeft, device_type, void, SizeType>;
    using StaticCrsGraphType = staticcrsgraph_type;
    using row_map_type = typename staticcrsgraph_type::row_map_type;
    using index_type = typename staticcrsgraph_type::entries_type;
    using values_type = Kokkos::View<Scalar*, device_type>;
    using HostMirror = CrsMatrix;

    staticcrsgraph_type graph;
    values_type values;
    Ordinal numCols_ = 0;

    CrsMatrix() = default;
    template <class V>
    CrsMatrix(const std::string&, Ordinal ncols, const V& vals, const staticcrsgraph_type& g)
        : graph(g), values(vals), numCols_(ncols) {}
    template <class S2, class O2, class D2, class M2, class Z2>
    CrsMatrix(const CrsMatrix<S2, O2, D2, M2, Z2>& o) : graph(o.graph.entries, o.graph.row_map), values(o.values), numCols_(o.numCols_) {}

    Ordinal numRows() const { return graph.numRows(); }
    Ordinal numCols() const { return numCols_; }
    SizeType nnz() const { return (SizeType)graph.entries.extent(0); }
};

}  // namespace KokkosSparse
