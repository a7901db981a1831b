// graph.cuh -- device graph views, hierarchy levels and per-level degree bins.
#pragma once
#include "jet_common.cuh"

namespace jetb {

// Read-only view of one CSR level (both edge directions stored, no loops).
template <class O, class E, class W>
struct GView {
    O n;
    E m;
    const E* row;
    const O* adj;
    const W* val;
    const W* vw;
};

// One level of the coarsening hierarchy (src/contract.hpp:85-91).  The finest
// level borrows the caller's arrays; coarser levels own theirs.
template <class O, class E, class W>
struct Level {
    O n = 0;
    E m = 0;
    const E* row = nullptr;
    const O* adj = nullptr;
    const W* val = nullptr;
    const W* vw = nullptr;
    DBuf<E> own_row;
    DBuf<O> own_adj;
    DBuf<W> own_val;
    DBuf<W> own_vw;
    DBuf<O> map;           // previous (finer) level -> this level
    bool uniform = false;  // all edge weights equal (finest level only)
    // degree bins (src/contract.hpp:383, src/jet_refiner.hpp:985 choose by
    // average degree; here every vertex is classed by its own degree)
    DBuf<O> warp_list;     // THREAD_DEG < deg <= HUB_DEG
    DBuf<O> hub_list;      // deg > HUB_DEG
    O n_warp = 0, n_hub = 0;
    int group = 4;         // threads per vertex for edge-parallel kernels
    E max_deg = 0;
    GView<O, E, W> view() const { return GView<O, E, W>{n, m, row, adj, val, vw}; }
};

template <class O, class E>
__global__ void k_bin_degrees(O n, const E* row, O* warp_list, O* n_warp, O* hub_list, O* n_hub, E* max_deg) {
    E local_max = 0;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t rounds = ceil_div<int64_t>((int64_t)n, stride);
    for (int64_t r = 0; r < rounds; r++) {
        int64_t i = start + r * stride;
        E d = 0;
        if (i < n) d = row[i + 1] - row[i];
        if (d > local_max) local_max = d;
        O s = warp_append(n_warp, i < n && d > THREAD_DEG && d <= HUB_DEG);
        if (s >= 0) warp_list[s] = (O)i;
        O h = warp_append(n_hub, i < n && d > HUB_DEG);
        if (h >= 0) hub_list[h] = (O)i;
    }
    for (int o = 16; o > 0; o >>= 1) {
        E y = __shfl_xor_sync(0xffffffffu, local_max, o);
        if (y > local_max) local_max = y;
    }
    if ((threadIdx.x & 31) == 0 && local_max > 0) {
        if (sizeof(E) == 4) atomicMax((int*)max_deg, (int)local_max);
        else atomicMax((unsigned long long*)max_deg, (unsigned long long)local_max);
    }
}

}  // namespace jetb
