// prof.cuh -- device-side counts for the profiling pass.
//
// When kernel-class timing is on (jet_prof_enable) and a level runs on the
// host-driven loop, every refinement kernel class of an iteration is
// bracketed by CUDA events, and these kernels -- launched outside the
// brackets -- count what the algorithmic byte model of each class needs:
// uncached vertices and their table sizes (LP select), candidates and their
// summed degree (afterburner), moves and their summed degree (moves, table
// updates, cut change), rows marked for a rebuild with their degree and
// capacity (update_large).  Nothing here runs when timing is off.
#pragma once
#include "refine.cuh"

namespace jetb {

struct ProfCounts {
    unsigned long long uncached, size_uncached, csize_all;
    unsigned long long cand, cand_deg;
    unsigned long long moves, moves_deg;
    unsigned long long marked, marked_deg, marked_cap;
    unsigned long long reb_cand;  // rebalance candidates (vertices with a bucket)
};

// Block-wide sum of up to three values, one atomic each per block.
__device__ __forceinline__ void prof_block_add(unsigned long long a, unsigned long long b, unsigned long long c,
                                               unsigned long long* pa, unsigned long long* pb, unsigned long long* pc) {
    __shared__ unsigned long long s[3][32];
    for (int m = 16; m > 0; m >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, m);
        b += __shfl_xor_sync(0xffffffffu, b, m);
        c += __shfl_xor_sync(0xffffffffu, c, m);
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) { s[0][w] = a; s[1][w] = b; s[2][w] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long ta = 0, tb = 0, tc = 0;
        for (int i = 0; i < nw; i++) { ta += s[0][i]; tb += s[1][i]; tc += s[2][i]; }
        if (ta && pa) atomicAdd(pa, ta);
        if (tb && pb) atomicAdd(pb, tb);
        if (tc && pc) atomicAdd(pc, tc);
    }
}

// Before LP select: vertices without a cached destination and the sizes of
// their tables, and the summed table sizes of all vertices.
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_prof_select(RefArgs<O, E, W> a, ProfCounts* c) {
    unsigned long long u = 0, su = 0, sa = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)a.g.n; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long sz = (unsigned long long)a.csize[i];
        sa += sz;
        if (a.dest_cache[i] == NULL_PART) { u++; su += sz; }
    }
    prof_block_add(u, su, sa, &c->uncached, &c->size_uncached, &c->csize_all);
}

// Count and summed degree of list[0 .. *count).
template <class O, class E>
__global__ void __launch_bounds__(BLOCK) k_prof_list(const E* row, const O* list, const O* count, unsigned long long* cnt,
                                                     unsigned long long* deg) {
    const int64_t n = (int64_t)*count;
    unsigned long long d = 0;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        O i = list[x];
        d += (unsigned long long)(row[i + 1] - row[i]);
    }
    prof_block_add(blockIdx.x == 0 && threadIdx.x == 0 ? (unsigned long long)n : 0ull, d, 0ull, cnt, deg, nullptr);
}

// Rows marked for an update_large rebuild: count, summed degree, capacity.
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_prof_marked(RefArgs<O, E, W> a, ProfCounts* c) {
    unsigned long long m = 0, d = 0, cap = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)a.g.n; i += (int64_t)gridDim.x * blockDim.x) {
        if (a.mark[i]) {
            m++;
            d += (unsigned long long)(a.g.row[i + 1] - a.g.row[i]);
            cap += (unsigned long long)(a.coff[i + 1] - a.coff[i]);
        }
    }
    prof_block_add(m, d, cap, &c->marked, &c->marked_deg, &c->marked_cap);
}

// Rebalance candidates: vertices given a bucket by the selection.
template <class O>
__global__ void __launch_bounds__(BLOCK) k_prof_bid(const O* bid, int64_t n, unsigned long long* cnt) {
    unsigned long long c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) c += bid[i] >= 0;
    prof_block_add(c, 0ull, 0ull, cnt, nullptr, nullptr);
}

}  // namespace jetb
