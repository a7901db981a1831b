// sort.cuh -- stable LSD radix sort of (key, value) pairs, 8-bit digits.
//
// Per pass: per-tile digit histograms (digit-major), one exclusive scan over
// them, then a scatter in which every element's rank among equal digits of its
// tile follows tile order (warp match.any peers + per-warp digit counts), so
// equal keys keep their input order.  Used where the reference's result
// depends on processing order (rebalance scores) to reproduce its in-order
// semantics deterministically.
#pragma once
#include "jet_common.cuh"

namespace jetb {

static constexpr int RS_THREADS = 256;
static constexpr int RS_ITEMS = 8;
static constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
static constexpr int RS_BINS = 256;

template <class K>
__device__ __forceinline__ int rs_digit(K k, int shift) { return (int)((k >> shift) & (K)(RS_BINS - 1)); }

// First pass may read keys through a functor (value = element index).
template <class K, class GetKey>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(GetKey get, int64_t n, int shift, int64_t ntiles, uint32_t* hist) {
    __shared__ uint32_t h[RS_BINS];
    h[threadIdx.x] = 0;
    __syncthreads();
    int64_t base = (int64_t)blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ITEMS; r++) {
        int64_t i = base + (int64_t)r * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[rs_digit<K>(get(i), shift)], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

template <class K, class V, class GetKey, class GetVal>
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(GetKey get, GetVal getv, int64_t n, int shift, int64_t ntiles,
                                                           const uint32_t* offs, K* kout, V* vout) {
    __shared__ uint32_t cnt[RS_THREADS / 32][RS_BINS];
    __shared__ uint32_t run[RS_BINS];
    __shared__ uint32_t base_off[RS_BINS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    base_off[threadIdx.x] = offs[(int64_t)threadIdx.x * ntiles + blockIdx.x];
    run[threadIdx.x] = 0;
    int64_t tbase = (int64_t)blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ITEMS; r++) {
        for (int w = 0; w < RS_THREADS / 32; w++) cnt[w][threadIdx.x] = 0;
        __syncthreads();
        int64_t i = tbase + (int64_t)r * RS_THREADS + threadIdx.x;
        bool in = i < n;
        K key = in ? get(i) : (K)0;
        int d = in ? rs_digit<K>(key, shift) : RS_BINS;  // RS_BINS never matches a real digit
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int rank = __popc(peers & ((1u << lane) - 1));
        if (in && rank == 0) cnt[wid][d] = __popc(peers);
        __syncthreads();
        // exclusive prefix over warps for digit threadIdx.x
        {
            uint32_t acc = 0;
            int dd = threadIdx.x;
            for (int w = 0; w < RS_THREADS / 32; w++) { uint32_t c = cnt[w][dd]; cnt[w][dd] = acc; acc += c; }
            // acc = this round's total for digit dd
            __syncthreads();
            if (in) {
                uint32_t pos = base_off[d] + run[d] + cnt[wid][d] + rank;
                kout[pos] = key;
                vout[pos] = getv(i);
            }
            __syncthreads();
            run[dd] += acc;
        }
        __syncthreads();
    }
}

template <class T>
struct GetIndex {
    __device__ __forceinline__ T operator()(int64_t i) const { return (T)i; }
};

struct RadixScratch {
    DBuf<uint32_t> hist;
};

// Sorts n pairs by key bits [0, bits).  The first pass reads keys/values
// through functors; the result lands in (k0, v0) or (k1, v1) -- the return
// value says which (0 or 1).
template <class K, class V, class GetKey, class GetVal>
int radix_sort_pairs(GetKey get0, GetVal getv0, int64_t n, int bits, K* k0, V* v0, K* k1, V* v1, RadixScratch& rs,
                     ScanScratch& sc, cudaStream_t s) {
    if (n <= 0 || bits <= 0) return -1;
    int64_t ntiles = ceil_div<int64_t>(n, RS_TILE);
    int64_t hn = ntiles * RS_BINS;
    if (rs.hist.n < hn + 1) rs.hist.alloc(hn + 1024, s);
    int passes = (bits + 7) / 8;
    int cur = -1;  // -1: functor input
    for (int p = 0; p < passes; p++) {
        int shift = 8 * p;
        K* kd = (cur == 0) ? k1 : k0;
        V* vd = (cur == 0) ? v1 : v0;
        if (cur < 0) {
            k_rs_hist<K, GetKey><<<(unsigned)ntiles, RS_THREADS, 0, s>>>(get0, n, shift, ntiles, rs.hist.p); count_launch();
            JET_LAUNCH_CHECK();
            exclusive_scan_array<uint32_t>(rs.hist.p, hn, rs.hist.p, nullptr, sc, s);
            k_rs_scatter<K, V, GetKey, GetVal><<<(unsigned)ntiles, RS_THREADS, 0, s>>>(get0, getv0, n, shift, ntiles, rs.hist.p, kd, vd); count_launch();
        } else {
            K* ks = cur == 0 ? k0 : k1;
            V* vs = cur == 0 ? v0 : v1;
            k_rs_hist<K, GetArray<K>><<<(unsigned)ntiles, RS_THREADS, 0, s>>>(GetArray<K>{ks}, n, shift, ntiles, rs.hist.p); count_launch();
            JET_LAUNCH_CHECK();
            exclusive_scan_array<uint32_t>(rs.hist.p, hn, rs.hist.p, nullptr, sc, s);
            k_rs_scatter<K, V, GetArray<K>, GetArray<V>><<<(unsigned)ntiles, RS_THREADS, 0, s>>>(GetArray<K>{ks}, GetArray<V>{vs}, n, shift, ntiles, rs.hist.p, kd, vd); count_launch();
        }
        JET_LAUNCH_CHECK();
        cur = (kd == k0) ? 0 : 1;
    }
    return cur;
}

inline int bits_for(uint64_t maxval) {
    int b = 0;
    while (b < 64 && (maxval >> b) != 0) b++;
    return b;
}

}  // namespace jetb
