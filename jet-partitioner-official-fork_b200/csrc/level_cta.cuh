// level_cta.cuh -- the whole refinement loop of a small level in one CTA.
//
// For levels of at most CTA_MAX_N vertices the per-iteration work is a few
// microseconds of memory traffic, and a loop of separate kernel launches is
// bound by launch and dependency latency.  Here one 1024-thread block runs
// jet_refine's loop (src/jet_refiner.hpp:1094-1134) end to end: every phase
// is the same device function the grid kernels use, separated by
// __syncthreads instead of kernel boundaries, and the rebalance tail (bucket
// offsets, candidate order, eviction scores, destination draws) is done in
// shared memory.  Results are identical to the multi-kernel path.
#pragma once
#include "refine.cuh"

namespace jetb {

static constexpr int CTA_MAX_N = 16384;   // candidate sort buffer: CTA_MAX_N x 8 B in shared memory
static constexpr int64_t CTA_MAX_M = 262144;  // beyond this many entries one SM's bandwidth is the limit
static constexpr int CTA_MAX_K = 256;     // per-warp connectivity tables: 32 warps x k slots
static constexpr int CTA_THREADS = 1024;

template <class O>
struct LevelLists {
    const O* warp_list;
    O n_warp;
    const O* hub_list;
    O n_hub;
    int group;
};

// Exclusive scan of in[0..n) into out (may alias), over the block: each
// thread sums a contiguous run, one block scan of the run sums, then each
// thread writes its run's prefixes (one barrier round for any n).
template <class T>
__device__ __forceinline__ void block_scan_global(const T* in, T* out, int64_t n) {
    __shared__ T sw[32];
    const int64_t per = (n + blockDim.x - 1) / blockDim.x;
    const int64_t lo = (int64_t)threadIdx.x * per;
    const int64_t hi = lo + per < n ? lo + per : n;
    T s = 0;
    for (int64_t i = lo; i < hi; i++) s += in[i];
    T tot;
    T ex = block_exclusive_scan<T>(s, sw, tot);
    for (int64_t i = lo; i < hi; i++) {
        const T v = in[i];
        out[i] = ex;
        ex += v;
    }
    __syncthreads();
}

// Bucket offsets, candidates in (bucket, vertex) order and their eviction
// scores: the block-level form of sort_candidates + k_evict_sorted (+ the
// strong rebalance's cookie cutter and destination draws).
template <bool STRONG, class O, class E, class W>
__device__ __forceinline__ void d_reb_tail(RefArgs<O, E, W> a, RebArgs<O, W> rb, uint64_t* keys, int P, PhaseClock& pc) {
    __shared__ W sw[32];
    const O n = a.g.n;
    block_scan_global<W>(rb.buckets, rb.boff, (int64_t)rb.t_minibuckets + 1);
    pc.mark(PH_REB_SCAN);
    if (rb.queue) {
        // only the candidates whose in-bucket order matters are sorted (they
        // fit: at most n <= P of them)
        __shared__ O s_count;
        __shared__ int s_fb;
        d_reb_classify<STRONG, O, E, W>(a, rb, threadIdx.x, blockDim.x);
        __syncthreads();
        if (threadIdx.x == 0) {
            s_count = a.dev->nord;
            s_fb = a.dev->reb_fb;
            a.dev->nord_last = s_count;
            a.dev->reb_fb_taken = s_fb;
            a.dev->nord = 0;
            a.dev->reb_fb = 0;
            if (s_fb) a.dev->nmoves = 0;  // the full sort below decides every move again
        }
        __syncthreads();
        pc.mark(PH_REB_SORT);
        if (!s_fb) {
            d_reb_queue_tail<STRONG, O, E, W>(a, rb, s_count, keys, P, &pc);
            return;
        }
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        uint64_t key = ~0ull;
        if (i < n) {
            O b = rb.bid[i];
            key = ((uint64_t)(b < 0 ? rb.none_key : (uint32_t)b) << 32) | (uint32_t)i;
        }
        keys[i] = key;
    }
    if (STRONG) for (int p = threadIdx.x; p < a.k; p += blockDim.x) rb.evict_adjust[p] = 0;
    __syncthreads();
    block_sort_keys<uint64_t>(keys, P);
    pc.mark(PH_REB_SORT);
    W carry = 0;
    for (int base = 0; base < (int)n; base += blockDim.x) {
        int q = base + threadIdx.x;
        uint32_t key = q < (int)n ? (uint32_t)(keys[q] >> 32) : rb.none_key;
        bool cand = key != rb.none_key;
        O i = cand ? (O)(uint32_t)(keys[q] & 0xffffffffu) : 0;
        W w = cand ? a.g.vw[i] : (W)0;
        W tot;
        W ex = block_exclusive_scan<W>(w, sw, tot);
        bool take = false;
        if (cand) {
            O b = (O)key;
            part_t p = a.part[i];
            O begin = (O)p * rb.width;
            W within = carry + ex - bucket_start<O, W>(rb, b);
            if (STRONG) rb.score[i] = within;
            W score = within + bucket_pos<O, W>(rb, b) - bucket_pos<O, W>(rb, begin);
            W limit = a.sizes[p] - rb.size_max;
            if (score < limit) {
                take = true;
                if (STRONG && score + w >= limit) rb.evict_adjust[p] = score + w;
            }
        }
        O s = warp_append(&a.dev->nmoves, take);
        if (take) a.moves[s] = i;
        carry += tot;
    }
    __syncthreads();
    pc.mark(PH_REB_EVICT);
    if (STRONG) {
        d_cookie<O, E, W>(a, rb);
        __syncthreads();
        pc.mark(PH_COOKIE);
        d_strong_first<O, E, W>(a, rb);
        __syncthreads();
        pc.mark(PH_STRONG_FIRST);
        d_strong_redraw<O, E, W>(a, rb);
        __syncthreads();
        pc.mark(PH_REDRAW);
    }
}

template <class O, class E, class W>
__device__ __forceinline__ void cta_zero_buckets(const RebArgs<O, W>& rb) {
    int64_t m = (int64_t)rb.t_minibuckets + 1 + rb.width;
    for (int64_t i = threadIdx.x; i < m; i += blockDim.x) rb.buckets[i] = 0;
    __syncthreads();
}

// Where the single-CTA loop keeps the level's mutable state.  The loop is
// bound by the latency of its dependent accesses, phase after phase; arrays
// placed in shared memory (byte offsets past the phase scratch at offset 0)
// are read and written there for the whole loop instead of through L2.
// NO_SMEM leaves an array in global memory.  Only the single CTA of the
// launch touches these arrays, so moving them cannot change a result.
static constexpr uint32_t NO_SMEM = 0xffffffffu;
struct CtaSmemPlan {
    uint32_t part, dest, csize, dest_cache, save_gain, pregain, lock, mark;
    uint32_t cand, moves, bid, score, sizes, dev, ctl, slots, buckets, boff;
    int64_t nslots, nbuckets;
    size_t total;  // dynamic shared memory the launch needs
};

template <class T>
__device__ __forceinline__ void cta_place(unsigned char* base, uint32_t off, T*& ptr, int64_t count) {
    if (off == NO_SMEM) return;
    T* dst = (T*)(base + off);
    const T* src = ptr;
    for (int64_t i = threadIdx.x; i < count; i += blockDim.x) dst[i] = src[i];
    ptr = dst;
}

template <class O, class E, class W>
__global__ void __launch_bounds__(CTA_THREADS, 1)
k_level_cta(RefArgs<O, E, W> a, LevelLists<O> li, RebArgs<O, W> rbw, RebArgs<O, W> rbs, Ctl<W>* c, part_t* best_part,
            W* sizes_best, int P, int max_iters, CtaSmemPlan plan) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* keys = (uint64_t*)smem_raw;
    __shared__ int s_mode, s_more, s_copy;
    const O n = a.g.n;
    Ctl<W>* const c_global = c;
    RefDev<O, W>* const dev_global = a.dev;
    {
        // move the planned arrays into shared memory
        cta_place(smem_raw, plan.part, a.part, n);
        cta_place(smem_raw, plan.dest, a.dest, n);
        cta_place(smem_raw, plan.csize, a.csize, n);
        cta_place(smem_raw, plan.dest_cache, a.dest_cache, n);
        cta_place(smem_raw, plan.save_gain, a.save_gain, n);
        cta_place(smem_raw, plan.pregain, a.pregain, n);
        cta_place(smem_raw, plan.lock, a.lock, n);
        cta_place(smem_raw, plan.mark, a.mark, n);
        cta_place(smem_raw, plan.cand, a.cand, n);
        cta_place(smem_raw, plan.moves, a.moves, n);
        cta_place(smem_raw, plan.sizes, a.sizes, a.k);
        cta_place(smem_raw, plan.dev, a.dev, 1);
        cta_place(smem_raw, plan.ctl, c, 1);
        cta_place(smem_raw, plan.slots, a.slots, plan.nslots);
        cta_place(smem_raw, plan.bid, rbw.bid, n);
        cta_place(smem_raw, plan.score, rbw.score, n);
        cta_place(smem_raw, plan.buckets, rbw.buckets, plan.nbuckets);
        cta_place(smem_raw, plan.boff, rbw.boff, plan.nbuckets);
        rbs.bid = rbw.bid; rbs.score = rbw.score; rbs.buckets = rbw.buckets; rbs.boff = rbw.boff;
        if (plan.ctl != NO_SMEM) a.filter = &c->filter;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ctl_begin_logic(c);
        s_mode = c->mode;
        s_more = c->more;
    }
    __syncthreads();
    PhaseClock pc(a.pclk, 0, threadIdx.x == 0);
    int iters = 0;
    while (s_more) {
        const int mode = s_mode;
        if (mode == MODE_LP) {
            d_lp_select_thread<O, E, W>(a);
            d_lp_select_warp<O, E, W>(a, li.warp_list, li.n_warp);
            d_lp_select_warp<O, E, W>(a, li.hub_list, li.n_hub);
            __syncthreads();
            pc.mark(PH_LP_SELECT);
            switch (li.group) {
                case 4: d_afterburn<4, O, E, W>(a); break;
                case 8: d_afterburn<8, O, E, W>(a); break;
                case 16: d_afterburn<16, O, E, W>(a); break;
                default: d_afterburn<32, O, E, W>(a); break;
            }
            __syncthreads();
            pc.mark(PH_AFTERBURN);
            d_afterburn_hub<O, E, W>(a);
            __syncthreads();
            pc.mark(PH_AFTERBURN_HUB);
        } else if (mode == MODE_WEAK) {
            cta_zero_buckets<O, E, W>(rbw);
            d_weak_prep<O, E, W>(a, rbw);
            __syncthreads();
            pc.mark(PH_REB_PREP);
            d_weak_select_thread<O, E, W>(a, rbw);
            d_weak_select_warp<O, E, W>(a, rbw, li.warp_list, li.n_warp);
            d_weak_select_warp<O, E, W>(a, rbw, li.hub_list, li.n_hub);
            __syncthreads();
            pc.mark(PH_REB_SELECT);
            d_reb_tail<false, O, E, W>(a, rbw, keys, P, pc);
        } else {
            cta_zero_buckets<O, E, W>(rbs);
            d_strong_prep<O, E, W>(a, rbs);
            __syncthreads();
            pc.mark(PH_REB_PREP);
            d_strong_score_thread<O, E, W>(a, rbs);
            d_strong_score_warp<O, E, W>(a, rbs, li.warp_list, li.n_warp);
            d_strong_score_warp<O, E, W>(a, rbs, li.hub_list, li.n_hub);
            __syncthreads();
            pc.mark(PH_REB_SELECT);
            d_reb_tail<true, O, E, W>(a, rbs, keys, P, pc);
        }
        // perform_moves (src/jet_refiner.hpp:905-955)
        d_apply_moves<O, E, W>(a, 0);
        __syncthreads();
        pc.mark(PH_APPLY);
        switch (li.group) {
            case 4: d_update_small<4, false, O, E, W>(a); break;
            case 8: d_update_small<8, false, O, E, W>(a); break;
            case 16: d_update_small<16, false, O, E, W>(a); break;
            default: d_update_small<32, false, O, E, W>(a); break;
        }
        d_update_small_hub<false, O, E, W>(a);
        __syncthreads();
        pc.mark(PH_UPDATE_SUB);
        switch (li.group) {
            case 4: d_update_small<4, true, O, E, W>(a); d_mark_neighbors<4, O, E, W>(a); break;
            case 8: d_update_small<8, true, O, E, W>(a); d_mark_neighbors<8, O, E, W>(a); break;
            case 16: d_update_small<16, true, O, E, W>(a); d_mark_neighbors<16, O, E, W>(a); break;
            default: d_update_small<32, true, O, E, W>(a); d_mark_neighbors<32, O, E, W>(a); break;
        }
        d_update_small_hub<true, O, E, W>(a);
        d_mark_neighbors_hub<O, E, W>(a);
        __syncthreads();
        pc.mark(PH_UPDATE_ADD);
        d_conn_warp<O, E, W>(a, nullptr, n, 1, &a.dev->large);  // update_large: rebuild marked rows
        __syncthreads();
        pc.mark(PH_REBUILD);
        d_cut_after<O, E, W>(a);
        __syncthreads();
        pc.mark(PH_CUT);
        W mx = block_max_sizes<W>(a.sizes, a.k);
        if (threadIdx.x == 0) {
            ctl_end_logic<O, W>(c, a.dev, mx);
            s_mode = c->mode;
            s_more = c->more && ++iters < max_iters;
            s_copy = c->copy;
            if (c->more && iters >= max_iters) atomicOr(&a.dev->err, ERRF_SPIN);
        }
        __syncthreads();
        pc.mark(PH_CTL);
        if (s_copy) {
            for (int64_t i = threadIdx.x; i < n; i += blockDim.x) best_part[i] = a.part[i];
            for (int p = threadIdx.x; p < a.k; p += blockDim.x) sizes_best[p] = a.sizes[p];
        }
        __syncthreads();
        pc.mark(PH_COPY);
    }
    pc.flush();
    // the host reads the control state and the error flags after the level
    if (threadIdx.x == 0) {
        if (plan.ctl != NO_SMEM) *c_global = *c;
        if (plan.dev != NO_SMEM && a.dev->err) atomicOr(&dev_global->err, a.dev->err);
    }
}

// Places the loop's arrays in shared memory, most latency-critical first,
// while they fit beside the phase scratch; the rest stay in global memory.
template <class O, class W>
inline CtaSmemPlan plan_cta_smem(int64_t n, int64_t nslots, int64_t nbuckets, int k, size_t scratch, size_t budget,
                                 bool enable) {
    CtaSmemPlan pl;
    uint32_t* fields[] = {&pl.part, &pl.dest, &pl.csize, &pl.dest_cache, &pl.save_gain, &pl.pregain, &pl.lock, &pl.mark,
                          &pl.cand, &pl.moves, &pl.bid, &pl.score, &pl.sizes, &pl.dev, &pl.ctl, &pl.slots,
                          &pl.buckets, &pl.boff};
    for (uint32_t* f : fields) *f = NO_SMEM;
    pl.nslots = nslots;
    pl.nbuckets = nbuckets;
    pl.total = scratch;
    if (!enable) return pl;
    size_t off = (scratch + 15) & ~(size_t)15;
    auto take = [&](uint32_t& f, size_t bytes) {
        size_t end = off + ((bytes + 15) & ~(size_t)15);
        if (end > budget) return;
        f = (uint32_t)off;
        off = end;
    };
    take(pl.dev, sizeof(RefDev<O, W>));
    take(pl.ctl, sizeof(Ctl<W>));
    take(pl.sizes, (size_t)k * sizeof(W));
    take(pl.part, n * sizeof(part_t));
    take(pl.dest, n * sizeof(part_t));
    take(pl.csize, n * sizeof(part_t));
    take(pl.dest_cache, n * sizeof(part_t));
    take(pl.lock, n);
    take(pl.mark, n);
    take(pl.pregain, n * sizeof(W));
    take(pl.save_gain, n * sizeof(W));
    take(pl.slots, nslots * sizeof(Slot<W>));
    take(pl.cand, n * sizeof(O));
    take(pl.moves, n * sizeof(O));
    take(pl.bid, n * sizeof(O));
    take(pl.score, n * sizeof(W));
    take(pl.buckets, nbuckets * sizeof(W));
    take(pl.boff, nbuckets * sizeof(W));
    pl.total = off;
    return pl;
}


template <class O, class W>
constexpr size_t level_cta_smem(int P, int k) {
    size_t sort_b = (size_t)P * 8;
    size_t conn_b = (((size_t)(CTA_THREADS / 32) * k * sizeof(part_t) + 15) & ~(size_t)15) + (size_t)(CTA_THREADS / 32) * k * sizeof(W);
    return sort_b > conn_b ? sort_b : conn_b;
}

}  // namespace jetb
