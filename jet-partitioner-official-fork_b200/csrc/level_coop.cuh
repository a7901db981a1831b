// level_coop.cuh -- the refinement loop of a level as one persistent grid
// kernel, in two launch forms: one thread-block cluster of 8-16 CTAs whose
// phases meet at the hardware cluster barrier (mid-size levels), or a
// cooperative launch of one 1024-thread CTA per SM with a software grid
// barrier.
//
// Same phases and results as the single-CTA loop (level_cta.cuh) and the
// multi-kernel path; phases are separated by a grid barrier instead of kernel
// boundaries, and the order-dependent parts of rebalancing (bucket offsets,
// candidate order, eviction scores) use grid-level scans and a stable radix
// sort whose blocks own contiguous ranges.  The launch is cooperative, so all
// CTAs are resident; every barrier wait is still bounded and, on timeout,
// raises ERRF_SPIN and makes every CTA leave the loop.
#pragma once
#include "level_cta.cuh"

namespace jetb {

struct GridBar {
    unsigned int count;
    unsigned int gen;
    int abort;
    unsigned int cut_done;       // blocks done with the cut change this iteration
    int64_t nmarked;             // rows queued for rebuild this iteration
};

// Returns false when the loop must stop (a barrier timed out somewhere).
// A wait gives up after spin_cap polls (2^26, about 4 s, by default).
//
// Thread 0 of each block arrives with a release-acquire atomic add on the
// arrival counter: the block's earlier writes, ordered before it by
// __syncthreads, are released with it.  The last block to arrive resets the
// counter and publishes the next generation with a release store; the others
// poll the generation with acquire loads, so every block's writes are
// visible to every block after the barrier.
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool grid_sync(GridBar* gb, int* err, long long spin_cap = (1ll << 26)) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int g = ld_acquire_gpu(&gb->gen);
        unsigned int arrived = atom_add_acq_rel_gpu(&gb->count, 1u) + 1u;
        if (arrived == gridDim.x) {
            gb->count = 0;  // ordered before the release below; nobody arrives again before it
            st_release_gpu(&gb->gen, g + 1u);
        } else {
            long long spins = 0;
            while (ld_acquire_gpu(&gb->gen) == g) {
                if ((spins & 63) == 63 && ((volatile int*)&gb->abort)[0]) break;
                if (++spins > spin_cap) {
                    atomicOr(err, ERRF_SPIN);
                    atomicExch(&gb->abort, 1);
                    break;
                }
                if (spins > 256) __nanosleep(32);
            }
        }
    }
    __syncthreads();
    return ((volatile int*)&gb->abort)[0] == 0;
}

// Barrier between phases: a hardware cluster barrier when the whole launch is
// one thread-block cluster (CL), else the bounded software grid barrier.
// barrier.cluster with release/acquire orders every memory access of the
// cluster's threads, global memory included.
template <bool CL>
__device__ __forceinline__ bool level_sync(GridBar* gb, int* err) {
    if constexpr (CL) {
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
        return true;
    } else {
        return grid_sync(gb, err);
    }
}

// Grid-wide exclusive scan of get(0..n) into out: each block owns a
// contiguous range; block offsets come from the per-block sums.
template <bool CL, class T, class Get>
__device__ __forceinline__ bool grid_scan(Get get, int64_t n, T* out, T* block_sums, GridBar* gb, int* err) {
    __shared__ T sw[32];
    __shared__ T s_off;
    const int64_t chunk = ceil_div<int64_t>(n, (int64_t)gridDim.x);
    const int64_t lo = chunk * blockIdx.x, hi = lo + chunk < n ? lo + chunk : n;
    T s = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += get(i);
    T tot;
    block_exclusive_scan<T>(s, sw, tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
    if (!level_sync<CL>(gb, err)) return false;
    // offset of this block: sum of earlier blocks' sums
    T o = 0;
    for (unsigned b = threadIdx.x; b < blockIdx.x; b += blockDim.x) o += block_sums[b];
    T otot;
    block_exclusive_scan<T>(o, sw, otot);
    if (threadIdx.x == 0) s_off = otot;
    __syncthreads();
    T carry = s_off;
    for (int64_t base = lo; base < hi; base += blockDim.x) {
        int64_t i = base + threadIdx.x;
        T v = i < hi ? get(i) : T(0);
        T t2;
        T ex = block_exclusive_scan<T>(v, sw, t2);
        if (i < hi) out[i] = carry + ex;
        carry += t2;
    }
    return level_sync<CL>(gb, err);
}

// One stable LSD pass over 8 bits: keys/values from the functors into
// (kd, vd).  Blocks own contiguous ranges, processed in order in tiles of
// blockDim elements, so equal digits keep their input order.
template <bool CL, class K, class V, class GetK, class GetV>
__device__ __forceinline__ bool grid_radix_pass(GetK getk, GetV getv, int64_t n, int shift, K* kd, V* vd, uint32_t* hist,
                                                uint32_t (*cnt)[RS_BINS], GridBar* gb, int* err) {
    __shared__ uint32_t base_off[RS_BINS];
    __shared__ uint32_t run[RS_BINS];
    __shared__ uint32_t tile_tot[RS_BINS];
    __shared__ uint32_t sw32[32];
    const int nb = gridDim.x;
    const int64_t chunk = ceil_div<int64_t>(n, (int64_t)nb);
    const int64_t lo = chunk * blockIdx.x, hi = lo + chunk < n ? lo + chunk : n;
    for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) base_off[d] = 0;
    __syncthreads();
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&base_off[rs_digit<K>(getk(i), shift)], 1u);
    __syncthreads();
    for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) hist[(int64_t)d * nb + blockIdx.x] = base_off[d];
    if (!level_sync<CL>(gb, err)) return false;
    // start of each digit for this block: every smaller digit + this digit in earlier blocks
    {
        const int d = threadIdx.x;  // blockDim >= RS_BINS
        uint32_t tot_d = 0, before = 0;
        if (d < RS_BINS)
            for (int b = 0; b < nb; b++) {
                uint32_t v = hist[(int64_t)d * nb + b];
                tot_d += v;
                if (b < (int)blockIdx.x) before += v;
            }
        uint32_t all;
        uint32_t ex = block_exclusive_scan<uint32_t>(d < RS_BINS ? tot_d : 0u, sw32, all);
        if (d < RS_BINS) { base_off[d] = ex + before; run[d] = 0; }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t base = lo; base < hi; base += blockDim.x) {
        for (int w = 0; w < nw; w++)
            for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) cnt[w][d] = 0;
        __syncthreads();
        int64_t i = base + threadIdx.x;
        bool in = i < hi;
        K key = in ? getk(i) : (K)0;
        int dg = in ? rs_digit<K>(key, shift) : RS_BINS;
        unsigned peers = __match_any_sync(0xffffffffu, dg);
        int rank = __popc(peers & ((1u << lane) - 1));
        if (in && rank == 0) cnt[wid][dg] = __popc(peers);
        __syncthreads();
        for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) {
            uint32_t acc = 0;
            for (int w = 0; w < nw; w++) { uint32_t c = cnt[w][d]; cnt[w][d] = acc; acc += c; }
            tile_tot[d] = acc;
        }
        __syncthreads();
        if (in) {
            uint32_t pos = base_off[dg] + run[dg] + cnt[wid][dg] + rank;
            kd[pos] = key;
            vd[pos] = getv(i);
        }
        __syncthreads();
        for (int d = threadIdx.x; d < RS_BINS; d += blockDim.x) run[d] += tile_tot[d];
        __syncthreads();
    }
    return level_sync<CL>(gb, err);
}

template <class O, class E, class W>
struct CoopScratch {
    GridBar* bar;
    W* wsum;             // per-block sums for W scans
    uint32_t* hist;      // 256 x gridDim
    uint32_t* sk0;       // sort buffers (n)
    uint32_t* sk1;
    O* sv0;
    O* sv1;
    W* wpre;             // prefix of candidate weights in sorted order (n)
    O* marked;           // rows to rebuild after a large move set (n)
    int qcap;            // queued candidates block 0 can order in its dynamic shared memory
    int64_t boff_cap;    // bucket offsets each block can keep in shared memory (0: none)
    int64_t boff_off;    // their byte offset: past the queue keys and the radix counters
};

// Rebalance tail over the grid (sort_candidates + k_evict_sorted [+ strong]).
template <bool CL, bool STRONG, class O, class E, class W>
__device__ __forceinline__ bool coop_reb_tail(RefArgs<O, E, W>& a, RebArgs<O, W>& rb, CoopScratch<O, E, W>& cs, int bits,
                                              PhaseClock& pc) {
    int* err = &a.dev->err;
    const int64_t n = a.g.n;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if ((int64_t)rb.t_minibuckets + 1 <= cs.boff_cap) {
        // every block scans the bucket totals into its own shared copy of the
        // offsets (no grid barrier); all later readers in this rebalance
        // (classification, ordering, eviction, cookie cutter, destinations)
        // read the copy of their own block
        W* boff_s = (W*)(smem_raw + cs.boff_off);
        block_scan_global<W>(rb.buckets, boff_s, (int64_t)rb.t_minibuckets + 1);
        rb.boff = boff_s;
    } else if (!grid_scan<CL, W>(GetArray<W>{rb.buckets}, (int64_t)rb.t_minibuckets + 1, rb.boff, cs.wsum, cs.bar, err)) {
        return false;
    }
    pc.mark(PH_REB_SCAN);
    if (rb.queue) {
        // the grid classifies; block 0 orders the queue (when it fits) and
        // finishes the rebalance while the other blocks wait at the barrier
        d_reb_classify<STRONG, O, E, W>(a, rb, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
        if (!level_sync<CL>(cs.bar, err)) return false;
        pc.mark(PH_REB_SORT);
        volatile RefDev<O, W>* vd = a.dev;
        const O count = vd->nord;
        const int fb = vd->reb_fb || count > (O)cs.qcap;
        if (!fb && blockIdx.x == 0) d_reb_queue_tail<STRONG, O, E, W>(a, rb, count, (uint64_t*)smem_raw, cs.qcap, &pc);
        // every block has read the queue state before block 0 resets it
        if (!level_sync<CL>(cs.bar, err)) return false;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.dev->nord_last = count;
            a.dev->reb_fb_taken = fb;
            a.dev->nord = 0;
            a.dev->reb_fb = 0;
            if (fb) a.dev->nmoves = 0;  // the full sort below decides every move again
        }
        if (!fb) return true;
    }
    uint32_t(*cnt)[RS_BINS] = (uint32_t(*)[RS_BINS])smem_raw;  // 32 x 256 counters (dynamic shared memory)
    // stable sort of (bucket id, vertex) pairs
    int passes = (bits + 7) / 8;
    uint32_t* kin = nullptr;
    O* vin = nullptr;
    for (int p = 0; p < passes; p++) {
        uint32_t* kd = (p & 1) ? cs.sk1 : cs.sk0;
        O* vd = (p & 1) ? cs.sv1 : cs.sv0;
        bool ok;
        if (p == 0)
            ok = grid_radix_pass<CL, uint32_t, O>(GetBidKey<O>{rb.bid, rb.none_key}, GetIndex<O>{}, n, 0, kd, vd, cs.hist, cnt, cs.bar, err);
        else
            ok = grid_radix_pass<CL, uint32_t, O>(GetArray<uint32_t>{kin}, GetArray<O>{vin}, n, 8 * p, kd, vd, cs.hist, cnt, cs.bar, err);
        if (!ok) return false;
        kin = kd;
        vin = vd;
    }
    pc.mark(PH_REB_SORT);
    rb.skey = kin;
    rb.sval = vin;
    if (!grid_scan<CL, W>(GetSortedWeight<O, W>{kin, vin, a.g.vw, rb.none_key}, n, cs.wpre, cs.wsum, cs.bar, err)) return false;
    pc.mark(PH_WEIGHT_SCAN);
    rb.wpre = cs.wpre;
    if (STRONG) {
        for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.k; p += gridDim.x * blockDim.x) rb.evict_adjust[p] = 0;
        if (!level_sync<CL>(cs.bar, err)) return false;
    }
    if (STRONG) d_evict_sorted<true, O, E, W>(a, rb);
    else d_evict_sorted<false, O, E, W>(a, rb);
    if (!level_sync<CL>(cs.bar, err)) return false;
    pc.mark(PH_REB_EVICT);
    if (STRONG) {
        if (blockIdx.x == 0) d_cookie<O, E, W>(a, rb);
        if (!level_sync<CL>(cs.bar, err)) return false;
        pc.mark(PH_COOKIE);
        d_strong_first<O, E, W>(a, rb);
        if (!level_sync<CL>(cs.bar, err)) return false;
        pc.mark(PH_STRONG_FIRST);
        if (blockIdx.x == 0) d_strong_redraw<O, E, W>(a, rb);
        if (!level_sync<CL>(cs.bar, err)) return false;
        pc.mark(PH_REDRAW);
    }
    return true;
}

template <class O, class E, class W>
__device__ __forceinline__ void coop_zero(W* p, int64_t m) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) p[i] = 0;
}

template <bool CL, class O, class E, class W>
__global__ void __launch_bounds__(CTA_THREADS, 1)
k_level_coop(RefArgs<O, E, W> a, LevelLists<O> li, RebArgs<O, W> rbw, RebArgs<O, W> rbs, Ctl<W>* c, part_t* best_part,
             W* sizes_best, CoopScratch<O, E, W> cs, int bits, int max_iters) {
    int* err = &a.dev->err;
    const O n = a.g.n;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl_begin_logic(c);
    if (!level_sync<CL>(cs.bar, err)) return;
    PhaseClock pc(a.pclk, CL ? 2 * PHASE_SLOTS : 4 * PHASE_SLOTS, blockIdx.x == 0 && threadIdx.x == 0);
    while (true) {
        const int more = ((volatile Ctl<W>*)c)->more;
        const int mode = ((volatile Ctl<W>*)c)->mode;
        if (!more) break;
        if (mode == MODE_LP) {
            d_lp_select_thread<O, E, W>(a);
            d_lp_select_warp<O, E, W>(a, li.warp_list, li.n_warp);
            d_lp_select_warp<O, E, W>(a, li.hub_list, li.n_hub);
            if (!level_sync<CL>(cs.bar, err)) return;
            pc.mark(PH_LP_SELECT);
            switch (li.group) {
                case 4: d_afterburn<4, O, E, W>(a); break;
                case 8: d_afterburn<8, O, E, W>(a); break;
                case 16: d_afterburn<16, O, E, W>(a); break;
                default: d_afterburn<32, O, E, W>(a); break;
            }
            if (!level_sync<CL>(cs.bar, err)) return;
            pc.mark(PH_AFTERBURN);
            if (li.n_hub > 0) {
                d_afterburn_hub<O, E, W>(a);
                if (!level_sync<CL>(cs.bar, err)) return;
                pc.mark(PH_AFTERBURN_HUB);
            }
        } else {
            RebArgs<O, W>& rb = mode == MODE_WEAK ? rbw : rbs;
            // bucket totals cleared while block 0 lists the parts (neither
            // reads what the other writes)
            coop_zero<O, E, W>(rb.buckets, (int64_t)rb.t_minibuckets + 1 + rb.width);
            if (blockIdx.x == 0) {
                if (mode == MODE_WEAK) d_weak_prep<O, E, W>(a, rb);
                else d_strong_prep<O, E, W>(a, rb);
            }
            if (!level_sync<CL>(cs.bar, err)) return;
            pc.mark(PH_REB_PREP);
            if (mode == MODE_WEAK) {
                d_weak_select_thread<O, E, W>(a, rb);
                d_weak_select_warp<O, E, W>(a, rb, li.warp_list, li.n_warp);
                d_weak_select_warp<O, E, W>(a, rb, li.hub_list, li.n_hub);
            } else {
                d_strong_score_thread<O, E, W>(a, rb);
                d_strong_score_warp<O, E, W>(a, rb, li.warp_list, li.n_warp);
                d_strong_score_warp<O, E, W>(a, rb, li.hub_list, li.n_hub);
            }
            if (!level_sync<CL>(cs.bar, err)) return;
            pc.mark(PH_REB_SELECT);
            bool ok = mode == MODE_WEAK ? coop_reb_tail<CL, false, O, E, W>(a, rb, cs, bits, pc)
                                        : coop_reb_tail<CL, true, O, E, W>(a, rb, cs, bits, pc);
            if (!ok) return;
        }
        // perform_moves (src/jet_refiner.hpp:905-955)
        d_apply_moves<O, E, W>(a, 0);
        if (!level_sync<CL>(cs.bar, err)) return;
        pc.mark(PH_APPLY);
        switch (li.group) {
            case 4: d_update_small<4, false, O, E, W>(a); break;
            case 8: d_update_small<8, false, O, E, W>(a); break;
            case 16: d_update_small<16, false, O, E, W>(a); break;
            default: d_update_small<32, false, O, E, W>(a); break;
        }
        d_update_small_hub<false, O, E, W>(a);
        if (!level_sync<CL>(cs.bar, err)) return;
        pc.mark(PH_UPDATE_SUB);
        switch (li.group) {
            case 4: d_update_small<4, true, O, E, W>(a); d_mark_neighbors<4, O, E, W>(a); break;
            case 8: d_update_small<8, true, O, E, W>(a); d_mark_neighbors<8, O, E, W>(a); break;
            case 16: d_update_small<16, true, O, E, W>(a); d_mark_neighbors<16, O, E, W>(a); break;
            default: d_update_small<32, true, O, E, W>(a); d_mark_neighbors<32, O, E, W>(a); break;
        }
        d_update_small_hub<true, O, E, W>(a);
        d_mark_neighbors_hub<O, E, W>(a);
        if (!level_sync<CL>(cs.bar, err)) return;
        pc.mark(PH_UPDATE_ADD);
        if (a.dev->large) {
            // update_large: queue the marked rows (one coalesced pass), then
            // rebuild them one warp per row
            for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
                int64_t i = base + threadIdx.x;
                bool take = i < n && a.mark[i];
                int64_t s = warp_append(&cs.bar->nmarked, take);
                if (take) cs.marked[s] = (O)i;
            }
            if (!level_sync<CL>(cs.bar, err)) return;
            d_conn_warp<O, E, W>(a, cs.marked, (O)((volatile GridBar*)cs.bar)->nmarked, 1, nullptr);
            if (!level_sync<CL>(cs.bar, err)) return;
        }
        pc.mark(PH_REBUILD);
        d_cut_after<O, E, W>(a);
        // the last block to finish its share of the cut change closes the
        // iteration (one barrier instead of two): its fence and counter add
        // come after every other block's cut atomics
        {
            __shared__ int s_last;
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                s_last = atomicAdd(&cs.bar->cut_done, 1u) == gridDim.x - 1;
            }
            __syncthreads();
            if (s_last) {
                __threadfence();
                W mx = block_max_sizes<W>(a.sizes, a.k);
                if (threadIdx.x == 0) {
                    cs.bar->cut_done = 0;
                    ctl_end_logic<O, W>(c, a.dev, mx);
                    cs.bar->nmarked = 0;
                    if (c->more && c->iter_count >= max_iters) { c->more = 0; atomicOr(err, ERRF_SPIN); }
                }
            }
        }
        if (!level_sync<CL>(cs.bar, err)) return;
        pc.mark(PH_CUT);
        // the copy of the best state needs no barrier of its own: what it
        // reads (parts, sizes) is next written by the apply phase, at least
        // one barrier later, and nothing reads what it writes during the loop
        if (((volatile Ctl<W>*)c)->copy) {
            for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
                best_part[i] = a.part[i];
            for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.k; p += gridDim.x * blockDim.x) sizes_best[p] = a.sizes[p];
        }
        pc.mark(PH_COPY);
    }
    pc.flush();
}

}  // namespace jetb
