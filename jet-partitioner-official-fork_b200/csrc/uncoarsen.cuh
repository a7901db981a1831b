// uncoarsen.cuh -- Jet refinement driver (src/jet_refiner.hpp:1050-1142),
// the uncoarsening loop (src/uncoarsen.hpp:88-158) and the whole partition
// (src/partitioner.hpp:61-125).
#pragma once
#include <cstdlib>
#include "partitioner.cuh"
#include "sort.cuh"
#include "level_coop.cuh"
#include "prof.cuh"

namespace jetb {

template <class O, class E, class W>
struct Refiner {
    Engine<O, E, W>& e;
    cudaStream_t s;
    part_t k;
    O n_max;
    int64_t slots_cap;
    DBuf<E> coff;
    DBuf<Slot<W>> slots;
    DBuf<part_t> csize, dest_cache, part_work, dest, undersized;
    DBuf<uint8_t> lock, mark;
    DBuf<W> save_gain, pregain, score, sizes_curr, sizes_best, evict_adjust, evict_start, buckets;
    DBuf<O> cand, cand_hub, moves, moves_hub, bid, sv0, sv1, redraw, ordl;
    DBuf<uint32_t> sk0, sk1;
    DBuf<W> boff, wpre;
    DBuf<part_t> redraw_p;
    RadixScratch rsort;
    DBuf<RefDev<O, W>> dev;
    DBuf<Ctl<W>> ctl;
    Ctl<W>* hctl = nullptr;  // pinned mirror
    int pslot = -1;
    int64_t bucket_cap = 0;
    bool verbose = false;
    bool use_graph = true;
    bool use_cta = true;
    bool use_coop = true;
    bool use_cluster = true;
    DBuf<GridBar> cbar;
    DBuf<W> cwsum;
    DBuf<uint32_t> chist;
    DBuf<O> cmarked;
    // rows of degree > THREAD_DEG longest first (per level) and the work
    // counters of the persistent table-build kernel
    DBuf<O> lorder;
    DBuf<unsigned> lctr;
    // rows of 9-16 and of 17-32 edges (per level) and their counts
    DBuf<O> s16, s32, scnt;
    DBuf<unsigned> cdone;  // k_cut_finalize_ctl's block counter
    O n_lorder = 0;
    mutable int long_grid_cache = -1;
    // 1: the total edge weight of the finest level is below 2^31, so every
    // row sum of every level fits in 32 bits (contraction only merges and
    // drops edge weight); 0: not; -1: not yet known
    int narrow_state = -1;

    struct HostState {
        W cut = 0;
        W total_imb = 0;
        W total_size = 0;
        bool init = false;
    };
    HostState best, curr;
    int64_t total_iters = 0;

    Refiner(Engine<O, E, W>& eng, O nmax, int64_t mmax, part_t kk) : e(eng), s(eng.s), k(kk), n_max(nmax) {
        int64_t n1 = nmax > 0 ? nmax : 1;
        coff.alloc(n1 + 1, s);
        slots_cap = mmax > 0 ? mmax : 1;
        slots.alloc(slots_cap, s);
        csize.alloc(n1, s); dest_cache.alloc(n1, s); part_work.alloc(n1, s); dest.alloc(n1, s);
        lock.alloc(n1, s); mark.alloc(n1, s); mark.zero();
        save_gain.alloc(n1, s); pregain.alloc(n1, s); score.alloc(n1, s);
        cand.alloc(n1, s); cand_hub.alloc(n1, s); moves.alloc(n1, s); moves_hub.alloc(n1, s); bid.alloc(n1, s);
        sizes_curr.alloc(k, s); sizes_best.alloc(k, s); undersized.alloc(k, s); evict_adjust.alloc(k, s);
        evict_start.alloc(k + 1, s);
        O sections, tmb;
        sections_for(nmax, sections, tmb);
        bucket_cap = (int64_t)tmb + 1 + (int64_t)MAX_BUCKETS * sections;
        buckets.alloc(bucket_cap, s);
        boff.alloc(bucket_cap, s);
        sk0.alloc(n1, s); sk1.alloc(n1, s); sv0.alloc(n1, s); sv1.alloc(n1, s); wpre.alloc(n1, s);
        redraw.alloc(n1, s); redraw_p.alloc(n1, s); ordl.alloc(n1, s);
        lorder.alloc(n1, s);
        s16.alloc(n1, s);
        s32.alloc(n1, s);
        scnt.alloc(2, s);
        cdone.alloc(1, s);
        cdone.zero();
        lctr.alloc(2, s);
        lctr.zero();
        dev.alloc(1, s);
        dev.zero();
        ctl.alloc(1, s);
        ctl.zero();
        pcount.alloc(1, s);
        ph_reset();
        int drv = refine_drivers();
        use_cta = (drv & JET_DRIVER_CTA) != 0;
        use_coop = (drv & JET_DRIVER_COOP) != 0;
        use_cluster = (drv & JET_DRIVER_CLUSTER) != 0;
        use_graph = (drv & JET_DRIVER_GRAPH) != 0;
        pslot = pinned_acquire(sizeof(Ctl<W>));
        hctl = (Ctl<W>*)pinned_ptr(pslot);
        std::memset(hctl, 0, sizeof(Ctl<W>));
        // scratch for every scan and sort an iteration may run, sized up front
        // so that iterations can be captured into a graph (no allocation inside)
        int64_t scan_max = (n1 + 1 > bucket_cap ? n1 + 1 : bucket_cap);
        int64_t tiles = ceil_div<int64_t>(scan_max, SCAN_TILE) + 1024;
        if (e.scan.buf.n < tiles) e.scan.buf.alloc(tiles, s);
        int64_t rs_h = ceil_div<int64_t>(n1, RS_TILE) * RS_BINS + 1024;
        if (rsort.hist.n < rs_h) rsort.hist.alloc(rs_h, s);
    }
    ~Refiner() {
        cudaStreamSynchronize(s);
        pinned_release(pslot);
    }

    // src/jet_refiner.hpp:425-430 and :559-564
    void sections_for(O n, O& sections, O& t_minibuckets) const {
        sections = MAX_SECTIONS;
        O section_size = (n + sections * k) / (sections * k);
        if (section_size < 4096) {
            section_size = 4096;
            sections = (n + section_size * k) / (section_size * k);
        }
        t_minibuckets = MAX_BUCKETS * k * sections;
    }

    RefArgs<O, E, W> args(const Level<O, E, W>& L) {
        RefArgs<O, E, W> a;
        a.g = L.view(); a.k = k; a.coff = coff.p; a.slots = slots.p; a.csize = csize.p; a.dest_cache = dest_cache.p;
        a.lock = lock.p; a.mark = mark.p; a.part = part_work.p; a.dest = dest.p; a.save_gain = save_gain.p;
        a.pregain = pregain.p; a.sizes = sizes_curr.p; a.cand = cand.p; a.cand_hub = cand_hub.p; a.moves = moves.p;
        a.moves_hub = moves_hub.p; a.dev = dev.p; a.filter = &ctl.p->filter;
        a.narrow = narrow_state > 0 ? 1 : 0;
        a.pclk = phase_clk_ptr();
        return a;
    }

    size_t warp_smem() const {
        int kw = k < WARP_TABLE ? k : WARP_TABLE;
        return (size_t)(BLOCK / 32) * kw * (sizeof(part_t) + sizeof(W)) + 16;
    }
    size_t cta_smem() const { return (((size_t)k * sizeof(part_t) + 15) & ~(size_t)15) + (size_t)k * sizeof(W); }

    bool attrs_done = false;
    void set_attrs() {
        if (attrs_done) return;
        JET_CUDA(cudaFuncSetAttribute(k_conn_warp<O, E, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)warp_smem_max()));
        JET_CUDA(cudaFuncSetAttribute(k_conn_cta<O, E, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      device_info().max_smem_optin - 1024));
        JET_CUDA(cudaFuncSetAttribute(k_reb_ordered<false, O, E, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(QUEUE_KEYS * sizeof(uint64_t))));
        JET_CUDA(cudaFuncSetAttribute(k_reb_ordered<true, O, E, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(QUEUE_KEYS * sizeof(uint64_t))));
        attrs_done = true;
    }
    static size_t warp_smem_max() { return (size_t)(BLOCK / 32) * WARP_TABLE * (sizeof(part_t) + sizeof(W)) + 16; }

    // Builds (or, with only_marked, rebuilds the marked rows of) every table.
    void build_tables(const Level<O, E, W>& L, int only_marked, const int* gate) {
        set_attrs();
        auto a = args(L);
        if (cta_smem() > (size_t)device_info().max_smem_optin - 1024)
            throw JetError{JET_ERR_INVALID, "num_parts too large for the shared-memory connectivity tables"};
        k_conn_thread<8, 256, O, E, W><<<grid_persistent(L.n, 8), 256, 0, s>>>(a, -1, 8, only_marked, gate, nullptr, nullptr); count_launch();
        if (L.max_deg > 8) {
            k_conn_thread<16, 256, O, E, W><<<grid_persistent(L.n, 8), 256, 0, s>>>(a, 8, 16, only_marked, gate, s16.p, scnt.p); count_launch();
        }
        if (L.max_deg > 16) {
            k_conn_thread<32, 128, O, E, W><<<grid_persistent(L.n, 16), 128, 0, s>>>(a, 16, THREAD_DEG, only_marked, gate, s32.p,
                                                                                  scnt.p + 1); count_launch();
        }
        JET_LAUNCH_CHECK();
        if (k <= WARP_TABLE && n_lorder > 0) {
            const int threads = long_threads();
            k_conn_long<O, E, W><<<long_grid(), threads, conn_long_smem<W>(threads / 32, k), s>>>(a, lorder.p, n_lorder, only_marked, gate,
                                                                                             lctr.p, LONG_BLOCK_MIN); count_launch();
            JET_LAUNCH_CHECK();
            return;
        }
        if (L.n_warp > 0) {
            if (k <= WARP_TABLE) {
                k_conn_warp<O, E, W><<<grid_persistent((int64_t)L.n_warp * 32, 16), BLOCK, warp_smem(), s>>>(a, L.warp_list.p, L.n_warp, only_marked, gate, INT64_MAX); count_launch();
            } else {
                k_conn_cta<O, E, W><<<grid_for(L.n_warp, 1) < 4096 ? grid_for(L.n_warp, 1) : 4096, 256, cta_smem(), s>>>(a, L.warp_list.p, L.n_warp, only_marked, gate, 0, 0); count_launch();
            }
            JET_LAUNCH_CHECK();
        }
        if (L.n_hub > 0) {
            // rows of the hub bin up to WARP_ROW_MAX edges still go one warp
            // per row (thousands of warps beat one CTA per row on dense levels);
            // only the longest rows get a whole CTA
            int64_t cta_from = 0;
            if (k <= WARP_TABLE) {
                k_conn_warp<O, E, W><<<grid_persistent((int64_t)L.n_hub * 32, 16), BLOCK, warp_smem(), s>>>(a, L.hub_list.p, L.n_hub, only_marked, gate, WARP_ROW_MAX); count_launch();
                cta_from = WARP_ROW_MAX;
            }
            if ((int64_t)L.max_deg > cta_from) {
                const int priv = k <= WARP_TABLE ? 1 : 0;
                const size_t sm = cta_smem() + (priv ? (((size_t)32 * k * sizeof(W) + 15) & ~(size_t)15) : 0);
                k_conn_cta<O, E, W><<<grid_for(L.n_hub, 1) < 4096 ? grid_for(L.n_hub, 1) : 4096, 1024, sm, s>>>(a, L.hub_list.p, L.n_hub, only_marked, gate, cta_from, priv); count_launch();
            }
            JET_LAUNCH_CHECK();
        }
    }
    static constexpr int64_t WARP_ROW_MAX = 16384;
    // rows of at least this many edges get a whole block in k_conn_long (a
    // power of two >= WARP_TABLE, so whole degree classes go one way)
    static constexpr int64_t LONG_BLOCK_MIN = 4096;
    // levels with fewer rows of degree > THREAD_DEG keep the per-list kernels
    static constexpr int64_t LONG_MIN_ROWS = 1024;
    // 1024 threads, two blocks per SM (measured against 512 x 4: faster on
    // levels dominated by single-warp rows, about 10% slower on a level of
    // whole-block rows, which are rarer)
    int long_threads() const { return 1024; }
    int long_grid() const {
        if (long_grid_cache >= 0) return long_grid_cache;
        const void* f = (const void*)k_conn_long<O, E, W>;
        JET_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dynamic_smem(f)));
        int per_sm = 0;
        JET_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, long_threads(), conn_long_smem<W>(long_threads() / 32, k)));
        long_grid_cache = device_info().sms * (per_sm > 0 ? per_sm : 1);
        return long_grid_cache;
    }
    // Per-level row lists for the table builds: rows of 9-16 and of 17-32
    // edges (k_bin_short), and rows of degree > THREAD_DEG longest first
    // (stable radix sort by power-of-two degree class) for k_conn_long.
    void order_long_rows(const Level<O, E, W>& L) {
        n_lorder = 0;
        if (L.max_deg > 8) {
            JET_CUDA(cudaMemsetAsync(scnt.p, 0, 2 * sizeof(O), s));
            k_bin_short<O, E><<<grid_persistent(L.n, 8), BLOCK, 0, s>>>(L.n, L.row, s16.p, s32.p, scnt.p); count_launch();
            JET_LAUNCH_CHECK();
        }
        const int64_t cnt = (int64_t)L.n_warp + (int64_t)L.n_hub;
        if (k > WARP_TABLE || cnt < LONG_MIN_ROWS) return;
        GetLongKey<O, E> key{L.warp_list.p, L.hub_list.p, L.n_warp, L.row};
        GetLongRow<O> val{L.warp_list.p, L.hub_list.p, L.n_warp};
        // six key bits: one pass, the rows land in lorder
        int which = radix_sort_pairs<uint32_t, O>(key, val, cnt, 6, sk0.p, lorder.p, sk1.p, sv1.p, rsort, e.scan, s);
        if (which != 0) JET_CUDA(cudaMemcpyAsync(lorder.p, sv1.p, sizeof(O) * cnt, cudaMemcpyDeviceToDevice, s));
        n_lorder = (O)cnt;
    }

    // Sets narrow_state from a level's total edge weight (the finest level's
    // bounds every coarser one).
    void set_weight_bound(const Level<O, E, W>& L) {
        if (sizeof(W) < 8) { narrow_state = 0; return; }
        W* sum = e.template dslot<W>(54);
        JET_CUDA(cudaMemsetAsync(sum, 0, sizeof(int64_t), s));
        if (L.m > 0) { k_sum<W><<<grid_persistent((int64_t)L.m, 8), BLOCK, 0, s>>>(L.val, (int64_t)L.m, sum); count_launch(); }
        JET_LAUNCH_CHECK();
        JET_CUDA(cudaMemcpyAsync(e.hscal, sum, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        e.sync();
        narrow_state = (int64_t)*(W*)e.hscal < ((int64_t)1 << 31) ? 1 : 0;
    }

    // init_conn_data, src/jet_refiner.hpp:958-1048.  Returns sum of capacities.
    int64_t init_conn(const Level<O, E, W>& L) {
        if (narrow_state < 0) set_weight_bound(L);
        exclusive_scan<E, GetConnCap<O, E>>(GetConnCap<O, E>{L.row, k}, L.n, coff.p, coff.p + L.n, e.scan, s);
        JET_CUDA(cudaMemcpyAsync(&e.hscal[0], coff.p + L.n, sizeof(E), cudaMemcpyDeviceToHost, s));
        e.sync();
        E C = *(E*)&e.hscal[0];
        // events bracket exactly the table-build kernels
        const double bytes =
            (double)L.n * (3 * sizeof(E) + 4) + (double)L.m * (sizeof(O) + sizeof(W) + 4) + (double)C * sizeof(Slot<W>);
        const bool finest = (int64_t)L.n == (int64_t)n_max;
        order_long_rows(L);
        int h = prof_begin(s);
        int hf = finest ? prof_begin(s) : -1;
        build_tables(L, 0, nullptr);
        if (finest) prof_end(hf, PK_CONN_FINEST, bytes, s);
        prof_end(h, PK_CONN_BUILD, bytes, s);
        fill<part_t>(dest_cache.p, L.n, NULL_PART, s);
        JET_CUDA(cudaMemsetAsync(lock.p, 0, L.n, s));
        last_slots = (int64_t)C;
        return (int64_t)C;
    }
    int64_t last_slots = 0;  // table slots of the level init_conn built last

    // Profiling-pass handles of the current iteration's class brackets.
    int ph[PK_COUNT];
    int ph_mark = -1;
    DBuf<ProfCounts> pcount;
    void ph_reset() { for (int i = 0; i < PK_COUNT; i++) ph[i] = -1; ph_mark = -1; phq[0] = phq[1] = -1; }

    void lp(const Level<O, E, W>& L) {
        auto a = args(L);
        int h = prof_begin(s);
        ph[PK_LP_SELECT] = h;
        k_lp_select_thread<O, E, W><<<grid_persistent(L.n, 16), BLOCK, 0, s>>>(a); count_launch();
        JET_LAUNCH_CHECK();
        if (L.n_warp > 0) { k_lp_select_warp<O, E, W><<<grid_persistent((int64_t)L.n_warp * 32, 16), BLOCK, 0, s>>>(a, L.warp_list.p, L.n_warp); count_launch(); }
        if (L.n_hub > 0) { k_lp_select_warp<O, E, W><<<grid_persistent((int64_t)L.n_hub * 32, 16), BLOCK, 0, s>>>(a, L.hub_list.p, L.n_hub); count_launch(); }
        JET_LAUNCH_CHECK();
        prof_end(h, PK_LP_SELECT, 0, s);
        h = prof_begin(s);
        ph[PK_AFTERBURN] = h;
        unsigned grid = grid_persistent((int64_t)L.n * L.group, 16);
        switch (L.group) {
            case 4: k_afterburn<4, O, E, W><<<grid, BLOCK, 0, s>>>(a); count_launch(); break;
            case 8: k_afterburn<8, O, E, W><<<grid, BLOCK, 0, s>>>(a); count_launch(); break;
            case 16: k_afterburn<16, O, E, W><<<grid, BLOCK, 0, s>>>(a); count_launch(); break;
            default: k_afterburn<32, O, E, W><<<grid, BLOCK, 0, s>>>(a); count_launch(); break;
        }
        JET_LAUNCH_CHECK();
        if (L.n_hub > 0) {
            k_afterburn_hub<O, E, W><<<device_info().sms * 2, 1024, 0, s>>>(a); count_launch();
            JET_LAUNCH_CHECK();
        }
        prof_end(h, PK_AFTERBURN, 0, s);
    }

    // max_dest of src/jet_refiner.hpp:575-578 (weak) and :437 (strong)
    static W weak_max_dest(W size_max) {
        W md = (W)((double)size_max * 0.99);
        if (md < size_max - 100) md = size_max - 100;
        return md;
    }
    static W strong_max_dest(W opt, W size_max) {
        W md = (W)((double)size_max * 0.99);
        return opt + 1 > md ? opt + 1 : md;
    }

    RebArgs<O, W> reb_args(const Level<O, E, W>& L, W max_dest, W opt, W size_max, bool clear = true) {
        RebArgs<O, W> rb;
        O sections, tmb;
        sections_for(L.n, sections, tmb);
        rb.size_max = size_max; rb.opt = opt; rb.max_dest = max_dest; rb.sections = sections; rb.t_minibuckets = tmb;
        rb.width = MAX_BUCKETS * sections; rb.buckets = buckets.p; rb.boff = boff.p; rb.bid = bid.p; rb.score = score.p;
        rb.undersized = undersized.p; rb.evict_adjust = evict_adjust.p; rb.evict_start = evict_start.p;
        rb.redraw = redraw.p; rb.redraw_p = redraw_p.p;
        rb.skey = nullptr; rb.sval = nullptr; rb.wpre = wpre.p;
        rb.none_key = (uint32_t)((int64_t)tmb + rb.width + 1);
        rb.ordl = ordl.p;
        // queue keys pack (bucket id, vertex) into 32 bits each
        rb.queue = reb_queue_enabled() && (int64_t)L.n <= (int64_t)UINT32_MAX && bucket_cap <= (int64_t)UINT32_MAX;
        if ((int64_t)tmb + 1 + rb.width > bucket_cap) throw JetError{JET_ERR_INVALID, "bucket array too small"};
        if (clear) JET_CUDA(cudaMemsetAsync(buckets.p, 0, sizeof(W) * ((size_t)tmb + 1 + rb.width), s));
        return rb;
    }

    // Bucket offsets, then candidates sorted by bucket id (stable in vertex
    // id) with the prefix of their weights: the in-order bucket scores.
    void sort_candidates(const Level<O, E, W>& L, RebArgs<O, W>& rb) {
        exclusive_scan_array<W>(buckets.p, (int64_t)rb.t_minibuckets + 1, boff.p, nullptr, e.scan, s);
        int bits = bits_for((uint64_t)rb.none_key);
        int which = radix_sort_pairs<uint32_t, O>(GetBidKey<O>{bid.p, rb.none_key}, GetIndex<O>{}, (int64_t)L.n, bits, sk0.p, sv0.p,
                                                  sk1.p, sv1.p, rsort, e.scan, s);
        rb.skey = which == 0 ? sk0.p : sk1.p;
        rb.sval = which == 0 ? sv0.p : sv1.p;
        exclusive_scan<W, GetSortedWeight<O, W>>(GetSortedWeight<O, W>{rb.skey, rb.sval, L.vw, rb.none_key}, (int64_t)L.n, wpre.p,
                                                 nullptr, e.scan, s);
    }

    // rebalance_weak, src/jet_refiner.hpp:551-645: destinations and bucket
    // scores, then the eviction (the queue path, else the full sort).
    void weak_select(const Level<O, E, W>& L, RebArgs<O, W>& rb) {
        auto a = args(L);
        int h = ph[PK_REB_SELECT] = prof_begin(s);
        k_weak_prep<O, E, W><<<1, 1024, 0, s>>>(a, rb); count_launch();
        k_weak_select_thread<O, E, W><<<grid_persistent(L.n, 16), BLOCK, 0, s>>>(a, rb); count_launch();
        if (L.n_warp > 0) { k_weak_select_warp<O, E, W><<<grid_persistent((int64_t)L.n_warp * 32, 16), BLOCK, 0, s>>>(a, rb, L.warp_list.p, L.n_warp); count_launch(); }
        if (L.n_hub > 0) { k_weak_select_warp<O, E, W><<<grid_persistent((int64_t)L.n_hub * 32, 16), BLOCK, 0, s>>>(a, rb, L.hub_list.p, L.n_hub); count_launch(); }
        JET_LAUNCH_CHECK();
        prof_end(h, PK_REB_SELECT, 0, s);
    }
    void weak_full(const Level<O, E, W>& L, RebArgs<O, W>& rb) {
        auto a = args(L);
        int h = ph[PK_REB_SORT] = prof_begin(s);
        sort_candidates(L, rb);
        prof_end(h, PK_REB_SORT, reb_sort_bytes(L, rb), s);
        h = ph[PK_REB_EVICT] = prof_begin(s);
        k_evict_sorted<false, O, E, W><<<grid_persistent(L.n, 16), BLOCK, 0, s>>>(a, rb); count_launch();
        JET_LAUNCH_CHECK();
        prof_end(h, PK_REB_EVICT, 0, s);
    }
    void weak(const Level<O, E, W>& L, W opt, W size_max) {
        auto rb = reb_args(L, weak_max_dest(size_max), opt, size_max);
        weak_select(L, rb);
        if (!rb.queue || !reb_queue<false>(L, rb)) weak_full(L, rb);
    }

    // Algorithmic bytes of sort_candidates: the bucket scan, each radix pass
    // reading and writing (key, vertex) pairs, and the weight prefix.
    double reb_sort_bytes(const Level<O, E, W>& L, const RebArgs<O, W>& rb) const {
        const double n = (double)L.n;
        const int passes = (bits_for((uint64_t)rb.none_key) + 7) / 8;
        return 2.0 * ((double)rb.t_minibuckets + 1) * sizeof(W) + passes * n * 2.0 * (4 + sizeof(O)) +
               n * (4 + sizeof(O) + 2 * sizeof(W));
    }

    // rebalance_strong, src/jet_refiner.hpp:417-546.
    void strong_select(const Level<O, E, W>& L, RebArgs<O, W>& rb) {
        auto a = args(L);
        int h = ph[PK_REB_SELECT] = prof_begin(s);
        k_strong_prep<O, E, W><<<1, 1024, 0, s>>>(a, rb); count_launch();
        k_strong_score_thread<O, E, W><<<grid_persistent(L.n, 16), BLOCK, 0, s>>>(a, rb); count_launch();
        if (L.n_warp > 0) { k_strong_score_warp<O, E, W><<<grid_persistent((int64_t)L.n_warp * 32, 16), BLOCK, 0, s>>>(a, rb, L.warp_list.p, L.n_warp); count_launch(); }
        if (L.n_hub > 0) { k_strong_score_warp<O, E, W><<<grid_persistent((int64_t)L.n_hub * 32, 16), BLOCK, 0, s>>>(a, rb, L.hub_list.p, L.n_hub); count_launch(); }
        JET_LAUNCH_CHECK();
        prof_end(h, PK_REB_SELECT, 0, s);
    }
    void strong_full(const Level<O, E, W>& L, RebArgs<O, W>& rb) {
        auto a = args(L);
        int h = ph[PK_REB_SORT] = prof_begin(s);
        sort_candidates(L, rb);
        prof_end(h, PK_REB_SORT, reb_sort_bytes(L, rb), s);
        h = ph[PK_REB_EVICT] = prof_begin(s);
        JET_CUDA(cudaMemsetAsync(evict_adjust.p, 0, sizeof(W) * k, s));
        k_evict_sorted<true, O, E, W><<<grid_persistent(L.n, 16), BLOCK, 0, s>>>(a, rb); count_launch();
        k_cookie<O, E, W><<<1, 1024, 0, s>>>(a, rb); count_launch();
        k_strong_first<O, E, W><<<grid_persistent(L.n, 8), BLOCK, 0, s>>>(a, rb); count_launch();
        k_strong_redraw<O, E, W><<<1, 1024, 0, s>>>(a, rb); count_launch();
        JET_LAUNCH_CHECK();
        prof_end(h, PK_REB_EVICT, 0, s);
    }
    void strong(const Level<O, E, W>& L, W opt, W size_max) {
        auto rb = reb_args(L, strong_max_dest(opt, size_max), opt, size_max);
        strong_select(L, rb);
        if (!rb.queue || !reb_queue<true>(L, rb)) strong_full(L, rb);
    }

    // The queue path of the eviction (d_reb_classify, k_reb_ordered): bucket
    // offsets, the classification over every vertex, then one block orders
    // the queue and finishes.  In a graph (h given) the ordering kernel sets
    // h for the fallback's IF node; on the host loop this reads back whether
    // the fallback must run, and returns false if so.
    static constexpr int QUEUE_KEYS = 8192;  // 64 KiB of keys in k_reb_ordered's shared memory
    int phq[2] = {-1, -1};                  // profiling brackets of the queue path
    template <bool STRONG>
    bool reb_queue(const Level<O, E, W>& L, RebArgs<O, W>& rb, cudaGraphConditionalHandle h = 0, bool in_graph = false) {
        auto a = args(L);
        set_attrs();
        if (prof_active()) {
            k_prof_bid<O><<<grid_persistent(L.n, 4), BLOCK, 0, s>>>(rb.bid, (int64_t)L.n, &pcount.p->reb_cand); count_launch();
            JET_LAUNCH_CHECK();
        }
        phq[0] = prof_begin(s);
        exclusive_scan_array<W>(buckets.p, (int64_t)rb.t_minibuckets + 1, boff.p, nullptr, e.scan, s);
        k_reb_classify<STRONG, O, E, W><<<grid_persistent(L.n, 16), BLOCK, 0, s>>>(a, rb); count_launch();
        JET_LAUNCH_CHECK();
        prof_end(phq[0], PK_REB_SORT, 0, s);
        phq[1] = prof_begin(s);
        k_reb_ordered<STRONG, O, E, W><<<1, 1024, QUEUE_KEYS * sizeof(uint64_t), s>>>(a, rb, QUEUE_KEYS, h, in_graph ? 1 : 0);
        count_launch();
        JET_LAUNCH_CHECK();
        prof_end(phq[1], PK_REB_EVICT, 0, s);
        if (in_graph) return true;
        JET_CUDA(cudaMemcpyAsync(e.hscal, dev.p, sizeof(RefDev<O, W>), cudaMemcpyDeviceToHost, s));
        e.sync();
        const RefDev<O, W>* d = (const RefDev<O, W>*)e.hscal;
        q_last = (int64_t)d->nord_last;
        q_fb_last = d->reb_fb_taken;
        return !d->reb_fb_taken;
    }
    int64_t q_last = 0;
    int q_fb_last = 0;

    // perform_moves, src/jet_refiner.hpp:905-955, in four parts: the moves
    // themselves (apply_moves_kernel, which also decides update_small versus
    // update_large), the small update (subtract pass over all moved vertices,
    // hubs included, then the add pass), the large update (mark the
    // neighbours, rebuild their tables) and the cut change.  Both updates'
    // kernels test the device-side decision, so running both is correct.
    void apply_moves_kernel(const Level<O, E, W>& L) {
        auto a = args(L);
        int hist = (size_t)k * sizeof(W) <= 32 * 1024;
        k_apply_moves<O, E, W><<<grid_persistent(L.n, 8), BLOCK, hist ? (size_t)k * sizeof(W) : 0, s>>>(a, hist); count_launch();
        JET_LAUNCH_CHECK();
    }
    void small_update_kernels(const Level<O, E, W>& L) {
        auto a = args(L);
        unsigned grid = grid_persistent((int64_t)L.n * L.group / 4 + 1, 16);
        const unsigned hub_grid = device_info().sms * 2;
        // every subtraction before any addition (src/jet_refiner.hpp:786, :810)
        switch (L.group) {
            case 4: k_update_small<4, false, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            case 8: k_update_small<8, false, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            case 16: k_update_small<16, false, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            default: k_update_small<32, false, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
        }
        count_launch();
        if (L.n_hub > 0) { k_update_small_hub<false, O, E, W><<<hub_grid, 1024, 0, s>>>(a); count_launch(); }
        switch (L.group) {
            case 4: k_update_small<4, true, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            case 8: k_update_small<8, true, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            case 16: k_update_small<16, true, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            default: k_update_small<32, true, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
        }
        count_launch();
        if (L.n_hub > 0) { k_update_small_hub<true, O, E, W><<<hub_grid, 1024, 0, s>>>(a); count_launch(); }
        JET_LAUNCH_CHECK();
    }
    void large_update_kernels(const Level<O, E, W>& L) {
        auto a = args(L);
        unsigned grid = grid_persistent((int64_t)L.n * L.group / 4 + 1, 16);
        switch (L.group) {
            case 4: k_mark_neighbors<4, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            case 8: k_mark_neighbors<8, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            case 16: k_mark_neighbors<16, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
            default: k_mark_neighbors<32, O, E, W><<<grid, BLOCK, 0, s>>>(a); break;
        }
        count_launch();
        if (L.n_hub > 0) { k_mark_neighbors_hub<O, E, W><<<device_info().sms * 2, 1024, 0, s>>>(a); count_launch(); }
        JET_LAUNCH_CHECK();
        if (ph_mark >= 0) {
            // profiling pass: count the marked rows between the two brackets
            prof_end(ph_mark, PK_UPDATE_LARGE, 0, s);
            k_prof_marked<O, E, W><<<grid_persistent(L.n, 4), BLOCK, 0, s>>>(a, pcount.p); count_launch();
            JET_LAUNCH_CHECK();
            ph[PK_UPDATE_LARGE] = prof_begin(s);
        }
        build_tables(L, 1, &dev.p->large);
    }
    void cut_after_kernel(const Level<O, E, W>& L) {
        k_cut_after<O, E, W><<<grid_persistent(L.n, 8), BLOCK, 0, s>>>(args(L)); count_launch();
        JET_LAUNCH_CHECK();
    }
    void moves_kernels(const Level<O, E, W>& L) {
        ph[PK_UPDATE_LARGE] = -1;
        int h = ph[PK_APPLY] = prof_begin(s);
        apply_moves_kernel(L);
        prof_end(h, PK_APPLY, 0, s);
        h = ph[PK_UPDATE] = prof_begin(s);
        small_update_kernels(L);
        prof_end(h, PK_UPDATE, 0, s);
        ph_mark = prof_begin(s);
        large_update_kernels(L);
        if (ph[PK_UPDATE_LARGE] >= 0) prof_end(ph[PK_UPDATE_LARGE], PK_UPDATE_LARGE, 0, s);
        h = ph[PK_CUT_AFTER] = prof_begin(s);
        cut_after_kernel(L);
        prof_end(h, PK_CUT_AFTER, 0, s);
    }

    // Profiling pass, after an iteration's sync: the device counts turned
    // into each class bracket's algorithmic bytes (each array element counted
    // once per bracket: reads of what the class must read, writes of what it
    // produces; a table probe counts one slot).
    void prof_account(const Level<O, E, W>& L, int kind, const IterResult& r) {
        ProfCounts c;
        JET_CUDA(cudaMemcpyAsync(e.hscal, pcount.p, sizeof(ProfCounts), cudaMemcpyDeviceToHost, s));
        e.sync();
        std::memcpy(&c, e.hscal, sizeof(ProfCounts));
        const double so = sizeof(O), se = sizeof(E), sw = sizeof(W), sl = sizeof(Slot<W>);
        const double n = (double)L.n, T = (double)c.moves, Td = (double)c.moves_deg;
        if (kind == 0) {
            // LP select: for every vertex its row offset (degree class),
            // cache test, destination write, lock and pre-gain; the uncached
            // ones read part, offset, size and their table and write gain and
            // cache; candidates read their saved gain and are appended
            prof_add_bytes(ph[PK_LP_SELECT], n * (se + 4 + 4 + 1 + sw) + (double)c.uncached * (4 + se + 4 + sw + 4) +
                                                 (double)c.size_uncached * sl + (double)c.cand * (sw + so));
            // afterburner: each candidate's row, pregain, part and destination;
            // per edge the neighbour, weight and the neighbour's pregain,
            // destination and part; the kept ones are locked and appended
            prof_add_bytes(ph[PK_AFTERBURN], (double)c.cand * (so + 2 * se + sw + 4 + 4) +
                                                 (double)c.cand_deg * (so + sw + sw + 4 + 4) + T * (1 + so));
        } else {
            // weak select / strong scores: every vertex's part, weight, table
            // offset and size and its whole table; bucket id and score out
            prof_add_bytes(ph[PK_REB_SELECT], n * (4 + sw + se + 4 + 4 + sw) + (double)c.csize_all * sl);
            const double evict_full = n * (4 + so + sw + 4) + T * (so + 4);
            if (phq[0] >= 0) {
                O sections, tmb;
                sections_for(L.n, sections, tmb);
                const double nb = (double)tmb + 1, m = (double)q_last, cand = (double)c.reb_cand;
                // queue path: bucket scan (read, write), every vertex's bucket
                // id, each candidate's part and weight, the bucket offsets and
                // totals and the part sizes once, the queued and the directly
                // evicted vertices appended
                prof_add_bytes(phq[0], 2 * nb * sw + n * so + cand * (4 + sw) + 2 * nb * sw + k * sw + (T + m) * so);
                // ordering block: each queued vertex's id, bucket, weight and
                // part and its two bucket offsets, the moves appended (strong:
                // the score writes, the cookie cutter over the parts and each
                // move's destination draw)
                double ob = m * (so + so + sw + 4 + 2 * sw) + T * so;
                if (kind == 2) ob += m * sw + 4.0 * k * sw + T * (so + 4 + 3 * sw + 4);
                prof_add_bytes(phq[1], q_fb_last ? 0.0 : ob);
                if (q_fb_last) prof_add_bytes(ph[PK_REB_EVICT], evict_full);
            } else {
                // eviction filter over the sorted candidates; the moves appended
                prof_add_bytes(ph[PK_REB_EVICT], evict_full);
            }
        }
        // apply: per move its vertex, part, destination and weight, the part
        // and destination writes, the two size updates
        prof_add_bytes(ph[PK_APPLY], T * (so + 4 + 4 + sw + 4 + 4 + 4) + 2.0 * k * sw);
        if (r.large) {
            // mark: each moved vertex's row and its neighbours' marks
            prof_add_bytes(ph_mark, Td * (so + 1) + T * 2 * se);
            // rebuild: each marked row, its neighbours' parts and the table
            prof_add_bytes(ph[PK_UPDATE_LARGE], (double)c.marked * (2 * se + 1 + 4) +
                                                    (double)c.marked_deg * (so + sw + 4) + (double)c.marked_cap * sl);
        } else {
            // small update, subtract then add: per moved edge the neighbour,
            // weight, the neighbour's table offset, size and one slot
            // read-modify-write, twice
            prof_add_bytes(ph[PK_UPDATE], 2.0 * Td * (so + sw + se + 4 + 2 * sl) + T * (so + 2 * se + 8));
        }
        // cut change part 2: per move two lookups in its own table
        prof_add_bytes(ph[PK_CUT_AFTER], T * (so + se + 4 + 8 + 2 * sl));
    }

    // Host-driven iteration end: results to pinned memory, one host sync.
    IterResult perform_moves(const Level<O, E, W>& L) {
        moves_kernels(L);
        if (ph[PK_APPLY] >= 0) {
            auto a = args(L);
            k_prof_list<O, E><<<grid_persistent(L.n, 4), BLOCK, 0, s>>>(a.g.row, a.moves, &a.dev->nmoves, &pcount.p->moves,
                                                                       &pcount.p->moves_deg);
            count_launch();
            JET_LAUNCH_CHECK();
        }
        k_finalize<O, E, W><<<1, 1024, 0, s>>>(args(L), e.hres); count_launch();
        JET_LAUNCH_CHECK();
        e.sync();
        IterResult r = *e.hres;
        if (r.err & ~16) throw JetError{JET_ERR_OVERFLOW, "connectivity table update exceeded its bounds"};
        return r;
    }

    W total_cut(const Level<O, E, W>& L, const part_t* part) {
        W* out = e.template dslot<W>(50);
        JET_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
        unsigned grid = grid_persistent((int64_t)L.n * L.group, 16);
        switch (L.group) {
            case 4: k_total_cut<4, O, E, W><<<grid, BLOCK, 0, s>>>(L.view(), part, out); count_launch(); break;
            case 8: k_total_cut<8, O, E, W><<<grid, BLOCK, 0, s>>>(L.view(), part, out); count_launch(); break;
            case 16: k_total_cut<16, O, E, W><<<grid, BLOCK, 0, s>>>(L.view(), part, out); count_launch(); break;
            default: k_total_cut<32, O, E, W><<<grid, BLOCK, 0, s>>>(L.view(), part, out); count_launch(); break;
        }
        JET_LAUNCH_CHECK();
        JET_CUDA(cudaMemcpyAsync(&e.hscal[0], out, sizeof(W), cudaMemcpyDeviceToHost, s));
        e.sync();
        return *(W*)&e.hscal[0];
    }

    void part_sizes(const Level<O, E, W>& L, const part_t* part, W* sizes) {
        JET_CUDA(cudaMemsetAsync(sizes, 0, sizeof(W) * k, s));
        int hist = (size_t)k * sizeof(W) <= 32 * 1024;
        k_part_sizes<O, W><<<grid_persistent(L.n, 8), BLOCK, hist ? (size_t)k * sizeof(W) : 0, s>>>(L.n, L.vw, part, k, sizes, hist); count_launch();
        JET_LAUNCH_CHECK();
    }

    W sum_vw(const Level<O, E, W>& L) {
        W* out = e.template dslot<W>(51);
        JET_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
        k_sum<W><<<grid_persistent(L.n, 8), BLOCK, 0, s>>>(L.vw, L.n, out); count_launch();
        JET_LAUNCH_CHECK();
        JET_CUDA(cudaMemcpyAsync(&e.hscal[0], out, sizeof(W), cudaMemcpyDeviceToHost, s));
        e.sync();
        return *(W*)&e.hscal[0];
    }

    W max_of_sizes(const W* sizes) {
        std::vector<W> h(k);
        JET_CUDA(cudaMemcpyAsync(h.data(), sizes, sizeof(W) * k, cudaMemcpyDeviceToHost, s));
        e.sync();
        W mx = 0;
        for (W x : h) if (x > mx) mx = x;
        return mx;
    }

    void check_parts(const Level<O, E, W>& L, const part_t* part) {
        int* err = e.template dslot<int>(52);
        JET_CUDA(cudaMemsetAsync(err, 0, sizeof(int64_t), s));
        k_check_parts<<<grid_persistent(L.n, 8), BLOCK, 0, s>>>((int64_t)L.n, part, k, err); count_launch();
        JET_LAUNCH_CHECK();
        JET_CUDA(cudaMemcpyAsync(&e.hscal[0], err, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        e.sync();
        if (*(int*)&e.hscal[0]) throw JetError{JET_ERR_INVALID, "part id out of range"};
    }

    // Sets up refinement state for a level (problem values and tables).
    struct Prob {
        W opt, size_max, imb_max;
    };
    Prob begin_level(const Level<O, E, W>& L, part_t* best_part, double imb) {
        if (!best.init) {
            check_parts(L, best_part);
            best.cut = total_cut(L, best_part);
            part_sizes(L, best_part, sizes_best.p);
            best.total_size = sum_vw(L);
        }
        Prob pb;
        O opt = (O)(((O)best.total_size + k - 1) / k);  // optimal_size, ordinal arithmetic (src/part_stat.hpp:111-114)
        O size_max = (O)((double)opt * imbalance_guard(imb));
        pb.opt = opt;
        pb.size_max = size_max;
        pb.imb_max = (W)size_max - (W)opt;
        if (!best.init) {
            best.init = true;
            W mx = max_of_sizes(sizes_best.p);
            best.total_imb = mx > pb.opt ? mx - pb.opt : 0;
            if (verbose)
                printf("Initial %lld %.6f %lld\n", (long long)(best.cut / 2), (double)best.total_imb / (double)pb.opt, (long long)L.n);
        }
        curr = best;
        JET_CUDA(cudaMemcpyAsync(sizes_curr.p, sizes_best.p, sizeof(W) * k, cudaMemcpyDeviceToDevice, s));
        JET_CUDA(cudaMemcpyAsync(part_work.p, best_part, sizeof(part_t) * L.n, cudaMemcpyDeviceToDevice, s));
        init_conn(L);
        return pb;
    }
    static double imbalance_guard(double imb) { return imb; }

    // One iteration body of jet_refine (src/jet_refiner.hpp:1106-1120).
    int iterate(const Level<O, E, W>& L, const Prob& pb, double filter_ratio, int& balance_counter, int& lab_counter) {
        int kind;
        ph_reset();
        const bool pf = prof_active();
        if (pf) {
            auto a = args(L);
            JET_CUDA(cudaMemsetAsync(pcount.p, 0, sizeof(ProfCounts), s));
            k_prof_select<O, E, W><<<grid_persistent(L.n, 4), BLOCK, 0, s>>>(a, pcount.p); count_launch();
            JET_LAUNCH_CHECK();
        }
        if (curr.total_imb <= pb.imb_max) {
            hctl->filter = filter_ratio;
            JET_CUDA(cudaMemcpyAsync(&ctl.p->filter, &hctl->filter, sizeof(double), cudaMemcpyHostToDevice, s));
            lp(L);
            if (pf) {
                auto a = args(L);
                k_prof_list<O, E><<<grid_persistent(L.n, 4), BLOCK, 0, s>>>(a.g.row, a.cand, &a.dev->ncand, &pcount.p->cand,
                                                                           &pcount.p->cand_deg);
                count_launch();
                JET_LAUNCH_CHECK();
            }
            balance_counter = 0;
            lab_counter++;
            kind = 0;
        } else {
            if (balance_counter < 2) { weak(L, pb.opt, pb.size_max); kind = 1; }
            else { strong(L, pb.opt, pb.size_max); kind = 2; }
            balance_counter++;
        }
        IterResult r = perform_moves(L);
        if (pf) prof_account(L, kind, r);
        curr.cut -= (W)r.cut_change;
        W mx = (W)r.max_part;
        curr.total_imb = mx > pb.opt ? mx - pb.opt : 0;
        last_moves = r.nmoves;
        total_iters++;
        return kind;
    }
    int64_t last_moves = 0;

    void save_best(const Level<O, E, W>& L, part_t* best_part) {
        best = curr;
        JET_CUDA(cudaMemcpyAsync(sizes_best.p, sizes_curr.p, sizeof(W) * k, cudaMemcpyDeviceToDevice, s));
        JET_CUDA(cudaMemcpyAsync(best_part, part_work.p, sizeof(part_t) * L.n, cudaMemcpyDeviceToDevice, s));
    }

    // ------------------------------------------------------------ single-CTA loop
    // Levels above CTA_PREFER_N vertices run faster on a 16-CTA cluster when
    // one is available (measured on meshes: 77 vs 127 us per iteration at
    // 4k vertices, 82 vs 104 in favour of one CTA at 835).  Batch and server
    // workers keep one CTA up to CTA_MAX_N: with many partitions sharing the
    // GPU, one SM per level gives more throughput than sixteen.
    static constexpr int64_t CTA_PREFER_N = 2048;
    // The drivers' size bounds, each overridable once per process by an
    // environment variable of the same name with a JET_ prefix (for tuning
    // on other parts; the defaults are the measured crossovers on B200).
    static int64_t bound(const char* env, int64_t def) {
        const char* v = std::getenv(env);
        return (v && *v) ? std::atoll(v) : def;
    }
    static int64_t cta_prefer_n() { static const int64_t v = bound("JET_CTA_PREFER_N", CTA_PREFER_N); return v; }
    static int64_t cluster_max_n() {
        // batch and server workers share the GPU: their bound is separate
        static const int64_t v = bound("JET_CLUSTER_MAX_N", CLUSTER_MAX_N);
        static const int64_t vb = bound("JET_BATCH_CLUSTER_MAX_N", CLUSTER_MAX_N);
        return batch_thread() ? vb : v;
    }
    static int64_t coop_max_n() { static const int64_t v = bound("JET_COOP_MAX_N", COOP_MAX_N); return v; }
    static int64_t cluster_max_m() { static const int64_t v = bound("JET_PERSISTENT_MAX_M", CLUSTER_MAX_M); return v; }
    static int64_t coop_max_m() { static const int64_t v = bound("JET_PERSISTENT_MAX_M", COOP_MAX_M); return v; }
    bool cta_eligible(const Level<O, E, W>& L) const {
        int64_t cap = (use_cluster && !batch_thread() && cluster_size() > 0) ? cta_prefer_n() : CTA_MAX_N;
        return use_cta && (int64_t)L.n <= cap && (int64_t)L.m <= CTA_MAX_M && k <= CTA_MAX_K;
    }

    void ctl_init(const Prob& pb, const std::vector<double>& temps, double tol) {
        Ctl<W>& c = *hctl;
        std::memset(&c, 0, sizeof(c));
        c.curr_cut = curr.cut; c.curr_imb = curr.total_imb; c.best_cut = best.cut; c.best_imb = best.total_imb;
        c.opt = pb.opt; c.imb_max = pb.imb_max; c.tol = tol;
        c.n_temps = (int)(temps.size() < (size_t)MAX_TEMPS ? temps.size() : MAX_TEMPS);
        for (int i = 0; i < c.n_temps; i++) c.temps[i] = temps[i];
        JET_CUDA(cudaMemcpyAsync(ctl.p, hctl, sizeof(Ctl<W>), cudaMemcpyHostToDevice, s));
    }

    void ctl_finish() {
        JET_CUDA(cudaMemcpyAsync(hctl, ctl.p, sizeof(Ctl<W>), cudaMemcpyDeviceToHost, s));
        JET_CUDA(cudaMemcpyAsync(e.hres, &dev.p->err, sizeof(int), cudaMemcpyDeviceToHost, s));
        e.sync();
        int err = *(int*)e.hres;
        if (err & ERRF_SPIN) throw JetError{JET_ERR_TIMEOUT, "a bounded device loop or grid barrier gave up"};
        if (err & ~16) throw JetError{JET_ERR_OVERFLOW, "refinement exceeded a device bound"};
        Ctl<W>& c = *hctl;
        best.cut = c.best_cut;
        best.total_imb = c.best_imb;
        curr.cut = c.curr_cut;
        curr.total_imb = c.curr_imb;
        total_iters += c.iter_count;
    }

    void run_level_cta(const Level<O, E, W>& L, part_t* best_part, const Prob& pb, const std::vector<double>& temps, double tol) {
        ctl_init(pb, temps, tol);
        LevelLists<O> li{L.warp_list.p, L.n_warp, L.hub_list.p, L.n_hub, L.group};
        RebArgs<O, W> rbw = reb_args(L, weak_max_dest(pb.size_max), pb.opt, pb.size_max, false);
        RebArgs<O, W> rbs = reb_args(L, strong_max_dest(pb.opt, pb.size_max), pb.opt, pb.size_max, false);
        int P = 1;
        while (P < (int)L.n) P <<= 1;
        size_t scratch = level_cta_smem<O, W>(P, k) + 64;
        // the attribute is per function and process-wide: always the device
        // maximum, so concurrent callers with different sizes cannot race
        const size_t smax = max_dynamic_smem((const void*)k_level_cta<O, E, W>);
        JET_CUDA(cudaFuncSetAttribute(k_level_cta<O, E, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
        // the level's table slots, as init_conn counted them
        const int64_t nslots = last_slots;
        const int64_t nbuckets = (int64_t)rbw.t_minibuckets + 1 + rbw.width;
        CtaSmemPlan plan = plan_cta_smem<O, W>((int64_t)L.n, nslots, nbuckets, k, scratch, smax, cta_smem_resident());
        k_level_cta<O, E, W><<<1, CTA_THREADS, plan.total, s>>>(args(L), li, rbw, rbs, ctl.p, best_part, sizes_best.p, P,
                                                                 1 << 22, plan);
        count_launch();
        JET_LAUNCH_CHECK();
        ctl_finish();
    }

    // ------------------------------------------------------------ cooperative loop
    // Above these the multi-kernel graph is faster (128^3 mesh: the 241,769-
    // vertex level, 3.1 M entries, runs 86 against 111 us per iteration here;
    // the 749,582-vertex level gains nothing and the 2 M one loses).
    static constexpr int64_t COOP_MAX_N = (int64_t)1 << 18;
    static constexpr int64_t COOP_MAX_M = (int64_t)1 << 22;
    size_t coop_smem() const {
        int kw = k < WARP_TABLE ? k : WARP_TABLE;
        size_t nw = CTA_THREADS / 32;
        size_t conn = ((nw * kw * sizeof(part_t) + 15) & ~(size_t)15) + nw * kw * sizeof(W);
        size_t q = (size_t)coop_boff_off() + (size_t)coop_boff_cap() * sizeof(W);
        return (conn > q ? conn : q) + 64;
    }
    // the per-block bucket offsets sit past both the queue keys and the full
    // sort's radix counters (32 warps x 256 digits), which share offset 0
    static size_t coop_boff_off() {
        size_t keys = (size_t)COOP_QUEUE_KEYS * sizeof(uint64_t);
        size_t rs = (size_t)32 * RS_BINS * sizeof(uint32_t);
        return ((keys > rs ? keys : rs) + 15) & ~(size_t)15;
    }
    // rebalance candidates block 0 of the persistent grid orders in shared memory
    // (2048 keys hold every queue seen on meshes and geometric graphs at
    // these sizes; more shared memory here would come out of the L1 cache
    // the loop's global accesses hit)
    static constexpr int COOP_QUEUE_KEYS = 2048;
    int coop_qcap() const { return COOP_QUEUE_KEYS; }
    // bucket offsets every block of the persistent grid keeps in shared
    // memory after the keys: room for the largest level the grid drivers
    // take, within 128 KiB (else those levels scan them across the grid)
    int64_t coop_boff_cap() const {
        int64_t nmax = (int64_t)n_max;
        const int64_t lim = coop_max_n() > cluster_max_n() ? coop_max_n() : cluster_max_n();
        if (nmax > lim) nmax = lim;
        O sections, tmb;
        sections_for((O)nmax, sections, tmb);
        const int64_t want = (int64_t)tmb + 1;
        return want * (int64_t)sizeof(W) <= ((int64_t)128 << 10) ? want : 0;
    }
    size_t coop_static_smem() const {
        static size_t bytes = [] {
            cudaFuncAttributes fa;
            return cudaFuncGetAttributes(&fa, k_level_coop<false, O, E, W>) == cudaSuccess ? fa.sharedSizeBytes : (size_t)1 << 30;
        }();
        return bytes;
    }
    bool coop_eligible(const Level<O, E, W>& L) const {
        return use_coop && device_info().coop && !cta_eligible(L) && (int64_t)L.n <= coop_max_n() &&
               (int64_t)L.m <= coop_max_m() && k <= WARP_TABLE &&
               coop_smem() + coop_static_smem() <= (size_t)device_info().max_smem_optin;
    }

    // ------------------------------------------------------------ cluster loop
    // Beyond these the cluster's 16 SMs lose to the whole GPU (graph driver):
    // 260 vs 131 us per iteration at 242k mesh vertices; 2x slower on dense
    // power-law levels of tens of millions of entries.
    static constexpr int64_t CLUSTER_MAX_N = (int64_t)1 << 16;
    static constexpr int64_t CLUSTER_MAX_M = (int64_t)1 << 21;
    // CTAs in the level cluster: 16 where the device allows it, else 8, 0 if
    // no cluster of 1024-thread CTAs with this shared memory fits.
    mutable int cluster_cache = -1;
    int cluster_size() const {
        if (cluster_cache >= 0) return cluster_cache;
        cluster_cache = [this] {
            const void* f = (const void*)k_level_coop<true, O, E, W>;
            if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dynamic_smem(f)) != cudaSuccess) return 0;
            cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            for (int want : {16, 8}) {
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3(want);
                cfg.blockDim = dim3(CTA_THREADS);
                cfg.dynamicSmemBytes = coop_smem();
                cudaLaunchAttribute at;
                at.id = cudaLaunchAttributeClusterDimension;
                at.val.clusterDim.x = want;
                at.val.clusterDim.y = 1;
                at.val.clusterDim.z = 1;
                cfg.attrs = &at;
                cfg.numAttrs = 1;
                int n = 0;
                if (cudaOccupancyMaxActiveClusters(&n, (void*)f, &cfg) == cudaSuccess && n > 0) return want;
            }
            cudaGetLastError();
            return 0;
        }();
        return cluster_cache;
    }
    bool cluster_eligible(const Level<O, E, W>& L) const {
        return use_cluster && !cta_eligible(L) && (int64_t)L.n <= cluster_max_n() && (int64_t)L.m <= cluster_max_m() &&
               k <= WARP_TABLE &&
               coop_smem() + coop_static_smem() <= (size_t)device_info().max_smem_optin && cluster_size() > 0;
    }

    // The whole level loop as one persistent launch: a single cluster
    // (hardware barriers) or a cooperative grid of one 1024-thread CTA per SM
    // (bounded software barriers).
    void run_level_coop(const Level<O, E, W>& L, part_t* best_part, const Prob& pb, const std::vector<double>& temps, double tol,
                        bool cluster = false) {
        size_t smem = coop_smem();
        int grid = 0;
        if (cluster) {
            grid = cluster_size();
        } else {
            JET_CUDA(cudaFuncSetAttribute(k_level_coop<false, O, E, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          max_dynamic_smem((const void*)k_level_coop<false, O, E, W>)));
            int per_sm = 0;
            JET_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_level_coop<false, O, E, W>, CTA_THREADS, smem));
            if (per_sm < 1) throw JetError{JET_ERR_CUDA, "cooperative level kernel does not fit on an SM"};
            grid = device_info().sms * per_sm;
        }
        if (cbar.n < 1) cbar.alloc(1, s);
        if (cwsum.n < grid) cwsum.alloc(grid, s);
        if (chist.n < (int64_t)grid * RS_BINS) chist.alloc((int64_t)grid * RS_BINS, s);
        if (cmarked.n < (int64_t)n_max) cmarked.alloc(n_max > 0 ? n_max : 1, s);
        JET_CUDA(cudaMemsetAsync(cbar.p, 0, sizeof(GridBar), s));
        ctl_init(pb, temps, tol);
        LevelLists<O> li{L.warp_list.p, L.n_warp, L.hub_list.p, L.n_hub, L.group};
        RebArgs<O, W> rbw = reb_args(L, weak_max_dest(pb.size_max), pb.opt, pb.size_max, false);
        RebArgs<O, W> rbs = reb_args(L, strong_max_dest(pb.opt, pb.size_max), pb.opt, pb.size_max, false);
        CoopScratch<O, E, W> cs{cbar.p, cwsum.p, chist.p, sk0.p, sk1.p, sv0.p, sv1.p, wpre.p, cmarked.p, coop_qcap(),
                                coop_boff_cap(), (int64_t)coop_boff_off()};
        int bits = bits_for((uint64_t)rbw.none_key);
        int max_iters = 1 << 22;
        RefArgs<O, E, W> a = args(L);
        Ctl<W>* cp = ctl.p;
        part_t* bp = best_part;
        W* sb = sizes_best.p;
        if (cluster) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(grid);
            cfg.blockDim = dim3(CTA_THREADS);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = s;
            cudaLaunchAttribute at;
            at.id = cudaLaunchAttributeClusterDimension;
            at.val.clusterDim.x = grid;
            at.val.clusterDim.y = 1;
            at.val.clusterDim.z = 1;
            cfg.attrs = &at;
            cfg.numAttrs = 1;
            JET_CUDA(cudaLaunchKernelEx(&cfg, k_level_coop<true, O, E, W>, a, li, rbw, rbs, cp, bp, sb, cs, bits, max_iters));
        } else {
            void* params[] = {&a, &li, &rbw, &rbs, &cp, &bp, &sb, &cs, &bits, &max_iters};
            JET_CUDA(cudaLaunchCooperativeKernel((const void*)k_level_coop<false, O, E, W>, dim3(grid), dim3(CTA_THREADS), params, smem, s));
        }
        count_launch();
        ctl_finish();
    }

    // ------------------------------------------------------------ graph-resident loop
    // Captures `fn` (which launches on this->s) into `g` after `deps` on the
    // capture stream; returns the tail nodes and the number of kernels captured.
    template <class F>
    std::vector<cudaGraphNode_t> capture_into(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, F&& fn, int64_t* nkernels) {
        cudaStream_t cs = capture_stream();
        JET_CUDA(cudaStreamBeginCaptureToGraph(cs, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                               cudaStreamCaptureModeRelaxed));
        cudaStream_t saved = s;
        s = cs;
        capturing() = true;
        int64_t l0 = launch_counter();
        try {
            fn();
        } catch (...) {
            capturing() = false;
            s = saved;
            cudaGraph_t dummy;
            cudaStreamEndCapture(cs, &dummy);
            throw;
        }
        *nkernels = launch_counter() - l0;
        capturing() = false;
        s = saved;
        cudaStreamCaptureStatus st;
        const cudaGraphNode_t* tail = nullptr;
        size_t ntail = 0;
        JET_CUDA(cudaStreamGetCaptureInfo(cs, &st, nullptr, nullptr, &tail, &ntail));
        std::vector<cudaGraphNode_t> out(tail, tail + ntail);
        cudaGraph_t gout;
        JET_CUDA(cudaStreamEndCapture(cs, &gout));
        return out;
    }

    static cudaGraphNode_t add_conditional(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, cudaGraphConditionalHandle h,
                                           cudaGraphConditionalNodeType type, cudaGraph_t* body) {
        cudaGraphNodeParams p = {};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = type;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        JET_CUDA(cudaGraphAddNode(&node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &p));
        *body = p.conditional.phGraph_out[0];
        return node;
    }

    // The refinement loop of one level as one graph launch: no host
    // round trip per iteration (the reference syncs about three times per
    // iteration, src/jet_refiner.hpp:199, :416, :550, :904).
    void run_level_graph(const Level<O, E, W>& L, part_t* best_part, const Prob& pb, const std::vector<double>& temps, double tol) {
        Ctl<W>& c = *hctl;
        std::memset(&c, 0, sizeof(c));
        c.curr_cut = curr.cut; c.curr_imb = curr.total_imb; c.best_cut = best.cut; c.best_imb = best.total_imb;
        c.opt = pb.opt; c.imb_max = pb.imb_max; c.tol = tol;
        c.n_temps = (int)(temps.size() < (size_t)MAX_TEMPS ? temps.size() : MAX_TEMPS);
        for (int i = 0; i < c.n_temps; i++) c.temps[i] = temps[i];
        JET_CUDA(cudaMemcpyAsync(ctl.p, hctl, sizeof(Ctl<W>), cudaMemcpyHostToDevice, s));
        set_attrs();
        cudaGraph_t G;
        JET_CUDA(cudaGraphCreate(&G, 0));
        cudaGraphExec_t X = nullptr;
        try {
            CtlHandles h;
            JET_CUDA(cudaGraphConditionalHandleCreate(&h.loop, G, 0, cudaGraphCondAssignDefault));
            JET_CUDA(cudaGraphConditionalHandleCreate(&h.lp, G, 0, cudaGraphCondAssignDefault));
            JET_CUDA(cudaGraphConditionalHandleCreate(&h.weak, G, 0, cudaGraphCondAssignDefault));
            JET_CUDA(cudaGraphConditionalHandleCreate(&h.strong, G, 0, cudaGraphCondAssignDefault));
            JET_CUDA(cudaGraphConditionalHandleCreate(&h.copy, G, 0, cudaGraphCondAssignDefault));
            // the rebalance bodies end in an IF node holding the full sort,
            // which k_reb_ordered opens when the queue cannot be used
            // (a handle must belong to a node: made only where the IF exists)
            RebArgs<O, W> rbw = reb_args(L, weak_max_dest(pb.size_max), pb.opt, pb.size_max, false);
            RebArgs<O, W> rbs = reb_args(L, strong_max_dest(pb.opt, pb.size_max), pb.opt, pb.size_max, false);
            cudaGraphConditionalHandle fbw = 0, fbs = 0;
            if (rbw.queue) JET_CUDA(cudaGraphConditionalHandleCreate(&fbw, G, 0, cudaGraphCondAssignDefault));
            if (rbs.queue) JET_CUDA(cudaGraphConditionalHandleCreate(&fbs, G, 0, cudaGraphCondAssignDefault));
            JET_CUDA(cudaMemsetAsync(dev.p->reb_fb_count, 0, 2 * sizeof(int), s));
            int64_t kb = 0, klp = 0, kw = 0, ks = 0, km = 0, kfw = 0, kfs = 0;
            Ctl<W>* cp = ctl.p;
            auto t0 = capture_into(G, {}, [&] { k_ctl_begin<W><<<1, 1, 0, s>>>(cp, h); count_launch(); JET_LAUNCH_CHECK(); }, &kb);
            cudaGraph_t body, b_lp, b_weak, b_strong, b_copy, b_fbw, b_fbs;
            add_conditional(G, t0, h.loop, cudaGraphCondTypeWhile, &body);
            cudaGraphNode_t n_lp = add_conditional(body, {}, h.lp, cudaGraphCondTypeIf, &b_lp);
            capture_into(b_lp, {}, [&] { lp(L); }, &klp);
            cudaGraphNode_t n_weak = add_conditional(body, {n_lp}, h.weak, cudaGraphCondTypeIf, &b_weak);
            auto tw = capture_into(b_weak, {}, [&] {
                rbw = reb_args(L, weak_max_dest(pb.size_max), pb.opt, pb.size_max);
                weak_select(L, rbw);
                if (rbw.queue) reb_queue<false>(L, rbw, fbw, true);
                else weak_full(L, rbw);
            }, &kw);
            if (rbw.queue) {
                add_conditional(b_weak, tw, fbw, cudaGraphCondTypeIf, &b_fbw);
                capture_into(b_fbw, {}, [&] { weak_full(L, rbw); }, &kfw);
            }
            cudaGraphNode_t n_strong = add_conditional(body, {n_weak}, h.strong, cudaGraphCondTypeIf, &b_strong);
            auto ts = capture_into(b_strong, {}, [&] {
                rbs = reb_args(L, strong_max_dest(pb.opt, pb.size_max), pb.opt, pb.size_max);
                strong_select(L, rbs);
                if (rbs.queue) reb_queue<true>(L, rbs, fbs, true);
                else strong_full(L, rbs);
            }, &ks);
            if (rbs.queue) {
                add_conditional(b_strong, ts, fbs, cudaGraphCondTypeIf, &b_fbs);
                capture_into(b_fbs, {}, [&] { strong_full(L, rbs); }, &kfs);
            }
            // (the update_small / update_large kernels all run and test the
            // device-side decision: conditional nodes around them cost more
            // than the kernels that return at once)
            auto tm = capture_into(body, {n_strong}, [&] {
                apply_moves_kernel(L);
                int hp = prof_begin(s);
                small_update_kernels(L);
                large_update_kernels(L);
                prof_end(hp, PK_UPDATE, 0, s);
                k_cut_finalize_ctl<O, E, W><<<grid_persistent(L.n, 8), BLOCK, 0, s>>>(args(L), cp, h, cdone.p); count_launch();
                JET_LAUNCH_CHECK();
            }, &km);
            add_conditional(body, tm, h.copy, cudaGraphCondTypeIf, &b_copy);
            int64_t kc = 0;
            capture_into(b_copy, {}, [&] {
                JET_CUDA(cudaMemcpyAsync(best_part, part_work.p, sizeof(part_t) * L.n, cudaMemcpyDeviceToDevice, s));
                JET_CUDA(cudaMemcpyAsync(sizes_best.p, sizes_curr.p, sizeof(W) * k, cudaMemcpyDeviceToDevice, s));
            }, &kc);
            JET_CUDA(cudaGraphInstantiate(&X, G, 0));
            JET_CUDA(cudaGraphLaunch(X, s));
            JET_CUDA(cudaMemcpyAsync(hctl, ctl.p, sizeof(Ctl<W>), cudaMemcpyDeviceToHost, s));
            JET_CUDA(cudaMemcpyAsync(e.hres, &dev.p->err, sizeof(int), cudaMemcpyDeviceToHost, s));
            JET_CUDA(cudaMemcpyAsync(e.hscal, dev.p->reb_fb_count, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
            e.sync();
            // kernels the graph ran: captured once, executed once per iteration
            // of their kind, the full sorts once per fallback
            const int* nfb = (const int*)e.hscal;
            add_launches(kb + klp * c.lab_counter + kw * c.weak_iters + ks * c.strong_iters + km * c.iter_count +
                         kfw * nfb[0] + kfs * nfb[1] - (kb + klp + kw + ks + km + kfw + kfs));
        } catch (...) {
            if (X) cudaGraphExecDestroy(X);
            cudaGraphDestroy(G);
            throw;
        }
        cudaGraphExecDestroy(X);
        cudaGraphDestroy(G);
        if (*(int*)e.hres & ~16) throw JetError{JET_ERR_OVERFLOW, "connectivity table update exceeded its bounds"};
        best.cut = c.best_cut;
        best.total_imb = c.best_imb;
        curr.cut = c.curr_cut;
        curr.total_imb = c.curr_imb;
        total_iters += c.iter_count;
    }

    // jet_refine, src/jet_refiner.hpp:1050-1142.  best_part in/out.
    jet_level_stats_c refine(const Level<O, E, W>& L, part_t* best_part, double imb, double tol, bool ultra) {
        auto t0 = clk::now();
        Prob pb = begin_level(L, best_part, imb);
        auto t1 = clk::now();
        std::vector<double> temps;
        if (ultra) { for (double t = 0.85; t > 0; t -= 0.05) temps.push_back(t); }
        else if (L.uniform) temps.push_back(0.25);
        else temps.push_back(0.75);
        if (cta_eligible(L) || cluster_eligible(L) || coop_eligible(L) || use_graph) {
            if (cta_eligible(L)) run_level_cta(L, best_part, pb, temps, tol);
            else if (cluster_eligible(L)) run_level_coop(L, best_part, pb, temps, tol, true);
            else if (coop_eligible(L)) run_level_coop(L, best_part, pb, temps, tol);
            else run_level_graph(L, best_part, pb, temps, tol);
            jet_level_stats_c cl;
            cl.edge_cut = (int64_t)(best.cut / 2);
            cl.imb = (double)best.total_imb / (double)pb.opt;
            cl.num_edges = (uint64_t)L.m;
            cl.num_vertices = (uint64_t)L.n;
            cl.total_ref_time = since(t0);
            cl.iterations_time = since(t1);
            cl.total_iterations = hctl->iter_count;
            cl.lp_iterations = hctl->lab_counter;
            return cl;
        }
        int iter_count = 0, balance_counter = 0, lab_counter = 0;
        for (double fr : temps) {
            int count = 0;
            while (count++ <= 11) {
                iter_count++;
                iterate(L, pb, fr, balance_counter, lab_counter);
                if (best.total_imb > pb.imb_max && curr.total_imb < best.total_imb) {
                    save_best(L, best_part);
                    count = 0;
                } else if (curr.cut < best.cut && (curr.total_imb <= pb.imb_max || curr.total_imb <= best.total_imb)) {
                    if ((double)curr.cut < tol * (double)best.cut) count = 0;
                    save_best(L, best_part);
                }
            }
        }
        e.sync();
        jet_level_stats_c cl;
        cl.edge_cut = (int64_t)(best.cut / 2);
        cl.imb = (double)best.total_imb / (double)pb.opt;
        cl.num_edges = (uint64_t)L.m;
        cl.num_vertices = (uint64_t)L.n;
        cl.total_ref_time = since(t0);
        cl.iterations_time = since(t1);
        cl.total_iterations = iter_count;
        cl.lp_iterations = lab_counter;
        return cl;
    }
};

// ---------------------------------------------------------------- partition
template <class O, class E, class W>
struct GraphIn {
    O n;
    E m;
    const E* row;
    const O* adj;
    const W* val;
    const W* vw;
    bool uniform;
};

// metis_init, src/initial_partition.hpp:92-114: values pass through `int`
// as in the reference, then widen to this Metis build's 64-bit idx_t.
template <class O, class E, class W>
void metis_coarsest(const Level<O, E, W>& L, part_t k, double imb, part_t* part_dev, cudaStream_t s) {
    std::vector<E> row(L.n + 1);
    std::vector<O> adj(L.m);
    std::vector<W> val(L.m), vw(L.n);
    JET_CUDA(cudaMemcpyAsync(row.data(), L.row, sizeof(E) * (L.n + 1), cudaMemcpyDeviceToHost, s));
    if (L.m) {
        JET_CUDA(cudaMemcpyAsync(adj.data(), L.adj, sizeof(O) * L.m, cudaMemcpyDeviceToHost, s));
        JET_CUDA(cudaMemcpyAsync(val.data(), L.val, sizeof(W) * L.m, cudaMemcpyDeviceToHost, s));
    }
    JET_CUDA(cudaMemcpyAsync(vw.data(), L.vw, sizeof(W) * L.n, cudaMemcpyDeviceToHost, s));
    stream_wait(s);
    std::vector<int64_t> xadj(L.n + 1), madj(L.m), madjw(L.m), mvw(L.n), pm(L.n > 0 ? L.n : 1, 0);
    // the reference hands Metis int arrays (src/initial_partition.hpp:65, :103-105)
    for (O i = 0; i <= L.n; i++) xadj[i] = (int)row[i];
    for (E j = 0; j < L.m; j++) { madj[j] = (int)adj[j]; madjw[j] = (int)val[j]; }
    for (O i = 0; i < L.n; i++) mvw[i] = (int)vw[i];
    int64_t obj = 0;
    int ret = metis_kway((int64_t)L.n, (int64_t)L.m, xadj.data(), madj.data(), mvw.data(), madjw.data(), (int64_t)k,
                         (float)imb, &obj, pm.data());
    if (ret != 1) throw JetError{JET_ERR_METIS, "Metis could not partition coarsest graph"};
    std::vector<part_t> p(L.n);
    for (O i = 0; i < L.n; i++) p[i] = (part_t)pm[i];
    JET_CUDA(cudaMemcpyAsync(part_dev, p.data(), sizeof(part_t) * L.n, cudaMemcpyHostToDevice, s));
    stream_wait(s);
}

struct Cfg {
    int alg;
    part_t k;
    double imb;
    double tol;
    bool ultra;
    bool verbose;
    bool dump = false;  // config_t::dump_coarse
};

// Writes the hierarchy levels[0..last] in the reference's binary layout
// (src/binary_dump.hpp:61-90): int32 level count, then per level N, M,
// row_map[N+1], entries[M], values[M], vertex weights[N] (tier types) and,
// from the second level on, the map from the previous level.
template <class O, class E, class W>
void dump_hierarchy(const std::vector<std::unique_ptr<Level<O, E, W>>>& levels, int last, const char* path, cudaStream_t s) {
    FILE* f = fopen(path, "wb");
    if (!f) throw JetError{JET_ERR_INVALID, "cannot open the hierarchy dump file"};
    int size = last + 1;
    bool ok = fwrite(&size, sizeof(int), 1, f) == 1;
    for (int l = 0; ok && l <= last; l++) {
        const Level<O, E, W>& L = *levels[l];
        O n = L.n;
        E m = L.m;
        std::vector<E> row(n + 1);
        std::vector<O> adj(m), map(l > 0 ? levels[l - 1]->n : 0);
        std::vector<W> val(m), vw(n);
        JET_CUDA(cudaMemcpyAsync(row.data(), L.row, sizeof(E) * (n + 1), cudaMemcpyDeviceToHost, s));
        if (m) {
            JET_CUDA(cudaMemcpyAsync(adj.data(), L.adj, sizeof(O) * m, cudaMemcpyDeviceToHost, s));
            JET_CUDA(cudaMemcpyAsync(val.data(), L.val, sizeof(W) * m, cudaMemcpyDeviceToHost, s));
        }
        if (n) JET_CUDA(cudaMemcpyAsync(vw.data(), L.vw, sizeof(W) * n, cudaMemcpyDeviceToHost, s));
        if (!map.empty()) JET_CUDA(cudaMemcpyAsync(map.data(), L.map.p, sizeof(O) * map.size(), cudaMemcpyDeviceToHost, s));
        stream_wait(s);
        ok = fwrite(&n, sizeof(O), 1, f) == 1 && fwrite(&m, sizeof(E), 1, f) == 1 &&
             fwrite(row.data(), sizeof(E), n + 1, f) == (size_t)(n + 1) && fwrite(adj.data(), sizeof(O), m, f) == (size_t)m &&
             fwrite(val.data(), sizeof(W), m, f) == (size_t)m && fwrite(vw.data(), sizeof(W), n, f) == (size_t)n &&
             fwrite(map.data(), sizeof(O), map.size(), f) == map.size();
    }
    if (fclose(f) != 0) ok = false;
    if (!ok) throw JetError{JET_ERR_INVALID, "writing the hierarchy dump failed"};
}

// The partition of one level as part_t values (src/binary_dump.hpp:91-97).
inline void dump_part(const part_t* part_dev, int64_t n, const char* path, cudaStream_t s) {
    std::vector<part_t> h(n);
    if (n) JET_CUDA(cudaMemcpyAsync(h.data(), part_dev, sizeof(part_t) * n, cudaMemcpyDeviceToHost, s));
    stream_wait(s);
    FILE* f = fopen(path, "wb");
    bool ok = f && fwrite(h.data(), sizeof(part_t), n, f) == (size_t)n;
    if (f && fclose(f) != 0) ok = false;
    if (!ok) throw JetError{JET_ERR_INVALID, "writing the coarse partition dump failed"};
}

// multilevel_jet + uncoarsen (src/uncoarsen.hpp:88-158): refine from the
// coarsest level down, projecting between levels.  `pa` holds the coarsest
// partition; `pb` is a second buffer of the finest size.  With cfg.dump the
// hierarchy and partition are written, as the reference does, at the first
// level (from the coarsest) whose partition is balanced before refinement.
template <class O, class E, class W>
W uncoarsen_levels(Engine<O, E, W>& eng, const Cfg& cfg, std::vector<std::unique_ptr<Level<O, E, W>>>& levels, DBuf<part_t>& pa,
                   DBuf<part_t>& pb, part_t* part_out, jet_stats_c* st, double* meas, clk::time_point t_start,
                   double t_coarsen, int64_t coarsest_n) {
    cudaStream_t s = eng.s;
    part_t k = cfg.k;
    Level<O, E, W>& L0 = *levels[0];
    auto tr = clk::now();
    Refiner<O, E, W> ref(eng, L0.n, (int64_t)L0.m, k);
    ref.verbose = cfg.verbose;
    ref.set_weight_bound(L0);
    part_t* cur_part = pa.p;
    part_t* other = pb.p;
    int nl = (int)levels.size();
    if (st) st->num_levels = nl;
    bool dumped = !cfg.dump;
    for (int l = nl - 1; l >= 0; l--) {
        if (!dumped) {
            // src/uncoarsen.hpp:96-111 (imbalance as get_max_imb, :69-80)
            Level<O, E, W>& L = *levels[l];
            ref.part_sizes(L, cur_part, ref.sizes_curr.p);
            std::vector<W> hs(k);
            JET_CUDA(cudaMemcpyAsync(hs.data(), ref.sizes_curr.p, sizeof(W) * k, cudaMemcpyDeviceToHost, s));
            eng.sync();
            W mx = 0, tot = 0;
            for (W x : hs) { if (x > mx) mx = x; tot += x; }
            O opt = (O)(((O)tot + k - 1) / k);
            if ((double)mx / (double)opt <= cfg.imb) {
                dump_part(cur_part, (int64_t)L.n, "coarse_part.out", s);
                dump_hierarchy<O, E, W>(levels, l, "coarse_graphs.out", s);
                dumped = true;
            }
        }
        jet_level_stats_c cl = ref.refine(*levels[l], cur_part, cfg.imb, cfg.tol, cfg.ultra);
        int idx = nl - 1 - l;
        if (st && idx < JET_MAX_LEVELS) st->levels[idx] = cl;
        if (l > 0) {
            Level<O, E, W>& fine = *levels[l - 1];
            k_project<O><<<grid_persistent(fine.n, 16), BLOCK, 0, s>>>(fine.n, levels[l]->map.p, cur_part, other); count_launch();
            JET_LAUNCH_CHECK();
            std::swap(cur_part, other);
            if (l - 1 > 0) { levels[l].reset(); }
        }
    }
    eng.sync();
    meas[M_REFINE] += since(tr);
    JET_CUDA(cudaMemcpyAsync(part_out, cur_part, sizeof(part_t) * L0.n, cudaMemcpyDeviceToDevice, s));
    W cut_half = ref.best.cut / 2;
    if (st) {
        std::vector<W> hs(k);
        JET_CUDA(cudaMemcpyAsync(hs.data(), ref.sizes_best.p, sizeof(W) * k, cudaMemcpyDeviceToHost, s));
        eng.sync();
        W largest = 0, smallest = ref.best.total_size;
        for (W x : hs) { if (x > largest) largest = x; if (x < smallest) smallest = x; }
        double opt = (double)(O)(((O)ref.best.total_size + k - 1) / k);
        st->edge_cut = (int64_t)cut_half;
        st->imb_ratio = (double)largest / opt;
        st->largest_part = (int64_t)largest;
        st->smallest_part = (int64_t)smallest;
        st->coarsest_vertices = coarsest_n;
        st->refine_iterations = ref.total_iters;
        meas[M_COARSEN] = t_coarsen;
        meas[M_TOTAL] = since(t_start);
        for (int i = 0; i < JET_NUM_MEASUREMENTS; i++) st->measurements[i] = meas[i];
    }
    eng.sync();
    return cut_half;
}

template <class O, class E, class W>
W run_partition(Engine<O, E, W>& eng, const Cfg& cfg, const GraphIn<O, E, W>& in, uint64_t seed, part_t* part_out,
                jet_stats_c* st) {
    cudaStream_t s = eng.s;
    auto t_start = clk::now();
    double meas[JET_NUM_MEASUREMENTS] = {0};
    part_t k = cfg.k;
    std::vector<std::unique_ptr<Level<O, E, W>>> levels;
    levels.emplace_back(new Level<O, E, W>());
    Level<O, E, W>& L0 = *levels[0];
    L0.n = in.n; L0.m = in.m; L0.row = in.row; L0.adj = in.adj; L0.val = in.val; L0.vw = in.vw; L0.uniform = in.uniform;
    eng.prepare_level(L0);
    eng.narrow_w = -1;  // set from this graph's finest level by the first contraction
    // coarsening cutoff, src/partitioner.hpp:88-94
    int cutoff = k * 8;
    if (cutoff > 1024) { cutoff = k * 2; cutoff = cutoff > 1024 ? cutoff : 1024; }
    O min_allowed = cutoff / 4;
    int alg = cfg.alg;
    if (alg < 0 || alg > 2) alg = 0;
    DBuf<O> skey(L0.m > 0 ? L0.m : 1, s);
    DBuf<W> sval(L0.m > 0 ? L0.m : 1, s);
    if (debug_timing()) {
        eng.sync();
        fprintf(stderr, "jet: finest level prepared %.3f ms\n", since(t_start) * 1e3);
    }
    // level loop, src/contract.hpp:494-533
    while (levels.back()->n > (O)cutoff) {
        Level<O, E, W>& cur = *levels.back();
        DBuf<O> map(cur.n, s);
        auto tm = clk::now();
        int h = prof_begin(s);
        O nc = eng.coarsen_map(cur, alg, seed, (int)levels.size(), map.p, nullptr, meas);
        prof_end(h, PK_HEC, 0, s);
        meas[M_MAP] += since(tm);
        if (debug_timing())
            fprintf(stderr, "jet: level %d n %lld m %lld map %.3f ms nc %lld\n", (int)levels.size(), (long long)cur.n,
                    (long long)cur.m, since(tm) * 1e3, (long long)nc);
        if (nc < min_allowed) break;
        auto tb = clk::now();
        std::unique_ptr<Level<O, E, W>> next(new Level<O, E, W>());
        h = prof_begin(s);
        eng.contract(cur, map.p, nc, *next, &skey, &sval);
        prof_end(h, PK_CONTRACT, 0, s);
        next->map = std::move(map);
        eng.prepare_level(*next);
        meas[M_BUILD] += since(tb);
        if (debug_timing()) fprintf(stderr, "jet: level %d contract+prepare %.3f ms\n", (int)levels.size(), since(tb) * 1e3);
        levels.push_back(std::move(next));
        if (levels.size() > 200) break;
    }
    double t_rel0 = since(t_start);
    skey.release();
    sval.release();
    double t_rel1 = since(t_start);
    eng.sync();
    double t_coarsen = since(t_start);
    if (debug_timing())
        fprintf(stderr, "jet: coarsening done %.3f ms (loop end %.3f, after release %.3f)\n", t_coarsen * 1e3, t_rel0 * 1e3,
                t_rel1 * 1e3);
    // initial partition
    auto ti = clk::now();
    Level<O, E, W>& coarsest = *levels.back();
    const int64_t coarsest_n = (int64_t)coarsest.n;
    DBuf<part_t> pa(L0.n > 0 ? L0.n : 1, s), pb(L0.n > 0 ? L0.n : 1, s);
    metis_coarsest(coarsest, k, cfg.imb, pa.p, s);
    meas[M_INITPARTITION] += since(ti);
    return uncoarsen_levels<O, E, W>(eng, cfg, levels, pa, pb, part_out, st, meas, t_start, t_coarsen, coarsest_n);
}

}  // namespace jetb
