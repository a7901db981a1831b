// partitioner.cuh -- host orchestration: coarsening level loop, Metis on the
// coarsest graph, uncoarsening with Jet refinement and projection.
// Mirrors src/partitioner.hpp, src/contract.hpp:448-533,
// src/uncoarsen.hpp:88-158 and src/jet_refiner.hpp:1050-1142.
#pragma once
#include <chrono>
#include <vector>
#include <memory>
#include "coarsen.cuh"
#include "contract.cuh"
#include "refine.cuh"
#include "../../include/jet_b200.h"


namespace jetb {

struct JetError {
    int code;
    const char* what;
};

using clk = std::chrono::steady_clock;
inline double since(clk::time_point a) { return std::chrono::duration<double>(clk::now() - a).count(); }

// Measurement slots, header/experiment_data.hpp:50-72.
enum Meas { M_MAP = 0, M_BUILD, M_COUNT, M_PREFIX, M_BUCKET, M_DEDUPE, M_RADIXSORT, M_RADIXDEDUPE, M_WRITEGRAPH, M_PERMUTE,
            M_MAPCONSTRUCT, M_HEAVY, M_INITTRANSFER, M_HASHMAPALLOC, M_HASHMAPINSERT, M_INITPARTITION, M_COARSEN, M_REFINE,
            M_FREEGRAPH, M_TOTAL };

template <class O, class E, class W>
struct Engine {
    cudaStream_t s;
    ScanScratch scan;
    RadixScratch rsort;
    DBuf<int64_t> dscal;   // small device scalars
    int64_t* hscal = nullptr;  // pinned mirror
    IterResult* hres = nullptr;
    int slot0 = -1;

    // side streams for the independent contraction bins of large levels
    // (made on first use), with the fork and join events
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[3] = {nullptr, nullptr, nullptr};

    explicit Engine(cudaStream_t st) : s(st) {
        dscal.alloc(64, s);
        slot0 = pinned_acquire(64 * sizeof(int64_t) + sizeof(IterResult) + 64);
        hscal = (int64_t*)pinned_ptr(slot0);
        hres = (IterResult*)(hscal + 64);
    }
    ~Engine() {
        cudaStreamSynchronize(s);
        for (int i = 0; i < 3; i++) {
            if (side[i]) { cudaStreamSynchronize(side[i]); cudaStreamDestroy(side[i]); }
            if (ev_join[i]) cudaEventDestroy(ev_join[i]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        pinned_release(slot0);
    }
    bool side_streams() {
        if (ev_fork) return true;
        for (int i = 0; i < 3; i++) {
            if (cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&ev_join[i], cudaEventDisableTiming) != cudaSuccess)
                return false;
        }
        return cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) == cudaSuccess;
    }
    template <class T> T* dslot(int i) { return (T*)(dscal.p + i); }
    void sync() { stream_wait(s); }
    // copies `cnt` device scalars starting at slot 0 to the host mirror
    void pull(int cnt) {
        JET_CUDA(cudaMemcpyAsync(hscal, dscal.p, sizeof(int64_t) * cnt, cudaMemcpyDeviceToHost, s));
        sync();
    }

    // ------------------------------------------------------------ level prep
    void prepare_level(Level<O, E, W>& L) {
        L.warp_list.alloc(L.n > 0 ? L.n : 1, s);
        L.hub_list.alloc(L.n > 0 ? L.n : 1, s);
        JET_CUDA(cudaMemsetAsync(dscal.p, 0, 3 * sizeof(int64_t), s));
        if (L.n > 0) {
            k_bin_degrees<O, E><<<grid_persistent(L.n, 8), BLOCK, 0, s>>>(L.n, L.row, L.warp_list.p, dslot<O>(0), L.hub_list.p,
                                                                          dslot<O>(1), dslot<E>(2)); count_launch();
            JET_LAUNCH_CHECK();
        }
        pull(3);
        L.n_warp = *(O*)&hscal[0];
        L.n_hub = *(O*)&hscal[1];
        L.max_deg = *(E*)&hscal[2];
        double avg = L.n > 0 ? (double)L.m / (double)L.n : 0.0;
        L.group = group_for_avg_degree(avg);
    }

    // ------------------------------------------------------------ coarsening
    O hec_map(Level<O, E, W>& L, uint64_t seed, int level, O* vcmap, O* hn_out, double* t_heavy, double* t_construct) {
        auto g = L.view();
        O n = L.n;
        DBuf<O> hn_own;
        O* hn = hn_out;
        if (!hn) { hn_own.alloc(n, s); hn = hn_own.p; }
        auto t0 = clk::now();
        if (L.uniform) {
            k_hec_uniform<O, E, W><<<grid_persistent(n, 16), BLOCK, 0, s>>>(g, seed, rng_stream(level, RNG_HEC_RANDOM, 0), hn); count_launch();
            JET_LAUNCH_CHECK();
        } else {
            W* vsum = dslot<W>(8);
            JET_CUDA(cudaMemsetAsync(vsum, 0, sizeof(int64_t), s));
            k_sum<W><<<grid_persistent(n, 8), BLOCK, 0, s>>>(g.vw, n, vsum); count_launch();
            JET_LAUNCH_CHECK();
            unsigned grid = grid_persistent((int64_t)n * L.group, 16);
            switch (L.group) {
                case 4: k_hec_heavy<4, O, E, W><<<grid, BLOCK, 0, s>>>(g, vsum, hn); count_launch(); break;
                case 8: k_hec_heavy<8, O, E, W><<<grid, BLOCK, 0, s>>>(g, vsum, hn); count_launch(); break;
                case 16: k_hec_heavy<16, O, E, W><<<grid, BLOCK, 0, s>>>(g, vsum, hn); count_launch(); break;
                default: k_hec_heavy<32, O, E, W><<<grid, BLOCK, 0, s>>>(g, vsum, hn); count_launch(); break;
            }
            JET_LAUNCH_CHECK();
            if (L.n_hub > 0) {
                k_hec_heavy_hub<O, E, W><<<grid_for(L.n_hub, 1), 1024, 0, s>>>(g, vsum, L.hub_list.p, L.n_hub, hn); count_launch();
                JET_LAUNCH_CHECK();
            }
        }
        if (t_heavy) { sync(); *t_heavy += since(t0); }
        auto t1 = clk::now();
        hec_aggregate(n, hn, vcmap);
        O nc = number_roots(vcmap, n);
        if (t_construct) *t_construct += since(t1);
        return nc;
    }

    // parallel_map_construct (src/heuristics.hpp:89-169) with the result of its
    // in-order execution; vcmap receives each vertex's root.
    void hec_aggregate(O n, const O* hn, O* vcmap) {
        fill<O>(vcmap, n, ord_max<O>(), s);
        DBuf<O> nxt(n, s), cnt(n, s), min_free(n, s);
        DBuf<int> has_free(n, s);
        DBuf<uint8_t> inB(n, s);
        unsigned grid = grid_persistent(n, 16);
        k_hec_p1_init<O><<<grid, BLOCK, 0, s>>>(n, hn, nxt.p, vcmap); count_launch();
        JET_LAUNCH_CHECK();
        int* changed = dslot<int>(18);
        for (int round = 0;; round++) {
            JET_CUDA(cudaMemsetAsync(changed, 0, sizeof(int64_t), s));
            k_hec_p1_jump<O><<<grid, BLOCK, 0, s>>>(n, nxt.p, changed); count_launch();
            JET_LAUNCH_CHECK();
            JET_CUDA(cudaMemcpyAsync(hscal, changed, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
            sync();
            if (*(int*)hscal == 0) break;
            if (round > 64) throw JetError{JET_ERR_TIMEOUT, "HEC pointer jumping did not converge"};
        }
        k_hec_p1_final<O><<<grid, BLOCK, 0, s>>>(n, nxt.p, vcmap); count_launch();
        cnt.zero();
        k_hec_p2_count<O><<<grid, BLOCK, 0, s>>>(n, hn, vcmap, inB.p, cnt.p, min_free.p, has_free.p); count_launch();
        k_hec_p2_walk<O><<<grid, BLOCK, 0, s>>>(n, hn, inB.p, cnt.p, min_free.p, has_free.p); count_launch();
        k_hec_p2_roots<O><<<grid, BLOCK, 0, s>>>(n, hn, inB.p, min_free.p, has_free.p, vcmap); count_launch();
        JET_LAUNCH_CHECK();
    }

    O number_roots(O* vcmap, O n) {
        DBuf<O> ids(n + 1, s);
        O* total = dslot<O>(20);
        exclusive_scan<O, GetIsRoot<O>>(GetIsRoot<O>{vcmap}, n, ids.p, total, scan, s);
        k_assign_ids<O><<<grid_persistent(n, 16), BLOCK, 0, s>>>(n, ids.p, vcmap); count_launch();
        JET_LAUNCH_CHECK();
        JET_CUDA(cudaMemcpyAsync(hscal, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        sync();
        return *(O*)hscal;
    }

    template <bool INITIAL, bool UNIFORM>
    void pick(Level<O, E, W>& L, const O* perm, const O* perm_len, O max_len, const O* vcmap, O* hn, uint64_t seed, uint64_t stream) {
        auto g = L.view();
        unsigned grid = grid_persistent((int64_t)max_len * L.group, 16);
        switch (L.group) {
            case 4: k_pick_match<4, INITIAL, UNIFORM, O, E, W><<<grid, BLOCK, 0, s>>>(g, perm, perm_len, vcmap, hn, seed, stream); count_launch(); break;
            case 8: k_pick_match<8, INITIAL, UNIFORM, O, E, W><<<grid, BLOCK, 0, s>>>(g, perm, perm_len, vcmap, hn, seed, stream); count_launch(); break;
            case 16: k_pick_match<16, INITIAL, UNIFORM, O, E, W><<<grid, BLOCK, 0, s>>>(g, perm, perm_len, vcmap, hn, seed, stream); count_launch(); break;
            default: k_pick_match<32, INITIAL, UNIFORM, O, E, W><<<grid, BLOCK, 0, s>>>(g, perm, perm_len, vcmap, hn, seed, stream); count_launch(); break;
        }
        JET_LAUNCH_CHECK();
        if (L.n_hub > 0) {
            k_pick_match_hub<INITIAL, UNIFORM, O, E, W><<<grid_for(L.n_hub, 1), 1024, 0, s>>>(g, L.hub_list.p, L.n_hub, vcmap, hn, seed, stream); count_launch();
            JET_LAUNCH_CHECK();
        }
    }

    // coarsen_match, src/heuristics.hpp:427-671.
    O match_map(Level<O, E, W>& L, bool two_hop, uint64_t seed, int level, O* vcmap, O* hn_init_out) {
        auto g = L.view();
        O n = L.n;
        const O MAXV = ord_max<O>();
        DBuf<O> hn(n, s);
        fill<O>(hn.p, n, MAXV, s);
        fill<O>(vcmap, n, MAXV, s);
        if (L.uniform) {
            k_match_uniform_init<O, E, W><<<grid_persistent(n, 16), BLOCK, 0, s>>>(g, seed, rng_stream(level, RNG_MATCH_RANDOM, 0), hn.p); count_launch();
            JET_LAUNCH_CHECK();
        } else {
            pick<true, false>(L, nullptr, nullptr, n, vcmap, hn.p, seed, rng_stream(level, RNG_MATCH_PICK, 0));
        }
        if (hn_init_out) JET_CUDA(cudaMemcpyAsync(hn_init_out, hn.p, sizeof(O) * n, cudaMemcpyDeviceToDevice, s));
        DBuf<O> perm_a(n, s), perm_b(n, s), winner(n, s);
        O* cur = nullptr;
        O* cur_len = dslot<O>(16);
        O* nxt_len = dslot<O>(17);
        O len = n;
        int outer = 0;
        while (len > 0) {
            unsigned grid = grid_persistent(len, 16);
            for (int r = 0; r < 4; r++) {
                k_commit1<O><<<grid, BLOCK, 0, s>>>(n, cur, cur_len, hn.p, vcmap, winner.p, r); count_launch();
                k_commit2a<O><<<grid, BLOCK, 0, s>>>(n, cur, cur_len, hn.p, vcmap, winner.p); count_launch();
                k_commit2<O><<<grid, BLOCK, 0, s>>>(n, cur, cur_len, hn.p, vcmap, winner.p); count_launch();
                k_commit3<O><<<grid, BLOCK, 0, s>>>(n, cur, cur_len, vcmap); count_launch();
                JET_LAUNCH_CHECK();
            }
            outer++;
            uint64_t st = rng_stream(level, RNG_MATCH_PICK, outer);
            if (L.uniform) pick<false, true>(L, cur, cur_len, len, vcmap, hn.p, seed, st);
            else pick<false, false>(L, cur, cur_len, len, vcmap, hn.p, seed, st);
            O* nxt = (cur == perm_a.p) ? perm_b.p : perm_a.p;
            JET_CUDA(cudaMemsetAsync(nxt_len, 0, sizeof(int64_t), s));
            k_match_remaining<O><<<grid, BLOCK, 0, s>>>(n, cur, cur_len, hn.p, vcmap, nxt, nxt_len); count_launch();
            JET_LAUNCH_CHECK();
            JET_CUDA(cudaMemcpyAsync(cur_len, nxt_len, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
            JET_CUDA(cudaMemcpyAsync(hscal, nxt_len, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
            sync();
            len = *(O*)hscal;
            cur = nxt;
            if (outer > 100000) throw JetError{JET_ERR_TIMEOUT, "matching did not settle"};
        }
        if (debug_timing()) fprintf(stderr, "jet:   matching n %lld outer %d\n", (long long)n, outer);
        if (two_hop) two_hop_passes(L, vcmap);
        k_singletons<O><<<grid_persistent(n, 16), BLOCK, 0, s>>>(n, vcmap); count_launch();
        JET_LAUNCH_CHECK();
        return number_roots(vcmap, n);
    }

    O count_unmatched(O n, const O* vcmap) {
        O* c = dslot<O>(24);
        JET_CUDA(cudaMemsetAsync(c, 0, sizeof(int64_t), s));
        k_count_unmatched<O><<<grid_persistent(n, 8), BLOCK, 0, s>>>(n, vcmap, c); count_launch();
        JET_LAUNCH_CHECK();
        JET_CUDA(cudaMemcpyAsync(hscal, c, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        sync();
        return *(O*)hscal;
    }

    // Unmatched vertices (leaves only: of degree 1) in vertex order; pos_out,
    // if given, receives each vertex's position in the list.
    O unmatched_list(Level<O, E, W>& L, const O* vcmap, int leaves_only, DBuf<O>& list, DBuf<O>* pos_out = nullptr) {
        O n = L.n;
        DBuf<O> pos_own;
        DBuf<O>& pos = pos_out ? *pos_out : pos_own;
        pos.alloc(n > 0 ? n : 1, s);
        O* total = dslot<O>(25);
        exclusive_scan<O, GetUnmatched<O, E>>(GetUnmatched<O, E>{vcmap, L.row, leaves_only}, n, pos.p, total, scan, s);
        JET_CUDA(cudaMemcpyAsync(hscal, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        sync();
        O cnt = *(O*)hscal;
        list.alloc(cnt > 0 ? cnt : 1, s);
        k_scatter_unmatched<O, E><<<grid_persistent(n, 16), BLOCK, 0, s>>>(n, vcmap, L.row, leaves_only, pos.p, list.p); count_launch();
        JET_LAUNCH_CHECK();
        return cnt;
    }

    // matchHash in list order (see k_pair_groups).  The null digest sorts as
    // `null_as` (a value no other digest takes); keys use `bits` bits.
    template <class H>
    void match_hash(const O* list, const H* hashes, O mappable, H nullkey, H null_as, int bits, O* vcmap) {
        if (mappable <= 0) return;
        DBuf<H> k0(mappable, s), k1(mappable, s);
        DBuf<O> v0(mappable, s), v1(mappable, s), ex(mappable, s), start(mappable, s);
        int which = radix_sort_pairs<H, O>(GetDigestKey<O, H>{hashes, nullkey, null_as}, GetIndex<O>{}, (int64_t)mappable, bits,
                                           k0.p, v0.p, k1.p, v1.p, rsort, scan, s);
        const H* sk = which == 0 ? k0.p : k1.p;
        const O* sx = which == 0 ? v0.p : v1.p;
        exclusive_scan<O, GetGroupHead<H, O>>(GetGroupHead<H, O>{sk}, (int64_t)mappable, ex.p, nullptr, scan, s);
        k_group_starts<H, O><<<grid_persistent(mappable, 16), BLOCK, 0, s>>>(sk, (int64_t)mappable, ex.p, start.p); count_launch();
        k_pair_groups<H, O><<<grid_persistent(mappable, 16), BLOCK, 0, s>>>(sk, sx, list, (int64_t)mappable, ex.p, start.p, vcmap); count_launch();
        JET_LAUNCH_CHECK();
    }

    void two_hop_passes(Level<O, E, W>& L, O* vcmap) {
        struct Report {
            clk::time_point t;
            ~Report() { if (debug_timing()) fprintf(stderr, "jet:   two-hop %.3f ms\n", since(t) * 1e3); }
        } rep{clk::now()};
        auto g = L.view();
        O n = L.n;
        const O MAXV = ord_max<O>();
        O unmapped = count_unmatched(n, vcmap);
        if ((double)unmapped / (double)n > 0.25) {  // leaves, src/heuristics.hpp:539-560
            DBuf<O> list;
            O cnt = unmatched_list(L, vcmap, 1, list);
            if (cnt > 0) {
                DBuf<O> hs(cnt, s);
                k_leaf_hash<O, E, W><<<grid_persistent(cnt, 16), BLOCK, 0, s>>>(g, list.p, cnt, hs.p); count_launch();
                JET_LAUNCH_CHECK();
                match_hash<O>(list.p, hs.p, cnt, MAXV, n, bits_for((uint64_t)n), vcmap);
            }
        }
        unmapped = count_unmatched(n, vcmap);
        if ((double)unmapped / (double)n > 0.25) {  // twins, src/heuristics.hpp:565-598
            DBuf<O> list;
            DBuf<O> pos;
            O cnt = unmatched_list(L, vcmap, 0, list, &pos);
            if (cnt > 0) {
                DBuf<uint64_t> hs(cnt, s);
                k_twin_hash<O, E, W><<<grid_persistent((int64_t)cnt * 32, 16), BLOCK, 0, s>>>(g, list.p, cnt, hs.p); count_launch();
                JET_LAUNCH_CHECK();
                if (L.n_hub > 0) {
                    k_twin_hash_hub<O, E, W><<<grid_for(L.n_hub, 1) < 4096 ? grid_for(L.n_hub, 1) : 4096, 1024, 0, s>>>(
                        g, L.hub_list.p, L.n_hub, vcmap, pos.p, hs.p); count_launch();
                    JET_LAUNCH_CHECK();
                }
                match_hash<uint64_t>(list.p, hs.p, cnt, (uint64_t)0, (uint64_t)0, 64, vcmap);
            }
        }
        unmapped = count_unmatched(n, vcmap);
        if ((double)unmapped / (double)n > 0.25) {  // relatives, src/heuristics.hpp:603-640
            DBuf<O> list;
            O cnt = unmatched_list(L, vcmap, 0, list);
            if (cnt > 0) {
                DBuf<O> hs(cnt, s);
                k_relative_hash<O, E, W><<<grid_persistent(cnt, 16), BLOCK, 0, s>>>(g, list.p, cnt, hs.p); count_launch();
                JET_LAUNCH_CHECK();
                match_hash<O>(list.p, hs.p, cnt, MAXV, n, bits_for((uint64_t)n), vcmap);
            }
        }
    }

    // generate_coarse_mapping, src/contract.hpp:448-492.
    O coarsen_map(Level<O, E, W>& L, int alg, uint64_t seed, int level, O* vcmap, O* hn_out, double* meas) {
        if (alg == 1) return hec_map(L, seed, level, vcmap, hn_out, meas ? &meas[M_HEAVY] : nullptr, meas ? &meas[M_MAPCONSTRUCT] : nullptr);
        return match_map(L, alg == 0, seed, level, vcmap, hn_out);
    }

    // Hub rows of a level with many coarse ids (see k_hub_keys): keys, one
    // radix sort, reduce-by-key into the rows' scratch regions.
    void contract_hubs_sorted(GView<O, E, W> g, const O* map, const O* lh, const O* nh, const O* moff, const O* members,
                              const E* hrow, O nc, O* skey, W* sval, O* ucnt) {
        JET_CUDA(cudaMemcpyAsync(&hscal[6], nh, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        sync();
        int64_t nhub = (int64_t)*(O*)&hscal[6];
        if (nhub <= 0) return;
        DBuf<E> hoff(nhub + 1, s);
        E* tot = dslot<E>(46);
        exclusive_scan<E, GetHubDu<O, E>>(GetHubDu<O, E>{lh, hrow}, nhub, hoff.p, tot, scan, s);
        JET_CUDA(cudaMemcpyAsync(&hscal[7], tot, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        sync();
        int64_t total = (int64_t)*(E*)&hscal[7];
        if (total <= 0) return;
        const int nb = bits_for((uint64_t)nc);
        const uint64_t sentinel = (uint64_t)nhub << nb;
        const int bits = bits_for(sentinel);
        if (bits > 64) throw JetError{JET_ERR_INVALID, "hub row sort key exceeds 64 bits"};
        DBuf<uint64_t> kin(total, s), k0(total, s), k1(total, s);
        DBuf<W> vin(total, s), v0(total, s), v1(total, s);
        k_hub_keys<O, E, W><<<device_info().sms * 2, 1024, 0, s>>>(g, map, lh, nh, moff, members, hoff.p, nb, sentinel, kin.p,
                                                                   vin.p); count_launch();
        JET_LAUNCH_CHECK();
        int which = radix_sort_pairs<uint64_t, W>(GetArray<uint64_t>{kin.p}, GetArray<W>{vin.p}, total, bits, k0.p, v0.p, k1.p,
                                                  v1.p, rsort, scan, s);
        const uint64_t* sk = which == 0 ? k0.p : k1.p;
        const W* sv = which == 0 ? v0.p : v1.p;
        DBuf<int64_t> seg(total, s), row_first(nhub, s);
        exclusive_scan<int64_t, GetKeyHead<uint64_t, int64_t>>(GetKeyHead<uint64_t, int64_t>{sk, sentinel}, total, seg.p, nullptr,
                                                               scan, s);
        unsigned grid = grid_persistent(total, 16);
        k_hub_row_first<<<grid, BLOCK, 0, s>>>(sk, total, nb, sentinel, seg.p, row_first.p); count_launch();
        k_hub_reduce<O, E, W><<<grid, BLOCK, 0, s>>>(sk, sv, total, nb, sentinel, seg.p, row_first.p, lh, hrow, skey, sval, ucnt); count_launch();
        JET_LAUNCH_CHECK();
    }

    // ------------------------------------------------------------ contraction
    static constexpr int DENSE_PASSES = 8;
    // 1: the graph being coarsened has total edge weight below 2^31, so every
    // coarse row sum fits in 32 bits (acc_add); -1: not known yet (set from the
    // first level contracted, which for a partition is the finest)
    int narrow_w = -1;
    int weight_fits_32(const Level<O, E, W>& L) {
        if (sizeof(W) < 8) return 0;
        W* sum = dslot<W>(55);
        JET_CUDA(cudaMemsetAsync(sum, 0, sizeof(int64_t), s));
        if (L.m > 0) { k_sum<W><<<grid_persistent((int64_t)L.m, 8), BLOCK, 0, s>>>(L.val, (int64_t)L.m, sum); count_launch(); }
        JET_LAUNCH_CHECK();
        JET_CUDA(cudaMemcpyAsync(hscal, sum, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        sync();
        return (int64_t)*(W*)hscal < ((int64_t)1 << 31) ? 1 : 0;
    }
    // build_coarse_graph, src/contract.hpp:347-446.
    static constexpr int64_t CONTRACT_FORK_M = (int64_t)1 << 22;
    void contract(const Level<O, E, W>& L, const O* map, O nc, Level<O, E, W>& C, DBuf<O>* skey_buf, DBuf<W>* sval_buf) {
        if (narrow_w < 0) narrow_w = weight_fits_32(L);
        auto g = L.view();
        O n = L.n;
        DBuf<O> cnt(nc + 1, s), moff(nc + 1, s), members(n > 0 ? n : 1, s), ucnt(nc + 1, s);
        DBuf<E> du(nc + 1, s), hrow(nc + 1, s);
        C.own_vw.alloc(nc, s);
        cnt.zero(); du.zero(); C.own_vw.zero(); ucnt.zero();
        k_contract_count<O, E, W><<<grid_persistent(n, 16), BLOCK, 0, s>>>(g, map, cnt.p, du.p, C.own_vw.p); count_launch();
        JET_LAUNCH_CHECK();
        exclusive_scan_array<O>(cnt.p, nc + 1, moff.p, nullptr, scan, s);
        exclusive_scan_array<E>(du.p, nc + 1, hrow.p, nullptr, scan, s);
        k_contract_members<O><<<grid_persistent(n, 16), BLOCK, 0, s>>>(n, map, moff.p, cnt.p, members.p); count_launch();
        JET_LAUNCH_CHECK();
        // scratch for unique entries, sized by the fine nnz (the bound on sum du)
        DBuf<O> skey_own;
        DBuf<W> sval_own;
        O* skey;
        W* sval;
        if (skey_buf && skey_buf->n >= (int64_t)L.m) { skey = skey_buf->p; sval = sval_buf->p; }
        else { skey_own.alloc(L.m > 0 ? L.m : 1, s); sval_own.alloc(L.m > 0 ? L.m : 1, s); skey = skey_own.p; sval = sval_own.p; }
        DBuf<O> l1(nc, s), l2a(nc, s), l2b(nc, s), l2(nc, s), lh(nc, s);
        O* n1 = dslot<O>(40);
        O* n2 = dslot<O>(41);
        O* nh = dslot<O>(42);
        int* err = dslot<int>(43);
        O* n2a = dslot<O>(45);
        O* n2b = dslot<O>(47);
        // hub rows: a dense shared-memory accumulator when the coarse id range
        // takes at most DENSE_PASSES chunks, else (row, neighbour) keys + radix sort
        int dense_chunk = (max_dynamic_smem((const void*)k_contract_dense<O, E, W>) - 1024) / (int)sizeof(W);
        dense_chunk &= ~1023;
        const bool dense = dense_chunk > 0 && (int64_t)nc <= (int64_t)DENSE_PASSES * dense_chunk;
        if (dense)
            JET_CUDA(cudaFuncSetAttribute(k_contract_dense<O, E, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          max_dynamic_smem((const void*)k_contract_dense<O, E, W>)));
        JET_CUDA(cudaMemsetAsync(n1, 0, 8 * sizeof(int64_t), s));  // slots 40-47 (44 and 46 are scan totals, set later)
        k_contract_bin<O, E><<<grid_persistent(nc, 8), BLOCK, 0, s>>>(nc, hrow.p, l1.p, n1, l2a.p, n2a, l2b.p, n2b, l2.p, n2, lh.p, nh);
        count_launch();
        JET_LAUNCH_CHECK();
        // The bins write disjoint rows: on a large level they run side by side
        // (the warp bin and the hub rows on this stream, the shared-memory
        // bins on three side streams), so that one bin's tail overlaps the
        // others' work.  Batch workers keep one stream each.
        const bool fork = (int64_t)L.m >= CONTRACT_FORK_M && !batch_thread() && !capturing() && side_streams();
        cudaStream_t sa = s, sb = s, sc = s;
        // joins the side streams back into s on every way out of this
        // function (an exception included) before the bins' buffers are freed
        struct Join {
            Engine* e;
            bool on;
            ~Join() {
                if (!on) return;
                for (int i = 0; i < 3; i++) {
                    cudaEventRecord(e->ev_join[i], e->side[i]);
                    cudaStreamWaitEvent(e->s, e->ev_join[i], 0);
                }
            }
        } join{this, false};
        if (fork) {
            JET_CUDA(cudaEventRecord(ev_fork, s));
            for (int i = 0; i < 3; i++) JET_CUDA(cudaStreamWaitEvent(side[i], ev_fork, 0));
            join.on = true;
            sa = side[0];
            sb = side[1];
            sc = side[2];
        }
        k_contract_warp<O, E, W><<<grid_persistent((int64_t)nc * 32, 16), BLOCK, 0, s>>>(g, map, nc, moff.p, members.p, hrow.p, skey, sval, ucnt.p); count_launch();
        JET_LAUNCH_CHECK();
        {
            size_t sm1 = contract_smem_bytes<O, W>(CT_S1_SLOTS), sm2a = contract_smem_bytes<O, W>(CT_S2A_SLOTS),
                   sm2b = contract_smem_bytes<O, W>(CT_S2B_SLOTS), sm2 = contract_smem_bytes<O, W>(CT_S2_SLOTS);
            JET_CUDA(cudaFuncSetAttribute(k_contract_smem<CT_S2B_THREADS, CT_S2B_SLOTS, O, E, W>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2b));
            JET_CUDA(cudaFuncSetAttribute(k_contract_smem<CT_S2_THREADS, CT_S2_SLOTS, O, E, W>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
            JET_CUDA(cudaFuncSetAttribute(k_contract_smem<CT_S2A_THREADS, CT_S2A_SLOTS, O, E, W>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2a));
            int per_sm = 0;
            JET_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contract_smem<CT_S1_THREADS, CT_S1_SLOTS, O, E, W>,
                                                                   CT_S1_THREADS, sm1));
            k_contract_smem<CT_S1_THREADS, CT_S1_SLOTS, O, E, W><<<device_info().sms * (per_sm > 0 ? per_sm : 1), CT_S1_THREADS, sm1, sa>>>(
                g, map, l1.p, n1, moff.p, members.p, hrow.p, skey, sval, ucnt.p, nc, narrow_w); count_launch();
            JET_LAUNCH_CHECK();
            JET_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contract_smem<CT_S2A_THREADS, CT_S2A_SLOTS, O, E, W>,
                                                                   CT_S2A_THREADS, sm2a));
            k_contract_smem<CT_S2A_THREADS, CT_S2A_SLOTS, O, E, W><<<device_info().sms * (per_sm > 0 ? per_sm : 1), CT_S2A_THREADS, sm2a, sb>>>(
                g, map, l2a.p, n2a, moff.p, members.p, hrow.p, skey, sval, ucnt.p, nc, narrow_w); count_launch();
            JET_LAUNCH_CHECK();
            JET_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_contract_smem<CT_S2B_THREADS, CT_S2B_SLOTS, O, E, W>,
                                                                   CT_S2B_THREADS, sm2b));
            k_contract_smem<CT_S2B_THREADS, CT_S2B_SLOTS, O, E, W><<<device_info().sms * (per_sm > 0 ? per_sm : 1), CT_S2B_THREADS, sm2b, sc>>>(
                g, map, l2b.p, n2b, moff.p, members.p, hrow.p, skey, sval, ucnt.p, nc, narrow_w); count_launch();
            JET_LAUNCH_CHECK();
            k_contract_smem<CT_S2_THREADS, CT_S2_SLOTS, O, E, W><<<device_info().sms * 2, CT_S2_THREADS, sm2, sb>>>(
                g, map, l2.p, n2, moff.p, members.p, hrow.p, skey, sval, ucnt.p, nc, narrow_w); count_launch();
            JET_LAUNCH_CHECK();
            if (dense) {
                k_contract_dense<O, E, W><<<device_info().sms, 1024, (size_t)dense_chunk * sizeof(W), s>>>(
                    g, map, lh.p, nh, moff.p, members.p, hrow.p, nc, dense_chunk, skey, sval, ucnt.p, narrow_w); count_launch();
                JET_LAUNCH_CHECK();
            } else {
                contract_hubs_sorted(g, map, lh.p, nh, moff.p, members.p, hrow.p, nc, skey, sval, ucnt.p);
            }
        }
        if (fork) {
            join.on = false;
            for (int i = 0; i < 3; i++) {
                JET_CUDA(cudaEventRecord(ev_join[i], side[i]));
                JET_CUDA(cudaStreamWaitEvent(s, ev_join[i], 0));
            }
        }
        // coarse row offsets and nnz
        C.own_row.alloc(nc + 1, s);
        E* tot = dslot<E>(44);
        exclusive_scan<E, GetCast<O, E>>(GetCast<O, E>{ucnt.p}, nc + 1, C.own_row.p, tot, scan, s);
        JET_CUDA(cudaMemcpyAsync(hscal, dscal.p + 40, sizeof(int64_t) * 5, cudaMemcpyDeviceToHost, s));
        sync();
        if (*(int*)&hscal[3]) throw JetError{JET_ERR_OVERFLOW, "contraction hash table overflow"};
        E mc = *(E*)&hscal[4];
        C.n = nc;
        C.m = mc;
        C.own_adj.alloc(mc > 0 ? mc : 1, s);
        C.own_val.alloc(mc > 0 ? mc : 1, s);
        // every row's unique entries are packed at its scratch offset, in
        // neighbour order; rows of at most 2048 member edges only (the
        // counts of the two largest bins are zero): one warp per row
        const bool short_rows = *(O*)&hscal[1] == 0 && *(O*)&hscal[2] == 0;
        if (mc > 0 && short_rows) {
            k_contract_copy_rows<O, E, W><<<grid_persistent((int64_t)nc * 32, 16), BLOCK, 0, s>>>(nc, hrow.p, skey, sval, C.own_row.p,
                                                                                              C.own_adj.p, C.own_val.p);
            count_launch();
            JET_LAUNCH_CHECK();
        } else if (mc > 0) {
            const int64_t chunks = ((int64_t)mc + CT_COPY_CHUNK - 1) / CT_COPY_CHUNK;
            DBuf<O> chunk_row(chunks, s);
            k_copy_chunk_rows<O, E><<<grid_persistent(nc, 8), BLOCK, 0, s>>>(nc, C.own_row.p, chunk_row.p); count_launch();
            k_contract_copy<O, E, W><<<grid_persistent(chunks * 32, 16), BLOCK, 0, s>>>(nc, mc, chunk_row.p, hrow.p, skey, sval,
                                                                                      C.own_row.p, C.own_adj.p, C.own_val.p);
            count_launch();
            JET_LAUNCH_CHECK();
        }
        C.row = C.own_row.p;
        C.adj = C.own_adj.p;
        C.val = C.own_val.p;
        C.vw = C.own_vw.p;
        C.uniform = false;
    }
};

}  // namespace jetb
