// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points over the Jet reference's OWN code: the unmodified reference
// headers (src/*.hpp) and entry translation unit (src/jet.cpp, compiled beside
// this file) built with g++ against the host-only Kokkos stand-in in
// oracle/kokkos_shim/.  oracle/ref.mk builds two copies into oracle/_ref/:
//   libjet_ref_serial.so  -- Kokkos::Serial: every loop in index order; the
//                            reference's single-thread semantics (jet_serial)
//   libjet_ref_host.so    -- OpenMP on every host core (jet_host), used as the
//                            timed CPU baseline.
// Tests use these to pin the CPU oracle (oracle/jet_oracle.cpp) and the GPU
// path to the reference's own results.  Nothing in the product loads them.
//
// Each function mirrors an orc_* function of the oracle with the same
// arguments; tiers are 0 (int32 everywhere), 1 (int64 offsets and weights),
// 2 (also int64 ordinals).  The reference prints progress to stdout inside
// jet_refine (src/jet_refiner.hpp:1075-1076); `quiet` calls send that to
// /dev/null.
#include <fcntl.h>
#include <unistd.h>

#include <csetjmp>
#include <csignal>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <list>
#include <string>
#include <vector>

#include "jet_defs.h"
#include "jet.h"
#include "partitioner.hpp"
#include "io.hpp"

using namespace jet_partitioner;

#if defined(SERIAL)
using RefSpace = Kokkos::Serial;
#else
using RefSpace = Kokkos::DefaultHostExecutionSpace;
#endif

namespace {

template <class O, class E, class W>
using Mat = KokkosSparse::CrsMatrix<W, O, RefSpace, void, E>;

// Redirects stdout to /dev/null for its lifetime.
struct Quiet {
    int saved = -1;
    explicit Quiet(bool on) {
        if (!on) return;
        fflush(stdout);
        saved = dup(1);
        int nul = open("/dev/null", O_WRONLY);
        dup2(nul, 1);
        close(nul);
    }
    ~Quiet() {
        if (saved < 0) return;
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

// The reference divides by zero in rebalance_weak when no part is undersized
// (src/jet_refiner.hpp:618), which raises SIGFPE.  A call made under
// FPE_GUARD turns that into status REF_SIGFPE when the fault is on the
// calling thread (always so for the Serial build); the reference's
// allocations of the abandoned call are leaked.
static constexpr int REF_SIGFPE = 8;
thread_local sigjmp_buf* t_fpe_jmp = nullptr;
void on_fpe(int sig) {
    if (t_fpe_jmp) siglongjmp(*t_fpe_jmp, sig);
    std::signal(sig, SIG_DFL);
    std::raise(sig);
}
struct FpeHandler {
    struct sigaction old {};
    FpeHandler() {
        struct sigaction sa {};
        sa.sa_handler = on_fpe;
        sigemptyset(&sa.sa_mask);
        sa.sa_flags = SA_NODEFER;
        sigaction(SIGFPE, &sa, &old);
    }
    ~FpeHandler() { sigaction(SIGFPE, &old, nullptr); }
};
#define FPE_GUARD(...)                                 \
    {                                                  \
        FpeHandler fpe_handler_;                       \
        sigjmp_buf fpe_jb_;                            \
        if (sigsetjmp(fpe_jb_, 1)) {                   \
            t_fpe_jmp = nullptr;                       \
            return REF_SIGFPE;                         \
        }                                              \
        t_fpe_jmp = &fpe_jb_;                          \
        __VA_ARGS__;                                   \
        t_fpe_jmp = nullptr;                           \
    }

template <class T, class V>
V to_view(const void* src, int64_t n, const char* label) {
    V v(Kokkos::ViewAllocateWithoutInitializing(label), (size_t)n);
    if (n > 0) std::memcpy(v.data(), src, (size_t)n * sizeof(T));
    return v;
}

template <class O, class E, class W>
Mat<O, E, W> make_mat(int64_t n, const void* row, const void* adj, const void* val) {
    using M = Mat<O, E, W>;
    using dev = typename M::device_type;
    int64_t m = ((const E*)row)[n];
    auto r = to_view<E, Kokkos::View<E*, dev>>(row, n + 1, "row map");
    auto a = to_view<O, Kokkos::View<O*, dev>>(adj, m, "entries");
    auto v = to_view<W, Kokkos::View<W*, dev>>(val, m, "values");
    typename M::staticcrsgraph_type gr(a, r);
    return M("g", (O)n, v, gr);
}

template <class O, class E, class W>
Kokkos::View<W*, typename Mat<O, E, W>::device_type> make_w(const void* vw, int64_t n) {
    return to_view<W, Kokkos::View<W*, typename Mat<O, E, W>::device_type>>(vw, n, "vertex weights");
}

config_t make_cfg(int alg, int k, double imb, double tol, int ultra) {
    config_t c;
    c.coarsening_alg = alg;
    c.num_parts = k;
    c.max_imb_ratio = imb;
    c.refine_tolerance = tol;
    c.ultra_settings = ultra != 0;
    c.verbose = false;
    c.dump_coarse = false;
    c.num_iter = 1;
    return c;
}

void set_seed(uint64_t seed) {
    std::string s = std::to_string((unsigned long long)seed);
    setenv("JET_SEED", s.c_str(), 1);
}

}  // namespace

#define REF_TIER_DISPATCH(tier, ...)                                                       \
    switch (tier) {                                                                        \
        case 0: { typedef int32_t O; typedef int32_t E; typedef int32_t W; __VA_ARGS__; } \
        case 1: { typedef int32_t O; typedef int64_t E; typedef int64_t W; __VA_ARGS__; } \
        case 2: { typedef int64_t O; typedef int64_t E; typedef int64_t W; __VA_ARGS__; } \
        default: return 1;                                                                 \
    }

extern "C" {

// Number of threads the reference's execution space runs on.
int ref_concurrency() { return RefSpace().concurrency(); }

// partitioner::partition (src/partitioner.hpp:61-125) through the reference's
// own entry instantiation.  The coarsening RNG pool is seeded with `seed`
// (the reference seeds it from the clock, src/contract.hpp:503).
// Returns 0, or 8 when the reference raised SIGFPE (its division by zero in
// rebalance_weak, src/jet_refiner.hpp:618); *seconds_out is the wall time of
// the partition call alone.
int ref_partition(int tier, int alg, int k, double imb, double tol, int ultra, int64_t n, const void* row,
                  const void* adj, const void* val, const void* vw, int uniform_ew, uint64_t seed, int32_t* part_out,
                  int64_t* cut_out, double* imb_out, double* seconds_out, int quiet) {
    config_t cfg = make_cfg(alg, k, imb, tol, ultra);
    set_seed(seed);
    REF_TIER_DISPATCH(tier, {
        auto g = make_mat<O, E, W>(n, row, adj, val);
        auto w = make_w<O, E, W>(vw, n);
        experiment_data<W> exp;
        W cut = 0;
        Quiet q(quiet != 0);
        typename partitioner<Mat<O, E, W>, part_t>::part_vt part;
        auto t0 = std::chrono::steady_clock::now();
        FPE_GUARD(part = partitioner<Mat<O, E, W>, part_t>::partition(cut, cfg, g, w, uniform_ew != 0, exp));
        auto t1 = std::chrono::steady_clock::now();
        std::memcpy(part_out, part.data(), (size_t)n * sizeof(int32_t));
        *cut_out = (int64_t)cut;
        if (imb_out) {
            using stat = part_stat<Mat<O, E, W>, part_t>;
            auto sizes = stat::get_part_sizes(g, w, part, k);
            double opt = (double)stat::optimal_size(stat::get_total_size(g, w), k);
            *imb_out = (double)stat::largest_part_size(sizes) / opt;
        }
        if (seconds_out) *seconds_out = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    });
}

// One coarsening map (generate_coarse_mapping, src/contract.hpp:448-492):
// alg 0 = 2-hop matching (MtMetis), 1 = HEC, 2 = plain matching.
int ref_coarsen(int tier, int alg, uint64_t seed, int64_t n, const void* row, const void* adj, const void* val,
                const void* vw, int uniform, void* map_out, int64_t* nc_out) {
    set_seed(seed);
    REF_TIER_DISPATCH(tier, {
        using C = contracter<Mat<O, E, W>>;
        auto g = make_mat<O, E, W>(n, row, adj, val);
        auto w = make_w<O, E, W>(vw, n);
        C c;
        c.set_heuristic(alg == 1 ? C::HECv1 : (alg == 2 ? C::Match : C::MtMetis));
        experiment_data<W> exp;
        typename C::pool_t pool(seed);
        auto cm = c.generate_coarse_mapping(g, w, uniform != 0, pool, exp);
        std::memcpy(map_out, cm.map.data(), (size_t)n * sizeof(O));
        *nc_out = (int64_t)cm.coarse_vtx;
        return 0;
    });
}

// build_coarse_graph (src/contract.hpp:347-446) for a given map.  Output
// arrays as orc_contract; rows come out in the reference's hash-slot order.
int ref_contract(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
                 const void* map, int64_t nc, void* crow, void* cadj, void* cval, void* cvw, int64_t* cnnz) {
    REF_TIER_DISPATCH(tier, {
        using C = contracter<Mat<O, E, W>>;
        using dev = typename Mat<O, E, W>::device_type;
        auto g = make_mat<O, E, W>(n, row, adj, val);
        typename C::coarse_level_triple lvl;
        lvl.mtx = g;
        lvl.vtx_w = make_w<O, E, W>(vw, n);
        lvl.level = 1;
        typename C::coarse_map cm;
        cm.coarse_vtx = (O)nc;
        cm.map = to_view<O, Kokkos::View<O*, dev>>(map, n, "map");
        typename C::scratch_mem scratch;
        scratch.htable = Kokkos::View<O*, dev>("htable scratch", (size_t)g.nnz());
        scratch.hvals = Kokkos::View<W*, dev>("hvals scratch", (size_t)g.nnz());
        scratch.hrow_map = Kokkos::View<E*, dev>("hrow_map scratch", (size_t)n + 1);
        experiment_data<W> exp;
        C c;
        auto next = c.build_coarse_graph(lvl, cm, scratch, exp);
        int64_t m = (int64_t)next.mtx.nnz();
        std::memcpy(crow, next.mtx.graph.row_map.data(), (size_t)(nc + 1) * sizeof(E));
        if (m) std::memcpy(cadj, next.mtx.graph.entries.data(), (size_t)m * sizeof(O));
        if (m) std::memcpy(cval, next.mtx.values.data(), (size_t)m * sizeof(W));
        std::memcpy(cvw, next.vtx_w.data(), (size_t)nc * sizeof(W));
        *cnnz = m;
        return 0;
    });
}

// init_conn_data (src/jet_refiner.hpp:958-1048) for a partition.  Output as
// orc_conn_build: off n+1, ent/val C = off[n], size n.
int ref_conn_build(int tier, int64_t n, const void* row, const void* adj, const void* val, const int32_t* part, int k,
                   void* off_out, int32_t* ent_out, void* val_out, int32_t* size_out) {
    REF_TIER_DISPATCH(tier, {
        using R = jet_refiner<Mat<O, E, W>, part_t>;
        using dev = typename Mat<O, E, W>::device_type;
        auto g = make_mat<O, E, W>(n, row, adj, val);
        auto p = to_view<int32_t, Kokkos::View<int32_t*, dev>>(part, n, "part");
        R r(g, k);
        auto cd = r.init_conn_data(r.perm_cdata, g, p, k);
        int64_t c = (int64_t)cd.conn_offsets((size_t)n);
        std::memcpy(off_out, cd.conn_offsets.data(), (size_t)(n + 1) * sizeof(E));
        if (c) std::memcpy(ent_out, cd.conn_entries.data(), (size_t)c * sizeof(int32_t));
        if (c) std::memcpy(val_out, cd.conn_vals.data(), (size_t)c * sizeof(W));
        std::memcpy(size_out, cd.conn_table_sizes.data(), (size_t)n * sizeof(int32_t));
        return 0;
    });
}

// `iters` iterations of jet_refine's body (src/jet_refiner.hpp:1106-1119)
// from `part` (in/out), without the best-state bookkeeping: LP while the
// imbalance is within bounds, else weak rebalancing twice, then strong; then
// perform_moves.  Outputs as orc_refine_iters.
int ref_refine_iters(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
                     int32_t* part, int k, double imb, double filter_ratio, int iters, void* sizes_out,
                     int64_t* cut_out, void* off_out, int32_t* ent_out, void* cval_out, int32_t* size_out,
                     int32_t* dest_cache_out, int64_t* moves_out, int32_t* kind_out) {
    REF_TIER_DISPATCH(tier, {
        using M = Mat<O, E, W>;
        using R = jet_refiner<M, part_t>;
        using stat = part_stat<M, part_t>;
        using dev = typename M::device_type;
        using gain_t = typename R::gain_t;
        auto g = make_mat<O, E, W>(n, row, adj, val);
        auto w = make_w<O, E, W>(vw, n);
        auto p = to_view<int32_t, Kokkos::View<int32_t*, dev>>(part, n, "part");
        R r(g, k);
        typename R::refine_data st;
        st.cut = stat::get_total_cut(g, p);
        st.part_sizes = stat::get_part_sizes(g, w, p, k);
        st.total_size = stat::get_total_size(g, w);
        typename R::problem prob;
        prob.g = g;
        prob.k = k;
        prob.imb = imb;
        prob.vtx_w = w;
        prob.opt = stat::optimal_size(st.total_size, k);
        prob.size_max = prob.opt * imb;
        gain_t mx = stat::largest_part_size(st.part_sizes);
        st.total_imb = mx > prob.opt ? mx - prob.opt : 0;
        st.init = true;
        gain_t imb_max = prob.size_max - prob.opt;
        auto cd = r.init_conn_data(r.perm_cdata, g, p, k);
        int bal = 0;
        for (int it = 0; it < iters; it++) {
            typename R::vtx_vt moves;
            int kind;
            if (st.total_imb <= imb_max) {
                moves = r.jet_lp(prob, p, cd, r.perm_scratch, filter_ratio);
                bal = 0;
                kind = 0;
            } else if (bal < 2) {
                FPE_GUARD(moves = r.rebalance_weak(prob, p, cd, r.perm_scratch, st.part_sizes));
                bal++;
                kind = 1;
            } else {
                moves = r.rebalance_strong(prob, p, cd, r.perm_scratch, st.part_sizes);
                bal++;
                kind = 2;
            }
            r.perform_moves(prob, p, moves, r.perm_scratch.dest_part, r.perm_scratch, cd, st);
            if (moves_out) moves_out[it] = (int64_t)moves.extent(0);
            if (kind_out) kind_out[it] = kind;
        }
        std::memcpy(part, p.data(), (size_t)n * sizeof(int32_t));
        for (int q = 0; q < k; q++) ((W*)sizes_out)[q] = (W)st.part_sizes(q);
        *cut_out = (int64_t)st.cut;
        int64_t c = (int64_t)cd.conn_offsets((size_t)n);
        if (off_out) std::memcpy(off_out, cd.conn_offsets.data(), (size_t)(n + 1) * sizeof(E));
        if (ent_out && c) std::memcpy(ent_out, cd.conn_entries.data(), (size_t)c * sizeof(int32_t));
        if (cval_out && c) std::memcpy(cval_out, cd.conn_vals.data(), (size_t)c * sizeof(W));
        if (size_out) std::memcpy(size_out, cd.conn_table_sizes.data(), (size_t)n * sizeof(int32_t));
        if (dest_cache_out) std::memcpy(dest_cache_out, cd.dest_cache.data(), (size_t)n * sizeof(int32_t));
        return 0;
    });
}

// One full jet_refine (src/jet_refiner.hpp:1050-1142) at a single level from
// `part` (in/out), fresh refine data.  *cut_out counts each cut edge twice.
int ref_refine_level(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
                     int32_t* part, int k, double imb, double tol, int ultra, int uniform_ew, int64_t* cut_out,
                     int32_t* iters_out) {
    config_t cfg = make_cfg(1, k, imb, tol, ultra);
    REF_TIER_DISPATCH(tier, {
        using M = Mat<O, E, W>;
        using R = jet_refiner<M, part_t>;
        using dev = typename M::device_type;
        auto g = make_mat<O, E, W>(n, row, adj, val);
        auto w = make_w<O, E, W>(vw, n);
        auto p = to_view<int32_t, Kokkos::View<int32_t*, dev>>(part, n, "part");
        R r(g, k);
        typename R::refine_data st;
        experiment_data<W> exp;
        {
            Quiet q(true);
            FPE_GUARD(r.jet_refine(g, cfg, w, p, uniform_ew != 0, st, exp));
        }
        std::memcpy(part, p.data(), (size_t)n * sizeof(int32_t));
        *cut_out = (int64_t)st.cut;
        if (iters_out) *iters_out = -1;  // experiment_data keeps its level records private
        return 0;
    });
}

// uncoarsener::uncoarsen (src/uncoarsen.hpp:127-158) over a fixed hierarchy,
// as the reference's jet_import app does (app/import_coarse.cpp:49-132).
// Level 0 is the finest; maps[l] (l >= 1) sends level l-1's vertices to level
// l.  coarsest_part has ns[nlevels-1] entries; part_out receives ns[0].
int ref_uncoarsen(int tier, int nlevels, const int64_t* ns, const void* const* rows, const void* const* adjs,
                  const void* const* vals, const void* const* vws, const void* const* maps,
                  const int32_t* coarsest_part, int k, double imb, double tol, int ultra, int uniform_finest,
                  int32_t* part_out, int64_t* cut_out) {
    config_t cfg = make_cfg(1, k, imb, tol, ultra);
    REF_TIER_DISPATCH(tier, {
        using M = Mat<O, E, W>;
        using C = contracter<M>;
        using U = uncoarsener<M, part_t>;
        using dev = typename M::device_type;
        std::list<typename C::coarse_level_triple> levels;
        for (int l = 0; l < nlevels; l++) {
            typename C::coarse_level_triple lv;
            lv.level = l + 1;
            lv.mtx = make_mat<O, E, W>(ns[l], rows[l], adjs[l], vals[l]);
            lv.vtx_w = make_w<O, E, W>(vws[l], ns[l]);
            lv.uniform_weights = (l == 0) && uniform_finest;
            if (l > 0) {
                lv.interp_mtx.coarse_vtx = (O)ns[l];
                lv.interp_mtx.map = to_view<O, Kokkos::View<O*, dev>>(maps[l], ns[l - 1], "map");
            }
            levels.push_back(lv);
        }
        auto cp = to_view<int32_t, Kokkos::View<int32_t*, dev>>(coarsest_part, ns[nlevels - 1], "coarsest part");
        experiment_data<W> exp;
        W cut = 0;
        Quiet q(true);
        typename U::part_vt part;
        FPE_GUARD(part = U::uncoarsen(levels, cp, cfg, cut, exp));
        std::memcpy(part_out, part.data(), (size_t)ns[0] * sizeof(int32_t));
        *cut_out = (int64_t)cut;
        return 0;
    });
}

// pstat quantities (app/part_eval.cpp:73-110 over src/part_stat.hpp).
// out: [cut (each edge once), max part cut, comm size, largest, smallest, total]
int ref_pstat(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
              const int32_t* part, int k, int64_t* out) {
    REF_TIER_DISPATCH(tier, {
        using M = Mat<O, E, W>;
        using stat = part_stat<M, part_t>;
        using dev = typename M::device_type;
        auto g = make_mat<O, E, W>(n, row, adj, val);
        auto w = make_w<O, E, W>(vw, n);
        auto p = to_view<int32_t, Kokkos::View<int32_t*, dev>>(part, n, "part");
        out[0] = (int64_t)(stat::get_total_cut(g, p) / 2);
        out[1] = (int64_t)stat::max_part_cut(g, p, k);
        out[2] = (int64_t)stat::comm_size(g, p, k);
        auto sizes = stat::get_part_sizes(g, w, p, k);
        int64_t largest = 0, smallest = INT64_MAX, total = 0;
        for (int q = 0; q < k; q++) {
            int64_t s = (int64_t)sizes(q);
            largest = std::max(largest, s);
            smallest = std::min(smallest, s);
            total += s;
        }
        out[3] = largest;
        out[4] = smallest;
        out[5] = total;
        return 0;
    });
}

// jet_refiner::gain_bucket (src/jet_refiner.hpp:326-356).
int ref_gain_bucket32(int32_t gain, int32_t vwgt) {
    return jet_refiner<Mat<int32_t, int32_t, int32_t>, part_t>::gain_bucket(gain, vwgt);
}
int ref_gain_bucket64(int64_t gain, int64_t vwgt) {
    return jet_refiner<Mat<int32_t, int64_t, int64_t>, part_t>::gain_bucket(gain, vwgt);
}

// The reference's own METIS reader (app/io.hpp:99-217), std tier.  Returns
// 0 and fills n, nnz and the arrays (capacity given by the caller: row_cap
// entries of row, nnz_cap of adj and val), or 1 when the reader rejects the
// file, or 2 when the capacity is too small.
int ref_load_metis(const char* path, int64_t* n, int64_t* nnz, int32_t* row, int64_t row_cap, int32_t* adj,
                   int32_t* val, int64_t nnz_cap, int* uniform_ew) {
    matrix_t g;
    bool uni = false;
    bool ok;
    {
        Quiet q(true);
        ok = load_metis_graph(g, uni, path);
    }
    if (!ok) return 1;
    *n = g.numRows();
    *nnz = g.nnz();
    if (*n + 1 > row_cap || *nnz > nnz_cap) return 2;
    std::memcpy(row, g.graph.row_map.data(), (size_t)(*n + 1) * sizeof(int32_t));
    std::memcpy(adj, g.graph.entries.data(), (size_t)*nnz * sizeof(int32_t));
    std::memcpy(val, g.values.data(), (size_t)*nnz * sizeof(int32_t));
    *uniform_ew = uni ? 1 : 0;
    return 0;
}

// Kokkos::pod_hash of an int32 as the stand-in computes it.
uint32_t ref_pod_hash32(int32_t x) { return Kokkos::pod_hash<int32_t>()(x); }

}  // extern "C"
