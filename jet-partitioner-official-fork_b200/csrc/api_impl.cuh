// api_impl.cuh -- templated bodies of the C ABI (include/jet_b200.h).
// Each tier's translation unit instantiates them with its integer types.
#pragma once
#include "uncoarsen.cuh"
#include <string>

namespace jetb {

void set_last_error(const std::string& msg);
cudaStream_t default_stream();

// Maps exceptions to status codes; the message goes to jet_last_error().
template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const JetError& e) {
        set_last_error(e.what);
        return e.code;
    } catch (const CudaError& e) {
        set_last_error(std::string(e.where) + ": " + cudaGetErrorString(e.e));
        if (e.e == cudaErrorMemoryAllocation) { cudaGetLastError(); return JET_ERR_OOM; }
        return JET_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return JET_ERR_OOM;
    }
}

inline cudaStream_t pick_stream(void* s) { return s ? (cudaStream_t)s : default_stream(); }

// ---------------------------------------------------------------- validation
// Rejects graphs the refinement cannot handle: non-monotone offsets, neighbour
// ids out of range, non-positive vertex or edge weights (a zero vertex weight
// would make gain_bucket divide by zero and never terminate).
// Vertices and entries are checked in two flat passes, so hub rows cost no
// more than any other entries.
template <class O, class E, class W>
__global__ void k_validate(O n, E m, const E* row, const O* adj, const W* val, const W* vw, int* err) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        E a = row[i], b = row[i + 1];
        if (b < a || a < 0 || b > m) bad |= 1;
        if (vw[i] <= 0) bad |= 4;
    }
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < (int64_t)m; j += stride) {
        O v = adj[j];
        if (v < 0 || v >= n) bad |= 2;
        if (val[j] <= 0) bad |= 8;
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicOr(err, bad);
    if (blockIdx.x == 0 && threadIdx.x == 0 && (row[0] != 0 || row[n] != m)) atomicOr(err, 1);
}

template <class O, class E, class W>
void validate(Engine<O, E, W>& eng, O n, E m, const E* row, const O* adj, const W* val, const W* vw) {
    int* err = eng.template dslot<int>(60);
    JET_CUDA(cudaMemsetAsync(err, 0, sizeof(int64_t), eng.s));
    k_validate<O, E, W><<<grid_persistent((int64_t)m + n + 1, 8), BLOCK, 0, eng.s>>>(n, m, row, adj, val, vw, err); count_launch();
    JET_LAUNCH_CHECK();
    JET_CUDA(cudaMemcpyAsync(&eng.hscal[0], err, sizeof(int64_t), cudaMemcpyDeviceToHost, eng.s));
    eng.sync();
    int e = *(int*)&eng.hscal[0];
    if (e & 1) throw JetError{JET_ERR_INVALID, "row_map is not a valid CSR offset array"};
    if (e & 2) throw JetError{JET_ERR_INVALID, "neighbour id out of range"};
    if (e & 4) throw JetError{JET_ERR_INVALID, "vertex weights must be positive"};
    if (e & 8) throw JetError{JET_ERR_INVALID, "edge weights must be positive"};
}

// Device copies of host inputs (or borrowed device pointers).
template <class O, class E, class W>
struct Inputs {
    DBuf<E> row;
    DBuf<O> adj;
    DBuf<W> val, vw;
    const E* prow;
    const O* padj;
    const W* pval;
    const W* pvw;
    E m;
    void load(O n, const E* r, const O* a, const W* v, const W* w, int mem, cudaStream_t s) {
        if (mem == JET_MEM_DEVICE) {
            prow = r; padj = a; pval = v; pvw = w;
            JET_CUDA(cudaMemcpyAsync(&m, r + n, sizeof(E), cudaMemcpyDeviceToHost, s));
            stream_wait(s);
            return;
        }
        m = r[n];
        if (m < 0) throw JetError{JET_ERR_INVALID, "negative nnz"};
        row.alloc(n + 1, s); adj.alloc(m > 0 ? m : 1, s); val.alloc(m > 0 ? m : 1, s); vw.alloc(n > 0 ? n : 1, s);
        JET_CUDA(cudaMemcpyAsync(row.p, r, sizeof(E) * (n + 1), cudaMemcpyHostToDevice, s));
        if (m > 0) {
            JET_CUDA(cudaMemcpyAsync(adj.p, a, sizeof(O) * m, cudaMemcpyHostToDevice, s));
            JET_CUDA(cudaMemcpyAsync(val.p, v, sizeof(W) * m, cudaMemcpyHostToDevice, s));
        }
        if (n > 0) JET_CUDA(cudaMemcpyAsync(vw.p, w, sizeof(W) * n, cudaMemcpyHostToDevice, s));
        prow = row.p; padj = adj.p; pval = val.p; pvw = vw.p;
    }
};

// partitioner::partition (src/partitioner.hpp:61-125) behind the C ABI.
template <class O, class E, class W>
int partition_impl(const jet_config_c* cfg, O n, const E* row, const O* adj, const W* val, const W* vw, int uniform_ew,
                   int mem, uint64_t seed, void* stream, part_t* part_out, W* cut_out, jet_stats_c* st) {
    return guarded([&]() -> int {
        if (!cfg || !row || !part_out || !cut_out || n < 0) throw JetError{JET_ERR_INVALID, "null argument"};
        if (cfg->num_parts < 1) throw JetError{JET_ERR_INVALID, "num_parts must be >= 1"};
        if (mem != JET_MEM_HOST && mem != JET_MEM_DEVICE) throw JetError{JET_ERR_INVALID, "mem must be JET_MEM_HOST or JET_MEM_DEVICE"};
        if (st) std::memset(st, 0, sizeof(*st));
        cudaStream_t s = pick_stream(stream);
        Engine<O, E, W> eng(s);
        auto t0 = clk::now();
        Inputs<O, E, W> in;
        in.load(n, row, adj, val, vw, mem, s);
        double t_load = since(t0);
        validate<O, E, W>(eng, n, in.m, in.prow, in.padj, in.pval, in.pvw);
        double t_transfer = since(t0);
        if (debug_timing()) fprintf(stderr, "jet: load %.3f ms validate %.3f ms\n", t_load * 1e3, (t_transfer - t_load) * 1e3);
        if (n == 0) { *cut_out = 0; return JET_OK; }
        DBuf<part_t> part_dev;
        part_t* pout = part_out;
        if (mem == JET_MEM_HOST) { part_dev.alloc(n, s); pout = part_dev.p; }
        Cfg c{cfg->coarsening_alg, cfg->num_parts, cfg->max_imb_ratio, cfg->refine_tolerance, cfg->ultra_settings != 0,
              cfg->verbose != 0, cfg->dump_coarse != 0};
        if (c.k == 1) {
            // a single part: everything in part 0, nothing cut
            JET_CUDA(cudaMemsetAsync(pout, 0, sizeof(part_t) * n, s));
            *cut_out = 0;
        } else {
            GraphIn<O, E, W> gi{n, in.m, in.prow, in.padj, in.pval, in.pvw, uniform_ew != 0};
            *cut_out = run_partition<O, E, W>(eng, c, gi, seed, pout, st);
        }
        if (mem == JET_MEM_HOST) {
            JET_CUDA(cudaMemcpyAsync(part_out, pout, sizeof(part_t) * n, cudaMemcpyDeviceToHost, s));
        }
        eng.sync();
        if (st) {
            st->measurements[M_INITTRANSFER] += t_transfer;
            if (cfg->verbose) {
                int64_t out[6];
                pstat_impl_dev(eng, n, in.m, in.prow, in.padj, in.pval, in.pvw, pout, cfg->num_parts, out);
                st->max_part_cut = out[1];
                st->objective = out[2];
            }
        }
        return JET_OK;
    });
}

// Partition statistics over device arrays (app/part_eval.cpp:73-110,
// src/part_stat.hpp:77-239).
template <class O, class E, class W>
__global__ void k_cut_per_part(GView<O, E, W> g, const part_t* part, W* per) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        part_t pi = part[i];
        W acc = 0;
        for (E j = g.row[i]; j < g.row[i + 1]; j++) if (part[g.adj[j]] != pi) acc += g.val[j];
        if (acc) atomic_add(&per[pi], acc);
    }
}
template <class O, class E, class W>
__global__ void k_comm_count(GView<O, E, W> g, const part_t* part, const E* coff, const Slot<W>* slots, const part_t* csize,
                             long long* out) {
    long long c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        const Slot<W>* b = slots + coff[i];
        part_t pi = part[i];
        for (part_t s = 0; s < csize[i]; s++) if (b[s].p >= 0 && b[s].p != pi) c++;
    }
    c = group_sum<long long>(c, 32);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd((unsigned long long*)out, (unsigned long long)c);
}

template <class O, class E, class W>
void pstat_impl_dev(Engine<O, E, W>& eng, O n, E m, const E* row, const O* adj, const W* val, const W* vw, const part_t* part,
                    part_t k, int64_t* out) {
    cudaStream_t s = eng.s;
    Level<O, E, W> L;
    L.n = n; L.m = m; L.row = row; L.adj = adj; L.val = val; L.vw = vw;
    eng.prepare_level(L);
    Refiner<O, E, W> ref(eng, n, (int64_t)m, k);
    ref.check_parts(L, part);
    W cut = ref.total_cut(L, part);
    DBuf<W> per(k, s);
    per.zero();
    k_cut_per_part<O, E, W><<<grid_persistent(n, 8), BLOCK, 0, s>>>(L.view(), part, per.p); count_launch();
    JET_LAUNCH_CHECK();
    std::vector<W> hper(k), hs(k);
    JET_CUDA(cudaMemcpyAsync(hper.data(), per.p, sizeof(W) * k, cudaMemcpyDeviceToHost, s));
    ref.part_sizes(L, part, ref.sizes_best.p);
    JET_CUDA(cudaMemcpyAsync(hs.data(), ref.sizes_best.p, sizeof(W) * k, cudaMemcpyDeviceToHost, s));
    JET_CUDA(cudaMemcpyAsync(ref.part_work.p, part, sizeof(part_t) * n, cudaMemcpyDeviceToDevice, s));
    ref.init_conn(L);
    long long* cc = eng.template dslot<long long>(61);
    JET_CUDA(cudaMemsetAsync(cc, 0, sizeof(int64_t), s));
    k_comm_count<O, E, W><<<grid_persistent(n, 8), BLOCK, 0, s>>>(L.view(), part, ref.coff.p, ref.slots.p, ref.csize.p, cc); count_launch();
    JET_LAUNCH_CHECK();
    JET_CUDA(cudaMemcpyAsync(&eng.hscal[1], cc, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    eng.sync();
    W mx = 0, largest = 0, smallest = std::numeric_limits<W>::max(), total = 0;
    for (W x : hper) mx = x > mx ? x : mx;
    for (W x : hs) { largest = x > largest ? x : largest; smallest = x < smallest ? x : smallest; total += x; }
    out[0] = (int64_t)(cut / 2); out[1] = (int64_t)mx; out[2] = eng.hscal[1];
    out[3] = (int64_t)largest; out[4] = (int64_t)smallest; out[5] = (int64_t)total;
}

// ---------------------------------------------------------------- components
template <class O, class E, class W>
struct Tier {
    static Level<O, E, W> borrow(int64_t n, int64_t m, const void* row, const void* adj, const void* val, const void* vw, bool uniform) {
        Level<O, E, W> L;
        L.n = (O)n; L.m = (E)m; L.row = (const E*)row; L.adj = (const O*)adj; L.val = (const W*)val; L.vw = (const W*)vw;
        L.uniform = uniform;
        return L;
    }

    static int coarsen_map(int alg, int level, uint64_t seed, int64_t n, int64_t m, const void* row, const void* adj,
                           const void* val, const void* vw, int uniform, void* map_out, void* hn_out, int64_t* nc, void* stream) {
        return guarded([&]() -> int {
            Engine<O, E, W> eng(pick_stream(stream));
            Level<O, E, W> L = borrow(n, m, row, adj, val, vw, uniform != 0);
            eng.prepare_level(L);
            O c = eng.coarsen_map(L, alg, seed, level, (O*)map_out, (O*)hn_out, nullptr);
            *nc = (int64_t)c;
            eng.sync();
            return JET_OK;
        });
    }

    static int contract(int64_t n, int64_t m, const void* row, const void* adj, const void* val, const void* vw, const void* map,
                        int64_t nc, void* crow, void* cadj, void* cval, void* cvw, int64_t* cnnz, void* stream) {
        return guarded([&]() -> int {
            Engine<O, E, W> eng(pick_stream(stream));
            cudaStream_t s = eng.s;
            Level<O, E, W> L = borrow(n, m, row, adj, val, vw, false);
            Level<O, E, W> C;
            eng.contract(L, (const O*)map, (O)nc, C, nullptr, nullptr);
            JET_CUDA(cudaMemcpyAsync(crow, C.row, sizeof(E) * (nc + 1), cudaMemcpyDeviceToDevice, s));
            if (C.m) {
                JET_CUDA(cudaMemcpyAsync(cadj, C.adj, sizeof(O) * C.m, cudaMemcpyDeviceToDevice, s));
                JET_CUDA(cudaMemcpyAsync(cval, C.val, sizeof(W) * C.m, cudaMemcpyDeviceToDevice, s));
            }
            if (nc) JET_CUDA(cudaMemcpyAsync(cvw, C.vw, sizeof(W) * nc, cudaMemcpyDeviceToDevice, s));
            *cnnz = (int64_t)C.m;
            eng.sync();
            return JET_OK;
        });
    }

    // Unpacks {part, weight} slots into separate arrays.
    static void unpack(cudaStream_t s, const Slot<W>* slots, int64_t C, int32_t* ent, W* val) {
        if (C <= 0) return;
        std::vector<Slot<W>> h(C);
        JET_CUDA(cudaMemcpyAsync(h.data(), slots, sizeof(Slot<W>) * C, cudaMemcpyDeviceToHost, s));
        stream_wait(s);
        std::vector<int32_t> he(C);
        std::vector<W> hv(C);
        for (int64_t i = 0; i < C; i++) { he[i] = h[i].p; hv[i] = h[i].v; }
        if (ent) JET_CUDA(cudaMemcpyAsync(ent, he.data(), sizeof(int32_t) * C, cudaMemcpyHostToDevice, s));
        if (val) JET_CUDA(cudaMemcpyAsync(val, hv.data(), sizeof(W) * C, cudaMemcpyHostToDevice, s));
        stream_wait(s);
    }

    static int conn_build(int64_t n, int64_t m, const void* row, const void* adj, const void* val, const int32_t* part, int32_t k,
                          void* off, int32_t* ent, void* cval, int32_t* size, void* stream) {
        return guarded([&]() -> int {
            Engine<O, E, W> eng(pick_stream(stream));
            cudaStream_t s = eng.s;
            Level<O, E, W> L = borrow(n, m, row, adj, val, nullptr, false);
            eng.prepare_level(L);
            Refiner<O, E, W> ref(eng, (O)n, m, k);
            JET_CUDA(cudaMemcpyAsync(ref.part_work.p, part, sizeof(part_t) * n, cudaMemcpyDeviceToDevice, s));
            ref.check_parts(L, ref.part_work.p);
            int64_t C = ref.init_conn(L);
            JET_CUDA(cudaMemcpyAsync(off, ref.coff.p, sizeof(E) * (n + 1), cudaMemcpyDeviceToDevice, s));
            JET_CUDA(cudaMemcpyAsync(size, ref.csize.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
            unpack(s, ref.slots.p, C, ent, (W*)cval);
            eng.sync();
            return JET_OK;
        });
    }

    static int refine_iters(int64_t n, int64_t m, const void* row, const void* adj, const void* val, const void* vw, int32_t* part,
                            int32_t k, double imb, double filter_ratio, int32_t iters, void* sizes, int64_t* cut, void* off,
                            int32_t* ent, void* cval, int32_t* size, int32_t* dest_cache, int64_t* moves, int32_t* kinds,
                            void* stream) {
        return guarded([&]() -> int {
            Engine<O, E, W> eng(pick_stream(stream));
            cudaStream_t s = eng.s;
            Level<O, E, W> L = borrow(n, m, row, adj, val, vw, false);
            eng.prepare_level(L);
            Refiner<O, E, W> ref(eng, (O)n, m, k);
            auto pb = ref.begin_level(L, part, imb);
            int bal = 0, lab = 0;
            std::vector<int64_t> hm(iters > 0 ? iters : 1);
            std::vector<int32_t> hk(iters > 0 ? iters : 1);
            for (int it = 0; it < iters; it++) {
                hk[it] = ref.iterate(L, pb, filter_ratio, bal, lab);
                hm[it] = ref.last_moves;
            }
            JET_CUDA(cudaMemcpyAsync(part, ref.part_work.p, sizeof(part_t) * n, cudaMemcpyDeviceToDevice, s));
            JET_CUDA(cudaMemcpyAsync(sizes, ref.sizes_curr.p, sizeof(W) * k, cudaMemcpyDeviceToDevice, s));
            *cut = (int64_t)ref.curr.cut;
            if (moves && iters > 0) std::memcpy(moves, hm.data(), sizeof(int64_t) * iters);
            if (kinds && iters > 0) std::memcpy(kinds, hk.data(), sizeof(int32_t) * iters);
            if (off) JET_CUDA(cudaMemcpyAsync(off, ref.coff.p, sizeof(E) * (n + 1), cudaMemcpyDeviceToDevice, s));
            if (size) JET_CUDA(cudaMemcpyAsync(size, ref.csize.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
            if (dest_cache) JET_CUDA(cudaMemcpyAsync(dest_cache, ref.dest_cache.p, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
            if (ent || cval) {
                E C = 0;
                JET_CUDA(cudaMemcpyAsync(&C, ref.coff.p + n, sizeof(E), cudaMemcpyDeviceToHost, s));
                stream_wait(s);
                unpack(s, ref.slots.p, (int64_t)C, ent, (W*)cval);
            }
            eng.sync();
            return JET_OK;
        });
    }

    static int refine_level(int64_t n, int64_t m, const void* row, const void* adj, const void* val, const void* vw, int32_t* part,
                            int32_t k, double imb, double tol, int uniform_ew, int64_t* cut, int32_t* iters, void* stream) {
        return guarded([&]() -> int {
            Engine<O, E, W> eng(pick_stream(stream));
            Level<O, E, W> L = borrow(n, m, row, adj, val, vw, uniform_ew != 0);
            eng.prepare_level(L);
            Refiner<O, E, W> ref(eng, (O)n, m, k);
            jet_level_stats_c cl = ref.refine(L, part, imb, tol, false);
            *cut = (int64_t)ref.best.cut;
            if (iters) *iters = cl.total_iterations;
            eng.sync();
            return JET_OK;
        });
    }

    static int pstat(int64_t n, int64_t m, const void* row, const void* adj, const void* val, const void* vw, const int32_t* part,
                     int32_t k, int64_t* out, void* stream) {
        return guarded([&]() -> int {
            Engine<O, E, W> eng(pick_stream(stream));
            pstat_impl_dev<O, E, W>(eng, (O)n, (E)m, (const E*)row, (const O*)adj, (const W*)val, (const W*)vw, part, k, out);
            return JET_OK;
        });
    }

    static int project(int64_t n_fine, const void* map, const int32_t* coarse, int32_t* fine, void* stream) {
        return guarded([&]() -> int {
            cudaStream_t s = pick_stream(stream);
            if (n_fine > 0) {
                k_project<O><<<grid_persistent(n_fine, 16), BLOCK, 0, s>>>((O)n_fine, (const O*)map, coarse, fine); count_launch();
                JET_LAUNCH_CHECK();
            }
            stream_wait(s);
            return JET_OK;
        });
    }

    // app/import_coarse.cpp:49-132: load a dumped hierarchy (reference
    // layout, this tier's types) and its coarsest partition, then uncoarsen.
    static int refine_hierarchy(const jet_config_c* cfg, const char* graphs_path, const char* part_path, int32_t* part_out,
                                int64_t part_capacity, int64_t* n_out, int64_t* cut_out, jet_stats_c* st, void* stream) {
        return guarded([&]() -> int {
            if (!cfg || !part_out || !cut_out) throw JetError{JET_ERR_INVALID, "null argument"};
            if (st) std::memset(st, 0, sizeof(*st));
            const char* gp = graphs_path ? graphs_path : "coarse_graphs.out";
            const char* pp = part_path ? part_path : "coarse_part.out";
            Engine<O, E, W> eng(pick_stream(stream));
            cudaStream_t s = eng.s;
            auto t_start = clk::now();
            double meas[JET_NUM_MEASUREMENTS] = {0};
            FILE* f = fopen(gp, "rb");
            if (!f) throw JetError{JET_ERR_INVALID, "cannot open the hierarchy file"};
            std::vector<std::unique_ptr<Level<O, E, W>>> levels;
            int size = 0;
            bool ok = fread(&size, sizeof(int), 1, f) == 1 && size > 0 && size <= 1000;
            O prev_n = 0;
            for (int l = 0; ok && l < size; l++) {
                O n = 0;
                E m = 0;
                ok = fread(&n, sizeof(O), 1, f) == 1 && fread(&m, sizeof(E), 1, f) == 1 && n >= 0 && m >= 0;
                if (!ok) break;
                std::vector<E> row(n + 1);
                std::vector<O> adj(m), map(l > 0 ? prev_n : 0);
                std::vector<W> val(m), vw(n);
                ok = fread(row.data(), sizeof(E), n + 1, f) == (size_t)(n + 1) && fread(adj.data(), sizeof(O), m, f) == (size_t)m &&
                     fread(val.data(), sizeof(W), m, f) == (size_t)m && fread(vw.data(), sizeof(W), n, f) == (size_t)n &&
                     fread(map.data(), sizeof(O), map.size(), f) == map.size();
                if (!ok) break;
                std::unique_ptr<Level<O, E, W>> L(new Level<O, E, W>());
                L->n = n;
                L->m = m;
                L->own_row.alloc(n + 1, s);
                L->own_adj.alloc(m > 0 ? m : 1, s);
                L->own_val.alloc(m > 0 ? m : 1, s);
                L->own_vw.alloc(n > 0 ? n : 1, s);
                JET_CUDA(cudaMemcpyAsync(L->own_row.p, row.data(), sizeof(E) * (n + 1), cudaMemcpyHostToDevice, s));
                if (m) {
                    JET_CUDA(cudaMemcpyAsync(L->own_adj.p, adj.data(), sizeof(O) * m, cudaMemcpyHostToDevice, s));
                    JET_CUDA(cudaMemcpyAsync(L->own_val.p, val.data(), sizeof(W) * m, cudaMemcpyHostToDevice, s));
                }
                if (n) JET_CUDA(cudaMemcpyAsync(L->own_vw.p, vw.data(), sizeof(W) * n, cudaMemcpyHostToDevice, s));
                if (l > 0) {
                    L->map.alloc(prev_n > 0 ? prev_n : 1, s);
                    if (prev_n) JET_CUDA(cudaMemcpyAsync(L->map.p, map.data(), sizeof(O) * prev_n, cudaMemcpyHostToDevice, s));
                }
                stream_wait(s);  // host vectors go out of scope
                L->row = L->own_row.p;
                L->adj = L->own_adj.p;
                L->val = L->own_val.p;
                L->vw = L->own_vw.p;
                L->uniform = false;  // imported levels carry no uniform flag (reference default)
                eng.prepare_level(*L);
                levels.push_back(std::move(L));
                prev_n = n;
            }
            fclose(f);
            if (!ok) throw JetError{JET_ERR_INVALID, "malformed hierarchy file"};
            validate<O, E, W>(eng, levels[0]->n, levels[0]->m, levels[0]->row, levels[0]->adj, levels[0]->val, levels[0]->vw);
            O n0 = levels[0]->n, nc = levels.back()->n;
            if (n_out) *n_out = (int64_t)n0;
            if ((int64_t)n0 > part_capacity) throw JetError{JET_ERR_INVALID, "part_out too small for the finest level"};
            DBuf<part_t> pa(n0 > 0 ? n0 : 1, s), pb(n0 > 0 ? n0 : 1, s), pout(n0 > 0 ? n0 : 1, s);
            {
                std::vector<part_t> cp(nc);
                FILE* pf = fopen(pp, "rb");
                bool pok = pf && fread(cp.data(), sizeof(part_t), nc, pf) == (size_t)nc;
                if (pf) fclose(pf);
                if (!pok) throw JetError{JET_ERR_INVALID, "cannot read the coarse partition file"};
                for (part_t p : cp)
                    if (p < 0 || p >= cfg->num_parts) throw JetError{JET_ERR_INVALID, "part id out of range in the coarse partition"};
                if (nc) JET_CUDA(cudaMemcpyAsync(pa.p, cp.data(), sizeof(part_t) * nc, cudaMemcpyHostToDevice, s));
                stream_wait(s);
            }
            Cfg c{cfg->coarsening_alg, cfg->num_parts, cfg->max_imb_ratio, cfg->refine_tolerance, cfg->ultra_settings != 0,
                  cfg->verbose != 0, false};
            double t_load = since(t_start);
            W cut = uncoarsen_levels<O, E, W>(eng, c, levels, pa, pb, pout.p, st, meas, t_start, 0.0, (int64_t)nc);
            if (st) st->measurements[M_INITPARTITION] = t_load;
            if (n0) JET_CUDA(cudaMemcpyAsync(part_out, pout.p, sizeof(part_t) * n0, cudaMemcpyDeviceToHost, s));
            stream_wait(s);
            *cut_out = (int64_t)cut;
            return JET_OK;
        });
    }
};

// Per-tier function table used by the tier-generic entry points.
struct TierOps {
    int (*coarsen_map)(int, int, uint64_t, int64_t, int64_t, const void*, const void*, const void*, const void*, int, void*, void*,
                       int64_t*, void*);
    int (*contract)(int64_t, int64_t, const void*, const void*, const void*, const void*, const void*, int64_t, void*, void*, void*,
                    void*, int64_t*, void*);
    int (*conn_build)(int64_t, int64_t, const void*, const void*, const void*, const int32_t*, int32_t, void*, int32_t*, void*,
                      int32_t*, void*);
    int (*refine_iters)(int64_t, int64_t, const void*, const void*, const void*, const void*, int32_t*, int32_t, double, double,
                        int32_t, void*, int64_t*, void*, int32_t*, void*, int32_t*, int32_t*, int64_t*, int32_t*, void*);
    int (*refine_level)(int64_t, int64_t, const void*, const void*, const void*, const void*, int32_t*, int32_t, double, double, int,
                        int64_t*, int32_t*, void*);
    int (*pstat)(int64_t, int64_t, const void*, const void*, const void*, const void*, const int32_t*, int32_t, int64_t*, void*);
    int (*project)(int64_t, const void*, const int32_t*, int32_t*, void*);
    int (*refine_hierarchy)(const jet_config_c*, const char*, const char*, int32_t*, int64_t, int64_t*, int64_t*, jet_stats_c*,
                            void*);
};

template <class O, class E, class W>
TierOps make_ops() {
    using T = Tier<O, E, W>;
    return TierOps{&T::coarsen_map, &T::contract, &T::conn_build, &T::refine_iters, &T::refine_level, &T::pstat, &T::project,
                   &T::refine_hierarchy};
}

TierOps ops_i32();
TierOps ops_big();
TierOps ops_biggest();

}  // namespace jetb
