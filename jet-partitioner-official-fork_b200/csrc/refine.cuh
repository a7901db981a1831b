// refine.cuh -- Jet refinement kernels (src/jet_refiner.hpp of the reference).
//
// Connectivity tables: vertex i owns cap(i) = min(deg(i), k) slots starting at
// coff[i]; the first csize[i] of them form an open-addressed table part ->
// summed edge weight (home slot slot_home(p, size, k), linear probing;
// direct-mapped when size == k; the reference uses p % size, and only the
// slot layout differs).  Slots are {part, weight} pairs so a probe and its update touch
// one cache line.  Table sizes follow the reference exactly: built at cap,
// shrunk to used + max(used/4, 3) when that is smaller, grown by appends when
// an incremental insert finds no free slot.
//
// Ties between equally connected destination parts go to the lowest part id
// (the reference takes the first hash slot, which depends on slot layout).
#pragma once
#include "graph.cuh"

namespace jetb {

template <class W>
struct Slot {
    part_t p;
    W v;
};

// Visits slots [0, sz) of a table in order, loading four at a time before
// the first use: a one-thread scan of a row's table is a chain of dependent
// waits otherwise (each use stalls the next load's issue).
template <class W, class F>
__device__ __forceinline__ void scan_slots(const Slot<W>* base, part_t sz, F&& body) {
    for (part_t s0 = 0; s0 < sz; s0 += 4) {
        Slot<W> sl[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (s0 + u < sz) sl[u] = base[s0 + u];
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (s0 + u < sz) body(sl[u]);
    }
}

// Home slot of part p in a table of `size` slots: p itself when the table is
// direct-mapped (size == k), else a multiplicative hash scaled to the size
// (no division).  Only the slot layout depends on this choice, never a
// table's contents or size.
__host__ __device__ __forceinline__ part_t slot_home(part_t p, part_t size, part_t k) {
    if (size == k) return p;
    return (part_t)(((uint64_t)((uint32_t)p * 0x9E3779B1u) * (uint64_t)(uint32_t)size) >> 32);
}

__host__ __device__ __forceinline__ part_t shrunk_size(part_t used, part_t cap) {
    part_t q = used / 4;
    if (q < 3) q = 3;
    part_t s = used + q;
    return s < cap ? s : cap;
}

template <class E>
__host__ __device__ __forceinline__ part_t conn_cap(E deg, part_t k) { return deg > (E)k ? k : (part_t)deg; }

template <class O, class E>
struct GetConnCap {
    const E* row;
    part_t k;
    __device__ __forceinline__ E operator()(int64_t i) const { return (E)conn_cap<E>(row[i + 1] - row[i], k); }
};

// Device-resident per-iteration counters and results.
template <class O, class W>
struct RefDev {
    O ncand;
    O nmoves;
    O ncand_hub;
    O nmoves_hub;
    O nredraw;
    W cut1, cut2;
    W vw_cursor;          // strong rebalance: next free position past the evictions
    W max_vwgt;
    part_t total_undersized;
    int err;
    int large;            // this iteration used update_large
    O nord;               // rebalance: candidates queued for in-bucket ordering
    O nord_last;          // (their count in the last rebalance, for profiling)
    int reb_fb;           // rebalance: the queue cannot be used (fallback to the full sort)
    int reb_fb_taken;     // the last rebalance took the fallback
    int reb_fb_count[2];  // fallbacks taken inside the current level graph (weak, strong)
};
// Copied to pinned host memory once per iteration.
struct IterResult {
    int64_t nmoves;
    int64_t cut_change;
    int64_t max_part;
    int32_t err;
    int32_t large;
};

template <class O, class E, class W>
struct RefArgs {
    GView<O, E, W> g;
    part_t k;
    const E* coff;
    Slot<W>* slots;
    part_t* csize;
    part_t* dest_cache;
    uint8_t* lock;
    uint8_t* mark;
    part_t* part;
    part_t* dest;
    W* save_gain;
    W* pregain;
    W* sizes;
    O* cand;
    O* cand_hub;
    O* moves;
    O* moves_hub;
    RefDev<O, W>* dev;
    const double* filter;  // LP filter ratio, read on the device (it changes per iteration with ultra settings)
    int narrow;            // every row's summed edge weight fits in 32 bits (see acc_add)
    unsigned long long* pclk;  // per-phase clock totals of the persistent level loops, or null (jet_prof_phases)
};

// Per-phase clock totals of a persistent level loop, kept by one thread in
// local memory and added to a.pclk when the loop ends (phase-time profiling
// only; nothing is recorded without a.pclk).  Slots [base + id] hold cycles,
// [base + PHASE_SLOTS + id] the number of times the phase ran.
static constexpr int PHASE_SLOTS = 24;
enum PhaseId : int {
    PH_LP_SELECT = 0, PH_AFTERBURN, PH_AFTERBURN_HUB, PH_REB_PREP, PH_REB_SELECT, PH_REB_SCAN, PH_REB_SORT, PH_REB_EVICT,
    PH_STRONG_TAIL, PH_APPLY, PH_UPDATE_SUB, PH_UPDATE_ADD, PH_REBUILD, PH_CUT, PH_CTL, PH_COPY,
    PH_COOKIE, PH_STRONG_FIRST, PH_REDRAW, PH_WEIGHT_SCAN, PH_COUNT
};
struct PhaseClock {
    unsigned long long* out;
    int base;
    bool on;
    long long last;
    unsigned long long cyc[PH_COUNT];
    unsigned cnt[PH_COUNT];
    __device__ PhaseClock(unsigned long long* p, int b, bool owner) : out(p), base(b), on(p != nullptr && owner), last(0) {
        if (on) {
            for (int i = 0; i < PH_COUNT; i++) { cyc[i] = 0; cnt[i] = 0; }
            last = clock64();
        }
    }
    __device__ __forceinline__ void mark(int id) {
        if (!on) return;
        long long t = clock64();
        cyc[id] += (unsigned long long)(t - last);
        cnt[id]++;
        last = t;
    }
    __device__ void flush() {
        if (!on) return;
        for (int i = 0; i < PH_COUNT; i++) {
            atomicAdd(&out[base + i], cyc[i]);
            atomicAdd(&out[base + PHASE_SLOTS + i], (unsigned long long)cnt[i]);
        }
    }
};


// ---------------------------------------------------------------- table build
// Rows with dlo < deg <= dhi (dhi <= SET <= 32): one thread per vertex, its
// distinct parts gathered in a private SET-entry shared-memory set
// (interleaved so threads hit distinct banks; multiplicative hash into a
// power-of-two set, no division).  Three instances cover deg <= 32: SET = 8
// (256 threads, small enough for full occupancy) for deg <= 8, SET = 16 (256
// threads) for 8 < deg <= 16 and SET = 32 (128 threads) for 16 < deg <= 32,
// the last two launched only when the level has such rows.
// Neighbours are read in batches of 8 with every load issued before the first
// use, so a row costs about two memory latencies instead of two per entry.
// The final table (at most 32 slots) is laid out with a register bitmask of
// occupied slots and written once, with no read-back.
template <int SET>
__device__ __forceinline__ int set_home(part_t p) {
    constexpr int bits = SET == 8 ? 3 : (SET == 16 ? 4 : 5);
    return (int)(((uint32_t)p * 0x9E3779B1u) >> (32 - bits));
}

// With a list (rows of one degree class, *list_count of them, from
// k_bin_short) the threads walk the list instead of every vertex, so whole
// warps stay busy.
template <int SET, int THREADS, class O, class E, class W>
__global__ void __launch_bounds__(THREADS) k_conn_thread(RefArgs<O, E, W> a, int dlo, int dhi, int only_marked, const int* gate,
                                                        const O* list, const O* list_count) {
    __shared__ part_t sk[SET][THREADS];
    __shared__ W sv[SET][THREADS];
    if (gate && !*gate) return;
    const int t = threadIdx.x;
    const int64_t count = list ? (int64_t)*list_count : (int64_t)a.g.n;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + t; x < count; x += (int64_t)gridDim.x * blockDim.x) {
        O i = list ? list[x] : (O)x;
        E rs = a.g.row[i], re = a.g.row[i + 1];
        E deg = re - rs;
        if (deg <= dlo || deg > dhi) continue;
        if (only_marked && !a.mark[i]) continue;
#pragma unroll
        for (int s = 0; s < SET; s++) sk[s][t] = NULL_PART;
        int used = 0;
        for (E j0 = rs; j0 < re; j0 += 8) {
            O vb[8];
            W wb[8];
            part_t pb[8];
#pragma unroll
            for (int u = 0; u < 8; u++) vb[u] = j0 + u < re ? a.g.adj[j0 + u] : (O)0;
#pragma unroll
            for (int u = 0; u < 8; u++) wb[u] = j0 + u < re ? a.g.val[j0 + u] : (W)0;
#pragma unroll
            for (int u = 0; u < 8; u++) pb[u] = j0 + u < re ? a.part[vb[u]] : NULL_PART;
#pragma unroll
            for (int u = 0; u < 8; u++) {
                part_t p = pb[u];
                if (p == NULL_PART) continue;
                int h = set_home<SET>(p);
                // at most deg <= SET distinct parts: a free or matching slot is always found
                while (sk[h][t] != NULL_PART && sk[h][t] != p) h = (h + 1) & (SET - 1);
                if (sk[h][t] == NULL_PART) { sk[h][t] = p; sv[h][t] = wb[u]; used++; }
                else sv[h][t] += wb[u];
            }
        }
        part_t cap = conn_cap<E>(deg, a.k);
        part_t size = cap == 0 ? 0 : shrunk_size(used, cap);
        Slot<W>* base = a.slots + a.coff[i];
        uint32_t occ = 0;  // size <= cap <= 32
        bool ok = true;
#pragma unroll
        for (int s = 0; s < SET; s++) {
            part_t p = sk[s][t];
            if (p == NULL_PART || !ok) continue;
            int po = slot_home(p, size, a.k);
            if (size < a.k) {
                int guard = 0;
                while ((occ >> po) & 1u) {
                    po = po + 1 == size ? 0 : po + 1;
                    if (++guard > size) { ok = false; break; }
                }
                if (!ok) continue;
            }
            occ |= 1u << po;
            Slot<W> sl;
            sl.p = p;
            sl.v = sv[s][t];
            base[po] = sl;
        }
        for (int s = 0; s < cap; s++) {
            if ((occ >> s) & 1u) continue;
            Slot<W> sl;
            sl.p = NULL_PART;
            sl.v = 0;
            base[s] = sl;
        }
        if (!ok) atomicOr(&a.dev->err, ERRF_OVERFLOW);
        a.csize[i] = size;
        if (only_marked) { a.mark[i] = 0; a.dest_cache[i] = NULL_PART; }
    }
}

// Rows of 9-16 and of 17-32 edges into two lists (counts in cnt[0], cnt[1])
// for the SET = 16 and SET = 32 table builds.
template <class O, class E>
__global__ void k_bin_short(O n, const E* row, O* l16, O* l32, O* cnt) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t rounds = ceil_div<int64_t>((int64_t)n, stride);
    for (int64_t r = 0; r < rounds; r++) {
        int64_t i = start + r * stride;
        E d = 0;
        if (i < n) d = row[i + 1] - row[i];
        O s = warp_append(&cnt[0], i < n && d > 8 && d <= 16);
        if (s >= 0) l16[s] = (O)i;
        s = warp_append(&cnt[1], i < n && d > 16 && d <= THREAD_DEG);
        if (s >= 0) l32[s] = (O)i;
    }
}

// Inserts p into a shared-memory table of `cap` slots (direct-mapped when
// cap == k); returns true when this call claimed a new slot.
// `err` receives ERRF_OVERFLOW if the probe sequence exceeds its bound (the
// table always has room: cap >= number of distinct neighbour parts).
template <class W>
__device__ __forceinline__ bool smem_table_add(part_t* keys, W* vals, part_t cap, part_t k, part_t p, W w, int* err,
                                               int narrow = 0) {
    volatile part_t* vk = keys;
    part_t po = slot_home(p, cap, k);
    bool claimed = false;
    if (cap == k) {
        if (vk[po] == NULL_PART && atomicCAS((int*)&keys[po], NULL_PART, p) == NULL_PART) claimed = true;
    } else {
        int guard = 0;
        while (true) {
            part_t px = vk[po];
            while (px != p && px != NULL_PART) {
                po = po + 1 == cap ? 0 : po + 1;
                px = vk[po];
                if (++guard > 2 * cap) { atomicOr(err, ERRF_OVERFLOW); return false; }
            }
            if (px == p) break;
            px = atomicCAS((int*)&keys[po], NULL_PART, p);
            if (px == NULL_PART) { claimed = true; break; }
            if (px == p) break;
            po = po + 1 == cap ? 0 : po + 1;
            if (++guard > 2 * cap) { atomicOr(err, ERRF_OVERFLOW); return false; }
        }
    }
    acc_add<W>(&vals[po], w, narrow);
    return claimed;
}

// Copies a shared-memory table (cap slots, `used` parts) to the vertex's
// global region at its final size.  `tid`/`nt` are the cooperating threads.
template <class W>
__device__ __forceinline__ void smem_table_flush(const part_t* keys, const W* vals, part_t cap, part_t used, part_t k,
                                                 Slot<W>* base, part_t* size_out, int tid, int nt, bool sync_block, int* err) {
    part_t size = shrunk_size(used, cap);
    if (size == cap) {
        for (int s = tid; s < cap; s += nt) { base[s].p = keys[s]; base[s].v = vals[s]; }
    } else {
        for (int s = tid; s < cap; s += nt) { base[s].p = NULL_PART; base[s].v = 0; }
        if (sync_block) __syncthreads(); else __syncwarp();
        for (int s = tid; s < cap; s += nt) {
            part_t p = keys[s];
            if (p == NULL_PART) continue;
            part_t po = slot_home(p, size, k);
            int guard = 0;
            bool placed = true;
            while (true) {
                part_t old = atomicCAS((int*)&base[po].p, NULL_PART, p);
                if (old == NULL_PART) break;
                po = po + 1 == size ? 0 : po + 1;
                if (++guard > size) { atomicOr(err, ERRF_OVERFLOW); placed = false; break; }
            }
            if (placed) base[po].v = vals[s];
        }
    }
    if (tid == 0) *size_out = size;
}

// Adds edges rs+t, rs+t+nt, ... of a row into a shared-memory table; four
// edges per thread per round with every load issued before the first use
// (the part gather depends on the neighbour id load).  Returns the slots this
// thread claimed.
template <class O, class E, class W>
__device__ __forceinline__ int table_add_edges(const RefArgs<O, E, W>& a, part_t* keys, W* vals, part_t cap, E rs, E re, int t,
                                               int nt) {
    int mine = 0;
    for (E j0 = rs + t; j0 < re; j0 += 4 * (E)nt) {
        O v[4];
        W w[4];
        part_t p[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            E j = j0 + (E)u * nt;
            v[u] = j < re ? a.g.adj[j] : (O)0;
            w[u] = j < re ? a.g.val[j] : (W)0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) p[u] = j0 + (E)u * nt < re ? a.part[v[u]] : NULL_PART;
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (p[u] != NULL_PART) mine += smem_table_add<W>(keys, vals, cap, a.k, p[u], w[u], &a.dev->err, a.narrow);
    }
    return mine;
}

// 32 < deg <= 4096 and k <= WARP_TABLE: one warp per vertex, table in shared memory.
static constexpr int WARP_TABLE = 512;

// Writes a row's table from a direct-mapped accumulator: vals[p] is the
// row's summed weight to part p (p < k; zero = absent).  A table of size k
// stays direct-mapped; a smaller one is laid out in keys[0, size) by
// inserting every present part from its home (shared-memory CAS, linear
// probing), then every slot is written once, its weight read back through its
// key.  The region holds cap = min(deg, k) slots; [size, cap) is cleared.
// `t`/`nt` are the cooperating threads (a warp or the block; `block` picks the
// barrier).
// With `clear`, every weight read is zeroed, leaving vals all zero.
template <class W>
__device__ __forceinline__ void direct_table_write(part_t* keys, W* vals, part_t k, part_t cap, part_t used, Slot<W>* base,
                                                   part_t* size_out, int t, int nt, bool block, int* err, bool clear = false) {
    const part_t size = shrunk_size(used, cap);
    if (size == k) {
        for (int p = t; p < k; p += nt) {
            Slot<W> sl;
            sl.v = vals[p];
            sl.p = sl.v != 0 ? (part_t)p : NULL_PART;
            base[p] = sl;
            if (clear && sl.v != 0) vals[p] = 0;
        }
    } else {
        for (int q = t; q < size; q += nt) keys[q] = NULL_PART;
        if (block) __syncthreads(); else __syncwarp();
        for (int p = t; p < k; p += nt) {
            if (vals[p] == 0) continue;
            part_t po = slot_home((part_t)p, size, k);
            int guard = 0;
            while (atomicCAS((int*)&keys[po], NULL_PART, p) != NULL_PART) {
                po = po + 1 == size ? 0 : po + 1;
                if (++guard > size) { atomicOr(err, ERRF_OVERFLOW); break; }
            }
        }
        if (block) __syncthreads(); else __syncwarp();
        for (int q = t; q < cap; q += nt) {
            Slot<W> sl;
            sl.p = q < size ? keys[q] : NULL_PART;
            sl.v = sl.p >= 0 ? vals[sl.p] : (W)0;
            base[q] = sl;
            if (clear && sl.p >= 0) vals[sl.p] = 0;  // each present part sits in one slot
        }
    }
    if (t == 0) *size_out = size;
}

// Writes a row's table from a shared-memory hash table of cap slots (keys,
// vals [0, cap), `used` parts present).  When the table shrinks it is
// rehashed into keys/vals [cap, cap + size) (the caller guarantees the room)
// and every slot of the row's region is then written once.
template <class W>
__device__ __forceinline__ void hashed_table_write(part_t* keys, W* vals, part_t cap, part_t used, part_t k, Slot<W>* base,
                                                   part_t* size_out, int t, int nt, int* err) {
    const part_t size = shrunk_size(used, cap);
    if (size == cap) {
        for (int q = t; q < cap; q += nt) {
            Slot<W> sl;
            sl.p = keys[q];
            sl.v = vals[q];
            base[q] = sl;
            vals[q] = 0;
        }
    } else {
        part_t* tk = keys + cap;
        W* tv = vals + cap;
        for (int q = t; q < size; q += nt) tk[q] = NULL_PART;
        __syncwarp();
        for (int q = t; q < cap; q += nt) {
            const part_t p = keys[q];
            if (p == NULL_PART) continue;
            part_t po = slot_home(p, size, k);
            int guard = 0;
            bool placed = true;
            while (atomicCAS((int*)&tk[po], NULL_PART, p) != NULL_PART) {
                po = po + 1 == size ? 0 : po + 1;
                if (++guard > size) { atomicOr(err, ERRF_OVERFLOW); placed = false; break; }
            }
            if (placed) tv[po] = vals[q];
        }
        __syncwarp();
        for (int q = t; q < cap; q += nt) {
            Slot<W> sl;
            sl.p = q < size ? tk[q] : NULL_PART;
            sl.v = sl.p >= 0 ? tv[q] : (W)0;
            base[q] = sl;
            vals[q] = 0;
            if (q < size) tv[q] = 0;
        }
    }
    if (t == 0) *size_out = size;
}

// One row's table built by one warp in its own shared-memory slice (`keys`,
// `vals`: k entries each, k <= WARP_TABLE; vals all zero on entry, and left
// all zero).  Rows with cap >= k / 4: every edge adds its weight at its
// part's index (no hashing, no slot claiming), the nonzero entries are
// counted, and the table is written by direct_table_write, which clears what
// it reads (no clearing pass per row).  Shorter rows, for which scanning k entries would
// dominate: a hash table of cap slots, rehashed in the slice's upper part
// when it shrinks (2 cap < k).
template <class O, class E, class W>
__device__ __forceinline__ void conn_warp_row(const RefArgs<O, E, W>& a, O i, E rs, E re, part_t* keys, W* vals, int lane,
                                              int only_marked) {
    const part_t k = a.k;
    const part_t cap = conn_cap<E>(re - rs, k);
    if (4 * cap < k) {
        for (int s = lane; s < cap; s += 32) { keys[s] = NULL_PART; vals[s] = 0; }
        __syncwarp();
        int mine = table_add_edges<O, E, W>(a, keys, vals, cap, rs, re, lane, 32);
        __syncwarp();
        const int used = group_sum<int>(mine, 32);
        hashed_table_write<W>(keys, vals, cap, used, k, a.slots + a.coff[i], &a.csize[i], lane, 32, &a.dev->err);
        if (only_marked && lane == 0) { a.mark[i] = 0; a.dest_cache[i] = NULL_PART; }
        __syncwarp();
        return;
    }
    for (E j0 = rs + lane; j0 < re; j0 += 4 * 32) {
        O v[4];
        W w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            E j = j0 + (E)u * 32;
            v[u] = j < re ? a.g.adj[j] : (O)0;
            w[u] = j < re ? a.g.val[j] : (W)0;
        }
        part_t p[4];
#pragma unroll
        for (int u = 0; u < 4; u++) p[u] = j0 + (E)u * 32 < re ? a.part[v[u]] : NULL_PART;
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (p[u] != NULL_PART) acc_add<W>(&vals[p[u]], w[u], a.narrow);
    }
    __syncwarp();
    int mine = 0;
    for (int s = lane; s < k; s += 32) mine += vals[s] != 0;
    const int used = group_sum<int>(mine, 32);
    direct_table_write<W>(keys, vals, k, cap, used, a.slots + a.coff[i], &a.csize[i], lane, 32, false, &a.dev->err, true);
    if (only_marked && lane == 0) { a.mark[i] = 0; a.dest_cache[i] = NULL_PART; }
    __syncwarp();
}

template <class O, class E, class W>
__device__ __forceinline__ void d_conn_warp(RefArgs<O, E, W> a, const O* list, O count, int only_marked, const int* gate,
                                            int64_t max_deg = INT64_MAX) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (gate && !*gate) return;
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kw = a.k < WARP_TABLE ? a.k : WARP_TABLE;
    const int nw = (int)(blockDim.x >> 5);
    part_t* keys = (part_t*)smem_raw + wid * kw;
    W* vals = (W*)(smem_raw + (((size_t)nw * kw * sizeof(part_t) + 15) & ~(size_t)15)) + wid * kw;
    for (int s = lane; s < kw; s += 32) vals[s] = 0;  // conn_warp_row keeps it zero
    __syncwarp();
    const int64_t warps = (int64_t)gridDim.x * nw;
    for (int64_t x = blockIdx.x * (int64_t)nw + wid; x < count; x += warps) {
        O i = list ? list[x] : (O)x;  // no list: every vertex
        if (only_marked && !a.mark[i]) continue;
        E rs = a.g.row[i], re = a.g.row[i + 1];
        if ((int64_t)(re - rs) > max_deg) continue;  // left to the CTA-per-row kernel
        conn_warp_row<O, E, W>(a, i, rs, re, keys, vals, lane, only_marked);
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_conn_warp(RefArgs<O, E, W> a, const O* list, O count, int only_marked, const int* gate,
                                                     int64_t max_deg) {
    d_conn_warp<O, E, W>(a, list, count, only_marked, gate, max_deg);
}

// One row with cap == k built by a whole block: every warp accumulates its
// share of the edges into its own direct-mapped array of k weights in `acc`
// (no slot claiming, no contention between warps); the arrays are summed into
// the table (`keys`, `vals`: k entries each) and the table is written out.
// Edge weights are positive, so a nonzero sum marks a present part.
template <class O, class E, class W>
__device__ __forceinline__ void conn_block_row_priv(const RefArgs<O, E, W>& a, O i, E rs, E re, W* acc, part_t* keys, W* vals,
                                                    int* s_used, int only_marked) {
    // acc is all zero on entry (conn_priv_zero before the first row) and is
    // left all zero: the merge clears every entry it reads
    const int nw = (int)(blockDim.x >> 5), wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) *s_used = 0;
    W* my = acc + wid * a.k;
    for (E j0 = rs + threadIdx.x; j0 < re; j0 += 4 * (E)blockDim.x) {
        O v[4];
        W w[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            E j = j0 + (E)u * blockDim.x;
            v[u] = j < re ? a.g.adj[j] : (O)0;
            w[u] = j < re ? a.g.val[j] : (W)0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (j0 + (E)u * blockDim.x < re) acc_add<W>(&my[a.part[v[u]]], w[u], a.narrow);
    }
    __syncthreads();
    // merge: one thread per part sums the nw arrays (consecutive parts on
    // consecutive lanes: no bank conflicts), clearing each entry it reads
    int used = 0;
    for (int p = threadIdx.x; p < a.k; p += blockDim.x) {
        W sum = 0;
        for (int w = 0; w < nw; w++) { sum += acc[w * a.k + p]; acc[w * a.k + p] = 0; }
        vals[p] = sum;
        used += sum != 0;
    }
    used = group_sum<int>(used, 32);
    if ((threadIdx.x & 31) == 0 && used) atomicAdd(s_used, used);
    __syncthreads();
    direct_table_write<W>(keys, vals, a.k, a.k, *s_used, a.slots + a.coff[i], &a.csize[i], threadIdx.x, blockDim.x, true,
                          &a.dev->err);
    if (only_marked && threadIdx.x == 0) { a.mark[i] = 0; a.dest_cache[i] = NULL_PART; }
    __syncthreads();
}

// Clears the per-warp accumulators of conn_block_row_priv once per block.
template <class W>
__device__ __forceinline__ void conn_priv_zero(W* acc, int entries) {
    for (int s = threadIdx.x; s < entries; s += blockDim.x) acc[s] = 0;
    __syncthreads();
}

// Rows of degree > THREAD_DEG (k <= WARP_TABLE), one persistent launch.
// `order` lists them longest first (by power-of-two degree class); a shared
// counter hands them out.  Rows of at least `block_min` edges (block_min >= k,
// so their tables are direct-mapped) go to a whole block each, the rest to
// single warps: a block draws rows until it draws one below block_min, gives
// that one to its warp 0, and from then on every warp draws its own rows.
// Longest-first keeps the long rows off the critical path's end.  The last
// block to finish zeroes the counters for the next launch.
//
// Shared memory: the larger of nw * k weights + one k-entry table (block
// rows) and nw per-warp tables of k entries (warp rows); the second is larger.
template <class O, class E, class W>
__global__ void __launch_bounds__(1024, 2) k_conn_long(RefArgs<O, E, W> a, const O* order, O count, int only_marked,
                                                   const int* gate, unsigned* ctr, int64_t block_min) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned s_x;
    __shared__ int s_used;
    if (gate && !*gate) return;
    const int nw = (int)(blockDim.x >> 5), wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = a.k;
    const size_t key_bytes = ((size_t)nw * k * sizeof(part_t) + 15) & ~(size_t)15;
    bool warp_mode = false;
    O pending = 0;  // warp 0: the first warp row, drawn by the whole block
    bool has_pending = false;
    conn_priv_zero<W>((W*)smem_raw, nw * k);
    while (true) {
        if (threadIdx.x == 0) s_x = atomicAdd(&ctr[0], 1u);
        __syncthreads();
        const unsigned x = s_x;
        __syncthreads();
        if (x >= (unsigned)count) break;
        const O i = order[x];
        const E rs = a.g.row[i], re = a.g.row[i + 1];
        if ((int64_t)(re - rs) < block_min) {
            if (wid == 0) { pending = i; has_pending = true; }
            warp_mode = true;
            break;
        }
        if (only_marked && !a.mark[i]) continue;
        W* acc = (W*)smem_raw;
        unsigned char* tbl = smem_raw + (((size_t)nw * k * sizeof(W) + 15) & ~(size_t)15);
        conn_block_row_priv<O, E, W>(a, i, rs, re, acc, (part_t*)tbl, (W*)(tbl + (((size_t)k * sizeof(part_t) + 15) & ~(size_t)15)),
                                     &s_used, only_marked);
    }
    if (warp_mode) {
        part_t* keys = (part_t*)smem_raw + wid * k;
        W* vals = (W*)(smem_raw + key_bytes) + wid * k;
        __syncthreads();  // block rows are done with the shared memory
        for (int s = lane; s < k; s += 32) vals[s] = 0;  // conn_warp_row keeps it zero
        __syncwarp();
        while (true) {
            O i;
            if (has_pending) {
                i = pending;
                has_pending = false;
            } else {
                unsigned x = 0;
                if (lane == 0) x = atomicAdd(&ctr[0], 1u);
                x = __shfl_sync(0xffffffffu, x, 0);
                if (x >= (unsigned)count) break;
                i = order[x];
            }
            if (only_marked && !a.mark[i]) continue;
            conn_warp_row<O, E, W>(a, i, a.g.row[i], a.g.row[i + 1], keys, vals, lane, only_marked);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctr[1], 1u) == gridDim.x - 1) {
            ctr[0] = 0;
            ctr[1] = 0;
            __threadfence();
        }
    }
}
template <class W>
__host__ __device__ constexpr size_t conn_long_smem(int nw, int k) {
    return ((((size_t)nw * k * sizeof(part_t) + 15) & ~(size_t)15) + (size_t)nw * k * sizeof(W) + 16);
}

// Power-of-two degree class of a row of the warp or hub list, as a sort key
// that puts longer rows first.
template <class O, class E>
struct GetLongKey {
    const O* warp_list;
    const O* hub_list;
    O n_warp;
    const E* row;
    __device__ __forceinline__ uint32_t operator()(int64_t x) const {
        O i = x < n_warp ? warp_list[x] : hub_list[x - n_warp];
        uint64_t d = (uint64_t)(row[i + 1] - row[i]);
        return (uint32_t)__clzll((long long)d);  // 63 - floor(log2 d), d > 0
    }
};
template <class O>
struct GetLongRow {
    const O* warp_list;
    const O* hub_list;
    O n_warp;
    __device__ __forceinline__ O operator()(int64_t x) const { return x < n_warp ? warp_list[x] : hub_list[x - n_warp]; }
};

// Any degree: one CTA per vertex, table of cap <= k slots in shared memory.
// With `priv` (the launch gave nw * k weights of shared memory beyond the
// table) a row with cap == k accumulates into one private direct-mapped
// array per warp (no slot claiming, no contention between warps), which are
// summed into the table afterwards; edge weights are positive, so a nonzero
// sum marks a present part.
__device__ __forceinline__ size_t conn_cta_priv_bytes(int nw, int k, size_t wbytes) {
    return (((size_t)nw * k * wbytes + 15) & ~(size_t)15);
}
template <class O, class E, class W>
__device__ __forceinline__ void d_conn_cta(RefArgs<O, E, W> a, const O* list, O count, int only_marked, const int* gate,
                                           int64_t min_deg = 0, int priv = 0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_used;
    if (gate && !*gate) return;
    const int nw = (int)(blockDim.x >> 5);
    W* acc = (W*)smem_raw;  // priv: nw x k
    unsigned char* tbl = smem_raw + (priv ? conn_cta_priv_bytes(nw, a.k, sizeof(W)) : 0);
    part_t* keys = (part_t*)tbl;
    W* vals = (W*)(tbl + ((a.k * sizeof(part_t) + 15) & ~(size_t)15));
    if (priv) conn_priv_zero<W>(acc, nw * a.k);
    for (O x = blockIdx.x; x < count; x += gridDim.x) {
        O i = list[x];
        if (only_marked && !a.mark[i]) continue;
        if ((int64_t)(a.g.row[i + 1] - a.g.row[i]) <= min_deg) continue;  // done by the warp kernel
        E rs = a.g.row[i], re = a.g.row[i + 1];
        part_t cap = conn_cap<E>(re - rs, a.k);
        if (priv && cap == a.k) {
            conn_block_row_priv<O, E, W>(a, i, rs, re, acc, keys, vals, &s_used, only_marked);
            continue;
        }
        for (int s = threadIdx.x; s < cap; s += blockDim.x) { keys[s] = NULL_PART; vals[s] = 0; }
        if (threadIdx.x == 0) s_used = 0;
        __syncthreads();
        int mine = 0;
        mine += table_add_edges<O, E, W>(a, keys, vals, cap, rs, re, threadIdx.x, blockDim.x);
        mine = group_sum<int>(mine, 32);
        if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&s_used, mine);
        __syncthreads();
        smem_table_flush<W>(keys, vals, cap, s_used, a.k, a.slots + a.coff[i], &a.csize[i], threadIdx.x, blockDim.x, true, &a.dev->err);
        if (only_marked && threadIdx.x == 0) { a.mark[i] = 0; a.dest_cache[i] = NULL_PART; }
        __syncthreads();
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_conn_cta(RefArgs<O, E, W> a, const O* list, O count, int only_marked, const int* gate,
                                                   int64_t min_deg, int priv) {
    d_conn_cta<O, E, W>(a, list, count, only_marked, gate, min_deg, priv);
}

// ---------------------------------------------------------------- lookups
template <class W>
__device__ __forceinline__ W table_lookup(const Slot<W>* base, part_t target, part_t size, part_t k) {  // src/jet_refiner.hpp:891-901
    if (size <= 0) return 0;
    part_t pi = slot_home(target, size, k);
    for (part_t q = 0; q < size; q++) {
        part_t e = base[pi].p;
        if (e == target) return base[pi].v;
        if (e == NULL_PART) return 0;
        pi = pi + 1 == size ? 0 : pi + 1;
    }
    return 0;
}

// ---------------------------------------------------------------- LP select
// Best destination (most connected part other than the own one; ties to the
// lowest part id) and the filter of src/jet_refiner.hpp:206-251, then the
// candidate list of :255-266.
template <class W>
__device__ __forceinline__ bool lp_better(W c, part_t e, W bc, part_t be) {
    return c > 0 && (c > bc || (c == bc && e < be));
}

template <class O, class E, class W>
__device__ __forceinline__ void lp_finish(const RefArgs<O, E, W>& a, O i, part_t best, W b_conn, W p_conn, double filter_ratio,
                                          bool computed) {
    if (computed) {
        W sg = 0;
        if (best != NO_MOVE) {
            if (b_conn >= p_conn || ((double)(p_conn - b_conn) < floor(filter_ratio * (double)p_conn))) sg = b_conn - p_conn;
            else best = NO_MOVE;
        }
        a.save_gain[i] = sg;
        a.dest_cache[i] = best;
    }
    a.dest[i] = best;
}

template <class O, class E, class W>
__device__ __forceinline__ void d_lp_select_thread(RefArgs<O, E, W> a) {
    const W GAIN_MIN = std::numeric_limits<W>::lowest();
    const double filter_ratio = *a.filter;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t rounds = ceil_div<int64_t>((int64_t)a.g.n, stride);
    for (int64_t r = 0; r < rounds; r++) {
        int64_t x = start + r * stride;
        bool cand = false;
        O i = (O)x;
        if (x < a.g.n && a.g.row[i + 1] - a.g.row[i] <= THREAD_DEG) {
            part_t best = a.dest_cache[i];
            if (best != NULL_PART) {
                lp_finish<O, E, W>(a, i, best, 0, 0, filter_ratio, false);
            } else {
                part_t p = a.part[i];
                best = NO_MOVE;
                W b_conn = 0, p_conn = 0;
                const Slot<W>* base = a.slots + a.coff[i];
                part_t sz = a.csize[i];
                scan_slots<W>(base, sz, [&](const Slot<W>& sl) {
                    if (sl.p != p) { if (lp_better<W>(sl.v, sl.p, b_conn, best)) { best = sl.p; b_conn = sl.v; } }
                    else if (sl.v > 0) p_conn = sl.v;
                });
                lp_finish<O, E, W>(a, i, best, b_conn, p_conn, filter_ratio, true);
                best = a.dest[i];
            }
            cand = best != NO_MOVE && a.lock[i] == 0;
            if (cand) a.pregain[i] = a.save_gain[i];
            else { a.pregain[i] = GAIN_MIN; a.lock[i] = 0; }
        }
        O s = warp_append(&a.dev->ncand, cand);
        if (cand) a.cand[s] = i;
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_lp_select_thread(RefArgs<O, E, W> a) { d_lp_select_thread<O, E, W>(a); }

// Vertices with deg > 32: one warp per vertex scans its table.
template <class O, class E, class W>
__device__ __forceinline__ void d_lp_select_warp(RefArgs<O, E, W> a, const O* list, O count) {
    const W GAIN_MIN = std::numeric_limits<W>::lowest();
    const double filter_ratio = *a.filter;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (int)(blockDim.x >> 5);
    for (int64_t x = blockIdx.x * (int64_t)(int)(blockDim.x >> 5) + (threadIdx.x >> 5); x < count; x += warps) {
        O i = list[x];
        part_t best = a.dest_cache[i];
        if (best != NULL_PART) {
            if (lane == 0) lp_finish<O, E, W>(a, i, best, 0, 0, filter_ratio, false);
        } else {
            part_t p = a.part[i];
            best = NO_MOVE;
            W b_conn = 0, p_conn = 0;
            const Slot<W>* base = a.slots + a.coff[i];
            part_t sz = a.csize[i];
            for (part_t s = lane; s < sz; s += 32) {
                Slot<W> sl = base[s];
                if (sl.p != p) { if (lp_better<W>(sl.v, sl.p, b_conn, best)) { best = sl.p; b_conn = sl.v; } }
                else if (sl.v > 0) p_conn = sl.v;
            }
            for (int m = 16; m > 0; m >>= 1) {
                W c2 = shfl_xor(b_conn, m, 32);
                part_t e2 = shfl_xor(best, m, 32);
                if (lp_better<W>(c2, e2, b_conn, best)) { b_conn = c2; best = e2; }
                W pc2 = shfl_xor(p_conn, m, 32);
                if (pc2 > p_conn) p_conn = pc2;
            }
            if (lane == 0) lp_finish<O, E, W>(a, i, best, b_conn, p_conn, filter_ratio, true);
        }
        __syncwarp();
        if (lane == 0) {
            best = a.dest[i];
            bool cand = best != NO_MOVE && a.lock[i] == 0;
            if (cand) {
                a.pregain[i] = a.save_gain[i];
                O s = atomic_add(&a.dev->ncand, (O)1);
                a.cand[s] = i;
            } else {
                a.pregain[i] = GAIN_MIN;
                a.lock[i] = 0;
            }
        }
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_lp_select_warp(RefArgs<O, E, W> a, const O* list, O count) { d_lp_select_warp<O, E, W>(a, list, count); }

// ---------------------------------------------------------------- afterburner
// src/jet_refiner.hpp:275-307: a candidate keeps its move if its gain,
// recomputed assuming every higher-priority candidate (larger pre-gain, then
// smaller id) has already moved, is non-negative.
// A candidate's gain change from its edges j0, j0 + stride, ... < e: an
// edge to a higher-priority neighbour v counts -w / +w for v's destination
// and +w / -w for v's current part being the candidate's part p / best.
// Four edges per round, with every round's loads (neighbours, weights, their
// pregains, then their destinations and parts where needed) issued before
// the first use.
template <class O, class E, class W>
__device__ __forceinline__ W afterburn_edges(const RefArgs<O, E, W>& a, O i, W igain, part_t p, part_t best, E j0, E e, E stride) {
    W ch = 0;
    for (; j0 < e; j0 += 4 * stride) {
        O v[4];
        W w[4], vg[4];
        part_t vd[4], vp[4];
        bool take[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const E j = j0 + (E)u * stride;
            v[u] = j < e ? a.g.adj[j] : (O)-1;
            w[u] = j < e ? a.g.val[j] : (W)0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) vg[u] = v[u] >= 0 ? a.pregain[v[u]] : (W)0;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            take[u] = v[u] >= 0 && (vg[u] > igain || (vg[u] == igain && v[u] < i));
            vd[u] = take[u] ? a.dest[v[u]] : NULL_PART;
            vp[u] = take[u] ? a.part[v[u]] : NULL_PART;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (!take[u]) continue;
            if (vd[u] == p) ch -= w[u]; else if (vd[u] == best) ch += w[u];
            if (vp[u] == p) ch += w[u]; else if (vp[u] == best) ch -= w[u];
        }
    }
    return ch;
}

template <int G, class O, class E, class W>
__device__ __forceinline__ void d_afterburn(RefArgs<O, E, W> a) {
    O count = a.dev->ncand;
#define AB_BODY(x, in, lane)                                                                \
    {                                                                                       \
        O i = 0; E s = 0, e = 0; W igain = 0; part_t p = 0, best = 0; bool act = false;     \
        if (in) {                                                                           \
            i = a.cand[x]; s = a.g.row[i]; e = a.g.row[i + 1];                              \
            act = e - s <= HUB_DEG;                                                         \
            igain = a.pregain[i]; p = a.part[i]; best = a.dest[i];                          \
        }                                                                                   \
        W ch = 0;                                                                           \
        if (act) ch = afterburn_edges<O, E, W>(a, i, igain, p, best, s + lane, e, (E)G);   \
        ch = group_sum<W>(ch, G);                                                           \
        bool keep = act && lane == 0 && igain + ch >= 0;                                    \
        if (keep) a.lock[i] = 1;                                                            \
        O sl = warp_append(&a.dev->nmoves, keep);                                           \
        if (keep) a.moves[sl] = i;                                                          \
        if (in && lane == 0 && !act) { O hs = atomic_add(&a.dev->ncand_hub, (O)1); a.cand_hub[hs] = i; } \
    }
    JET_GROUP_LOOP(G, count, AB_BODY)
#undef AB_BODY
}
template <int G, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_afterburn(RefArgs<O, E, W> a) { d_afterburn<G, O, E, W>(a); }

template <class O, class E, class W>
__device__ __forceinline__ void d_afterburn_hub(RefArgs<O, E, W> a) {
    __shared__ W part_sum[32];
    O count = a.dev->ncand_hub;
    for (O x = blockIdx.x; x < count; x += gridDim.x) {
        O i = a.cand_hub[x];
        W igain = a.pregain[i];
        part_t p = a.part[i], best = a.dest[i];
        W ch = 0;
        ch = afterburn_edges<O, E, W>(a, i, igain, p, best, a.g.row[i] + threadIdx.x, a.g.row[i + 1], (E)blockDim.x);
        ch = group_sum<W>(ch, 32);
        if ((threadIdx.x & 31) == 0) part_sum[threadIdx.x >> 5] = ch;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); w++) ch += part_sum[w];
            if (igain + ch >= 0) {
                a.lock[i] = 1;
                O s = atomic_add(&a.dev->nmoves, (O)1);
                a.moves[s] = i;
            }
        }
        __syncthreads();
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_afterburn_hub(RefArgs<O, E, W> a) { d_afterburn_hub<O, E, W>(a); }

// ---------------------------------------------------------------- gain buckets
// src/jet_refiner.hpp:326-356 with C++ semantics kept: the float gain is
// scaled by the double literal 1.5 in double and rounded back to float.
template <class W>
__host__ __device__ __forceinline__ int gain_bucket(W gx, W vwgt) {
    float gain = (float)gx / (float)vwgt;
    int t;
    if (gain > 0.0) t = 0;
    else if (gain == 0.0) t = 1;
    else {
        t = MID_BUCKET;
        gain = fabsf(gain);
        if (gain < 1.0) {
            while (gain < 1.0) { gain = (float)((double)gain * 1.5); t--; }
            if (t < 2) t = 2;
        } else {
            while (gain > 1.0) { gain = (float)((double)gain / 1.5); t++; }
            if (t > MAX_BUCKETS) t = MAX_BUCKETS - 1;
        }
    }
    return t;
}

// ---------------------------------------------------------------- rebalance
template <class O, class W>
struct RebArgs {
    W size_max;
    W opt;
    W max_dest;
    O sections;
    O t_minibuckets;
    O width;          // MAX_BUCKETS * sections
    W* buckets;       // raw bucket totals, t_minibuckets + 1 + width entries
    W* boff;          // exclusive offsets of buckets[0 .. t_minibuckets]
    O* bid;
    W* score;         // in-bucket score (weight of the bucket's earlier vertices)
    part_t* undersized;
    W* evict_adjust;  // k
    W* evict_start;   // k + 1
    const uint32_t* skey;  // candidates sorted by bucket id (stable in vertex id)
    const O* sval;
    const W* wpre;         // exclusive prefix of vertex weights in sorted order
    uint32_t none_key;     // key of non-candidates (sorted last)
    O* redraw;             // strong rebalance: vertices needing a re-drawn position
    part_t* redraw_p;      // and the chunk they stopped at
    O* ordl;               // candidates whose in-bucket order decides their eviction
    int queue;             // eviction from the queue allowed (else the full sort)
};

// B(x): the offset the reference reads for bucket x -- scanned for
// x <= t_minibuckets, the raw total past it (the scan does not reach there).
template <class O, class W>
__device__ __forceinline__ W bucket_pos(const RebArgs<O, W>& rb, O x) { return x <= rb.t_minibuckets ? rb.boff[x] : rb.buckets[x]; }

// Weight of the vertices that precede bucket b in bucket order.
template <class O, class W>
__device__ __forceinline__ W bucket_start(const RebArgs<O, W>& rb, O b) {
    if (b <= rb.t_minibuckets) return rb.boff[b];
    W s = rb.boff[rb.t_minibuckets] + rb.buckets[rb.t_minibuckets];
    for (O x = rb.t_minibuckets + 1; x < b; x++) s += rb.buckets[x];
    return s;
}

template <class O>
struct GetBidKey {
    const O* bid;
    uint32_t none;
    __device__ __forceinline__ uint32_t operator()(int64_t i) const { O b = bid[i]; return b < 0 ? none : (uint32_t)b; }
};
template <class O, class W>
struct GetSortedWeight {
    const uint32_t* key;
    const O* val;
    const W* vw;
    uint32_t none;
    __device__ __forceinline__ W operator()(int64_t q) const { return key[q] == none ? (W)0 : vw[val[q]]; }
};

// Undersized parts in index order (src/jet_refiner.hpp:584-598).
template <class O, class E, class W>
__device__ __forceinline__ void d_weak_prep(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    __shared__ int sw[32];
    int carry = 0;
    for (int base = 0; base < a.k; base += 1024) {
        int p = base + threadIdx.x;
        int f = (p < a.k && a.sizes[p] < rb.max_dest) ? 1 : 0;
        int tot;
        int ex = block_exclusive_scan<int>(f, sw, tot);
        if (f) rb.undersized[carry + ex] = p;
        carry += tot;
    }
    if (threadIdx.x == 0) a.dev->total_undersized = carry;
}
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_weak_prep(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_weak_prep<O, E, W>(a, rb); }

// Destination choice and bucket score (src/jet_refiner.hpp:599-645), one
// thread per vertex (tables of vertices with deg > 32 are scanned by a warp).
template <class O, class E, class W>
__device__ __forceinline__ void weak_score(const RefArgs<O, E, W>& a, const RebArgs<O, W>& rb, O i, part_t p, part_t best,
                                           W gain, W p_gain, bool eligible) {
    part_t dest = p;
    W sg = 0;
    if (eligible) {
        if (gain > 0) { dest = best; sg = gain - p_gain; }
        else {
            part_t tu = a.dev->total_undersized;
            if (tu > 0) { dest = rb.undersized[(int64_t)i % tu]; sg = -p_gain; }
        }
    }
    a.dest[i] = dest;
    if (dest != p) {
        int gt = gain_bucket<W>(sg, a.g.vw[i]);
        O gid = (MAX_BUCKETS * (O)p + gt) * rb.sections + (O)(i % rb.sections);
        rb.bid[i] = gid;
        atomic_add(&rb.buckets[gid], a.g.vw[i]);  // bucket total; in-bucket order comes from the sort
    } else {
        rb.bid[i] = -1;
    }
}

template <class O, class E, class W>
__device__ __forceinline__ void d_weak_select_thread(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < a.g.n; x += (int64_t)gridDim.x * blockDim.x) {
        O i = (O)x;
        if (a.g.row[i + 1] - a.g.row[i] > THREAD_DEG) continue;
        part_t p = a.part[i];
        W sp = a.sizes[p];
        bool elig = sp > rb.size_max && (double)a.g.vw[i] < 1.5 * (double)(sp - rb.opt);
        W gain = 0, p_gain = 0;
        part_t best = p;
        if (elig) {
            const Slot<W>* base = a.slots + a.coff[i];
            part_t sz = a.csize[i];
            scan_slots<W>(base, sz, [&](const Slot<W>& sl) {
                if (sl.p > NULL_PART && a.sizes[sl.p] < rb.max_dest) {
                    if (sl.v > gain || (sl.v == gain && sl.v > 0 && sl.p < best)) { best = sl.p; gain = sl.v; }
                }
                if (sl.p == p) p_gain = sl.v;
            });
        }
        weak_score<O, E, W>(a, rb, i, p, best, gain, p_gain, elig);
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_weak_select_thread(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_weak_select_thread<O, E, W>(a, rb); }

template <class O, class E, class W>
__device__ __forceinline__ void d_weak_select_warp(RefArgs<O, E, W> a, RebArgs<O, W> rb, const O* list, O count) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (int)(blockDim.x >> 5);
    for (int64_t x = blockIdx.x * (int64_t)(int)(blockDim.x >> 5) + (threadIdx.x >> 5); x < count; x += warps) {
        O i = list[x];
        part_t p = a.part[i];
        W sp = a.sizes[p];
        bool elig = sp > rb.size_max && (double)a.g.vw[i] < 1.5 * (double)(sp - rb.opt);
        W gain = 0, p_gain = 0;
        part_t best = p;
        if (elig) {
            const Slot<W>* base = a.slots + a.coff[i];
            part_t sz = a.csize[i];
            for (part_t s = lane; s < sz; s += 32) {
                Slot<W> sl = base[s];
                if (sl.p > NULL_PART && a.sizes[sl.p] < rb.max_dest) {
                    if (sl.v > gain || (sl.v == gain && sl.v > 0 && sl.p < best)) { best = sl.p; gain = sl.v; }
                }
                if (sl.p == p) p_gain = sl.v;
            }
            for (int m = 16; m > 0; m >>= 1) {
                W g2 = shfl_xor(gain, m, 32);
                part_t b2 = shfl_xor(best, m, 32);
                if (g2 > gain || (g2 == gain && g2 > 0 && b2 < best)) { gain = g2; best = b2; }
                W pg2 = shfl_xor(p_gain, m, 32);
                if (pg2 != 0) p_gain = pg2;
            }
        }
        if (lane == 0) weak_score<O, E, W>(a, rb, i, p, best, gain, p_gain, elig);
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_weak_select_warp(RefArgs<O, E, W> a, RebArgs<O, W> rb, const O* list, O count) { d_weak_select_warp<O, E, W>(a, rb, list, count); }

// max_vwgt: largest room left in a part below max_dest (src/jet_refiner.hpp:442-451).
template <class O, class E, class W>
__device__ __forceinline__ void d_strong_prep(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    __shared__ W sm[32];
    __shared__ int sany[32];
    W best = std::numeric_limits<W>::lowest();
    int any = 0;
    for (int p = threadIdx.x; p < a.k; p += blockDim.x) {
        W s = a.sizes[p];
        if (s < rb.max_dest) { W cap = rb.max_dest - s; if (!any || cap > best) best = cap; any = 1; }
    }
    for (int m = 16; m > 0; m >>= 1) {
        W b2 = shfl_xor(best, m, 32);
        int a2 = shfl_xor(any, m, 32);
        if (a2 && (!any || b2 > best)) best = b2;
        any |= a2;
    }
    if ((threadIdx.x & 31) == 0) { sm[threadIdx.x >> 5] = best; sany[threadIdx.x >> 5] = any; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++)
            if (sany[w] && (!any || sm[w] > best)) { best = sm[w]; any = 1; }
        a.dev->max_vwgt = any ? best : std::numeric_limits<W>::lowest();
        a.dev->total_undersized = any;
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_strong_prep(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_strong_prep<O, E, W>(a, rb); }

// Eviction score: average loss to adjacent non-full parts (unsigned
// division, src/jet_refiner.hpp:452-480).
template <class O, class E, class W>
__device__ __forceinline__ void strong_score(const RefArgs<O, E, W>& a, const RebArgs<O, W>& rb, O i, part_t p, uint64_t tg,
                                             uint64_t tk, W p_gain) {
    if (tk == 0) tk = 1;
    W gain = (W)((tg / tk) - (uint64_t)p_gain);
    W w = a.g.vw[i];
    W lim = a.sizes[p] - rb.size_max;
    int gt = gain_bucket<W>(gain, w < lim ? w : lim);
    if (gt < MAX_BUCKETS) {
        O gid = (MAX_BUCKETS * (O)p + gt) * rb.sections + (O)(i % rb.sections) + 1;
        rb.bid[i] = gid;
        atomic_add(&rb.buckets[gid], w);
    }
}

template <class O, class E, class W>
__device__ __forceinline__ bool strong_eligible(const RefArgs<O, E, W>& a, const RebArgs<O, W>& rb, O i, part_t p) {
    W sp = a.sizes[p];
    W w = a.g.vw[i];
    if (!a.dev->total_undersized) return false;  // no part below max_dest
    W mv = a.dev->max_vwgt;
    return sp > rb.size_max && w <= 2 * mv && w < 2 * (sp - rb.opt);
}

template <class O, class E, class W>
__device__ __forceinline__ void d_strong_score_thread(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < a.g.n; x += (int64_t)gridDim.x * blockDim.x) {
        O i = (O)x;
        if (a.g.row[i + 1] - a.g.row[i] > THREAD_DEG) continue;
        part_t p = a.part[i];
        rb.bid[i] = -1;
        if (!strong_eligible<O, E, W>(a, rb, i, p)) continue;
        uint64_t tk = 0, tg = 0;
        W p_gain = 0;
        const Slot<W>* base = a.slots + a.coff[i];
        part_t sz = a.csize[i];
        scan_slots<W>(base, sz, [&](const Slot<W>& sl) {
            if (sl.p == p) p_gain = sl.v;
            else if (sl.p > NULL_PART && a.sizes[sl.p] < rb.max_dest) { tg += (uint64_t)sl.v; tk += 1; }
        });
        strong_score<O, E, W>(a, rb, i, p, tg, tk, p_gain);
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_strong_score_thread(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_strong_score_thread<O, E, W>(a, rb); }

template <class O, class E, class W>
__device__ __forceinline__ void d_strong_score_warp(RefArgs<O, E, W> a, RebArgs<O, W> rb, const O* list, O count) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (int)(blockDim.x >> 5);
    for (int64_t x = blockIdx.x * (int64_t)(int)(blockDim.x >> 5) + (threadIdx.x >> 5); x < count; x += warps) {
        O i = list[x];
        part_t p = a.part[i];
        if (lane == 0) rb.bid[i] = -1;
        if (!strong_eligible<O, E, W>(a, rb, i, p)) continue;
        uint64_t tk = 0, tg = 0;
        W p_gain = 0;
        const Slot<W>* base = a.slots + a.coff[i];
        part_t sz = a.csize[i];
        for (part_t s = lane; s < sz; s += 32) {
            Slot<W> sl = base[s];
            if (sl.p == p) p_gain = sl.v;
            else if (sl.p > NULL_PART && a.sizes[sl.p] < rb.max_dest) { tg += (uint64_t)sl.v; tk += 1; }
        }
        tg = group_sum<uint64_t>(tg, 32);
        tk = group_sum<uint64_t>(tk, 32);
        p_gain = group_sum<W>(p_gain, 32);  // own part appears in at most one slot
        if (lane == 0) strong_score<O, E, W>(a, rb, i, p, tg, tk, p_gain);
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_strong_score_warp(RefArgs<O, E, W> a, RebArgs<O, W> rb, const O* list, O count) { d_strong_score_warp<O, E, W>(a, rb, list, count); }

// get_evictions (src/jet_refiner.hpp:392-409).  The reference's in-bucket
// score is an atomic fetch-add whose order, run in index order, is the
// weight of the bucket's earlier vertices; here it is read off the stable
// sort by bucket id: wpre[q] - (weight of all earlier buckets).
template <bool ADJUST, class O, class E, class W>
__device__ __forceinline__ void d_evict_sorted(RefArgs<O, E, W> a, RebArgs<O, W> rb);
template <bool ADJUST, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_evict_sorted(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_evict_sorted<ADJUST, O, E, W>(a, rb); }
template <bool ADJUST, class O, class E, class W>
__device__ __forceinline__ void d_evict_sorted(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t rounds = ceil_div<int64_t>((int64_t)a.g.n, stride);
    for (int64_t r = 0; r < rounds; r++) {
        int64_t q = start + r * stride;
        bool take = false;
        O i = 0;
        if (q < a.g.n && rb.skey[q] != rb.none_key) {
            O b = (O)rb.skey[q];
            i = rb.sval[q];
            part_t p = a.part[i];
            O begin = (O)p * rb.width;
            W within = rb.wpre[q] - bucket_start<O, W>(rb, b);
            if (ADJUST) rb.score[i] = within;
            W score = within + bucket_pos<O, W>(rb, b) - bucket_pos<O, W>(rb, begin);
            W limit = a.sizes[p] - rb.size_max;
            if (score < limit) {
                take = true;
                if (ADJUST && score + a.g.vw[i] >= limit) rb.evict_adjust[p] = score + a.g.vw[i];
            }
        }
        O s = warp_append(&a.dev->nmoves, take);
        if (take) a.moves[s] = i;
    }
}

// "cookie cutter" (src/jet_refiner.hpp:491-518): prefix positions of the
// evicted weight per part and of the free room per undersized part.
template <class O, class E, class W>
__device__ __forceinline__ void d_cookie(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    __shared__ W sw[32];
    W carry = 0;
    for (int base = 0; base < a.k; base += 1024) {
        int p = base + threadIdx.x;
        W add = 0;
        O begin = (O)p * rb.width;
        if (p < a.k) {
            add = rb.evict_adjust[p];
            if (add == 0) add = rb.boff[begin + rb.width] - rb.boff[begin];
        }
        W tot;
        W ex = block_exclusive_scan<W>(add, sw, tot);
        if (p < a.k) rb.evict_adjust[p] = rb.boff[begin] - (carry + ex);
        carry += tot;
    }
    if (threadIdx.x == 0) a.dev->vw_cursor = carry;
    W carry2 = 0;
    for (int base = 0; base < a.k; base += 1024) {
        int p = base + threadIdx.x;
        W add = 0;
        if (p < a.k && rb.max_dest > a.sizes[p]) add = rb.max_dest - a.sizes[p];
        W tot;
        W ex = block_exclusive_scan<W>(add, sw, tot);
        if (p < a.k) rb.evict_start[p + 1] = carry2 + ex + add;
        carry2 += tot;
    }
    if (threadIdx.x == 0) rb.evict_start[0] = 0;
}
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_cookie(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_cookie<O, E, W>(a, rb); }

// Adjust scores and pick destinations by chunk (src/jet_refiner.hpp:519-544).
// A vertex less than half inside its chunk draws a new position past the
// end; only those draws depend on order (they advance one shared cursor),
// so they are queued here and replayed in vertex order by k_strong_redraw.
template <class O, class E, class W>
__device__ __forceinline__ void d_strong_first(RefArgs<O, E, W> a, RebArgs<O, W> rb, int64_t start, int64_t stride) {
    O count = a.dev->nmoves;
    for (int64_t x = start; x < count; x += stride) {
        O v = a.moves[x];
        part_t pv = a.part[v];
        W sc = rb.score[v] + rb.boff[rb.bid[v]] - rb.evict_adjust[pv];
        W w = a.g.vw[v];
        // the chunk holding position sc: the last p with evict_start[p] <= sc
        // (evict_start is a prefix of non-negative capacities, so a binary
        // search finds what a scan from p = 0 would)
        int lo = 0, hi = a.k + 1;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (rb.evict_start[mid] <= sc) lo = mid + 1;
            else hi = mid;
        }
        int p = lo - 1;
        part_t dest = pv;
        if (p < 0) atomicOr(&a.dev->err, ERRF_SPIN);  // positions are never negative
        else if (p < a.k) {
            if (w / 2 <= rb.evict_start[p + 1] - sc) dest = p;
            else {
                O s = atomic_add(&a.dev->nredraw, (O)1);
                rb.redraw[s] = v;
                rb.redraw_p[v] = p;
            }
        }
        rb.score[v] = sc;
        a.dest[v] = dest;
    }
}
template <class O, class E, class W>
__device__ __forceinline__ void d_strong_first(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    d_strong_first<O, E, W>(a, rb, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}
template <class O, class E, class W>
__global__ void k_strong_first(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_strong_first<O, E, W>(a, rb); }

// One block: sorts the queued vertices by id and replays their draws in order.
static constexpr int REDRAW_CAP = 4096;
template <class K>
__device__ __forceinline__ void block_sort_keys(K* key, int P) {
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    bool up = (i & k) == 0;
                    K x = key[i], y = key[ixj];
                    if ((x > y) == up) { key[i] = y; key[ixj] = x; }
                }
            }
            __syncthreads();
        }
    }
}
// The chunk scan of the destination draw (src/jet_refiner.hpp:529-531):
// from p, step while es[p] <= sc, then step back one.  es is a prefix of
// non-negative capacities (non-decreasing), so the first index past p whose
// bound exceeds sc is found by a binary search; the result is the scan's.
template <class W>
__device__ __forceinline__ int chunk_scan(const W* es, int p, int k, W sc) {
    if (p > k || es[p] > sc) return p - 1;
    int lo = p + 1, hi = k + 1;  // es[lo - 1] <= sc; find the first q in [lo, k] with es[q] > sc, else k + 1
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (es[mid] <= sc) lo = mid + 1;
        else hi = mid;
    }
    return lo - 1;
}

// The replay is one thread's serial walk (each draw advances the shared
// cursor), so what it reads is staged first: the chunk bounds in shared
// memory (when k fits) and, given `stage` shared memory for it, each queued
// vertex's weight and chunk, with the chosen chunks written back there and
// stored by the whole block; without it each vertex's data is loaded one
// vertex ahead of its use.
static constexpr int REDRAW_ES_CAP = 513;
template <class O, class E, class W>
__device__ __forceinline__ void d_strong_redraw(RefArgs<O, E, W> a, RebArgs<O, W> rb, unsigned char* stage = nullptr,
                                                size_t stage_bytes = 0) {
    __shared__ O list[REDRAW_CAP];
    __shared__ W es_s[REDRAW_ES_CAP];
    O cnt = a.dev->nredraw;
    if (cnt == 0) return;
    const bool es_in = a.k + 1 <= REDRAW_ES_CAP;
    if (es_in)
        for (int p = threadIdx.x; p <= a.k; p += blockDim.x) es_s[p] = rb.evict_start[p];
    const W* es = es_in ? es_s : rb.evict_start;
    bool fits = cnt <= REDRAW_CAP;
    if (fits) {
        int P = 1;
        while (P < (int)cnt) P <<= 1;
        for (int i = threadIdx.x; i < P; i += blockDim.x) list[i] = i < (int)cnt ? rb.redraw[i] : std::numeric_limits<O>::max();
        __syncthreads();
        block_sort_keys<O>(list, P);
    } else {
        __syncthreads();
        if (threadIdx.x == 0) atomicOr(&a.dev->err, 16);  // more draws than the replay buffer: order falls back to queue order
    }
    if (fits && stage && (size_t)cnt * (sizeof(W) + sizeof(int)) <= stage_bytes) {
        W* sw = (W*)stage;
        int* sp = (int*)(stage + (size_t)cnt * sizeof(W));
        for (int x = threadIdx.x; x < (int)cnt; x += blockDim.x) {
            const O v = list[x];
            sw[x] = a.g.vw[v];
            sp[x] = rb.redraw_p[v];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            W cursor = a.dev->vw_cursor;
            for (int x = 0; x < (int)cnt; x++) {
                const W w = sw[x];
                int p = sp[x];
                int dest = -1;
                int guard = 0;
                while (p < a.k) {
                    W sc = cursor;
                    cursor += w;
                    p = chunk_scan<W>(es, p, a.k, sc);
                    if (p < a.k && w / 2 <= es[p + 1] - sc) { dest = p; break; }
                    if (++guard > 4 * a.k + 64) { atomicOr(&a.dev->err, ERRF_SPIN); break; }
                }
                sp[x] = dest;
            }
            a.dev->vw_cursor = cursor;
        }
        __syncthreads();
        for (int x = threadIdx.x; x < (int)cnt; x += blockDim.x) {
            const O v = list[x];
            a.dest[v] = sp[x] >= 0 ? (part_t)sp[x] : a.part[v];
        }
        return;
    }
    if (threadIdx.x != 0) return;
    W cursor = a.dev->vw_cursor;
    O v = fits ? list[0] : rb.redraw[0];
    W w = a.g.vw[v];
    int p = rb.redraw_p[v];
    part_t pv = a.part[v];
    for (O x = 0; x < cnt; x++) {
        O vn = v;
        W wn = w;
        int pn = p;
        part_t pvn = pv;
        if (x + 1 < cnt) {
            vn = fits ? list[x + 1] : rb.redraw[x + 1];
            wn = a.g.vw[vn];
            pn = rb.redraw_p[vn];
            pvn = a.part[vn];
        }
        part_t dest = pv;
        int guard = 0;
        while (p < a.k) {
            W sc = cursor;
            cursor += w;
            p = chunk_scan<W>(es, p, a.k, sc);
            if (p < a.k && w / 2 <= es[p + 1] - sc) { dest = p; break; }
            if (++guard > 4 * a.k + 64) { atomicOr(&a.dev->err, ERRF_SPIN); break; }
        }
        a.dest[v] = dest;
        v = vn;
        w = wn;
        p = pn;
        pv = pvn;
    }
    a.dev->vw_cursor = cursor;
}
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_strong_redraw(RefArgs<O, E, W> a, RebArgs<O, W> rb) { d_strong_redraw<O, E, W>(a, rb); }

// ---------------------------------------------------------------- eviction from a short queue
// A candidate's eviction score (get_evictions, src/jet_refiner.hpp:392-409)
// is the offset of its bucket inside its part's bucket range plus "within",
// the weight of the bucket's candidates before it in vertex order; it leaves
// while the score is below its part's excess.  Weights are non-negative, so
// within lies in [0, bucket total - own weight]: a bucket whose offset
// reaches the excess keeps every candidate, and (weak) a bucket that ends
// below the excess loses every one, whatever their order.  Only the
// candidates of the buckets in between -- weak: the bucket that straddles the
// excess, one per part; strong: also every bucket that leaves, since the
// destination draw reads each evicted vertex's score -- need their place in
// the bucket.  d_reb_classify decides the rest and queues those on rb.ordl;
// d_reb_ordered orders the queue in one block.  The moves, scores and
// adjustments are those of the full sort (sort_candidates + d_evict_sorted),
// which stays as the fallback for what this cannot take: a weak bucket id
// past its part's range (gain bucket 50 shares the next part's first bucket,
// so one bucket would hold two parts' candidates), a negative vertex weight,
// or a queue longer than the block holds.
template <bool STRONG, class O, class E, class W>
__device__ __forceinline__ void d_reb_classify(RefArgs<O, E, W> a, RebArgs<O, W> rb, int64_t start, int64_t stride) {
    const int64_t n = a.g.n;
    const int64_t rounds = ceil_div<int64_t>(n, stride);
    for (int64_t r = 0; r < rounds; r++) {  // the same count in every lane: warp_append needs the whole warp
        const int64_t q = start + r * stride;
        bool take = false, order = false;
        O b = -1;
        if (q < n) b = rb.bid[q];
        if (b >= 0) {
            const O i = (O)q;
            const part_t p = a.part[i];
            const O begin = (O)p * rb.width;
            const W w = a.g.vw[i];
            if ((!STRONG && b >= begin + rb.width) || w < 0) {
                atomicOr(&a.dev->reb_fb, 1);
            } else {
                const W base = rb.boff[b] - rb.boff[begin];
                const W limit = a.sizes[p] - rb.size_max;
                if (base < limit) {
                    if (!STRONG && base + rb.buckets[b] < limit) take = true;
                    else order = true;
                }
            }
        }
        O s = warp_append(&a.dev->nmoves, take);
        if (take) a.moves[s] = (O)q;
        O t = warp_append(&a.dev->nord, order);
        if (order) rb.ordl[t] = (O)q;
    }
}

// Inclusive sum of v over runs that begin where head is set, across the
// block (every thread calls it, one value each).  carry is the sum of the
// run left open by the previous call and is updated for the next call.
template <class T>
__device__ __forceinline__ T block_seg_scan(T v, bool head, T& carry) {
    __shared__ T sv[32];
    __shared__ int sf[32];
    __shared__ T s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T x = v;
    int f = head ? 1 : 0;
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        int g = __shfl_up_sync(0xffffffffu, f, o);
        if (lane >= o) {
            if (!f) x += y;
            f |= g;
        }
    }
    if (lane == 31) { sv[wid] = x; sf[wid] = f; }
    __syncthreads();
    if (wid == 0) {
        T y = lane < nw ? sv[lane] : T(0);
        int g = lane < nw ? sf[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            T y2 = __shfl_up_sync(0xffffffffu, y, o);
            int g2 = __shfl_up_sync(0xffffffffu, g, o);
            if (lane >= o) {
                if (!g) y += y2;
                g |= g2;
            }
        }
        if (lane < nw) { sv[lane] = y; sf[lane] = g; }
    }
    __syncthreads();
    if (!f && wid > 0) { x += sv[wid - 1]; f = sf[wid - 1]; }
    if (!f) x += carry;
    if (threadIdx.x == blockDim.x - 1) s_last = x;
    __syncthreads();
    carry = s_last;
    return x;
}

// One block: the queued candidates sorted by (bucket, vertex) in shared
// memory (keys: at least count entries rounded up to a power of two), the
// weight prefix inside each bucket, and the eviction test of
// d_evict_sorted for them (strong: with the scores and part adjustments).
template <bool STRONG, class O, class E, class W>
__device__ __forceinline__ void d_reb_ordered(RefArgs<O, E, W> a, RebArgs<O, W> rb, O count, uint64_t* keys) {
    int P = 1;
    while (P < (int)count) P <<= 1;
    for (int q = threadIdx.x; q < P; q += blockDim.x) {
        uint64_t key = ~0ull;
        if (q < (int)count) {
            const O i = rb.ordl[q];
            key = ((uint64_t)(uint32_t)rb.bid[i] << 32) | (uint32_t)i;
        }
        keys[q] = key;
    }
    if (STRONG)
        for (int p = threadIdx.x; p < a.k; p += blockDim.x) rb.evict_adjust[p] = 0;
    __syncthreads();
    block_sort_keys<uint64_t>(keys, P);
    W carry = 0;
    for (int base = 0; base < (int)count; base += blockDim.x) {
        const int q = base + threadIdx.x;
        const bool in = q < (int)count;
        const uint64_t key = in ? keys[q] : 0ull;
        const uint32_t b32 = (uint32_t)(key >> 32);
        const bool head = in && (q == 0 || (uint32_t)(keys[q - 1] >> 32) != b32);
        const O i = (O)(uint32_t)key;
        const W w = in ? a.g.vw[i] : W(0);
        const W incl = block_seg_scan<W>(w, head, carry);
        bool take = false;
        if (in) {
            const O b = (O)b32;
            const part_t p = a.part[i];
            const O begin = (O)p * rb.width;
            const W within = incl - w;
            if (STRONG) rb.score[i] = within;
            const W score = within + rb.boff[b] - rb.boff[begin];
            const W limit = a.sizes[p] - rb.size_max;
            if (score < limit) {
                take = true;
                if (STRONG && score + w >= limit) rb.evict_adjust[p] = score + w;
            }
        }
        O s = warp_append(&a.dev->nmoves, take);
        if (take) a.moves[s] = i;
    }
    __syncthreads();
}

// The ordered eviction and, for strong rebalancing, the cookie cutter and the
// destination draws, all in one block.  keys: key_cap 64-bit entries of
// shared memory (at least count), reused by the draws once the order is done.
template <bool STRONG, class O, class E, class W>
__device__ __forceinline__ void d_reb_queue_tail(RefArgs<O, E, W> a, RebArgs<O, W> rb, O count, uint64_t* keys, int key_cap,
                                                 PhaseClock* pc) {
    d_reb_ordered<STRONG, O, E, W>(a, rb, count, keys);
    if (pc) pc->mark(PH_REB_EVICT);
    if (STRONG) {
        d_cookie<O, E, W>(a, rb);
        __syncthreads();
        if (pc) pc->mark(PH_COOKIE);
        d_strong_first<O, E, W>(a, rb, threadIdx.x, blockDim.x);
        __syncthreads();
        if (pc) pc->mark(PH_STRONG_FIRST);
        d_strong_redraw<O, E, W>(a, rb, (unsigned char*)keys, (size_t)key_cap * sizeof(uint64_t));
        __syncthreads();
        if (pc) pc->mark(PH_REDRAW);
    }
}

template <bool STRONG, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_reb_classify(RefArgs<O, E, W> a, RebArgs<O, W> rb) {
    d_reb_classify<STRONG, O, E, W>(a, rb, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// One block of 1024 threads after k_reb_classify.  When the queue fits `cap`
// keys of dynamic shared memory and nothing asked for the fallback, it
// finishes the rebalance; otherwise it drops the moves the classification
// queued and raises reb_fb_taken (and, inside a graph, the conditional
// handle of the fallback's IF node).  Either way it resets the queue.
template <bool STRONG, class O, class E, class W>
__global__ void __launch_bounds__(1024) k_reb_ordered(RefArgs<O, E, W> a, RebArgs<O, W> rb, int cap, cudaGraphConditionalHandle h,
                                                      int in_graph) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ O s_count;
    __shared__ int s_fb;
    if (threadIdx.x == 0) {
        const O count = a.dev->nord;
        const int fb = a.dev->reb_fb || count > (O)cap;
        s_count = count;
        s_fb = fb;
        a.dev->nord_last = count;
        a.dev->reb_fb_taken = fb;
        a.dev->nord = 0;
        a.dev->reb_fb = 0;
        if (fb) a.dev->nmoves = 0;
        if (in_graph) {
            cudaGraphSetConditional(h, fb ? 1u : 0u);
            a.dev->reb_fb_count[STRONG ? 1 : 0] += fb;
        }
    }
    __syncthreads();
    if (s_fb) return;
    d_reb_queue_tail<STRONG, O, E, W>(a, rb, s_count, (uint64_t*)smem_raw, cap, nullptr);
}

// ---------------------------------------------------------------- moves
// perform_moves part 1 (src/jet_refiner.hpp:910-931): cut change from the old
// tables, apply the moves, part-size deltas through a shared histogram.
template <class O, class E, class W>
__device__ __forceinline__ void d_apply_moves(RefArgs<O, E, W> a, int hist) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    W* hs = (W*)smem_raw;
    if (hist) {
        for (int p = threadIdx.x; p < a.k; p += blockDim.x) hs[p] = 0;
        __syncthreads();
    }
    O count = a.dev->nmoves;
    W c1 = 0;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < count; x += stride) {
        O i = a.moves[x];
        part_t p = a.part[i], b = a.dest[i];
        const Slot<W>* base = a.slots + a.coff[i];
        part_t sz = a.csize[i];
        c1 += table_lookup<W>(base, b, sz, a.k) - table_lookup<W>(base, p, sz, a.k);
        a.dest_cache[i] = NULL_PART;
        W w = a.g.vw[i];
        if (hist) { atomic_add(&hs[p], -w); atomic_add(&hs[b], w); }
        else { atomic_add(&a.sizes[p], -w); atomic_add(&a.sizes[b], w); }
        a.part[i] = b;
        a.dest[i] = p;
        if (a.g.row[i + 1] - a.g.row[i] > HUB_DEG) { O s = atomic_add(&a.dev->nmoves_hub, (O)1); a.moves_hub[s] = i; }
    }
    c1 = group_sum<W>(c1, 32);
    if ((threadIdx.x & 31) == 0 && c1) atomic_add(&a.dev->cut1, c1);
    if (hist) {
        __syncthreads();
        for (int p = threadIdx.x; p < a.k; p += blockDim.x) if (hs[p]) atomic_add(&a.sizes[p], hs[p]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.dev->large = count > (O)(a.g.n / 10);
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_apply_moves(RefArgs<O, E, W> a, int hist) { d_apply_moves<O, E, W>(a, hist); }

// update_small subtract (src/jet_refiner.hpp:786-808).
template <class O, class E, class W>
__device__ __forceinline__ void conn_sub(const RefArgs<O, E, W>& a, O v, part_t p, W w) {
    Slot<W>* base = a.slots + a.coff[v];
    part_t vsize = a.csize[v];
    part_t po = slot_home(p, vsize, a.k);
    part_t guard = 0;
    while (ld_cg(&base[po].p) != p) {
        po = po + 1 == vsize ? 0 : po + 1;
        if (++guard > vsize) { atomicOr(&a.dev->err, ERRF_PROBE); return; }
    }
    W x = atomic_add(&base[po].v, -w);
    if (vsize < a.k && x == w) st_v(&base[po].p, HASH_RECLAIM);
}

// update_small add (src/jet_refiner.hpp:811-887).
template <class O, class E, class W>
__device__ __forceinline__ void conn_add(const RefArgs<O, E, W>& a, O v, part_t best, W w) {
    a.dest_cache[v] = NULL_PART;
    E vs = a.coff[v];
    Slot<W>* base = a.slots + vs;
    part_t vsize = ld_cg(&a.csize[v]);
    const part_t home = slot_home(best, vsize, a.k);
    part_t po = home;
    bool success = false;
    for (part_t q = 0, pi = home; q < vsize; q++) {
        part_t e = ld_cg(&base[pi].p);
        if (e == best) { success = true; po = pi; break; }
        else if (e == NULL_PART) break;
        pi = pi + 1 == vsize ? 0 : pi + 1;
    }
    part_t count = 0;
    while (!success && count < vsize) {
        part_t px = ld_cg(&base[po].p);
        while (px != best && px > NULL_PART && count++ < vsize) {
            po = po + 1 == vsize ? 0 : po + 1;
            px = ld_cg(&base[po].p);
        }
        if (px == best) success = true;
        else if (px <= NULL_PART) {
            part_t old = atomicCAS((int*)&base[po].p, px, best);
            if (old == best || old <= NULL_PART) success = true;
            else { po = po + 1 == vsize ? 0 : po + 1; count++; }
        }
    }
    if (!success) {
        // no free slot: append past the table's end (capacity min(deg,k) always suffices)
        part_t cap = (part_t)(a.coff[v + 1] - vs);
        po = vsize;
        while (!success) {
            if (po >= cap) { atomicOr(&a.dev->err, ERRF_OVERFLOW); return; }
            part_t px = ld_cg(&base[po].p);
            while (px != best && px > NULL_PART) {
                if (++po >= cap) { atomicOr(&a.dev->err, ERRF_OVERFLOW); return; }
                px = ld_cg(&base[po].p);
            }
            if (px == best) success = true;
            else {
                part_t py = atomicCAS((int*)&base[po].p, px, best);
                if (py == px) { py = best; atomicAdd((int*)&a.csize[v], 1); }
                if (py == best) success = true;
                else po++;
            }
        }
    }
    atomic_add(&base[po].v, w);
}

template <int G, bool ADD, class O, class E, class W>
__device__ __forceinline__ void d_update_small(RefArgs<O, E, W> a) {
    if (a.dev->large) return;
    O count = a.dev->nmoves;
#define UPD_BODY(x, in, lane)                                                               \
    {                                                                                       \
        if (in) {                                                                           \
            O i = a.moves[x];                                                               \
            E s = a.g.row[i], e = a.g.row[i + 1];                                           \
            if (e - s <= HUB_DEG) {                                                         \
                part_t pp = ADD ? a.part[i] : a.dest[i];                                    \
                for (E j = s + lane; j < e; j += G) {                                       \
                    if (ADD) conn_add<O, E, W>(a, a.g.adj[j], pp, a.g.val[j]);              \
                    else conn_sub<O, E, W>(a, a.g.adj[j], pp, a.g.val[j]);                  \
                }                                                                           \
            }                                                                               \
        }                                                                                   \
    }
    JET_GROUP_LOOP(G, count, UPD_BODY)
#undef UPD_BODY
}
template <int G, bool ADD, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_update_small(RefArgs<O, E, W> a) { d_update_small<G, ADD, O, E, W>(a); }

template <bool ADD, class O, class E, class W>
__device__ __forceinline__ void d_update_small_hub(RefArgs<O, E, W> a) {
    if (a.dev->large) return;
    O count = a.dev->nmoves_hub;
    for (O x = blockIdx.x; x < count; x += gridDim.x) {
        O i = a.moves_hub[x];
        part_t pp = ADD ? a.part[i] : a.dest[i];
        for (E j = a.g.row[i] + threadIdx.x; j < a.g.row[i + 1]; j += blockDim.x) {
            if (ADD) conn_add<O, E, W>(a, a.g.adj[j], pp, a.g.val[j]);
            else conn_sub<O, E, W>(a, a.g.adj[j], pp, a.g.val[j]);
        }
    }
}
template <bool ADD, class O, class E, class W>
__global__ void __launch_bounds__(1024) k_update_small_hub(RefArgs<O, E, W> a) { d_update_small_hub<ADD, O, E, W>(a); }

// update_large (src/jet_refiner.hpp:743-777): mark every neighbour of a
// moved vertex; the marked rows are rebuilt by the table builders.
template <int G, class O, class E, class W>
__device__ __forceinline__ void d_mark_neighbors(RefArgs<O, E, W> a) {
    if (!a.dev->large) return;
    O count = a.dev->nmoves;
#define MARK_BODY(x, in, lane)                                                              \
    {                                                                                       \
        if (in) {                                                                           \
            O i = a.moves[x];                                                               \
            E rs = a.g.row[i], re = a.g.row[i + 1];                                         \
            if (re - rs <= HUB_DEG)  /* hubs: one CTA each (d_mark_neighbors_hub) */         \
                for (E j0 = rs + lane; j0 < re; j0 += 4 * G) {                              \
                    /* four neighbours per lane, every load issued before the first use */  \
                    O v[4];                                                                 \
                    uint8_t mk[4];                                                          \
                    _Pragma("unroll") for (int u = 0; u < 4; u++)                           \
                        v[u] = j0 + (E)u * G < re ? a.g.adj[j0 + (E)u * G] : (O)-1;         \
                    _Pragma("unroll") for (int u = 0; u < 4; u++)                           \
                        mk[u] = v[u] >= 0 ? a.mark[v[u]] : (uint8_t)1;                      \
                    /* read first: few lines get dirtied */                                 \
                    _Pragma("unroll") for (int u = 0; u < 4; u++)                           \
                        if (!mk[u]) a.mark[v[u]] = 1;                                       \
                }                                                                           \
        }                                                                                   \
    }
    JET_GROUP_LOOP(G, count, MARK_BODY)
#undef MARK_BODY
}
template <int G, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_mark_neighbors(RefArgs<O, E, W> a) { d_mark_neighbors<G, O, E, W>(a); }

template <class O, class E, class W>
__device__ __forceinline__ void d_mark_neighbors_hub(RefArgs<O, E, W> a) {
    if (!a.dev->large) return;
    O count = a.dev->nmoves_hub;
    for (O x = blockIdx.x; x < count; x += gridDim.x) {
        O i = a.moves_hub[x];
        const E re = a.g.row[i + 1];
        for (E j0 = a.g.row[i] + threadIdx.x; j0 < re; j0 += 4 * (E)blockDim.x) {
            O v[4];
            uint8_t mk[4];
#pragma unroll
            for (int u = 0; u < 4; u++) v[u] = j0 + (E)u * blockDim.x < re ? a.g.adj[j0 + (E)u * blockDim.x] : (O)-1;
#pragma unroll
            for (int u = 0; u < 4; u++) mk[u] = v[u] >= 0 ? a.mark[v[u]] : (uint8_t)1;
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (!mk[u]) a.mark[v[u]] = 1;
        }
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_mark_neighbors_hub(RefArgs<O, E, W> a) { d_mark_neighbors_hub<O, E, W>(a); }

// perform_moves part 2 (src/jet_refiner.hpp:937-946): cut change from the
// updated tables.
template <class O, class E, class W>
__device__ __forceinline__ void d_cut_after(RefArgs<O, E, W> a) {
    O count = a.dev->nmoves;
    W c2 = 0;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < count; x += (int64_t)gridDim.x * blockDim.x) {
        O i = a.moves[x];
        const Slot<W>* base = a.slots + a.coff[i];
        part_t sz = a.csize[i];
        c2 += table_lookup<W>(base, a.part[i], sz, a.k) - table_lookup<W>(base, a.dest[i], sz, a.k);
    }
    c2 = group_sum<W>(c2, 32);
    if ((threadIdx.x & 31) == 0 && c2) atomic_add(&a.dev->cut2, c2);
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_cut_after(RefArgs<O, E, W> a) { d_cut_after<O, E, W>(a); }

// Largest part, results to the host mirror, counters reset.
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_finalize(RefArgs<O, E, W> a, IterResult* out) {
    __shared__ W sm[32];
    W mx = std::numeric_limits<W>::lowest();
    for (int p = threadIdx.x; p < a.k; p += blockDim.x) { W s = a.sizes[p]; if (s > mx) mx = s; }
    for (int m = 16; m > 0; m >>= 1) { W y = shfl_xor(mx, m, 32); if (y > mx) mx = y; }
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) if (sm[w] > mx) mx = sm[w];
        RefDev<O, W>* d = a.dev;
        out->nmoves = (int64_t)d->nmoves;
        out->cut_change = (int64_t)(d->cut1 + d->cut2);
        out->max_part = (int64_t)mx;
        out->err = d->err;
        out->large = d->large;
        d->ncand = 0; d->nmoves = 0; d->ncand_hub = 0; d->nmoves_hub = 0; d->nredraw = 0;
        d->cut1 = 0; d->cut2 = 0; d->large = 0;
    }
}

// ---------------------------------------------------------------- device-side control
// The iteration control of jet_refine (src/jet_refiner.hpp:1094-1134) run on
// the device, so a whole level refines inside one CUDA graph: a WHILE node
// repeats the iteration, IF nodes select LP / weak / strong and the copy of
// an improved state.  State lives in Ctl; handles are set with
// cudaGraphSetConditional.
enum { MODE_LP = 0, MODE_WEAK = 1, MODE_STRONG = 2 };
static constexpr int MAX_TEMPS = 24;

template <class W>
struct Ctl {
    W curr_cut, curr_imb, best_cut, best_imb;
    W opt, imb_max;
    double tol;
    double filter;
    double temps[MAX_TEMPS];
    int n_temps, temp_idx;
    int count, balance_counter, lab_counter, iter_count;
    int weak_iters, strong_iters;
    int mode, copy, more;
};

struct CtlHandles {
    cudaGraphConditionalHandle loop, lp, weak, strong, copy;
};

// Mode of the next iteration, decided the way the loop body starts
// (src/jet_refiner.hpp:1106-1117).
template <class W>
__device__ __forceinline__ void ctl_next_mode(Ctl<W>* c) {
    c->iter_count++;
    if (c->curr_imb <= c->imb_max) {
        c->mode = MODE_LP;
        c->balance_counter = 0;
        c->lab_counter++;
    } else {
        c->mode = c->balance_counter < 2 ? MODE_WEAK : MODE_STRONG;
        if (c->mode == MODE_WEAK) c->weak_iters++; else c->strong_iters++;
        c->balance_counter++;
    }
}

template <class W>
__device__ __forceinline__ void ctl_set_handles(const Ctl<W>* c, const CtlHandles& h, bool in_graph) {
    if (!in_graph) return;
    cudaGraphSetConditional(h.lp, c->more && c->mode == MODE_LP);
    cudaGraphSetConditional(h.weak, c->more && c->mode == MODE_WEAK);
    cudaGraphSetConditional(h.strong, c->more && c->mode == MODE_STRONG);
    cudaGraphSetConditional(h.copy, c->copy);
    cudaGraphSetConditional(h.loop, c->more);
}

// Before the first iteration: the first `count++ <= 11` check passes.
template <class W>
__device__ __forceinline__ void ctl_begin_logic(Ctl<W>* c) {
    c->count = 1;
    c->temp_idx = 0;
    c->filter = c->temps[0];
    c->more = 1;
    c->copy = 0;
    ctl_next_mode(c);
}
template <class W>
__global__ void k_ctl_begin(Ctl<W>* c, CtlHandles h) {
    ctl_begin_logic(c);
    ctl_set_handles(c, h, true);
}

// After an iteration: applies the cut change and largest part, keeps the best
// state (src/jet_refiner.hpp:1120-1132), evaluates the loop condition and the
// next mode, and resets the per-iteration counters.
template <class O, class W>
__device__ __forceinline__ void ctl_end_logic(Ctl<W>* c, RefDev<O, W>* d, W mx) {
    // the cut changes were summed by other blocks' atomics: read past L1
    c->curr_cut -= ld_cg(&d->cut1) + ld_cg(&d->cut2);
    c->curr_imb = mx > c->opt ? mx - c->opt : 0;
    c->copy = 0;
    if (c->best_imb > c->imb_max && c->curr_imb < c->best_imb) {
        c->best_cut = c->curr_cut;
        c->best_imb = c->curr_imb;
        c->copy = 1;
        c->count = 0;
    } else if (c->curr_cut < c->best_cut && (c->curr_imb <= c->imb_max || c->curr_imb <= c->best_imb)) {
        if ((double)c->curr_cut < c->tol * (double)c->best_cut) c->count = 0;
        c->best_cut = c->curr_cut;
        c->best_imb = c->curr_imb;
        c->copy = 1;
    }
    int more = 1;
    if (!(c->count++ <= 11)) {
        c->temp_idx++;
        if (c->temp_idx < c->n_temps) {
            c->filter = c->temps[c->temp_idx];
            c->count = 1;
        } else {
            more = 0;
        }
    }
    c->more = more;
    if (more) ctl_next_mode(c);
    d->ncand = 0; d->nmoves = 0; d->ncand_hub = 0; d->nmoves_hub = 0; d->nredraw = 0;
    d->cut1 = 0; d->cut2 = 0; d->large = 0;
}

// Largest part size, reduced over the block (result valid in thread 0).
template <class W>
__device__ __forceinline__ W block_max_sizes(const W* sizes, int k) {
    __shared__ W sm[32];
    W mx = std::numeric_limits<W>::lowest();
    for (int p = threadIdx.x; p < k; p += blockDim.x) { W s = sizes[p]; if (s > mx) mx = s; }
    for (int m = 16; m > 0; m >>= 1) { W y = shfl_xor(mx, m, 32); if (y > mx) mx = y; }
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) if (sm[w] > mx) mx = sm[w];
    __syncthreads();
    return mx;
}

// Closes an iteration inside the level graph and sets the graph's handles.
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_finalize_ctl(RefArgs<O, E, W> a, Ctl<W>* c, CtlHandles h) {
    W mx = block_max_sizes<W>(a.sizes, a.k);
    if (threadIdx.x != 0) return;
    ctl_end_logic<O, W>(c, a.dev, mx);
    ctl_set_handles(c, h, true);
}

// k_cut_after and k_finalize_ctl in one launch (one graph node less per
// iteration): every block adds its cut change, and the last block to finish
// (a counter, reset by that block) closes the iteration.
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_cut_finalize_ctl(RefArgs<O, E, W> a, Ctl<W>* c, CtlHandles h, unsigned* done) {
    __shared__ int s_last;
    d_cut_after<O, E, W>(a);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    W mx = block_max_sizes<W>(a.sizes, a.k);
    if (threadIdx.x != 0) return;
    *done = 0;
    ctl_end_logic<O, W>(c, a.dev, mx);
    ctl_set_handles(c, h, true);
}


// ---------------------------------------------------------------- statistics
// Cut counted from both endpoints (src/part_stat.hpp:77-108).
template <int G, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_total_cut(GView<O, E, W> g, const part_t* part, W* out) {
    W acc = 0;
#define CUT_BODY(x, in, lane)                                                               \
    {                                                                                       \
        if (in) {                                                                           \
            O i = (O)x; part_t pi = part[i];                                                \
            for (E j = g.row[i] + lane; j < g.row[i + 1]; j += G) if (part[g.adj[j]] != pi) acc += g.val[j]; \
        }                                                                                   \
    }
    JET_GROUP_LOOP(G, g.n, CUT_BODY)
#undef CUT_BODY
    acc = group_sum<W>(acc, 32);
    if ((threadIdx.x & 31) == 0 && acc) atomic_add(out, acc);
}

template <class O, class W>
__global__ void __launch_bounds__(BLOCK) k_part_sizes(O n, const W* vw, const part_t* part, part_t k, W* sizes, int hist) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    W* hs = (W*)smem_raw;
    if (hist) { for (int p = threadIdx.x; p < k; p += blockDim.x) hs[p] = 0; __syncthreads(); }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (hist) atomic_add(&hs[part[i]], vw[i]);
        else atomic_add(&sizes[part[i]], vw[i]);
    }
    if (hist) {
        __syncthreads();
        for (int p = threadIdx.x; p < k; p += blockDim.x) if (hs[p]) atomic_add(&sizes[p], hs[p]);
    }
}

// Projection to the finer level (src/uncoarsen.hpp:82-86).
template <class O>
__global__ void k_project(O n_fine, const O* map, const part_t* coarse, part_t* fine) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_fine; i += (int64_t)gridDim.x * blockDim.x)
        fine[i] = coarse[map[i]];
}

// Part ids out of range are rejected before refinement starts.
static __global__ void k_check_parts(int64_t n, const part_t* part, part_t k, int* err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (part[i] < 0 || part[i] >= k) atomicOr(err, 8);
}

}  // namespace jetb
