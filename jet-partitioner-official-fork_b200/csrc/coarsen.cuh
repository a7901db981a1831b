// coarsen.cuh -- coarsening maps: HEC (heavy-edge clustering), heavy/random
// matching with hash-phased commit rounds, and the 2-hop leaf / twin /
// relative passes.  Restates src/heuristics.hpp of the reference.
//
// Group kernels: G consecutive lanes cooperate on one vertex; loops are
// warp-uniform so shuffles always see all 32 lanes.  Vertices of degree above
// HUB_DEG are skipped by group kernels and handled by one CTA each.
#pragma once
#include "graph.cuh"
#include "sort.cuh"

namespace jetb {

template <class O> __host__ __device__ constexpr O ord_max() { return std::numeric_limits<O>::max(); }

// Iterates vertices in warp-uniform rounds; `body(i, valid, lane)` is invoked
// by every lane of every group.
#define JET_GROUP_LOOP(G, COUNT, BODY)                                                        \
    {                                                                                         \
        const int _lane = threadIdx.x & ((G) - 1);                                            \
        const int64_t _groups_per_grid = ((int64_t)gridDim.x * blockDim.x) / (G);             \
        const int64_t _gid0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / (G);         \
        const int64_t _rounds = ceil_div<int64_t>((int64_t)(COUNT), _groups_per_grid);        \
        for (int64_t _r = 0; _r < _rounds; _r++) {                                            \
            const int64_t _x = _gid0 + _r * _groups_per_grid;                                 \
            const bool _in = _x < (int64_t)(COUNT);                                           \
            BODY(_x, _in, _lane);                                                             \
        }                                                                                     \
    }

// ---------------------------------------------------------------- HEC
// Random heavy neighbour when all weights are equal, src/heuristics.hpp:197-210.
template <class O, class E, class W>
__global__ void k_hec_uniform(GView<O, E, W> g, uint64_t seed, uint64_t stream, O* hn) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t r = jet_rng(seed, stream, (uint64_t)i);
        E s = g.row[i], d = g.row[i + 1] - s;
        hn[i] = d > 0 ? g.adj[s + (E)(r % (uint64_t)d)] : (O)(r % (uint64_t)g.n);
    }
}

template <class W>
__global__ void k_sum(const W* a, int64_t n, W* out) {
    W s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += a[i];
    s = group_sum<W>(s, 32);
    if ((threadIdx.x & 31) == 0) atomic_add(out, s);
}

// Heaviest eligible edge (neighbour weight below 6x average); ties go to the
// later edge, as the reference's ">=" ValLoc scan does in index order
// (src/heuristics.hpp:211-249).
template <class O, class E, class W>
__device__ __forceinline__ void argmax_merge(W& bw, E& bj, W w2, E j2) {
    if (j2 >= 0 && (bj < 0 || w2 > bw || (w2 == bw && j2 > bj))) { bw = w2; bj = j2; }
}

// Heaviest eligible edge among j0, j0 + stride, ... < e (argmax_merge is a
// total order, so the edge order does not matter), four edges per round with
// the neighbour ids, weights and neighbour weights all loaded before the first use.
template <class O, class E, class W>
__device__ __forceinline__ void heavy_edges(const GView<O, E, W>& g, W max_allowed, E j0, E e, E stride, W& bw, E& bj) {
    for (; j0 < e; j0 += 4 * stride) {
        O v[4];
        W w[4], vw[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const E j = j0 + (E)u * stride;
            v[u] = j < e ? g.adj[j] : (O)-1;
            w[u] = j < e ? g.val[j] : (W)0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) vw[u] = v[u] >= 0 ? g.vw[v[u]] : max_allowed;
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (vw[u] < max_allowed) argmax_merge<O, E, W>(bw, bj, w[u], j0 + (E)u * stride);
    }
}

template <int G, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_hec_heavy(GView<O, E, W> g, const W* vsum, O* hn) {
    W max_allowed = (W)(6 * (*vsum)) / (W)g.n;
#define HEC_BODY(x, in, lane)                                                               \
    {                                                                                       \
        O i = (O)x;                                                                         \
        E s = 0, e = 0;                                                                     \
        bool act = false;                                                                   \
        if (in) { s = g.row[i]; e = g.row[i + 1]; act = (e - s) > 0 && (e - s) <= HUB_DEG && g.vw[i] < max_allowed; } \
        W bw = 0; E bj = -1;                                                                \
        if (act) heavy_edges<O, E, W>(g, max_allowed, s + lane, e, (E)G, bw, bj);          \
        for (int m = G >> 1; m > 0; m >>= 1) {                                              \
            W w2 = shfl_xor(bw, m, G); E j2 = shfl_xor(bj, m, G);                           \
            argmax_merge<O, E, W>(bw, bj, w2, j2);                                          \
        }                                                                                   \
        if (in && lane == 0 && (e - s) <= HUB_DEG) hn[i] = (act && bj >= 0) ? g.adj[bj] : i; \
    }
    JET_GROUP_LOOP(G, g.n, HEC_BODY)
#undef HEC_BODY
}

template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_hec_heavy_hub(GView<O, E, W> g, const W* vsum, const O* hubs, O nhub, O* hn) {
    __shared__ W sw[32];
    __shared__ E sj[32];
    W max_allowed = (W)(6 * (*vsum)) / (W)g.n;
    for (O h = blockIdx.x; h < nhub; h += gridDim.x) {
        O i = hubs[h];
        E s = g.row[i], e = g.row[i + 1];
        bool act = g.vw[i] < max_allowed;
        W bw = 0; E bj = -1;
        if (act)
            for (E j = s + threadIdx.x; j < e; j += blockDim.x) {
                O v = g.adj[j];
                if (g.vw[v] < max_allowed) argmax_merge<O, E, W>(bw, bj, g.val[j], j);
            }
        for (int m = 16; m > 0; m >>= 1) {
            W w2 = shfl_xor(bw, m, 32); E j2 = shfl_xor(bj, m, 32);
            argmax_merge<O, E, W>(bw, bj, w2, j2);
        }
        if ((threadIdx.x & 31) == 0) { sw[threadIdx.x >> 5] = bw; sj[threadIdx.x >> 5] = bj; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); w++) argmax_merge<O, E, W>(bw, bj, sw[w], sj[w]);
            hn[i] = (act && bj >= 0) ? g.adj[bj] : i;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- HEC, in-order semantics
// The reference's aggregation rounds (src/heuristics.hpp:101-126) executed in
// index order settle every vertex within two rounds, and both rounds have a
// data-parallel formulation that yields exactly the in-order result:
//
// Round 1 (swap = 1) processes A = {u : hn[u] <= u}.  Every u in A is still
// free at its turn (claims go to smaller indices), and it ends in the
// aggregate found by following hn through A: the chain stops at t with
// hn[t] == t (root t) or at h = hn[t] outside A (h is claimed as a partner and
// becomes the root).  Resolved by pointer jumping.
//
// Round 2 (swap = 0) processes the rest, B, all with hn[u] > u, in index order.
// u is claimed by its smallest free child (a free w in B with hn[w] == u) if
// one exists; otherwise u is free and pairs with hn[u] when it is its parent's
// smallest free child and the parent is in B, else joins the parent's
// aggregate.  "free" is a NOR over children, evaluated bottom-up in one pass in
// which the last child to finish continues with the parent.
template <class O>
__device__ __forceinline__ O hec_enc(O root) { return (O)(-2) - root; }  // terminal marker (< -1)

template <class O>
__global__ void k_hec_p1_init(O n, const O* hn, O* nxt, O* vcmap) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        O u = (O)x;
        O h = hn[u];
        if (h > u) { nxt[u] = (O)-1; continue; }  // not in A
        if (h == u) { nxt[u] = hec_enc<O>(u); continue; }
        if (hn[h] <= h) { nxt[u] = h; continue; }  // parent inside A
        nxt[u] = hec_enc<O>(h);
        vcmap[h] = h;  // h is claimed as a partner: root of its aggregate
    }
}

template <class O>
__global__ void k_hec_p1_jump(O n, O* nxt, int* changed) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        O p = ld_cg(&nxt[x]);
        if (p < 0) continue;
        O q = ld_cg(&nxt[p]);
        if (q != p) { st_v(&nxt[x], q); *changed = 1; }
    }
}

template <class O>
__global__ void k_hec_p1_final(O n, const O* nxt, O* vcmap) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        O e = nxt[x];
        if (e < -1) vcmap[x] = (O)(-2) - e;
    }
}

template <class O>
__global__ void k_hec_p2_count(O n, const O* hn, const O* vcmap, uint8_t* inB, O* cnt, O* min_free, int* has_free) {
    const O MAXV = ord_max<O>();
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        O u = (O)x;
        bool b = vcmap[u] == MAXV;
        inB[u] = b;
        min_free[u] = MAXV;
        has_free[u] = 0;
        if (b) {
            O v = hn[u];
            if (vcmap[v] == MAXV) atomic_add(&cnt[v], (O)1);
        }
    }
}

template <class O>
__device__ __forceinline__ void atomic_min_o(int32_t* p, int32_t v) { atomicMin((int*)p, v); }
template <class O>
__device__ __forceinline__ void atomic_min_o(int64_t* p, int64_t v) { atomicMin((long long*)p, (long long)v); }

// has_free[u]: bit 0 = u has a free child; bit 1 = u's walk step was claimed.
// A vertex is stepped through exactly once: either its own thread finds
// cnt == 0 or its last child continues into it, and both happen only after
// every child finished; the claim bit keeps the second arrival out.
template <class O>
__global__ void k_hec_p2_walk(O n, const O* hn, const uint8_t* inB, O* cnt, O* min_free, int* has_free) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        O cur = (O)x;
        if (!inB[cur] || ld_cg(&cnt[cur]) != 0) continue;  // children pending: the last one continues here
        while (true) {
            if (atomicOr(&has_free[cur], 2) & 2) break;  // already stepped through
            __threadfence();
            bool is_free = (ld_cg(&has_free[cur]) & 1) == 0;
            O v = hn[cur];
            if (!inB[v]) break;
            if (is_free) {
                atomic_min_o<O>(&min_free[v], cur);
                atomicOr(&has_free[v], 1);
            }
            __threadfence();
            if (atomic_add(&cnt[v], (O)-1) != 1) break;  // another child finishes v later
            __threadfence();
            cur = v;
        }
    }
}

template <class O>
__global__ void k_hec_p2_roots(O n, const O* hn, const uint8_t* inB, const O* min_free, const int* has_free, O* vcmap) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        O u = (O)x;
        if (!inB[u]) continue;
        O root;
        if (has_free[u] & 1) {
            root = min_free[u];
        } else {
            O v = hn[u];
            if (inB[v]) root = (min_free[v] == u) ? u : min_free[v];
            else root = vcmap[v];
        }
        vcmap[u] = root;
    }
}

// Roots (vcmap[u] == u) are numbered in index order; others take their
// root's number (src/heuristics.hpp:147-165, :655-665).
template <class O>
struct GetIsRoot {
    const O* vcmap;
    __device__ __forceinline__ O operator()(int64_t i) const { return vcmap[i] == (O)i ? (O)1 : (O)0; }
};
template <class O>
__global__ void k_assign_ids(O n, const O* ids, O* vcmap) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x)
        vcmap[u] = ids[vcmap[u]];
}
template <class O>
__global__ void k_singletons(O n, O* vcmap) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x)
        if (vcmap[u] == ord_max<O>()) vcmap[u] = (O)u;
}

// ---------------------------------------------------------------- matching
template <class O, class E, class W>
__global__ void k_match_uniform_init(GView<O, E, W> g, uint64_t seed, uint64_t stream, O* hn) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        E s = g.row[i], d = g.row[i + 1] - s;
        if (d == 0) continue;
        uint64_t r = jet_rng(seed, stream, (uint64_t)i);
        hn[i] = g.adj[s + (E)(r % (uint64_t)d)];
    }
}

// pickMatch (src/heuristics.hpp:321-425): among eligible neighbours, the
// lexicographic maximum of (edge weight, xorshift(v + r), edge index) --
// what the reference's in-order scan with ">=" tie-breaking selects.  For
// uniform weights the weight term is ignored.
struct PickKey {
    int64_t w;
    uint32_t h;
    int64_t j;
};
__device__ __forceinline__ bool pick_better(int64_t w2, uint32_t h2, int64_t j2, int64_t w, uint32_t h, int64_t j) {
    if (j2 < 0) return false;
    if (j < 0) return true;
    if (w2 != w) return w2 > w;
    if (h2 != h) return h2 > h;
    return j2 > j;
}

template <bool INITIAL, bool UNIFORM, class O, class E, class W>
__device__ __forceinline__ bool pick_skip(O u, const O* vcmap, const O* hn) {
    if (INITIAL) return false;
    const O MAXV = ord_max<O>();
    return vcmap[u] != MAXV || hn[u] == MAXV || vcmap[hn[u]] == MAXV;
}

// The best (weight, hash, edge) of a vertex's eligible edges j0, j0 + stride,
// ... < e (pick_better's total order, so the edge order does not matter),
// four edges per round with the neighbour ids, weights and match states all
// loaded before the first use.
template <bool INITIAL, bool UNIFORM, class O, class E, class W>
__device__ __forceinline__ void pick_edges(const GView<O, E, W>& g, const O* vcmap, uint32_t r, E j0, E e, E stride, int64_t& bw,
                                           uint32_t& bh, int64_t& bj) {
    const O MAXV = ord_max<O>();
    for (; j0 < e; j0 += 4 * stride) {
        O v[4];
        int64_t w[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const E j = j0 + (E)u * stride;
            v[u] = j < e ? g.adj[j] : (O)-1;
            w[u] = (!UNIFORM && j < e) ? (int64_t)g.val[j] : 0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) ok[u] = v[u] >= 0 && (INITIAL || vcmap[v[u]] == MAXV);
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (!ok[u]) continue;
            const uint32_t h = xorshift32((uint32_t)((uint64_t)v[u] + r));
            const int64_t j = (int64_t)(j0 + (E)u * stride);
            if (pick_better(w[u], h, j, bw, bh, bj)) { bw = w[u]; bh = h; bj = j; }
        }
    }
}

template <int G, bool INITIAL, bool UNIFORM, class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_pick_match(GView<O, E, W> g, const O* perm, const O* perm_len, const O* vcmap, O* hn,
                                                      uint64_t seed, uint64_t stream) {
    const O MAXV = ord_max<O>();
    O len = perm ? *perm_len : g.n;
#define PICK_BODY(x, in, lane)                                                              \
    {                                                                                       \
        O u = 0; E s = 0, e = 0; bool act = false; uint32_t r = 0;                          \
        if (in) {                                                                           \
            u = perm ? perm[x] : (O)x;                                                      \
            s = g.row[u]; e = g.row[u + 1];                                                 \
            act = (e - s) <= HUB_DEG && !pick_skip<INITIAL, UNIFORM, O, E, W>(u, vcmap, hn); \
            r = (uint32_t)jet_rng(seed, stream, (uint64_t)u);                               \
        }                                                                                   \
        int64_t bw = 0; uint32_t bh = 0; int64_t bj = -1;                                   \
        if (act) pick_edges<INITIAL, UNIFORM, O, E, W>(g, vcmap, r, s + lane, e, (E)G, bw, bh, bj); \
        for (int m = G >> 1; m > 0; m >>= 1) {                                              \
            int64_t w2 = shfl_xor(bw, m, G); uint32_t h2 = shfl_xor(bh, m, G);              \
            int64_t j2 = shfl_xor(bj, m, G);                                                \
            if (pick_better(w2, h2, j2, bw, bh, bj)) { bw = w2; bh = h2; bj = j2; }         \
        }                                                                                   \
        if (act && lane == 0) hn[u] = bj >= 0 ? g.adj[bj] : MAXV;                           \
    }
    JET_GROUP_LOOP(G, len, PICK_BODY)
#undef PICK_BODY
}

template <bool INITIAL, bool UNIFORM, class O, class E, class W>
__global__ void __launch_bounds__(1024) k_pick_match_hub(GView<O, E, W> g, const O* hubs, O nhub, const O* vcmap, O* hn,
                                                         uint64_t seed, uint64_t stream) {
    const O MAXV = ord_max<O>();
    __shared__ int64_t sw[32], sj[32];
    __shared__ uint32_t sh[32];
    for (O x = blockIdx.x; x < nhub; x += gridDim.x) {
        O u = hubs[x];
        bool act = INITIAL || !pick_skip<INITIAL, UNIFORM, O, E, W>(u, vcmap, hn);
        // in the non-initial case only vertices still proposing take part
        if (!INITIAL && act) act = vcmap[u] == MAXV && hn[u] != MAXV;
        uint32_t r = (uint32_t)jet_rng(seed, stream, (uint64_t)u);
        int64_t bw = 0; uint32_t bh = 0; int64_t bj = -1;
        if (act) pick_edges<INITIAL, UNIFORM, O, E, W>(g, vcmap, r, g.row[u] + threadIdx.x, g.row[u + 1], (E)blockDim.x, bw, bh, bj);
        for (int m = 16; m > 0; m >>= 1) {
            int64_t w2 = shfl_xor(bw, m, 32); uint32_t h2 = shfl_xor(bh, m, 32); int64_t j2 = shfl_xor(bj, m, 32);
            if (pick_better(w2, h2, j2, bw, bh, bj)) { bw = w2; bh = h2; bj = j2; }
        }
        if ((threadIdx.x & 31) == 0) { sw[threadIdx.x >> 5] = bw; sh[threadIdx.x >> 5] = bh; sj[threadIdx.x >> 5] = bj; }
        __syncthreads();
        if (threadIdx.x == 0 && act) {
            for (int w = 1; w < (int)(blockDim.x >> 5); w++)
                if (pick_better(sw[w], sh[w], sj[w], bw, bh, bj)) { bw = sw[w]; bh = sh[w]; bj = sj[w]; }
            hn[u] = bj >= 0 ? g.adj[bj] : MAXV;
        }
        __syncthreads();
    }
}

// Commit rounds, src/heuristics.hpp:462-501.  Part 1 marks inactive
// vertices; in part 2 an inactive v goes to the first active proposer in
// index order (what the reference's in-order pass yields), found with
// atomicMin so the outcome does not depend on thread timing.
template <class O>
__global__ void k_commit1(O n, const O* perm, const O* perm_len, const O* hn, O* vcmap, O* winner, int r) {
    const O MAXV = ord_max<O>();
    O len = perm ? *perm_len : n;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < len; x += (int64_t)gridDim.x * blockDim.x) {
        O u = perm ? perm[x] : (O)x;
        winner[u] = MAXV;
        O v = hn[u];
        if (v == MAXV || vcmap[u] != MAXV) continue;
        bool cond = r > 0 ? (pod_hash((O)(u + r)) < pod_hash((O)(v + r))) : (u < v);
        if (!cond) vcmap[u] = MAXV - 1;
    }
}
template <class O>
__global__ void k_commit2a(O n, const O* perm, const O* perm_len, const O* hn, const O* vcmap, O* winner) {
    const O MAXV = ord_max<O>();
    O len = perm ? *perm_len : n;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < len; x += (int64_t)gridDim.x * blockDim.x) {
        O u = perm ? perm[x] : (O)x;
        O v = hn[u];
        if (v == MAXV || vcmap[u] != MAXV) continue;
        if (vcmap[v] == MAXV - 1) atomic_min_o<O>(&winner[v], u);
    }
}
template <class O>
__global__ void k_commit2(O n, const O* perm, const O* perm_len, const O* hn, O* vcmap, const O* winner) {
    const O MAXV = ord_max<O>();
    O len = perm ? *perm_len : n;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < len; x += (int64_t)gridDim.x * blockDim.x) {
        O u = perm ? perm[x] : (O)x;
        O v = hn[u];
        if (v == MAXV || vcmap[u] != MAXV) continue;
        if (winner[v] == u) {
            O cv = u < v ? u : v;
            vcmap[v] = cv;
            vcmap[u] = cv;
        }
    }
}
template <class O>
__global__ void k_commit3(O n, const O* perm, const O* perm_len, O* vcmap) {
    const O MAXV = ord_max<O>();
    O len = perm ? *perm_len : n;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < len; x += (int64_t)gridDim.x * blockDim.x) {
        O u = perm ? perm[x] : (O)x;
        if (vcmap[u] == MAXV - 1) vcmap[u] = MAXV;
    }
}
// Remaining proposers: unmatched with a valid proposal (src/heuristics.hpp:524-531).
template <class O>
__global__ void k_match_remaining(O n, const O* perm, const O* perm_len, const O* hn, const O* vcmap, O* next, O* next_len) {
    const O MAXV = ord_max<O>();
    O len = perm ? *perm_len : n;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t rounds = ceil_div<int64_t>((int64_t)len, stride);
    for (int64_t r = 0; r < rounds; r++) {
        int64_t x = start + r * stride;
        O u = 0;
        bool keep = false;
        if (x < len) { u = perm ? perm[x] : (O)x; keep = vcmap[u] == MAXV && hn[u] != MAXV; }
        O s = warp_append(next_len, keep);
        if (keep) next[s] = u;
    }
}

// ---------------------------------------------------------------- 2-hop
template <class O>
__global__ void k_count_unmatched(O n, const O* vcmap, O* out) {
    O c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        c += vcmap[i] == ord_max<O>();
    c = group_sum<O>(c, 32);
    if ((threadIdx.x & 31) == 0 && c) atomic_add(out, c);
}

// Unmatched vertices (optionally only degree-1 ones) in index order, via a
// scan so that list positions match the reference's scan order
// (src/heuristics.hpp:545-552, :569-576, :607-614).
template <class O, class E>
struct GetUnmatched {
    const O* vcmap;
    const E* row;
    int leaves_only;
    __device__ __forceinline__ O operator()(int64_t i) const {
        bool um = vcmap[i] == ord_max<O>();
        if (leaves_only) um = um && (row[i + 1] - row[i] == 1);
        return um ? (O)1 : (O)0;
    }
};
template <class O, class E>
__global__ void k_scatter_unmatched(O n, const O* vcmap, const E* row, int leaves_only, const O* pos, O* list) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        bool um = vcmap[i] == ord_max<O>();
        if (leaves_only) um = um && (row[i + 1] - row[i] == 1);
        if (um) list[pos[i]] = (O)i;
    }
}

template <class O, class E, class W>
__global__ void k_leaf_hash(GView<O, E, W> g, const O* list, O cnt, O* hashes) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < cnt; x += (int64_t)gridDim.x * blockDim.x)
        hashes[x] = g.adj[g.row[list[x]]];
}

// Order-free adjacency digest sum(h^2 + h), h = pod_hash(neighbour)
// (src/heuristics.hpp:580-594).  One warp per vertex; one CTA per hub.
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_twin_hash(GView<O, E, W> g, const O* list, O cnt, uint64_t* hashes) {
#define TWIN_BODY(x, in, lane)                                                              \
    {                                                                                       \
        uint64_t h = 0; O u = 0; E s = 0, e = 0;                                            \
        if (in) { u = list[x]; s = g.row[u]; e = g.row[u + 1]; if (e - s > HUB_DEG) e = s; } \
        for (E j = s + lane; j < e; j += 32) { uint64_t y = pod_hash(g.adj[j]); h += y * y + y; } \
        h = group_sum<uint64_t>(h, 32);                                                     \
        if (in && lane == 0 && g.row[u + 1] - s <= HUB_DEG) hashes[x] = h;                  \
    }
    JET_GROUP_LOOP(32, cnt, TWIN_BODY)
#undef TWIN_BODY
}
// Hub rows (deg > HUB_DEG) of the unmatched list, one CTA each: walks the
// level's hub list and writes each unmatched hub's digest at its list
// position pos[u].
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_twin_hash_hub(GView<O, E, W> g, const O* hub_list, O n_hub, const O* vcmap,
                                                        const O* pos, uint64_t* hashes) {
    __shared__ uint64_t part[32];
    for (O x = blockIdx.x; x < n_hub; x += gridDim.x) {
        O u = hub_list[x];
        if (vcmap[u] != ord_max<O>()) continue;
        E s = g.row[u], e = g.row[u + 1];
        uint64_t h = 0;
        for (E j = s + threadIdx.x; j < e; j += blockDim.x) { uint64_t y = pod_hash(g.adj[j]); h += y * y + y; }
        h = group_sum<uint64_t>(h, 32);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = h;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < (int)(blockDim.x >> 5); w++) h += part[w];
            hashes[pos[u]] = h;
        }
        __syncthreads();
    }
}

// Lowest-degree neighbour, heaviest edge among equals (first wins)
// (src/heuristics.hpp:615-637).
template <class O, class E, class W>
__global__ void k_relative_hash(GView<O, E, W> g, const O* list, O cnt, O* hashes) {
    const O MAXV = ord_max<O>();
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < cnt; x += (int64_t)gridDim.x * blockDim.x) {
        O u = list[x];
        O h = MAXV;
        W max_wgt = 0;
        O min_deg = MAXV;
        for (E j = g.row[u]; j < g.row[u + 1]; j++) {
            O v = g.adj[j];
            O vdeg = (O)(g.row[v + 1] - g.row[v]);
            if (min_deg > vdeg) { min_deg = vdeg; max_wgt = g.val[j]; h = v; }
            else if (min_deg == vdeg && max_wgt < g.val[j]) { h = v; max_wgt = g.val[j]; }
        }
        hashes[x] = h;
    }
}

// matchHash, src/heuristics.hpp:277-319, in list order: vertices with equal
// digests pair up consecutively (1st with 2nd, 3rd with 4th, ...), which is
// what the reference's table loop gives when run in list order with the
// entries whose digest equals the table's null key run last (those all share
// the first free slot past their home slot).  On the device: a stable radix
// sort by digest, then group ranks from a scan of group heads.
template <class O, class H>
struct GetDigestKey {
    const H* h;
    H nullkey;
    H null_as;  // key the null digest sorts under (its own group)
    __device__ __forceinline__ H operator()(int64_t i) const { H v = h[i]; return v == nullkey ? null_as : v; }
};
template <class K, class O>
struct GetGroupHead {
    const K* sk;
    __device__ __forceinline__ O operator()(int64_t q) const { return (q == 0 || sk[q] != sk[q - 1]) ? (O)1 : (O)0; }
};
template <class K, class O>
__global__ void k_group_starts(const K* sk, int64_t n, const O* ex, O* start) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        if (q == 0 || sk[q] != sk[q - 1]) start[ex[q]] = (O)q;
}
template <class K, class O>
__global__ void k_pair_groups(const K* sk, const O* sx, const O* list, int64_t n, const O* ex, const O* start, O* vcmap) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        bool head = q == 0 || sk[q] != sk[q - 1];
        O gid = ex[q] + (head ? 1 : 0) - 1;
        int64_t r = q - (int64_t)start[gid];
        if ((r & 1) || q + 1 >= n || sk[q + 1] != sk[q]) continue;
        O a = list[sx[q]], b = list[sx[q + 1]];
        O cv = a < b ? a : b;
        vcmap[a] = cv;
        vcmap[b] = cv;
    }
}

}  // namespace jetb
