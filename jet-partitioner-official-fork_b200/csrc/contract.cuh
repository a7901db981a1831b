// contract.cuh -- contraction of a level under a fine->coarse map
// (src/contract.hpp:147-446 of the reference).
//
// Coarse vertex weights are sums of member weights.  Each coarse row holds
// the distinct coarse neighbours other than itself with summed edge weights.
// Work per coarse row c scales with du(c) = sum of member degrees:
//   du <= 32        one warp per row, dedupe with match.any (rows come out sorted)
//   32 < du <= 256  128-thread CTA, 512-slot shared-memory hash table
//   256 < du <= 4K  512-thread CTA, 8192-slot shared-memory hash table
//   du > 4K         1024-thread CTA, hash table in global scratch (size du)
// Unique entries land in a scratch array at the row's upper-bound offset,
// then a copy pass packs them into the coarse CSR.
#pragma once
#include "graph.cuh"

namespace jetb {

static constexpr int CT_S1_DU = 256, CT_S1_SLOTS = 512, CT_S1_THREADS = 128;
static constexpr int CT_S2_DU = 4096, CT_S2_SLOTS = 8192, CT_S2_THREADS = 512;
__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }
// hash table (slots) plus a sort buffer of slots/2 entries (a row in the bin
// has at most slots/2 distinct neighbours)
template <class O, class W>
constexpr size_t contract_smem_bytes(int slots) {
    return align16((size_t)slots * sizeof(O)) + align16((size_t)slots * sizeof(W)) + align16((size_t)(slots / 2) * sizeof(O)) +
           (size_t)(slots / 2) * sizeof(W);
}

// Sorts P (a power of two) key/value pairs in shared memory by key.
template <int THREADS, class K, class V>
__device__ __forceinline__ void block_bitonic_sort(K* key, V* val, int P) {
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += THREADS) {
                int ixj = i ^ j;
                if (ixj > i) {
                    bool up = (i & k) == 0;
                    K a = key[i], b = key[ixj];
                    if ((a > b) == up) {
                        key[i] = b; key[ixj] = a;
                        V t = val[i]; val[i] = val[ixj]; val[ixj] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
}

template <class O, class E, class W>
__global__ void k_contract_count(GView<O, E, W> g, const O* map, O* cnt, E* du, W* cvw) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < g.n; i += (int64_t)gridDim.x * blockDim.x) {
        O c = map[i];
        atomic_add(&cnt[c], (O)1);
        atomic_add(&du[c], (E)(g.row[i + 1] - g.row[i]));
        atomic_add(&cvw[c], g.vw[i]);
    }
}

template <class O>
__global__ void k_contract_members(O n, const O* map, const O* moff, O* cnt, O* members) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        O c = map[i];
        O pos = atomic_add(&cnt[c], (O)-1) - 1;
        members[moff[c] + pos] = (O)i;
    }
}

template <class O, class E>
__global__ void k_contract_bin(O nc, const E* hrow, O* l1, O* n1, O* l2, O* n2, O* lh, O* nh) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t rounds = ceil_div<int64_t>((int64_t)nc, stride);
    for (int64_t r = 0; r < rounds; r++) {
        int64_t c = start + r * stride;
        E d = 0;
        if (c < nc) d = hrow[c + 1] - hrow[c];
        O s = warp_append(n1, c < nc && d > 32 && d <= CT_S1_DU);
        if (s >= 0) l1[s] = (O)c;
        s = warp_append(n2, c < nc && d > CT_S1_DU && d <= CT_S2_DU);
        if (s >= 0) l2[s] = (O)c;
        s = warp_append(nh, c < nc && d > CT_S2_DU);
        if (s >= 0) lh[s] = (O)c;
    }
}

// du <= 32: one warp per coarse row.
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_contract_warp(GView<O, E, W> g, const O* map, O nc, const O* moff, const O* members,
                                                        const E* hrow, O* skey, W* sval, O* ucnt) {
#define CW_BODY(x, in, lane)                                                                \
    {                                                                                       \
        O c = (O)x;                                                                         \
        E d = 0, hs = 0;                                                                    \
        if (in) { hs = hrow[c]; d = hrow[c + 1] - hs; }                                     \
        bool row_ok = in && d <= 32;                                                        \
        O key = (O)-1; W w = 0;                                                             \
        if (row_ok && (E)lane < d) {                                                        \
            O m0 = moff[c], m1 = moff[c + 1];                                               \
            E acc = 0, t = (E)lane;                                                         \
            for (O m = m0; m < m1; m++) {                                                   \
                O i = members[m];                                                           \
                E rs = g.row[i], dd = g.row[i + 1] - rs;                                    \
                if (t < acc + dd) {                                                         \
                    E j = rs + (t - acc);                                                   \
                    O u = map[g.adj[j]];                                                    \
                    if (u != c) { key = u; w = g.val[j]; }                                  \
                    break;                                                                  \
                }                                                                           \
                acc += dd;                                                                  \
            }                                                                               \
        }                                                                                   \
        unsigned grp = __match_any_sync(0xffffffffu, key);                                  \
        bool leader = key != (O)-1 && (__ffs(grp) - 1) == lane;                             \
        W sum = 0; int rank = 0;                                                            \
        unsigned leaders = __ballot_sync(0xffffffffu, leader);                              \
        for (int sl = 0; sl < 32; sl++) {                                                   \
            W ws = __shfl_sync(0xffffffffu, w, sl);                                         \
            O ks = __shfl_sync(0xffffffffu, key, sl);                                       \
            if ((grp >> sl) & 1u) sum += ws;                                                \
            if (((leaders >> sl) & 1u) && ks < key) rank++;                                 \
        }                                                                                   \
        if (row_ok && leader) { skey[hs + rank] = key; sval[hs + rank] = sum; }             \
        if (row_ok && lane == 0) ucnt[c] = (O)__popc(leaders);                              \
    }
    JET_GROUP_LOOP(32, nc, CW_BODY)
#undef CW_BODY
}

__device__ __forceinline__ uint32_t slot_hash(uint64_t k) {
    k *= 0x9E3779B97F4A7C15ull;
    return (uint32_t)(k >> 32);
}

// Walks the concatenated adjacency of a coarse row's members with the whole
// CTA: members are taken blockDim at a time, their degrees prefix-summed in
// shared memory, and each thread locates its edge by binary search.
template <int THREADS, class O, class E, class W, class F>
__device__ __forceinline__ void cta_for_row_edges(GView<O, E, W> g, const O* members, O m0, O m1, E* s_pref, O* s_mem,
                                                  F&& f) {
    for (O mb = m0; mb < m1; mb += THREADS) {
        O cnt = m1 - mb < THREADS ? m1 - mb : THREADS;
        E d = 0;
        if ((O)threadIdx.x < cnt) {
            O i = members[mb + threadIdx.x];
            s_mem[threadIdx.x] = i;
            d = g.row[i + 1] - g.row[i];
        }
        // inclusive prefix of degrees in shared memory (Hillis-Steele)
        s_pref[threadIdx.x] = d;
        __syncthreads();
        for (int o = 1; o < THREADS; o <<= 1) {
            E v = threadIdx.x >= (unsigned)o ? s_pref[threadIdx.x - o] : 0;
            __syncthreads();
            s_pref[threadIdx.x] += v;
            __syncthreads();
        }
        E total = s_pref[cnt - 1];
        for (E t = threadIdx.x; t < total; t += THREADS) {
            int lo = 0, hi = (int)cnt - 1;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (s_pref[mid] > t) hi = mid; else lo = mid + 1;
            }
            E before = lo > 0 ? s_pref[lo - 1] : 0;
            O i = s_mem[lo];
            f(g.row[i] + (t - before));
        }
        __syncthreads();
    }
}

template <int THREADS, int SLOTS, class O, class E, class W>
__global__ void __launch_bounds__(THREADS) k_contract_smem(GView<O, E, W> g, const O* map, const O* list, const O* count,
                                                          const O* moff, const O* members, const E* hrow, O* skey, W* sval,
                                                          O* ucnt) {
    extern __shared__ __align__(16) unsigned char ct_smem[];
    O* keys = (O*)ct_smem;
    W* vals = (W*)(ct_smem + align16((size_t)SLOTS * sizeof(O)));
    O* sk = (O*)((unsigned char*)vals + align16((size_t)SLOTS * sizeof(W)));
    W* sv = (W*)((unsigned char*)sk + align16((size_t)(SLOTS / 2) * sizeof(O)));
    __shared__ E s_pref[THREADS];
    __shared__ O s_mem[THREADS];
    __shared__ int s_cnt;
    O total_rows = *count;
    for (O x = blockIdx.x; x < total_rows; x += gridDim.x) {
        O c = list[x];
        E hs = hrow[c], d = hrow[c + 1] - hs;
        int ts = 64;
        while (ts < 2 * d) ts <<= 1;
        if (ts > SLOTS) ts = SLOTS;
        for (int s = threadIdx.x; s < ts; s += THREADS) { keys[s] = (O)-1; vals[s] = 0; }
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        cta_for_row_edges<THREADS>(g, members, moff[c], moff[c + 1], s_pref, s_mem, [&](E j) {
            O u = map[g.adj[j]];
            if (u == c) return;
            W w = g.val[j];
            uint32_t slot = slot_hash((uint64_t)u) & (ts - 1);
            for (int probe = 0; probe < ts; probe++) {
                O k = keys[slot];
                if (k == (O)-1) {
                    O old = atomic_cas(&keys[slot], (O)-1, u);
                    if (old == (O)-1 || old == u) { atomic_add(&vals[slot], w); return; }
                } else if (k == u) {
                    atomic_add(&vals[slot], w);
                    return;
                }
                slot = (slot + 1) & (ts - 1);
            }
        });
        __syncthreads();
        // pack the occupied slots, sort them by neighbour id, write the row
        for (int base = 0; base < ts; base += THREADS) {
            int s = base + threadIdx.x;
            bool occ = s < ts && keys[s] != (O)-1;
            unsigned b = __ballot_sync(0xffffffffu, occ);
            int wpos = 0;
            if ((threadIdx.x & 31) == 0 && b) wpos = atomicAdd(&s_cnt, __popc(b));
            wpos = __shfl_sync(0xffffffffu, wpos, 0);
            if (occ) {
                int p = wpos + __popc(b & ((1u << (threadIdx.x & 31)) - 1));
                sk[p] = keys[s];
                sv[p] = vals[s];
            }
        }
        __syncthreads();
        int u = s_cnt;
        int P = 1;
        while (P < u) P <<= 1;
        for (int i = u + threadIdx.x; i < P; i += THREADS) sk[i] = std::numeric_limits<O>::max();
        __syncthreads();
        block_bitonic_sort<THREADS>(sk, sv, P);
        for (int i = threadIdx.x; i < u; i += THREADS) { skey[hs + i] = sk[i]; sval[hs + i] = sv[i]; }
        __syncthreads();
        if (threadIdx.x == 0) ucnt[c] = (O)u;
        __syncthreads();
    }
}

// du > 4096: open-addressed table of size du in the row's scratch region.
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_contract_hub(GView<O, E, W> g, const O* map, const O* list, const O* count,
                                                       const O* moff, const O* members, const E* hrow, O* skey, W* sval,
                                                       O* ucnt, int* err) {
    __shared__ E s_pref[1024];
    __shared__ O s_mem[1024];
    __shared__ unsigned long long s_cnt;
    O total_rows = *count;
    for (O x = blockIdx.x; x < total_rows; x += gridDim.x) {
        O c = list[x];
        E hs = hrow[c], d = hrow[c + 1] - hs;
        for (E s = threadIdx.x; s < d; s += blockDim.x) { skey[hs + s] = (O)-1; sval[hs + s] = 0; }
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        cta_for_row_edges<1024>(g, members, moff[c], moff[c + 1], s_pref, s_mem, [&](E j) {
            O u = map[g.adj[j]];
            if (u == c) return;
            W w = g.val[j];
            E slot = (E)(slot_hash((uint64_t)u) % (uint64_t)d);
            for (E probe = 0; probe < d; probe++) {
                O k = ld_cg(&skey[hs + slot]);
                if (k == (O)-1) {
                    O old = atomic_cas(&skey[hs + slot], (O)-1, u);
                    if (old == (O)-1) { atomicAdd(&s_cnt, 1ull); atomic_add(&sval[hs + slot], w); return; }
                    if (old == u) { atomic_add(&sval[hs + slot], w); return; }
                } else if (k == u) {
                    atomic_add(&sval[hs + slot], w);
                    return;
                }
                slot++;
                if (slot >= d) slot = 0;
            }
            atomicOr(err, ERRF_OVERFLOW);
        });
        __syncthreads();
        if (threadIdx.x == 0) ucnt[c] = (O)s_cnt;
        __syncthreads();
    }
}

// Packs each row's unique entries into the coarse CSR.
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_contract_copy(O nc, const E* hrow, const O* skey, const W* sval, const E* crow,
                                                        O* cadj, W* cval) {
#define CC_BODY(x, in, lane)                                                                \
    {                                                                                       \
        if (in) {                                                                           \
            O c = (O)x;                                                                     \
            E hs = hrow[c];                                                                 \
            if (hrow[c + 1] - hs <= CT_S2_DU) {                                             \
                E o = crow[c], cnt = crow[c + 1] - o;                                       \
                for (E t = lane; t < cnt; t += 32) { cadj[o + t] = skey[hs + t]; cval[o + t] = sval[hs + t]; } \
            }                                                                               \
        }                                                                                   \
    }
    JET_GROUP_LOOP(32, nc, CC_BODY)
#undef CC_BODY
}

template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_contract_copy_hub(const O* list, const O* count, const E* hrow, const O* skey,
                                                            const W* sval, const E* crow, O* cadj, W* cval) {
    __shared__ unsigned long long s_pos;
    O total_rows = *count;
    for (O x = blockIdx.x; x < total_rows; x += gridDim.x) {
        O c = list[x];
        E hs = hrow[c], d = hrow[c + 1] - hs, o = crow[c];
        if (threadIdx.x == 0) s_pos = 0;
        __syncthreads();
        for (E base = 0; base < d; base += blockDim.x) {
            E s = base + threadIdx.x;
            bool occ = s < d && skey[hs + s] != (O)-1;
            unsigned b = __ballot_sync(0xffffffffu, occ);
            unsigned long long wpos = 0;
            if ((threadIdx.x & 31) == 0 && b) wpos = atomicAdd(&s_pos, (unsigned long long)__popc(b));
            wpos = __shfl_sync(0xffffffffu, wpos, 0);
            if (occ) {
                E p = (E)wpos + __popc(b & ((1u << (threadIdx.x & 31)) - 1));
                cadj[o + p] = skey[hs + s];
                cval[o + p] = sval[hs + s];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- hub rows in neighbour order
// Rows built in the global table (du > 4096) come out in slot order; these
// put them in neighbour-id order like every other row.  Hub row x (coarse
// vertex list[x]) owns entries [hoff[x], hoff[x+1]) of the enumeration.
template <class O, class E>
struct GetHubRowSize {
    const O* list;
    const E* crow;
    __device__ __forceinline__ E operator()(int64_t x) const { O c = list[x]; return crow[c + 1] - crow[c]; }
};
template <class E>
__device__ __forceinline__ int64_t hub_row_of(const E* hoff, int64_t nhub, int64_t q) {
    int64_t lo = 0, hi = nhub - 1;  // last x with hoff[x] <= q
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) >> 1;
        if ((int64_t)hoff[mid] <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
}
template <class O, class E>
struct GetHubKey {
    const O* list;
    const E* crow;
    const E* hoff;
    int64_t nhub;
    const O* cadj;
    int nb;  // bits of a neighbour id
    __device__ __forceinline__ uint64_t operator()(int64_t q) const {
        int64_t x = hub_row_of<E>(hoff, nhub, q);
        E pos = crow[list[x]] + (E)(q - (int64_t)hoff[x]);
        return ((uint64_t)x << nb) | (uint64_t)cadj[pos];
    }
};
template <class O, class E, class W>
__global__ void k_hub_gather(const O* list, const E* crow, const E* hoff, int64_t nhub, int64_t total, const int64_t* sq,
                             const W* cval, W* tval) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t q = sq[t];
        int64_t x = hub_row_of<E>(hoff, nhub, q);
        tval[t] = cval[crow[list[x]] + (E)(q - (int64_t)hoff[x])];
    }
}
template <class O, class E, class W>
__global__ void k_hub_place(const O* list, const E* crow, const E* hoff, int64_t total, const uint64_t* skey,
                            const W* tval, int nb, O* cadj, W* cval) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        uint64_t key = skey[t];
        int64_t x = (int64_t)(key >> nb);
        E pos = crow[list[x]] + (E)(t - (int64_t)hoff[x]);
        cadj[pos] = (O)(key & ((1ull << nb) - 1ull));
        cval[pos] = tval[t];
    }
}

}  // namespace jetb
