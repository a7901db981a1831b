// contract.cuh -- contraction of a level under a fine->coarse map
// (src/contract.hpp:147-446 of the reference).
//
// Coarse vertex weights are sums of member weights.  Each coarse row holds
// the distinct coarse neighbours other than itself with summed edge weights.
// Work per coarse row c scales with du(c) = sum of member degrees:
//   du <= 32        one warp per row, dedupe with match.any
//   32 < du <= 256  128-thread CTA, 512-slot shared-memory hash table, sorted
//   256 < du <= 4K  512-thread CTA, 8192-slot shared-memory hash table, sorted
//   du > 4K         few coarse ids: a dense shared-memory accumulator per row;
//                   many: (row, neighbour) keys, a radix sort, reduce-by-key
// Unique entries land, in neighbour order, in a scratch array at the row's
// upper-bound offset; a copy pass packs them into the coarse CSR.
#pragma once
#include "graph.cuh"

namespace jetb {

static constexpr int CT_S1_DU = 256, CT_S1_SLOTS = 512, CT_S1_THREADS = 128;
static constexpr int CT_S2A_DU = 1024, CT_S2A_SLOTS = 2048, CT_S2A_THREADS = 256;
static constexpr int CT_S2B_DU = 2048, CT_S2B_SLOTS = 4096, CT_S2B_THREADS = 512;
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

// Stable LSD radix sort of u (key, value) pairs in shared memory, 8-bit
// digits over key bits [0, bits).  Each warp owns a contiguous chunk of the
// input; per pass it counts its digits (match.any peers, one counter per warp
// and digit, digit-major), one block scan turns the counts into offsets, and
// a second sweep scatters every element to its offset plus its rank among
// equal digits before it in the chunk.  `hist` holds THREADS / 32 * 256
// counters.  Returns the buffer that holds the result: 0 = (ka, va), 1 = (kb, vb).
template <int THREADS, class K, class V>
__device__ __forceinline__ int block_radix_sort_pairs(K* ka, V* va, K* kb, V* vb, int u, int bits, uint32_t* hist,
                                                      uint32_t* s_sw) {
    constexpr int NW = THREADS / 32;
    constexpr int PER = NW * 256 / THREADS;  // counters per thread in the scan
    static_assert(NW * 256 % THREADS == 0, "scan tiling");
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int chunk = (u + NW - 1) / NW;
    const int c0 = wid * chunk < u ? wid * chunk : u;
    const int c1 = c0 + chunk < u ? c0 + chunk : u;
    int cur = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        K* ks = cur == 0 ? ka : kb;
        V* vs = cur == 0 ? va : vb;
        K* kd = cur == 0 ? kb : ka;
        V* vd = cur == 0 ? vb : va;
        for (int i = threadIdx.x; i < NW * 256; i += THREADS) hist[i] = 0;
        __syncthreads();
        for (int b = c0; b < c1; b += 32) {
            const int e = b + lane;
            const bool in = e < c1;
            const int d = in ? (int)((ks[e] >> shift) & (K)255) : 256;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (in && (peers & ((1u << lane) - 1u)) == 0) hist[d * NW + wid] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        uint32_t loc[PER];
        uint32_t sum = 0;
#pragma unroll
        for (int q = 0; q < PER; q++) { loc[q] = hist[threadIdx.x * PER + q]; sum += loc[q]; }
        uint32_t tot;
        uint32_t run = block_exclusive_scan<uint32_t>(sum, s_sw, tot);
#pragma unroll
        for (int q = 0; q < PER; q++) { hist[threadIdx.x * PER + q] = run; run += loc[q]; }
        __syncthreads();
        for (int b = c0; b < c1; b += 32) {
            const int e = b + lane;
            const bool in = e < c1;
            const K key = in ? ks[e] : (K)0;
            const int d = in ? (int)((key >> shift) & (K)255) : 256;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int rank = __popc(peers & ((1u << lane) - 1u));
            const uint32_t base = in ? hist[d * NW + wid] : 0u;
            if (in) { kd[base + rank] = key; vd[base + rank] = vs[e]; }
            __syncwarp();
            if (in && rank == 0) hist[d * NW + wid] = base + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        cur ^= 1;
    }
    return cur;
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
__global__ void k_contract_bin(O nc, const E* hrow, O* l1, O* n1, O* l2a, O* n2a, O* l2b, O* n2b, O* l2, O* n2, O* lh, O* nh) {
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t rounds = ceil_div<int64_t>((int64_t)nc, stride);
    for (int64_t r = 0; r < rounds; r++) {
        int64_t c = start + r * stride;
        E d = 0;
        if (c < nc) d = hrow[c + 1] - hrow[c];
        O s = warp_append(n1, c < nc && d > 32 && d <= CT_S1_DU);
        if (s >= 0) l1[s] = (O)c;
        s = warp_append(n2a, c < nc && d > CT_S1_DU && d <= CT_S2A_DU);
        if (s >= 0) l2a[s] = (O)c;
        s = warp_append(n2b, c < nc && d > CT_S2A_DU && d <= CT_S2B_DU);
        if (s >= 0) l2b[s] = (O)c;
        s = warp_append(n2, c < nc && d > CT_S2B_DU && d <= CT_S2_DU);
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
// CTA.  A row of at most FEW_MEMBERS members (a matched pair or a singleton) is
// walked member by member with the CTA striding over each member's edges;
// otherwise members are taken blockDim at a time, their degrees
// prefix-summed in shared memory, and each thread locates its edge by binary
// search.  The row's member count is CTA-uniform, so is the choice.
static constexpr int FEW_MEMBERS = 2;
template <int THREADS, class O, class E, class W, class F>
__device__ __forceinline__ void cta_for_row_edges(GView<O, E, W> g, const O* members, O m0, O m1, E* s_pref, O* s_mem,
                                                  F&& f) {
    if (m1 - m0 <= FEW_MEMBERS) {
        for (O mi = m0; mi < m1; mi++) {
            O i = members[mi];
            for (E j = g.row[i] + threadIdx.x; j < g.row[i + 1]; j += THREADS) f(j);
        }
        return;
    }
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
                                                          O* ucnt, O nc, int narrow) {
    extern __shared__ __align__(16) unsigned char ct_smem[];
    O* keys = (O*)ct_smem;
    W* vals = (W*)(ct_smem + align16((size_t)SLOTS * sizeof(O)));
    O* sk = (O*)((unsigned char*)vals + align16((size_t)SLOTS * sizeof(W)));
    W* sv = (W*)((unsigned char*)sk + align16((size_t)(SLOTS / 2) * sizeof(O)));
    __shared__ E s_pref[THREADS];
    __shared__ O s_mem[THREADS];
    __shared__ int s_cnt;
    __shared__ int s_sw[32];
    // the radix sort's second buffers and counters must fit the hash table's space
    constexpr size_t kb_bytes = align16((size_t)(SLOTS / 2) * sizeof(O));
    constexpr size_t vb_bytes = align16((size_t)(SLOTS / 2) * sizeof(W));
    constexpr bool radix_fits = THREADS >= 256 && kb_bytes + vb_bytes + (size_t)(THREADS / 32) * 256 * sizeof(uint32_t) <=
                                                      align16((size_t)SLOTS * sizeof(O)) + (size_t)SLOTS * sizeof(W);
    O total_rows = *count;
    int id_bits = 0;
    while (id_bits < 63 && (((int64_t)nc - 1) >> id_bits) > 0) id_bits++;
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
                    if (old == (O)-1 || old == u) { acc_add<W>(&vals[slot], w, narrow); return; }
                } else if (k == u) {
                    acc_add<W>(&vals[slot], w, narrow);
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
        const int64_t words = ((int64_t)nc + 31) >> 5;
        if (words * 8 <= (int64_t)(align16((size_t)SLOTS * sizeof(O)) + (size_t)SLOTS * sizeof(W))) {
            // Rank by bitmap: the row's distinct ids set bits in an nc-bit
            // map (in the freed hash-table space); an id's rank is the number
            // of set bits before it (per-word prefix counts + popcount), so the
            // row is written in id order with no comparison sort.
            uint32_t* bm = (uint32_t*)ct_smem;
            int* wpre = (int*)(bm + words);
            for (int64_t w = threadIdx.x; w < words; w += THREADS) bm[w] = 0;
            __syncthreads();
            for (int e = threadIdx.x; e < u; e += THREADS) atomicOr(&bm[sk[e] >> 5], 1u << (sk[e] & 31));
            __syncthreads();
            const int per = (int)((words + THREADS - 1) / THREADS);
            const int64_t w0 = (int64_t)threadIdx.x * per, w1 = w0 + per < words ? w0 + per : words;
            int cntb = 0;
            for (int64_t w = w0; w < w1; w++) cntb += __popc(bm[w]);
            int totb;
            int run = block_exclusive_scan<int>(cntb, s_sw, totb);
            for (int64_t w = w0; w < w1; w++) { wpre[w] = run; run += __popc(bm[w]); }
            __syncthreads();
            for (int e = threadIdx.x; e < u; e += THREADS) {
                O key = sk[e];
                int64_t w = key >> 5;
                int r = wpre[w] + __popc(bm[w] & ((1u << (key & 31)) - 1u));
                skey[hs + r] = key;
                sval[hs + r] = sv[e];
            }
        } else if (radix_fits && u > 128) {
            // radix sort by id: the second key/value buffers and the digit
            // counters live in the freed hash-table space
            O* kb = (O*)ct_smem;
            W* vb = (W*)(ct_smem + kb_bytes);
            uint32_t* hist = (uint32_t*)(ct_smem + kb_bytes + vb_bytes);
            int which = block_radix_sort_pairs<radix_fits ? THREADS : 256, O, W>(sk, sv, kb, vb, u, id_bits, hist,
                                                                                (uint32_t*)s_sw);
            const O* rk = which == 0 ? sk : kb;
            const W* rv = which == 0 ? sv : vb;
            for (int i = threadIdx.x; i < u; i += THREADS) { skey[hs + i] = rk[i]; sval[hs + i] = rv[i]; }
        } else {
            int P = 1;
            while (P < u) P <<= 1;
            for (int i = u + threadIdx.x; i < P; i += THREADS) sk[i] = std::numeric_limits<O>::max();
            __syncthreads();
            block_bitonic_sort<THREADS>(sk, sv, P);
            for (int i = threadIdx.x; i < u; i += THREADS) { skey[hs + i] = sk[i]; sval[hs + i] = sv[i]; }
        }
        __syncthreads();
        if (threadIdx.x == 0) ucnt[c] = (O)u;
        __syncthreads();
    }
}

// du > 4096 on a level with few coarse vertices: a dense accumulator.  The
// coarse id range is walked in chunks of `chunk` ids; per chunk the CTA adds
// every member edge whose coarse neighbour falls in the chunk into a
// shared-memory array indexed by id, then writes the nonzero entries in id
// order (edge weights are positive, so a nonzero sum marks a neighbour).
// Rows come out sorted with no hashing and no sort; the cost is one read of
// the row's edges per chunk.
template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_contract_dense(GView<O, E, W> g, const O* map, const O* list, const O* count,
                                                         const O* moff, const O* members, const E* hrow, O nc, int chunk,
                                                         O* skey, W* sval, O* ucnt, int narrow) {
    extern __shared__ __align__(16) unsigned char ct_smem[];
    W* acc = (W*)ct_smem;
    __shared__ E s_pref[1024];
    __shared__ O s_mem[1024];
    __shared__ int s_sw[32];
    O total_rows = *count;
    for (O x = blockIdx.x; x < total_rows; x += gridDim.x) {
        O c = list[x];
        const O m0 = moff[c], m1 = moff[c + 1];
        E out = hrow[c];
        for (O base = 0; base < nc; base += chunk) {
            const O top = nc - base < (O)chunk ? nc : base + chunk;
            const int len = (int)(top - base);
            for (int i = threadIdx.x; i < len; i += blockDim.x) acc[i] = 0;
            __syncthreads();
            auto add = [&](E j) {
                O u = map[g.adj[j]];
                if (u != c && u >= base && u < top) acc_add<W>(&acc[u - base], g.val[j], narrow);
            };
            if (m1 - m0 <= 32) {
                // few members (the usual case for dense rows): stride over each member's edges
                for (O mi = m0; mi < m1; mi++) {
                    O i = members[mi];
                    for (E j = g.row[i] + threadIdx.x; j < g.row[i + 1]; j += blockDim.x) add(j);
                }
            } else {
                cta_for_row_edges<1024>(g, members, m0, m1, s_pref, s_mem, add);
            }
            __syncthreads();
            // id-ordered compaction, one 1024-entry tile at a time
            for (int t0 = 0; t0 < len; t0 += blockDim.x) {
                int i = t0 + threadIdx.x;
                W v = i < len ? acc[i] : (W)0;
                int tot;
                int ex = block_exclusive_scan<int>(v != 0 ? 1 : 0, s_sw, tot);
                if (v != 0) { skey[out + ex] = base + (O)i; sval[out + ex] = v; }
                out += tot;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) ucnt[c] = (O)(out - hrow[c]);
        __syncthreads();
    }
}

// Packs each row's unique entries into the coarse CSR as a flat copy of the
// output in chunks of CT_COPY_CHUNK slots, one warp per chunk, so that work
// is even whatever the row lengths.  chunk_row[j] is the row holding the
// chunk's first slot (k_copy_chunk_rows).  The warp walks the rows from there
// 32 at a time: lane l holds row r + l's output start, and each slot finds its
// row by a five-step binary search over the lanes (shuffles); loads and
// stores stay coalesced.
static constexpr int CT_COPY_CHUNK = 2048;
// The same packing with one warp per row, for levels whose rows are all
// short (no row above 2048 member edges): no row search, one pass.
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_contract_copy_rows(O nc, const E* hrow, const O* skey, const W* sval, const E* crow,
                                                             O* cadj, W* cval) {
#define CC_BODY(x, in, lane)                                                                \
    {                                                                                       \
        if (in) {                                                                           \
            const O c = (O)x;                                                               \
            const E hs = hrow[c], o = crow[c], cnt = crow[c + 1] - o;                      \
            for (E t = lane; t < cnt; t += 32) { cadj[o + t] = skey[hs + t]; cval[o + t] = sval[hs + t]; } \
        }                                                                                   \
    }
    JET_GROUP_LOOP(32, nc, CC_BODY)
#undef CC_BODY
}
template <class O, class E>
__global__ void k_copy_chunk_rows(O nc, const E* crow, O* chunk_row) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        const E s = crow[c], t = crow[c + 1];
        if (t <= s) continue;
        for (E j = (s + CT_COPY_CHUNK - 1) / CT_COPY_CHUNK; j * CT_COPY_CHUNK < t; j++) chunk_row[j] = (O)c;
    }
}
template <class O, class E, class W>
__global__ void __launch_bounds__(BLOCK) k_contract_copy(O nc, E mc, const O* chunk_row, const E* hrow, const O* skey,
                                                        const W* sval, const E* crow, O* cadj, W* cval) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t chunks = ((int64_t)mc + CT_COPY_CHUNK - 1) / CT_COPY_CHUNK;
    for (int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < chunks; j += warps) {
        const E e1 = (E)((j + 1) * CT_COPY_CHUNK < (int64_t)mc ? (j + 1) * CT_COPY_CHUNK : (int64_t)mc);
        E e = (E)(j * CT_COPY_CHUNK);
        for (int64_t r = chunk_row[j]; e < e1; r += 32) {
            const int64_t c = r + lane;
            const E os = c < nc ? crow[c] : mc;  // past the last row: never <= a live slot
            const E hs = c < nc ? hrow[c] : (E)0;
            const E wend = r + 32 < (int64_t)nc ? crow[r + 32] : mc;
            const E lim = wend < e1 ? wend : e1;
            for (E base = e; base < lim; base += 32) {
                const E x = base + lane;
                int lo = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const E v = __shfl_sync(0xffffffffu, os, lo + step);
                    if (v <= x) lo += step;
                }
                const E ro = __shfl_sync(0xffffffffu, os, lo);
                const E rh = __shfl_sync(0xffffffffu, hs, lo);
                if (x < lim) {
                    const E src = rh + (x - ro);
                    cadj[x] = skey[src];
                    cval[x] = sval[src];
                }
            }
            e = lim;
        }
    }
}

// ---------------------------------------------------------------- hub rows, many coarse ids
// du > 4096 on a level with many coarse vertices: every hub-row edge becomes
// a (row rank, coarse neighbour) key, one stable radix sort brings equal keys
// together in neighbour order, and a reduce-by-key writes each row's unique
// entries, sorted, into its scratch region.  Work is spread over the whole
// GPU whatever the row sizes.  hoff[x] is the exclusive prefix of du over
// the hub list; self-loops and padding get the sentinel key (past every row).
template <class O, class E>
struct GetHubDu {
    const O* list;
    const E* hrow;
    __device__ __forceinline__ E operator()(int64_t x) const { O c = list[x]; return hrow[c + 1] - hrow[c]; }
};

template <class O, class E, class W>
__global__ void __launch_bounds__(1024) k_hub_keys(GView<O, E, W> g, const O* map, const O* list, const O* count,
                                                   const O* moff, const O* members, const E* hoff, int nb, uint64_t sentinel,
                                                   uint64_t* key, W* val) {
    O total_rows = *count;
    for (O x = blockIdx.x; x < total_rows; x += gridDim.x) {
        O c = list[x];
        E out = hoff[x];
        for (O mi = moff[c]; mi < moff[c + 1]; mi++) {
            O i = members[mi];
            E rs = g.row[i], d = g.row[i + 1] - rs;
            for (E t = threadIdx.x; t < d; t += blockDim.x) {
                O u = map[g.adj[rs + t]];
                key[out + t] = u == c ? sentinel : (((uint64_t)x << nb) | (uint64_t)u);
                val[out + t] = g.val[rs + t];
            }
            out += d;
        }
    }
}

template <class K, class O>
struct GetKeyHead {
    const K* key;
    K sentinel;
    __device__ __forceinline__ O operator()(int64_t q) const {
        K k = key[q];
        return (k != sentinel && (q == 0 || key[q - 1] != k)) ? (O)1 : (O)0;
    }
};

// First segment index of every row present in the sorted keys.
static __global__ void k_hub_row_first(const uint64_t* key, int64_t total, int nb, uint64_t sentinel, const int64_t* seg,
                                int64_t* row_first) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = key[q];
        if (k == sentinel) continue;
        if (q == 0 || (key[q - 1] >> nb) != (k >> nb)) row_first[k >> nb] = seg[q];
    }
}

template <class O, class E, class W>
__global__ void k_hub_reduce(const uint64_t* key, const W* val, int64_t total, int nb, uint64_t sentinel, const int64_t* seg,
                             const int64_t* row_first, const O* list, const E* hrow, O* skey, W* sval, O* ucnt) {
    const uint64_t mask = (1ull << nb) - 1ull;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = key[q];
        if (k == sentinel || (q > 0 && key[q - 1] == k)) continue;
        W sum = 0;
        for (int64_t r = q; r < total && key[r] == k; r++) sum += val[r];
        int64_t x = (int64_t)(k >> nb);
        O c = list[x];
        E pos = hrow[c] + (E)(seg[q] - row_first[x]);
        skey[pos] = (O)(k & mask);
        sval[pos] = sum;
        atomic_add(&ucnt[c], (O)1);
    }
}

}  // namespace jetb
