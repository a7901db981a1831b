// jet_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A single-threaded CPU restatement of the Jet multilevel k-way partitioner's
// hot path (coarsening, contraction, Metis initial partition, Jet refinement,
// projection, partition statistics).  It is the checker for the CUDA library:
// only tests, the smoke check and the benchmark's CPU-baseline leg may load it.
// Nothing in the product links or calls it.
//
// Parity status: PINNED to the reference's own code.  oracle/ref.mk compiles
// the unmodified reference sources against a host-only Kokkos stand-in
// (oracle/kokkos_shim/) into oracle/_ref/, and tests/test_ref_pin.py runs
// every step below through both and demands identical results: pstat,
// gain_bucket, contraction given a map, connectivity tables given a partition,
// coarsening maps, LP / weak / strong refinement iterations, a full refinement
// level and uncoarsening a fixed hierarchy (the last four with edge weights
// under which no two parts tie, since ties are broken differently -- below),
// plus the 8-seed median cut within 2% of the reference's.
//
// Semantics follow the reference executed on one thread (its Serial execution
// space): every "parallel" loop runs in index order and every atomic is a plain
// read-modify-write.  Deliberate deviations, all in places where the reference's
// behaviour is an artefact of hash-slot layout or thread timing:
//   * RNG: a counter-based splitmix64 stream jet_rng(seed, stream, index)
//     replaces Kokkos' time-seeded XorShift64 pool (src/contract.hpp:503);
//     the CUDA library draws the same numbers.
//   * Ties between equally connected destination parts (LP select,
//     src/jet_refiner.hpp:222-230; weak rebalance, :606-613) go to the lowest
//     part id instead of the first hash slot, so results do not depend on the
//     connectivity table's slot layout.
//   * Contraction emits each coarse row sorted by neighbour id (the reference
//     emits hash-slot order, src/contract.hpp:320-327).
//   * rebalance_weak with no undersized part leaves the vertex in place (the
//     reference divides by zero there, src/jet_refiner.hpp:618).
//   * matchHash (src/heuristics.hpp:277-319) runs the entries whose digest
//     equals the table's null key after all others, so each digest value
//     pairs its members consecutively in list order.
// Reference files are cited as path:line inside the reference project.

#include <cstdint>
#include <cstring>
#include <cmath>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <limits>
#include <chrono>
#include <type_traits>

typedef int64_t metis_idx_t;
typedef float metis_real_t;
extern "C" int METIS_PartGraphKway(metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*,
                                   metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*,
                                   metis_real_t*, metis_real_t*, metis_idx_t*, metis_idx_t*,
                                   metis_idx_t*);

namespace orc {

typedef int32_t part_t;
static const part_t NULL_PART = -1;     // src/jet_refiner.hpp:87
static const part_t HASH_RECLAIM = -2;  // src/jet_refiner.hpp:88
static const part_t NO_MOVE = -3;       // src/jet_refiner.hpp:89
static const int MAX_SECTIONS = 128;    // src/jet_refiner.hpp:91
static const int MAX_BUCKETS = 50;      // src/jet_refiner.hpp:92
static const int MID_BUCKET = 25;       // src/jet_refiner.hpp:93

// ---------------------------------------------------------------- hashing / RNG
// src/heuristics.hpp:49-56
static inline uint32_t xorshift32(uint32_t x) {
    x ^= x << 13; x ^= x >> 17; x ^= x << 5; return x;
}
// MurmurHash3_x86_32 (Austin Appleby, public domain) over the key bytes with
// seed 0: the byte hash Kokkos::pod_hash applies (src/heuristics.hpp:73).
static inline uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
static inline uint32_t murmur3_words(const uint32_t* w, int nwords) {
    const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    uint32_t h = 0;
    for (int i = 0; i < nwords; i++) {
        uint32_t k = w[i];
        k *= c1; k = rotl32(k, 15); k *= c2;
        h ^= k; h = rotl32(h, 13); h = h * 5 + 0xe6546b64u;
    }
    h ^= (uint32_t)(nwords * 4);
    h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
    return h;
}
template <class O> static inline uint32_t pod_hash(O x) {
    uint32_t w[sizeof(O) / 4];
    std::memcpy(w, &x, sizeof(O));
    return murmur3_words(w, (int)(sizeof(O) / 4));
}
// splitmix64 finaliser (S. Vigna) over a (seed, stream, index) counter.
static inline uint64_t jet_rng(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (stream * 0x100000001B3ull + idx + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline uint64_t rng_stream(int level, int kind, int round) {
    return ((uint64_t)(uint32_t)level << 40) | ((uint64_t)(uint32_t)kind << 32) | (uint32_t)round;
}
enum { RNG_HEC_RANDOM = 1, RNG_MATCH_RANDOM = 2, RNG_MATCH_PICK = 3 };

// ---------------------------------------------------------------- graph
template <class O, class E, class W>
struct Csr {
    O n = 0;
    std::vector<E> row;
    std::vector<O> adj;
    std::vector<W> val;
    E nnz() const { return row.empty() ? 0 : row[n]; }
};

template <class O, class E, class W>
struct Level {
    Csr<O, E, W> g;
    std::vector<W> vw;
    std::vector<O> map;  // fine (previous level) -> this level; empty at level 1
    bool uniform = false;
};

// ---------------------------------------------------------------- statistics
// src/part_stat.hpp:77-108 (cut counted from both endpoints)
template <class O, class E, class W>
W total_cut(const Csr<O, E, W>& g, const part_t* part) {
    W cut = 0;
    for (O i = 0; i < g.n; i++)
        for (E j = g.row[i]; j < g.row[i + 1]; j++)
            if (part[i] != part[g.adj[j]]) cut += g.val[j];
    return cut;
}
// src/part_stat.hpp:111-114 -- ordinal arithmetic, as the reference declares it.
template <class O> O optimal_size(O total, part_t k) { return (total + k - 1) / k; }

template <class O, class E, class W>
std::vector<W> part_sizes(const Csr<O, E, W>& g, const W* vw, const part_t* part, part_t k) {
    std::vector<W> s(k, 0);
    for (O i = 0; i < g.n; i++) s[part[i]] += vw[i];
    return s;
}

// ---------------------------------------------------------------- coarsening
// HEC heavy-neighbour proposal, src/heuristics.hpp:196-250.
template <class O, class E, class W>
void hec_propose(const Csr<O, E, W>& g, const W* vw, bool uniform, uint64_t seed, int level, O* hn) {
    O n = g.n;
    if (uniform) {
        for (O i = 0; i < n; i++) {
            uint64_t r = jet_rng(seed, rng_stream(level, RNG_HEC_RANDOM, 0), (uint64_t)i);
            E deg = g.row[i + 1] - g.row[i];
            if (deg > 0) hn[i] = g.adj[g.row[i] + (E)(r % (uint64_t)deg)];
            else hn[i] = (O)(r % (uint64_t)n);
        }
        return;
    }
    W sum = 0;
    for (O i = 0; i < n; i++) sum += vw[i];
    W max_allowed = 6 * sum / n;
    for (O i = 0; i < n; i++) {
        E start = g.row[i], end = g.row[i + 1];
        if (end - start > 0 && vw[i] < max_allowed) {
            // ValLoc reduction evaluated in index order with ">=": the last
            // heaviest eligible edge wins.
            bool any = false; W best = 0; E loc = end;
            for (E j = start; j < end; j++) {
                W w = g.val[j];
                O v = g.adj[j];
                if ((!any || w >= best) && vw[v] < max_allowed) { best = w; loc = j; any = true; }
            }
            hn[i] = any ? g.adj[loc] : i;
        } else {
            hn[i] = i;
        }
    }
}

// Lock-free aggregation rounds, src/heuristics.hpp:89-169, run on one thread.
// vcmap receives, per vertex, the root vertex of its aggregate.
template <class O, class E, class W>
O hec_aggregate(O n, const O* hn, O* vcmap) {
    const O ORD_MAX = std::numeric_limits<O>::max();
    for (O i = 0; i < n; i++) vcmap[i] = ORD_MAX;
    std::vector<O> perm(n), next;
    for (O i = 0; i < n; i++) perm[i] = i;
    int swap = 1;
    while (!perm.empty()) {
        for (size_t x = 0; x < perm.size(); x++) {
            O u = perm[x];
            O v = hn[u];
            int condition = u < v;
            if (condition ^ swap) {
                if (vcmap[u] == ORD_MAX) {
                    vcmap[u] = ORD_MAX - 1;
                    if (u == v || vcmap[v] == ORD_MAX) {
                        vcmap[v] = ORD_MAX - 1;
                        O cv = v < u ? v : u;
                        vcmap[u] = cv;
                        vcmap[v] = cv;
                    } else {
                        if (vcmap[v] < n) vcmap[u] = vcmap[v];
                        else vcmap[u] = ORD_MAX;
                    }
                }
            }
        }
        next.clear();
        for (size_t x = 0; x < perm.size(); x++)
            if (vcmap[perm[x]] >= n) next.push_back(perm[x]);
        swap ^= 1;
        perm.swap(next);
    }
    return 0;
}

// Root numbering: roots (vcmap[u] == u) numbered in index order, everybody
// else takes its root's number (src/heuristics.hpp:147-165, :655-665).
template <class O>
O number_roots(O n, O* vcmap) {
    std::vector<O> id(n, -1);
    O nc = 0;
    for (O u = 0; u < n; u++) if (vcmap[u] == u) id[u] = nc++;
    for (O u = 0; u < n; u++) vcmap[u] = id[vcmap[u]];
    return nc;
}

// pickMatch, thread-per-vertex form, src/heuristics.hpp:397-425.
template <class O, class E, class W>
O pick_match(const Csr<O, E, W>& g, const O* vcmap, bool initial, bool uniform, uint32_t r, O u) {
    const O ORD_MAX = std::numeric_limits<O>::max();
    O h = ORD_MAX;
    W max_ewt = 0;
    uint32_t tiebreaker = 0;
    for (E j = g.row[u]; j < g.row[u + 1]; j++) {
        O v = g.adj[j];
        if (initial || vcmap[v] == ORD_MAX) {
            if (!uniform && max_ewt < g.val[j]) {
                max_ewt = g.val[j];
                h = v;
                tiebreaker = xorshift32((uint32_t)((uint64_t)v + r));
            } else if (uniform || max_ewt == g.val[j]) {
                uint32_t sim = xorshift32((uint32_t)((uint64_t)v + r));
                if (sim >= tiebreaker) { h = v; tiebreaker = sim; }
            }
        }
    }
    return h;
}

// matchHash, src/heuristics.hpp:277-319, one thread.
template <class O, class H>
void match_hash(const std::vector<O>& list, const std::vector<H>& hashes, H nullkey, O* vcmap) {
    O mappable = (O)list.size();
    if (mappable == 0) return;
    std::vector<H> htable(mappable, nullkey);
    std::vector<O> twins(mappable, -1);
    // List order, except that entries whose digest equals the null key run
    // after all others (one of the orders the reference's parallel loop can
    // take): they then all meet in one free slot, so every digest value forms
    // its own group and members pair up consecutively.
    for (int pass = 0; pass < 2; pass++)
    for (O x = 0; x < mappable; x++) {
        O i = list[x];
        H h = hashes[x];
        if ((h == nullkey) != (pass == 1)) continue;
        O key = (O)(h % (H)mappable);
        while (true) {
            if (htable[key] == nullkey) htable[key] = h;
            if (htable[key] == h) break;
            key++;
            if (key >= mappable) key -= mappable;
        }
        O twin = twins[key];
        if (twin == -1) {
            twins[key] = i;
        } else {
            O cv = twin < i ? twin : i;
            vcmap[twin] = cv;
            vcmap[i] = cv;
            twins[key] = -1;
        }
    }
}

// coarsen_match, src/heuristics.hpp:427-671.  two_hop selects the leaf/twin/
// relative passes (heuristic MtMetis).  hn_init (optional) receives the
// initial proposals.  Returns the number of coarse vertices; vcmap is the map.
template <class O, class E, class W>
O coarsen_match(const Csr<O, E, W>& g, bool uniform, bool two_hop, uint64_t seed, int level,
                O* vcmap, O* hn_init) {
    const O ORD_MAX = std::numeric_limits<O>::max();
    O n = g.n;
    std::vector<O> hn(n, ORD_MAX);
    for (O i = 0; i < n; i++) vcmap[i] = ORD_MAX;
    if (uniform) {
        for (O i = 0; i < n; i++) {
            E deg = g.row[i + 1] - g.row[i];
            if (deg == 0) continue;
            uint64_t r = jet_rng(seed, rng_stream(level, RNG_MATCH_RANDOM, 0), (uint64_t)i);
            hn[i] = g.adj[g.row[i] + (E)(r % (uint64_t)deg)];
        }
    } else {
        for (O i = 0; i < n; i++) {
            uint32_t r = (uint32_t)jet_rng(seed, rng_stream(level, RNG_MATCH_PICK, 0), (uint64_t)i);
            hn[i] = pick_match(g, vcmap, true, false, r, i);
        }
    }
    if (hn_init) for (O i = 0; i < n; i++) hn_init[i] = hn[i];
    std::vector<O> perm(n), next;
    for (O i = 0; i < n; i++) perm[i] = i;
    int outer = 0;
    while (!perm.empty()) {
        for (int r = 0; r < 4; r++) {
            for (O u : perm) {
                O v = hn[u];
                if (v == ORD_MAX || vcmap[u] != ORD_MAX) continue;
                bool condition = (r > 0) ? (pod_hash<O>((O)(u + r)) < pod_hash<O>((O)(v + r))) : (u < v);
                if (!condition) vcmap[u] = ORD_MAX - 1;
            }
            for (O u : perm) {
                O v = hn[u];
                if (v == ORD_MAX || vcmap[u] != ORD_MAX) continue;
                O cv = u < v ? u : v;
                if (vcmap[v] == ORD_MAX - 1) { vcmap[v] = cv; vcmap[u] = cv; }
            }
            for (O u : perm) if (vcmap[u] == ORD_MAX - 1) vcmap[u] = ORD_MAX;
        }
        outer++;
        for (O u : perm) {
            if (vcmap[u] != ORD_MAX || hn[u] == ORD_MAX || vcmap[hn[u]] == ORD_MAX) continue;
            uint32_t r = (uint32_t)jet_rng(seed, rng_stream(level, RNG_MATCH_PICK, outer), (uint64_t)u);
            hn[u] = pick_match(g, vcmap, false, uniform, r, u);
        }
        next.clear();
        for (O u : perm) if (vcmap[u] == ORD_MAX && hn[u] != ORD_MAX) next.push_back(u);
        perm.swap(next);
    }
    if (two_hop) {
        auto count_unmatched = [&]() { O c = 0; for (O i = 0; i < n; i++) c += (vcmap[i] == ORD_MAX); return c; };
        O unmapped = count_unmatched();
        // leaves, src/heuristics.hpp:539-560
        if ((double)unmapped / (double)n > 0.25) {
            std::vector<O> list; std::vector<O> hs;
            for (O i = 0; i < n; i++)
                if (vcmap[i] == ORD_MAX && g.row[i + 1] - g.row[i] == 1) { list.push_back(i); hs.push_back(g.adj[g.row[i]]); }
            match_hash<O, O>(list, hs, ORD_MAX, vcmap);
        }
        unmapped = count_unmatched();
        // twins, src/heuristics.hpp:565-598
        if ((double)unmapped / (double)n > 0.25) {
            std::vector<O> list; std::vector<uint64_t> hs;
            for (O i = 0; i < n; i++) {
                if (vcmap[i] != ORD_MAX) continue;
                uint64_t h = 0;
                for (E j = g.row[i]; j < g.row[i + 1]; j++) {
                    uint64_t y = pod_hash<O>(g.adj[j]);
                    y = y * y + y;
                    h += y;
                }
                list.push_back(i); hs.push_back(h);
            }
            match_hash<O, uint64_t>(list, hs, 0, vcmap);
        }
        unmapped = count_unmatched();
        // relatives, src/heuristics.hpp:603-640
        if ((double)unmapped / (double)n > 0.25) {
            std::vector<O> list; std::vector<O> hs;
            for (O i = 0; i < n; i++) {
                if (vcmap[i] != ORD_MAX) continue;
                O h = ORD_MAX; W max_wgt = 0; O min_deg = ORD_MAX;
                for (E j = g.row[i]; j < g.row[i + 1]; j++) {
                    O v = g.adj[j];
                    O vdeg = (O)(g.row[v + 1] - g.row[v]);
                    if (min_deg > vdeg) { min_deg = vdeg; max_wgt = g.val[j]; h = v; }
                    else if (min_deg == vdeg && max_wgt < g.val[j]) { h = v; max_wgt = g.val[j]; }
                }
                list.push_back(i); hs.push_back(h);
            }
            match_hash<O, O>(list, hs, ORD_MAX, vcmap);
        }
    }
    for (O i = 0; i < n; i++) if (vcmap[i] == ORD_MAX) vcmap[i] = i;
    return number_roots<O>(n, vcmap);
}

template <class O, class E, class W>
O coarsen_hec(const Csr<O, E, W>& g, const W* vw, bool uniform, uint64_t seed, int level, O* vcmap, O* hn_out) {
    std::vector<O> hn(g.n);
    hec_propose(g, vw, uniform, seed, level, hn.data());
    if (hn_out) std::copy(hn.begin(), hn.end(), hn_out);
    hec_aggregate<O, E, W>(g.n, hn.data(), vcmap);
    return number_roots<O>(g.n, vcmap);
}

// Contraction, src/contract.hpp:347-446: coarse vertex weights are sums of
// member weights; each coarse row holds the distinct coarse neighbours other
// than itself with summed edge weights.  Rows are emitted sorted.
template <class O, class E, class W>
void contract(const Csr<O, E, W>& g, const W* vw, const O* map, O nc, Csr<O, E, W>& c, std::vector<W>& cvw) {
    O n = g.n;
    cvw.assign(nc, 0);
    for (O i = 0; i < n; i++) cvw[map[i]] += vw[i];
    std::vector<O> cnt(nc + 1, 0);
    for (O i = 0; i < n; i++) cnt[map[i] + 1]++;
    for (O x = 0; x < nc; x++) cnt[x + 1] += cnt[x];
    std::vector<O> members(n);
    {
        std::vector<O> pos(cnt.begin(), cnt.end() - 1);
        for (O i = 0; i < n; i++) members[pos[map[i]]++] = i;
    }
    std::vector<W> acc(nc, 0);
    std::vector<char> seen(nc, 0);
    std::vector<O> keys;
    c.n = nc;
    c.row.assign(nc + 1, 0);
    c.adj.clear(); c.val.clear();
    for (O x = 0; x < nc; x++) {
        keys.clear();
        for (O m = cnt[x]; m < cnt[x + 1]; m++) {
            O i = members[m];
            for (E j = g.row[i]; j < g.row[i + 1]; j++) {
                O u = map[g.adj[j]];
                if (u == x) continue;
                if (!seen[u]) { seen[u] = 1; keys.push_back(u); }
                acc[u] += g.val[j];
            }
        }
        std::sort(keys.begin(), keys.end());
        for (O u : keys) { c.adj.push_back(u); c.val.push_back(acc[u]); acc[u] = 0; seen[u] = 0; }
        c.row[x + 1] = (E)c.adj.size();
    }
}

// ---------------------------------------------------------------- refinement
template <class O, class E, class W>
struct Conn {
    std::vector<E> off;        // n+1, capacity min(deg,k) per vertex
    std::vector<part_t> ent;   // C
    std::vector<W> val;        // C
    std::vector<part_t> size;  // current table size
    std::vector<part_t> dest_cache;
    std::vector<O> lock;
};

// Table sizing rule shared by both reference builders
// (src/jet_refiner.hpp:1008-1013 and :701-705).
static inline part_t shrunk_size(part_t used, part_t cap) {
    part_t q = used / 4;
    if (q < 3) q = 3;
    part_t s = used + q;
    return s < cap ? s : cap;
}

// Builds one vertex's table at the final size, inserting distinct parts in
// order of first occurrence with linear probing from p % size.
template <class O, class E, class W>
void build_row(const Csr<O, E, W>& g, const part_t* part, part_t k, Conn<O, E, W>& cd, O i,
               std::vector<W>& scratch_w, std::vector<char>& mark, std::vector<part_t>& order) {
    E s = cd.off[i];
    part_t cap = (part_t)(cd.off[i + 1] - s);
    for (part_t j = 0; j < cap; j++) { cd.ent[s + j] = NULL_PART; cd.val[s + j] = 0; }
    order.clear();
    for (E j = g.row[i]; j < g.row[i + 1]; j++) {
        part_t p = part[g.adj[j]];
        if (!mark[p]) { mark[p] = 1; order.push_back(p); }
        scratch_w[p] += g.val[j];
    }
    part_t used = (part_t)order.size();
    part_t size = cap == 0 ? 0 : shrunk_size(used, cap);
    for (part_t p : order) {
        part_t po = p % size;
        if (size < k) while (cd.ent[s + po] != NULL_PART) po = (po + 1) % size;
        cd.ent[s + po] = p;
        cd.val[s + po] = scratch_w[p];
        scratch_w[p] = 0;
        mark[p] = 0;
    }
    cd.size[i] = size;
}

// init_conn_data, src/jet_refiner.hpp:958-1048.
template <class O, class E, class W>
void init_conn(const Csr<O, E, W>& g, const part_t* part, part_t k, Conn<O, E, W>& cd) {
    O n = g.n;
    cd.off.assign(n + 1, 0);
    for (O i = 0; i < n; i++) {
        E deg = g.row[i + 1] - g.row[i];
        cd.off[i + 1] = cd.off[i] + (deg > (E)k ? (E)k : deg);
    }
    cd.ent.assign(cd.off[n], NULL_PART);
    cd.val.assign(cd.off[n], 0);
    cd.size.assign(n, 0);
    cd.dest_cache.assign(n, NULL_PART);
    cd.lock.assign(n, 0);
    std::vector<W> sw(k, 0);
    std::vector<char> mark(k, 0);
    std::vector<part_t> order;
    for (O i = 0; i < n; i++) build_row(g, part, k, cd, i, sw, mark, order);
}

// src/jet_refiner.hpp:891-901
template <class W>
W lookup(const part_t* keys, const W* vals, part_t target, part_t size) {
    for (part_t q = 0; q < size; q++) {
        part_t pi = (target + q) % size;
        if (keys[pi] == target) return vals[pi];
        if (keys[pi] == NULL_PART) return 0;
    }
    return 0;
}

template <class O, class E, class W>
struct Problem {
    const Csr<O, E, W>* g;
    const W* vw;
    part_t k;
    double imb;
    O opt;
    O size_max;
};

template <class O, class E, class W>
struct State {
    std::vector<W> sizes;
    W total_size = 0;
    W cut = 0;
    W total_imb = 0;
    bool init = false;
};

template <class O, class W>
struct Scratch {
    std::vector<W> gain1, gain2, gain_persistent, evict_start, evict_end;
    std::vector<O> vtx1, vtx2;
    std::vector<part_t> dest, undersized;
};

// jet_lp, src/jet_refiner.hpp:200-323.  Returns the list of moves.
template <class O, class E, class W>
std::vector<O> jet_lp(const Problem<O, E, W>& pb, const part_t* part, Conn<O, E, W>& cd, Scratch<O, W>& sc, double filter_ratio) {
    const Csr<O, E, W>& g = *pb.g;
    O n = g.n;
    const W GAIN_MIN = std::numeric_limits<W>::lowest();
    std::vector<W>& save = sc.gain_persistent;
    for (O i = 0; i < n; i++) {
        part_t best = cd.dest_cache[i];
        if (best != NULL_PART) { sc.dest[i] = best; continue; }
        part_t p = part[i];
        best = NO_MOVE;
        W b_conn = 0, p_conn = 0;
        E s = cd.off[i];
        for (E j = s; j < s + cd.size[i]; j++) {
            W c = cd.val[j];
            part_t e = cd.ent[j];
            if (e != p && c > 0 && (c > b_conn || (c == b_conn && e < best))) { best = e; b_conn = c; }
            else if (c > 0 && e == p) p_conn = c;
        }
        save[i] = 0;
        if (best != NO_MOVE) {
            if (b_conn >= p_conn || ((double)(p_conn - b_conn) < std::floor(filter_ratio * (double)p_conn)))
                save[i] = b_conn - p_conn;
            else
                best = NO_MOVE;
        }
        cd.dest_cache[i] = best;
        sc.dest[i] = best;
    }
    std::vector<W>& pregain = sc.gain1;
    std::vector<O> cand;
    for (O i = 0; i < n; i++) {
        if (sc.dest[i] != NO_MOVE && cd.lock[i] == 0) { cand.push_back(i); pregain[i] = save[i]; }
        else { pregain[i] = GAIN_MIN; cd.lock[i] = 0; }
    }
    for (O i : cand) {
        W change = 0;
        part_t best = sc.dest[i], p = part[i];
        W igain = pregain[i];
        for (E j = g.row[i]; j < g.row[i + 1]; j++) {
            O v = g.adj[j];
            W vgain = pregain[v];
            if (vgain > igain || (vgain == igain && v < i)) {
                part_t vp = sc.dest[v];
                W w = g.val[j];
                if (vp == p) change -= w; else if (vp == best) change += w;
                vp = part[v];
                if (vp == p) change += w; else if (vp == best) change -= w;
            }
        }
        if (igain + change >= 0) cd.lock[i] = 1;
    }
    std::vector<O> moves;
    for (O i : cand) if (cd.lock[i]) moves.push_back(i);
    return moves;
}

// src/jet_refiner.hpp:326-356.  C++ float/double semantics kept as written:
// "gain *= 1.5" multiplies in double and rounds back to float.
template <class W>
int gain_bucket(W gx, W vwgt) {
    float gain = (float)gx / (float)vwgt;
    int t = 0;
    if (gain > 0.0) t = 0;
    else if (gain == 0.0) t = 1;
    else {
        t = MID_BUCKET;
        gain = std::fabs(gain);
        if (gain < 1.0) {
            while (gain < 1.0) { gain *= 1.5; t--; }
            if (t < 2) t = 2;
        } else {
            while (gain > 1.0) { gain /= 1.5; t++; }
            if (t > MAX_BUCKETS) t = MAX_BUCKETS - 1;
        }
    }
    return t;
}

template <class O>
static void sections_for(O n, part_t k, O& sections) {
    sections = MAX_SECTIONS;
    O section_size = (n + sections * k) / (sections * k);
    if (section_size < 4096) {
        section_size = 4096;
        sections = (n + section_size * k) / (section_size * k);
    }
}

// get_evictions, src/jet_refiner.hpp:358-412.  buckets holds t_minibuckets+1
// sizes and is turned into exclusive offsets in place.
template <bool adjust, class O, class E, class W>
std::vector<O> get_evictions(const Problem<O, E, W>& pb, const part_t* part, Scratch<O, W>& sc, const std::vector<W>& sizes,
                             std::vector<W>& buckets, O t_minibuckets, O width, W size_max,
                             const std::vector<O>& bid, const std::vector<W>& score_in, std::vector<W>& evict_adjust) {
    W acc = 0;
    for (O i = 0; i <= t_minibuckets; i++) { W x = buckets[i]; buckets[i] = acc; acc += x; }
    if (adjust) std::fill(evict_adjust.begin(), evict_adjust.end(), 0);
    std::vector<O> moves;
    for (O i = 0; i < pb.g->n; i++) {
        O b = bid[i];
        if (b == -1) continue;
        part_t p = part[i];
        O begin = p * width;
        W score = score_in[i] + buckets[b] - buckets[begin];
        W limit = sizes[p] - size_max;
        if (score < limit) {
            if (adjust && score + pb.vw[i] >= limit) evict_adjust[p] = score + pb.vw[i];
            moves.push_back(i);
        }
    }
    return moves;
}

// rebalance_weak, src/jet_refiner.hpp:551-645.
template <class O, class E, class W>
std::vector<O> rebalance_weak(const Problem<O, E, W>& pb, const part_t* part, Conn<O, E, W>& cd, Scratch<O, W>& sc, const std::vector<W>& sizes) {
    const Csr<O, E, W>& g = *pb.g;
    part_t k = pb.k;
    W opt = pb.opt;
    O n = g.n;
    O sections; sections_for<O>(n, k, sections);
    O t_minibuckets = MAX_BUCKETS * k * sections;
    // + MAX_BUCKETS*sections slack: a gain_type of exactly 50 indexes past the
    // part's own range, as it does in the reference.
    std::vector<W> buckets(t_minibuckets + 1 + MAX_BUCKETS * sections, 0);
    W size_max = pb.size_max;
    W max_dest = (W)(size_max * 0.99);
    if (max_dest < size_max - 100) max_dest = size_max - 100;
    std::vector<part_t> undersized;
    for (part_t p = 0; p < k; p++) if (sizes[p] < max_dest) undersized.push_back(p);
    part_t total_undersized = (part_t)undersized.size();
    std::vector<W>& save = sc.gain2;
    for (O i = 0; i < n; i++) {
        part_t p = part[i];
        W p_gain = 0, gain = 0;
        part_t best = p;
        if (sizes[p] > size_max && (double)pb.vw[i] < 1.5 * (double)(sizes[p] - opt)) {
            E s = cd.off[i];
            for (E j = s; j < s + cd.size[i]; j++) {
                part_t pj = cd.ent[j];
                if (pj > NULL_PART && sizes[pj] < max_dest) {
                    W jg = cd.val[j];
                    if (jg > gain || (jg == gain && jg > 0 && pj < best)) { best = pj; gain = jg; }
                }
                if (pj == p) p_gain = cd.val[j];
            }
            if (gain > 0) { sc.dest[i] = best; save[i] = gain - p_gain; }
            else if (total_undersized > 0) { sc.dest[i] = undersized[i % total_undersized]; save[i] = -p_gain; }
            else sc.dest[i] = p;
        } else {
            sc.dest[i] = p;
        }
    }
    std::vector<O> bid(n, -1);
    std::vector<W> score(n, 0);
    for (O i = 0; i < n; i++) {
        part_t p = part[i];
        if (p != sc.dest[i]) {
            int gt = gain_bucket<W>(save[i], pb.vw[i]);
            O gid = (MAX_BUCKETS * p + gt) * sections + (i % sections);
            bid[i] = gid;
            score[i] = buckets[gid];
            buckets[gid] += pb.vw[i];
        }
    }
    std::vector<W> dummy;
    return get_evictions<false>(pb, part, sc, sizes, buckets, t_minibuckets, (O)(MAX_BUCKETS * sections), size_max, bid, score, dummy);
}

// rebalance_strong, src/jet_refiner.hpp:417-546.
template <class O, class E, class W>
std::vector<O> rebalance_strong(const Problem<O, E, W>& pb, const part_t* part, Conn<O, E, W>& cd, Scratch<O, W>& sc, const std::vector<W>& sizes) {
    const Csr<O, E, W>& g = *pb.g;
    part_t k = pb.k;
    W opt = pb.opt;
    O n = g.n;
    const W GAIN_MIN = std::numeric_limits<W>::lowest();
    O sections; sections_for<O>(n, k, sections);
    O t_minibuckets = MAX_BUCKETS * k * sections;
    std::vector<W> buckets(t_minibuckets + 1 + MAX_BUCKETS * sections, 0);
    W size_max = pb.size_max;
    W max_dest = std::max<W>(opt + 1, (W)(pb.size_max * 0.99));
    bool any = false; W max_vwgt = GAIN_MIN;
    for (part_t p = 0; p < k; p++) {
        if (sizes[p] < max_dest) {
            W cap = max_dest - sizes[p];
            if (!any || cap > max_vwgt) max_vwgt = cap;
            any = true;
        }
    }
    std::vector<O> bid(n, -1);
    std::vector<W> save(n, 0);
    for (O i = 0; i < n; i++) {
        part_t p = part[i];
        W w = pb.vw[i];
        if (sizes[p] > size_max && any && w <= 2 * max_vwgt && w < 2 * (sizes[p] - opt)) {
            uint64_t tk = 0, tg = 0;
            W p_gain = 0;
            E s = cd.off[i];
            for (E j = s; j < s + cd.size[i]; j++) {
                part_t pj = cd.ent[j];
                if (pj == p) p_gain = cd.val[j];
                else if (pj > NULL_PART && sizes[pj] < max_dest) { tg += (uint64_t)cd.val[j]; tk += 1; }
            }
            if (tk == 0) tk = 1;
            W gain = (W)((tg / tk) - (uint64_t)p_gain);
            W lim = sizes[p] - size_max;
            int gt = gain_bucket<W>(gain, w < lim ? w : lim);
            if (gt < MAX_BUCKETS) {
                O gid = (MAX_BUCKETS * p + gt) * sections + (i % sections) + 1;
                bid[i] = gid;
                save[i] = buckets[gid];
                buckets[gid] += w;
            }
        }
    }
    std::vector<W> evict_adjust(k, 0);
    O width = MAX_BUCKETS * sections;
    std::vector<O> moves = get_evictions<true>(pb, part, sc, sizes, buckets, t_minibuckets, width, size_max, bid, save, evict_adjust);
    // cookie cutter, src/jet_refiner.hpp:491-518
    W upd = 0;
    for (part_t p = 0; p < k; p++) {
        W add = evict_adjust[p];
        O begin = MAX_BUCKETS * p * sections;
        if (add == 0) add = buckets[begin + width] - buckets[begin];
        evict_adjust[p] = buckets[begin] - upd;
        upd += add;
    }
    W vw_cursor = upd;
    std::vector<W> evict_start(k + 1, 0);
    W acc = 0;
    for (part_t p = 0; p < k; p++) {
        if (max_dest > sizes[p]) acc += max_dest - sizes[p];
        evict_start[p + 1] = acc;
    }
    for (O v : moves) save[v] = save[v] + buckets[bid[v]] - evict_adjust[part[v]];
    // select destination parts (rs), src/jet_refiner.hpp:526-544
    for (O v : moves) {
        int p = 0;
        bool done = false;
        while (p < k) {
            while (p <= k && evict_start[p] <= save[v]) p++;
            p--;
            if (p < k && pb.vw[v] / 2 <= evict_start[p + 1] - save[v]) { sc.dest[v] = p; done = true; break; }
            else if (p < k) { save[v] = vw_cursor; vw_cursor += pb.vw[v]; }
        }
        if (!done) sc.dest[v] = part[v];
    }
    return moves;
}

// update_small, src/jet_refiner.hpp:781-888.  Returns false on a corrupt table.
template <class O, class E, class W>
bool update_small(const Problem<O, E, W>& pb, const part_t* part, const std::vector<O>& moves, const std::vector<part_t>& dest, Conn<O, E, W>& cd) {
    const Csr<O, E, W>& g = *pb.g;
    part_t k = pb.k;
    for (O i : moves) {
        part_t p = dest[i];
        for (E j = g.row[i]; j < g.row[i + 1]; j++) {
            O v = g.adj[j];
            W w = g.val[j];
            E vs = cd.off[v];
            part_t vsize = cd.size[v];
            part_t po = p % vsize;
            part_t guard = 0;
            while (cd.ent[vs + po] != p) { po = (po + 1) % vsize; if (++guard > vsize) return false; }
            W x = cd.val[vs + po];
            cd.val[vs + po] -= w;
            if (vsize < k && x == w) cd.ent[vs + po] = HASH_RECLAIM;
        }
    }
    for (O i : moves) {
        part_t best = part[i];
        for (E j = g.row[i]; j < g.row[i + 1]; j++) {
            O v = g.adj[j];
            W w = g.val[j];
            cd.dest_cache[v] = NULL_PART;
            E vs = cd.off[v];
            part_t vsize = cd.size[v];
            part_t po = best % vsize;
            bool success = false;
            for (part_t q = 0; q < vsize; q++) {
                part_t pi = (best + q) % vsize;
                if (cd.ent[vs + pi] == best) { success = true; po = pi; break; }
                else if (cd.ent[vs + pi] == NULL_PART) break;
            }
            part_t count = 0;
            while (!success && count < vsize) {
                part_t px = cd.ent[vs + po];
                while (px != best && px > NULL_PART && count++ < vsize) {
                    po = (po + 1) % vsize;
                    px = cd.ent[vs + po];
                }
                if (px == best) success = true;
                else if (px <= NULL_PART) { cd.ent[vs + po] = best; success = true; }
            }
            if (!success) {
                po = vsize;
                E cap = cd.off[v + 1] - vs;
                while (true) {
                    if ((E)po >= cap) return false;
                    part_t px = cd.ent[vs + po];
                    if (px == best) break;
                    if (px <= NULL_PART) { cd.ent[vs + po] = best; cd.size[v] += 1; break; }
                    po++;
                }
            }
            cd.val[vs + po] += w;
        }
    }
    return true;
}

// update_large, src/jet_refiner.hpp:743-777.
template <class O, class E, class W>
void update_large(const Problem<O, E, W>& pb, const part_t* part, const std::vector<O>& moves, Conn<O, E, W>& cd) {
    const Csr<O, E, W>& g = *pb.g;
    std::vector<char> mark(g.n, 0);
    for (O i : moves) for (E j = g.row[i]; j < g.row[i + 1]; j++) mark[g.adj[j]] = 1;
    std::vector<W> sw(pb.k, 0);
    std::vector<char> pmark(pb.k, 0);
    std::vector<part_t> order;
    for (O i = 0; i < g.n; i++) {
        if (!mark[i]) continue;
        build_row(g, part, pb.k, cd, i, sw, pmark, order);
        cd.dest_cache[i] = NULL_PART;
    }
}

// perform_moves, src/jet_refiner.hpp:905-955.
template <class O, class E, class W>
bool perform_moves(const Problem<O, E, W>& pb, part_t* part, const std::vector<O>& moves, Scratch<O, W>& sc, Conn<O, E, W>& cd, State<O, E, W>& st) {
    const Csr<O, E, W>& g = *pb.g;
    W c1 = 0;
    for (O i : moves) {
        E s = cd.off[i];
        W pc = lookup<W>(&cd.ent[s], &cd.val[s], part[i], cd.size[i]);
        W bc = lookup<W>(&cd.ent[s], &cd.val[s], sc.dest[i], cd.size[i]);
        c1 += bc - pc;
    }
    for (O i : moves) {
        part_t p = part[i], best = sc.dest[i];
        cd.dest_cache[i] = NULL_PART;
        st.sizes[p] -= pb.vw[i];
        st.sizes[best] += pb.vw[i];
        part[i] = best;
        sc.dest[i] = p;
    }
    bool ok = true;
    if ((O)moves.size() > (O)(g.n / 10)) update_large(pb, part, moves, cd);
    else ok = update_small(pb, part, moves, sc.dest, cd);
    W c2 = 0;
    for (O i : moves) {
        E s = cd.off[i];
        W pc = lookup<W>(&cd.ent[s], &cd.val[s], sc.dest[i], cd.size[i]);
        W bc = lookup<W>(&cd.ent[s], &cd.val[s], part[i], cd.size[i]);
        c2 += bc - pc;
    }
    W mx = std::numeric_limits<W>::lowest();
    for (W s : st.sizes) if (s > mx) mx = s;
    st.total_imb = mx > pb.opt ? mx - pb.opt : 0;
    st.cut -= c1 + c2;
    return ok;
}

struct LevelRecord {
    int64_t cut_half, nnz, n;
    double imb;
    int32_t iters, lp_iters;
};

template <class O, class E, class W>
struct Refiner {
    Scratch<O, W> sc;
    Conn<O, E, W> cd;
    int iter_log_cap = 0;
    explicit Refiner(O n_max, part_t k) {
        sc.gain1.assign(std::max<O>(n_max, (O)(k * MAX_SECTIONS * MAX_BUCKETS)), 0);
        sc.gain2.assign(n_max, 0);
        sc.gain_persistent.assign(n_max, 0);
        sc.vtx1.assign(n_max, 0);
        sc.vtx2.assign(std::max<O>(n_max, (O)(k * MAX_SECTIONS * MAX_BUCKETS)), 0);
        sc.dest.assign(n_max, 0);
    }

    // jet_refine, src/jet_refiner.hpp:1050-1142.  best_part is in/out.
    bool refine(const Csr<O, E, W>& g, const W* vw, part_t k, double imb_ratio, double tol, bool ultra,
                bool uniform_ew, part_t* best_part, State<O, E, W>& best, LevelRecord* rec, bool verbose) {
        if (!best.init) {
            best.cut = total_cut(g, best_part);
            best.sizes = part_sizes(g, vw, best_part, k);
            best.total_size = 0;
            for (O i = 0; i < g.n; i++) best.total_size += vw[i];
        }
        Problem<O, E, W> pb;
        pb.g = &g; pb.vw = vw; pb.k = k; pb.imb = imb_ratio;
        pb.opt = optimal_size<O>((O)best.total_size, k);
        pb.size_max = (O)(pb.opt * imb_ratio);
        if (!best.init) {
            best.init = true;
            W mx = 0;
            for (W s : best.sizes) if (s > mx) mx = s;
            best.total_imb = mx > pb.opt ? mx - pb.opt : 0;
            if (verbose)
                printf("Initial %lld %.6f %lld\n", (long long)(best.cut / 2),
                       (double)best.total_imb / (double)pb.opt, (long long)g.n);
        }
        State<O, E, W> curr = best;
        W imb_max = (W)pb.size_max - (W)pb.opt;
        std::vector<part_t> part(best_part, best_part + g.n);
        init_conn(g, part.data(), k, cd);
        int iter_count = 0, balance_counter = 0, lab_counter = 0;
        std::vector<double> temps;
        if (ultra) { for (double t = 0.85; t > 0; t -= 0.05) temps.push_back(t); }
        else if (uniform_ew) temps.push_back(0.25);
        else temps.push_back(0.75);
        bool ok = true;
        for (double fr : temps) {
            int count = 0;
            while (count++ <= 11) {
                iter_count++;
                std::vector<O> moves;
                if (curr.total_imb <= imb_max) {
                    moves = jet_lp(pb, part.data(), cd, sc, fr);
                    balance_counter = 0;
                    lab_counter++;
                } else {
                    if (balance_counter < 2) moves = rebalance_weak(pb, part.data(), cd, sc, curr.sizes);
                    else moves = rebalance_strong(pb, part.data(), cd, sc, curr.sizes);
                    balance_counter++;
                }
                ok = perform_moves(pb, part.data(), moves, sc, cd, curr) && ok;
                if (best.total_imb > imb_max && curr.total_imb < best.total_imb) {
                    best = curr;
                    std::copy(part.begin(), part.end(), best_part);
                    count = 0;
                } else if (curr.cut < best.cut && (curr.total_imb <= imb_max || curr.total_imb <= best.total_imb)) {
                    if ((double)curr.cut < tol * (double)best.cut) count = 0;
                    best = curr;
                    std::copy(part.begin(), part.end(), best_part);
                }
            }
        }
        if (rec) {
            rec->cut_half = (int64_t)(best.cut / 2);
            rec->imb = (double)best.total_imb / (double)pb.opt;
            rec->nnz = (int64_t)g.nnz();
            rec->n = (int64_t)g.n;
            rec->iters = iter_count;
            rec->lp_iters = lab_counter;
        }
        return ok;
    }
};

// metis_init, src/initial_partition.hpp:92-114: values go through `int`
// as in the reference, then widen to this Metis build's 64-bit idx_t.
template <class O, class E, class W>
int metis_init(const Csr<O, E, W>& g, const W* vw, part_t k, double imb, part_t* part) {
    metis_idx_t n = g.n, ncon = 1, nparts = k, obj = 0;
    std::vector<metis_idx_t> xadj(g.n + 1), adj(g.nnz()), adjw(g.nnz()), vwg(g.n), pm(g.n, 0);
    for (O i = 0; i <= g.n; i++) xadj[i] = (int)g.row[i];
    for (E j = 0; j < g.nnz(); j++) { adj[j] = (int)g.adj[j]; adjw[j] = (int)g.val[j]; }
    for (O i = 0; i < g.n; i++) vwg[i] = (int)vw[i];
    metis_real_t ub = (metis_real_t)imb;
    int ret = METIS_PartGraphKway(&n, &ncon, xadj.data(), adj.data(), vwg.data(), nullptr, adjw.data(),
                                  &nparts, nullptr, &ub, nullptr, &obj, pm.data());
    if (ret != 1) return -1;
    for (O i = 0; i < g.n; i++) part[i] = (part_t)pm[i];
    return 0;
}

}  // namespace orc

// ================================================================ C interface
extern "C" {

typedef struct orc_config {
    int32_t coarsening_alg;
    int32_t num_parts;
    double max_imb_ratio;
    double refine_tolerance;
    int32_t ultra_settings;
    int32_t verbose;
} orc_config;

typedef struct orc_stats {
    int64_t cut;           // final edge cut (each cut edge once)
    int64_t largest, smallest;
    double imb;            // largest / optimal
    int32_t levels;
    int32_t coarsest_n;
    double t_coarsen, t_init, t_refine, t_total;
    int64_t level_cut[256];
    int64_t level_n[256];
    int64_t level_nnz[256];
    int32_t level_iters[256];
    int32_t level_lp_iters[256];
} orc_stats;

}

namespace {

using clk = std::chrono::steady_clock;
static double secs(clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); }

template <class O, class E, class W>
orc::Csr<O, E, W> make_csr(int64_t n, const void* row, const void* adj, const void* val) {
    orc::Csr<O, E, W> g;
    g.n = (O)n;
    const E* r = (const E*)row;
    g.row.assign(r, r + n + 1);
    g.adj.assign((const O*)adj, (const O*)adj + g.row[n]);
    g.val.assign((const W*)val, (const W*)val + g.row[n]);
    return g;
}

// uncoarsener::multilevel_jet (src/uncoarsen.hpp:88-125): refine each level,
// coarsest first, then project onto the next finer level.  `part` holds the
// coarsest level's partition on entry and the finest level's on exit.
template <class O, class E, class W>
bool uncoarsen_levels(const std::vector<orc::Level<O, E, W>>& levels, const orc_config* cfg,
                      std::vector<orc::part_t>& part, orc::State<O, E, W>& best, orc_stats* st) {
    using namespace orc;
    part_t k = cfg->num_parts;
    Refiner<O, E, W> ref(levels[0].g.n, k);
    int nl = (int)levels.size();
    bool ok = true;
    for (int l = nl - 1; l >= 0; l--) {
        LevelRecord rec;
        ok = ref.refine(levels[l].g, levels[l].vw.data(), k, cfg->max_imb_ratio, cfg->refine_tolerance,
                        cfg->ultra_settings != 0, levels[l].uniform, part.data(), best, &rec, cfg->verbose != 0) && ok;
        if (st && nl - 1 - l < 256) {
            int idx = nl - 1 - l;
            st->level_cut[idx] = rec.cut_half; st->level_n[idx] = rec.n; st->level_nnz[idx] = rec.nnz;
            st->level_iters[idx] = rec.iters; st->level_lp_iters[idx] = rec.lp_iters;
        }
        if (l > 0) {
            const std::vector<O>& map = levels[l].map;
            std::vector<part_t> fine(levels[l - 1].g.n);
            for (size_t i = 0; i < fine.size(); i++) fine[i] = part[map[i]];
            part.swap(fine);
        }
    }
    return ok;
}

// partitioner::partition, src/partitioner.hpp:61-125, with contracter::
// generate_coarse_graphs (src/contract.hpp:494-533) and uncoarsener::
// uncoarsen (src/uncoarsen.hpp:88-158).
template <class O, class E, class W>
int run_partition(const orc_config* cfg, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
                  int uniform_ew, uint64_t seed, int32_t* part_out, int64_t* cut_out, orc_stats* st) {
    using namespace orc;
    auto t0 = clk::now();
    part_t k = cfg->num_parts;
    std::vector<Level<O, E, W>> levels(1);
    levels[0].g = make_csr<O, E, W>(n, row, adj, val);
    levels[0].vw.assign((const W*)vw, (const W*)vw + n);
    levels[0].uniform = uniform_ew != 0;
    int cutoff = k * 8;
    if (cutoff > 1024) { cutoff = k * 2; cutoff = std::max(1024, cutoff); }
    O min_allowed = cutoff / 4;
    int alg = cfg->coarsening_alg;
    if (alg < 0 || alg > 2) alg = 0;
    while (levels.back().g.n > (O)cutoff) {
        Level<O, E, W>& cur = levels.back();
        int lvl = (int)levels.size();
        std::vector<O> map(cur.g.n);
        O nc;
        if (alg == 1) nc = coarsen_hec(cur.g, cur.vw.data(), cur.uniform, seed, lvl, map.data(), (O*)nullptr);
        else nc = coarsen_match(cur.g, cur.uniform, alg == 0, seed, lvl, map.data(), (O*)nullptr);
        if (nc < min_allowed) break;
        Level<O, E, W> next;
        contract(cur.g, cur.vw.data(), map.data(), nc, next.g, next.vw);
        next.map.swap(map);
        next.uniform = false;
        levels.push_back(std::move(next));
        if (levels.size() > 200) break;
    }
    auto t1 = clk::now();
    Level<O, E, W>& coarsest = levels.back();
    std::vector<part_t> part(coarsest.g.n, 0);
    if (metis_init(coarsest.g, coarsest.vw.data(), k, cfg->max_imb_ratio, part.data()) != 0) return 3;
    auto t2 = clk::now();
    State<O, E, W> best;
    bool ok = uncoarsen_levels(levels, cfg, part, best, st);
    auto t3 = clk::now();
    std::copy(part.begin(), part.end(), part_out);
    *cut_out = (int64_t)(best.cut / 2);
    if (st) {
        W largest = 0, smallest = best.total_size;
        for (W s : best.sizes) { largest = std::max(largest, s); smallest = std::min(smallest, s); }
        st->cut = (int64_t)(best.cut / 2);
        st->largest = (int64_t)largest;
        st->smallest = (int64_t)smallest;
        st->imb = (double)largest / (double)optimal_size<O>((O)best.total_size, k);
        st->levels = (int32_t)levels.size();
        st->coarsest_n = (int32_t)coarsest.g.n;
        st->t_coarsen = secs(t0, t1); st->t_init = secs(t1, t2); st->t_refine = secs(t2, t3); st->t_total = secs(t0, t3);
    }
    return ok ? 0 : 4;
}

}  // namespace

#define ORC_TIER_DISPATCH(tier, ...)                                   \
    switch (tier) {                                                    \
        case 0: { typedef int32_t O; typedef int32_t E; typedef int32_t W; __VA_ARGS__; } \
        case 1: { typedef int32_t O; typedef int64_t E; typedef int64_t W; __VA_ARGS__; } \
        case 2: { typedef int64_t O; typedef int64_t E; typedef int64_t W; __VA_ARGS__; } \
        default: return 1;                                             \
    }

extern "C" {

// Full partition of one graph (tier 0: int32 everywhere; 1: int64 offsets and
// weights; 2: also int64 ordinals).  Returns 0 on success, 3 on Metis failure,
// 4 on a corrupt connectivity table.
int orc_partition(int tier, const orc_config* cfg, int64_t n, const void* row, const void* adj, const void* val,
                  const void* vw, int uniform_ew, uint64_t seed, int32_t* part_out, int64_t* cut_out, orc_stats* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    ORC_TIER_DISPATCH(tier, return (run_partition<O, E, W>(cfg, n, row, adj, val, vw, uniform_ew, seed, part_out, cut_out, st)));
}

// One coarsening map: alg 0 = 2-hop matching, 1 = HEC, 2 = plain matching.
// hn_out (nullable) receives the initial heavy-neighbour proposals.
int orc_coarsen(int tier, int alg, int level, uint64_t seed, int64_t n, const void* row, const void* adj, const void* val,
                const void* vw, int uniform, void* map_out, void* hn_out, int64_t* nc_out) {
    ORC_TIER_DISPATCH(tier, {
        auto g = make_csr<O, E, W>(n, row, adj, val);
        O nc;
        if (alg == 1) nc = orc::coarsen_hec(g, (const W*)vw, uniform != 0, seed, level, (O*)map_out, (O*)hn_out);
        else nc = orc::coarsen_match(g, uniform != 0, alg == 0, seed, level, (O*)map_out, (O*)hn_out);
        *nc_out = (int64_t)nc;
        return 0;
    });
}

// Contraction of a graph under a given map.  Output arrays must hold nc+1,
// nnz(g) and nnz(g) entries; rows come out sorted.
int orc_contract(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
                 const void* map, int64_t nc, void* crow, void* cadj, void* cval, void* cvw, int64_t* cnnz) {
    ORC_TIER_DISPATCH(tier, {
        auto g = make_csr<O, E, W>(n, row, adj, val);
        orc::Csr<O, E, W> c; std::vector<W> w;
        orc::contract(g, (const W*)vw, (const O*)map, (O)nc, c, w);
        std::copy(c.row.begin(), c.row.end(), (E*)crow);
        std::copy(c.adj.begin(), c.adj.end(), (O*)cadj);
        std::copy(c.val.begin(), c.val.end(), (W*)cval);
        std::copy(w.begin(), w.end(), (W*)cvw);
        *cnnz = (int64_t)c.nnz();
        return 0;
    });
}

// Connectivity tables for a partition.  off_out: n+1; ent_out/val_out: C =
// off_out[n] (at most nnz); size_out: n.
int orc_conn_build(int tier, int64_t n, const void* row, const void* adj, const void* val, const int32_t* part, int k,
                   void* off_out, int32_t* ent_out, void* val_out, int32_t* size_out) {
    ORC_TIER_DISPATCH(tier, {
        auto g = make_csr<O, E, W>(n, row, adj, val);
        orc::Conn<O, E, W> cd;
        orc::init_conn(g, part, k, cd);
        std::copy(cd.off.begin(), cd.off.end(), (E*)off_out);
        std::copy(cd.ent.begin(), cd.ent.end(), ent_out);
        std::copy(cd.val.begin(), cd.val.end(), (W*)val_out);
        std::copy(cd.size.begin(), cd.size.end(), size_out);
        return 0;
    });
}

// Runs `iters` refinement iterations at one level from `part` (in/out)
// without the best-state bookkeeping: each iteration is LP when the current
// imbalance is within bounds, else weak (twice) then strong rebalancing --
// exactly the iteration body of jet_refine.  Outputs the final part sizes (k),
// cut (both directions), connectivity tables (as orc_conn_build) and per
// iteration the move count and kind (0 LP, 1 weak, 2 strong).
int orc_refine_iters(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
                     int32_t* part, int k, double imb, double filter_ratio, int iters, void* sizes_out, int64_t* cut_out,
                     void* off_out, int32_t* ent_out, void* cval_out, int32_t* size_out, int32_t* dest_cache_out,
                     int64_t* moves_out, int32_t* kind_out) {
    ORC_TIER_DISPATCH(tier, {
        auto g = make_csr<O, E, W>(n, row, adj, val);
        const W* w = (const W*)vw;
        orc::Refiner<O, E, W> ref((O)n, k);
        orc::State<O, E, W> st;
        st.cut = orc::total_cut(g, part);
        st.sizes = orc::part_sizes(g, w, part, k);
        for (O i = 0; i < g.n; i++) st.total_size += w[i];
        orc::Problem<O, E, W> pb;
        pb.g = &g; pb.vw = w; pb.k = k; pb.imb = imb;
        pb.opt = orc::optimal_size<O>((O)st.total_size, k);
        pb.size_max = (O)(pb.opt * imb);
        W mx = 0; for (W s : st.sizes) mx = std::max(mx, s);
        st.total_imb = mx > pb.opt ? mx - pb.opt : 0;
        W imb_max = (W)pb.size_max - (W)pb.opt;
        orc::init_conn(g, part, k, ref.cd);
        int bal = 0;
        bool ok = true;
        for (int it = 0; it < iters; it++) {
            std::vector<O> moves;
            int kind;
            if (st.total_imb <= imb_max) { moves = orc::jet_lp(pb, part, ref.cd, ref.sc, filter_ratio); bal = 0; kind = 0; }
            else if (bal < 2) { moves = orc::rebalance_weak(pb, part, ref.cd, ref.sc, st.sizes); bal++; kind = 1; }
            else { moves = orc::rebalance_strong(pb, part, ref.cd, ref.sc, st.sizes); bal++; kind = 2; }
            ok = orc::perform_moves(pb, part, moves, ref.sc, ref.cd, st) && ok;
            if (moves_out) moves_out[it] = (int64_t)moves.size();
            if (kind_out) kind_out[it] = kind;
        }
        std::copy(st.sizes.begin(), st.sizes.end(), (W*)sizes_out);
        *cut_out = (int64_t)st.cut;
        if (off_out) std::copy(ref.cd.off.begin(), ref.cd.off.end(), (E*)off_out);
        if (ent_out) std::copy(ref.cd.ent.begin(), ref.cd.ent.end(), ent_out);
        if (cval_out) std::copy(ref.cd.val.begin(), ref.cd.val.end(), (W*)cval_out);
        if (size_out) std::copy(ref.cd.size.begin(), ref.cd.size.end(), size_out);
        if (dest_cache_out) std::copy(ref.cd.dest_cache.begin(), ref.cd.dest_cache.end(), dest_cache_out);
        return ok ? 0 : 4;
    });
}

// One full jet_refine at a single level starting from `part` (in/out).
int orc_refine_level(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw,
                     int32_t* part, int k, double imb, double tol, int uniform_ew, int64_t* cut_out, int32_t* iters_out) {
    ORC_TIER_DISPATCH(tier, {
        auto g = make_csr<O, E, W>(n, row, adj, val);
        orc::Refiner<O, E, W> ref((O)n, k);
        orc::State<O, E, W> st;
        orc::LevelRecord rec;
        bool ok = ref.refine(g, (const W*)vw, k, imb, tol, false, uniform_ew != 0, part, st, &rec, false);
        *cut_out = (int64_t)st.cut;
        if (iters_out) *iters_out = rec.iters;
        return ok ? 0 : 4;
    });
}

// uncoarsener::uncoarsen (src/uncoarsen.hpp:127-158) over a fixed hierarchy,
// as the reference's jet_import app does (app/import_coarse.cpp:49-132).
// Level 0 is the finest; maps[l] (l >= 1) sends level l-1's vertices to level
// l.  coarsest_part has ns[nlevels-1] entries; part_out receives ns[0];
// *cut_out counts each cut edge once.
int orc_uncoarsen(int tier, int nlevels, const int64_t* ns, const void* const* rows, const void* const* adjs,
                  const void* const* vals, const void* const* vws, const void* const* maps,
                  const int32_t* coarsest_part, const orc_config* cfg, int uniform_finest, int32_t* part_out,
                  int64_t* cut_out) {
    ORC_TIER_DISPATCH(tier, {
        std::vector<orc::Level<O, E, W>> levels(nlevels);
        for (int l = 0; l < nlevels; l++) {
            levels[l].g = make_csr<O, E, W>(ns[l], rows[l], adjs[l], vals[l]);
            levels[l].vw.assign((const W*)vws[l], (const W*)vws[l] + ns[l]);
            levels[l].uniform = (l == 0) && uniform_finest;
            if (l > 0) levels[l].map.assign((const O*)maps[l], (const O*)maps[l] + ns[l - 1]);
        }
        std::vector<orc::part_t> part(coarsest_part, coarsest_part + ns[nlevels - 1]);
        orc::State<O, E, W> best;
        bool ok = uncoarsen_levels(levels, cfg, part, best, nullptr);
        std::copy(part.begin(), part.end(), part_out);
        *cut_out = (int64_t)(best.cut / 2);
        return ok ? 0 : 4;
    });
}

// pstat quantities, app/part_eval.cpp:73-110 over src/part_stat.hpp.
// out: [cut (each edge once), max part cut, comm size, largest, smallest, total]
int orc_pstat(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw, const int32_t* part,
              int k, int64_t* out) {
    ORC_TIER_DISPATCH(tier, {
        auto g = make_csr<O, E, W>(n, row, adj, val);
        const W* w = (const W*)vw;
        W cut = orc::total_cut(g, part);
        std::vector<W> per(k, 0);
        int64_t comm = 0;
        std::vector<char> seen(k, 0);
        std::vector<int32_t> touched;
        for (O i = 0; i < g.n; i++) {
            touched.clear();
            for (E j = g.row[i]; j < g.row[i + 1]; j++) {
                int32_t p = part[g.adj[j]];
                if (p != part[i]) {
                    per[part[i]] += g.val[j];
                    if (!seen[p]) { seen[p] = 1; touched.push_back(p); }
                }
            }
            comm += (int64_t)touched.size();
            for (int32_t p : touched) seen[p] = 0;
        }
        W mx = 0; for (W x : per) mx = std::max(mx, x);
        std::vector<W> s = orc::part_sizes(g, w, part, k);
        W largest = 0, smallest = std::numeric_limits<W>::max(), total = 0;
        for (W x : s) { largest = std::max(largest, x); smallest = std::min(smallest, x); total += x; }
        out[0] = (int64_t)(cut / 2); out[1] = (int64_t)mx; out[2] = comm;
        out[3] = (int64_t)largest; out[4] = (int64_t)smallest; out[5] = (int64_t)total;
        return 0;
    });
}

int orc_gain_bucket64(int64_t gain, int64_t vwgt) { return orc::gain_bucket<int64_t>(gain, vwgt); }
int orc_gain_bucket32(int32_t gain, int32_t vwgt) { return orc::gain_bucket<int32_t>(gain, vwgt); }
uint32_t orc_pod_hash32(int32_t x) { return orc::pod_hash<int32_t>(x); }
uint64_t orc_rng(uint64_t seed, uint64_t stream, uint64_t idx) { return orc::jet_rng(seed, stream, idx); }

// Metis on a small graph (host), as the reference's initial partitioner.
int orc_metis(int tier, int64_t n, const void* row, const void* adj, const void* val, const void* vw, int k, double imb,
              int32_t* part) {
    ORC_TIER_DISPATCH(tier, {
        auto g = make_csr<O, E, W>(n, row, adj, val);
        return orc::metis_init(g, (const W*)vw, k, imb, part) == 0 ? 0 : 3;
    });
}

}  // extern "C"
