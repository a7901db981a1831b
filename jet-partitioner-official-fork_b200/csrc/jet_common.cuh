// jet_common.cuh -- shared device/host machinery for the B200 Jet partitioner.
//
// Types follow the reference's three integer tiers (header/jet_defs.h:47-92):
//   O  ordinal (vertex id)      int32 or int64
//   E  edge offset (row_map)    int32 or int64
//   W  weight (vertex/edge)     int32 or int64; gains use the same signed type
// Part ids are int32 (header/jet_defs.h:77).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <limits>
#include <type_traits>
#include "../../include/jet_b200.h"

namespace jetb {

typedef int32_t part_t;
static constexpr part_t NULL_PART = -1;     // src/jet_refiner.hpp:87
static constexpr part_t HASH_RECLAIM = -2;  // src/jet_refiner.hpp:88
static constexpr part_t NO_MOVE = -3;       // src/jet_refiner.hpp:89
static constexpr int MAX_SECTIONS = 128;    // src/jet_refiner.hpp:91
static constexpr int MAX_BUCKETS = 50;      // src/jet_refiner.hpp:92
static constexpr int MID_BUCKET = 25;       // src/jet_refiner.hpp:93

// Degree classes used to pick thread / warp / CTA per vertex.
static constexpr int THREAD_DEG = 32;    // deg <= 32: one thread per vertex (tables, selects)
static constexpr int HUB_DEG = 4096;     // deg > 4096: one CTA per vertex
static constexpr int BLOCK = 256;

// Device error flags (bit set in Ctx::err).
enum : int {
    ERRF_PROBE = 1,      // a hash probe ran past its bound (corrupt table)
    ERRF_OVERFLOW = 2,   // a table had no room
    ERRF_SPIN = 4,       // a bounded wait gave up
};

struct CudaError {
    cudaError_t e;
    const char* where;
};

#define JET_CUDA(call)                                                       \
    do {                                                                     \
        cudaError_t _e = (call);                                             \
        if (_e != cudaSuccess) throw ::jetb::CudaError{_e, #call};           \
    } while (0)

#define JET_LAUNCH_CHECK() JET_CUDA(cudaGetLastError())

// ------------------------------------------------------------------ hashing / RNG
// Both are restated identically in the CPU oracle so that the two draw the
// same numbers for the same (seed, stream, index).
__host__ __device__ __forceinline__ uint32_t xorshift32(uint32_t x) {  // src/heuristics.hpp:49-56
    x ^= x << 13; x ^= x >> 17; x ^= x << 5; return x;
}
__host__ __device__ __forceinline__ uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }
// MurmurHash3_x86_32 (public domain algorithm) with seed 0 over 4- or 8-byte
// keys: the byte hash that Kokkos::pod_hash applies (src/heuristics.hpp:73).
__host__ __device__ __forceinline__ uint32_t murmur_block(uint32_t h, uint32_t k) {
    k *= 0xcc9e2d51u; k = rotl32(k, 15); k *= 0x1b873593u;
    h ^= k; h = rotl32(h, 13); return h * 5 + 0xe6546b64u;
}
__host__ __device__ __forceinline__ uint32_t murmur_final(uint32_t h, uint32_t len) {
    h ^= len; h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16; return h;
}
__host__ __device__ __forceinline__ uint32_t pod_hash(int32_t x) {
    return murmur_final(murmur_block(0, (uint32_t)x), 4);
}
__host__ __device__ __forceinline__ uint32_t pod_hash(int64_t x) {
    uint64_t u = (uint64_t)x;
    return murmur_final(murmur_block(murmur_block(0, (uint32_t)u), (uint32_t)(u >> 32)), 8);
}
// splitmix64 finaliser over a (seed, stream, index) counter.
__host__ __device__ __forceinline__ uint64_t jet_rng(uint64_t seed, uint64_t stream, uint64_t idx) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (stream * 0x100000001B3ull + idx + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t rng_stream(int level, int kind, int round) {
    return ((uint64_t)(uint32_t)level << 40) | ((uint64_t)(uint32_t)kind << 32) | (uint32_t)round;
}
enum { RNG_HEC_RANDOM = 1, RNG_MATCH_RANDOM = 2, RNG_MATCH_PICK = 3 };

// ------------------------------------------------------------------ atomics
__device__ __forceinline__ int32_t atomic_cas(int32_t* p, int32_t c, int32_t v) { return atomicCAS((int*)p, c, v); }
__device__ __forceinline__ int64_t atomic_cas(int64_t* p, int64_t c, int64_t v) {
    return (int64_t)atomicCAS((unsigned long long*)p, (unsigned long long)c, (unsigned long long)v);
}
__device__ __forceinline__ uint64_t atomic_cas(uint64_t* p, uint64_t c, uint64_t v) {
    return (uint64_t)atomicCAS((unsigned long long*)p, (unsigned long long)c, (unsigned long long)v);
}
__device__ __forceinline__ int32_t atomic_add(int32_t* p, int32_t v) { return atomicAdd((int*)p, v); }
__device__ __forceinline__ int64_t atomic_add(int64_t* p, int64_t v) {
    return (int64_t)atomicAdd((unsigned long long*)p, (unsigned long long)v);
}

// Adds w to a shared-memory accumulator that starts at zero.  With 64-bit
// weights and `narrow` (the graph's total edge weight is below 2^31, so no
// partial sum reaches 2^32) the add is a 32-bit atomic on the low word: the
// high word stays zero and the 64-bit value is exact.  A 64-bit shared
// atomic add costs several times as much.
template <class W>
__device__ __forceinline__ void acc_add(W* p, W w, int narrow) {
    if (sizeof(W) == 8 && narrow) atomicAdd((unsigned*)p, (unsigned)w);
    else atomic_add(p, w);
}
// Loads that bypass L1 so other SMs' atomics are observed within a kernel.
template <class T> __device__ __forceinline__ T ld_cg(const T* p) { return *(const volatile T*)p; }
template <class T> __device__ __forceinline__ void st_v(T* p, T v) { *(volatile T*)p = v; }

// Warp-aggregated append: every lane of the warp must call it (pred may be
// false).  Returns the slot for lanes with pred, -1 otherwise.
template <class C>
__device__ __forceinline__ C warp_append(C* counter, bool pred) {
    unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (mask == 0) return (C)-1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    C base = 0;
    if (lane == leader) base = atomic_add(counter, (C)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!pred) return (C)-1;
    return base + (C)__popc(mask & ((1u << lane) - 1));
}

template <class T> __device__ __forceinline__ T shfl_xor(T v, int m, int w) { return __shfl_xor_sync(0xffffffffu, v, m, w); }
template <class T> __device__ __forceinline__ T group_sum(T v, int w) {
    for (int m = w >> 1; m > 0; m >>= 1) v += shfl_xor(v, m, w);
    return v;
}

template <class T> __host__ __device__ __forceinline__ T ceil_div(T a, T b) { return (a + b - 1) / b; }

// ------------------------------------------------------------------ launch geometry
// Every kernel launch site calls count_launch() (read by jet_launch_count).
// While a graph is being captured the count is provisional: the capturing
// code corrects it by the number of times the captured kernels ran.
void count_launch();
int64_t launch_counter();
// Which level-loop drivers refinement may use (JET_DRIVER_* bits).
int refine_drivers();
// The one-CTA level loop may keep its state in shared memory (JET_DRIVER_CTA_SMEM).
bool cta_smem_resident();
// Rebalancing may order only the queued candidates (JET_DRIVER_REB_QUEUE).
bool reb_queue_enabled();
// JET_DEBUG_TIMING set in the environment: phase timings go to stderr.
bool debug_timing();
// Host clock in milliseconds (steady).
double host_ms();
// Largest dynamic shared memory a launch of `func` can request on the
// current device (opt-in maximum minus the kernel's static shared memory).
int max_dynamic_smem(const void* func);
// METIS_PartGraphKway with int64 arrays.  Metis keeps global random state,
// so concurrent in-process calls would change each other's results: a
// thread in batch mode sends its call to a helper process (one graph per
// helper at a time); other threads call in process, one at a time.
int metis_kway(int64_t n, int64_t m, int64_t* xadj, int64_t* adj, int64_t* vw, int64_t* ew, int64_t nparts, float ub,
               int64_t* obj, int64_t* part);
// Waits for a stream; batch-mode threads block on an event instead of
// spinning, leaving the host cores to the other workers and Metis helpers.
void stream_wait(cudaStream_t s);
// True on a batch or server worker thread.
bool batch_thread();
void add_launches(int64_t n);
// True while this thread captures work into a CUDA graph (profiling event
// records are skipped: they are not allowed inside conditional bodies).
bool& capturing();
// Per-device stream used only to capture graphs.
cudaStream_t capture_stream();
// Pinned, device-mapped host buffers reused across calls (cudaHostAlloc costs
// milliseconds): acquire returns a slot of at least `bytes`, release frees it
// for reuse by a later caller on the same thread.
int pinned_acquire(size_t bytes);
void* pinned_ptr(int slot);
void pinned_release(int slot);

struct Dev {
    int sms = 148;
    int max_smem_optin = 227 * 1024;
    int coop = 0;  // cooperative launches supported
    size_t total_mem = (size_t)180 << 30;
};
Dev& device_info();

inline unsigned grid_for(int64_t items, int per_block = BLOCK) {
    int64_t b = (items + per_block - 1) / per_block;
    if (b < 1) b = 1;
    if (b > 0x7fffffff) b = 0x7fffffff;
    return (unsigned)b;
}
// Grid for grid-stride loops whose item count lives on the device.
inline unsigned grid_persistent(int64_t max_items, int blocks_per_sm = 8) {
    int64_t cap = (int64_t)device_info().sms * blocks_per_sm;
    int64_t b = (max_items + BLOCK - 1) / BLOCK;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

// Threads per vertex for edge-parallel kernels, from the average degree.
inline int group_for_avg_degree(double avg) {
    if (avg <= 6.0) return 4;
    if (avg <= 14.0) return 8;
    if (avg <= 28.0) return 16;
    return 32;
}

// ------------------------------------------------------------------ memory
// Stream-ordered allocations from a library-owned pool that keeps freed
// memory for reuse, so per-level and per-call buffers cost no cudaMalloc
// after warm-up.
struct Pool {
    cudaMemPool_t pool = nullptr;
    int device = -1;
};
cudaMemPool_t pool_for_current_device();
// Large buffers (>= BIG_BYTES) are kept across calls: mapping hundreds of MB
// into the stream-ordered pool costs milliseconds per allocation.  A block
// freed on one stream is handed to the next request that fits (within 2x),
// whose stream first waits for the freeing stream's work.
static constexpr size_t BIG_BYTES = (size_t)32 << 20;
void* big_alloc(size_t bytes, cudaStream_t s, size_t* got);
void big_free(void* p, size_t bytes, cudaStream_t s);

template <class T>
struct DBuf {
    T* p = nullptr;
    int64_t n = 0;
    cudaStream_t s = nullptr;
    size_t big = 0;  // bytes of a cached large block (0: from the pool)
    DBuf() {}
    DBuf(int64_t count, cudaStream_t st) { alloc(count, st); }
    void alloc(int64_t count, cudaStream_t st) {
        release();
        s = st;
        n = count;
        if (count > 0) {
            size_t bytes = sizeof(T) * (size_t)count;
            double t0 = debug_timing() ? host_ms() : 0;
            if (bytes >= BIG_BYTES) p = (T*)big_alloc(bytes, st, &big);
            else JET_CUDA(cudaMallocFromPoolAsync((void**)&p, bytes, pool_for_current_device(), st));
            if (debug_timing()) {
                double dt = host_ms() - t0;
                if (dt > 1.0) fprintf(stderr, "jet: slow device allocation %.1f MB took %.3f ms\n", bytes / 1e6, dt);
            }
        }
    }
    void release() {
        if (p) {
            if (big) big_free(p, big, s);
            else cudaFreeAsync(p, s);
        }
        p = nullptr;
        n = 0;
        big = 0;
    }
    ~DBuf() { release(); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s), big(o.big) { o.p = nullptr; o.n = 0; o.big = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; s = o.s; big = o.big; o.p = nullptr; o.n = 0; o.big = 0; }
        return *this;
    }
    void zero() { if (n) JET_CUDA(cudaMemsetAsync(p, 0, sizeof(T) * (size_t)n, s)); }
    void fill_bytes(int b) { if (n) JET_CUDA(cudaMemsetAsync(p, b, sizeof(T) * (size_t)n, s)); }
};

// ------------------------------------------------------------------ kernels: fill / iota
template <class T>
__global__ void k_fill(T* p, int64_t n, T v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
template <class T>
inline void fill(T* p, int64_t n, T v, cudaStream_t s) {
    if (n <= 0) return;
    k_fill<T><<<grid_persistent(n, 16), BLOCK, 0, s>>>(p, n, v); count_launch();
    JET_LAUNCH_CHECK();
}

// ------------------------------------------------------------------ scan
// Exclusive prefix sum in three launches: per-tile sums, one-block scan of the
// tile sums, per-tile scan plus carry.  `in` may alias `out`; `total` (device,
// nullable) receives the grand total.  Input element i is get(i).
static constexpr int SCAN_TILE = 2048;  // items per tile (256 threads x 8)

template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem_warp, T& block_total) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T x = v;
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int nw = blockDim.x >> 5;
        T s = lane < nw ? smem_warp[lane] : T(0);
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) smem_warp[lane] = s;
    }
    __syncthreads();
    T warp_prefix = wid > 0 ? smem_warp[wid - 1] : T(0);
    block_total = smem_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

template <class T, class Get>
__global__ void __launch_bounds__(BLOCK) k_scan_tiles(Get get, int64_t n, T* tile_sums) {
    __shared__ T sw[32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    T s = 0;
    for (int j = 0; j < SCAN_TILE / BLOCK; j++) {
        int64_t i = base + (int64_t)threadIdx.x * (SCAN_TILE / BLOCK) + j;
        if (i < n) s += get(i);
    }
    T tot;
    block_exclusive_scan<T>(s, sw, tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

template <class T>
__global__ void __launch_bounds__(1024) k_scan_sums(T* sums, int64_t ntiles, T* total) {
    __shared__ T sw[32];
    T carry = 0;
    for (int64_t b = 0; b < ntiles; b += 1024) {
        int64_t i = b + threadIdx.x;
        T v = i < ntiles ? sums[i] : T(0);
        T tot;
        T ex = block_exclusive_scan<T>(v, sw, tot);
        if (i < ntiles) sums[i] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class T, class Get>
__global__ void __launch_bounds__(BLOCK) k_scan_apply(Get get, int64_t n, const T* tile_offsets, T* out) {
    __shared__ T sw[32];
    int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    constexpr int PER = SCAN_TILE / BLOCK;
    T v[PER];
    T s = 0;
    for (int j = 0; j < PER; j++) {
        int64_t i = base + (int64_t)threadIdx.x * PER + j;
        v[j] = i < n ? get(i) : T(0);
        s += v[j];
    }
    T tot;
    T ex = block_exclusive_scan<T>(s, sw, tot) + tile_offsets[blockIdx.x];
    for (int j = 0; j < PER; j++) {
        int64_t i = base + (int64_t)threadIdx.x * PER + j;
        if (i < n) out[i] = ex;
        ex += v[j];
    }
}

// Small scans in one launch: one 1024-thread block walks the input in chunks
// of 4096 (four items per thread) with a running carry.
static constexpr int64_t SCAN_ONE_BLOCK_MAX = 16384;
template <class T, class Get>
__global__ void __launch_bounds__(1024) k_scan_one(Get get, int64_t n, T* out, T* total) {
    __shared__ T sw[32];
    T carry = 0;
    for (int64_t base = 0; base < n; base += 4 * 1024) {
        T v[4];
        T s = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t i = base + (int64_t)threadIdx.x * 4 + j;
            v[j] = i < n ? get(i) : T(0);
            s += v[j];
        }
        T tot;
        T ex = block_exclusive_scan<T>(s, sw, tot) + carry;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t i = base + (int64_t)threadIdx.x * 4 + j;
            if (i < n) out[i] = ex;
            ex += v[j];
        }
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class T>
struct GetArray {
    const T* a;
    __device__ __forceinline__ T operator()(int64_t i) const { return a[i]; }
};

template <class A, class B>
struct GetCast {
    const A* a;
    __device__ __forceinline__ B operator()(int64_t i) const { return (B)a[i]; }
};

// Scratch for scans: tile sums.  One per context, grown on demand.
struct ScanScratch {
    DBuf<int64_t> buf;
};

template <class T, class Get>
inline void exclusive_scan(Get get, int64_t n, T* out, T* total, ScanScratch& sc, cudaStream_t s) {
    if (n <= 0) {
        if (total) JET_CUDA(cudaMemsetAsync(total, 0, sizeof(T), s));
        return;
    }
    if (n <= SCAN_ONE_BLOCK_MAX) {
        k_scan_one<T, Get><<<1, 1024, 0, s>>>(get, n, out, total); count_launch();
        JET_LAUNCH_CHECK();
        return;
    }
    int64_t ntiles = ceil_div<int64_t>(n, SCAN_TILE);
    if (sc.buf.n < ntiles) sc.buf.alloc(ntiles + 1024, s);
    T* sums = (T*)sc.buf.p;
    k_scan_tiles<T, Get><<<(unsigned)ntiles, BLOCK, 0, s>>>(get, n, sums); count_launch();
    JET_LAUNCH_CHECK();
    k_scan_sums<T><<<1, 1024, 0, s>>>(sums, ntiles, total); count_launch();
    JET_LAUNCH_CHECK();
    k_scan_apply<T, Get><<<(unsigned)ntiles, BLOCK, 0, s>>>(get, n, sums, out); count_launch();
    JET_LAUNCH_CHECK();
}

template <class T>
inline void exclusive_scan_array(const T* in, int64_t n, T* out, T* total, ScanScratch& sc, cudaStream_t s) {
    exclusive_scan<T, GetArray<T>>(GetArray<T>{in}, n, out, total, sc, s);
}

// ------------------------------------------------------------------ profiling hooks
// Optional CUDA-event timing of selected kernel classes, on the stream the
// kernels run on.  Used by the benchmark to measure the dominant kernel.
enum ProfKernel : int {
    PK_CONN_BUILD = 0,
    PK_LP_SELECT,
    PK_AFTERBURN,
    PK_UPDATE,       // update_small (both passes)
    PK_CONTRACT,
    PK_HEC,
    PK_CONN_FINEST,  // the table build of the finest level alone
    PK_REB_SELECT,   // weak destination select / strong eviction scores
    PK_REB_SORT,     // bucket offsets, candidate sort, weight prefix
    PK_REB_EVICT,    // eviction filter (+ strong: cookie cutter, draws)
    PK_APPLY,        // apply moves and part sizes
    PK_UPDATE_LARGE, // update_large: mark neighbours, rebuild their rows
    PK_CUT_AFTER,    // cut change part 2
    PK_COUNT
};
// Marks the start/end of a timed launch group.  bytes = algorithmic bytes;
// prof_add_bytes adds to a group already ended (counts known only after the
// iteration's sync).
int prof_begin(cudaStream_t s);
void prof_end(int h, ProfKernel k, double bytes, cudaStream_t s);
void prof_add_bytes(int h, double bytes);
bool prof_active();
// Device buffer of the persistent level loops' phase clocks (jet_prof_phases), or null.
unsigned long long* phase_clk_ptr();
void prof_collect();  // after a stream sync: folds event pairs into the slots

}  // namespace jetb
