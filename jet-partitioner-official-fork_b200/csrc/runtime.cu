// runtime.cu -- process-wide runtime pieces: device properties, the
// stream-ordered memory pool, the default stream, error strings, kernel-class
// profiling and the tier-generic C entry points.
#include "api_impl.cuh"
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

namespace jetb {

static std::mutex g_mu;

Dev& device_info() {
    static thread_local int cached_dev = -1;
    static thread_local Dev d;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != cached_dev) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, dev) == cudaSuccess) {
            d.sms = p.multiProcessorCount;
            d.max_smem_optin = (int)p.sharedMemPerBlockOptin;
            d.coop = p.cooperativeLaunch;
        }
        cached_dev = dev;
    }
    return d;
}

// One pool per device, keeping freed memory (release threshold = max).
cudaMemPool_t pool_for_current_device() {
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        JET_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        uint64_t thr = UINT64_MAX;
        JET_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &thr));
    }
    return pools[dev];
}

cudaStream_t default_stream() {
    static cudaStream_t streams[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!streams[dev]) JET_CUDA(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
    return streams[dev];
}

static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
int64_t launch_counter() { return g_launches.load(); }
static std::atomic<int> g_drivers{JET_DRIVER_ALL};
int refine_drivers() { return g_drivers.load(); }
bool debug_timing() {
    static const bool on = getenv("JET_DEBUG_TIMING") != nullptr;
    return on;
}
void add_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

bool& capturing() {
    static thread_local bool c = false;
    return c;
}

cudaStream_t capture_stream() {
    static cudaStream_t streams[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!streams[dev]) JET_CUDA(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking));
    return streams[dev];
}

struct PinnedSlot {
    void* p = nullptr;
    size_t bytes = 0;
    bool used = false;
};
static thread_local std::vector<PinnedSlot> g_pinned;

int pinned_acquire(size_t bytes) {
    for (size_t i = 0; i < g_pinned.size(); i++) {
        PinnedSlot& sl = g_pinned[i];
        if (!sl.used && sl.bytes >= bytes) { sl.used = true; return (int)i; }
    }
    PinnedSlot sl;
    size_t b = bytes < 4096 ? 4096 : bytes;
    JET_CUDA(cudaHostAlloc(&sl.p, b, cudaHostAllocMapped));
    sl.bytes = b;
    sl.used = true;
    g_pinned.push_back(sl);
    return (int)g_pinned.size() - 1;
}
void* pinned_ptr(int slot) { return g_pinned[slot].p; }
void pinned_release(int slot) {
    if (slot >= 0 && slot < (int)g_pinned.size()) g_pinned[slot].used = false;
}

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

// ---------------------------------------------------------------- profiling
struct ProfState {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    struct Pending { int ev; int kind; double bytes; };
    std::vector<Pending> pending;
    int next = 0;
    double ms[PK_COUNT] = {0};
    double bytes[PK_COUNT] = {0};
    int64_t launches[PK_COUNT] = {0};
};
static ProfState g_prof;

int prof_begin(cudaStream_t s) {
    if (!g_prof.on || capturing()) return -1;
    if (g_prof.next + 2 > (int)g_prof.pool.size()) {
        int old = (int)g_prof.pool.size();
        g_prof.pool.resize(old + 512);
        for (int i = old; i < old + 512; i++) cudaEventCreate(&g_prof.pool[i]);
    }
    int h = g_prof.next;
    g_prof.next += 2;
    cudaEventRecord(g_prof.pool[h], s);
    return h;
}

void prof_end(int h, ProfKernel k, double bytes, cudaStream_t s) {
    if (h < 0 || !g_prof.on || capturing()) return;
    cudaEventRecord(g_prof.pool[h + 1], s);
    g_prof.pending.push_back({h, (int)k, bytes});
}

void prof_collect() {
    if (!g_prof.on) return;
    for (auto& p : g_prof.pending) {
        cudaEventSynchronize(g_prof.pool[p.ev + 1]);
        float ms = 0;
        if (cudaEventElapsedTime(&ms, g_prof.pool[p.ev], g_prof.pool[p.ev + 1]) == cudaSuccess) {
            g_prof.ms[p.kind] += ms;
            g_prof.bytes[p.kind] += p.bytes;
            g_prof.launches[p.kind] += 1;
        }
    }
    g_prof.pending.clear();
    g_prof.next = 0;
}

}  // namespace jetb

using namespace jetb;

static TierOps* ops_for(int tier) {
    static TierOps t[3] = {ops_i32(), ops_big(), ops_biggest()};
    if (tier < 0 || tier > 2) return nullptr;
    return &t[tier];
}

extern "C" {

const char* jet_version(void) { return "jet-b200 1.1.0 (sm_100a)"; }
const char* jet_last_error(void) { return g_last_error.c_str(); }

int jet_device_ok(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return JET_ERR_NOT_BUILT; }
    return JET_OK;
}

int jet_coarsen_map(int tier, int alg, int level, uint64_t seed, int64_t n, int64_t nnz, const void* row_map, const void* entries,
                    const void* values, const void* vweights, int uniform, void* map_out, void* hn_out, int64_t* nc, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->coarsen_map(alg, level, seed, n, nnz, row_map, entries, values, vweights, uniform, map_out, hn_out, nc, stream);
}

int jet_contract(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values, const void* vweights,
                 const void* map, int64_t nc, void* crow, void* cadj, void* cval, void* cvw, int64_t* cnnz, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->contract(n, nnz, row_map, entries, values, vweights, map, nc, crow, cadj, cval, cvw, cnnz, stream);
}

int jet_conn_build(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values, const int32_t* part,
                   int32_t k, void* off, int32_t* ent, void* val, int32_t* size, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->conn_build(n, nnz, row_map, entries, values, part, k, off, ent, val, size, stream);
}

int jet_refine_iters(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                     const void* vweights, int32_t* part, int32_t k, double imb, double filter_ratio, int32_t iters, void* sizes,
                     int64_t* cut, void* off, int32_t* ent, void* val, int32_t* size, int32_t* dest_cache, int64_t* moves,
                     int32_t* kinds, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->refine_iters(n, nnz, row_map, entries, values, vweights, part, k, imb, filter_ratio, iters, sizes, cut, off, ent, val,
                           size, dest_cache, moves, kinds, stream);
}

int jet_refine_level(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                     const void* vweights, int32_t* part, int32_t k, double imb, double tol, int uniform_ew, int64_t* cut,
                     int32_t* iters, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->refine_level(n, nnz, row_map, entries, values, vweights, part, k, imb, tol, uniform_ew, cut, iters, stream);
}

int jet_pstat(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values, const void* vweights,
              const int32_t* part, int32_t k, int64_t* out, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->pstat(n, nnz, row_map, entries, values, vweights, part, k, out, stream);
}

int jet_project(int tier, int64_t n_fine, const void* map, const int32_t* coarse, int32_t* fine, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->project(n_fine, map, coarse, fine, stream);
}

int64_t jet_launch_count(void) { return g_launches.load(); }

int jet_set_refine_drivers(int mask) { return g_drivers.exchange(mask & JET_DRIVER_ALL); }

int jet_prof_enable(int on) {
    prof_collect();
    g_prof.on = on != 0;
    for (int i = 0; i < PK_COUNT; i++) { g_prof.ms[i] = 0; g_prof.bytes[i] = 0; g_prof.launches[i] = 0; }
    return JET_OK;
}

int jet_prof_read(double* ms, double* bytes, int64_t* launches) {
    prof_collect();
    for (int i = 0; i < PK_COUNT; i++) {
        if (ms) ms[i] = g_prof.ms[i];
        if (bytes) bytes[i] = g_prof.bytes[i];
        if (launches) launches[i] = g_prof.launches[i];
    }
    return JET_OK;
}

}  // extern "C"
