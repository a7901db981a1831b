// runtime.cu -- process-wide runtime pieces: device properties, the
// stream-ordered memory pool, the default stream, error strings, kernel-class
// profiling and the tier-generic C entry points.
#include "api_impl.cuh"
#include <atomic>
#include <cerrno>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <dlfcn.h>
#include <spawn.h>
#include <signal.h>
#include <sys/socket.h>
#include <sys/wait.h>
#include <unistd.h>

extern char** environ;
typedef int64_t metis_idx_t;
typedef float metis_real_t;
extern "C" int METIS_PartGraphKway(metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*, metis_idx_t*,
                                   metis_idx_t*, metis_idx_t*, metis_real_t*, metis_real_t*, metis_idx_t*, metis_idx_t*,
                                   metis_idx_t*);

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
            d.total_mem = p.totalGlobalMem;
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

namespace {
struct BigBlock {
    void* p;
    size_t bytes;
    int dev;
    cudaEvent_t ev;  // recorded on the freeing stream
};
std::mutex g_big_mu;
std::vector<BigBlock> g_big_free;
size_t g_big_cached = 0;
}  // namespace

void* big_alloc(size_t bytes, cudaStream_t s, size_t* got) {
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(g_big_mu);
        int best = -1;
        for (size_t i = 0; i < g_big_free.size(); i++) {
            const BigBlock& b = g_big_free[i];
            if (b.dev == dev && b.bytes >= bytes && b.bytes <= 2 * bytes && (best < 0 || b.bytes < g_big_free[best].bytes))
                best = (int)i;
        }
        if (best >= 0) {
            BigBlock b = g_big_free[best];
            g_big_free.erase(g_big_free.begin() + best);
            g_big_cached -= b.bytes;
            JET_CUDA(cudaStreamWaitEvent(s, b.ev, 0));
            cudaEventDestroy(b.ev);
            *got = b.bytes;
            return b.p;
        }
    }
    // round up to one of four size classes per power of two, so that later
    // requests of similar size find this block in the cache
    size_t cls = (size_t)1 << (63 - __builtin_clzll((unsigned long long)bytes));
    size_t step = cls / 4;
    size_t want = (bytes + step - 1) / step * step;
    void* p = nullptr;
    JET_CUDA(cudaMallocFromPoolAsync(&p, want, pool_for_current_device(), s));
    *got = want;
    return p;
}

void big_free(void* p, size_t bytes, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess || cudaEventRecord(ev, s) != cudaSuccess) {
        cudaFreeAsync(p, s);
        return;
    }
    std::lock_guard<std::mutex> lk(g_big_mu);
    g_big_free.push_back({p, bytes, dev, ev});
    g_big_cached += bytes;
    // keep at most a quarter of this device's memory cached; oldest blocks go
    // first (the device size comes from the cached properties: querying free
    // memory here stalled for tens of milliseconds)
    const size_t total_b = device_info().total_mem;
    size_t mine = 0;
    for (const BigBlock& b : g_big_free) if (b.dev == dev) mine += b.bytes;
    for (size_t i = 0; i < g_big_free.size() && mine > total_b / 4;) {
        BigBlock b = g_big_free[i];
        if (b.dev != dev) { i++; continue; }
        g_big_free.erase(g_big_free.begin() + i);
        g_big_cached -= b.bytes;
        mine -= b.bytes;
        cudaStreamWaitEvent(s, b.ev, 0);
        cudaFreeAsync(b.p, s);
        cudaEventDestroy(b.ev);
    }
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
static thread_local int t_driver_mask = JET_DRIVER_ALL;
int refine_drivers() { return g_drivers.load() & t_driver_mask; }
bool cta_smem_resident() { return (g_drivers.load() & JET_DRIVER_CTA_SMEM) != 0; }
bool reb_queue_enabled() { return (g_drivers.load() & JET_DRIVER_REB_QUEUE) != 0; }
double host_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
bool debug_timing() {
    static const bool on = getenv("JET_DEBUG_TIMING") != nullptr;
    return on;
}
void add_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int max_dynamic_smem(const void* func) {
    cudaFuncAttributes fa;
    JET_CUDA(cudaFuncGetAttributes(&fa, func));
    return device_info().max_smem_optin - (int)fa.sharedSizeBytes;
}

// ---------------------------------------------------------------- Metis
static std::mutex g_metis_inproc;
static thread_local bool t_batch = false;
bool batch_thread() { return t_batch; }

namespace {
struct Helper {
    pid_t pid = -1;
    int fd = -1;
    bool busy = false;
};
std::mutex g_hmu;
std::condition_variable g_hcv;
std::vector<Helper> g_helpers;
bool g_helpers_broken = false;

std::string helper_path() {
    Dl_info info;
    if (!dladdr((void*)&helper_path, &info) || !info.dli_fname) return "";
    std::string so = info.dli_fname;
    size_t slash = so.rfind('/');
    return (slash == std::string::npos ? std::string(".") : so.substr(0, slash)) + "/jet_metis_helper";
}

bool spawn_helper(Helper& h) {
    static const std::string path = helper_path();
    if (path.empty() || access(path.c_str(), X_OK) != 0) return false;
    int sv[2];
    if (socketpair(AF_UNIX, SOCK_STREAM | SOCK_CLOEXEC, 0, sv) != 0) return false;
    posix_spawn_file_actions_t fa;
    posix_spawn_file_actions_init(&fa);
    posix_spawn_file_actions_adddup2(&fa, sv[1], 0);
    posix_spawn_file_actions_adddup2(&fa, sv[1], 1);
    char* argv[] = {(char*)path.c_str(), nullptr};
    pid_t pid = -1;
    int rc = posix_spawn(&pid, path.c_str(), &fa, nullptr, argv, environ);
    posix_spawn_file_actions_destroy(&fa);
    close(sv[1]);
    if (rc != 0) { close(sv[0]); return false; }
    h.pid = pid;
    h.fd = sv[0];
    return true;
}

// Both retry a transfer that a signal interrupted.
bool send_all(int fd, const void* p, size_t bytes) {
    const char* c = (const char*)p;
    while (bytes > 0) {
        ssize_t r = send(fd, c, bytes, MSG_NOSIGNAL);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        c += r;
        bytes -= (size_t)r;
    }
    return true;
}

bool recv_all(int fd, void* p, size_t bytes) {
    char* c = (char*)p;
    while (bytes > 0) {
        ssize_t r = recv(fd, c, bytes, 0);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        c += r;
        bytes -= (size_t)r;
    }
    return true;
}

// Index of a helper now marked busy (its socket in *fd), or -1 when none can
// be had.
int acquire_helper(int* fd) {
    std::unique_lock<std::mutex> lk(g_hmu);
    size_t cap = std::thread::hardware_concurrency();
    if (cap < 1) cap = 1;
    if (cap > 32) cap = 32;
    while (true) {
        if (g_helpers_broken) return -1;
        for (size_t i = 0; i < g_helpers.size(); i++)
            if (!g_helpers[i].busy && g_helpers[i].fd >= 0) {
                g_helpers[i].busy = true;
                *fd = g_helpers[i].fd;
                return (int)i;
            }
        if (g_helpers.size() < cap) {
            Helper h;
            if (!spawn_helper(h)) { g_helpers_broken = true; return -1; }
            h.busy = true;
            *fd = h.fd;
            g_helpers.push_back(h);
            return (int)g_helpers.size() - 1;
        }
        g_hcv.wait(lk);
    }
}

std::atomic<int64_t> g_helper_calls{0}, g_helper_failures{0}, g_inproc_calls{0}, g_helper_metis_errors{0};

void release_helper(int i, bool ok) {
    std::lock_guard<std::mutex> lk(g_hmu);
    Helper& h = g_helpers[i];
    if (!ok) {
        // this helper is gone: close it and let the next request start a
        // fresh one in its place (the failed call runs in-process)
        g_helper_failures++;
        close(h.fd);
        h.fd = -1;
        if (h.pid > 0) { kill(h.pid, SIGKILL); waitpid(h.pid, nullptr, 0); }
        h.pid = -1;
        if (spawn_helper(h)) h.busy = false;
        else g_helpers_broken = true;  // helpers cannot be started: in-process calls from now on
    }
    h.busy = false;
    g_hcv.notify_one();
}
}  // namespace

// Failures injected by jet_test_inject_metis_failures: the next calls
// report METIS_ERROR without running Metis.
static std::atomic<int> g_metis_fail{0};

int metis_kway(int64_t n, int64_t m, int64_t* xadj, int64_t* adj, int64_t* vw, int64_t* ew, int64_t nparts, float ub,
               int64_t* obj, int64_t* part) {
    for (int f = g_metis_fail.load(); f > 0; f = g_metis_fail.load())
        if (g_metis_fail.compare_exchange_weak(f, f - 1)) return -4;  // METIS_ERROR
    if (t_batch) {
        int fd = -1;
        int hi = acquire_helper(&fd);
        if (hi >= 0) {
            int64_t hdr[3] = {n, m, nparts};
            int64_t out[2] = {0, 0};
            bool ok = send_all(fd, hdr, sizeof(hdr)) && send_all(fd, &ub, sizeof(ub)) &&
                      send_all(fd, xadj, sizeof(int64_t) * (n + 1)) && send_all(fd, adj, sizeof(int64_t) * m) &&
                      send_all(fd, vw, sizeof(int64_t) * n) && send_all(fd, ew, sizeof(int64_t) * m) &&
                      recv_all(fd, out, sizeof(out)) && recv_all(fd, part, sizeof(int64_t) * n);
            const bool metis_ok = ok && out[0] == 1;  // METIS_OK
            // a helper whose Metis reported an error is replaced too: Metis
            // state left from its earlier calls must not reach later ones
            release_helper(hi, metis_ok);
            if (metis_ok) {
                g_helper_calls++;
                *obj = out[1];
                return 1;
            }
            if (ok) {
                // Metis failed in the helper: rerun the call once in-process
                g_helper_calls++;
                g_helper_metis_errors++;
                g_helper_failures--;  // release_helper counted it as a transfer failure
            }
        }
    }
    g_inproc_calls++;
    std::lock_guard<std::mutex> lk(g_metis_inproc);
    metis_idx_t nn = n, ncon = 1, np = nparts;
    metis_real_t u = ub;
    return METIS_PartGraphKway(&nn, &ncon, xadj, adj, vw, nullptr, ew, &np, nullptr, &u, nullptr, obj, part);
}

void stream_wait(cudaStream_t s) {
    if (!t_batch) {
        JET_CUDA(cudaStreamSynchronize(s));
        return;
    }
    static thread_local cudaEvent_t ev[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!ev[dev]) JET_CUDA(cudaEventCreateWithFlags(&ev[dev], cudaEventBlockingSync | cudaEventDisableTiming));
    JET_CUDA(cudaEventRecord(ev[dev], s));
    JET_CUDA(cudaEventSynchronize(ev[dev]));
}

bool& capturing() {
    static thread_local bool c = false;
    return c;
}

// One per thread and device: threads that partition concurrently capture
// their level graphs independently.
cudaStream_t capture_stream() {
    static thread_local cudaStream_t streams[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
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
    int open = 0;  // begun, not yet ended
};
static ProfState g_prof;
static std::recursive_mutex g_prof_mu;  // host threads may partition concurrently

int prof_begin(cudaStream_t s) {
    std::lock_guard<std::recursive_mutex> lk(g_prof_mu);
    if (!g_prof.on || capturing()) return -1;
    if (g_prof.next + 2 > (int)g_prof.pool.size()) {
        int old = (int)g_prof.pool.size();
        g_prof.pool.resize(old + 512);
        for (int i = old; i < old + 512; i++) cudaEventCreate(&g_prof.pool[i]);
    }
    int h = g_prof.next;
    g_prof.next += 2;
    g_prof.open++;
    cudaEventRecord(g_prof.pool[h], s);
    return h;
}

static unsigned long long* g_pclk = nullptr;  // phase clocks of the persistent level loops
unsigned long long* phase_clk_ptr() { return g_pclk; }

bool prof_active() {
    std::lock_guard<std::recursive_mutex> lk(g_prof_mu);
    return g_prof.on && !capturing();
}

void prof_add_bytes(int h, double bytes) {
    std::lock_guard<std::recursive_mutex> lk(g_prof_mu);
    if (h < 0 || !g_prof.on) return;
    for (auto it = g_prof.pending.rbegin(); it != g_prof.pending.rend(); ++it)
        if (it->ev == h) { it->bytes += bytes; return; }
}

void prof_end(int h, ProfKernel k, double bytes, cudaStream_t s) {
    std::lock_guard<std::recursive_mutex> lk(g_prof_mu);
    if (h < 0 || !g_prof.on || capturing()) return;
    cudaEventRecord(g_prof.pool[h + 1], s);
    g_prof.pending.push_back({h, (int)k, bytes});
    g_prof.open--;
}

void prof_collect() {
    std::lock_guard<std::recursive_mutex> lk(g_prof_mu);
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
    if (g_prof.open == 0) g_prof.next = 0;  // events still open elsewhere keep their slots
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

int jet_refine_hierarchy(int tier, const jet_config_c* config, const char* graphs_path, const char* part_path, int32_t* part_out,
                         int64_t part_capacity, int64_t* n_out, int64_t* edge_cut, jet_stats_c* stats, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->refine_hierarchy(config, graphs_path, part_path, part_out, part_capacity, n_out, edge_cut, stats, stream);
}

int jet_project(int tier, int64_t n_fine, const void* map, const int32_t* coarse, int32_t* fine, void* stream) {
    TierOps* o = ops_for(tier);
    if (!o) return JET_ERR_INVALID;
    return o->project(n_fine, map, coarse, fine, stream);
}

int64_t jet_launch_count(void) { return g_launches.load(); }

int jet_prof_phases(int on, uint64_t* out) {
    const size_t bytes = sizeof(unsigned long long) * 6 * PHASE_SLOTS;
    if (on) {
        if (!g_pclk && cudaMalloc(&g_pclk, bytes) != cudaSuccess) { g_pclk = nullptr; return JET_ERR_OOM; }
        return cudaMemset(g_pclk, 0, bytes) == cudaSuccess ? JET_OK : JET_ERR_CUDA;
    }
    if (!g_pclk) return JET_OK;
    cudaDeviceSynchronize();
    int rc = JET_OK;
    if (out && cudaMemcpy(out, g_pclk, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) rc = JET_ERR_CUDA;
    cudaFree(g_pclk);
    g_pclk = nullptr;
    return rc;
}

int jet_metis_call_stats(int64_t* out) {
    if (!out) return JET_ERR_INVALID;
    out[0] = g_helper_calls.load();
    out[1] = g_helper_failures.load();
    out[2] = g_inproc_calls.load();
    {
        std::lock_guard<std::mutex> lk(g_hmu);
        out[3] = (int64_t)g_helpers.size();
        out[4] = g_helpers_broken ? 1 : 0;
    }
    out[5] = g_helper_metis_errors.load();
    return JET_OK;
}

int jet_test_inject_metis_failures(int count) { return g_metis_fail.exchange(count < 0 ? 0 : count); }

int jet_device_alloc(int64_t bytes, void** ptr) {
    if (!ptr || bytes < 0) return JET_ERR_INVALID;
    *ptr = nullptr;
    if (bytes == 0) return JET_OK;
    cudaError_t e = cudaMalloc(ptr, (size_t)bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        g_last_error = std::string("jet_device_alloc: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? JET_ERR_OOM : JET_ERR_CUDA;
    }
    return JET_OK;
}

int jet_device_free(void* ptr) {
    if (ptr && cudaFree(ptr) != cudaSuccess) {
        cudaGetLastError();
        return JET_ERR_CUDA;
    }
    return JET_OK;
}

int jet_copy(void* dst, const void* src, int64_t bytes) {
    if (bytes < 0 || (bytes > 0 && (!dst || !src))) return JET_ERR_INVALID;
    if (bytes == 0) return JET_OK;
    cudaError_t e = cudaMemcpy(dst, src, (size_t)bytes, cudaMemcpyDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        g_last_error = std::string("jet_copy: ") + cudaGetErrorString(e);
        return JET_ERR_CUDA;
    }
    return JET_OK;
}

int jet_set_refine_drivers(int mask) { return g_drivers.exchange(mask & JET_DRIVER_ALL); }

// Batch and server workers run many partitions side by side.  A cooperative
// level kernel needs every SM at once and would stall the other streams, and
// building a level graph costs more host time than its launches save when
// the GPU is shared, and a 16-CTA cluster must wait for 16 free SMs, so their
// threads keep only the one-CTA level loop (the host loop takes the larger
// levels).  They also wait on streams without
// spinning and send Metis calls to helper processes.
void jet_thread_batch_mode(int on) {
    // one CTA for small levels, a 16-CTA cluster for mid-size ones (it needs
    // 16 SMs, not the whole GPU), the host loop above; the loops' options
    // (state in shared memory, the rebalance queue) as everywhere else
    // (JET_BATCH_DRIVERS, read once per process, replaces this mask for tuning)
    static const int batch_mask = [] {
        const char* v = std::getenv("JET_BATCH_DRIVERS");
        return (v && *v) ? (std::atoi(v) & JET_DRIVER_ALL)
                         : (JET_DRIVER_CTA | JET_DRIVER_CLUSTER | JET_DRIVER_CTA_SMEM | JET_DRIVER_REB_QUEUE);
    }();
    t_driver_mask = on ? batch_mask : JET_DRIVER_ALL;
    t_batch = on != 0;
}

int jet_prof_enable(int on) {
    prof_collect();
    std::lock_guard<std::recursive_mutex> lk(g_prof_mu);
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
