// noalloc.cu -- partition statistics without any device allocation.
//
// jet_pstat computes the pstat quantities (cut, largest per-part cut,
// communication volume, part sizes) with scratch memory it allocates per
// call.  Some callers cannot let a library allocate device memory: services
// that reserve the GPU's memory up front for their own pool (a framework's
// caching allocator that has taken the whole device, a real-time loop that
// must never block inside the driver's allocator) and forbid allocation
// afterwards.  jet_pstat_noalloc serves them: its scratch lives in the
// file-scope array below, which every GPU that loads this module holds until
// the process exits, so a call allocates nothing.
//
// Under CUDA's lazy module loading (the default since CUDA 12) the module,
// and with it the array's device memory, is loaded on the first call on each
// device, which also looks up the array's device address.  That first call
// (or running with CUDA_MODULE_LOADING=EAGER) must therefore come before the
// caller reserves the rest of the device's memory.
#include "api_impl.cuh"
#include <climits>
#include <mutex>

namespace jetb {
namespace noalloc {

// Largest part count the scratch array serves.
static constexpr int MAX_PARTS = 16384;
// Layout (int64 words): [0] cut, [1] comm volume, [2] error flags,
// [8 .. 8+MAX_PARTS) per-part cut, [8+MAX_PARTS .. 8+2*MAX_PARTS) part sizes,
// [8+2*MAX_PARTS .. +6) results.  2 * 16384 + 16 words = 256.1 KiB.
static constexpr int SCRATCH_WORDS = 8 + 2 * MAX_PARTS + 8;

// Shared by every call on a device; calls that overlap on the GPU race on it.
static __device__ __align__(256) long long g_scratch[SCRATCH_WORDS];

static constexpr int WARPS = 8;
static constexpr int BITMAP_WORDS = MAX_PARTS / 32;

// One warp per vertex.  Distinct foreign parts are counted with a per-warp
// shared-memory bitmap: a lane that flips a bit from 0 to 1 found a new part;
// the same lanes clear their bits again before the next vertex.
template <class O, class E, class W>
__global__ void __launch_bounds__(WARPS * 32) k_pstat_na(O n, const E* row, const O* adj, const W* val, const W* vw,
                                                         const int32_t* part, int32_t k, long long* scr) {
    __shared__ uint32_t bitmap[WARPS][BITMAP_WORDS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int w = lane; w < BITMAP_WORDS; w += 32) bitmap[wid][w] = 0;
    __syncwarp();
    long long* per_cut = scr + 8;
    long long* sizes = scr + 8 + MAX_PARTS;
    long long cut_acc = 0, comm_acc = 0;
    const int64_t warps = (int64_t)gridDim.x * WARPS;
    for (int64_t x = (int64_t)blockIdx.x * WARPS + wid; x < n; x += warps) {
        int32_t own = part[x];
        if (own < 0 || own >= k) {
            if (lane == 0) atomicOr((unsigned long long*)&scr[2], 1ull);
            continue;
        }
        E s = row[x], e = row[x + 1];
        long long wsum = 0, fresh = 0;
        bool bad = false;
        for (E j = s + lane; j < e; j += 32) {
            int32_t p = part[adj[j]];
            if (p < 0 || p >= k) { bad = true; continue; }
            if (p == own) continue;
            wsum += (long long)val[j];
            uint32_t bit = 1u << (p & 31);
            uint32_t old = atomicOr(&bitmap[wid][p >> 5], bit);
            if (!(old & bit)) fresh++;
        }
        __syncwarp();
        for (E j = s + lane; j < e; j += 32) {
            int32_t p = part[adj[j]];
            if (p >= 0 && p < k && p != own) atomicAnd(&bitmap[wid][p >> 5], ~(1u << (p & 31)));
        }
        __syncwarp();
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr((unsigned long long*)&scr[2], 1ull);
        wsum = group_sum<long long>(wsum, 32);
        fresh = group_sum<long long>(fresh, 32);
        if (lane == 0) {
            if (wsum) atomicAdd((unsigned long long*)&per_cut[own], (unsigned long long)wsum);
            atomicAdd((unsigned long long*)&sizes[own], (unsigned long long)(long long)vw[x]);
            cut_acc += wsum;
            comm_acc += fresh;
        }
    }
    if (lane == 0) {
        if (cut_acc) atomicAdd((unsigned long long*)&scr[0], (unsigned long long)cut_acc);
        if (comm_acc) atomicAdd((unsigned long long*)&scr[1], (unsigned long long)comm_acc);
    }
}

// out = {cut / 2, largest per-part cut, comm volume, largest, smallest, total}
__global__ void __launch_bounds__(1024) k_pstat_na_final(int32_t k, long long* scr) {
    __shared__ long long smx[32], slg[32], ssm[32], stot[32];
    const long long* per_cut = scr + 8;
    const long long* sizes = scr + 8 + MAX_PARTS;
    long long mx = 0, lg = 0, sm = LLONG_MAX, tot = 0;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
        long long c = per_cut[p], z = sizes[p];
        mx = c > mx ? c : mx;
        lg = z > lg ? z : lg;
        sm = z < sm ? z : sm;
        tot += z;
    }
    for (int m = 16; m > 0; m >>= 1) {
        long long a = __shfl_xor_sync(0xffffffffu, mx, m), b = __shfl_xor_sync(0xffffffffu, lg, m);
        long long c = __shfl_xor_sync(0xffffffffu, sm, m), d = __shfl_xor_sync(0xffffffffu, tot, m);
        mx = a > mx ? a : mx; lg = b > lg ? b : lg; sm = c < sm ? c : sm; tot += d;
    }
    if ((threadIdx.x & 31) == 0) { smx[threadIdx.x >> 5] = mx; slg[threadIdx.x >> 5] = lg; ssm[threadIdx.x >> 5] = sm; stot[threadIdx.x >> 5] = tot; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
            mx = smx[w] > mx ? smx[w] : mx; lg = slg[w] > lg ? slg[w] : lg; sm = ssm[w] < sm ? ssm[w] : sm; tot += stot[w];
        }
        long long* res = scr + 8 + 2 * MAX_PARTS;
        res[0] = scr[0] / 2; res[1] = mx; res[2] = scr[1]; res[3] = lg; res[4] = sm; res[5] = tot; res[6] = scr[2];
    }
}

// Device address of g_scratch, looked up once per device with that device
// current (a host-side reference to g_scratch is only a stand-in symbol).
static long long* scratch_ptr(int* status) {
    static long long* ptrs[64] = {};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_last_error("jet_pstat_noalloc: no usable current device");
        *status = JET_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("jet_pstat_noalloc: scratch array lookup failed: ") + cudaGetErrorString(e));
            *status = JET_ERR_CUDA;
            return nullptr;
        }
        ptrs[dev] = (long long*)p;
    }
    *status = JET_OK;
    return ptrs[dev];
}

static int cuda_fail(const char* where, cudaError_t e) {
    set_last_error(std::string("jet_pstat_noalloc: ") + where + ": " + cudaGetErrorString(e));
    return JET_ERR_CUDA;
}

template <class O, class E, class W>
static int run(int64_t n, int64_t nnz, const void* row, const void* adj, const void* val, const void* vw, const int32_t* part,
               int32_t k, int64_t* out, cudaStream_t s) {
    int st = JET_OK;
    long long* scr = scratch_ptr(&st);
    if (st != JET_OK) return st;
    cudaError_t e = cudaMemsetAsync(scr, 0, sizeof(long long) * (8 + 2 * (size_t)MAX_PARTS), s);
    if (e != cudaSuccess) return cuda_fail("clearing the scratch array", e);
    if (n > 0) {
        int sms = device_info().sms;
        int64_t blocks = (n + WARPS - 1) / WARPS;
        if (blocks > (int64_t)sms * 8) blocks = (int64_t)sms * 8;
        k_pstat_na<O, E, W><<<(unsigned)blocks, WARPS * 32, 0, s>>>((O)n, (const E*)row, (const O*)adj, (const W*)val,
                                                                    (const W*)vw, part, k, scr);
        count_launch();
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail("statistics kernel launch", e);
    }
    k_pstat_na_final<<<1, 1024, 0, s>>>(k, scr);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail("final reduction launch", e);
    long long res[7];
    e = cudaMemcpyAsync(res, scr + 8 + 2 * MAX_PARTS, sizeof(res), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return cuda_fail("copying the results", e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail("stream synchronisation", e);
    if (res[6]) {
        set_last_error("jet_pstat_noalloc: a part id lies outside [0, k)");
        return JET_ERR_INVALID;
    }
    (void)nnz;
    for (int i = 0; i < 6; i++) out[i] = (int64_t)res[i];
    return JET_OK;
}

}  // namespace noalloc
}  // namespace jetb

extern "C" int jet_pstat_noalloc(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                                 const void* vweights, const int32_t* part, int32_t k, int64_t* out, void* stream) {
    using namespace jetb::noalloc;
    if (!out || n < 0 || nnz < 0 || (n > 0 && (!row_map || !part || !vweights)) || (nnz > 0 && (!entries || !values))) {
        jetb::set_last_error("jet_pstat_noalloc: null array or negative size");
        return JET_ERR_INVALID;
    }
    if (k < 1 || k > MAX_PARTS) {  // the scratch array serves at most MAX_PARTS parts
        jetb::set_last_error("jet_pstat_noalloc: num_parts must lie in [1, 16384]");
        return JET_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;  // NULL: the legacy default stream
    switch (tier) {
        case 0: return run<int32_t, int32_t, int32_t>(n, nnz, row_map, entries, values, vweights, part, k, out, s);
        case 1: return run<int32_t, int64_t, int64_t>(n, nnz, row_map, entries, values, vweights, part, k, out, s);
        case 2: return run<int64_t, int64_t, int64_t>(n, nnz, row_map, entries, values, vweights, part, k, out, s);
        default:
            jetb::set_last_error("jet_pstat_noalloc: tier must be 0, 1 or 2");
            return JET_ERR_INVALID;
    }
}
