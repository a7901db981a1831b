// test_hooks.cu -- entry points that let tests drive the library's failure
// handling without faulting, trapping or hanging a GPU.  No counterpart in
// the reference, which has no failure handling to test (a Metis failure
// exits the process, src/initial_partition.hpp:106-109).
//
//   jet_test_grid_barrier   runs the cooperative level driver's software grid
//                           barrier with a short poll limit; with one block
//                           told not to arrive, every other block's wait must
//                           run out, flag ERRF_SPIN and return, and the call
//                           must report JET_ERR_TIMEOUT with the context
//                           still usable.
//   jet_test_table_overflow inserts `nparts` distinct parts into a shared-
//                           memory connectivity table of `cap` slots with the
//                           table-build insert (smem_table_add); with more
//                           parts than slots the probe bound must flag
//                           ERRF_OVERFLOW (JET_ERR_OVERFLOW), writing nothing
//                           outside the table.
#include "uncoarsen.cuh"
#include <string>

namespace jetb {

void set_last_error(const std::string& msg);

__global__ void k_test_grid_barrier(GridBar* gb, int* err, int absent, long long spin_cap, int rounds, int* passed) {
    if ((int)blockIdx.x == absent) return;  // this block never arrives
    for (int r = 0; r < rounds; r++) {
        if (!grid_sync(gb, err, spin_cap)) return;
        if (threadIdx.x == 0) atomicAdd(passed, 1);
    }
}

template <class W>
__global__ void k_test_table(int cap, int k, int nparts, int* err, int* claimed) {
    extern __shared__ int smem[];
    part_t* keys = (part_t*)smem;
    W* vals = (W*)(smem + ((cap + 1) & ~1));
    for (int s = threadIdx.x; s < cap; s += blockDim.x) { keys[s] = NULL_PART; vals[s] = 0; }
    __syncthreads();
    for (int p = threadIdx.x; p < nparts; p += blockDim.x)
        if (smem_table_add<W>(keys, vals, (part_t)cap, (part_t)k, (part_t)p, (W)1, err)) atomicAdd(claimed, 1);
}

}  // namespace jetb

using namespace jetb;

extern "C" int jet_test_grid_barrier(int blocks, int absent_block, int spin_cap_log2, int rounds, int* passed_out) {
    if (blocks < 1 || blocks > 64 || spin_cap_log2 < 1 || spin_cap_log2 > 26 || rounds < 1 || rounds > 1000)
        return JET_ERR_INVALID;
    struct Buf { GridBar gb; int err; int passed; };
    Buf* d = nullptr;
    if (cudaMalloc(&d, sizeof(Buf)) != cudaSuccess) return JET_ERR_OOM;
    cudaMemset(d, 0, sizeof(Buf));
    GridBar* gb = &d->gb;
    int* err = &d->err;
    int* passed = &d->passed;
    long long cap = 1ll << spin_cap_log2;
    void* args[] = {&gb, &err, &absent_block, &cap, &rounds, &passed};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_test_grid_barrier, dim3(blocks), dim3(128), args, 0, 0);
    count_launch();
    Buf h{};
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(Buf), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_last_error(std::string("jet_test_grid_barrier: ") + cudaGetErrorString(e));
        return JET_ERR_CUDA;
    }
    if (passed_out) *passed_out = h.passed;
    if (h.err & ERRF_SPIN) {
        set_last_error("a bounded grid barrier wait gave up");
        return JET_ERR_TIMEOUT;
    }
    return JET_OK;
}

extern "C" int jet_test_table_overflow(int cap, int k, int nparts, int* claimed_out) {
    if (cap < 1 || cap > 4096 || k < cap || nparts < 0 || nparts > k) return JET_ERR_INVALID;
    int* d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(int)) != cudaSuccess) return JET_ERR_OOM;
    cudaMemset(d, 0, 2 * sizeof(int));
    size_t smem = sizeof(int) * (size_t)((cap + 1) & ~1) + sizeof(int64_t) * (size_t)cap;
    k_test_table<int64_t><<<1, 128, smem>>>(cap, k, nparts, d, d + 1);
    count_launch();
    int h[2] = {0, 0};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        set_last_error(std::string("jet_test_table_overflow: ") + cudaGetErrorString(e));
        return JET_ERR_CUDA;
    }
    if (claimed_out) *claimed_out = h[1];
    if (h[0] & ERRF_OVERFLOW) {
        set_last_error("a connectivity table had no room");
        return JET_ERR_OVERFLOW;
    }
    return JET_OK;
}
