// batch.cu -- many independent partitions at once: the batched entry point
// and the request-serving loop around it.
//
// Each graph is one ordinary partition (the same code path and result as
// jet_partition_*), run by a host worker thread on that worker's own CUDA
// stream.  Several workers keep several graphs' kernels in flight, so small
// graphs that leave most SMs idle on their own fill the GPU together, and one
// graph's host-side Metis call overlaps the others' device work.  Admission
// is by estimated device footprint against a byte budget.
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <cstring>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>
#include "../../include/jet_b200.h"

extern "C" void jet_thread_batch_mode(int on);

namespace {

using clk = std::chrono::steady_clock;

int tier_bytes(int tier, int* ob, int* eb, int* wb) {
    if (tier == 0) { *ob = 4; *eb = 4; *wb = 4; return 1; }
    if (tier == 1) { *ob = 4; *eb = 8; *wb = 8; return 1; }
    if (tier == 2) { *ob = 8; *eb = 8; *wb = 8; return 1; }
    return 0;
}

int64_t footprint(int tier, int64_t n, int64_t nnz, int32_t k) {
    int ob, eb, wb;
    if (!tier_bytes(tier, &ob, &eb, &wb)) return -1;
    int64_t input = (n + 1) * eb + nnz * (ob + wb) + n * wb;
    // coarse hierarchy (kept until refinement) and contraction scratch,
    // refinement state per vertex, connectivity slots (<= nnz), buckets
    int64_t hierarchy = 3 * input + nnz * (ob + wb);
    int64_t per_vertex = n * (int64_t)(12 * ob + 8 * wb + 48);
    int64_t slots = (nnz + n) * (int64_t)(4 + wb) + n * eb;
    int64_t buckets = (int64_t)k * 50 * 128 * wb * 2;
    return input + hierarchy + per_vertex + slots + buckets + ((int64_t)16 << 20);
}

int run_one(int tier, int mem, jet_graph_desc& d, cudaStream_t s) {
    if (tier == 0 || tier == 1) {
        if (d.n < 0 || d.n > INT32_MAX) return JET_ERR_INVALID;
    }
    if (tier == 0) {
        int32_t cut = 0;
        int rc = jet_partition_i32(&d.config, (int32_t)d.n, (const int32_t*)d.row_map, (const int32_t*)d.entries,
                                   (const int32_t*)d.values, (const int32_t*)d.vweights, d.uniform_ew, mem, d.seed, s,
                                   d.part_out, &cut, nullptr);
        d.edge_cut = cut;
        return rc;
    }
    if (tier == 1) {
        int64_t cut = 0;
        int rc = jet_partition_big(&d.config, (int32_t)d.n, (const int64_t*)d.row_map, (const int32_t*)d.entries,
                                   (const int64_t*)d.values, (const int64_t*)d.vweights, d.uniform_ew, mem, d.seed, s,
                                   d.part_out, &cut, nullptr);
        d.edge_cut = cut;
        return rc;
    }
    if (tier == 2) {
        int64_t cut = 0;
        int rc = jet_partition_biggest(&d.config, d.n, (const int64_t*)d.row_map, (const int64_t*)d.entries,
                                       (const int64_t*)d.values, (const int64_t*)d.vweights, d.uniform_ew, mem, d.seed, s,
                                       d.part_out, &cut, nullptr);
        d.edge_cut = cut;
        return rc;
    }
    return JET_ERR_INVALID;
}

int64_t nnz_of(int tier, int mem, const jet_graph_desc& d) {
    if (!d.row_map || d.n < 0) return 0;
    int64_t m = 0;
    if (mem == JET_MEM_HOST) {
        m = tier == 0 ? (int64_t)((const int32_t*)d.row_map)[d.n] : ((const int64_t*)d.row_map)[d.n];
    } else if (tier == 0) {
        int32_t v = 0;
        cudaMemcpy(&v, (const int32_t*)d.row_map + d.n, sizeof(v), cudaMemcpyDeviceToHost);
        m = v;
    } else {
        cudaMemcpy(&m, (const int64_t*)d.row_map + d.n, sizeof(m), cudaMemcpyDeviceToHost);
    }
    return m;
}

}  // namespace

struct jet_server {
    struct Req {
        jet_graph_desc d;
        int64_t fp = 0;
        clk::time_point submit;
        bool done = false;
    };
    int tier = 0, mem = 0, device = 0;
    int64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, Req> reqs;
    int64_t next_ticket = 0, in_use = 0;
    int inflight = 0;
    bool stop = false;
    jet_server_stats st = {};
    std::vector<std::thread> threads;

    void worker() {
        cudaSetDevice(device);
        jet_thread_batch_mode(1);
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) s = nullptr;
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            // oldest first; it waits until its footprint fits (no overtaking)
            cv_work.wait(lk, [&] {
                if (queue.empty()) return stop;
                const Req& r = reqs[queue.front()];
                return in_use + r.fp <= budget || inflight == 0;
            });
            if (queue.empty()) break;
            int64_t t = queue.front();
            queue.pop_front();
            Req& r = reqs[t];
            in_use += r.fp;
            inflight++;
            if (in_use > st.peak_footprint_bytes) st.peak_footprint_bytes = in_use;
            if (inflight > st.peak_concurrent) st.peak_concurrent = inflight;
            jet_graph_desc d = r.d;
            int64_t fp = r.fp;
            auto t_submit = r.submit;
            lk.unlock();
            int rc = s ? run_one(tier, mem, d, s) : JET_ERR_CUDA;
            auto t_end = clk::now();
            d.error[0] = 0;
            if (rc != JET_OK) {
                const char* msg = s ? jet_last_error() : "worker stream creation failed";
                std::strncpy(d.error, msg ? msg : "", sizeof(d.error) - 1);
                d.error[sizeof(d.error) - 1] = 0;
            }
            lk.lock();
            Req& r2 = reqs[t];
            r2.d = d;
            r2.d.status = rc;
            r2.d.latency_ms = std::chrono::duration<double, std::milli>(t_end - t_submit).count();
            r2.done = true;
            in_use -= fp;
            inflight--;
            if (rc == JET_OK) st.completed++; else st.failed++;
            cv_done.notify_all();
            cv_work.notify_all();
        }
        lk.unlock();
        if (s) cudaStreamDestroy(s);
    }

    // Queues a request; `at` is its submission time (the batch start for
    // jet_partition_batch).
    int64_t submit(const jet_graph_desc& d, clk::time_point at) {
        int64_t m = nnz_of(tier, mem, d);
        int64_t fp = footprint(tier, d.n, m, d.config.num_parts);
        std::lock_guard<std::mutex> lk(mu);
        st.submitted++;
        if (fp < 0) { st.refused++; return -(int64_t)JET_ERR_INVALID; }
        if (fp > budget) { st.refused++; return -(int64_t)JET_ERR_OOM; }
        int64_t t = next_ticket++;
        Req& r = reqs[t];
        r.d = d;
        r.d.status = -1;
        r.fp = fp;
        r.submit = at;
        queue.push_back(t);
        cv_work.notify_one();
        return t;
    }

    int wait(int64_t t, jet_graph_desc* out, double timeout_ms) {
        std::unique_lock<std::mutex> lk(mu);
        auto it = reqs.find(t);
        if (it == reqs.end()) return JET_ERR_INVALID;
        auto ready = [&] { return reqs[t].done; };
        if (timeout_ms < 0) cv_done.wait(lk, ready);
        else if (!cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) return JET_ERR_TIMEOUT;
        if (out) *out = reqs[t].d;
        reqs.erase(t);
        return JET_OK;
    }

    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_work.notify_all();
        for (auto& th : threads) th.join();
        threads.clear();
    }
};

extern "C" {

int64_t jet_server_footprint(int tier, int64_t n, int64_t nnz, int32_t num_parts) { return footprint(tier, n, nnz, num_parts); }

jet_server* jet_server_create(int tier, int mem, int workers, int64_t mem_budget_bytes) {
    int ob, eb, wb;
    if (!tier_bytes(tier, &ob, &eb, &wb) || (mem != JET_MEM_HOST && mem != JET_MEM_DEVICE) || mem_budget_bytes <= 0)
        return nullptr;
    jet_server* srv = new jet_server();
    srv->tier = tier;
    srv->mem = mem;
    srv->budget = mem_budget_bytes;
    cudaGetDevice(&srv->device);
    int w = workers > 0 ? workers : 8;
    for (int i = 0; i < w; i++) srv->threads.emplace_back([srv] { srv->worker(); });
    return srv;
}

int64_t jet_server_submit(jet_server* srv, const jet_graph_desc* req) {
    if (!srv || !req) return -(int64_t)JET_ERR_INVALID;
    return srv->submit(*req, clk::now());
}

int jet_server_wait(jet_server* srv, int64_t ticket, jet_graph_desc* out, double timeout_ms) {
    if (!srv) return JET_ERR_INVALID;
    return srv->wait(ticket, out, timeout_ms);
}

int jet_server_stats_get(jet_server* srv, jet_server_stats* out) {
    if (!srv || !out) return JET_ERR_INVALID;
    std::lock_guard<std::mutex> lk(srv->mu);
    *out = srv->st;
    return JET_OK;
}

int jet_server_destroy(jet_server* srv) {
    if (!srv) return JET_ERR_INVALID;
    srv->shutdown();
    delete srv;
    return JET_OK;
}

int jet_partition_batch(int tier, int64_t count, jet_graph_desc* graphs, int mem, int workers) {
    if (count < 0 || (count > 0 && !graphs)) return JET_ERR_INVALID;
    if (count == 0) return JET_OK;
    jet_server* srv = jet_server_create(tier, mem, workers, INT64_MAX);
    if (!srv) return JET_ERR_INVALID;
    // largest first, so the long partitions start early
    std::vector<std::pair<int64_t, int64_t>> order;
    for (int64_t i = 0; i < count; i++) order.push_back({nnz_of(tier, mem, graphs[i]), i});
    std::stable_sort(order.begin(), order.end(), [](auto& a, auto& b) { return a.first > b.first; });
    auto t0 = clk::now();
    std::vector<int64_t> tickets(count, -1);
    for (auto& o : order) tickets[o.second] = srv->submit(graphs[o.second], t0);
    int first_err = JET_OK;
    for (int64_t i = 0; i < count; i++) {
        if (tickets[i] < 0) {
            graphs[i].status = (int32_t)(-tickets[i]);
        } else {
            jet_graph_desc out;
            if (srv->wait(tickets[i], &out, -1.0) == JET_OK) graphs[i] = out;
            else graphs[i].status = JET_ERR_INVALID;
        }
        if (graphs[i].status != JET_OK && first_err == JET_OK) first_err = graphs[i].status;
    }
    jet_server_destroy(srv);
    return first_err;
}

}  // extern "C"
