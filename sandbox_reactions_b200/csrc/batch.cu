// batch.cu — many independent worlds advanced together on one GPU: one context and stream per world, a pool of host
// threads each stepping its share of the worlds (greedy balance by cell count), so that the worlds' kernels overlap on
// the device and one world's host-side solver decisions never stall the others.
#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

struct sr_batch {
    std::vector<sr_ctx*> ctx;
    std::vector<std::vector<uint32_t>> share;  // worlds per thread
    cudaStream_t join = nullptr;
    cudaEvent_t start = nullptr, end = nullptr;
    std::vector<cudaEvent_t> done;
    std::string error;
};

extern "C" cudaStream_t sr_ctx_stream(sr_ctx* c);

namespace {

// Longest-processing-time-first: worlds sorted by cells, each to the thread with the fewest cells so far.
std::vector<std::vector<uint32_t>> balance(const std::vector<size_t>& cells, uint32_t threads) {
    std::vector<uint32_t> order(cells.size());
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cells[a] > cells[b]; });
    std::vector<std::vector<uint32_t>> share(threads);
    std::vector<size_t> load(threads, 0);
    for (uint32_t i : order) {
        uint32_t t = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
        share[t].push_back(i);
        load[t] += cells[i];
    }
    return share;
}

}  // namespace

extern "C" {

sr_status sr_batch_create(const sr_config* cfgs, uint32_t count, uint32_t threads, sr_batch** out) {
    if (!cfgs || !out || count == 0) {
        sr_set_global_error("sr_batch_create: no worlds");
        return SR_E_INVALID;
    }
    *out = nullptr;
    sr_batch* b = new sr_batch();
    std::vector<size_t> cells;
    for (uint32_t i = 0; i < count; i++) {
        sr_ctx* c = nullptr;
        sr_status st = sr_create(&cfgs[i], &c);
        if (st != SR_OK) {
            std::string msg = std::string("world ") + std::to_string(i) + ": " + sr_last_error(nullptr);
            sr_batch_destroy(b);
            sr_set_global_error(msg);
            return st;
        }
        b->ctx.push_back(c);
        cells.push_back((size_t)cfgs[i].width * cfgs[i].height);
    }
    if (threads == 0) threads = std::min<uint32_t>(count, 16);
    threads = std::min(threads, count);
    b->share = balance(cells, threads);
    if (cudaStreamCreateWithFlags(&b->join, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->start) != cudaSuccess || cudaEventCreate(&b->end) != cudaSuccess) {
        sr_batch_destroy(b);
        sr_set_global_error("sr_batch_create: stream or event creation failed");
        return SR_E_CUDA;
    }
    b->done.resize(count);
    for (auto& e : b->done) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    *out = b;
    return SR_OK;
}

void sr_batch_destroy(sr_batch* b) {
    if (!b) return;
    for (sr_ctx* c : b->ctx) sr_destroy(c);
    for (auto e : b->done) cudaEventDestroy(e);
    if (b->start) cudaEventDestroy(b->start);
    if (b->end) cudaEventDestroy(b->end);
    if (b->join) cudaStreamDestroy(b->join);
    delete b;
}

sr_status sr_batch_upload(sr_batch* b, uint32_t index, const float* planes, const float* kappa) {
    if (!b || index >= b->ctx.size()) return SR_E_INVALID;
    sr_status st = sr_upload(b->ctx[index], planes, 4);
    if (st == SR_OK && kappa) st = sr_upload_opacity(b->ctx[index], kappa);
    if (st != SR_OK) b->error = sr_last_error(b->ctx[index]);
    return st;
}

sr_status sr_batch_step(sr_batch* b, uint32_t steps, double* device_ms) {
    if (!b) return SR_E_INVALID;
    // every world's stream starts after `start`; `end` follows every world's last work
    cudaEventRecord(b->start, b->join);
    for (sr_ctx* c : b->ctx) cudaStreamWaitEvent(sr_ctx_stream(c), b->start, 0);
    std::vector<sr_status> status(b->ctx.size(), SR_OK);
    std::vector<std::thread> pool;
    for (const auto& mine : b->share) {
        pool.emplace_back([&, mine] {
            for (uint32_t i : mine) status[i] = sr_step(b->ctx[i], steps);
        });
    }
    for (auto& t : pool) t.join();
    for (size_t i = 0; i < b->ctx.size(); i++) {
        cudaEventRecord(b->done[i], sr_ctx_stream(b->ctx[i]));
        cudaStreamWaitEvent(b->join, b->done[i], 0);
    }
    cudaEventRecord(b->end, b->join);
    cudaEventSynchronize(b->end);
    for (size_t i = 0; i < b->ctx.size(); i++)
        if (status[i] != SR_OK) {
            b->error = "world " + std::to_string(i) + ": " + sr_last_error(b->ctx[i]);
            sr_set_global_error(b->error);
            return status[i];
        }
    if (device_ms) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, b->start, b->end);
        *device_ms = ms;
    }
    return SR_OK;
}

sr_status sr_batch_readback(sr_batch* b, uint32_t index, float* planes) {
    if (!b || index >= b->ctx.size()) return SR_E_INVALID;
    return sr_readback(b->ctx[index], planes, 4);
}

sr_ctx* sr_batch_ctx(sr_batch* b, uint32_t index) {
    if (!b || index >= b->ctx.size()) return nullptr;
    return b->ctx[index];
}

}  // extern "C"
