// batch.cu — many independent worlds advanced together on one GPU, each with its own context.
//
// After the worlds' first step (which tunes each world's multigrid), a batch step is ONE captured CUDA graph: from the
// batch's stream it forks to every world's stream, each branch holds that world's whole step — P1 to P9, the implicit
// step under device control with its conditional loops — and the branches join again. The graph is captured once per
// combination of the worlds' state buffers (two, as the worlds alternate them in step) and replayed; the worlds'
// kernels interleave on the device with no host decision between them. Until then (the first step, or a world whose
// step cannot be captured: the learned preconditioner) the worlds step on a pool of host threads, one context per
// world, balanced by cell count.
#include <map>
#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

struct BatchGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> launches;  // per world, per replay, outside the implicit steps' loops
    std::vector<unsigned> generation;  // the worlds' capture generations it was built at
};

struct sr_batch {
    std::vector<sr_ctx*> ctx;
    std::map<std::vector<int>, BatchGraph> graphs;  // keyed by the worlds' state buffers
    std::vector<std::vector<uint32_t>> share;  // worlds per thread
    cudaStream_t join = nullptr;
    cudaEvent_t start = nullptr, end = nullptr, start_fork = nullptr;
    std::vector<cudaEvent_t> done;
    std::string error;
};

extern "C" cudaStream_t sr_ctx_stream(sr_ctx* c);
long long sr_ctx_capture_step(sr_ctx* c, int cur, cudaStream_t s, cudaGraph_t root);
bool sr_ctx_prepare_capture(sr_ctx* c);
void sr_ctx_graph_steps_done(sr_ctx* c, uint32_t steps, long long launches_per_step);
sr_status sr_ctx_after_steps(sr_ctx* c);
unsigned sr_ctx_generation(const sr_ctx* c);
int sr_ctx_state(const sr_ctx* c);
bool sr_ctx_uploaded(const sr_ctx* c);

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

void drop_graphs(sr_batch* b) {
    if (!b->graphs.empty()) cudaStreamSynchronize(b->join);
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second.exec);
    b->graphs.clear();
}

// The batch step's graph for the worlds' current state buffers, captured on first use (every world must be ready for
// capture); null when some world cannot be captured.
BatchGraph* batch_graph(sr_batch* b) {
    std::vector<int> key;
    for (sr_ctx* c : b->ctx) key.push_back(sr_ctx_state(c));
    auto it = b->graphs.find(key);
    if (it != b->graphs.end()) {
        bool fresh = true;
        for (size_t i = 0; i < b->ctx.size(); i++) fresh &= it->second.generation[i] == sr_ctx_generation(b->ctx[i]);
        if (fresh) return &it->second;
        drop_graphs(b);  // a world's settings changed since
    }
    // the worlds' control blocks are rewritten for the capture (on their own streams): no batch step may still be
    // running on the batch's stream
    SR_CUDA_TRY(cudaStreamSynchronize(b->join));
    for (sr_ctx* c : b->ctx)
        if (!sr_ctx_prepare_capture(c)) return nullptr;
    BatchGraph bg;
    cudaGraph_t g;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) throw SrError{SR_E_CUDA, "batch graph creation failed"};
    SR_CUDA_TRY(cudaStreamBeginCaptureToGraph(b->join, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    try {
        SR_CUDA_TRY(cudaEventRecord(b->start_fork, b->join));
        for (size_t i = 0; i < b->ctx.size(); i++) {
            cudaStream_t ws = sr_ctx_stream(b->ctx[i]);
            SR_CUDA_TRY(cudaStreamWaitEvent(ws, b->start_fork, 0));
            bg.launches.push_back(sr_ctx_capture_step(b->ctx[i], key[i], ws, g));
            bg.generation.push_back(sr_ctx_generation(b->ctx[i]));
            SR_CUDA_TRY(cudaEventRecord(b->done[i], ws));
            SR_CUDA_TRY(cudaStreamWaitEvent(b->join, b->done[i], 0));
        }
    } catch (...) {
        cudaGraph_t dead;
        cudaStreamEndCapture(b->join, &dead);
        cudaGraphDestroy(g);
        throw;
    }
    cudaGraph_t out;
    SR_CUDA_TRY(cudaStreamEndCapture(b->join, &out));
    const cudaError_t e = cudaGraphInstantiate(&bg.exec, g, 0);
    cudaGraphDestroy(g);
    SR_CUDA_TRY(e);
    return &(b->graphs[key] = bg);
}

// `steps` steps of every world on the pool of host threads (each world's own stream, after `start`).
void pool_steps(sr_batch* b, uint32_t steps, std::vector<sr_status>& status) {
    for (sr_ctx* c : b->ctx) cudaStreamWaitEvent(sr_ctx_stream(c), b->start, 0);
    std::vector<std::thread> pool;
    for (const auto& mine : b->share) {
        pool.emplace_back([&, mine] {
            for (uint32_t i : mine)
                if (status[i] == SR_OK) status[i] = sr_step(b->ctx[i], steps);
        });
    }
    for (auto& t : pool) t.join();
    for (size_t i = 0; i < b->ctx.size(); i++) {
        cudaEventRecord(b->done[i], sr_ctx_stream(b->ctx[i]));
        cudaStreamWaitEvent(b->join, b->done[i], 0);
    }
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
        if (cfgs[i].active_box) {  // a batch step is one graph over its worlds' whole steps: their boxes would refit
            sr_batch_destroy(b);
            sr_set_global_error("world " + std::to_string(i) + ": the active box is a single world's (batch worlds "
                                "step whole)");
            return SR_E_UNSUPPORTED;
        }
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
        cudaEventCreate(&b->start) != cudaSuccess || cudaEventCreate(&b->end) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->start_fork, cudaEventDisableTiming) != cudaSuccess) {
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
    drop_graphs(b);
    if (b->start_fork) cudaEventDestroy(b->start_fork);
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
    for (size_t i = 0; i < b->ctx.size(); i++)
        if (!sr_ctx_uploaded(b->ctx[i])) {
            b->error = "world " + std::to_string(i) + ": no state uploaded";
            sr_set_global_error(b->error);
            return SR_E_INVALID;
        }
    std::vector<sr_status> status(b->ctx.size(), SR_OK);
    cudaEventRecord(b->start, b->join);
    uint32_t done = 0;
    try {
        while (done < steps) {
            BatchGraph* g = batch_graph(b);
            if (!g) {  // a world not ready for capture (its first step tunes its multigrid): one step on the pool
                pool_steps(b, 1, status);
                done++;
                bool bad = false;
                for (sr_status st : status) bad |= st != SR_OK;
                if (bad) break;
                continue;
            }
            SR_CUDA_TRY(cudaGraphLaunch(g->exec, b->join));
            for (size_t i = 0; i < b->ctx.size(); i++) sr_ctx_graph_steps_done(b->ctx[i], 1, g->launches[i]);
            done++;
        }
    } catch (const SrError& e) {
        cudaStreamSynchronize(b->join);
        b->error = e.message;
        sr_set_global_error(b->error);
        return e.status;
    }
    cudaEventRecord(b->end, b->join);
    cudaEventSynchronize(b->end);
    // the worlds' own streams follow the batch (their readbacks and reports)
    for (sr_ctx* c : b->ctx) cudaStreamWaitEvent(sr_ctx_stream(c), b->end, 0);
    for (size_t i = 0; i < b->ctx.size(); i++) {
        if (status[i] == SR_OK) status[i] = sr_ctx_after_steps(b->ctx[i]);
        if (status[i] != SR_OK) {
            b->error = "world " + std::to_string(i) + ": " + sr_last_error(b->ctx[i]);
            sr_set_global_error(b->error);
            return status[i];
        }
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
