// Query server: several graphs resident in HBM, BFS/SSSP/MIS requests admitted against a
// device-memory budget, continuous batching across execution slots.
//
// The reference has no serving layer (one query per process run, test/*/run.sh); this is
// the systems layer around the plain entry points. A worker thread owns S execution slots
// (one apspie context, stream and 1/S of the persistent grid each, so batches on different
// slots overlap on the device). Whenever a slot is free it takes the (graph, kind) whose
// oldest pending request is oldest and folds every request of that pair that is waiting
// at that moment into one launch:
//   BFS  -> the batched BFS over up to max_batch sources, each depth row written straight
//           into its request's output buffer; fewer than bfs_min_batch waiting requests
//           (6 by default) run apspie_bfs each instead, which is faster for so few;
//   MIS  -> one apspie_mis (the fixed priorities make every MIS query on a graph the same
//           question), the set copied to every waiting request;
//   SSSP -> apspie_sssp_batch over up to sssp_fold sources (max_batch by default), rows
//           staged and copied into the requests' buffers, when at least sssp_min_batch
//           requests wait; fewer run apspie_sssp each, straight into their outputs. By
//           default graphs of at most 2^19 vertices fold from 4 * sqrt(m / 65536)
//           waiting requests (4 at R-MAT scale 16, 8 at 18: about where one multi-query
//           launch overtakes as many single-source launches); larger graphs do not fold,
//           because the multi-query kernel is throughput-bound and a slot holds only its
//           share of the SMs, while single-source queries spread over all slots.
// A launch is admitted only if resident graphs + the slots' reserved scratch + the batch's
// output staging fit the budget; otherwise it waits for a running launch to finish.
// Requests that arrive while launches run are picked up by the next free slot (no wait for
// a fixed batch boundary). Every answer is computed by the same kernels as the plain path,
// so it is identical whether the request ran alone or in a mix.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "../../include/apspie_server.h"

namespace apspie {
namespace {

using Clock = std::chrono::steady_clock;

struct Graph {
    apspie_csr view;  // device arrays owned below
    int32_t *row_ptr = nullptr, *col_ind = nullptr, *weights = nullptr;
    uint32_t *prio = nullptr;  // MIS priorities: mt19937(seed) outputs
    size_t bytes = 0;
};

struct Request {
    uint64_t ticket;
    int graph, kind, source;
    void *d_out;
    Clock::time_point t_submit;
};

struct Done {
    int status = 0;
    double latency_ms = 0.0;
    bool done = false;
};

struct Slot {
    apspie_ctx *ctx = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    std::vector<Request> batch;
    int kind = 0;
    int status = 0;
    size_t staged_bytes = 0;  // batch output staging counted against the budget
    void *stage = nullptr;
    size_t stage_cap = 0;
    int32_t *d_src = nullptr;  // device copy of a BFS batch's sources
    int src_cap = 0;
};

}  // namespace
}  // namespace apspie

struct apspie_server {
    int device = 0;
    int64_t budget = 0;
    int max_batch = 512;
    int sssp_fold = 1 << 30;  // SSSP requests per launch (also capped by max_batch)
    int bfs_min_batch = 6;     // fewer waiting BFS requests run the single-source kernel
    int sssp_min_batch = 0;    // fewer waiting SSSP requests run the single-source kernel (0: by size)
    std::vector<apspie::Graph> graphs;
    size_t graph_bytes = 0;
    std::vector<apspie::Slot> slots;
    size_t slot_reserve = 0;  // scratch reserved per slot (largest graph)

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<apspie::Request> incoming;
    std::unordered_map<uint64_t, apspie::Done> results;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
    bool started = false;
    apspie_server_stats st{};
    std::string last_error;
};

namespace apspie {
namespace {

// A launch of n requests of `kind` runs the batched kernel when n reaches the kind's
// minimum batch (MIS always folds); smaller launches run the single-source kernel once
// per request, straight into each request's output.
struct MinBatch {
    int bfs, sssp;
};
bool batched(int kind, int n, MinBatch mb) {
    return (kind == APSPIE_QUERY_BFS && n >= mb.bfs) || (kind == APSPIE_QUERY_SSSP && n >= mb.sssp && n > 1);
}
MinBatch min_batch(const apspie_server *s, const apspie_csr &g) {
    int sssp = s->sssp_min_batch;
    if (sssp <= 0)
        sssp = g.m > (1 << 19) ? std::numeric_limits<int>::max()
                               : std::max(2, static_cast<int>(std::lround(4.0 * std::sqrt(g.m / 65536.0))));
    return {s->bfs_min_batch, sssp};
}

// Scratch the launch reserves in the slot's arena.
size_t arena_need(const apspie_csr &g, int kind, int n, MinBatch mb) {
    if (kind == APSPIE_QUERY_MIS) return mis_scratch_need(g.m);
    if (!batched(kind, n, mb)) return traversal_scratch_need(g.m);
    return kind == APSPIE_QUERY_BFS ? bfs_batch_scratch_need(g.m, n) + 8192  // + the row-pointer table
                                    : sssp_batch_scratch_need(g.m, n);
}

// Batched SSSP launches stage their n rows before copying them out (batched BFS writes
// straight into the requests' buffers).
size_t stage_need(const apspie_csr &g, int kind, int n, MinBatch mb) {
    return kind == APSPIE_QUERY_SSSP && batched(kind, n, mb) ? static_cast<size_t>(n) * g.m * 4 : 0;
}

// Device bytes a slot holds now (its arena never shrinks; staging is kept for reuse).
size_t slot_held(const Slot &sl) {
    return static_cast<size_t>(apspie_ctx_scratch_bytes(sl.ctx)) + sl.stage_cap +
           static_cast<size_t>(sl.src_cap) * 4;
}

// Extra device bytes running (kind, n) on the slot would allocate (arena growth keeps
// 1/8 headroom, as scratch_reserve does).
size_t slot_growth(const Slot &sl, const apspie_csr &g, int kind, int n, MinBatch mb) {
    const size_t cur = static_cast<size_t>(apspie_ctx_scratch_bytes(sl.ctx));
    const size_t an = arena_need(g, kind, n, mb);
    const size_t sn = stage_need(g, kind, n, mb);
    return (an > cur ? an + an / 8 - cur : 0) + (sn > sl.stage_cap ? sn - sl.stage_cap : 0) +
           (batched(kind, n, mb) && sl.src_cap < n ? static_cast<size_t>(std::max(n, 512)) * 4 : 0);
}

void finish_batch(apspie_server *s, Slot &sl) {
    const auto now = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    for (const Request &r : sl.batch) {
        Done &d = s->results[r.ticket];
        d.status = sl.status;
        d.latency_ms = std::chrono::duration<double, std::milli>(now - r.t_submit).count();
        d.done = true;
        s->st.completed += 1;
        if (sl.status != APSPIE_OK) s->st.failed += 1;
    }
    s->st.launches += 1;
    sl.batch.clear();
    sl.busy = false;
    sl.staged_bytes = 0;
    s->cv_done.notify_all();
}

// Enqueues the work of one batch on the slot's stream and records its completion event.
void launch_batch(apspie_server *s, Slot &sl) {
    const Graph &g = s->graphs[sl.batch.front().graph];
    apspie_status st = APSPIE_OK;
    const int n = static_cast<int>(sl.batch.size());
    if (sl.kind != APSPIE_QUERY_MIS && !batched(sl.kind, n, min_batch(s, g.view))) {
        for (int i = 0; i < n && st == APSPIE_OK; ++i) {
            const Request &r = sl.batch[i];
            st = sl.kind == APSPIE_QUERY_BFS
                     ? apspie_bfs(sl.ctx, &g.view, r.source, 0, static_cast<int32_t *>(r.d_out), nullptr)
                     : apspie_sssp(sl.ctx, &g.view, r.source, static_cast<int32_t *>(r.d_out), nullptr);
        }
    } else if (sl.kind == APSPIE_QUERY_BFS || sl.kind == APSPIE_QUERY_SSSP) {
        std::vector<int32_t> srcs(n);
        for (int i = 0; i < n; ++i) srcs[i] = sl.batch[i].source;
        const bool staged_rows = sl.kind == APSPIE_QUERY_SSSP;  // BFS writes into the requests' rows
        const size_t rows = staged_rows ? static_cast<size_t>(n) * g.view.m * sizeof(int32_t) : 0;
        if (sl.stage_cap < rows) {
            cudaStreamSynchronize(sl.stream);
            if (sl.stage) cudaFree(sl.stage);
            sl.stage = nullptr;
            sl.stage_cap = 0;
            if (cudaMalloc(&sl.stage, rows) != cudaSuccess) {
                (void)cudaGetLastError();
                st = APSPIE_ERR_OOM;
            } else {
                sl.stage_cap = rows;
            }
        }
        if (st == APSPIE_OK && sl.src_cap < n) {
            cudaStreamSynchronize(sl.stream);
            if (sl.d_src) cudaFree(sl.d_src);
            sl.d_src = nullptr;
            sl.src_cap = 0;
            if (cudaMalloc(&sl.d_src, std::max(n, 512) * sizeof(int32_t)) != cudaSuccess) {
                (void)cudaGetLastError();
                st = APSPIE_ERR_OOM;
            } else {
                sl.src_cap = std::max(n, 512);
            }
        }
        if (st == APSPIE_OK) {
            cudaMemcpyAsync(sl.d_src, srcs.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, sl.stream);
            // the host vector must outlive the copy
            cudaStreamSynchronize(sl.stream);
            if (sl.kind == APSPIE_QUERY_BFS) {
                std::vector<int32_t *> out(n);
                for (int i = 0; i < n; ++i) out[i] = static_cast<int32_t *>(sl.batch[i].d_out);
                st = bfs_batch_impl(sl.ctx, &g.view, sl.d_src, n, 0, nullptr, out.data(), nullptr);
            } else {
                st = apspie_sssp_batch(sl.ctx, &g.view, sl.d_src, n, static_cast<int32_t *>(sl.stage), nullptr);
            }
        }
        if (st == APSPIE_OK && staged_rows)
            for (int i = 0; i < n; ++i)
                cudaMemcpyAsync(sl.batch[i].d_out, static_cast<char *>(sl.stage) + static_cast<size_t>(i) * g.view.m * 4,
                                static_cast<size_t>(g.view.m) * 4, cudaMemcpyDeviceToDevice, sl.stream);
    } else if (sl.kind == APSPIE_QUERY_MIS) {
        uint8_t *first = static_cast<uint8_t *>(sl.batch.front().d_out);
        st = apspie_mis(sl.ctx, &g.view, g.prio, first, nullptr);
        if (st == APSPIE_OK)
            for (int i = 1; i < n; ++i)
                cudaMemcpyAsync(sl.batch[i].d_out, first, g.view.m, cudaMemcpyDeviceToDevice, sl.stream);
    }
    sl.status = st;
    cudaEventRecord(sl.ev, sl.stream);
}

void worker_loop(apspie_server *s) {
    cudaSetDevice(s->device);
    std::map<std::pair<int, int>, std::deque<Request>> pending;  // (graph, kind) -> FIFO
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(s->mu);
            bool any_busy = false;
            for (auto &sl : s->slots) any_busy |= sl.busy;
            bool any_pending = false;
            for (auto &kv : pending) any_pending |= !kv.second.empty();
            if (!any_busy && !any_pending)
                s->cv_work.wait(lock, [&] { return s->stop || !s->incoming.empty(); });
            if (s->stop && s->incoming.empty() && !any_busy && !any_pending) return;
            while (!s->incoming.empty()) {
                Request r = s->incoming.front();
                s->incoming.pop_front();
                pending[{r.graph, r.kind}].push_back(r);
            }
        }
        // retire finished launches
        for (auto &sl : s->slots)
            if (sl.busy && cudaEventQuery(sl.ev) == cudaSuccess) finish_batch(s, sl);
        // admit new launches on free slots, oldest request first
        for (auto &sl : s->slots) {
            if (sl.busy) continue;
            auto best = pending.end();
            for (auto it = pending.begin(); it != pending.end(); ++it)
                if (!it->second.empty() &&
                    (best == pending.end() || it->second.front().t_submit < best->second.front().t_submit))
                    best = it;
            if (best == pending.end()) break;
            const int gi = best->first.first, kind = best->first.second;
            const Graph &g = s->graphs[gi];
            int n = static_cast<int>(best->second.size());
            if (kind != APSPIE_QUERY_MIS) n = std::min(n, s->max_batch);
            if (kind == APSPIE_QUERY_SSSP) n = std::min(n, s->sssp_fold);
            size_t held = s->graph_bytes;
            for (auto &other : s->slots) held += slot_held(other);
            size_t need = slot_growth(sl, g.view, kind, n, min_batch(s, g.view));
            // shrink the batch until its growth fits the budget
            while (n > 1 && held + need > static_cast<size_t>(s->budget)) {
                n /= 2;
                need = slot_growth(sl, g.view, kind, n, min_batch(s, g.view));
            }
            const size_t fixed = held;
            if (held + need > static_cast<size_t>(s->budget)) {
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.deferred += 1;
                break;  // wait for memory to free up
            }
            sl.kind = kind;
            sl.batch.assign(best->second.begin(), best->second.begin() + n);
            best->second.erase(best->second.begin(), best->second.begin() + n);
            sl.busy = true;
            sl.staged_bytes = need;
            launch_batch(s, sl);
            {
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.batched_queries += n;
                s->st.max_batch_seen = std::max<int64_t>(s->st.max_batch_seen, n);
                s->st.peak_bytes = std::max<int64_t>(s->st.peak_bytes, static_cast<int64_t>(fixed + need));
            }
        }
        bool any_busy = false;
        for (auto &sl : s->slots) any_busy |= sl.busy;
        if (any_busy) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_server_create(int device, int64_t memory_budget_bytes, int32_t num_slots, int32_t max_batch,
                                   apspie_server **out) {
    if (!out || memory_budget_bytes <= 0 || num_slots < 1 || num_slots > 16 || max_batch < 1)
        return APSPIE_ERR_INVALID_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return APSPIE_ERR_CUDA;
    apspie_server *s = new apspie_server();
    s->device = device;
    s->budget = memory_budget_bytes;
    s->max_batch = max_batch;
    s->slots.resize(num_slots);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    for (auto &sl : s->slots) {
        if (apspie_ctx_create(device, nullptr, &sl.ctx) != APSPIE_OK ||
            cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) {
            apspie_server_destroy(s);
            return APSPIE_ERR_CUDA;
        }
        sl.ctx->stream = sl.stream;
        // Concurrent persistent grids should all fit on the device at once: each slot's
        // grids take floor(per-SM occupancy / num_slots) blocks per SM, so every grid holds
        // at most 1/num_slots of each SM resource and the slots' grids together fit even
        // when their kernels differ in footprint. (A grid whose blocks could not all be
        // resident would end its wait at a grid barrier with APSPIE_ERR_TIMEOUT, not hang.)
        sl.ctx->grid_share = num_slots;
    }
    *out = s;
    return APSPIE_OK;
}

apspie_status apspie_server_add_graph(apspie_server *s, const apspie_host_csr *g, int32_t symmetric,
                                      uint32_t mis_seed, int32_t *graph_id) {
    if (!s || !g || !graph_id || s->started || g->m <= 0 || g->nnz < 0) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(s->device);
    Graph G;
    const size_t rp = (static_cast<size_t>(g->m) + 1) * 4, ci = static_cast<size_t>(g->nnz) * 4;
    const bool w = g->val_type == APSPIE_VAL_I32 && g->val;
    G.bytes = rp + ci + (w ? ci : 0) + static_cast<size_t>(g->m) * 4;
    if (s->graph_bytes + G.bytes > static_cast<size_t>(s->budget)) return APSPIE_ERR_OOM;
    bool ok = cudaMalloc(&G.row_ptr, rp) == cudaSuccess && cudaMalloc(&G.col_ind, std::max<size_t>(ci, 4)) == cudaSuccess &&
              cudaMalloc(&G.prio, static_cast<size_t>(g->m) * 4) == cudaSuccess &&
              (!w || cudaMalloc(&G.weights, std::max<size_t>(ci, 4)) == cudaSuccess);
    if (!ok) {
        (void)cudaGetLastError();
        cudaFree(G.row_ptr);
        cudaFree(G.col_ind);
        cudaFree(G.prio);
        cudaFree(G.weights);
        return APSPIE_ERR_OOM;
    }
    std::vector<uint32_t> pr(g->m);
    apspie_mt19937_u32(mis_seed, g->m, pr.data());
    cudaMemcpy(G.row_ptr, g->row_ptr, rp, cudaMemcpyHostToDevice);
    cudaMemcpy(G.col_ind, g->col_ind, ci, cudaMemcpyHostToDevice);
    cudaMemcpy(G.prio, pr.data(), static_cast<size_t>(g->m) * 4, cudaMemcpyHostToDevice);
    if (w) cudaMemcpy(G.weights, g->val, ci, cudaMemcpyHostToDevice);
    G.view.m = G.view.n = g->m;
    G.view.nnz = g->nnz;
    G.view.val_type = w ? APSPIE_VAL_I32 : APSPIE_VAL_NONE;
    G.view.row_ptr = G.row_ptr;
    G.view.col_ind = G.col_ind;
    G.view.val = G.weights;
    G.view.flags = symmetric ? APSPIE_CSR_SYMMETRIC : 0u;
    G.view.reserved = 0;
    s->graph_bytes += G.bytes;
    s->slot_reserve = std::max(s->slot_reserve, traversal_scratch_need(G.view.m));
    s->graphs.push_back(G);
    *graph_id = static_cast<int32_t>(s->graphs.size() - 1);
    return APSPIE_OK;
}

apspie_status apspie_server_set_sssp_fold(apspie_server *s, int32_t max_fold) {
    if (!s || s->started || max_fold < 1) return APSPIE_ERR_INVALID_ARG;
    s->sssp_fold = std::min(max_fold, s->max_batch);
    return APSPIE_OK;
}

apspie_status apspie_server_set_bfs_min_batch(apspie_server *s, int32_t min_batch) {
    if (!s || s->started || min_batch < 1) return APSPIE_ERR_INVALID_ARG;
    s->bfs_min_batch = min_batch;
    return APSPIE_OK;
}

apspie_status apspie_server_set_sssp_min_batch(apspie_server *s, int32_t min_batch) {
    if (!s || s->started || min_batch < 0) return APSPIE_ERR_INVALID_ARG;
    s->sssp_min_batch = min_batch;
    return APSPIE_OK;
}

apspie_status apspie_server_start(apspie_server *s) {
    if (!s || s->started) return APSPIE_ERR_INVALID_ARG;
    if (s->graph_bytes + s->slot_reserve * s->slots.size() > static_cast<size_t>(s->budget)) return APSPIE_ERR_OOM;
    // reserve each slot's scratch up front so admission accounting matches the device: the
    // largest launch (a full batch on the largest graph) when the budget allows it, so no
    // arena grows (with a device synchronisation) while requests wait; else the
    // single-query need, and batches then grow it only as far as the budget lets them
    int32_t mmax = 0;
    for (auto &g : s->graphs) mmax = std::max(mmax, g.view.m);
    size_t full = traversal_scratch_need(mmax);
    if (mmax > 0) {
        full = std::max(full, mis_scratch_need(mmax));
        full = std::max(full, bfs_batch_scratch_need(mmax, s->max_batch) + 8192);
        const int fold = std::min(s->sssp_fold, s->max_batch);
        if (fold > 1) full = std::max(full, sssp_batch_scratch_need(mmax, fold));
    }
    const size_t with_headroom = full + full / 8;
    const bool fits = s->graph_bytes + with_headroom * s->slots.size() <= static_cast<size_t>(s->budget);
    for (auto &sl : s->slots) {
        void *base;
        const apspie_status st =
            fits ? scratch_reserve(sl.ctx, full, &base) : apspie_ctx_reserve(sl.ctx, mmax, 0);
        if (st != APSPIE_OK) return APSPIE_ERR_OOM;
    }
    s->started = true;
    s->worker = std::thread(worker_loop, s);
    return APSPIE_OK;
}

apspie_status apspie_server_submit(apspie_server *s, int32_t graph_id, int32_t kind, int32_t source, void *d_out,
                                   uint64_t *ticket) {
    if (!s || !ticket || !d_out || !s->started) return APSPIE_ERR_INVALID_ARG;
    if (graph_id < 0 || graph_id >= static_cast<int32_t>(s->graphs.size())) return APSPIE_ERR_INVALID_ARG;
    if (kind != APSPIE_QUERY_BFS && kind != APSPIE_QUERY_SSSP && kind != APSPIE_QUERY_MIS) return APSPIE_ERR_INVALID_ARG;
    const Graph &g = s->graphs[graph_id];
    if (kind != APSPIE_QUERY_MIS && (source < 0 || source >= g.view.m)) return APSPIE_ERR_INVALID_ARG;
    if (kind == APSPIE_QUERY_SSSP && g.view.val_type != APSPIE_VAL_I32) return APSPIE_ERR_UNSUPPORTED;
    Request r;
    r.graph = graph_id;
    r.kind = kind;
    r.source = source;
    r.d_out = d_out;
    r.t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        r.ticket = s->next_ticket++;
        s->results[r.ticket] = Done();
        s->incoming.push_back(r);
        s->st.submitted += 1;
    }
    s->cv_work.notify_one();
    *ticket = r.ticket;
    return APSPIE_OK;
}

apspie_status apspie_server_wait(apspie_server *s, uint64_t ticket, int32_t timeout_ms, double *latency_ms) {
    if (!s) return APSPIE_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->results.find(ticket);
    if (it == s->results.end()) return APSPIE_ERR_INVALID_ARG;
    const bool ok = s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms < 0 ? 1 << 30 : timeout_ms),
                                        [&] { return s->results[ticket].done; });
    if (!ok) return APSPIE_ERR_TIMEOUT;
    Done d = s->results[ticket];
    s->results.erase(ticket);
    if (latency_ms) *latency_ms = d.latency_ms;
    return static_cast<apspie_status>(d.status);
}

apspie_status apspie_server_poll(apspie_server *s, uint64_t ticket, int32_t *done) {
    if (!s || !done) return APSPIE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->results.find(ticket);
    if (it == s->results.end()) return APSPIE_ERR_INVALID_ARG;
    *done = it->second.done ? 1 : 0;
    return APSPIE_OK;
}

apspie_status apspie_server_get_stats(apspie_server *s, apspie_server_stats *out) {
    if (!s || !out) return APSPIE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->st;
    size_t held = s->graph_bytes;
    for (auto &sl : s->slots) held += slot_held(sl);
    out->resident_bytes = static_cast<int64_t>(held);
    return APSPIE_OK;
}

void apspie_server_destroy(apspie_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    for (auto &sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.stage) cudaFree(sl.stage);
        if (sl.d_src) cudaFree(sl.d_src);
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.ctx) apspie_ctx_destroy(sl.ctx);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    for (auto &g : s->graphs) {
        cudaFree(g.row_ptr);
        cudaFree(g.col_ind);
        cudaFree(g.weights);
        cudaFree(g.prio);
    }
    delete s;
}

}  // extern "C"
