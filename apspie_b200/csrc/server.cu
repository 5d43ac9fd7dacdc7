// Query server: several graphs resident in HBM, BFS/SSSP/MIS requests admitted against a
// device-memory budget, continuous batching across execution slots.
//
// The reference has no serving layer (one query per process run, test/*/run.sh); this is
// the systems layer around the plain entry points. A worker thread owns S execution slots
// (one apspie context, stream and 1/S of the persistent grid each, so launches on
// different slots overlap on the device).
//
// BFS runs on a per-graph engine (msbfs.cu): the batched BFS kernel with 32 * W query
// slots, kept running while requests arrive. The worker posts BFS requests of that graph
// into the engine's host-mapped ring; at every level boundary the kernel retires the
// queries whose frontier died (the worker sees each completion as soon as it is posted)
// and admits waiting requests into the freed query slots, so a request that arrives while
// others are on the GPU joins the running launch at the next level instead of waiting
// for a whole batch. When fewer than bfs_min_batch BFS requests wait on a graph with no
// engine running, they run apspie_bfs each instead (faster for so few).
//   MIS  -> one apspie_mis (the fixed priorities make every MIS query on a graph the same
//           question), the set copied to every waiting request;
//   SSSP -> apspie_sssp_batch over up to sssp_fold sources, rows staged and copied into
//           the requests' buffers, when at least sssp_min_batch requests wait; fewer run
//           apspie_sssp each. By default graphs of at most 2^19 vertices fold from
//           4 * sqrt(m / 65536) waiting requests; larger graphs do not fold (the
//           multi-query kernel is throughput-bound and a slot holds only its share of the
//           SMs, while single-source queries spread over all slots).
// A BFS or SSSP request whose source has no edges is answered without a slot: one small
// kernel writes 0 at the source and -1 elsewhere, which is what the traversal returns.
// A free slot takes the (graph, kind) whose oldest waiting request is oldest. A launch is
// admitted only if resident graphs + the slots' scratch + the launch's own growth fit the
// budget; otherwise it shrinks (fewer requests, or fewer engine query slots) or waits for
// a running launch to finish. Single-source requests run at most kSingleSourcePerLaunch per
// slot launch. An engine stops admitting (finishes its queries and leaves the slot) once
// other work has waited for a slot longer than it has run, or when its waiting requests
// outgrow its query slots (it is relaunched with more), but only after kEngineMinRun; an
// engine started while nothing else runs or waits takes the whole device. Launches whose
// device-side wait ran out (a persistent grid that could not be co-resident, e.g. on a
// GPU shared with other work) are retried with half the grid. Every answer is computed by
// the same kernels as the plain path, so it is identical whether the request ran alone or
// in a mix.
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

struct Request {
    uint64_t ticket;
    int graph, kind, source;
    void *d_out;
    Clock::time_point t_submit;
};

struct Graph {
    apspie_csr view;  // device arrays owned below
    int32_t *row_ptr = nullptr, *col_ind = nullptr, *weights = nullptr;
    uint32_t *prio = nullptr;  // MIS priorities: mt19937(seed) outputs
    size_t bytes = 0;
    std::vector<int32_t> deg;  // host copy of the degrees (sources without edges)
    BfsEngine *eng = nullptr;  // BFS engine (ring in host-mapped memory)
    int eng_slot = -1;         // slot the engine runs on, -1 when not running
    int eng_W = 0;
    bool eng_accepting = false;
    Clock::time_point eng_t0;
    std::unordered_map<uint64_t, Request> in_engine;  // posted, not yet completed
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
    int engine_graph = -1;  // the launch is this graph's BFS engine
    void *stage = nullptr;
    size_t stage_cap = 0;
    int32_t *d_src = nullptr;  // device copy of a batch's sources
    int src_cap = 0;
    int retries = 0;
    int share = 1;  // the slot's persistent grids take 1/share of the device (doubled on a timeout)
};

constexpr int kSingleSourcePerLaunch = 16;
constexpr std::chrono::microseconds kEngineMinRun(5000);

// Rows answered without a traversal: sources without edges.
constexpr int kTrivialMax = 64;
struct TrivialArgs {
    int n, m;
    int src[kTrivialMax];
    int *row[kTrivialMax];
};

// Every entry -1 but the source's 0. Rows whose start is 16-byte aligned are written four
// entries per store.
__global__ void trivial_rows(TrivialArgs t) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (int k = 0; k < t.n; ++k) {
        int *row = t.row[k];
        const int src = t.src[k];
        int done = 0;
        if ((reinterpret_cast<uintptr_t>(row) & 15u) == 0) {
            const int n4 = t.m >> 2;
            for (int i = tid; i < n4; i += stride) {
                int4 x = make_int4(-1, -1, -1, -1);
                if (i == src >> 2) {
                    const int lane = src & 3;
                    x.x = lane == 0 ? 0 : -1;
                    x.y = lane == 1 ? 0 : -1;
                    x.z = lane == 2 ? 0 : -1;
                    x.w = lane == 3 ? 0 : -1;
                }
                reinterpret_cast<int4 *>(row)[i] = x;
            }
            done = n4 << 2;
        }
        for (int i = done + tid; i < t.m; i += stride) row[i] = i == src ? 0 : -1;
    }
}

struct TrivialLaunch {
    cudaEvent_t ev;
    std::vector<Request> reqs;
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
    cudaStream_t triv_stream = nullptr;
    std::deque<apspie::TrivialLaunch> trivial;
    std::vector<cudaEvent_t> free_events;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<apspie::Request> incoming;
    std::unordered_map<uint64_t, apspie::Done> results;
    std::deque<uint64_t> completed_order;  // completion order, for take_completed
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
    bool started = false;
    apspie_server_stats st{};
    std::string last_error;
};

namespace apspie {
namespace {

// A launch of n requests of `kind` runs a batched kernel when n reaches the kind's
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

// Scratch a launch reserves in the slot's arena (a BFS batch runs on the engine).
size_t arena_need(const apspie_csr &g, int kind, int n, MinBatch mb) {
    if (kind == APSPIE_QUERY_MIS) return mis_scratch_need(g.m);
    if (!batched(kind, n, mb)) return traversal_scratch_need(g.m);
    return kind == APSPIE_QUERY_BFS ? bfs_engine_scratch_need(g.m, bfs_engine_words(n))
                                    : sssp_batch_scratch_need(g.m, n);
}

// Batched SSSP launches stage their n rows before copying them out (the BFS engine writes
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
    const bool src_copy = kind == APSPIE_QUERY_SSSP && batched(kind, n, mb);
    return (an > cur ? an + an / 8 - cur : 0) + (sn > sl.stage_cap ? sn - sl.stage_cap : 0) +
           (src_copy && sl.src_cap < n ? static_cast<size_t>(std::max(n, 512)) * 4 : 0);
}

// Records one request's outcome (caller holds s->mu).
void complete_locked(apspie_server *s, const Request &r, int status, Clock::time_point now) {
    Done &d = s->results[r.ticket];
    d.status = status;
    d.latency_ms = std::chrono::duration<double, std::milli>(now - r.t_submit).count();
    d.done = true;
    s->completed_order.push_back(r.ticket);
    s->st.completed += 1;
    if (status != APSPIE_OK) s->st.failed += 1;
}

// Device status of the slot's last launch (its stream is idle): a device-side error
// raised by an asynchronous call, else OK.
apspie_status slot_device_status(Slot &sl) { return apspie_ctx_synchronize(sl.ctx); }

void finish_batch(apspie_server *s, Slot &sl, std::map<std::pair<int, int>, std::deque<Request>> &pending) {
    int status = sl.status;
    if (status == APSPIE_OK) status = slot_device_status(sl);
    if (status == APSPIE_OK) sl.retries = 0;
    if (status == APSPIE_ERR_TIMEOUT && sl.retries < 3) {
        // a persistent grid did not get all of its blocks at once: retry on half the grid
        sl.share *= 2;
        ++sl.retries;
        auto &q = pending[{sl.batch.front().graph, sl.kind}];
        for (auto it = sl.batch.rbegin(); it != sl.batch.rend(); ++it) q.push_front(*it);
        std::lock_guard<std::mutex> lock(s->mu);
        s->st.launches += 1;
    } else {
        const auto now = Clock::now();
        std::lock_guard<std::mutex> lock(s->mu);
        for (const Request &r : sl.batch) complete_locked(s, r, status, now);
        s->st.launches += 1;
        s->cv_done.notify_all();
    }
    sl.batch.clear();
    sl.busy = false;
}

// Enqueues the work of one batch (SSSP, MIS, or a few single-source BFS) on the slot's
// stream and records its completion event.
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
    } else if (sl.kind == APSPIE_QUERY_SSSP) {
        std::vector<int32_t> srcs(n);
        for (int i = 0; i < n; ++i) srcs[i] = sl.batch[i].source;
        const size_t rows = static_cast<size_t>(n) * g.view.m * sizeof(int32_t);
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
            st = apspie_sssp_batch(sl.ctx, &g.view, sl.d_src, n, static_cast<int32_t *>(sl.stage), nullptr);
        }
        if (st == APSPIE_OK)
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

// Posts waiting BFS requests of graph gi into its engine's ring; returns how many.
int feed_engine(apspie_server *s, int gi, std::deque<Request> &q) {
    Graph &g = s->graphs[gi];
    int n = 0;
    while (!q.empty() && bfs_engine_post(g.eng, q.front().source, static_cast<int *>(q.front().d_out), q.front().ticket)) {
        g.in_engine.emplace(q.front().ticket, q.front());
        q.pop_front();
        ++n;
    }
    return n;
}

// Collects the engine's posted completions.
void engine_completions(apspie_server *s, Graph &g) {
    unsigned long long ids[512];
    for (;;) {
        const int n = bfs_engine_completions(g.eng, ids, 512);
        if (n == 0) return;
        const auto now = Clock::now();
        std::lock_guard<std::mutex> lock(s->mu);
        for (int i = 0; i < n; ++i) {
            auto it = g.in_engine.find(ids[i]);
            if (it == g.in_engine.end()) continue;
            complete_locked(s, it->second, APSPIE_OK, now);
            g.in_engine.erase(it);
        }
        s->cv_done.notify_all();
    }
}

// Answers requests whose source has no edges (BFS / SSSP) without a slot.
void launch_trivial(apspie_server *s, std::vector<Request> &reqs) {
    size_t i = 0;
    while (i < reqs.size()) {
        TrivialLaunch tl;
        TrivialArgs t;
        t.m = s->graphs[reqs[i].graph].view.m;
        t.n = 0;
        while (i < reqs.size() && t.n < kTrivialMax && s->graphs[reqs[i].graph].view.m == t.m) {
            t.src[t.n] = reqs[i].source;
            t.row[t.n] = static_cast<int *>(reqs[i].d_out);
            ++t.n;
            tl.reqs.push_back(reqs[i]);
            ++i;
        }
        // 64-thread blocks: they fit beside a persistent grid (see side_room)
        const int blocks = std::min(2048, (t.m + 63) / 64);
        trivial_rows<<<blocks, 64, 0, s->triv_stream>>>(t);
        if (s->free_events.empty()) {
            cudaEvent_t ev;
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            s->free_events.push_back(ev);
        }
        tl.ev = s->free_events.back();
        s->free_events.pop_back();
        cudaEventRecord(tl.ev, s->triv_stream);
        s->trivial.push_back(std::move(tl));
    }
    reqs.clear();
}

void retire_trivial(apspie_server *s) {
    while (!s->trivial.empty() && cudaEventQuery(s->trivial.front().ev) == cudaSuccess) {
        TrivialLaunch &tl = s->trivial.front();
        const auto now = Clock::now();
        {
            std::lock_guard<std::mutex> lock(s->mu);
            for (const Request &r : tl.reqs) complete_locked(s, r, APSPIE_OK, now);
            s->st.launches += 1;
            s->cv_done.notify_all();
        }
        s->free_events.push_back(tl.ev);
        s->trivial.pop_front();
    }
}

// An engine's launch ended. Requests still waiting in its ring go back to the front of the
// graph's BFS queue (the next launch posts them again); after a device-side error so do
// the queries the launch took but did not finish (a timeout is retried on half the grid,
// up to three times, then the requests fail).
void engine_ended(apspie_server *s, Slot &sl, std::map<std::pair<int, int>, std::deque<Request>> &pending) {
    const int gi = sl.engine_graph;
    Graph &g = s->graphs[gi];
    engine_completions(s, g);
    apspie_run_stats rs;
    // the control block back (levels run) and the launch's device status
    apspie_status st = finish_call(sl.ctx, &rs, "bfs engine");
    if (st == APSPIE_OK) st = slot_device_status(sl);
    std::vector<Request> back;
    for (unsigned long long id : bfs_engine_take_back(g.eng)) {
        auto it = g.in_engine.find(id);
        if (it == g.in_engine.end()) continue;
        back.push_back(it->second);
        g.in_engine.erase(it);
    }
    bool fail = false;
    if (st != APSPIE_OK) {
        std::vector<Request> taken;
        for (auto &kv : g.in_engine) taken.push_back(kv.second);
        g.in_engine.clear();
        back.insert(back.end(), taken.begin(), taken.end());
        std::sort(back.begin(), back.end(), [](const Request &a, const Request &b) { return a.ticket < b.ticket; });
        if (st == APSPIE_ERR_TIMEOUT && sl.retries < 3) {
            sl.share *= 2;
            ++sl.retries;
        } else {
            fail = true;
        }
    } else {
        sl.retries = 0;
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->st.launches += 1;
        s->st.engine_launches += 1;
        s->st.engine_levels += rs.iterations;
        if (fail) {
            const auto now = Clock::now();
            for (const Request &r : back) complete_locked(s, r, st, now);
            back.clear();
            s->cv_done.notify_all();
        }
    }
    auto &q = pending[{gi, APSPIE_QUERY_BFS}];
    for (auto it = back.rbegin(); it != back.rend(); ++it) q.push_front(*it);
    g.eng_slot = -1;
    g.eng_accepting = false;
    sl.engine_graph = -1;
    sl.busy = false;
}

void worker_loop(apspie_server *s) {
    cudaSetDevice(s->device);
    std::map<std::pair<int, int>, std::deque<Request>> pending;  // (graph, kind) -> FIFO
    std::vector<Request> triv;
    for (;;) {
        bool any_busy = false, any_pending = false, any_outstanding = !s->trivial.empty();
        for (auto &sl : s->slots) any_busy |= sl.busy;
        for (auto &kv : pending) any_pending |= !kv.second.empty();
        for (auto &g : s->graphs) any_outstanding |= !g.in_engine.empty();
        {
            std::unique_lock<std::mutex> lock(s->mu);
            if (!any_busy && !any_pending && !any_outstanding)
                s->cv_work.wait(lock, [&] { return s->stop || !s->incoming.empty(); });
            if (s->stop && s->incoming.empty() && !any_busy && !any_pending && !any_outstanding) return;
            while (!s->incoming.empty()) {
                Request r = s->incoming.front();
                s->incoming.pop_front();
                const Graph &g = s->graphs[r.graph];
                if (r.kind != APSPIE_QUERY_MIS && g.deg[r.source] == 0)
                    triv.push_back(r);
                else
                    pending[{r.graph, r.kind}].push_back(r);
            }
        }
        if (!triv.empty()) {
            {
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.trivial += static_cast<int64_t>(triv.size());
            }
            launch_trivial(s, triv);
        }
        retire_trivial(s);
        // engines: completions, and launches that ended
        for (auto &g : s->graphs)
            if (g.eng && (g.eng_slot >= 0 || !g.in_engine.empty())) engine_completions(s, g);
        for (auto &sl : s->slots) {
            if (!sl.busy || cudaEventQuery(sl.ev) != cudaSuccess) continue;
            if (sl.engine_graph >= 0)
                engine_ended(s, sl, pending);
            else
                finish_batch(s, sl, pending);
        }
        // BFS requests of a graph whose engine runs go straight into its ring
        for (auto &kv : pending) {
            if (kv.first.second != APSPIE_QUERY_BFS || kv.second.empty()) continue;
            Graph &g = s->graphs[kv.first.first];
            if (g.eng_slot >= 0 && g.eng_accepting) {
                const int n = feed_engine(s, kv.first.first, kv.second);
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.joined_running += n;
                s->st.batched_queries += n;
            }
        }
        // admit new launches on free slots, oldest request first
        bool starved = false;  // work waits while every slot is busy
        for (auto &sl : s->slots) {
            if (sl.busy) continue;
            auto best = pending.end();
            for (auto it = pending.begin(); it != pending.end(); ++it) {
                if (it->second.empty()) continue;
                const Graph &g = s->graphs[it->first.first];
                if (it->first.second == APSPIE_QUERY_BFS && g.eng_slot >= 0) continue;  // draining engine
                if (best == pending.end() || it->second.front().t_submit < best->second.front().t_submit) best = it;
            }
            if (best == pending.end()) break;
            const int gi = best->first.first, kind = best->first.second;
            Graph &g = s->graphs[gi];
            const MinBatch mb = min_batch(s, g.view);
            int n = static_cast<int>(best->second.size());
            if (kind != APSPIE_QUERY_MIS) n = std::min(n, s->max_batch);
            if (kind == APSPIE_QUERY_SSSP) n = std::min(n, s->sssp_fold);
            // an engine gets query slots for twice the waiting requests (arrivals join it)
            if (kind == APSPIE_QUERY_BFS && batched(kind, n, mb)) n = std::min(s->max_batch, std::max(2 * n, 32));
            size_t held = s->graph_bytes;
            for (auto &other : s->slots) held += slot_held(other);
            size_t need = slot_growth(sl, g.view, kind, n, mb);
            // shrink the launch until its growth fits the budget
            while (n > 1 && held + need > static_cast<size_t>(s->budget)) {
                n /= 2;
                need = slot_growth(sl, g.view, kind, n, mb);
            }
            if (held + need > static_cast<size_t>(s->budget)) {
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.deferred += 1;
                break;  // wait for memory to free up
            }
            sl.busy = true;
            sl.ctx->grid_share = sl.share;
            if (kind == APSPIE_QUERY_BFS && batched(kind, n, mb)) {
                const int W = bfs_engine_words(n);
                feed_engine(s, gi, best->second);
                // an engine that starts while nothing else runs or waits takes the whole
                // device; work arriving later waits for it to drain (it is drained for such
                // work after kEngineMinRun)
                bool alone = true;
                for (auto &other : s->slots) alone &= &other == &sl || !other.busy;
                for (auto &kv : pending)
                    alone &= kv.second.empty() || (kv.first.first == gi && kv.first.second == APSPIE_QUERY_BFS);
                if (alone) sl.ctx->grid_share = std::max(1, sl.share / static_cast<int>(s->slots.size()));
                const apspie_status st = bfs_engine_launch(sl.ctx, &g.view, W, g.eng);
                if (st != APSPIE_OK) {
                    // the launch never started: every request in its ring fails
                    (void)bfs_engine_take_back(g.eng);
                    std::vector<Request> back;
                    for (auto &kv : g.in_engine) back.push_back(kv.second);
                    g.in_engine.clear();
                    const auto now = Clock::now();
                    std::lock_guard<std::mutex> lock(s->mu);
                    for (const Request &r : back) complete_locked(s, r, st, now);
                    s->cv_done.notify_all();
                    sl.busy = false;
                    continue;
                }
                cudaEventRecord(sl.ev, sl.stream);
                sl.engine_graph = gi;
                g.eng_slot = static_cast<int>(&sl - s->slots.data());
                g.eng_W = W;
                g.eng_accepting = true;
                g.eng_t0 = Clock::now();
                std::lock_guard<std::mutex> lock(s->mu);
                s->st.batched_queries += static_cast<int64_t>(g.in_engine.size());
                s->st.max_batch_seen = std::max<int64_t>(s->st.max_batch_seen, 32 * W);
                s->st.peak_bytes = std::max<int64_t>(s->st.peak_bytes, static_cast<int64_t>(held + need));
                continue;
            }
            // requests that run one single-source launch each: a few per slot launch, so
            // that slots turn over (a scale-22 SSSP takes about 2 ms)
            if (!batched(kind, n, mb) && kind != APSPIE_QUERY_MIS) n = std::min(n, kSingleSourcePerLaunch);
            if (kind == APSPIE_QUERY_BFS) n = std::min(n, static_cast<int>(best->second.size()));
            sl.kind = kind;
            sl.engine_graph = -1;
            sl.batch.assign(best->second.begin(), best->second.begin() + n);
            best->second.erase(best->second.begin(), best->second.begin() + n);
            launch_batch(s, sl);
            std::lock_guard<std::mutex> lock(s->mu);
            s->st.batched_queries += n;
            s->st.max_batch_seen = std::max<int64_t>(s->st.max_batch_seen, n);
            s->st.peak_bytes = std::max<int64_t>(s->st.peak_bytes, static_cast<int64_t>(held + need));
        }
        for (auto &kv : pending) {
            if (kv.second.empty()) continue;
            const Graph &g = s->graphs[kv.first.first];
            if (!(kv.first.second == APSPIE_QUERY_BFS && g.eng_slot >= 0 && g.eng_accepting)) starved = true;
        }
        // engines leave their slot when other work has waited longer than they have run,
        // or when their backlog outgrows their query slots (relaunched larger)
        const auto now = Clock::now();
        for (auto &g : s->graphs) {
            if (g.eng_slot < 0 || !g.eng_accepting) continue;
            bool drain = false;
            if (starved) {
                Clock::time_point oldest = now;
                for (auto &kv : pending)
                    if (!kv.second.empty() && !(kv.first.second == APSPIE_QUERY_BFS && &s->graphs[kv.first.first] == &g))
                        oldest = std::min(oldest, kv.second.front().t_submit);
                // other work may wait as long as the engine has run, at least 2 ms, at most
                // 50 ms; an engine always runs kEngineMinRun first (its first levels)
                const auto ran = std::chrono::duration_cast<std::chrono::microseconds>(now - g.eng_t0);
                const auto allow = std::max(std::chrono::microseconds(2000),
                                            std::min(std::chrono::microseconds(50000), ran));
                drain = ran >= kEngineMinRun && now - oldest > allow;
            }
            const int slots = 32 * g.eng_W;
            auto it = pending.find({static_cast<int>(&g - s->graphs.data()), APSPIE_QUERY_BFS});
            const size_t backlog = bfs_engine_waiting(g.eng) + (it == pending.end() ? 0 : it->second.size());
            if (slots < s->max_batch && backlog > static_cast<size_t>(2 * slots) && now - g.eng_t0 >= kEngineMinRun)
                drain = true;
            if (drain) {
                bfs_engine_set_accept(g.eng, 0);
                g.eng_accepting = false;
            }
        }
        bool busy = !s->trivial.empty();
        for (auto &sl : s->slots) busy |= sl.busy;
        if (busy) std::this_thread::sleep_for(std::chrono::microseconds(20));
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
    s->max_batch = std::min(max_batch, 512);
    s->slots.resize(num_slots);
    if (cudaStreamCreateWithFlags(&s->triv_stream, cudaStreamNonBlocking) != cudaSuccess) {
        apspie_server_destroy(s);
        return APSPIE_ERR_CUDA;
    }
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
        // resident ends its wait at a grid barrier with APSPIE_ERR_TIMEOUT; the launch is
        // then retried on half the grid.)
        sl.share = num_slots;
        sl.ctx->grid_share = num_slots;
        // a slot's grid that has the device to itself still leaves room for the answers of
        // sources without edges (a kernel on the side stream) and the caller's kernels
        sl.ctx->side_room = 1;
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
    if (bfs_engine_create(&G.eng) != APSPIE_OK) return APSPIE_ERR_OOM;
    bool ok = cudaMalloc(&G.row_ptr, rp) == cudaSuccess && cudaMalloc(&G.col_ind, std::max<size_t>(ci, 4)) == cudaSuccess &&
              cudaMalloc(&G.prio, static_cast<size_t>(g->m) * 4) == cudaSuccess &&
              (!w || cudaMalloc(&G.weights, std::max<size_t>(ci, 4)) == cudaSuccess);
    if (!ok) {
        (void)cudaGetLastError();
        cudaFree(G.row_ptr);
        cudaFree(G.col_ind);
        cudaFree(G.prio);
        cudaFree(G.weights);
        bfs_engine_destroy(G.eng);
        return APSPIE_ERR_OOM;
    }
    std::vector<uint32_t> pr(g->m);
    apspie_mt19937_u32(mis_seed, g->m, pr.data());
    cudaMemcpy(G.row_ptr, g->row_ptr, rp, cudaMemcpyHostToDevice);
    cudaMemcpy(G.col_ind, g->col_ind, ci, cudaMemcpyHostToDevice);
    cudaMemcpy(G.prio, pr.data(), static_cast<size_t>(g->m) * 4, cudaMemcpyHostToDevice);
    if (w) cudaMemcpy(G.weights, g->val, ci, cudaMemcpyHostToDevice);
    G.deg.resize(g->m);
    for (int i = 0; i < g->m; ++i) G.deg[i] = g->row_ptr[i + 1] - g->row_ptr[i];
    G.view.m = G.view.n = g->m;
    G.view.nnz = g->nnz;
    G.view.val_type = w ? APSPIE_VAL_I32 : APSPIE_VAL_NONE;
    G.view.row_ptr = G.row_ptr;
    G.view.col_ind = G.col_ind;
    G.view.val = G.weights;
    G.view.flags = symmetric ? APSPIE_CSR_SYMMETRIC : 0u;
    G.view.reserved = 0;
    s->graph_bytes += G.bytes;
    s->graphs.push_back(std::move(G));
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

apspie_status apspie_server_set_side_room(apspie_server *s, int32_t on) {
    if (!s || s->started) return APSPIE_ERR_INVALID_ARG;
    for (auto &sl : s->slots) sl.ctx->side_room = on != 0;
    return APSPIE_OK;
}

apspie_status apspie_server_start(apspie_server *s) {
    if (!s || s->started) return APSPIE_ERR_INVALID_ARG;
    // reserve each slot's scratch up front so admission accounting matches the device: the
    // largest launch (an engine with max_batch query slots, or the largest SSSP batch or
    // MIS, on the largest graph) when the budget allows it, so no arena grows (with a
    // device synchronisation) while requests wait; else the single-query need, and
    // launches then grow it only as far as the budget lets them
    int32_t mmax = 0;
    for (auto &g : s->graphs) mmax = std::max(mmax, g.view.m);
    size_t full = traversal_scratch_need(mmax), single = traversal_scratch_need(mmax);
    if (mmax > 0) {
        full = std::max(full, mis_scratch_need(mmax));
        single = std::max(single, mis_scratch_need(mmax));
        full = std::max(full, bfs_engine_scratch_need(mmax, bfs_engine_words(s->max_batch)));
        const int fold = std::min(s->sssp_fold, s->max_batch);
        if (fold > 1) full = std::max(full, sssp_batch_scratch_need(mmax, fold));
    }
    if (s->graph_bytes + (single + single / 8) * s->slots.size() > static_cast<size_t>(s->budget))
        return APSPIE_ERR_OOM;
    const size_t with_headroom = full + full / 8;
    const bool fits = s->graph_bytes + with_headroom * s->slots.size() <= static_cast<size_t>(s->budget);
    for (auto &sl : s->slots) {
        void *base;
        if (scratch_reserve(sl.ctx, fits ? full : single, &base) != APSPIE_OK) return APSPIE_ERR_OOM;
    }
    s->started = true;
    s->worker = std::thread(worker_loop, s);
    return APSPIE_OK;
}

apspie_status apspie_server_submit(apspie_server *s, int32_t graph_id, int32_t kind, int32_t source, void *d_out,
                                   uint64_t *ticket) {
    if (!ticket) return APSPIE_ERR_INVALID_ARG;
    return apspie_server_submit_many(s, 1, &graph_id, &kind, &source, &d_out, ticket);
}

apspie_status apspie_server_submit_many(apspie_server *s, int32_t n, const int32_t *graph_ids, const int32_t *kinds,
                                        const int32_t *sources, void *const *d_outs, uint64_t *tickets) {
    if (!s || n < 0 || !s->started) return APSPIE_ERR_INVALID_ARG;
    if (n == 0) return APSPIE_OK;
    if (!graph_ids || !kinds || !sources || !d_outs || !tickets) return APSPIE_ERR_INVALID_ARG;
    for (int32_t i = 0; i < n; ++i) {
        const int32_t gi = graph_ids[i], kind = kinds[i];
        if (!d_outs[i] || gi < 0 || gi >= static_cast<int32_t>(s->graphs.size())) return APSPIE_ERR_INVALID_ARG;
        if (kind != APSPIE_QUERY_BFS && kind != APSPIE_QUERY_SSSP && kind != APSPIE_QUERY_MIS)
            return APSPIE_ERR_INVALID_ARG;
        const Graph &g = s->graphs[gi];
        if (kind != APSPIE_QUERY_MIS && (sources[i] < 0 || sources[i] >= g.view.m)) return APSPIE_ERR_INVALID_ARG;
        if (kind == APSPIE_QUERY_SSSP && g.view.val_type != APSPIE_VAL_I32) return APSPIE_ERR_UNSUPPORTED;
    }
    const auto now = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        for (int32_t i = 0; i < n; ++i) {
            Request r;
            r.graph = graph_ids[i];
            r.kind = kinds[i];
            r.source = kinds[i] == APSPIE_QUERY_MIS ? 0 : sources[i];
            r.d_out = d_outs[i];
            r.t_submit = now;
            r.ticket = s->next_ticket++;
            s->results[r.ticket] = Done();
            s->incoming.push_back(r);
            tickets[i] = r.ticket;
        }
        s->st.submitted += n;
    }
    s->cv_work.notify_one();
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

apspie_status apspie_server_take_completed(apspie_server *s, int32_t timeout_ms, int32_t cap, uint64_t *tickets,
                                           int32_t *statuses, double *latencies_ms, int32_t *count) {
    if (!s || !count || cap < 1 || !tickets) return APSPIE_ERR_INVALID_ARG;
    *count = 0;
    std::unique_lock<std::mutex> lock(s->mu);
    auto ready = [&] {
        while (!s->completed_order.empty() && s->results.find(s->completed_order.front()) == s->results.end())
            s->completed_order.pop_front();  // already waited individually
        return !s->completed_order.empty();
    };
    if (!s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms < 0 ? 1 << 30 : timeout_ms), ready))
        return APSPIE_ERR_TIMEOUT;
    int n = 0;
    while (n < cap && !s->completed_order.empty()) {
        const uint64_t t = s->completed_order.front();
        s->completed_order.pop_front();
        auto it = s->results.find(t);
        if (it == s->results.end()) continue;
        tickets[n] = t;
        if (statuses) statuses[n] = it->second.status;
        if (latencies_ms) latencies_ms[n] = it->second.latency_ms;
        s->results.erase(it);
        ++n;
    }
    *count = n;
    return APSPIE_OK;
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
    if (s->triv_stream) {
        cudaStreamSynchronize(s->triv_stream);
        cudaStreamDestroy(s->triv_stream);
    }
    for (auto &tl : s->trivial) cudaEventDestroy(tl.ev);
    for (auto ev : s->free_events) cudaEventDestroy(ev);
    for (auto &g : s->graphs) {
        cudaFree(g.row_ptr);
        cudaFree(g.col_ind);
        cudaFree(g.weights);
        cudaFree(g.prio);
        bfs_engine_destroy(g.eng);
    }
    delete s;
}

}  // extern "C"
