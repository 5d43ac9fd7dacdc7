// Shared device/host plumbing for the apspie B200 kernels: the context object, the
// scratch arena, the bounded grid barrier used by the persistent traversal kernels, and
// block-wide scan helpers. sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/apspie.h"

namespace apspie {

constexpr int kTimeline = 128;
constexpr int kBandBins = 256;  // SSSP distance-band histogram bins

// ---------------------------------------------------------------------------------
// Per-call device control block. Reset by the host (one memset) before each launch.
// ---------------------------------------------------------------------------------
struct TravCtl {
    // grid barrier word: arrivals count in the low bits, the phase flips bit 31. It sits
    // next to `err` in one aligned 8-byte pair so a single load returns both.
    unsigned bar;
    int err;             // first apspie_status error raised on the device
    int err_where;       // kernel-defined location code of that error
    unsigned long long wait_limit_ns;  // bound of every grid-barrier wait (0: kBarrierTimeoutNs)
    int qlen[2];         // frontier queue lengths (ping-pong)
    int iterations;
    int push_iterations;
    int pull_iterations;
    int flen[2];         // far-pile lengths (SSSP, ping-pong)
    int delta;           // SSSP bucket width in use
    long long edges_expanded;
    long long edges_component;
    long long vertices_reached;
    long long aux[4];    // kernel-specific counters
    int tl_count;        // phase timeline: block 0 stamps every grid barrier it passes
    int tl_site[kTimeline];
    unsigned long long tl_ns[kTimeline];
    // SSSP distance band (ping-pong with the frontier queues): the least distance in each
    // queue and a degree-weighted histogram of its distances. Device-only.
    int sbase[2];
    unsigned long long shist[2][kBandBins];
    // Per-round list counters of kernels that keep several rounds' lists apart (MIS keeps
    // three: the lists a round fills, reads, and clears for the round after next). Device-only.
    int rcnt[12];
    unsigned long long rcnt64[3];
};
static_assert(offsetof(TravCtl, bar) == 0 && offsetof(TravCtl, err) == 4, "barrier word / error pair");
// Prefix of the control block the host reads back after a call.
constexpr size_t kCtlHostBytes = offsetof(TravCtl, sbase);

// Upper bound on a persistent grid (chunk sums are staged in shared memory).
constexpr int kMaxGrid = 1024;
// A grid barrier gives up after this long (ns) and raises APSPIE_ERR_TIMEOUT, unless the
// context sets another bound (apspie_ctx_set_wait_limit).
constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;

}  // namespace apspie

// Plan of the last apspie_spgemm_symbolic call, reused by the numeric call on the same
// operands while no other call has reserved scratch since (scratch_epoch unchanged).
struct apspie_spgemm_plan_cache {
    bool valid = false;
    unsigned long long epoch = 0;
    apspie_csr a{}, b{};
    void *dev[8] = {};        // plan buffers inside the scratch arenas
    long long host[12] = {};  // bin counts and sizes read back at planning
};

// One tuning-table entry: the knobs the autotuner chose for a (kind, shape bucket).
struct apspie_tune_entry {
    int kind, log_m, log_deg, symmetric;
    apspie_tune_params p;
    double ms;
};

struct apspie_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    std::string last_error;
    // scratch arena: one device allocation, carved per call, grown on demand
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    unsigned long long scratch_epoch = 0;  // bumped by every scratch reservation
    apspie_spgemm_plan_cache sg_cache;
    // secondary arena for variable-size tables (SpGEMM global tier, ...)
    void *scratch2 = nullptr;
    size_t scratch2_bytes = 0;
    // control block (device) + pinned host mirror
    apspie::TravCtl *d_ctl = nullptr;
    apspie::TravCtl *h_ctl = nullptr;
    int *d_sticky_err = nullptr;  // errors of asynchronous calls, read by synchronize
    int *h_word = nullptr;        // pinned scratch word for small device->host reads
    int validate = 0;
    float bfs_alpha = 14.0f;
    float bfs_beta = 24.0f;
    int sssp_delta = 0;  // <= 0: chosen on the device
    long long sssp_band = 0;  // 0: auto, < 0: off
    int max_grid = 0;    // 0: as many co-resident blocks as fit
    int grid_share = 1;  // persistent grids take 1/grid_share of the co-resident capacity
    int side_room = 0;   // persistent grids with the device to themselves leave kSideRoomRegs per SM
    float batch_push_frac = 0.05f;  // batched BFS: push while frontier edges < frac * nnz
    int spgemm_reg_max = 128;       // SpGEMM register tier: rows of <= this many products
    int spgemm_block_max = 1024;    // SpGEMM shared-table tier: rows of <= this many products
    int tc_task_work = 4096;        // TC wedges per warp task
    int tc_orient = 1;              // TC: re-orient L by degree
    int sssp_batch_groups = 0;      // batched SSSP: <= 0 multi-query kernel, > 0 query groups
    int use_tuning = 1;             // consult tune_table
    unsigned long long wait_limit_ns = 0;  // grid-barrier wait bound (0: kBarrierTimeoutNs)
    unsigned long long *h_limit = nullptr;  // pinned copy of it, the source of the per-call upload
    std::vector<apspie_tune_entry> tune_table;
};

namespace apspie {

// ---------------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------------
apspie_status set_error(apspie_ctx *ctx, apspie_status st, const std::string &msg);
apspie_status cuda_error(apspie_ctx *ctx, cudaError_t e, const char *what);
// The knobs a call of `kind` on A uses: the context's own, overridden by its tuning-table
// entry for A's shape bucket when there is one (and use_tuning is on).
apspie_tune_params effective_params(const apspie_ctx *ctx, int kind, const apspie_csr *A);
// Ensures the arena holds `bytes`; returns its base in *out.
apspie_status scratch_reserve(apspie_ctx *ctx, size_t bytes, void **out);
apspie_status scratch2_reserve(apspie_ctx *ctx, size_t bytes, void **out);
// Validates a CSR view on the device (synchronises). Used when ctx->validate is on.
apspie_status validate_csr(apspie_ctx *ctx, const apspie_csr *A, bool need_square);
// Checks host-visible CSR view fields (no device access).
apspie_status check_csr_view(apspie_ctx *ctx, const apspie_csr *A, const char *who);
// Co-resident blocks a persistent kernel with per_sm blocks per SM may launch on ctx.
// With ctx->side_room and the device to itself (grid_share 1), it takes fewer blocks per
// SM until kSideRoomRegs registers per SM stay free (regs_per_block: the kernel's register
// allocation per block), so that small kernels of other streams (the server's answers for
// sources without edges, a caller's own kernels) still find room on every SM.
constexpr int kSmRegs = 65536;        // registers per SM (sm_100a)
constexpr int kSideRoomRegs = 4096;   // e.g. two 64-thread blocks of up to 32 registers
int persistent_cap(const apspie_ctx *ctx, int per_sm, int regs_per_block = 0);
// Cooperative launch of a persistent kernel with the largest co-resident grid.
// `work` (edges the graph holds) sizes the grid: about one block per kWorkPerBlock edges,
// at least one per SM, at most the co-resident limit (barrier cost grows with blocks).
constexpr long long kWorkPerBlock = 4096;
// Clears the control block on the context's stream before a launch and, when the context
// sets its own wait bound, writes that bound into it.
apspie_status reset_ctl(apspie_ctx *ctx);
apspie_status launch_persistent(apspie_ctx *ctx, const void *func, int block, void **args,
                                long long work, int *grid_out = nullptr);
// Copies the control block back, synchronises, and turns a device error into a status.
apspie_status finish_call(apspie_ctx *ctx, apspie_run_stats *stats, const char *who);

// Scratch bytes the entry points reserve in a context's arena (for admission control).
size_t traversal_scratch_need(int m);        // apspie_bfs / apspie_sssp
size_t mis_scratch_need(int m);              // apspie_mis
size_t bfs_batch_scratch_need(int m, int nq);  // apspie_bfs_batch (nq <= 512 per launch)
// apspie_bfs_batch into per-query rows h_rows[q] (host array of device pointers) when
// h_rows is given, else into the query-major d_depths
apspie_status bfs_batch_impl(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources, int32_t num_sources,
                             int32_t depth_cap, int32_t *d_depths, int32_t *const *h_rows, apspie_run_stats *stats);
// The server's continuous BFS engine (msbfs.cu): a persistent batched BFS with 32 * W
// query slots that takes requests from a host-mapped ring at every level and posts each
// query's completion as soon as its frontier dies.
}  // namespace apspie
struct BfsEngine;
namespace apspie {
size_t bfs_engine_scratch_need(int m, int W);
int bfs_engine_words(int slots);  // W for at least `slots` query slots (32..512)
apspie_status bfs_engine_create(BfsEngine **out);
void bfs_engine_destroy(BfsEngine *e);
bool bfs_engine_post(BfsEngine *e, int source, int *row, unsigned long long id);
int bfs_engine_completions(BfsEngine *e, unsigned long long *ids, int cap);
unsigned long long bfs_engine_waiting(const BfsEngine *e);
void bfs_engine_set_accept(BfsEngine *e, int on);
std::vector<unsigned long long> bfs_engine_take_back(BfsEngine *e);  // untaken ring entries (launch ended)
apspie_status bfs_engine_launch(apspie_ctx *ctx, const apspie_csr *A, int W, BfsEngine *e);
size_t sssp_batch_scratch_need(int m, int nq);  // apspie_sssp_batch (nq <= 512 per launch)
// apspie_sssp_batch in query groups (each group of blocks runs single-source SSSPs)
size_t sssp_group_scratch_need(int m, int groups);
int sssp_group_count(const apspie_ctx *ctx, int nq);
apspie_status sssp_batch_grouped(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources, int32_t nq,
                                 int32_t *d_dists, apspie_run_stats *stats);

// Device-wide exclusive scan (scan.cu): out[0..n) = prefix of in, out[n] = total.
size_t scan_scratch_bytes(long long n);
apspie_status device_exclusive_scan(apspie_ctx *ctx, const int *in, long long n, int *out, void *tmp,
                                    int *overflow_flag);

// Carves aligned sub-buffers out of the scratch arena.
struct Carver {
    char *base;
    size_t off = 0;
    explicit Carver(void *b) : base(static_cast<char *>(b)) {}
    template <typename T>
    T *take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T *p = reinterpret_cast<T *>(base + off);
        off += count * sizeof(T);
        return p;
    }
    static size_t need(std::initializer_list<size_t> sizes) {
        size_t o = 0;
        for (size_t s : sizes) o = ((o + 255) & ~size_t(255)) + s;
        return o + 256;
    }
};

// ---------------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------------
#ifdef __CUDACC__

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_volatile_i32(const int *p) {
    return *reinterpret_cast<const volatile int *>(p);
}

// Block 0, thread 0: records (site, globaltimer) in the control block's timeline.
__device__ __forceinline__ void timeline_mark(TravCtl *ctl, int site) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int k = ctl->tl_count;
        if (k < kTimeline) {
            ctl->tl_site[k] = site;
            ctl->tl_ns[k] = globaltimer_ns();
            ctl->tl_count = k + 1;
        }
    }
}

__device__ __forceinline__ void raise_error(TravCtl *ctl, int *sticky, int status, int where) {
    if (atomicCAS(&ctl->err, 0, status) == 0) ctl->err_where = where;
    atomicCAS(sticky, 0, status);
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const void *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// The blocks that cooperate on one traversal: all of a launch's blocks, or one group of
// them when a launch runs several independent traversals side by side.
struct VGrid {
    int id;  // this block's index within the group
    int n;   // blocks in the group
};

__device__ __forceinline__ VGrid hw_grid() { return VGrid{static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x)}; }

// Grid-wide barrier for a cooperatively launched (co-resident) grid: a sense-reversing
// counter. Thread 0 of every block adds 1 to ctl->bar, except block 0, which adds
// 2^31 - (G - 1); the G additions sum to 2^31, so bit 31 flips exactly when the last block
// arrives and the low bits return to where they were (no reset). A waiter polls the pair
// (bar, err) with one 64-bit load until bit 31 differs from what it saw before arriving,
// or until an error is posted. Every wait is bounded (the control block's wait_limit_ns,
// else kBarrierTimeoutNs); on timeout it
// raises APSPIE_ERR_TIMEOUT. Returns false when any block has raised an error, so that all
// blocks leave the persistent loop together instead of hanging.
// With a VGrid group, the group's blocks synchronise on the group's own control block.
__device__ __forceinline__ bool grid_barrier(TravCtl *ctl, int *sticky, int where, VGrid vg = hw_grid()) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned inc = vg.id == 0 ? 0x80000000u - static_cast<unsigned>(vg.n - 1) : 1u;
        __threadfence();
        const unsigned before = atomicAdd(&ctl->bar, inc);
        unsigned long long pair;
        unsigned long long t0 = 0;
        const unsigned long long limit = ctl->wait_limit_ns ? ctl->wait_limit_ns : kBarrierTimeoutNs;
        for (unsigned spin = 1;; ++spin) {
            pair = ld_acquire_u64(&ctl->bar);
            if (((static_cast<unsigned>(pair) ^ before) & 0x80000000u) != 0u) break;
            if ((pair >> 32) != 0ull) break;  // an error was raised: leave now
            if ((spin & 1023u) == 0u) {
                const unsigned long long t = globaltimer_ns();
                if (t0 == 0) {
                    t0 = t;
                } else if (t - t0 > limit) {
                    raise_error(ctl, sticky, APSPIE_ERR_TIMEOUT, where);
                    pair = 1ull << 32;
                    break;
                }
            }
        }
        __threadfence();
        s_ok = (pair >> 32) == 0ull;
        timeline_mark(ctl, where);
    }
    __syncthreads();
    return s_ok != 0;
}

// Block-wide exclusive scan of one int per thread. `tmp` must hold 33 ints.
template <int BLOCK>
__device__ __forceinline__ int block_exclusive_scan(int x, int &total, int *tmp) {
    static_assert(BLOCK % 32 == 0 && BLOCK <= 1024, "block size");
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) tmp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int w = lane < NW ? tmp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < NW) tmp[lane] = wi - w;  // exclusive warp base
        if (lane == NW - 1) tmp[32] = wi;   // block total
    }
    __syncthreads();
    int res = tmp[wid] + incl - x;
    total = tmp[32];
    __syncthreads();
    return res;
}

// Block-wide inclusive scan of one 64-bit count per thread; `tmp` must hold 33 values and
// tmp[32] holds the block total on return.
template <int BLOCK>
__device__ __forceinline__ unsigned long long block_inclusive_scan_u64(unsigned long long x,
                                                                      unsigned long long *tmp) {
    static_assert(BLOCK % 32 == 0 && BLOCK <= 1024, "block size");
    constexpr int NW = BLOCK / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) tmp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const unsigned long long w = lane < NW ? tmp[lane] : 0ull;
        unsigned long long wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < NW) tmp[lane] = wi - w;
        if (lane == NW - 1) tmp[32] = wi;
    }
    __syncthreads();
    return tmp[wid] + incl;
}

// Warp-aggregated append of `v` to queue `q` for lanes with pred set. All 32 lanes of
// the warp must call it.
__device__ __forceinline__ void warp_append(bool pred, int v, int *q, int *qlen) {
    unsigned mask = __ballot_sync(0xffffffffu, pred);
    if (mask == 0) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(qlen, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (pred) q[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

// Per-warp staging buffer for queue appends: entries collect in shared memory and one
// atomicAdd on the queue length reserves room for up to QCAP of them at a time, instead
// of one contended global atomic per warp step. `count` is warp-uniform (a register of
// every lane). All 32 lanes must call push/flush.
template <int QCAP>
struct WarpQueue {
    int *buf;   // shared memory, QCAP entries, private to the warp
    int *q;     // global queue
    int *qlen;  // global queue length
    int count;

    __device__ __forceinline__ WarpQueue(int *b, int *queue, int *len)
        : buf(b), q(queue), qlen(len), count(0) {}

    __device__ __forceinline__ void flush() {
        __syncwarp();
        if (count == 0) return;
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == 0) base = atomicAdd(qlen, count);
        base = __shfl_sync(0xffffffffu, base, 0);
        for (int i = lane; i < count; i += 32) q[base + i] = buf[i];
        __syncwarp();
        count = 0;
    }

    __device__ __forceinline__ void push(bool pred, int v) {
        const unsigned mask = __ballot_sync(0xffffffffu, pred);
        if (mask == 0) return;
        if (count + 32 > QCAP) flush();
        const int lane = threadIdx.x & 31;
        if (pred) buf[count + __popc(mask & ((1u << lane) - 1u))] = v;
        count += __popc(mask);
    }
};

#endif  // __CUDACC__

}  // namespace apspie
