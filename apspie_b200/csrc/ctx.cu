// Context, scratch arena, CSR validation and the cooperative-launch helper.
//
// The context replaces the reference's mgpu::CudaContext (test/bfs/main.cu:27) and its
// per-call scratch (src/scratch.hpp:5-31, allocScratch src/util.cuh:646-672): the
// reference mallocs scratch inside every call (and cub temp storage inside every level,
// src/spmspvBfs.cuh:196-207); here one arena per context is grown on demand and reused.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "common.cuh"

namespace apspie {

apspie_status set_error(apspie_ctx *ctx, apspie_status st, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return st;
}

apspie_status cuda_error(apspie_ctx *ctx, cudaError_t e, const char *what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    (void)cudaGetLastError();  // clear non-sticky errors
    return set_error(ctx, e == cudaErrorMemoryAllocation ? APSPIE_ERR_OOM : APSPIE_ERR_CUDA, msg);
}

apspie_status scratch_reserve(apspie_ctx *ctx, size_t bytes, void **out) {
    ++ctx->scratch_epoch;
    if (bytes <= ctx->scratch_bytes && ctx->scratch) {
        *out = ctx->scratch;
        return APSPIE_OK;
    }
    // In-flight kernels may still use the old arena.
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "scratch_reserve sync");
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    size_t want = bytes + bytes / 8;  // headroom so slightly larger graphs reuse it
    e = cudaMalloc(&ctx->scratch, want);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        e = cudaMalloc(&ctx->scratch, bytes);
        want = bytes;
    }
    if (e != cudaSuccess) return cuda_error(ctx, e, "scratch_reserve cudaMalloc");
    ctx->scratch_bytes = want;
    *out = ctx->scratch;
    return APSPIE_OK;
}

apspie_status scratch2_reserve(apspie_ctx *ctx, size_t bytes, void **out) {
    ++ctx->scratch_epoch;
    if (bytes <= ctx->scratch2_bytes && ctx->scratch2) {
        *out = ctx->scratch2;
        return APSPIE_OK;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "scratch2_reserve sync");
    if (ctx->scratch2) cudaFree(ctx->scratch2);
    ctx->scratch2 = nullptr;
    ctx->scratch2_bytes = 0;
    e = cudaMalloc(&ctx->scratch2, bytes);
    if (e != cudaSuccess) return cuda_error(ctx, e, "scratch2_reserve cudaMalloc");
    ctx->scratch2_bytes = bytes;
    *out = ctx->scratch2;
    return APSPIE_OK;
}

apspie_status check_csr_view(apspie_ctx *ctx, const apspie_csr *A, const char *who) {
    if (!A) return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": NULL matrix");
    if (A->m < 0 || A->n < 0 || A->nnz < 0)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": negative size");
    if (!A->row_ptr || (A->nnz > 0 && !A->col_ind))
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": NULL CSR array");
    if (A->val_type < APSPIE_VAL_NONE || A->val_type > APSPIE_VAL_I32)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": unknown val_type");
    if (A->val_type != APSPIE_VAL_NONE && A->nnz > 0 && !A->val)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": NULL values");
    return APSPIE_OK;
}

// flags: 1 row_ptr[0] != 0, 2 row_ptr[m] != nnz, 4 decreasing offsets, 8 column out of
// range, 16 offset out of [0, nnz]
__global__ void validate_csr_kernel(int m, int n, int nnz, const int *__restrict__ row_ptr,
                                    const int *__restrict__ col_ind, int *flags) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    int f = 0;
    if (tid == 0) {
        if (row_ptr[0] != 0) f |= 1;
        if (row_ptr[m] != nnz) f |= 2;
    }
    for (int i = tid; i < m; i += stride) {
        int a = row_ptr[i], b = row_ptr[i + 1];
        if (b < a) f |= 4;
        if (a < 0 || a > nnz || b < 0 || b > nnz) f |= 16;
    }
    for (int e = tid; e < nnz; e += stride) {
        int c = col_ind[e];
        if (c < 0 || c >= n) f |= 8;
    }
    if (f) atomicOr(flags, f);
}

apspie_status validate_csr(apspie_ctx *ctx, const apspie_csr *A, bool need_square) {
    apspie_status st = check_csr_view(ctx, A, "validate");
    if (st != APSPIE_OK) return st;
    if (need_square && A->m != A->n)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "validate: matrix must be square");
    cudaError_t e = cudaMemsetAsync(ctx->d_ctl, 0, sizeof(TravCtl), ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "validate memset");
    int *flags = &ctx->d_ctl->err;
    int threads = 256;
    int blocks = ctx->num_sms * 8;
    validate_csr_kernel<<<blocks, threads, 0, ctx->stream>>>(A->m, A->n, A->nnz, A->row_ptr,
                                                              A->col_ind, flags);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(ctx, e, "validate launch");
    e = cudaMemcpyAsync(ctx->h_word, flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "validate copy");
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "validate sync");
    int f = *ctx->h_word;
    if (f) {
        std::string msg = "invalid CSR:";
        if (f & 1) msg += " row_ptr[0]!=0";
        if (f & 2) msg += " row_ptr[m]!=nnz";
        if (f & 4) msg += " decreasing row_ptr";
        if (f & 8) msg += " column index out of range";
        if (f & 16) msg += " row offset out of range";
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, msg);
    }
    return APSPIE_OK;
}

apspie_status reset_ctl(apspie_ctx *ctx) {
    cudaError_t e = cudaMemsetAsync(ctx->d_ctl, 0, sizeof(TravCtl), ctx->stream);
    if (e == cudaSuccess && ctx->wait_limit_ns != 0)
        e = cudaMemcpyAsync(&ctx->d_ctl->wait_limit_ns, ctx->h_limit, sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, ctx->stream);
    return e == cudaSuccess ? APSPIE_OK : cuda_error(ctx, e, "control reset");
}

// A cooperative grid that passes `rounds` grid barriers; block `absent` (when >= 0) leaves
// before its first arrival, so the others' first wait runs out.
__global__ void barrier_check_kernel(TravCtl *ctl, int *sticky, int rounds, int absent) {
    if (static_cast<int>(blockIdx.x) == absent) return;
    for (int r = 0; r < rounds; ++r)
        if (!grid_barrier(ctl, sticky, 900 + r)) return;
}

int persistent_cap(const apspie_ctx *ctx, int per_sm, int regs_per_block) {
    // a context that shares the device with grid_share - 1 others takes 1/grid_share of the
    // co-resident capacity, so that all of them fit at once. Whole blocks per SM: then each
    // kernel holds at most 1/grid_share of every per-SM resource (registers, shared memory,
    // threads), whichever limits it, and kernels of different footprints still fit together
    const int share = std::max(1, ctx->grid_share);
    if (share == 1 && ctx->side_room && regs_per_block > 0)
        while (per_sm > 1 && per_sm * regs_per_block > kSmRegs - kSideRoomRegs) --per_sm;
    if (per_sm >= share) return per_sm / share * ctx->num_sms;
    return std::max(1, per_sm * ctx->num_sms / share);
}

apspie_status launch_persistent(apspie_ctx *ctx, const void *func, int block, void **args,
                                long long work, int *grid_out) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, block, 0);
    if (e != cudaSuccess) return cuda_error(ctx, e, "occupancy query");
    if (per_sm < 1) return set_error(ctx, APSPIE_ERR_CUDA, "persistent kernel cannot be resident");
    int regs_per_block = 0;
    if (ctx->side_room) {
        cudaFuncAttributes fa;
        if ((e = cudaFuncGetAttributes(&fa, func)) != cudaSuccess) return cuda_error(ctx, e, "kernel attributes");
        // registers are allocated per warp in units of 256
        regs_per_block = (fa.numRegs * 32 + 255) / 256 * 256 * ((block + 31) / 32);
    }
    const int cap = persistent_cap(ctx, per_sm, regs_per_block);
    int grid = cap;
    const long long want = (work + kWorkPerBlock - 1) / kWorkPerBlock;
    if (want < grid) grid = static_cast<int>(want < ctx->num_sms ? ctx->num_sms : want);
    if (grid > cap) grid = cap;
    if (ctx->max_grid > 0 && grid > ctx->max_grid) grid = ctx->max_grid;
    if (grid > kMaxGrid) grid = kMaxGrid;
    e = cudaLaunchCooperativeKernel(func, dim3(grid), dim3(block), args, 0, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cooperative launch");
    if (grid_out) *grid_out = grid;
    return APSPIE_OK;
}

apspie_status finish_call(apspie_ctx *ctx, apspie_run_stats *stats, const char *who) {
    if (!stats) return APSPIE_OK;
    cudaError_t e = cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, kCtlHostBytes,
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "stats copy");
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "stats sync");
    const TravCtl &c = *ctx->h_ctl;
    stats->iterations = c.iterations;
    stats->push_iterations = c.push_iterations;
    stats->pull_iterations = c.pull_iterations;
    stats->reserved = 0;
    stats->edges_expanded = c.edges_expanded;
    stats->edges_component = c.edges_component;
    stats->vertices_reached = c.vertices_reached;
    if (c.err != 0) {
        // the error is reported here; clear the sticky copy so synchronize does not repeat it
        cudaMemsetAsync(ctx->d_sticky_err, 0, sizeof(int), ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        char buf[160];
        snprintf(buf, sizeof buf, "%s: device raised status %d at site %d", who, c.err,
                 c.err_where);
        return set_error(ctx, static_cast<apspie_status>(c.err), buf);
    }
    return APSPIE_OK;
}

}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_ctx_create(int device, void *cuda_stream, apspie_ctx **out) {
    if (!out) return APSPIE_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || device < 0 || device >= ndev) {
        (void)cudaGetLastError();
        return e == cudaSuccess ? APSPIE_ERR_INVALID_ARG : APSPIE_ERR_CUDA;
    }
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return APSPIE_ERR_CUDA;
    apspie_ctx *ctx = new apspie_ctx();
    ctx->device = device;
    ctx->stream = static_cast<cudaStream_t>(cuda_stream);
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    bool ok = cudaMalloc(&ctx->d_ctl, sizeof(TravCtl)) == cudaSuccess &&
              cudaMalloc(&ctx->d_sticky_err, sizeof(int)) == cudaSuccess &&
              cudaMallocHost(&ctx->h_ctl, sizeof(TravCtl)) == cudaSuccess &&
              cudaMallocHost(&ctx->h_word, 64) == cudaSuccess &&
              cudaMallocHost(&ctx->h_limit, 64) == cudaSuccess &&
              cudaMemset(ctx->d_sticky_err, 0, sizeof(int)) == cudaSuccess &&
              cudaMemset(ctx->d_ctl, 0, sizeof(TravCtl)) == cudaSuccess;
    if (!ok) {
        (void)cudaGetLastError();
        apspie_ctx_destroy(ctx);
        return APSPIE_ERR_OOM;
    }
    *out = ctx;
    return APSPIE_OK;
}

void apspie_ctx_destroy(apspie_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->scratch2) cudaFree(ctx->scratch2);
    if (ctx->d_ctl) cudaFree(ctx->d_ctl);
    if (ctx->d_sticky_err) cudaFree(ctx->d_sticky_err);
    if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
    if (ctx->h_word) cudaFreeHost(ctx->h_word);
    if (ctx->h_limit) cudaFreeHost(ctx->h_limit);
    delete ctx;
}

const char *apspie_ctx_last_error(const apspie_ctx *ctx) {
    return ctx ? ctx->last_error.c_str() : "NULL context";
}

apspie_status apspie_ctx_synchronize(apspie_ctx *ctx) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpyAsync(ctx->h_word, ctx->d_sticky_err, sizeof(int),
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "synchronize copy");
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "synchronize");
    int st = *ctx->h_word;
    if (st != 0) {
        cudaMemsetAsync(ctx->d_sticky_err, 0, sizeof(int), ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        return set_error(ctx, static_cast<apspie_status>(st),
                         "an asynchronous call raised a device-side error");
    }
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_validate(apspie_ctx *ctx, int on) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    ctx->validate = on ? 1 : 0;
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_bfs_tuning(apspie_ctx *ctx, float alpha, float beta) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    if (!(beta > 0.0f)) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "beta must be > 0");
    ctx->bfs_alpha = alpha;
    ctx->bfs_beta = beta;
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_sssp_delta(apspie_ctx *ctx, int32_t delta) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    ctx->sssp_delta = delta;
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_sssp_band(apspie_ctx *ctx, int64_t edges) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    ctx->sssp_band = edges;
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_sssp_batch_groups(apspie_ctx *ctx, int32_t groups) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    ctx->sssp_batch_groups = groups;
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_batch_push_frac(apspie_ctx *ctx, float frac) {
    if (!ctx || !(frac >= 0.0f)) return APSPIE_ERR_INVALID_ARG;
    ctx->batch_push_frac = frac;
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_max_grid(apspie_ctx *ctx, int32_t max_blocks) {
    if (!ctx || max_blocks < 0) return APSPIE_ERR_INVALID_ARG;
    ctx->max_grid = max_blocks;
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_wait_limit(apspie_ctx *ctx, int64_t ns) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    // calls already enqueued may still read the pinned copy
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "set_wait_limit");
    ctx->wait_limit_ns = ns > 0 ? static_cast<unsigned long long>(ns) : 0ull;
    *ctx->h_limit = ctx->wait_limit_ns;
    return APSPIE_OK;
}

apspie_status apspie_grid_barrier_check(apspie_ctx *ctx, int32_t rounds, int32_t absent_block, int32_t *grid) {
    if (!ctx || rounds < 0) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = reset_ctl(ctx);
    if (st != APSPIE_OK) return st;
    int g = 0;
    void *args[4];
    int *sticky = ctx->d_sticky_err;
    TravCtl *ctl = ctx->d_ctl;
    args[0] = &ctl;
    args[1] = &sticky;
    args[2] = &rounds;
    args[3] = &absent_block;
    st = launch_persistent(ctx, reinterpret_cast<const void *>(barrier_check_kernel), 256, args, 1LL << 40, &g);
    if (st != APSPIE_OK) return st;
    if (grid) *grid = g;
    apspie_run_stats rs;  // reads the control block back: the device's status
    return finish_call(ctx, &rs, "apspie_grid_barrier_check");
}

apspie_status apspie_ctx_timeline(const apspie_ctx *ctx, int32_t *sites, int64_t *ns, int32_t cap,
                                  int32_t *count) {
    if (!ctx || !count || cap < 0 || (cap > 0 && (!sites || !ns))) return APSPIE_ERR_INVALID_ARG;
    const TravCtl &c = *ctx->h_ctl;
    int n = c.tl_count < kTimeline ? c.tl_count : kTimeline;
    if (n > cap) n = cap;
    for (int i = 0; i < n; ++i) {
        sites[i] = c.tl_site[i];
        ns[i] = static_cast<int64_t>(c.tl_ns[i] - c.tl_ns[0]);
    }
    *count = n;
    return APSPIE_OK;
}

int64_t apspie_ctx_scratch_bytes(const apspie_ctx *ctx) {
    return ctx ? static_cast<int64_t>(ctx->scratch_bytes + ctx->scratch2_bytes) : 0;
}

apspie_status apspie_csr_validate(apspie_ctx *ctx, const apspie_csr *A) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    return validate_csr(ctx, A, false);
}

}  // extern "C"
