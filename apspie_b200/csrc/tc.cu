// Triangle counting as a masked SpGEMM: count = sum((L*L) .* L) for the strict lower
// triangle L of a symmetric graph, without materialising L*L.
//
// The reference builds L and U on the host (buildLower, test/tc/main.cu:39-55), forms
// D = U*L with cuSPARSE csrgemm (tc.cuh:62-165, D is materialised), intersects each
// column of D with the same column of U in one thread per column (ewiseMultTc,
// tc.cuh:168-199) and reduces a float vector (mgpu::Reduce, test/tc/main.cu:249).
//
// Here each row i of L is loaded into a hash set (its mask); every wedge (k in L(i,:),
// j in L(k,:)) probes the set, and hits are counted in int64. Rows are binned by mask size
// and wedge count: a warp with a 128-slot shared-memory set, a block with a 4096-slot
// shared set, or a block with a global set. Work per row = sum of deg_L(k) over its mask.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace apspie {
namespace {

constexpr int kTcBlock = 256;
constexpr int kEmpty = -1;
constexpr int kTcBins = 4;        // 0 nothing to do | 1 warp | 2 block/shared | 3 block/global
constexpr int kWarpSet = 128;     // slots (mask <= 64)
constexpr int kBlockSet = 4096;   // slots (mask <= 2048)
constexpr long long kWarpWork = 32768;

struct TcInfo {
    int bin_count[kTcBins];
    long long global_slots;
    unsigned long long count;
    int overflow;
};

__device__ __forceinline__ unsigned tc_hash(int key, int log2ts) {
    return (static_cast<unsigned>(key) * 2654435761u) >> (32 - log2ts);
}

__global__ void tc_rowinfo(int m, const int *__restrict__ rp, const int *__restrict__ ci, int *bin_rows,
                           long long *tbl_off, TcInfo *info) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < m; i += nwarps) {
        const int r0 = rp[i], r1 = rp[i + 1];
        const int d = r1 - r0;
        long long work = 0;
        if (d >= 2)
            for (int e = r0 + lane; e < r1; e += 32) {
                const int k = ci[e];
                work += rp[k + 1] - rp[k];
            }
        for (int o = 16; o; o >>= 1) work += __shfl_down_sync(0xffffffffu, work, o);
        if (lane == 0) {
            int b;
            if (d < 2 || work == 0)
                b = 0;
            else if (d <= kWarpSet / 2 && work <= kWarpWork)
                b = 1;
            else if (d <= kBlockSet / 2)
                b = 2;
            else
                b = 3;
            if (b) {
                const int pos = atomicAdd(&info->bin_count[b], 1);
                bin_rows[static_cast<long long>(b) * m + pos] = i;
            }
            if (b == 3) {
                long long ts = 64;
                while (ts < 2LL * d) ts <<= 1;
                tbl_off[i] = static_cast<long long>(
                    atomicAdd(reinterpret_cast<unsigned long long *>(&info->global_slots),
                              static_cast<unsigned long long>(ts)));
            }
        }
    }
}

__device__ __forceinline__ void set_insert(int *keys, long long ts, int log2ts, int key, TcInfo *info) {
    unsigned long long s = tc_hash(key, log2ts) & (ts - 1);
    for (long long p = 0; p <= ts; ++p) {
        const int old = atomicCAS(keys + s, kEmpty, key);
        if (old == kEmpty || old == key) return;
        s = (s + 1) & (ts - 1);
    }
    atomicOr(&info->overflow, 1);
}

template <bool COHERENT>
__device__ __forceinline__ bool set_find(const int *keys, long long ts, int log2ts, int key) {
    unsigned long long s = tc_hash(key, log2ts) & (ts - 1);
    for (long long p = 0; p <= ts; ++p) {
        const int k = COHERENT ? __ldcg(keys + s) : keys[s];
        if (k == key) return true;
        if (k == kEmpty) return false;
        s = (s + 1) & (ts - 1);
    }
    return false;
}

struct TcWarpSmem {
    int keys[kWarpSet];
    int rs[kWarpSet / 2];
    int soff[kWarpSet / 2 + 1];
};

// One warp per row (mask <= 64 entries, <= kWarpWork wedges).
__global__ void __launch_bounds__(kTcBlock) tc_warp(const int *__restrict__ rows, int nrows,
                                                    const int *__restrict__ rp, const int *__restrict__ ci,
                                                    TcInfo *info) {
    __shared__ TcWarpSmem smem[kTcBlock / 32];
    __shared__ unsigned long long bsum;
    const int lane = threadIdx.x & 31;
    TcWarpSmem &sm = smem[threadIdx.x >> 5];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    if (threadIdx.x == 0) bsum = 0;
    __syncthreads();
    constexpr int LOG = 7;  // log2(kWarpSet)
    unsigned long long hits = 0;
    for (int w = warp; w < nrows; w += nwarps) {
        const int i = rows[w];
        const int r0 = rp[i];
        const int d = rp[i + 1] - r0;
        for (int s = lane; s < kWarpSet; s += 32) sm.keys[s] = kEmpty;
        __syncwarp();
        int carry = 0;
        for (int base = 0; base < d; base += 32) {
            const int t = base + lane;
            int deg = 0;
            if (t < d) {
                const int k = ci[r0 + t];
                set_insert(sm.keys, kWarpSet, LOG, k, info);
                const int b0 = rp[k];
                sm.rs[t] = b0;
                deg = rp[k + 1] - b0;
            }
            int incl = deg;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (t < d) sm.soff[t] = carry + incl - deg;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncwarp();
        const int work = carry;
        for (int q = lane; q < work; q += 32) {
            int lo = 0, hi = d;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (sm.soff[mid] <= q)
                    lo = mid;
                else
                    hi = mid;
            }
            const int j = ci[sm.rs[lo] + (q - sm.soff[lo])];
            hits += set_find<false>(sm.keys, kWarpSet, LOG, j) ? 1 : 0;
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) hits += __shfl_down_sync(0xffffffffu, hits, o);
    if (lane == 0 && hits) atomicAdd(&bsum, hits);
    __syncthreads();
    if (threadIdx.x == 0 && bsum) atomicAdd(&info->count, bsum);
}

struct TcBlockSmem {
    int keys[kBlockSet];
    int rs[kTcBlock];
    int soff[kTcBlock + 1];
    int scan_tmp[33];
    unsigned long long bsum;
};

// One block per row; the mask set is in shared memory, or in scratch for GLOBAL rows.
template <bool GLOBAL>
__global__ void __launch_bounds__(kTcBlock) tc_block(const int *__restrict__ rows, int nrows,
                                                     const int *__restrict__ rp, const int *__restrict__ ci,
                                                     const long long *__restrict__ tbl_off, int *gkeys,
                                                     TcInfo *info) {
    __shared__ TcBlockSmem sm;
    const int tid = threadIdx.x;
    if (tid == 0) sm.bsum = 0;
    unsigned long long hits = 0;
    for (int w = blockIdx.x; w < nrows; w += gridDim.x) {
        const int i = rows[w];
        const int r0 = rp[i];
        const int d = rp[i + 1] - r0;
        long long ts = kBlockSet;
        int *keys = sm.keys;
        if (GLOBAL) {
            ts = 64;
            while (ts < 2LL * d) ts <<= 1;
            keys = gkeys + tbl_off[i];
        }
        int log2ts = 0;
        while ((1LL << log2ts) < ts) ++log2ts;
        if (log2ts > 31) log2ts = 31;
        for (long long s = tid; s < ts; s += kTcBlock) keys[s] = kEmpty;
        __syncthreads();
        for (int t = tid; t < d; t += kTcBlock) set_insert(keys, ts, log2ts, ci[r0 + t], info);
        __syncthreads();
        for (int c0 = 0; c0 < d; c0 += kTcBlock) {
            const int t = c0 + tid;
            int deg = 0;
            if (t < d) {
                const int k = ci[r0 + t];
                const int b0 = rp[k];
                sm.rs[tid] = b0;
                deg = rp[k + 1] - b0;
            }
            int tot;
            sm.soff[tid] = block_exclusive_scan<kTcBlock>(deg, tot, sm.scan_tmp);
            __syncthreads();
            const int nt = d - c0 < kTcBlock ? d - c0 : kTcBlock;
            for (int q = tid; q < tot; q += kTcBlock) {
                int lo = 0, hi = nt;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (sm.soff[mid] <= q)
                        lo = mid;
                    else
                        hi = mid;
                }
                const int j = ci[sm.rs[lo] + (q - sm.soff[lo])];
                hits += set_find<GLOBAL>(keys, ts, log2ts, j) ? 1 : 0;
            }
            __syncthreads();
        }
    }
    for (int o = 16; o; o >>= 1) hits += __shfl_down_sync(0xffffffffu, hits, o);
    if ((tid & 31) == 0 && hits) atomicAdd(&sm.bsum, hits);
    __syncthreads();
    if (tid == 0 && sm.bsum) atomicAdd(&info->count, sm.bsum);
}

// strict lower triangle extraction: counts, then copy
__global__ void lower_count(int m, const int *__restrict__ rp, const int *__restrict__ ci, int *cnt) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < m; i += nwarps) {
        int c = 0;
        for (int e = rp[i] + lane; e < rp[i + 1]; e += 32) c += ci[e] < i;
        for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) cnt[i] = c;
    }
}

__global__ void lower_copy(int m, const int *__restrict__ rp, const int *__restrict__ ci,
                           const int *__restrict__ lrp, int *lci) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < m; i += nwarps) {
        int out = lrp[i];
        for (int e0 = rp[i]; e0 < rp[i + 1]; e0 += 32) {
            const int e = e0 + lane;
            const bool keep = e < rp[i + 1] && ci[e] < i;
            const unsigned mask = __ballot_sync(0xffffffffu, keep);
            if (keep) lci[out + __popc(mask & ((1u << lane) - 1u))] = ci[e];
            out += __popc(mask);
        }
    }
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_tc(apspie_ctx *ctx, const apspie_csr *L, int64_t *count) {
    if (!ctx || !count) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_csr_view(ctx, L, "apspie_tc");
    if (st != APSPIE_OK) return st;
    if (L->m != L->n) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_tc: L must be square");
    if (ctx->validate && (st = validate_csr(ctx, L, true)) != APSPIE_OK) return st;
    const int m = L->m;
    const size_t mi = static_cast<size_t>(m) + 1;
    void *base;
    st = scratch_reserve(ctx, Carver::need({kTcBins * mi * 4, mi * 8, sizeof(TcInfo)}), &base);
    if (st != APSPIE_OK) return st;
    Carver c(base);
    int *bin_rows = c.take<int>(kTcBins * mi);
    long long *tbl_off = c.take<long long>(mi);
    TcInfo *info = c.take<TcInfo>(1);
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(TcInfo), ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "tc reset");
    if (m > 0) {
        const int blocks = std::min<long long>((static_cast<long long>(m) * 32 + 255) / 256, ctx->num_sms * 16LL);
        tc_rowinfo<<<blocks, 256, 0, ctx->stream>>>(m, L->row_ptr, L->col_ind, bin_rows, tbl_off, info);
    }
    TcInfo h;
    if ((e = cudaMemcpyAsync(&h, info, sizeof(TcInfo), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return cuda_error(ctx, e, "tc plan");
    int *gkeys = nullptr;
    if (h.global_slots > 0) {
        void *tb;
        if ((st = scratch2_reserve(ctx, static_cast<size_t>(h.global_slots) * 4 + 256, &tb)) != APSPIE_OK)
            return st;
        gkeys = static_cast<int *>(tb);
    }
    const int cap = ctx->num_sms * 8;
    if (h.bin_count[1] > 0)
        tc_warp<<<std::min((h.bin_count[1] + 7) / 8, cap), kTcBlock, 0, ctx->stream>>>(
            bin_rows + 1 * static_cast<size_t>(m), h.bin_count[1], L->row_ptr, L->col_ind, info);
    if (h.bin_count[2] > 0)
        tc_block<false><<<std::min(h.bin_count[2], cap), kTcBlock, 0, ctx->stream>>>(
            bin_rows + 2 * static_cast<size_t>(m), h.bin_count[2], L->row_ptr, L->col_ind, tbl_off, gkeys, info);
    if (h.bin_count[3] > 0)
        tc_block<true><<<std::min(h.bin_count[3], cap), kTcBlock, 0, ctx->stream>>>(
            bin_rows + 3 * static_cast<size_t>(m), h.bin_count[3], L->row_ptr, L->col_ind, tbl_off, gkeys, info);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(ctx, e, "tc launch");
    if ((e = cudaMemcpyAsync(&h, info, sizeof(TcInfo), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return cuda_error(ctx, e, "tc result");
    if (h.overflow) return set_error(ctx, APSPIE_ERR_HASH_OVERFLOW, "apspie_tc: mask set overflow");
    *count = static_cast<int64_t>(h.count);
    return APSPIE_OK;
}

apspie_status apspie_csr_strict_lower_device(apspie_ctx *ctx, const apspie_csr *A, apspie_csr_owned *L) {
    if (!ctx || !L) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    std::memset(L, 0, sizeof(*L));
    apspie_status st = check_csr_view(ctx, A, "apspie_csr_strict_lower_device");
    if (st != APSPIE_OK) return st;
    if (A->m != A->n) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "strict lower: A must be square");
    if (ctx->validate && (st = validate_csr(ctx, A, true)) != APSPIE_OK) return st;
    const int m = A->m;
    const size_t mi = static_cast<size_t>(m) + 1;
    void *base;
    st = scratch_reserve(ctx, Carver::need({mi * 4, scan_scratch_bytes(m) + 64, 64}), &base);
    if (st != APSPIE_OK) return st;
    Carver c(base);
    int *cnt = c.take<int>(mi);
    void *stmp = c.take<char>(scan_scratch_bytes(m) + 64);
    int *ovf = c.take<int>(16);
    cudaError_t e = cudaMemsetAsync(ovf, 0, sizeof(int), ctx->stream);
    int32_t *lrp = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&lrp, mi * sizeof(int32_t));
    if (e != cudaSuccess) return cuda_error(ctx, e, "strict lower alloc");
    const int blocks = std::max(1, std::min<int>((m * 32LL + 255) / 256, ctx->num_sms * 16));
    lower_count<<<blocks, 256, 0, ctx->stream>>>(m, A->row_ptr, A->col_ind, cnt);
    if ((st = device_exclusive_scan(ctx, cnt, m, lrp, stmp, ovf)) != APSPIE_OK) {
        cudaFree(lrp);
        return st;
    }
    int nnz = 0;
    if ((e = cudaMemcpyAsync(&nnz, lrp + m, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
        cudaFree(lrp);
        return cuda_error(ctx, e, "strict lower sync");
    }
    int32_t *lci = nullptr;
    if ((e = cudaMalloc(&lci, std::max(nnz, 1) * sizeof(int32_t))) != cudaSuccess) {
        cudaFree(lrp);
        return cuda_error(ctx, e, "strict lower alloc");
    }
    lower_copy<<<blocks, 256, 0, ctx->stream>>>(m, A->row_ptr, A->col_ind, lrp, lci);
    if ((e = cudaGetLastError()) != cudaSuccess) {
        cudaFree(lrp);
        cudaFree(lci);
        return cuda_error(ctx, e, "strict lower launch");
    }
    L->m = L->n = m;
    L->nnz = nnz;
    L->val_type = APSPIE_VAL_NONE;
    L->row_ptr = lrp;
    L->col_ind = lci;
    L->val = nullptr;
    return APSPIE_OK;
}

}  // extern "C"
