// Triangle counting as a masked SpGEMM: count = sum((L*L) .* L) for the strict lower
// triangle L of a symmetric graph, without materialising L*L.
//
// The reference builds L and U on the host (buildLower, test/tc/main.cu:39-55), forms
// D = U*L with cuSPARSE csrgemm (tc.cuh:62-165, D is materialised), intersects each
// column of D with the same column of U in one thread per column (ewiseMultTc,
// tc.cuh:168-199) and reduces a float vector (mgpu::Reduce, test/tc/main.cu:249).
//
// Here L's edges are first re-oriented on the device from the endpoint of lower
// (degree, id) rank to the higher one: D is another acyclic orientation of the same
// undirected edge set, so sum((D*D) .* D) is the same count, but every row of D has at
// most about sqrt(2 * nnz) entries and the wedge total drops (R-MAT scale 18: 1.11G wedges
// under L, 0.66G under D, largest row 8,083 -> 411). Each row i of D is loaded into a hash
// set (its mask); every wedge (k in D(i,:), j in D(k,:)) probes the set, and hits are
// counted in int64. Rows with masks of at most 256 entries are cut into warp tasks of at
// most task_work wedges (4096 unless tuned); each task loads its row's mask into a
// 512-slot shared-memory set, so skewed rows cannot unbalance the warps. Larger masks
// take a block with a 4096-slot shared set, or a block with a global set. An input with
// an entry on or above the diagonal is not a strict lower triangle; it is counted as
// given, sum((L*L) .* L), without re-orientation (also when orientation is tuned off).
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace apspie {
namespace {

constexpr int kTcBlock = 256;
constexpr int kEmpty = -1;
constexpr int kTcBins = 4;        // 0 nothing to do | 1 warp | 2 block/shared | 3 block/global
constexpr int kWarpSet = 512;     // slots (mask <= 256)
#ifndef APSPIE_TC_CHUNKS
#define APSPIE_TC_CHUNKS 4
#endif
constexpr int kTcChunks = APSPIE_TC_CHUNKS;  // 32-wedge chunks a warp gathers at once
constexpr int kBlockSet = 4096;   // slots (mask <= 2048)

struct TcInfo {
    int bin_count[kTcBins];
    long long global_slots;
    unsigned long long count;
    int overflow;
    int not_lower;  // an entry with column >= row
};

__device__ __forceinline__ unsigned tc_hash(int key, int log2ts) {
    return (static_cast<unsigned>(key) * 2654435761u) >> (32 - log2ts);
}

// 8 lanes per row: mask size d and wedge count; the row's bin goes to row_bin and, for a
// warp-tier row, its number of warp tasks (task_work wedges each) to ntask.
__global__ void tc_rowinfo(int m, const int *__restrict__ rp, const int *__restrict__ ci, int task_work,
                           unsigned char *row_bin, int *ntask, long long *tbl_off, TcInfo *info) {
    const int sub = threadIdx.x & 7;
    const int grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int ngrp = (gridDim.x * blockDim.x) >> 3;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    for (int i0 = grp - (grp & 3); i0 < m; i0 += ngrp) {  // the warp's 4 groups move together
        const int i = i0 + (grp & 3);
        int r0 = 0, r1 = 0;
        long long work = 0;
        if (i < m) {
            r0 = __ldg(rp + i);
            r1 = __ldg(rp + i + 1);
            if (r1 - r0 >= 2)
                for (int e = r0 + sub; e < r1; e += 8) {
                    const int k = __ldg(ci + e);
                    work += __ldg(rp + k + 1) - __ldg(rp + k);
                }
        }
        for (int o = 4; o; o >>= 1) work += __shfl_down_sync(gmask, work, o, 8);
        if (i < m && sub == 0) {
            const int d = r1 - r0;
            int b;
            if (d < 2 || work == 0)
                b = 0;
            else if (d <= kWarpSet / 2)
                b = 1;
            else if (d <= kBlockSet / 2)
                b = 2;
            else
                b = 3;
            row_bin[i] = static_cast<unsigned char>(b);
            ntask[i] = b == 1 ? static_cast<int>((work + task_work - 1) / task_work) : 0;
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

// Per-bin row lists (stride m, bin 0 skipped): warp ballots count a block's rows per
// bin, one global atomic per bin reserves their room.
__global__ void tc_binlists(int m, const unsigned char *__restrict__ row_bin, int *bin_rows, TcInfo *info) {
    __shared__ int cnt[kTcBins];
    __shared__ int base[kTcBins];
    const int lane = threadIdx.x & 31;
    for (int c0 = blockIdx.x * blockDim.x; c0 < m; c0 += gridDim.x * blockDim.x) {
        if (threadIdx.x < kTcBins) cnt[threadIdx.x] = 0;
        __syncthreads();
        const int i = c0 + threadIdx.x;
        const int b = i < m ? row_bin[i] : 0;
        int pos = 0;
#pragma unroll
        for (int k = 1; k < kTcBins; ++k) {
            const unsigned mk = __ballot_sync(0xffffffffu, b == k);
            int wbase = 0;
            if (mk && lane == __ffs(mk) - 1) wbase = atomicAdd(&cnt[k], __popc(mk));
            wbase = __shfl_sync(0xffffffffu, wbase, mk ? __ffs(mk) - 1 : 0);
            if (b == k) pos = wbase + __popc(mk & ((1u << lane) - 1u));
        }
        __syncthreads();
        if (threadIdx.x >= 1 && threadIdx.x < kTcBins && cnt[threadIdx.x])
            base[threadIdx.x] = atomicAdd(&info->bin_count[threadIdx.x], cnt[threadIdx.x]);
        __syncthreads();
        if (b > 0) bin_rows[static_cast<long long>(b) * m + base[b] + pos] = i;
        __syncthreads();
    }
}

// ---------------------------------------------------------------- degree orientation
// deg[v] = |L(v,:)| + |{i : v in L(i,:)}| (the undirected degree); flags entries with
// column >= row.
__global__ void tc_degree(int m, const int *__restrict__ rp, const int *__restrict__ ci, int *deg,
                          TcInfo *info) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    bool bad = false;
    for (int i = warp; i < m; i += nwarps) {
        const int r0 = __ldg(rp + i), r1 = __ldg(rp + i + 1);
        for (int e = r0 + lane; e < r1; e += 32) {
            const int j = __ldg(ci + e);
            bad |= j >= i;
            if (j >= 0 && j < m) atomicAdd(deg + j, 1);
        }
        if (lane == 0 && r1 > r0) atomicAdd(deg + i, r1 - r0);
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&info->not_lower, 1);
}

// PASS 0: out-degree counts of the orientation; PASS 1: scatter into D (rows unsorted).
// Edges leaving row i take one reservation per 32; edges entering i (from a lower-ranked
// column) one atomic each.
template <int PASS>
__global__ void tc_orient(int m, const int *__restrict__ rp, const int *__restrict__ ci,
                          const int *__restrict__ deg, int *cnt, const int *__restrict__ drp, int *dci) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < m; i += nwarps) {
        const int r0 = __ldg(rp + i), r1 = __ldg(rp + i + 1);
        const int di = __ldg(deg + i);
        const int drp_i = PASS == 1 ? __ldg(drp + i) : 0;
        int own = 0;
        for (int e0 = r0; e0 < r1; e0 += 32) {
            const int e = e0 + lane;
            const bool valid = e < r1;
            const int j = valid ? __ldg(ci + e) : 0;
            const int dj = valid ? __ldg(deg + j) : 0;
            const bool fwd = valid && (di < dj || (di == dj && i < j));
            const unsigned fm = __ballot_sync(0xffffffffu, fwd);
            if (PASS == 0) {
                if (valid && !fwd) atomicAdd(cnt + j, 1);
            } else {
                int b = 0;
                if (lane == 0 && fm) b = atomicAdd(cnt + i, __popc(fm));
                b = __shfl_sync(0xffffffffu, b, 0);
                if (fwd) dci[drp_i + b + __popc(fm & ((1u << lane) - 1u))] = j;
                if (valid && !fwd) dci[__ldg(drp + j) + atomicAdd(cnt + j, 1)] = i;
            }
            own += __popc(fm);
        }
        if (PASS == 0 && lane == 0 && own) atomicAdd(cnt + i, own);
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

// Warp tasks: task t belongs to the row r with task_ptr[r] <= t < task_ptr[r + 1] and
// covers wedges [c * task_work, (c + 1) * task_work) of it, c = t - task_ptr[r]. Each task
// loads its row's mask (<= 256 entries) into its warp's set, so tasks are independent and
// of bounded size, and warps stay balanced however skewed the rows are.
__global__ void __launch_bounds__(kTcBlock) tc_warp(const int *__restrict__ task_ptr, int m, int ntasks,
                                                    int task_work, const int *__restrict__ rp,
                                                    const int *__restrict__ ci, TcInfo *info) {
    __shared__ TcWarpSmem smem[kTcBlock / 32];
    const int lane = threadIdx.x & 31;
    TcWarpSmem &sm = smem[threadIdx.x >> 5];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    constexpr int LOG = kWarpSet == 512 ? 9 : (kWarpSet == 256 ? 8 : 7);  // log2(kWarpSet)
    static_assert((1 << LOG) == kWarpSet, "warp set size");
    unsigned long long hits = 0;
    for (int t = warp; t < ntasks; t += nwarps) {
        int lo = 0, hi = m;  // last row with task_ptr[row] <= t
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(task_ptr + mid) <= t)
                lo = mid;
            else
                hi = mid;
        }
        const int i = lo;
        const int w0 = (t - __ldg(task_ptr + i)) * task_work;
        const int r0 = __ldg(rp + i);
        const int d = __ldg(rp + i + 1) - r0;
        for (int s = lane; s < kWarpSet; s += 32) sm.keys[s] = kEmpty;
        __syncwarp();
        // mask into the set; rows k of the mask with entries are listed (row start, offset)
        int carry = 0, nv = 0;
        for (int base = 0; base < d; base += 32) {
            const int tt = base + lane;
            int len = 0, b0 = 0;
            if (tt < d) {
                const int k = __ldg(ci + r0 + tt);
                set_insert(sm.keys, kWarpSet, LOG, k, info);
                b0 = __ldg(rp + k);
                len = __ldg(rp + k + 1) - b0;
            }
            const unsigned nz = __ballot_sync(0xffffffffu, len > 0);
            int incl = len;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (len > 0) {
                const int slot = nv + __popc(nz & ((1u << lane) - 1u));
                sm.rs[slot] = b0;
                sm.soff[slot] = carry + incl - len;
            }
            nv += __popc(nz);
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) sm.soff[nv] = carry;
        __syncwarp();
        const int w1 = min(carry, w0 + task_work);
        // o0: the listed row holding wedge w0 (last with soff <= w0)
        int o0 = 0;
        {
            int a = 0, b = nv;
            while (b - a > 1) {
                const int mid = (a + b) >> 1;
                if (sm.soff[mid] <= w0)
                    a = mid;
                else
                    b = mid;
            }
            o0 = a;
        }
        // wedges in chunks of 32: the next 32 listed rows' starts that fall inside the
        // chunk are marked in a 32-bit word (distinct, since every listed row is
        // non-empty); each lane's row is o0 plus the marks at or before its position
        // kTcChunks chunks per step, so that each lane has that many gathers in flight
        const unsigned upto = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
        for (int base = w0; base < w1; base += 32 * kTcChunks) {
            int own[kTcChunks], q[kTcChunks];
#pragma unroll
            for (int h = 0; h < kTcChunks; ++h) {
                const int cb = base + 32 * h;
                const int nb = o0 + 1 + lane;
                const int st = nb <= nv ? sm.soff[nb] - cb : 32;
                const unsigned mark = (st >= 0 && st < 32) ? (1u << st) : 0u;
                const unsigned starts = __reduce_or_sync(0xffffffffu, mark);
                own[h] = o0 + __popc(starts & upto);
                q[h] = cb + lane;
                o0 += __popc(starts);
            }
            int j[kTcChunks];
#pragma unroll
            for (int h = 0; h < kTcChunks; ++h)
                j[h] = q[h] < w1 ? __ldg(ci + sm.rs[own[h]] + (q[h] - sm.soff[own[h]])) : -1;
#pragma unroll
            for (int h = 0; h < kTcChunks; ++h)
                if (q[h] < w1) hits += set_find<false>(sm.keys, kWarpSet, LOG, j[h]) ? 1 : 0;
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) hits += __shfl_down_sync(0xffffffffu, hits, o);
    if (lane == 0 && hits) atomicAdd(&info->count, hits);
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
    const size_t nz = static_cast<size_t>(L->nnz > 0 ? L->nnz : 1);
    void *base;
    st = scratch_reserve(ctx,
                         Carver::need({kTcBins * mi * 4, mi * 8, sizeof(TcInfo), mi, mi * 4, mi * 4, mi * 4,
                                       nz * 4, scan_scratch_bytes(m) + 64, mi * 4, mi * 4}),
                         &base);
    if (st != APSPIE_OK) return st;
    Carver c(base);
    int *bin_rows = c.take<int>(kTcBins * mi);
    long long *tbl_off = c.take<long long>(mi);
    TcInfo *info = c.take<TcInfo>(1);
    unsigned char *row_bin = c.take<unsigned char>(mi);
    int *deg = c.take<int>(mi);
    int *ocnt = c.take<int>(mi);
    int *drp = c.take<int>(mi);
    int *dci = c.take<int>(nz);
    void *stmp = c.take<char>(scan_scratch_bytes(m) + 64);
    int *ntask = c.take<int>(mi);
    int *task_ptr = c.take<int>(mi);
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(TcInfo), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(deg, 0, mi * 4, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ocnt, 0, mi * 4, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "tc reset");
    const int wblocks = std::max(1, std::min<int>((m * 32LL + 255) / 256, ctx->num_sms * 16));
    const int *rp = L->row_ptr, *ci = L->col_ind;
    const apspie_tune_params tp = effective_params(ctx, APSPIE_TUNE_TC, L);
    if (m > 0 && tp.tc_orient) {
        // D: L's edges oriented from lower to higher (degree, id) rank
        tc_degree<<<wblocks, 256, 0, ctx->stream>>>(m, rp, ci, deg, info);
        tc_orient<0><<<wblocks, 256, 0, ctx->stream>>>(m, rp, ci, deg, ocnt, nullptr, nullptr);
        if ((st = device_exclusive_scan(ctx, ocnt, m, drp, stmp, &info->overflow)) != APSPIE_OK) return st;
        if ((e = cudaMemsetAsync(ocnt, 0, mi * 4, ctx->stream)) != cudaSuccess) return cuda_error(ctx, e, "tc reset");
        tc_orient<1><<<wblocks, 256, 0, ctx->stream>>>(m, rp, ci, deg, ocnt, drp, dci);
        rp = drp;
        ci = dci;
    }
    const int rblocks = std::max(1, std::min<int>((m * 8LL + 255) / 256, ctx->num_sms * 16));
    const int lblocks = std::max(1, std::min<int>((m + 255LL) / 256, ctx->num_sms * 8));
    TcInfo h;
    int ntasks = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        if (m > 0) {
            tc_rowinfo<<<rblocks, 256, 0, ctx->stream>>>(m, rp, ci, tp.tc_task_work, row_bin, ntask, tbl_off,
                                                         info);
            tc_binlists<<<lblocks, 256, 0, ctx->stream>>>(m, row_bin, bin_rows, info);
            if ((st = device_exclusive_scan(ctx, ntask, m, task_ptr, stmp, &info->overflow)) != APSPIE_OK) return st;
            if ((e = cudaMemcpyAsync(&ntasks, task_ptr + m, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) !=
                cudaSuccess)
                return cuda_error(ctx, e, "tc plan");
        }
        if ((e = cudaMemcpyAsync(&h, info, sizeof(TcInfo), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
            return cuda_error(ctx, e, "tc plan");
        if (!h.not_lower || attempt == 1 || !tp.tc_orient) break;
        // not a strict lower triangle: count sum((L*L) .* L) on L as given
        rp = L->row_ptr;
        ci = L->col_ind;
        if ((e = cudaMemsetAsync(info, 0, sizeof(TcInfo), ctx->stream)) != cudaSuccess)
            return cuda_error(ctx, e, "tc reset");
    }
    int *gkeys = nullptr;
    if (h.global_slots > 0) {
        void *tb;
        if ((st = scratch2_reserve(ctx, static_cast<size_t>(h.global_slots) * 4 + 256, &tb)) != APSPIE_OK)
            return st;
        gkeys = static_cast<int *>(tb);
    }
    const int cap = ctx->num_sms * 8;
    if (ntasks > 0)
        tc_warp<<<std::min((ntasks + 7) / 8, cap), kTcBlock, 0, ctx->stream>>>(task_ptr, m, ntasks,
                                                                                 tp.tc_task_work, rp, ci, info);
    if (h.bin_count[2] > 0)
        tc_block<false><<<std::min(h.bin_count[2], cap), kTcBlock, 0, ctx->stream>>>(
            bin_rows + 2 * static_cast<size_t>(m), h.bin_count[2], rp, ci, tbl_off, gkeys, info);
    if (h.bin_count[3] > 0)
        tc_block<true><<<std::min(h.bin_count[3], cap), kTcBlock, 0, ctx->stream>>>(
            bin_rows + 3 * static_cast<size_t>(m), h.bin_count[3], rp, ci, tbl_off, gkeys, info);
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
