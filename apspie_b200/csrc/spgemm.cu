// Row-binned hash SpGEMM  C = A * B  (Gustavson, row by row).
//
// Replaces the reference's 2-D partitioned outer-product hash SpGEMM
// (src/spgemm.cuh:131-342, src/spgemmKernel.cuh:439-738: CSR->DCSC per partition,
// SetOpPairs, cudpp segmented scan, MergePathPartitions, KernelInsert into per-pair global
// tables of 131071 slots with <= 25 double-hash probes, then a segmented radix sort of
// every table and a COO->CSR rebuild) and its cuSPARSE csrgemm wrappers
// (src/spgemm.cuh:344-445, src/tc.cuh:62-165). Results: C's structure is the exact
// union of products; rows are sorted by column; int32 values are exact; FP32 values of a
// warp-tier row are summed in increasing position of A's row (the oracle's order, so
// bit-identical); block/global-tier rows accumulate with atomicAdd (order-dependent
// rounding only).
//
// Pipeline (all on the context stream):
//  1. rowinfo: per row, ub = sum of deg_B over A's row (products) -> bin; rows appended to
//     per-bin lists; global-tier rows get a hash table carved from scratch. One sync
//     reads the bin sizes.
//  2. symbolic: per bin, count distinct columns per row with a hash set -> cnt[]
//  3. scan cnt -> row_ptr(C); one sync reads nnz(C) (the caller may allocate C here)
//  4. numeric: per bin, accumulate values in the hash table, then emit the row sorted:
//     warp tier by a shared-memory bitonic sort, block/global tiers by ranking entries
//     against a 64K-column bitmap window (prefix popcounts).
// Bins: 0 no products | 1 ub <= 32: one warp, 64-slot table | 2 ub <= 128: one warp,
// 256-slot table | 3 ub <= 1024: one block, 2048-slot shared table | 4 larger: one block,
// global table of >= 2*ub slots (power of two). Tables stay at most half full.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace apspie {
namespace {

constexpr int kEmptyKey = -1;
constexpr int kBins = 5;
constexpr int kBlockTS = 2048;
constexpr int kSgBlock = 256;
constexpr int kWindowBits = 65536;  // columns per bitmap window
constexpr int kWindowWords = kWindowBits / 32;

struct SgInfo {
    int bin_count[kBins];
    int overflow;  // hash probe overflow or scan overflow
    long long global_slots;
};

__device__ __forceinline__ int bin_of(long long ub, int degA) {
    const long long w = ub > degA ? ub : degA;
    if (ub == 0) return 0;
    if (w <= 32) return 1;
    if (w <= 128) return 2;
    if (w <= 1024) return 3;
    return 4;
}

__device__ __forceinline__ unsigned hash_slot(int col, int log2ts) {
    return (static_cast<unsigned>(col) * 2654435761u) >> (32 - log2ts);
}

template <typename V>
__device__ __forceinline__ V vmul(V a, V b);
template <>
__device__ __forceinline__ float vmul<float>(float a, float b) { return __fmul_rn(a, b); }
template <>
__device__ __forceinline__ int vmul<int>(int a, int b) { return a * b; }
template <typename V>
__device__ __forceinline__ V vadd(V a, V b);
template <>
__device__ __forceinline__ float vadd<float>(float a, float b) { return __fadd_rn(a, b); }
template <>
__device__ __forceinline__ int vadd<int>(int a, int b) { return a + b; }

struct Mat {
    const int *rp;
    const int *ci;
    const void *val;
};

// ---------------------------------------------------------------- 1. row info / bins
__global__ void sg_rowinfo(int m, Mat A, Mat B, long long *ub, int *bin_rows, SgInfo *info,
                           long long *tbl_off) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < m; i += nwarps) {
        const int r0 = A.rp[i], r1 = A.rp[i + 1];
        long long s = 0;
        for (int e = r0 + lane; e < r1; e += 32) {
            const int k = A.ci[e];
            s += B.rp[k + 1] - B.rp[k];
        }
        for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) {
            ub[i] = s;
            const int b = bin_of(s, r1 - r0);
            const int pos = atomicAdd(&info->bin_count[b], 1);
            bin_rows[static_cast<long long>(b) * m + pos] = i;
            if (b == 4) {
                long long ts = 64;
                while (ts < 2 * s) ts <<= 1;
                tbl_off[i] = static_cast<long long>(
                    atomicAdd(reinterpret_cast<unsigned long long *>(&info->global_slots),
                              static_cast<unsigned long long>(ts)));
            }
        }
    }
}

// ---------------------------------------------------------------- warp tier
template <int PL, int TS, typename V>
struct WarpTierSmem {
    static constexpr int UB = 32 * PL;
    int keys[TS];
    V vals[TS];
    int sk_rs[UB];    // B row start of each A entry
    int soff[UB + 1]; // exclusive product offset of each A entry
    V sa[UB];         // A values
    int lk[UB];       // extraction list (sorted)
    V lv[UB];
};

// One warp per row. Products of A entry t are inserted only after every product of
// entries < t (the columns of one entry are distinct), so each output value is summed in
// increasing t exactly as the oracle does.
template <int PL, int TS, int LOG2TS, bool NUMERIC, typename V>
__global__ void __launch_bounds__(kSgBlock) sg_warp(const int *__restrict__ rows, int nrows, Mat A, Mat B,
                                                    int *cnt, const int *__restrict__ crp, int *cci,
                                                    V *cval, SgInfo *info) {
    using S = WarpTierSmem<PL, TS, V>;
    constexpr int UB = S::UB;
    __shared__ S smem[kSgBlock / 32];
    const int lane = threadIdx.x & 31;
    S &sm = smem[threadIdx.x >> 5];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const V *aval = static_cast<const V *>(A.val);
    const V *bval = static_cast<const V *>(B.val);
    for (int w = warp; w < nrows; w += nwarps) {
        const int i = rows[w];
        const int rA = A.rp[i];
        const int degA = A.rp[i + 1] - rA;  // <= UB by binning
        for (int t = lane; t < degA; t += 32) {
            const int k = A.ci[rA + t];
            const int b0 = B.rp[k];
            sm.sk_rs[t] = b0;
            sm.soff[t] = B.rp[k + 1] - b0;
            if (NUMERIC) sm.sa[t] = aval[rA + t];
        }
        for (int s = lane; s < TS; s += 32) {
            sm.keys[s] = kEmptyKey;
            if (NUMERIC) sm.vals[s] = V(0);
        }
        __syncwarp();
        int carry = 0;
        for (int base = 0; base < degA; base += 32) {
            const int t = base + lane;
            const int x = t < degA ? sm.soff[t] : 0;
            int incl = x;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (t < degA) sm.soff[t] = carry + incl - x;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        const int ub = carry;  // <= UB by binning
        if (lane == 0) sm.soff[degA] = ub;
        __syncwarp();
        int pc[PL], pt[PL];
        V pv[PL];
#pragma unroll
        for (int r = 0; r < PL; ++r) {
            const int q = r * 32 + lane;
            pc[r] = 0;
            pt[r] = -1;
            pv[r] = V(0);
            if (q < ub) {
                int lo = 0, hi = degA;  // last t with soff[t] <= q
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (sm.soff[mid] <= q)
                        lo = mid;
                    else
                        hi = mid;
                }
                const int e = sm.sk_rs[lo] + (q - sm.soff[lo]);
                pc[r] = B.ci[e];
                pt[r] = lo;
                if (NUMERIC) pv[r] = vmul<V>(sm.sa[lo], bval[e]);
            }
        }
        int fresh = 0;
#pragma unroll
        for (int r = 0; r < PL; ++r) {
            const int q0 = r * 32;
            if (q0 >= ub) break;
            const int last = (ub - 1 - q0) < 31 ? (ub - 1 - q0) : 31;
            const int t_lo = __shfl_sync(0xffffffffu, pt[r], 0);
            const int t_hi = __shfl_sync(0xffffffffu, pt[r], last);
            for (int t = t_lo; t <= t_hi; ++t) {
                if (pt[r] == t) {
                    unsigned s = hash_slot(pc[r], LOG2TS);
                    int probes = 0;
                    for (;;) {
                        const int k = sm.keys[s];
                        if (k == pc[r]) break;
                        if (k == kEmptyKey) {
                            const int old = atomicCAS(&sm.keys[s], kEmptyKey, pc[r]);
                            if (old == kEmptyKey) {
                                ++fresh;
                                break;
                            }
                            if (old == pc[r]) break;
                        }
                        s = (s + 1) & (TS - 1);
                        if (++probes > TS) {
                            atomicOr(&info->overflow, 1);
                            break;
                        }
                    }
                    if (NUMERIC) sm.vals[s] = vadd<V>(sm.vals[s], pv[r]);
                }
                __syncwarp();
            }
        }
        if (!NUMERIC) {
            for (int o = 16; o; o >>= 1) fresh += __shfl_down_sync(0xffffffffu, fresh, o);
            if (lane == 0) cnt[i] = fresh;
            __syncwarp();
            continue;
        }
        // compact the table (slot order), then bitonic-sort by column
        const int c0 = crp[i];
        const int nrow = crp[i + 1] - c0;
        int pos = 0;
        for (int s0 = 0; s0 < TS; s0 += 32) {
            const int k = sm.keys[s0 + lane];
            const bool v = k != kEmptyKey;
            const unsigned mask = __ballot_sync(0xffffffffu, v);
            if (v) {
                const int p = pos + __popc(mask & ((1u << lane) - 1u));
                if (p < UB) {
                    sm.lk[p] = k;
                    sm.lv[p] = sm.vals[s0 + lane];
                }
            }
            pos += __popc(mask);
        }
        for (int p = pos + lane; p < UB; p += 32) sm.lk[p] = 0x7fffffff;
        __syncwarp();
        for (int k2 = 2; k2 <= UB; k2 <<= 1) {
            for (int j = k2 >> 1; j > 0; j >>= 1) {
                for (int idx = lane; idx < UB / 2; idx += 32) {
                    const int a = 2 * idx - (idx & (j - 1));
                    const int b = a + j;
                    const bool up = (a & k2) == 0;
                    const int ka = sm.lk[a], kb = sm.lk[b];
                    if ((ka > kb) == up) {
                        sm.lk[a] = kb;
                        sm.lk[b] = ka;
                        const V t = sm.lv[a];
                        sm.lv[a] = sm.lv[b];
                        sm.lv[b] = t;
                    }
                }
                __syncwarp();
            }
        }
        for (int p = lane; p < nrow; p += 32) {
            cci[c0 + p] = sm.lk[p];
            cval[c0 + p] = sm.lv[p];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------- block / global tiers
template <typename V>
struct BlockTierSmem {
    int keys[kBlockTS];
    V vals[kBlockTS];
    int sk_rs[kSgBlock];
    int soff[kSgBlock + 1];
    V sa[kSgBlock];
    unsigned bits[kWindowWords];
    int wpre[kWindowWords];  // exclusive popcount prefix of the window's words
    int scan_tmp[33];
    int red[2];
};

template <typename V>
__device__ __forceinline__ void atomic_vadd(V *p, V v);
template <>
__device__ __forceinline__ void atomic_vadd<float>(float *p, float v) { atomicAdd(p, v); }
template <>
__device__ __forceinline__ void atomic_vadd<int>(int *p, int v) { atomicAdd(p, v); }

// One block per row. GLOBAL: the table lives in scratch at tbl_off[i] with a per-row size;
// otherwise it is the block's shared-memory table of kBlockTS slots. Products of all A
// entries are inserted concurrently (values by atomicAdd).
template <bool GLOBAL, bool NUMERIC, typename V>
__global__ void __launch_bounds__(kSgBlock) sg_block(const int *__restrict__ rows, int nrows, Mat A, Mat B,
                                                     const long long *__restrict__ ub_all,
                                                     const long long *__restrict__ tbl_off, int *gkeys,
                                                     V *gvals, int *cnt, const int *__restrict__ crp, int *cci,
                                                     V *cval, SgInfo *info) {
    __shared__ BlockTierSmem<V> sm;
    const V *aval = static_cast<const V *>(A.val);
    const V *bval = static_cast<const V *>(B.val);
    const int tid = threadIdx.x;
    for (int w = blockIdx.x; w < nrows; w += gridDim.x) {
        const int i = rows[w];
        int *keys = sm.keys;
        V *vals = sm.vals;
        long long ts = kBlockTS;
        if (GLOBAL) {
            const long long ub = ub_all[i];
            ts = 64;
            while (ts < 2 * ub) ts <<= 1;
            keys = gkeys + tbl_off[i];
            vals = gvals + tbl_off[i];
        }
        int log2ts = 0;
        while ((1LL << log2ts) < ts) ++log2ts;
        for (long long s = tid; s < ts; s += kSgBlock) {
            keys[s] = kEmptyKey;
            if (NUMERIC) vals[s] = V(0);
        }
        if (tid == 0) sm.red[0] = 0;
        __syncthreads();
        const int rA = A.rp[i];
        const int degA = A.rp[i + 1] - rA;
        int fresh = 0;
        for (int c0 = 0; c0 < degA; c0 += kSgBlock) {
            const int t = c0 + tid;
            int d = 0;
            if (t < degA) {
                const int k = A.ci[rA + t];
                const int b0 = B.rp[k];
                sm.sk_rs[tid] = b0;
                d = B.rp[k + 1] - b0;
                if (NUMERIC) sm.sa[tid] = aval[rA + t];
            }
            int tot;
            const int ex = block_exclusive_scan<kSgBlock>(d, tot, sm.scan_tmp);
            sm.soff[tid] = ex;
            if (tid == 0) sm.soff[kSgBlock] = tot;
            __syncthreads();
            const int nt = degA - c0 < kSgBlock ? degA - c0 : kSgBlock;
            for (int q = tid; q < tot; q += kSgBlock) {
                int lo = 0, hi = nt;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (sm.soff[mid] <= q)
                        lo = mid;
                    else
                        hi = mid;
                }
                const int e = sm.sk_rs[lo] + (q - sm.soff[lo]);
                const int col = B.ci[e];
                unsigned long long s = hash_slot(col, log2ts < 32 ? log2ts : 31) & (ts - 1);
                long long probes = 0;
                for (;;) {
                    const int k = GLOBAL ? __ldcg(keys + s) : keys[s];
                    if (k == col) break;
                    if (k == kEmptyKey) {
                        const int old = atomicCAS(keys + s, kEmptyKey, col);
                        if (old == kEmptyKey) {
                            ++fresh;
                            break;
                        }
                        if (old == col) break;
                    }
                    s = (s + 1) & (ts - 1);
                    if (++probes > ts) {
                        atomicOr(&info->overflow, 1);
                        break;
                    }
                }
                if (NUMERIC) atomic_vadd<V>(vals + s, vmul<V>(sm.sa[lo], bval[e]));
            }
            __syncthreads();
        }
        if (!NUMERIC) {
            for (int o = 16; o; o >>= 1) fresh += __shfl_down_sync(0xffffffffu, fresh, o);
            if ((tid & 31) == 0) atomicAdd(&sm.red[0], fresh);
            __syncthreads();
            if (tid == 0) cnt[i] = sm.red[0];
            __syncthreads();
            continue;
        }
        // emit the row sorted by column: rank entries inside 64K-column bitmap windows
        int cmin = 0x7fffffff, cmax = -1;
        for (long long s = tid; s < ts; s += kSgBlock) {
            const int k = GLOBAL ? __ldcg(keys + s) : keys[s];
            if (k != kEmptyKey) {
                cmin = min(cmin, k);
                cmax = max(cmax, k);
            }
        }
        for (int o = 16; o; o >>= 1) {
            cmin = min(cmin, __shfl_down_sync(0xffffffffu, cmin, o));
            cmax = max(cmax, __shfl_down_sync(0xffffffffu, cmax, o));
        }
        if (tid == 0) {
            sm.red[0] = 0x7fffffff;
            sm.red[1] = -1;
        }
        __syncthreads();
        if ((tid & 31) == 0) {
            atomicMin(&sm.red[0], cmin);
            atomicMax(&sm.red[1], cmax);
        }
        __syncthreads();
        cmin = sm.red[0];
        cmax = sm.red[1];
        const int c0 = crp[i];
        int done = 0;
        for (long long w0 = (cmax < 0 ? 1 : (cmin / kWindowBits)) * static_cast<long long>(kWindowBits);
             w0 <= cmax; w0 += kWindowBits) {
            for (int x = tid; x < kWindowWords; x += kSgBlock) sm.bits[x] = 0u;
            __syncthreads();
            for (long long s = tid; s < ts; s += kSgBlock) {
                const int k = GLOBAL ? __ldcg(keys + s) : keys[s];
                if (k != kEmptyKey && k >= w0 && k < w0 + kWindowBits) {
                    const int off = static_cast<int>(k - w0);
                    atomicOr(&sm.bits[off >> 5], 1u << (off & 31));
                }
            }
            __syncthreads();
            // exclusive prefix of popcounts over the window's words (WPT words per thread)
            constexpr int WPT = kWindowWords / kSgBlock;
            int local = 0;
#pragma unroll
            for (int x = 0; x < WPT; ++x) local += __popc(sm.bits[tid * WPT + x]);
            int tot;
            int run = block_exclusive_scan<kSgBlock>(local, tot, sm.scan_tmp);
#pragma unroll
            for (int x = 0; x < WPT; ++x) {
                sm.wpre[tid * WPT + x] = run;
                run += __popc(sm.bits[tid * WPT + x]);
            }
            __syncthreads();
            // every entry of the window lands at its column's rank
            for (long long s = tid; s < ts; s += kSgBlock) {
                const int k = GLOBAL ? __ldcg(keys + s) : keys[s];
                if (k != kEmptyKey && k >= w0 && k < w0 + kWindowBits) {
                    const int off = static_cast<int>(k - w0);
                    const int word = off >> 5;
                    const int rank = sm.wpre[word] + __popc(sm.bits[word] & ((1u << (off & 31)) - 1u));
                    cci[c0 + done + rank] = k;
                    cval[c0 + done + rank] = GLOBAL ? __ldcg(vals + s) : vals[s];
                }
            }
            done += tot;
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------- host side
struct SgPlan {
    long long *ub;
    int *bin_rows;
    long long *tbl_off;
    int *cnt;
    void *scan_tmp;
    int *gkeys;
    void *gvals;
    SgInfo *info;
    SgInfo h;
};

apspie_status check_pair(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, const char *who) {
    apspie_status st = check_csr_view(ctx, A, who);
    if (st != APSPIE_OK) return st;
    if ((st = check_csr_view(ctx, B, who)) != APSPIE_OK) return st;
    if (A->n != B->m) return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": A.n != B.m");
    if (A->val_type != B->val_type)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": A and B value types differ");
    if (ctx->validate) {
        if ((st = validate_csr(ctx, A, false)) != APSPIE_OK) return st;
        if ((st = validate_csr(ctx, B, false)) != APSPIE_OK) return st;
    }
    return APSPIE_OK;
}

// Runs rowinfo and sizes every buffer; leaves plan.h filled (synchronises once).
apspie_status sg_plan(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, SgPlan &p) {
    const int m = A->m;
    const size_t mi = static_cast<size_t>(m) + 1;
    const size_t base_need =
        Carver::need({mi * 8, static_cast<size_t>(kBins) * mi * 4, mi * 8, mi * 4,
                      scan_scratch_bytes(m) + 64, sizeof(SgInfo)});
    void *base;
    apspie_status st = scratch_reserve(ctx, base_need, &base);
    if (st != APSPIE_OK) return st;
    Carver c(base);
    p.ub = c.take<long long>(mi);
    p.bin_rows = c.take<int>(static_cast<size_t>(kBins) * mi);
    p.tbl_off = c.take<long long>(mi);
    p.cnt = c.take<int>(mi);
    p.scan_tmp = c.take<char>(scan_scratch_bytes(m) + 64);
    p.info = c.take<SgInfo>(1);
    cudaError_t e = cudaMemsetAsync(p.info, 0, sizeof(SgInfo), ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "spgemm info reset");
    Mat a{A->row_ptr, A->col_ind, A->val}, b{B->row_ptr, B->col_ind, B->val};
    if (m > 0) {
        const int blocks = std::min<long long>((static_cast<long long>(m) * 32 + 255) / 256, ctx->num_sms * 16LL);
        sg_rowinfo<<<blocks, 256, 0, ctx->stream>>>(m, a, b, p.ub, p.bin_rows, p.info, p.tbl_off);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(ctx, e, "spgemm rowinfo");
    }
    e = cudaMemcpyAsync(&p.h, p.info, sizeof(SgInfo), cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "spgemm info copy");
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_error(ctx, e, "spgemm sync");
    // global-tier hash tables live in the context's secondary arena
    const size_t gslots = static_cast<size_t>(p.h.global_slots);
    p.gkeys = nullptr;
    p.gvals = nullptr;
    if (gslots > 0) {
        void *tb;
        st = scratch2_reserve(ctx, Carver::need({gslots * 4, gslots * 4}), &tb);
        if (st != APSPIE_OK) return st;
        Carver c2(tb);
        p.gkeys = c2.take<int>(gslots);
        p.gvals = c2.take<char>(gslots * 4);
    }
    return APSPIE_OK;
}

template <bool NUMERIC, typename V>
apspie_status sg_run(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, SgPlan &p, const int *crp,
                     int *cci, V *cval) {
    const int m = A->m;
    Mat a{A->row_ptr, A->col_ind, A->val}, b{B->row_ptr, B->col_ind, B->val};
    const long long mi = static_cast<long long>(m) + 1;
    const int grid_cap = ctx->num_sms * 8;
    (void)mi;
    // per-bin lists are laid out with stride m (sg_rowinfo)
    auto rows = [&](int bin) { return p.bin_rows + static_cast<long long>(bin) * m; };
    int nb = p.h.bin_count[1];
    if (nb > 0) {
        const int g = std::min((nb + 7) / 8, grid_cap);
        sg_warp<1, 64, 6, NUMERIC, V><<<g, kSgBlock, 0, ctx->stream>>>(rows(1), nb, a, b, p.cnt, crp, cci, cval,
                                                                         p.info);
    }
    nb = p.h.bin_count[2];
    if (nb > 0) {
        const int g = std::min((nb + 7) / 8, grid_cap);
        sg_warp<4, 256, 8, NUMERIC, V><<<g, kSgBlock, 0, ctx->stream>>>(rows(2), nb, a, b, p.cnt, crp, cci, cval,
                                                                          p.info);
    }
    nb = p.h.bin_count[3];
    if (nb > 0) {
        const int g = std::min(nb, grid_cap);
        sg_block<false, NUMERIC, V><<<g, kSgBlock, 0, ctx->stream>>>(rows(3), nb, a, b, p.ub, p.tbl_off, p.gkeys,
                                                                      static_cast<V *>(p.gvals), p.cnt, crp, cci,
                                                                      cval, p.info);
    }
    nb = p.h.bin_count[4];
    if (nb > 0) {
        const int g = std::min(nb, grid_cap);
        sg_block<true, NUMERIC, V><<<g, kSgBlock, 0, ctx->stream>>>(rows(4), nb, a, b, p.ub, p.tbl_off, p.gkeys,
                                                                     static_cast<V *>(p.gvals), p.cnt, crp, cci,
                                                                     cval, p.info);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? APSPIE_OK : cuda_error(ctx, e, "spgemm launch");
}

__global__ void zero_empty_rows(const int *rows, int n, int *cnt) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) cnt[rows[k]] = 0;
}

apspie_status sg_symbolic(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, SgPlan &p, int *crp,
                          long long *nnz) {
    apspie_status st;
    const int m = A->m;
    if (p.h.bin_count[0] > 0) {
        const int n0 = p.h.bin_count[0];
        zero_empty_rows<<<std::min((n0 + 255) / 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(p.bin_rows, n0, p.cnt);
    }
    if (A->val_type == APSPIE_VAL_F32)
        st = sg_run<false, float>(ctx, A, B, p, nullptr, nullptr, nullptr);
    else
        st = sg_run<false, int>(ctx, A, B, p, nullptr, nullptr, nullptr);
    if (st != APSPIE_OK) return st;
    if ((st = device_exclusive_scan(ctx, p.cnt, m, crp, p.scan_tmp, &p.info->overflow)) != APSPIE_OK) return st;
    int tail[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(&tail[0], crp + m, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&p.h.overflow, &p.info->overflow, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "spgemm symbolic sync");
    if (p.h.overflow) return set_error(ctx, APSPIE_ERR_HASH_OVERFLOW, "spgemm: hash table or nnz(C) overflow");
    *nnz = tail[0];
    return APSPIE_OK;
}

apspie_status sg_numeric(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, SgPlan &p, const int *crp,
                         int *cci, void *cval) {
    apspie_status st;
    if (A->val_type == APSPIE_VAL_I32)
        st = sg_run<true, int>(ctx, A, B, p, crp, cci, static_cast<int *>(cval));
    else if (A->val_type == APSPIE_VAL_F32)
        st = sg_run<true, float>(ctx, A, B, p, crp, cci, static_cast<float *>(cval));
    else {
        // pattern only: reuse the int path with products of 1s written to a scratch sink
        return set_error(ctx, APSPIE_ERR_UNSUPPORTED, "spgemm numeric needs values (use symbolic for patterns)");
    }
    return st;
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_spgemm_symbolic(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B,
                                     int32_t *d_row_ptr_c, int64_t *nnz_c) {
    if (!ctx || !d_row_ptr_c || !nnz_c) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_pair(ctx, A, B, "apspie_spgemm_symbolic");
    if (st != APSPIE_OK) return st;
    SgPlan p;
    if ((st = sg_plan(ctx, A, B, p)) != APSPIE_OK) return st;
    long long nnz = 0;
    if ((st = sg_symbolic(ctx, A, B, p, d_row_ptr_c, &nnz)) != APSPIE_OK) return st;
    *nnz_c = nnz;
    return APSPIE_OK;
}

apspie_status apspie_spgemm_numeric(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B,
                                    const int32_t *d_row_ptr_c, int32_t *d_col_c, void *d_val_c) {
    if (!ctx || !d_row_ptr_c) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_pair(ctx, A, B, "apspie_spgemm_numeric");
    if (st != APSPIE_OK) return st;
    SgPlan p;
    if ((st = sg_plan(ctx, A, B, p)) != APSPIE_OK) return st;
    return sg_numeric(ctx, A, B, p, d_row_ptr_c, d_col_c, d_val_c);
}

apspie_status apspie_spgemm(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, apspie_csr_owned *C) {
    if (!ctx || !C) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    std::memset(C, 0, sizeof(*C));
    apspie_status st = check_pair(ctx, A, B, "apspie_spgemm");
    if (st != APSPIE_OK) return st;
    if (A->val_type == APSPIE_VAL_NONE)
        return set_error(ctx, APSPIE_ERR_UNSUPPORTED, "apspie_spgemm: values required (F32 or I32)");
    SgPlan p;
    if ((st = sg_plan(ctx, A, B, p)) != APSPIE_OK) return st;
    int32_t *rp = nullptr;
    cudaError_t e = cudaMalloc(&rp, (static_cast<size_t>(A->m) + 1) * sizeof(int32_t));
    if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_spgemm row_ptr");
    long long nnz = 0;
    if ((st = sg_symbolic(ctx, A, B, p, rp, &nnz)) != APSPIE_OK) {
        cudaFree(rp);
        return st;
    }
    int32_t *ci = nullptr;
    void *val = nullptr;
    const size_t n = static_cast<size_t>(nnz > 0 ? nnz : 1);
    if ((e = cudaMalloc(&ci, n * sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMalloc(&val, n * 4)) != cudaSuccess) {
        cudaFree(rp);
        if (ci) cudaFree(ci);
        return cuda_error(ctx, e, "apspie_spgemm C");
    }
    if ((st = sg_numeric(ctx, A, B, p, rp, ci, val)) != APSPIE_OK) {
        cudaFree(rp);
        cudaFree(ci);
        cudaFree(val);
        return st;
    }
    C->m = A->m;
    C->n = B->n;
    C->nnz = static_cast<int32_t>(nnz);
    C->val_type = A->val_type;
    C->row_ptr = rp;
    C->col_ind = ci;
    C->val = val;
    return APSPIE_OK;
}

void apspie_csr_free(apspie_csr_owned *C) {
    if (!C) return;
    if (C->row_ptr) cudaFree(C->row_ptr);
    if (C->col_ind) cudaFree(C->col_ind);
    if (C->val) cudaFree(C->val);
    std::memset(C, 0, sizeof(*C));
}

}  // extern "C"
