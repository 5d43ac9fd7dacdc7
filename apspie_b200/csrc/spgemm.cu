// Row-binned hash SpGEMM  C = A * B  (Gustavson, row by row).
//
// Replaces the reference's 2-D partitioned outer-product hash SpGEMM
// (src/spgemm.cuh:131-342, src/spgemmKernel.cuh:439-738: CSR->DCSC per partition,
// SetOpPairs, cudpp segmented scan, MergePathPartitions, KernelInsert into per-pair global
// tables of 131071 slots with <= 25 double-hash probes, then a segmented radix sort of
// every table and a COO->CSR rebuild) and its cuSPARSE csrgemm wrappers
// (src/spgemm.cuh:344-445, src/tc.cuh:62-165). Results: C's structure is the exact
// union of products; rows are sorted by column; int32 values are exact; FP32 values of a
// register-tier row (at most 128 products) are summed in increasing position of A's row
// (the oracle's order, so bit-identical); block/global-tier rows accumulate with
// atomicAdd (order-dependent rounding only).
//
// Pipeline (all on the context stream):
//  1. rowinfo: per row, ub = sum of deg_B over A's row (products) -> bin; rows appended to
//     per-bin lists; global-tier rows get a hash table carved from scratch. One sync
//     reads the bin sizes.
//  2. symbolic: per bin, count distinct columns per row with a hash set -> cnt[]
//  3. scan cnt -> row_ptr(C); one sync reads nnz(C) (the caller may allocate C here)
//  4. numeric: register tiers sort the products and sum each column's run; hash tiers
//     accumulate values in the table, then emit the row sorted by ranking entries against
//     a 64K-column bitmap window (prefix popcounts).
// Bins: 0 no products | 1-3 ub <= 32 / 64 / 128: one warp per row, the row's products
// held in registers (1, 2 or 4 per lane) and sorted by (column, product index) with a
// register bitonic network; duplicates are then adjacent and summed in product order |
// 4 ub <= 1024: one block, 2048-slot shared table | 5 larger: one block, global table of
// >= 2*ub slots (power of two). Tables stay at most half full.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace apspie {
namespace {

constexpr int kEmptyKey = -1;
constexpr int kBins = 6;
constexpr int kBinBlock = 4;   // shared-memory hash table tier
constexpr int kBinGlobal = 5;  // global-memory hash table tier
constexpr int kBlockTS = 2048;
constexpr int kSgBlock = 256;
constexpr int kWindowBits = 65536;  // columns per bitmap window
constexpr int kWindowWords = kWindowBits / 32;

struct SgInfo {
    int bin_count[kBins];
    int overflow;  // hash probe overflow or scan overflow
    long long global_slots;
};

// Rows of at most reg_max products (0, 32, 64 or 128) go to the register tiers (needs B
// with at most 2^24 columns, so that a key column << 7 | product stays below the padding
// key 0xffffffff; the host passes reg_max 0 otherwise), rows of at most block_max (<= 1024,
// the shared table holds 2048 slots) to the shared-memory table, longer rows to a global
// table.
__device__ __forceinline__ int bin_of(long long ub, int degA, int reg_max, int block_max) {
    const long long w = ub > degA ? ub : degA;
    if (ub == 0) return 0;
    if (w <= reg_max) return w <= 32 ? 1 : (w <= 64 ? 2 : 3);
    if (w <= block_max) return kBinBlock;
    return kBinGlobal;
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
// 8 lanes per row: ub = sum of deg_B over A's row, and the row's bin.
__global__ void sg_rowinfo(int m, Mat A, Mat B, int reg_max, int block_max, long long *ub,
                           unsigned char *row_bin, SgInfo *info, long long *tbl_off) {
    const int sub = threadIdx.x & 7;
    const int grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int ngrp = (gridDim.x * blockDim.x) >> 3;
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    for (int i0 = grp - (grp & 3); i0 < m; i0 += ngrp) {  // the warp's 4 groups move together
        const int i = i0 + (grp & 3);
        long long s = 0;
        int r0 = 0, r1 = 0;
        if (i < m) {
            r0 = __ldg(A.rp + i);
            r1 = __ldg(A.rp + i + 1);
            for (int e = r0 + sub; e < r1; e += 8) {
                const int k = __ldg(A.ci + e);
                s += __ldg(B.rp + k + 1) - __ldg(B.rp + k);
            }
        }
        for (int o = 4; o; o >>= 1) s += __shfl_down_sync(gmask, s, o, 8);
        if (i < m && sub == 0) {
            ub[i] = s;
            const int b = bin_of(s, r1 - r0, reg_max, block_max);
            row_bin[i] = static_cast<unsigned char>(b);
            if (b == kBinGlobal) {
                long long ts = 64;
                while (ts < 2 * s) ts <<= 1;
                tbl_off[i] = static_cast<long long>(
                    atomicAdd(reinterpret_cast<unsigned long long *>(&info->global_slots),
                              static_cast<unsigned long long>(ts)));
            }
        }
    }
}

// Per-bin row lists (stride m): each block counts its rows per bin with warp ballots,
// reserves room with one global atomic per bin, then scatters.
__global__ void sg_binlists(int m, const unsigned char *__restrict__ row_bin, int *bin_rows, SgInfo *info) {
    __shared__ int cnt[kBins];
    __shared__ int base[kBins];
    const int lane = threadIdx.x & 31;
    for (int c0 = blockIdx.x * blockDim.x; c0 < m; c0 += gridDim.x * blockDim.x) {
        if (threadIdx.x < kBins) cnt[threadIdx.x] = 0;
        __syncthreads();
        const int i = c0 + threadIdx.x;
        const int b = i < m ? row_bin[i] : -1;
        int pos = 0;
#pragma unroll
        for (int k = 0; k < kBins; ++k) {
            const unsigned mk = __ballot_sync(0xffffffffu, b == k);
            int wbase = 0;
            if (mk && lane == __ffs(mk) - 1) wbase = atomicAdd(&cnt[k], __popc(mk));
            wbase = __shfl_sync(0xffffffffu, wbase, mk ? __ffs(mk) - 1 : 0);
            if (b == k) pos = wbase + __popc(mk & ((1u << lane) - 1u));
        }
        __syncthreads();
        if (threadIdx.x < kBins && cnt[threadIdx.x])
            base[threadIdx.x] = atomicAdd(&info->bin_count[threadIdx.x], cnt[threadIdx.x]);
        __syncthreads();
        if (b >= 0) bin_rows[static_cast<long long>(b) * m + base[b] + pos] = i;
        __syncthreads();
    }
}

__device__ __forceinline__ void st_stream(float *p, float v) { __stcs(p, v); }
__device__ __forceinline__ void st_stream(int *p, int v) { __stcs(p, v); }

// ---------------------------------------------------------------- register (warp) tier
template <int PL, typename V>
struct RegTierSmem {
    static constexpr int N = 32 * PL;
    int soff[N + 1];  // exclusive product offset of each A entry
    int bs[N];        // B row start of each A entry
    V av[N];          // A values
    V pv[N];          // product values, by product index
    unsigned skey[N]; // sorted keys (numeric: walked by the head of each run)
    int tab[2 * N];   // symbolic: hash set of the row's columns
};

// One warp per row of at most N = 32 * PL products. Product q (element r * 32 + lane) of
// A entry t gets the key (column << QB) | q; after a bitonic sort of the keys in registers
// the products of one output column are adjacent and in increasing q, i.e. increasing
// position in A's row, so a run's head sums them in the oracle's order (bit-identical
// FP32). The symbolic pass only counts distinct columns, with a 2N-slot shared-memory hash
// set instead of the sort. Requires B->n <= 2^24 (see bin_of).
template <int PL, bool NUMERIC, typename V>
__global__ void __launch_bounds__(kSgBlock) sg_reg(const int *__restrict__ rows, int nrows, Mat A, Mat B,
                                                   int *cnt, const int *__restrict__ crp, int *cci, V *cval) {
    constexpr int N = 32 * PL;
    constexpr int QB = PL == 1 ? 5 : (PL == 2 ? 6 : 7);
    constexpr unsigned QMASK = (1u << QB) - 1u;
    constexpr unsigned PAD = 0xffffffffu;
    using S = RegTierSmem<PL, V>;
    __shared__ S smem[kSgBlock / 32];
    const int lane = threadIdx.x & 31;
    S &sm = smem[threadIdx.x >> 5];
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const V *aval = static_cast<const V *>(A.val);
    const V *bval = static_cast<const V *>(B.val);
    for (int w = warp; w < nrows; w += nwarps) {
        const int i = rows[w];
        const int rA = __ldg(A.rp + i);
        const int degA = __ldg(A.rp + i + 1) - rA;  // <= N by binning
        // A entries: B row start and length, A value
        int len[PL];
#pragma unroll
        for (int r = 0; r < PL; ++r) {
            const int t = r * 32 + lane;
            len[r] = 0;
            if (t < degA) {
                const int k = __ldg(A.ci + rA + t);
                const int b0 = __ldg(B.rp + k);
                len[r] = __ldg(B.rp + k + 1) - b0;
                sm.bs[t] = b0;
                if (NUMERIC) sm.av[t] = aval[rA + t];
            }
        }
        int carry = 0;
#pragma unroll
        for (int r = 0; r < PL; ++r) {
            int incl = len[r];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int t = r * 32 + lane;
            if (t < degA) sm.soff[t] = carry + incl - len[r];
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        const int ub = carry;  // <= N by binning
        if (lane == 0) sm.soff[degA] = ub;
        __syncwarp();
        // gather the products and build the keys
        unsigned key[PL];
#pragma unroll
        for (int r = 0; r < PL; ++r) {
            const int q = r * 32 + lane;
            key[r] = PAD;
            if (q < ub) {
                int lo = 0, hi = degA;  // last t with soff[t] <= q
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (sm.soff[mid] <= q)
                        lo = mid;
                    else
                        hi = mid;
                }
                const int e = sm.bs[lo] + (q - sm.soff[lo]);
                key[r] = (static_cast<unsigned>(__ldg(B.ci + e)) << QB) | static_cast<unsigned>(q);
                if (NUMERIC) sm.pv[q] = vmul<V>(sm.av[lo], bval[e]);
            }
        }
        if (!NUMERIC) {
            // count distinct columns: insert into the (half-full at most) set
#pragma unroll
            for (int r = 0; r < 2 * PL; ++r) sm.tab[r * 32 + lane] = -1;
            __syncwarp();
            int fresh = 0;
#pragma unroll
            for (int r = 0; r < PL; ++r) {
                if (key[r] == PAD) continue;
                const int col = static_cast<int>(key[r] >> QB);
                unsigned slot = (static_cast<unsigned>(col) * 2654435761u) >> (32 - (QB + 1));
                for (int probe = 0; probe < 2 * N; ++probe) {
                    const int old = atomicCAS(&sm.tab[slot], -1, col);
                    if (old == -1) {
                        ++fresh;
                        break;
                    }
                    if (old == col) break;
                    slot = (slot + 1) & (2 * N - 1);
                }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) fresh += __shfl_down_sync(0xffffffffu, fresh, o);
            if (lane == 0) cnt[i] = fresh;
            __syncwarp();
            continue;
        }
        // bitonic sort of the N keys, element index r * 32 + lane
#pragma unroll
        for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                if (j >= 32) {
#pragma unroll
                    for (int r = 0; r < PL; ++r) {
                        const int p = r ^ (j >> 5);
                        if (p > r) {
                            const bool up = (((r * 32) & k) == 0);
                            const unsigned a = key[r], b = key[p];
                            if ((a > b) == up) {
                                key[r] = b;
                                key[p] = a;
                            }
                        }
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < PL; ++r) {
                        const unsigned other = __shfl_xor_sync(0xffffffffu, key[r], j);
                        const bool up = (((r * 32 + lane) & k) == 0);
                        const bool lower = (lane & j) == 0;
                        key[r] = (lower == up) ? min(key[r], other) : max(key[r], other);
                    }
                }
            }
        }
        // run heads: first element of each column
        bool head[PL];
        unsigned hmask[PL];
#pragma unroll
        for (int r = 0; r < PL; ++r) {
            unsigned prev = __shfl_up_sync(0xffffffffu, key[r], 1);
            if (r > 0) {
                const unsigned last = __shfl_sync(0xffffffffu, key[r - 1], 31);
                if (lane == 0) prev = last;
            }
            head[r] = key[r] != PAD && ((r == 0 && lane == 0) || (prev >> QB) != (key[r] >> QB));
            hmask[r] = __ballot_sync(0xffffffffu, head[r]);
        }
#pragma unroll
        for (int r = 0; r < PL; ++r) sm.skey[r * 32 + lane] = key[r];
        __syncwarp();
        const int c0 = crp[i];
        int before = 0;
#pragma unroll
        for (int r = 0; r < PL; ++r) {
            if (head[r]) {
                const int rank = before + __popc(hmask[r] & ((1u << lane) - 1u));
                const unsigned col = key[r] >> QB;
                V sum = sm.pv[key[r] & QMASK];
                for (int f = r * 32 + lane + 1; f < ub; ++f) {
                    const unsigned kf = sm.skey[f];
                    if ((kf >> QB) != col) break;
                    sum = vadd<V>(sum, sm.pv[kf & QMASK]);
                }
                // streaming stores: C is written once and never re-read here, so it should
                // not push B (re-read by every row that names it) out of L2
                __stcs(cci + c0 + rank, static_cast<int>(col));
                st_stream(cval + c0 + rank, sum);
            }
            before += __popc(hmask[r]);
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
                    __stcs(cci + c0 + done + rank, k);
                    st_stream(cval + c0 + done + rank, GLOBAL ? __ldcg(vals + s) : vals[s]);
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
    unsigned char *row_bin;
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
                      scan_scratch_bytes(m) + 64, sizeof(SgInfo), mi});
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
    p.row_bin = c.take<unsigned char>(mi);
    cudaError_t e = cudaMemsetAsync(p.info, 0, sizeof(SgInfo), ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "spgemm info reset");
    Mat a{A->row_ptr, A->col_ind, A->val}, b{B->row_ptr, B->col_ind, B->val};
    if (m > 0) {
        const int blocks = std::min<long long>((static_cast<long long>(m) * 8 + 255) / 256, ctx->num_sms * 16LL);
        const apspie_tune_params tp = effective_params(ctx, APSPIE_TUNE_SPGEMM, A);
        const int reg_max = B->n <= (1 << 24) ? tp.spgemm_reg_max : 0;
        sg_rowinfo<<<blocks, 256, 0, ctx->stream>>>(m, a, b, reg_max, tp.spgemm_block_max, p.ub, p.row_bin,
                                                    p.info, p.tbl_off);
        const int lblocks = std::min<long long>((static_cast<long long>(m) + 255) / 256, ctx->num_sms * 8LL);
        sg_binlists<<<lblocks, 256, 0, ctx->stream>>>(m, p.row_bin, p.bin_rows, p.info);
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
    const int reg_cap = ctx->num_sms * 16;
    int nb = p.h.bin_count[1];
    if (nb > 0)
        sg_reg<1, NUMERIC, V><<<std::min((nb + 7) / 8, reg_cap), kSgBlock, 0, ctx->stream>>>(rows(1), nb, a, b,
                                                                                             p.cnt, crp, cci, cval);
    nb = p.h.bin_count[2];
    if (nb > 0)
        sg_reg<2, NUMERIC, V><<<std::min((nb + 7) / 8, reg_cap), kSgBlock, 0, ctx->stream>>>(rows(2), nb, a, b,
                                                                                             p.cnt, crp, cci, cval);
    nb = p.h.bin_count[3];
    if (nb > 0)
        sg_reg<4, NUMERIC, V><<<std::min((nb + 7) / 8, reg_cap), kSgBlock, 0, ctx->stream>>>(rows(3), nb, a, b,
                                                                                             p.cnt, crp, cci, cval);
    nb = p.h.bin_count[kBinBlock];
    if (nb > 0) {
        const int g = std::min(nb, grid_cap);
        sg_block<false, NUMERIC, V><<<g, kSgBlock, 0, ctx->stream>>>(rows(kBinBlock), nb, a, b, p.ub, p.tbl_off,
                                                                      p.gkeys, static_cast<V *>(p.gvals), p.cnt,
                                                                      crp, cci, cval, p.info);
    }
    nb = p.h.bin_count[kBinGlobal];
    if (nb > 0) {
        const int g = std::min(nb, grid_cap);
        sg_block<true, NUMERIC, V><<<g, kSgBlock, 0, ctx->stream>>>(rows(kBinGlobal), nb, a, b, p.ub, p.tbl_off,
                                                                     p.gkeys, static_cast<V *>(p.gvals), p.cnt,
                                                                     crp, cci, cval, p.info);
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

bool same_view(const apspie_csr &x, const apspie_csr *y) {
    return x.m == y->m && x.n == y->n && x.nnz == y->nnz && x.val_type == y->val_type &&
           x.row_ptr == y->row_ptr && x.col_ind == y->col_ind && x.val == y->val;
}

// The validation pass (ctx->validate) reserves no scratch, so it leaves the epoch alone.
void sg_cache_store(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, const SgPlan &p) {
    apspie_spgemm_plan_cache &c = ctx->sg_cache;
    c.a = *A;
    c.b = *B;
    c.dev[0] = p.ub;
    c.dev[1] = p.bin_rows;
    c.dev[2] = p.tbl_off;
    c.dev[3] = p.cnt;
    c.dev[4] = p.scan_tmp;
    c.dev[5] = p.gkeys;
    c.dev[6] = p.gvals;
    c.dev[7] = p.info;
    static_assert(kBins <= 8, "cache layout");
    for (int b = 0; b < kBins; ++b) c.host[b] = p.h.bin_count[b];
    c.host[8] = p.h.global_slots;
    c.host[9] = reinterpret_cast<long long>(p.row_bin);
    c.epoch = ctx->scratch_epoch;
    c.valid = true;
}

bool sg_cache_load(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B, SgPlan &p) {
    const apspie_spgemm_plan_cache &c = ctx->sg_cache;
    if (!c.valid || c.epoch != ctx->scratch_epoch || !same_view(c.a, A) || !same_view(c.b, B)) return false;
    p.ub = static_cast<long long *>(c.dev[0]);
    p.bin_rows = static_cast<int *>(c.dev[1]);
    p.tbl_off = static_cast<long long *>(c.dev[2]);
    p.cnt = static_cast<int *>(c.dev[3]);
    p.scan_tmp = c.dev[4];
    p.gkeys = static_cast<int *>(c.dev[5]);
    p.gvals = c.dev[6];
    p.info = static_cast<SgInfo *>(c.dev[7]);
    std::memset(&p.h, 0, sizeof(p.h));
    for (int b = 0; b < kBins; ++b) p.h.bin_count[b] = static_cast<int>(c.host[b]);
    p.h.global_slots = c.host[8];
    p.row_bin = reinterpret_cast<unsigned char *>(c.host[9]);
    return true;
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_spgemm_symbolic(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B,
                                     int32_t *d_row_ptr_c, int64_t *nnz_c) {
    if (!ctx || !d_row_ptr_c || !nnz_c) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    ctx->sg_cache.valid = false;
    apspie_status st = check_pair(ctx, A, B, "apspie_spgemm_symbolic");
    if (st != APSPIE_OK) return st;
    SgPlan p;
    if ((st = sg_plan(ctx, A, B, p)) != APSPIE_OK) return st;
    long long nnz = 0;
    if ((st = sg_symbolic(ctx, A, B, p, d_row_ptr_c, &nnz)) != APSPIE_OK) return st;
    *nnz_c = nnz;
    sg_cache_store(ctx, A, B, p);
    return APSPIE_OK;
}

apspie_status apspie_spgemm_numeric(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B,
                                    const int32_t *d_row_ptr_c, int32_t *d_col_c, void *d_val_c) {
    if (!ctx || !d_row_ptr_c) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_pair(ctx, A, B, "apspie_spgemm_numeric");
    if (st != APSPIE_OK) return st;
    SgPlan p;
    if (!sg_cache_load(ctx, A, B, p) && (st = sg_plan(ctx, A, B, p)) != APSPIE_OK) return st;
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
