// The frontier expander shared by the persistent BFS / SSSP / MIS kernels.
//
// It replaces the reference's per-level library chain (src/mXv.cuh:142-176,
// src/spmspvBfs.cuh:178-186, src/spmspvMis.cuh:245-263): Scan -> streamCompact ->
// IntervalGather(row lengths) -> Scan -> IntervalGather(row starts) ->
// IntervalGather/Expand(neighbours), with two D2H count reads per level. Here:
//
//  phase A  every block takes a contiguous chunk of the frontier queue, reads each
//           entry's CSR row start and length, and writes a block-local exclusive scan
//           of the lengths plus one chunk total (no host round trip);
//  barrier
//  phase B  every block loads the chunk totals (the second level of the scan), and the
//           (entries + edges) merge path is cut into tiles of BLOCK*VT items. Each tile
//           finds its two split points by binary search on the diagonal, stages its
//           entries' offsets/row starts in shared memory, merges them serially per
//           thread to label every edge slot with its owning entry, and then visits the
//           tile's edges strided across the block so that neighbour-index loads of a row
//           are coalesced. The semiring operation runs on each (entry, edge) pair in the
//           same pass (no materialised neighbour list, no sort).
#pragma once

#include "common.cuh"

namespace apspie {

constexpr int kSplitBatch = 256;

template <int BLOCK, int VT>
struct ExpandSmem {
    static constexpr int NV = BLOCK * VT;
    int base[kMaxGrid + 1];  // exclusive prefix of chunk totals
    int off[NV + 1];         // global edge offset of each staged entry
    int rs[NV + 1];          // CSR row start of each staged entry
    int aux[NV + 1];         // per-entry payload (vertex id, distance, ...)
    int seg[NV];             // tile edge slot -> staged entry
    int scan_tmp[33];
    int tsplit[kSplitBatch + 1];  // merge-path split of each tile of the current batch
};

// Phase A over this block's chunk of queue q[0, nf). hook(i, v, deg) may rewrite the
// degree (e.g. 0 for an entry that needs no expansion) and do per-entry work.
template <int BLOCK, class Hook>
__device__ __forceinline__ void frontier_phase_a(const int *__restrict__ q, int nf,
                                                 const int *__restrict__ row_ptr, int *rs,
                                                 int *loc_off, int *chunk_sum, int *scan_tmp,
                                                 Hook hook) {
    const int G = gridDim.x;
    const int C = (nf + G - 1) / G;
    const int c0 = min(static_cast<int>(blockIdx.x) * C, nf);
    const int c1 = min(c0 + C, nf);
    int carry = 0;
    for (int base = c0; base < c1; base += BLOCK) {
        const int i = base + threadIdx.x;
        int deg = 0;
        if (i < c1) {
            const int v = __ldcg(q + i);
            const int r0 = __ldg(row_ptr + v);
            deg = __ldg(row_ptr + v + 1) - r0;
            deg = hook(i, v, deg);
            rs[i] = r0;
        }
        int tot;
        const int ex = block_exclusive_scan<BLOCK>(deg, tot, scan_tmp);
        if (i < c1) loc_off[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) chunk_sum[blockIdx.x] = carry;
}

// Loads the chunk totals of phase A into base[] as an exclusive prefix; returns the total
// number of edges of the frontier.
template <int BLOCK>
__device__ __forceinline__ int frontier_chunk_bases(const int *__restrict__ chunk_sum, int *base,
                                                    int *scan_tmp) {
    const int G = gridDim.x;
    const int per = (G + BLOCK - 1) / BLOCK;
    const int t0 = threadIdx.x * per;
    int local = 0;
    for (int k = 0; k < per; ++k)
        if (t0 + k < G) local += __ldcg(chunk_sum + t0 + k);
    int tot;
    int run = block_exclusive_scan<BLOCK>(local, tot, scan_tmp);
    for (int k = 0; k < per; ++k)
        if (t0 + k < G) {
            base[t0 + k] = run;
            run += __ldcg(chunk_sum + t0 + k);
        }
    if (threadIdx.x == 0) base[G] = tot;
    __syncthreads();
    return tot;
}

// Number of entries among the first `diag` items of the merge of entry offsets
// (offset(j) = base[j / C] + loc_off[j]) with edge indices 0..E-1, entries first on ties.
__device__ __forceinline__ int frontier_merge_path(long long diag, int nf, int E,
                                                   const int *__restrict__ loc_off,
                                                   const int *base, int C) {
    long long lo = diag - E > 0 ? diag - E : 0;
    long long hi = diag < nf ? diag : nf;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        const int off = base[mid / C] + __ldcg(loc_off + mid);
        if (off <= diag - 1 - mid)
            lo = mid + 1;
        else
            hi = mid;
    }
    return static_cast<int>(lo);
}

// Phase B. load(j, k, sm) stages entry j's payload into sm.aux[k]; op(valid, k, idx, sm)
// handles the edge at CSR position idx owned by staged entry k. `op` is called by every
// thread of the block the same number of times (valid=false for idle slots), so it may
// use warp collectives.
//
// Block b owns a contiguous run of tiles. The split points of up to kSplitBatch tiles are
// found in parallel (one binary search per thread) before the tiles are walked, so the
// dependent global-memory search latency is paid once per batch rather than per tile.
template <int BLOCK, int VT, class Load, class Op>
__device__ __forceinline__ void frontier_expand(int nf, int E, const int *__restrict__ loc_off,
                                                const int *__restrict__ rs,
                                                ExpandSmem<BLOCK, VT> &sm, Load load, Op op) {
    constexpr int NV = BLOCK * VT;
    const int G = gridDim.x;
    const int C = (nf + G - 1) / G;
    const long long total = static_cast<long long>(nf) + E;
    const long long ntiles = (total + NV - 1) / NV;
    const long long per = (ntiles + G - 1) / G;
    const long long t_begin = static_cast<long long>(blockIdx.x) * per;
    const long long t_end = t_begin + per < ntiles ? t_begin + per : ntiles;
    for (long long tb = t_begin; tb < t_end; tb += kSplitBatch) {
        const long long te = tb + kSplitBatch < t_end ? tb + kSplitBatch : t_end;
        for (int s = threadIdx.x; s <= te - tb; s += BLOCK) {
            long long d = (tb + s) * NV;
            if (d > total) d = total;
            sm.tsplit[s] = frontier_merge_path(d, nf, E, loc_off, sm.base, C);
        }
        __syncthreads();
        for (long long tile = tb; tile < te; ++tile) {
            const long long d0 = tile * NV;
            const long long d1 = d0 + NV < total ? d0 + NV : total;
            const int a0 = sm.tsplit[tile - tb];
            const int a1 = sm.tsplit[tile - tb + 1];
            const int e0 = static_cast<int>(d0 - a0);
            const int e1 = static_cast<int>(d1 - a1);
            const int jb = a0 > 0 ? a0 - 1 : 0;
            const int ne = a1 - jb;
            for (int k = threadIdx.x; k < ne; k += BLOCK) {
                const int j = jb + k;
                sm.off[k] = sm.base[j / C] + __ldcg(loc_off + j);
                sm.rs[k] = __ldcg(rs + j);
                load(j, k, sm);
            }
            __syncthreads();
            const int tcount = static_cast<int>(d1 - d0);
            const int diag = threadIdx.x * VT;
            if (diag < tcount) {
                const int acount = a1 - a0, bcount = e1 - e0;
                int lo = diag - bcount > 0 ? diag - bcount : 0;
                int hi = diag < acount ? diag : acount;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (sm.off[a0 + mid - jb] <= e0 + diag - 1 - mid)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                int ja = a0 + lo, eb = e0 + diag - lo;
                int cur = ja - 1 - jb;
                const int end = diag + VT < tcount ? diag + VT : tcount;
                for (int it = diag; it < end; ++it) {
                    if (ja < a1 && sm.off[ja - jb] <= eb) {
                        cur = ja - jb;
                        ++ja;
                    } else {
                        sm.seg[eb - e0] = cur;
                        ++eb;
                    }
                }
            }
            __syncthreads();
            const int ned = e1 - e0;
            for (int k0 = 0; k0 < ned; k0 += BLOCK) {
                const int el = k0 + threadIdx.x;
                const bool valid = el < ned;
                int k = 0, idx = 0;
                if (valid) {
                    k = sm.seg[el];
                    idx = sm.rs[k] + (e0 + el - sm.off[k]);
                }
                op(valid, k, idx, sm);
            }
            __syncthreads();
        }
    }
}

}  // namespace apspie
