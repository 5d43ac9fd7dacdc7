// The frontier expander shared by the persistent BFS and SSSP kernels (single-source and
// batched).
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
//  phase B  every block loads the chunk totals (the second level of the scan). The merge
//           path of (frontier entries, edges) is cut into warp tiles of 32*VT items; each
//           block owns a contiguous run of them. The block finds the split point of every
//           tile of a batch in parallel (one two-level binary search per thread: chunk
//           bases in shared memory, then the chunk's local offsets), then each warp walks
//           its tiles on its own: it stages the tile's entries in its shared-memory slice,
//           merges them per lane to label every edge slot with its owning entry, and hands
//           each lane VT edges (strided, so a row's neighbour indices are read coalesced)
//           whose loads the operation issues back to back. No block barrier inside the
//           tile loop; the semiring operation runs on every (entry, edge) pair in the same
//           pass (no materialised neighbour list, no sort).
#pragma once

#include "common.cuh"

namespace apspie {

// Per-warp staging slice. EXTRA adds the second payload and the per-entry accumulator
// (batched BFS and SSSP); BFS and SSSP leave them out to keep shared memory (occupancy) down.
template <int WT, bool EXTRA>
struct WarpSlice {
    int off[WT + 1];   // global edge offset of each staged entry
    int rs[WT + 1];    // CSR row start of each staged entry
    int aux[WT + 1];   // per-entry payload (distance snapshot, vertex id, ...)
    int aux2[WT + 1];  // second payload (priority, ...)
    int flag[WT + 1];  // per-entry accumulator flushed after the tile
    int seg[WT];       // tile edge slot -> staged entry
};
template <int WT>
struct WarpSlice<WT, false> {
    int off[WT + 1];
    int rs[WT + 1];
    int aux[WT + 1];
    int seg[WT];
};

template <int BLOCK, int VT, bool EXTRA = true>
struct ExpandSmem {
    static constexpr int NWARP = BLOCK / 32;
    static constexpr int WT = 32 * VT;  // items (entries + edges) per warp tile
    static constexpr int BATCH = BLOCK; // warp tiles whose splits are found together
    using Warp = WarpSlice<WT, EXTRA>;
    static constexpr int QCAP = 128;  // per-warp queue staging (see WarpQueue)
    int qbuf[NWARP][2][QCAP];
    int base[kMaxGrid + 1];  // exclusive prefix of chunk totals
    int tsplit[BATCH + 1];   // merge-path split of each warp tile of the current batch
    int next_tile;           // tiles of the batch handed out so far (warps take them in turn)
    int scan_tmp[33];
    Warp w[NWARP];
};

struct RowIsEntry {
    __device__ __forceinline__ int operator()(int e) const { return e; }
};

// Phase A over this block's chunk of queue q[0, nf). hook(i, v, deg) may rewrite the
// degree (e.g. 0 for an entry that needs no expansion) and do per-entry work; the CSR row
// of queue entry e is row_of(e) (the entry itself unless the entry packs more).
template <int BLOCK, class Hook, class RowOf = RowIsEntry>
__device__ __forceinline__ void frontier_phase_a(const int *__restrict__ q, int nf,
                                                 const int *__restrict__ row_ptr, int *rs,
                                                 int *loc_off, int *chunk_sum, int *scan_tmp,
                                                 Hook hook, RowOf row_of = RowOf(), VGrid vg = hw_grid()) {
    const int G = vg.n;
    const int C = (nf + G - 1) / G;
    const int c0 = min(vg.id * C, nf);
    const int c1 = min(c0 + C, nf);
    int carry = 0;
    for (int base = c0; base < c1; base += BLOCK) {
        const int i = base + threadIdx.x;
        int deg = 0;
        if (i < c1) {
            const int v = __ldcg(q + i);
            const int row = row_of(v);
            const int r0 = __ldg(row_ptr + row);
            deg = __ldg(row_ptr + row + 1) - r0;
            deg = hook(i, v, deg);
            rs[i] = r0;
        }
        int tot;
        const int ex = block_exclusive_scan<BLOCK>(deg, tot, scan_tmp);
        if (i < c1) loc_off[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) chunk_sum[vg.id] = carry;
}

// Loads the chunk totals of phase A into base[] as an exclusive prefix; returns the total
// number of edges of the frontier.
template <int BLOCK>
__device__ __forceinline__ int frontier_chunk_bases(const int *__restrict__ chunk_sum, int *base,
                                                    int *scan_tmp, VGrid vg = hw_grid()) {
    const int G = vg.n;
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
// The first entry of every chunk has loc_off 0, so the search first bisects the chunk
// starts in shared memory and then at most one chunk's local offsets in global memory.
__device__ __forceinline__ int frontier_merge_path(long long diag, int nf, int E,
                                                   const int *__restrict__ loc_off,
                                                   const int *base, int C) {
    long long lo = diag - E > 0 ? diag - E : 0;
    long long hi = diag < nf ? diag : nf;
    if (lo >= hi) return static_cast<int>(lo);
    long long clo = (lo + C - 1) / C, chi = (hi - 1) / C;
    while (clo <= chi) {
        const long long c = (clo + chi) >> 1;
        if (base[c] <= diag - 1 - c * C) {
            lo = c * C + 1;
            clo = c + 1;
        } else {
            hi = c * C;
            chi = c - 1;
        }
    }
    if (lo < hi) {
        const int cb = base[lo / C];
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (cb + __ldcg(loc_off + mid) <= diag - 1 - mid)
                lo = mid + 1;
            else
                hi = mid;
        }
    }
    return static_cast<int>(lo);
}

// Phase B. load(j, k, ws) stages entry j's payload into the warp slice at k;
// op(valid, k, idx, ws) handles a lane's VT edges (CSR positions idx[], owning staged
// entries k[]); post(ne, ws) runs after the tile's edges (per-entry flushes). All three
// are called by every lane of the warp, so they may use warp collectives. DYN: warps claim
// the tiles of their block's batch in turn (else tile i goes to warp i % NWARP).
template <int BLOCK, int VT, bool EXTRA, bool DYN = true, class Load, class Op, class Post>
__device__ __forceinline__ void frontier_expand(int nf, int E, const int *__restrict__ loc_off,
                                                const int *__restrict__ rs,
                                                ExpandSmem<BLOCK, VT, EXTRA> &sm, Load load, Op op,
                                                Post post, VGrid vg = hw_grid()) {
    using S = ExpandSmem<BLOCK, VT, EXTRA>;
    constexpr int WT = S::WT;
    constexpr int NWARP = S::NWARP;
    constexpr int BATCH = S::BATCH;
    const int G = vg.n;
    const int C = (nf + G - 1) / G;
    const long long total = static_cast<long long>(nf) + E;
    const long long ntiles = (total + WT - 1) / WT;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    typename S::Warp &ws = sm.w[wid];
    // one warp tile: stage its entries, label its edge slots, run the operation
    auto run_tile = [&](long long tile, long long tb) {
        const long long d0 = tile * WT;
        const long long d1 = d0 + WT < total ? d0 + WT : total;
        const int a0 = sm.tsplit[tile - tb];
        const int a1 = sm.tsplit[tile - tb + 1];
        const int e0 = static_cast<int>(d0 - a0);
        const int e1 = static_cast<int>(d1 - a1);
        const int jb = a0 > 0 ? a0 - 1 : 0;
        const int ne = a1 - jb;
        for (int k = lane; k < ne; k += 32) {
            const int j = jb + k;
            ws.off[k] = sm.base[j / C] + __ldcg(loc_off + j);
            ws.rs[k] = __ldcg(rs + j);
            load(j, k, ws);
        }
        __syncwarp();
        const int tcount = static_cast<int>(d1 - d0);
        const int diag = lane * VT;
        if (diag < tcount) {
            const int acount = a1 - a0, bcount = e1 - e0;
            int lo = diag - bcount > 0 ? diag - bcount : 0;
            int hi = diag < acount ? diag : acount;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (ws.off[a0 + mid - jb] <= e0 + diag - 1 - mid)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            int ja = a0 + lo, eb = e0 + diag - lo;
            int cur = ja - 1 - jb;
            const int end = diag + VT < tcount ? diag + VT : tcount;
            for (int it = diag; it < end; ++it) {
                if (ja < a1 && ws.off[ja - jb] <= eb) {
                    cur = ja - jb;
                    ++ja;
                } else {
                    ws.seg[eb - e0] = cur;
                    ++eb;
                }
            }
        }
        __syncwarp();
        const int ned = e1 - e0;
        bool valid[VT];
        int kk[VT], idx[VT];
#pragma unroll
        for (int r = 0; r < VT; ++r) {
            const int el = r * 32 + lane;
            valid[r] = el < ned;
            kk[r] = 0;
            idx[r] = 0;
            if (valid[r]) {
                kk[r] = ws.seg[el];
                idx[r] = ws.rs[kk[r]] + (e0 + el - ws.off[kk[r]]);
            }
        }
        op(valid, kk, idx, ws);
        __syncwarp();
        post(ne, ws);
    };
    // the tiles [tb, te) of one batch: split points found together, then the warps
    auto run_batch = [&](long long tb, long long te) {
        for (int s = threadIdx.x; s <= te - tb; s += BLOCK) {
            long long d = (tb + s) * WT;
            if (d > total) d = total;
            sm.tsplit[s] = frontier_merge_path(d, nf, E, loc_off, sm.base, C);
        }
        if (threadIdx.x == 0) sm.next_tile = NWARP;
        __syncthreads();
        // a warp that finishes its tile takes the next unclaimed one, so tiles of uneven
        // cost (atomics, queue flushes) do not leave warps idle at the batch's barrier
        for (long long tile = tb + wid; tile < te;) {
            run_tile(tile, tb);
            if (DYN) {
                int nt = 0;
                if (lane == 0) nt = atomicAdd(&sm.next_tile, 1);
                tile = tb + __shfl_sync(0xffffffffu, nt, 0);
            } else {
                tile += NWARP;
            }
            __syncwarp();
        }
        __syncthreads();
    };
    const long long per = (ntiles + G - 1) / G;
    const long long t_begin = static_cast<long long>(vg.id) * per;
    const long long t_end = t_begin + per < ntiles ? t_begin + per : ntiles;
    for (long long tb = t_begin; tb < t_end; tb += BATCH) run_batch(tb, tb + BATCH < t_end ? tb + BATCH : t_end);
}

}  // namespace apspie
