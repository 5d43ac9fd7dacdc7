// Batched multi-source SSSP: many sources on one resident graph in ONE persistent launch.
//
// By default apspie_sssp_batch runs the multi-query kernel below: it reads each frontier
// row once for all of its changed queries and relaxes in label-correcting (Bellman-Ford)
// order. apspie_ctx_set_sssp_batch_groups(ctx, g > 0) runs the query groups of traverse.cu
// instead (g groups of blocks, each running the banded single-source SSSP on its share of
// the sources).
//
// Labels are vertex-major: the distances of one vertex for the 32 queries of word w sit in
// one 128-byte line, lab[(v * W + w) * 32 + q % 32]. Frontier entries are (vertex u, query
// word w) pairs whose "changed" bits (the queries whose distance at u dropped in the
// previous iteration) are non-zero; an entry's weight is deg(u), so the merge-path
// expander balances the edges. Each warp then walks its lanes' edges one at a time with
// the lanes standing for the word's 32 queries: lane q reads u's and v's labels of query q
// (two coalesced line reads shared by the whole word), relaxes nd = dist[q][u] + w(u,v) if
// q changed at u, and atomicMin's the label; a ballot collects the improved queries and the
// edge's own lane ORs them into v's next changed word, enqueueing (v, w) on the first bit.
// Every query reaches the same label-correcting fixed point as apspie_sssp computes alone
// (exact shortest distances for non-negative integer weights). A last pass transposes the
// labels into the query-major output out[q * m + v] (0xFFFFFFFF, -1 as int32, unreached).
// Each launch serves at most 32 * W queries with (nnz + m) * W < 2^31 (int32 item counts).
#include <algorithm>
#include <cstring>

#include "frontier.cuh"

namespace apspie {
namespace {

#ifndef APSPIE_SB_MINB
#define APSPIE_SB_MINB 5
#endif
#ifndef APSPIE_SB_UNROLL
#define APSPIE_SB_UNROLL 4
#endif
#ifndef APSPIE_SB_VT
#define APSPIE_SB_VT 2
#endif
constexpr int kSbBlock = 256;
constexpr int kSbVT = APSPIE_SB_VT;
constexpr int kSbUnroll = APSPIE_SB_UNROLL;  // edges whose label reads a warp issues together
// every lane's edge is visited exactly once per pass: a second visit would not record the
// queries it improves
static_assert(32 % kSbUnroll == 0, "the unroll must divide the warp");
using SbSmem = ExpandSmem<kSbBlock, kSbVT>;
using SbWarp = SbSmem::Warp;
using SbWQ = WarpQueue<SbSmem::QCAP>;

enum : int { kSiteSb = 500, kSiteSbNeg = 501, kSiteSbOverflow = 502, kSiteSbCap = 503, kSiteSbBadSource = 504 };

struct SbArgs {
    int m, nnz, nq, W;
    const int *__restrict__ row_ptr;
    const int *__restrict__ col_ind;
    const int *__restrict__ wt;
    const int *__restrict__ srcs;
    unsigned *lab;         // m x W x 32 labels, vertex-major, pre-filled with 0xFFFFFFFF
    unsigned *chg[2];      // m x W changed-query words (ping-pong)
    unsigned *cbits;       // per frontier entry: its changed word (copied in phase A)
    int *q[2];             // frontier entries u * W + w
    int *rs, *loc_off, *chunk_sum;
    TravCtl *ctl;
    int *sticky;
};

struct RowOfPacked {
    int W;
    __device__ __forceinline__ int operator()(int e) const { return e / W; }
};

__global__ void __launch_bounds__(kSbBlock, APSPIE_SB_MINB) sssp_batch_kernel(SbArgs a) {
    __shared__ SbSmem sm;
    timeline_mark(a.ctl, 0);
    const int G = gridDim.x;
    const int gtid = blockIdx.x * kSbBlock + threadIdx.x;
    const int gstride = G * kSbBlock;
    const int m = a.m, W = a.W;
    const long long mw = static_cast<long long>(m) * W;
    const int wid = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    for (long long i = gtid; i < mw; i += gstride) {
        a.chg[0][i] = 0u;
        a.chg[1][i] = 0u;
    }
    if (gtid == 0) a.ctl->qlen[0] = a.ctl->qlen[1] = 0;
    if (!grid_barrier(a.ctl, a.sticky, kSiteSb)) return;
    {
        SbWQ wq(sm.qbuf[wid][0], a.q[0], &a.ctl->qlen[0]);
        for (int base = blockIdx.x * kSbBlock; base < a.nq; base += gstride) {
            const int qi = base + threadIdx.x;
            bool fresh = false;
            int e = 0;
            if (qi < a.nq) {
                const int v = a.srcs[qi];
                if (v < 0 || v >= m) {  // reported; the barrier below then ends the launch
                    raise_error(a.ctl, a.sticky, APSPIE_ERR_INVALID_ARG, kSiteSbBadSource);
                } else {
                    e = v * W + (qi >> 5);
                    a.lab[static_cast<size_t>(e) * 32 + (qi & 31)] = 0u;
                    fresh = atomicOr(a.chg[0] + e, 1u << (qi & 31)) == 0u;
                }
            }
            wq.push(fresh, e);
        }
        wq.flush();
    }
    if (!grid_barrier(a.ctl, a.sticky, kSiteSb + 10)) return;

    int cur = 0, iters = 0;
    long long relaxed = 0;
    for (;;) {
        const int nf = ld_volatile_i32(&a.ctl->qlen[cur]);
        if (nf == 0) break;
        if (iters > m + 1) {
            if (gtid == 0) raise_error(a.ctl, a.sticky, APSPIE_ERR_NOT_CONVERGED, kSiteSbCap);
            break;
        }
        ++iters;
        int *qc = a.q[cur];
        int *qn = a.q[cur ^ 1];
        unsigned *cc = a.chg[cur];
        unsigned *cn = a.chg[cur ^ 1];
        unsigned *cbits = a.cbits;
        // phase A: take each entry's changed word (and clear it for reuse), row degrees
        frontier_phase_a<kSbBlock>(qc, nf, a.row_ptr, a.rs, a.loc_off, a.chunk_sum, sm.scan_tmp,
                                   [&](int i, int e, int deg) {
                                       const unsigned b = __ldcg(cc + e);
                                       cbits[i] = b;
                                       cc[e] = 0u;
                                       return b ? deg : 0;
                                   },
                                   RowOfPacked{W});
        if (gtid == 0) a.ctl->qlen[cur ^ 1] = 0;
        if (!grid_barrier(a.ctl, a.sticky, kSiteSb + 1)) return;
        const int E = frontier_chunk_bases<kSbBlock>(a.chunk_sum, sm.base, sm.scan_tmp);
        relaxed += E;
        SbWQ wq(sm.qbuf[wid][0], qn, &a.ctl->qlen[cur ^ 1]);
        const int *col = a.col_ind;
        const int *wt = a.wt;
        unsigned *lab = a.lab;
        TravCtl *ctl = a.ctl;
        int *sticky = a.sticky;
        frontier_expand<kSbBlock, kSbVT, true>(
            nf, E, a.loc_off, a.rs, sm,
            [&](int j, int k, SbWarp &ws) {
                const int e = __ldcg(qc + j);
                ws.aux[k] = e;                  // entry u * W + w
                ws.flag[k] = e - (e / W) * W;   // query word w
                ws.aux2[k] = static_cast<int>(__ldcg(cbits + j));
            },
            [&](const bool (&valid)[kSbVT], const int (&kk)[kSbVT], const int (&idx)[kSbVT], SbWarp &ws) {
                // this lane's edges: target entry (v, w), weight, source entry and its changed bits
                int tv[kSbVT], we[kSbVT], eu[kSbVT];
                unsigned bits[kSbVT];
#pragma unroll
                for (int r = 0; r < kSbVT; ++r) {
                    tv[r] = eu[r] = 0;
                    we[r] = 0;
                    bits[r] = 0u;
                    if (valid[r]) {
                        const int v = __ldg(col + idx[r]);
                        we[r] = __ldg(wt + idx[r]);
                        eu[r] = ws.aux[kk[r]];
                        tv[r] = v * W + ws.flag[kk[r]];
                        bits[r] = static_cast<unsigned>(ws.aux2[kk[r]]);
                        if (we[r] < 0) {  // reported once here; the edge is then left out
                            raise_error(ctl, sticky, APSPIE_ERR_INVALID_ARG, kSiteSbNeg);
                            bits[r] = 0u;
                        }
                    }
                }
                unsigned *lab_l = lab + lane;  // this lane's query in every label line
#pragma unroll
                for (int r = 0; r < kSbVT; ++r) {
                    const unsigned vmask = __ballot_sync(0xffffffffu, bits[r] != 0u);
                    if (vmask == 0u) continue;
                    unsigned mine = 0u;  // improved queries of this lane's edge r
#pragma unroll 1
                    for (int l0 = 0; l0 < 32; l0 += kSbUnroll) {
                        if (((vmask >> l0) & ((1u << kSbUnroll) - 1u)) == 0u) continue;
                        unsigned du[kSbUnroll], dv[kSbUnroll];
                        int ev[kSbUnroll], wl[kSbUnroll];
                        bool act[kSbUnroll];
#pragma unroll
                        for (int t = 0; t < kSbUnroll; ++t) {
                            const int l = l0 + t;
                            ev[t] = __shfl_sync(0xffffffffu, tv[r], l);
                            wl[t] = __shfl_sync(0xffffffffu, we[r], l);
                            const int u = __shfl_sync(0xffffffffu, eu[r], l);
                            const unsigned b = __shfl_sync(0xffffffffu, bits[r], l);
                            act[t] = (b >> lane) & 1u;
                            // coherent reads: a label lowered since the entry was queued must be
                            // seen (its change bit was consumed in phase A)
                            du[t] = act[t] ? __ldcg(lab_l + static_cast<size_t>(u) * 32) : 0u;
                            dv[t] = act[t] ? __ldcg(lab_l + static_cast<size_t>(ev[t]) * 32) : 0u;
                        }
                        // an improvement over the label just read is reported without waiting
                        // for the atomic's old value: if another edge lowered the label further
                        // meanwhile, v's query is only re-expanded once more (same values)
                        bool imp[kSbUnroll];
#pragma unroll
                        for (int t = 0; t < kSbUnroll; ++t) {
                            imp[t] = false;
                            // an active label is finite (< 2^31 - 1) and the weight is
                            // non-negative, so the 32-bit sum cannot wrap
                            const unsigned nd = du[t] + static_cast<unsigned>(wl[t]);
                            if (act[t]) {
                                if (nd >= 0x7fffffffu) {
                                    raise_error(ctl, sticky, APSPIE_ERR_INVALID_ARG, kSiteSbOverflow);
                                } else if (nd < dv[t]) {
                                    atomicMin(lab_l + static_cast<size_t>(ev[t]) * 32, nd);
                                    imp[t] = true;
                                }
                            }
                        }
#pragma unroll
                        for (int t = 0; t < kSbUnroll; ++t) {
                            const unsigned nb = __ballot_sync(0xffffffffu, imp[t]);
                            if (lane == l0 + t) mine = nb;
                        }
                    }
                    bool fresh = false;
                    if (mine) fresh = atomicOr(cn + tv[r], mine) == 0u;
                    wq.push(fresh, tv[r]);
                }
            },
            [](int, SbWarp &) {});
        wq.flush();
        if (!grid_barrier(a.ctl, a.sticky, kSiteSb + 2)) return;
        cur ^= 1;
    }
    if (gtid == 0) {
        a.ctl->iterations = iters;
        a.ctl->push_iterations = iters;
        a.ctl->edges_expanded = relaxed;
    }
}

// Labels (vertex-major, 32 queries per line) -> query-major rows out[q * m + v], one
// 32-vertex x 32-query tile at a time through shared memory (both sides coalesced).
__global__ void __launch_bounds__(256) sb_unpack(const unsigned *__restrict__ lab, int m, int W, int nq,
                                                 unsigned *out) {
    __shared__ unsigned t[32][33];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long long ntiles = static_cast<long long>((m + 31) / 32) * W;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int vb = static_cast<int>(tile / W) * 32;
        const int w = static_cast<int>(tile % W);
        for (int i = wid; i < 32; i += 8) {
            const int v = vb + i;
            t[i][lane] = v < m ? __ldcs(lab + (static_cast<size_t>(v) * W + w) * 32 + lane) : 0u;
        }
        __syncthreads();
        for (int i = wid; i < 32; i += 8) {
            const int q = w * 32 + i;
            if (q < nq && vb + lane < m) out[static_cast<size_t>(q) * m + vb + lane] = t[lane][i];
        }
        __syncthreads();
    }
}

}  // namespace

size_t sssp_batch_scratch_need(int m, int nq) {
    const int W = ((nq < 512 ? nq : 512) + 31) / 32;
    const size_t mw = static_cast<size_t>(m) * (W > 0 ? W : 1);
    const size_t multi =
        Carver::need({mw * 128, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, kMaxGrid * 4});
    // the grouped form (groups > 0): at most 4 groups are costed here
    const size_t grouped = sssp_group_scratch_need(m, std::max(1, std::min(nq, 4)));
    return std::max(multi, grouped);
}

}  // namespace apspie

using namespace apspie;

extern "C" apspie_status apspie_sssp_batch(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources,
                                           int32_t num_sources, int32_t *d_dists, apspie_run_stats *stats) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_csr_view(ctx, A, "apspie_sssp_batch");
    if (st != APSPIE_OK) return st;
    if (A->m != A->n || A->m <= 0)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp_batch: square, non-empty graph required");
    if (A->val_type != APSPIE_VAL_I32 || (A->nnz > 0 && !A->val))
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp_batch: int32 edge weights required");
    if (num_sources < 0 || (num_sources > 0 && (!d_sources || !d_dists)))
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp_batch: bad sources/output");
    if (ctx->validate && (st = validate_csr(ctx, A, true)) != APSPIE_OK) return st;
    if (ctx->sssp_batch_groups > 0) return sssp_batch_grouped(ctx, A, d_sources, num_sources, d_dists, stats);
    const int m = A->m;
    // queries per launch: W words with (nnz + m) * W below 2^31 (int32 item counts)
    long long wmax = 0x7fffffffLL / (static_cast<long long>(A->nnz) + m + 1);
    if (wmax > 16) wmax = 16;
    if (wmax < 1) return set_error(ctx, APSPIE_ERR_UNSUPPORTED, "apspie_sssp_batch: graph too large");
    const int per_launch = static_cast<int>(32 * wmax);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    for (int q0 = 0; q0 < num_sources; q0 += per_launch) {
        const int nq = std::min(per_launch, num_sources - q0);
        const int W = (nq + 31) / 32;
        const size_t mw = static_cast<size_t>(m) * W;
        void *base;
        st = scratch_reserve(
            ctx, Carver::need({mw * 128, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, kMaxGrid * 4}),
            &base);
        if (st != APSPIE_OK) return st;
        Carver c(base);
        SbArgs a;
        a.lab = c.take<unsigned>(mw * 32);
        a.chg[0] = c.take<unsigned>(mw);
        a.chg[1] = c.take<unsigned>(mw);
        a.cbits = c.take<unsigned>(mw);
        a.q[0] = c.take<int>(mw);
        a.q[1] = c.take<int>(mw);
        a.rs = c.take<int>(mw);
        a.loc_off = c.take<int>(mw);
        a.chunk_sum = c.take<int>(kMaxGrid);
        a.m = m;
        a.nnz = A->nnz;
        a.nq = nq;
        a.W = W;
        a.row_ptr = A->row_ptr;
        a.col_ind = A->col_ind;
        a.wt = static_cast<const int *>(A->val);
        a.srcs = d_sources + q0;
        a.ctl = ctx->d_ctl;
        a.sticky = ctx->d_sticky_err;
        cudaError_t e = cudaMemsetAsync(a.lab, 0xff, mw * 32 * sizeof(unsigned), ctx->stream);
        if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_sssp_batch reset");
        if ((st = reset_ctl(ctx)) != APSPIE_OK) return st;
        void *args[] = {&a};
        st = launch_persistent(ctx, reinterpret_cast<const void *>(sssp_batch_kernel), kSbBlock, args, 1LL << 40);
        if (st != APSPIE_OK) return st;
        const long long tiles = static_cast<long long>((m + 31) / 32) * W;
        const int ublocks = static_cast<int>(std::min<long long>(tiles, ctx->num_sms * 16LL));
        sb_unpack<<<ublocks, 256, 0, ctx->stream>>>(
            a.lab, m, W, nq, reinterpret_cast<unsigned *>(d_dists + static_cast<size_t>(q0) * m));
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(ctx, e, "apspie_sssp_batch unpack");
        if (stats) {
            apspie_run_stats part;
            if ((st = finish_call(ctx, &part, "apspie_sssp_batch")) != APSPIE_OK) return st;
            stats->iterations += part.iterations;
            stats->push_iterations += part.push_iterations;
            stats->edges_expanded += part.edges_expanded;
        }
    }
    return APSPIE_OK;
}
