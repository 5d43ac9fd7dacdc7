// Batched multi-source SSSP: many sources on one resident graph in ONE persistent launch.
//
// By default apspie_sssp_batch runs the query groups of traverse.cu (each group of blocks
// runs the banded single-source SSSP on its share of the sources). The multi-query kernel
// below (apspie_ctx_set_sssp_batch_groups(ctx, -1)) reads each frontier row once for
// all of its queries instead, but relaxes in Bellman-Ford order.
//
// Frontier entries are (vertex u, query word w) pairs whose "changed" bits (the queries
// whose distance at u dropped in the previous iteration) are non-zero; an entry's weight
// is deg(u), so the merge-path expander balances the edges, and every lane relaxes its
// edge (u, v) for each changed query of the word: nd = dist[q][u] + w(u,v), atomicMin into
// dist[q][v], and the first bit set in v's next word enqueues the entry (v, w). Every
// query is the same label-correcting fixed point as apspie_sssp computes alone (exact
// shortest distances for non-negative integer weights), but the column indices and weights
// of a frontier row are read once for all of its changed queries, and all queries share
// the iterations' barriers.
//
// Distances are kept as unsigned values in the query-major output out[q * m + v]
// initialised to 0xFFFFFFFF, which is -1 as int32: unreached vertices need no final pass.
// Each launch serves at most 32 * W queries with (nnz + m) * W < 2^31 (int32 item counts).
#include <algorithm>
#include <cstring>

#include "frontier.cuh"

namespace apspie {
namespace {

constexpr int kSbBlock = 256;
constexpr int kSbVT = 4;
using SbSmem = ExpandSmem<kSbBlock, kSbVT>;
using SbWarp = SbSmem::Warp;
using SbWQ = WarpQueue<SbSmem::QCAP>;

enum : int { kSiteSb = 500, kSiteSbNeg = 501, kSiteSbOverflow = 502, kSiteSbCap = 503 };

struct SbArgs {
    int m, nnz, nq, W;
    const int *__restrict__ row_ptr;
    const int *__restrict__ col_ind;
    const int *__restrict__ wt;
    const int *__restrict__ srcs;
    unsigned *dist;        // nq x m, pre-filled with 0xFFFFFFFF
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

__global__ void __launch_bounds__(kSbBlock) sssp_batch_kernel(SbArgs a) {
    __shared__ SbSmem sm;
    timeline_mark(a.ctl, 0);
    const int G = gridDim.x;
    const int gtid = blockIdx.x * kSbBlock + threadIdx.x;
    const int gstride = G * kSbBlock;
    const int m = a.m, W = a.W;
    const long long mw = static_cast<long long>(m) * W;
    const int wid = threadIdx.x >> 5;

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
                a.dist[static_cast<long long>(qi) * m + v] = 0u;
                e = v * W + (qi >> 5);
                fresh = atomicOr(a.chg[0] + e, 1u << (qi & 31)) == 0u;
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
        unsigned *dist = a.dist;
        TravCtl *ctl = a.ctl;
        int *sticky = a.sticky;
        frontier_expand<kSbBlock, kSbVT, true>(
            nf, E, a.loc_off, a.rs, sm,
            [&](int j, int k, SbWarp &ws) {
                const int e = __ldcg(qc + j);
                ws.aux[k] = e / W;           // vertex u
                ws.flag[k] = e - (e / W) * W;  // query word w
                ws.aux2[k] = static_cast<int>(__ldcg(cbits + j));
            },
            [&](const bool (&valid)[kSbVT], const int (&kk)[kSbVT], const int (&idx)[kSbVT], SbWarp &ws) {
                int v[kSbVT], w8[kSbVT];
#pragma unroll
                for (int r = 0; r < kSbVT; ++r) {
                    v[r] = valid[r] ? __ldg(col + idx[r]) : 0;
                    w8[r] = valid[r] ? __ldg(wt + idx[r]) : 0;
                }
#pragma unroll
                for (int r = 0; r < kSbVT; ++r) {
                    bool fresh = false;
                    int ent = 0;
                    if (valid[r]) {
                        const int u = ws.aux[kk[r]];
                        const int w = ws.flag[kk[r]];
                        unsigned bits = static_cast<unsigned>(ws.aux2[kk[r]]);
                        if (w8[r] < 0) {
                            raise_error(ctl, sticky, APSPIE_ERR_INVALID_ARG, kSiteSbNeg);
                            bits = 0u;
                        }
                        unsigned newbits = 0u;
                        while (bits) {
                            const int b = __ffs(bits) - 1;
                            bits &= bits - 1;
                            const long long qo = static_cast<long long>(w * 32 + b) * m;
                            const unsigned du = __ldcg(dist + qo + u);
                            const unsigned long long nd = static_cast<unsigned long long>(du) + w8[r];
                            if (nd >= 0x7fffffffull) {
                                raise_error(ctl, sticky, APSPIE_ERR_INVALID_ARG, kSiteSbOverflow);
                                continue;
                            }
                            const unsigned ndu = static_cast<unsigned>(nd);
                            if (ndu < dist[qo + v[r]] && ndu < atomicMin(dist + qo + v[r], ndu)) newbits |= 1u << b;
                        }
                        if (newbits) {
                            ent = v[r] * W + w;
                            fresh = atomicOr(cn + ent, newbits) == 0u;
                        }
                    }
                    wq.push(fresh, ent);
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

}  // namespace

size_t sssp_batch_scratch_need(int m, int nq) {
    const int W = ((nq < 512 ? nq : 512) + 31) / 32;
    const size_t mw = static_cast<size_t>(m) * (W > 0 ? W : 1);
    const size_t multi = Carver::need({mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, kMaxGrid * 4});
    // the default grouped form: up to 4 groups
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
    if (ctx->sssp_batch_groups >= 0) return sssp_batch_grouped(ctx, A, d_sources, num_sources, d_dists, stats);
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
        const size_t mi = static_cast<size_t>(m) + 1;
        const size_t mw = static_cast<size_t>(m) * W;
        void *base;
        st = scratch_reserve(ctx, Carver::need({mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, mw * 4, kMaxGrid * 4}),
                             &base);
        if (st != APSPIE_OK) return st;
        Carver c(base);
        SbArgs a;
        a.chg[0] = c.take<unsigned>(mw);
        a.chg[1] = c.take<unsigned>(mw);
        a.cbits = c.take<unsigned>(mw);
        a.q[0] = c.take<int>(mw);
        a.q[1] = c.take<int>(mw);
        a.rs = c.take<int>(mw);
        a.loc_off = c.take<int>(mw);
        a.chunk_sum = c.take<int>(kMaxGrid);
        (void)mi;
        a.m = m;
        a.nnz = A->nnz;
        a.nq = nq;
        a.W = W;
        a.row_ptr = A->row_ptr;
        a.col_ind = A->col_ind;
        a.wt = static_cast<const int *>(A->val);
        a.srcs = d_sources + q0;
        a.dist = reinterpret_cast<unsigned *>(d_dists + static_cast<size_t>(q0) * m);
        a.ctl = ctx->d_ctl;
        a.sticky = ctx->d_sticky_err;
        cudaError_t e = cudaMemsetAsync(a.dist, 0xff, static_cast<size_t>(nq) * m * sizeof(int32_t), ctx->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_ctl, 0, sizeof(TravCtl), ctx->stream);
        if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_sssp_batch reset");
        void *args[] = {&a};
        st = launch_persistent(ctx, reinterpret_cast<const void *>(sssp_batch_kernel), kSbBlock, args, 1LL << 40);
        if (st != APSPIE_OK) return st;
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
