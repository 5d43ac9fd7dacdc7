// Batched multi-source BFS: many sources on one resident graph in ONE persistent launch.
//
// The reference has no batched path (its drivers loop one source per process run,
// test/bfs/run.sh:30-35). Here every vertex carries W = ceil(nq/32) words of query bits:
// visited bits, and the frontier bits of the current level (ping-pong buffers). A level is
// a boolean SpMSpM (A^T times an m x nq frontier block) fused with the per-query visited
// mask:
//  push (few frontier vertices): merge-path expansion of the active list; for each edge
//       (u, v) the bits fr[u] & ~visited[v] are OR-ed into next[v] (one atomicOr per
//       non-zero word) and v is put on a touched list; a finalize pass turns next[v] into
//       the exact new bits, writes their depths and builds the next active list;
//  pull (many frontier vertices): one thread per vertex ORs its neighbours' frontier
//       words restricted to its still-unvisited queries and stops as soon as every such
//       query is covered.
// Depths go straight to the query-major output out[q * m + v] (warp-coalesced in pull).
// The per-query answers are exactly those of independent BFS runs.
//
// Active lists rotate through three queues so that the frontier buffer written at level L
// is zeroed (by the list of level L-2) in the same phase that resets the list length,
// without extra barriers.
#include <algorithm>
#include <cstring>

#include "frontier.cuh"

namespace apspie {
namespace {

constexpr int kMsBlock = 256;
constexpr int kMsVT = 4;
using MsSmem = ExpandSmem<kMsBlock, kMsVT>;
using MsWarp = MsSmem::Warp;
using MsWQ = WarpQueue<MsSmem::QCAP>;

enum : int { kSiteMs = 400, kSiteMsBadSource = 450 };
constexpr int kHeavyDeg = 128;  // pull: rows longer than this are scanned by a whole block

struct MsArgs {
    int m, nnz, nq, depth_cap;
    const int *__restrict__ row_ptr;
    const int *__restrict__ col_ind;
    const int *__restrict__ srcs;
    int *out;             // nq x m, pre-filled with -1 (when rows is null)
    int *const *rows;     // else: query q's depths go to rows[q][0..m), pre-filled with -1
    unsigned *vis;        // m x W
    unsigned *fr[2];      // m x W each
    unsigned *touched;    // m bits
    int *q[3];            // active lists (rotating)
    int *tq;              // touched list
    int *heavy;           // vertices with more than kHeavyDeg neighbours (pulled by a block)
    int *rs, *loc_off, *chunk_sum;
    TravCtl *ctl;         // qlen[0..1] + aux[0] used as qlen[2], aux[1] as touched length
    int *sticky;
    float push_frac;      // push while |active| * mean degree < push_frac * nnz
};

__device__ __forceinline__ int *depth_row(const MsArgs &a, int q) {
    return a.rows ? a.rows[q] : a.out + static_cast<long long>(q) * a.m;
}

// Bits of word w that belong to real queries (0..nq-1).
__device__ __forceinline__ unsigned query_mask(int nq, int w) {
    const int nbits = nq - w * 32;
    if (nbits >= 32) return ~0u;
    if (nbits <= 0) return 0u;
    return (1u << nbits) - 1u;
}

__device__ __forceinline__ int *qlen_ptr(TravCtl *ctl, int k) {
    return k < 2 ? &ctl->qlen[k] : reinterpret_cast<int *>(&ctl->aux[0]);
}

template <int W>
__global__ void __launch_bounds__(kMsBlock, W >= 16 ? 3 : 4) msbfs_kernel(MsArgs a) {
    __shared__ MsSmem sm;
    timeline_mark(a.ctl, 0);
    const int G = gridDim.x;
    const int gtid = blockIdx.x * kMsBlock + threadIdx.x;
    const int gstride = G * kMsBlock;
    const int m = a.m;
    const long long mw = static_cast<long long>(m) * W;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    int *tqlen = reinterpret_cast<int *>(&a.ctl->aux[1]);

    for (long long i = gtid; i < mw; i += gstride) {
        a.vis[i] = 0u;
        a.fr[0][i] = 0u;
        a.fr[1][i] = 0u;
    }
    for (int w = gtid; w < (m + 31) / 32; w += gstride) a.touched[w] = 0u;
    int *hlen = reinterpret_cast<int *>(&a.ctl->aux[2]);
    {
        MsWQ hq(sm.qbuf[wid][0], a.heavy, hlen);
        for (int base = blockIdx.x * kMsBlock; base < m; base += gstride) {
            const int v = base + threadIdx.x;
            const bool h = v < m && (__ldg(a.row_ptr + v + 1) - __ldg(a.row_ptr + v)) > kHeavyDeg;
            hq.push(h, v);
        }
        hq.flush();
    }
    if (gtid == 0) {
        a.ctl->qlen[0] = a.ctl->qlen[1] = 0;
        *qlen_ptr(a.ctl, 2) = 0;
        *tqlen = 0;
    }
    if (!grid_barrier(a.ctl, a.sticky, kSiteMs)) return;
    const int nheavy = ld_volatile_i32(hlen);
    // level 0: the sources
    {
        MsWQ wq(sm.qbuf[wid][0], a.q[0], qlen_ptr(a.ctl, 0));
        for (int base = blockIdx.x * kMsBlock; base < a.nq; base += gstride) {
            const int qi = base + threadIdx.x;
            bool first = false;
            int v = 0;
            if (qi < a.nq) {
                v = a.srcs[qi];
                if (v < 0 || v >= a.m) {  // reported; the barrier below then ends the launch
                    raise_error(a.ctl, a.sticky, APSPIE_ERR_INVALID_ARG, kSiteMsBadSource);
                    v = 0;
                } else {
                    const unsigned bit = 1u << (qi & 31);
                    atomicOr(a.vis + static_cast<long long>(v) * W + (qi >> 5), bit);
                    atomicOr(a.fr[0] + static_cast<long long>(v) * W + (qi >> 5), bit);
                    depth_row(a, qi)[v] = 0;
                    const unsigned tb = 1u << (v & 31);
                    first = !(atomicOr(a.touched + (v >> 5), tb) & tb);
                }
            }
            wq.push(first, v);
        }
        wq.flush();
    }
    if (!grid_barrier(a.ctl, a.sticky, kSiteMs + 1)) return;
    {
        const int n0 = ld_volatile_i32(qlen_ptr(a.ctl, 0));
        for (int i = gtid; i < n0; i += gstride) {
            const int v = __ldcg(a.q[0] + i);
            atomicAnd(a.touched + (v >> 5), ~(1u << (v & 31)));
        }
    }
    if (!grid_barrier(a.ctl, a.sticky, kSiteMs + 2)) return;

    const double mean_deg = m ? static_cast<double>(a.nnz) / m : 0.0;
    int prev_n = 0;  // length of the level L-1 list (all blocks read it at that level)
    int levels = 0, npush = 0, npull = 0;
    for (int L = 0;; ++L) {
        const int cur = L % 3, nxt = (L + 1) % 3, prv = (L + 2) % 3;
        const int nA = ld_volatile_i32(qlen_ptr(a.ctl, cur));
        if (nA == 0) break;
        if (a.depth_cap > 0 && L + 1 >= a.depth_cap) break;
        ++levels;
        const unsigned *frc = a.fr[L & 1];
        unsigned *frn = a.fr[(L + 1) & 1];
        // zero the level L-1 frontier words (buffer frn) and reset the next list
        if (L > 0) {
            const int *qp = a.q[prv];
            for (long long x = gtid; x < static_cast<long long>(prev_n) * W; x += gstride) {
                const int v = __ldcg(qp + x / W);
                frn[static_cast<long long>(v) * W + x % W] = 0u;
            }
        }
        const bool push = static_cast<double>(nA) * mean_deg < a.push_frac * a.nnz;
        int E = 0;
        if (push) {
            frontier_phase_a<kMsBlock>(a.q[cur], nA, a.row_ptr, a.rs, a.loc_off, a.chunk_sum, sm.scan_tmp,
                                       [](int, int, int deg) { return deg; });
        }
        if (gtid == 0) {
            *qlen_ptr(a.ctl, nxt) = 0;
            *tqlen = 0;
        }
        if (!grid_barrier(a.ctl, a.sticky, kSiteMs + 3)) return;
        if (push) {
            ++npush;
            E = frontier_chunk_bases<kMsBlock>(a.chunk_sum, sm.base, sm.scan_tmp);
            MsWQ tw(sm.qbuf[wid][0], a.tq, tqlen);
            const int *col = a.col_ind;
            const int *qc = a.q[cur];
            unsigned *vis = a.vis;
            unsigned *touched = a.touched;
            frontier_expand<kMsBlock, kMsVT, true>(
                nA, E, a.loc_off, a.rs, sm, [&](int j, int k, MsWarp &ws) { ws.aux[k] = __ldcg(qc + j); },
                [&](const bool (&valid)[kMsVT], const int (&kk)[kMsVT], const int (&idx)[kMsVT], MsWarp &ws) {
                    int v[kMsVT];
#pragma unroll
                    for (int r = 0; r < kMsVT; ++r) v[r] = valid[r] ? __ldg(col + idx[r]) : 0;
#pragma unroll
                    for (int r = 0; r < kMsVT; ++r) {
                        bool add = false;
                        if (valid[r]) {
                            const int u = ws.aux[kk[r]];
                            const unsigned *fu = frc + static_cast<long long>(u) * W;
                            const unsigned *vv = vis + static_cast<long long>(v[r]) * W;
                            unsigned *nv = frn + static_cast<long long>(v[r]) * W;
#pragma unroll
                            for (int w = 0; w < W; ++w) {
                                const unsigned bits = __ldcg(fu + w) & ~__ldcg(vv + w);
                                if (bits) {
                                    atomicOr(nv + w, bits);
                                    add = true;
                                }
                            }
                            if (add) {
                                const unsigned tb = 1u << (v[r] & 31);
                                add = !(atomicOr(touched + (v[r] >> 5), tb) & tb);
                            }
                        }
                        tw.push(add, v[r]);
                    }
                },
                [](int, MsWarp &) {});
            tw.flush();
            if (!grid_barrier(a.ctl, a.sticky, kSiteMs + 4)) return;
            // finalize the touched vertices
            const int nt = ld_volatile_i32(tqlen);
            MsWQ aw(sm.qbuf[wid][1], a.q[nxt], qlen_ptr(a.ctl, nxt));
            for (int base = blockIdx.x * kMsBlock; base < nt; base += gstride) {
                const int i = base + threadIdx.x;
                bool any = false;
                int v = 0;
                if (i < nt) {
                    v = __ldcg(a.tq + i);
                    atomicAnd(touched + (v >> 5), ~(1u << (v & 31)));
                    unsigned *nv = frn + static_cast<long long>(v) * W;
                    unsigned *vv = vis + static_cast<long long>(v) * W;
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        const unsigned nb = __ldcg(nv + w) & ~__ldcg(vv + w);
                        nv[w] = nb;
                        if (nb) {
                            vv[w] |= nb;
                            any = true;
                            unsigned b = nb;
                            while (b) {
                                const int bit = __ffs(b) - 1;
                                b &= b - 1;
                                depth_row(a, w * 32 + bit)[v] = L + 1;
                            }
                        }
                    }
                }
                aw.push(any, v);
            }
            aw.flush();
        } else {
            ++npull;
            MsWQ aw(sm.qbuf[wid][1], a.q[nxt], qlen_ptr(a.ctl, nxt));
            const unsigned lanemask_all = 0xffffffffu;
            for (int base = blockIdx.x * kMsBlock; base < m; base += gstride) {
                const int v = base + threadIdx.x;
                unsigned need[W], got[W];
                bool todo = false;
                if (v < m) {
                    const unsigned *vv = a.vis + static_cast<long long>(v) * W;
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        need[w] = ~__ldcg(vv + w) & query_mask(a.nq, w);
                        got[w] = 0u;
                        todo |= need[w] != 0u;
                    }
                } else {
#pragma unroll
                    for (int w = 0; w < W; ++w) need[w] = got[w] = 0u;
                }
                int r0 = 0, r1 = 0;
                if (todo) {
                    r0 = __ldg(a.row_ptr + v);
                    r1 = __ldg(a.row_ptr + v + 1);
                    if (r1 - r0 > kHeavyDeg) todo = false;  // handled by a block below
                }
                if (todo) {
                    // four neighbours per step: all their frontier words are loaded before the
                    // coverage test, so a thread keeps several loads in flight
                    constexpr int U = W >= 8 ? 2 : 4;
                    for (int e0 = r0; e0 < r1; e0 += U) {
                        int u[U];
#pragma unroll
                        for (int k = 0; k < U; ++k) u[k] = e0 + k < r1 ? __ldg(a.col_ind + e0 + k) : -1;
                        unsigned f[U][W];
#pragma unroll
                        for (int k = 0; k < U; ++k)
#pragma unroll
                            for (int w = 0; w < W; ++w)
                                f[k][w] = u[k] >= 0 ? __ldcg(frc + static_cast<long long>(u[k]) * W + w) : 0u;
                        bool done = true;
#pragma unroll
                        for (int w = 0; w < W; ++w) {
#pragma unroll
                            for (int k = 0; k < U; ++k) got[w] |= f[k][w] & need[w];
                            done &= got[w] == need[w];
                        }
                        if (done) break;
                    }
                }
                bool any = false;
                if (v < m) {
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        if (got[w]) {
                            any = true;
                            a.fr[(L + 1) & 1][static_cast<long long>(v) * W + w] = got[w];
                            a.vis[static_cast<long long>(v) * W + w] |= got[w];
                        }
                    }
                }
                // depths: one coalesced store per query that any lane of the warp found
#pragma unroll
                for (int w = 0; w < W; ++w) {
                    unsigned anyb = __reduce_or_sync(lanemask_all, got[w]);
                    while (anyb) {
                        const int bit = __ffs(anyb) - 1;
                        anyb &= anyb - 1;
                        if ((got[w] >> bit) & 1u) depth_row(a, w * 32 + bit)[v] = L + 1;
                    }
                }
                aw.push(any, v);
            }
            aw.flush();
            // heavy rows: one block per row, OR-reducing 256 neighbours per step and stopping
            // as soon as every still-unvisited query of the row is covered
            __shared__ unsigned s_need[W], s_acc[W];
            __shared__ int s_done;
            for (int h = blockIdx.x; h < nheavy; h += G) {
                const int v = __ldcg(a.heavy + h);
                unsigned *vv = a.vis + static_cast<long long>(v) * W;
                if (threadIdx.x < W) {
                    s_need[threadIdx.x] = ~__ldcg(vv + threadIdx.x) & query_mask(a.nq, threadIdx.x);
                    s_acc[threadIdx.x] = 0u;
                }
                __syncthreads();
                bool need_any = false;
#pragma unroll
                for (int w = 0; w < W; ++w) need_any |= s_need[w] != 0u;
                if (need_any) {
                    const int r0 = __ldg(a.row_ptr + v), r1 = __ldg(a.row_ptr + v + 1);
                    for (int e0 = r0; e0 < r1; e0 += kMsBlock) {
                        const int e = e0 + threadIdx.x;
                        unsigned bits[W];
                        if (e < r1) {
                            const unsigned *fu = frc + static_cast<long long>(__ldg(a.col_ind + e)) * W;
#pragma unroll
                            for (int w = 0; w < W; ++w) bits[w] = __ldcg(fu + w) & s_need[w];
                        } else {
#pragma unroll
                            for (int w = 0; w < W; ++w) bits[w] = 0u;
                        }
#pragma unroll
                        for (int w = 0; w < W; ++w) {
                            const unsigned r = __reduce_or_sync(0xffffffffu, bits[w]);
                            if (lane == 0 && r) atomicOr(&s_acc[w], r);
                        }
                        __syncthreads();
                        if (threadIdx.x == 0) {
                            int done = 1;
#pragma unroll
                            for (int w = 0; w < W; ++w) done &= s_acc[w] == s_need[w];
                            s_done = done;
                        }
                        __syncthreads();
                        if (s_done) break;
                    }
                    if (threadIdx.x < W) {
                        const unsigned got = s_acc[threadIdx.x];
                        if (got) {
                            a.fr[(L + 1) & 1][static_cast<long long>(v) * W + threadIdx.x] = got;
                            vv[threadIdx.x] |= got;
                            unsigned b = got;
                            while (b) {
                                const int bit = __ffs(b) - 1;
                                b &= b - 1;
                                depth_row(a, threadIdx.x * 32 + bit)[v] = L + 1;
                            }
                        }
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) {
                        bool any = false;
#pragma unroll
                        for (int w = 0; w < W; ++w) any |= s_acc[w] != 0u;
                        if (any) a.q[nxt][atomicAdd(qlen_ptr(a.ctl, nxt), 1)] = v;
                    }
                }
                __syncthreads();
            }
        }
        if (!grid_barrier(a.ctl, a.sticky, kSiteMs + 5)) return;
        prev_n = nA;
    }
    if (gtid == 0) {
        a.ctl->iterations = levels;
        a.ctl->push_iterations = npush;
        a.ctl->pull_iterations = npull;
    }
}

template <int W>
const void *msbfs_fn() {
    return reinterpret_cast<const void *>(msbfs_kernel<W>);
}

size_t batch_need(int m, int Wp) {
    const size_t mi = static_cast<size_t>(m) + 1;
    const size_t mw = static_cast<size_t>(m) * Wp;
    const size_t words = (static_cast<size_t>(m) + 31) / 32;
    return Carver::need({mw * 4, mw * 4, mw * 4, words * 4, mi * 4, mi * 4, mi * 4, mi * 4, mi * 4, mi * 4, mi * 4,
                         kMaxGrid * 4});
}

int padded_words(int nq) {
    const int W = (nq + 31) / 32;
    return W <= 1 ? 1 : W <= 2 ? 2 : W <= 4 ? 4 : W <= 8 ? 8 : 16;
}

}  // namespace

size_t bfs_batch_scratch_need(int m, int nq) { return batch_need(m, padded_words(nq < 512 ? nq : 512)); }

}  // namespace apspie

using namespace apspie;

namespace apspie {

// The batched BFS with either a query-major output (d_depths) or, when h_rows is given, one
// output row per query (h_rows[q], device pointers): the server writes each answer straight
// into its request's buffer this way.
apspie_status bfs_batch_impl(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources, int32_t num_sources,
                             int32_t depth_cap, int32_t *d_depths, int32_t *const *h_rows, apspie_run_stats *stats) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_csr_view(ctx, A, "apspie_bfs_batch");
    if (st != APSPIE_OK) return st;
    if (A->m != A->n || A->m <= 0)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_bfs_batch: square, non-empty graph required");
    if (num_sources < 0 || (num_sources > 0 && (!d_sources || (!d_depths && !h_rows))))
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_bfs_batch: bad sources/output");
    if (ctx->validate && (st = validate_csr(ctx, A, true)) != APSPIE_OK) return st;
    const int m = A->m;
    constexpr int kMaxQ = 512;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    for (int q0 = 0; q0 < num_sources; q0 += kMaxQ) {
        const int nq = std::min(kMaxQ, num_sources - q0);
        const int Wp = padded_words(nq);
        const size_t mi = static_cast<size_t>(m) + 1;
        const size_t mw = static_cast<size_t>(m) * Wp;
        const size_t words = (static_cast<size_t>(m) + 31) / 32;
        void *base;
        st = scratch_reserve(ctx, batch_need(m, Wp) + (h_rows ? Carver::need({kMaxQ * sizeof(int *)}) : 0), &base);
        if (st != APSPIE_OK) return st;
        Carver c(base);
        MsArgs a;
        a.rows = nullptr;
        a.vis = c.take<unsigned>(mw);
        a.fr[0] = c.take<unsigned>(mw);
        a.fr[1] = c.take<unsigned>(mw);
        a.touched = c.take<unsigned>(words);
        a.q[0] = c.take<int>(mi);
        a.q[1] = c.take<int>(mi);
        a.q[2] = c.take<int>(mi);
        a.tq = c.take<int>(mi);
        a.heavy = c.take<int>(mi);
        a.rs = c.take<int>(mi);
        a.loc_off = c.take<int>(mi);
        a.chunk_sum = c.take<int>(kMaxGrid);
        a.m = m;
        a.nnz = A->nnz;
        a.nq = nq;
        a.depth_cap = depth_cap;
        a.row_ptr = A->row_ptr;
        a.col_ind = A->col_ind;
        a.srcs = d_sources + q0;
        a.out = d_depths ? d_depths + static_cast<size_t>(q0) * m : nullptr;
        a.ctl = ctx->d_ctl;
        a.sticky = ctx->d_sticky_err;
        // pull levels scan a vertex's own row for parents: valid for symmetric patterns only
        a.push_frac = (A->flags & APSPIE_CSR_SYMMETRIC)
                          ? effective_params(ctx, APSPIE_TUNE_BFS_BATCH, A).batch_push_frac
                          : 1e30f;
        cudaError_t e = cudaSuccess;
        if (h_rows) {
            int32_t **table = c.take<int32_t *>(kMaxQ);
            // pageable source: the copy is staged before the call returns
            e = cudaMemcpyAsync(table, h_rows + q0, static_cast<size_t>(nq) * sizeof(int32_t *),
                                cudaMemcpyHostToDevice, ctx->stream);
            for (int q = 0; q < nq && e == cudaSuccess; ++q)
                e = cudaMemsetAsync(h_rows[q0 + q], 0xff, static_cast<size_t>(m) * sizeof(int32_t), ctx->stream);
            a.rows = table;
        } else {
            e = cudaMemsetAsync(a.out, 0xff, static_cast<size_t>(nq) * m * sizeof(int32_t), ctx->stream);
        }
        if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_bfs_batch reset");
        if ((st = reset_ctl(ctx)) != APSPIE_OK) return st;
        const void *fn = Wp == 1 ? msbfs_fn<1>() : Wp == 2 ? msbfs_fn<2>() : Wp == 4 ? msbfs_fn<4>()
                         : Wp == 8 ? msbfs_fn<8>() : msbfs_fn<16>();
        void *args[] = {&a};
        st = launch_persistent(ctx, fn, kMsBlock, args, 1LL << 40);
        if (st != APSPIE_OK) return st;
        if (stats) {
            apspie_run_stats part;
            if ((st = finish_call(ctx, &part, "apspie_bfs_batch")) != APSPIE_OK) return st;
            stats->iterations += part.iterations;
            stats->push_iterations += part.push_iterations;
            stats->pull_iterations += part.pull_iterations;
        }
    }
    return APSPIE_OK;
}

}  // namespace apspie

extern "C" apspie_status apspie_bfs_batch(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources,
                                          int32_t num_sources, int32_t depth_cap, int32_t *d_depths,
                                          apspie_run_stats *stats) {
    if (ctx && num_sources > 0 && !d_depths)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_bfs_batch: bad sources/output");
    return bfs_batch_impl(ctx, A, d_sources, num_sources, depth_cap, d_depths, nullptr, stats);
}
