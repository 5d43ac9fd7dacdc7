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
#include <atomic>
#include <cstring>
#include <vector>

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

// ---- continuous batching (the server's BFS engine) ----
// The engine is the same kernel with SERVE = true: instead of a fixed set of sources it
// keeps 32 * W query slots and, at the start of every level, block 0 retires the queries
// whose frontier died in the previous level (posting their ids to the host), then admits
// requests the host posted into a ring in host-mapped memory into free slots, while at most
// 1/kAdmitFrac of the slots are in flight (so that queries run in generations). An admitted
// query starts at that level (its depths are level - start), its output row is filled in
// the same level's first phase, and it runs alongside the queries already in flight. A
// retired slot keeps its visited bits until a sweep clears them; only swept slots are
// reused. The kernel ends when no query is in flight and nothing is waiting (or the host
// stopped admission); the host relaunches it when requests arrive later. Nothing on the
// device waits for the host: the ring is read once per level.
constexpr int kServeRing = 4096;  // request and completion ring entries
#ifndef APSPIE_ADMIT_FRAC
#define APSPIE_ADMIT_FRAC 64
#endif
constexpr int kAdmitFrac = APSPIE_ADMIT_FRAC;  // admissions while at most 1/kAdmitFrac of the slots are in flight
constexpr int kServeSlots = 512;  // upper bound of 32 * W

struct ServeRequest {
    int source;
    int pad;
    unsigned long long row;  // device pointer of the request's int32[m] output
    unsigned long long id;   // host's request id, echoed on completion
};

}  // namespace
}  // namespace apspie

// Host-mapped (cudaHostAllocMapped) ring between the server thread and a running engine.
struct apspie_serve_mailbox {
    volatile unsigned long long tail;   // host: requests posted so far
    volatile int accept;                // host: 0 = admit nothing more, finish and exit
    int pad0;
    volatile unsigned long long head;   // device: requests taken so far
    volatile unsigned long long ctail;  // device: completions posted so far
    unsigned long long pad1[4];
    apspie::ServeRequest req[apspie::kServeRing];
    volatile unsigned long long comp[apspie::kServeRing];  // ids of completed requests, in completion order
};

namespace apspie {
namespace {

// Device-side engine state (part of the engine's scratch; zeroed before each launch).
struct ServeState {
    int *rows[kServeSlots];                // output row of each slot's query
    int start[kServeSlots];                // level at which the slot's query started
    unsigned long long id[kServeSlots];
    unsigned active[16], dirty[16], sweeping[16], alive[2][16];
    int adm_n, exit_flag, pad[2];
    int adm_slot[kServeSlots], adm_src[kServeSlots];
    int *adm_row[kServeSlots];
    unsigned long long adm_id[kServeSlots];
    unsigned long long head, ctail;
};

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
    ServeState *sv;       // SERVE only: engine state
    apspie_serve_mailbox *mb;  // SERVE only: the host-mapped ring (device view)
    long long max_levels; // SERVE only: admission stops after this many levels
};

__device__ __forceinline__ unsigned long long ld_acquire_sys_u64(const volatile unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Block 0's bookkeeping at the start of level L of the engine (see ServeState): retire,
// post completions, admit, decide on a sweep and on the exit. The new sources' bits and
// queue entries are written here; every other block reads the outcome after the barrier.
template <int W>
__device__ void serve_admin(const MsArgs &a, int L, int cur) {
    __shared__ unsigned s_act[W], s_dirty[W], s_ret[W];
    __shared__ int s_nadm;
    __shared__ unsigned long long s_head, s_tail;
    __shared__ int s_accept;
    ServeState *sv = a.sv;
    apspie_serve_mailbox *mb = a.mb;
    constexpr int Q = 32 * W;
    if (threadIdx.x < W) {
        const int w = threadIdx.x;
        unsigned act = __ldcg(&sv->active[w]);
        unsigned ret = 0u;
        if (L > 0) {
            const unsigned alive = __ldcg(&sv->alive[(L - 1) & 1][w]);
            ret = act & ~alive;
            act &= ~ret;
            sv->alive[(L - 1) & 1][w] = 0u;
        }
        // slots swept in the previous level's first phase are clean now
        s_dirty[w] = (__ldcg(&sv->dirty[w]) & ~__ldcg(&sv->sweeping[w])) | ret;
        sv->sweeping[w] = 0u;
        s_act[w] = act;
        s_ret[w] = ret;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (L == 0) {  // a new launch continues the counters of the previous one
            sv->head = mb->head;
            sv->ctail = mb->ctail;
        }
        // completions: slot ids into the ring, then one fence, then the new count
        unsigned long long ct = sv->ctail;
        const unsigned long long ct0 = ct;
        for (int w = 0; w < W; ++w) {
            unsigned b = s_ret[w];
            while (b) {
                const int bit = __ffs(b) - 1;
                b &= b - 1;
                mb->comp[ct % kServeRing] = sv->id[w * 32 + bit];
                ++ct;
            }
        }
        if (ct != ct0) {
            __threadfence_system();
            mb->ctail = ct;
            sv->ctail = ct;
        }
        const unsigned long long tail = ld_acquire_sys_u64(&mb->tail);
        const int accept = mb->accept && L < a.max_levels;
        const unsigned long long head = sv->head;
        int free_clean = 0, in_flight = 0;
        for (int w = 0; w < W; ++w) {
            free_clean += __popc(~(s_act[w] | s_dirty[w]));
            in_flight += __popc(s_act[w]);
        }
        // new queries join only while at most 1/kAdmitFrac of the slots are in flight, so
        // that queries run in generations that start (nearly) together: their frontiers
        // grow and shrink together, and a bottom-up level serves them all. Queries started
        // at every level would keep some frontier small at every level, and the bottom-up
        // scans would read whole rows for them level after level. (Letting a generation
        // also admit at its second level, into the slots swept meanwhile, measured 20 %
        // fewer queries per second: one level of stagger already costs that much.)
        const bool gate = in_flight * kAdmitFrac <= Q;
        const unsigned long long waiting = tail > head ? tail - head : 0ull;
        s_nadm = accept && gate
                     ? static_cast<int>(waiting < static_cast<unsigned long long>(free_clean) ? waiting : free_clean)
                     : 0;
        s_head = head;
        s_tail = tail;
        s_accept = accept;
    }
    __syncthreads();
    // read the admitted requests in parallel (each a read of host memory)
    for (int k = threadIdx.x; k < s_nadm; k += blockDim.x) {
        const ServeRequest *r = &mb->req[(s_head + k) % kServeRing];
        sv->adm_src[k] = *reinterpret_cast<const volatile int *>(&r->source);
        sv->adm_row[k] = reinterpret_cast<int *>(*reinterpret_cast<const volatile unsigned long long *>(&r->row));
        sv->adm_id[k] = *reinterpret_cast<const volatile unsigned long long *>(&r->id);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // assign clean free slots in order
        int k = 0;
        for (int w = 0; w < W && k < s_nadm; ++w) {
            unsigned fr = ~(s_act[w] | s_dirty[w]);
            while (fr && k < s_nadm) {
                const int bit = __ffs(fr) - 1;
                fr &= fr - 1;
                const int slot = w * 32 + bit;
                sv->adm_slot[k] = slot;
                sv->rows[slot] = sv->adm_row[k];
                sv->id[slot] = sv->adm_id[k];
                sv->start[slot] = L;
                s_act[w] |= 1u << bit;
                ++k;
            }
        }
        const unsigned long long nh = s_head + s_nadm;
        sv->head = nh;
        mb->head = nh;
        sv->adm_n = s_nadm;
        int *qlen = cur < 2 ? &a.ctl->qlen[cur] : reinterpret_cast<int *>(&a.ctl->aux[0]);
        for (int j = 0; j < s_nadm; ++j) {
            const int slot = sv->adm_slot[j], v = sv->adm_src[j];
            const unsigned bit = 1u << (slot & 31);
            atomicOr(a.vis + static_cast<long long>(v) * W + (slot >> 5), bit);
            atomicOr(a.fr[L & 1] + static_cast<long long>(v) * W + (slot >> 5), bit);
            a.q[cur][atomicAdd(qlen, 1)] = v;
        }
        int nact = 0, ndirty = 0, nfree = 0;
        for (int w = 0; w < W; ++w) {
            nact += __popc(s_act[w]);
            ndirty += __popc(s_dirty[w]);
            nfree += __popc(~(s_act[w] | s_dirty[w]));
        }
        const bool pending = s_accept && s_tail > nh;
        const bool sweep = ndirty > 0 && (4 * ndirty >= Q || (pending && nfree == 0));
        for (int w = 0; w < W; ++w) {
            sv->active[w] = s_act[w];
            sv->dirty[w] = s_dirty[w];
            sv->sweeping[w] = sweep ? s_dirty[w] : 0u;
        }
        sv->exit_flag = nact == 0 && !pending && !sweep;
    }
}

__device__ __forceinline__ int *depth_row(const MsArgs &a, int q) {
    return a.rows ? a.rows[q] : a.out + static_cast<long long>(q) * a.m;
}

// Writes depth L + 1 of vertex v for query slot q (in the engine: relative to the level the
// query started at, and into the row its request gave; both are copied into shared memory
// at the start of every level: s_row, s_base).
template <bool SERVE>
__device__ __forceinline__ void put_depth(const MsArgs &a, int q, int v, int L, int *const *s_row,
                                          const int *s_base) {
    if (SERVE)
        s_row[q][v] = L + 1 - s_base[q];
    else
        depth_row(a, q)[v] = L + 1;
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

template <int W, bool SERVE>
__global__ void __launch_bounds__(kMsBlock, W >= 16 ? 3 : 4) msbfs_kernel(MsArgs a) {
    __shared__ MsSmem sm;
    __shared__ unsigned s_qmask[W];   // query slots in flight this level
    __shared__ unsigned s_alive[W];   // bits this block found in the next frontier (engine)
    __shared__ int *s_row[SERVE ? 32 * W : 1];  // engine: each slot's output row this level
    __shared__ int s_base[SERVE ? 32 * W : 1];  // engine: each slot's start level
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
    if (threadIdx.x < W) {
        s_qmask[threadIdx.x] = query_mask(a.nq, threadIdx.x);
        s_alive[threadIdx.x] = 0u;
    }
    if (!grid_barrier(a.ctl, a.sticky, kSiteMs)) return;
    const int nheavy = ld_volatile_i32(hlen);
    // level 0: the sources (the engine admits its queries level by level instead)
    if (!SERVE) {
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
    if (!SERVE) {
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
        if (SERVE) {
            if (blockIdx.x == 0) serve_admin<W>(a, L, cur);
            if (!grid_barrier(a.ctl, a.sticky, kSiteMs + 6)) return;
            if (ld_volatile_i32(&a.sv->exit_flag)) break;
            if (threadIdx.x < W) s_qmask[threadIdx.x] = __ldcg(&a.sv->active[threadIdx.x]);
            for (int q = threadIdx.x; q < 32 * W; q += blockDim.x) {
                s_row[SERVE ? q : 0] = reinterpret_cast<int *const volatile *>(a.sv->rows)[q];
                s_base[SERVE ? q : 0] = __ldcg(&a.sv->start[q]);
            }
            // first phase of the level: the admitted queries' output rows (0 at the source,
            // -1 elsewhere), and the sweep of retired slots' visited bits
            const int nadm = ld_volatile_i32(&a.sv->adm_n);
            for (int k = 0; k < nadm; ++k) {
                const int slot = __ldcg(&a.sv->adm_slot[k]);
                const int src = __ldcg(&a.sv->adm_src[k]);
                int *row = reinterpret_cast<int *const volatile *>(a.sv->rows)[slot];
                int done = 0;
                if ((reinterpret_cast<uintptr_t>(row) & 15u) == 0) {  // four entries per store
                    const int m4 = m >> 2;
                    for (int i = gtid; i < m4; i += gstride) {
                        int4 x = make_int4(-1, -1, -1, -1);
                        if (i == src >> 2) {
                            x.x = (src & 3) == 0 ? 0 : -1;
                            x.y = (src & 3) == 1 ? 0 : -1;
                            x.z = (src & 3) == 2 ? 0 : -1;
                            x.w = (src & 3) == 3 ? 0 : -1;
                        }
                        reinterpret_cast<int4 *>(row)[i] = x;
                    }
                    done = m4 << 2;
                }
                for (int i = done + gtid; i < m; i += gstride) row[i] = i == src ? 0 : -1;
            }
            unsigned sw[W];
            bool any_sw = false;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                sw[w] = __ldcg(&a.sv->sweeping[w]);
                any_sw |= sw[w] != 0u;
            }
            if (any_sw)
                for (long long x = gtid; x < mw; x += gstride) {
                    const unsigned c = sw[x % W];
                    if (c) a.vis[x] &= ~c;
                }
            __syncthreads();
        }
        const int nA = ld_volatile_i32(qlen_ptr(a.ctl, cur));
        if (!SERVE && nA == 0) break;
        if (!SERVE && a.depth_cap > 0 && L + 1 >= a.depth_cap) break;
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
                            if (SERVE) atomicOr(&s_alive[w], nb);
                            unsigned b = nb;
                            while (b) {
                                const int bit = __ffs(b) - 1;
                                b &= b - 1;
                                put_depth<SERVE>(a, w * 32 + bit, v, L, s_row, s_base);
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
                        need[w] = ~__ldcg(vv + w) & s_qmask[w];
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
                        if ((got[w] >> bit) & 1u) put_depth<SERVE>(a, w * 32 + bit, v, L, s_row, s_base);
                    }
                    if (SERVE) {
                        const unsigned wa = __reduce_or_sync(lanemask_all, got[w]);
                        if (lane == 0 && wa) atomicOr(&s_alive[w], wa);
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
                    s_need[threadIdx.x] = ~__ldcg(vv + threadIdx.x) & s_qmask[threadIdx.x];
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
                            if (SERVE) atomicOr(&s_alive[threadIdx.x], got);
                            unsigned b = got;
                            while (b) {
                                const int bit = __ffs(b) - 1;
                                b &= b - 1;
                                put_depth<SERVE>(a, threadIdx.x * 32 + bit, v, L, s_row, s_base);
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
        if (SERVE) {
            // this block's share of the next frontier's query bits: the queries still alive
            __syncthreads();
            if (threadIdx.x < W && s_alive[threadIdx.x]) {
                atomicOr(&a.sv->alive[L & 1][threadIdx.x], s_alive[threadIdx.x]);
                s_alive[threadIdx.x] = 0u;
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
    return reinterpret_cast<const void *>(msbfs_kernel<W, false>);
}

template <int W>
const void *msbfs_serve_fn() {
    return reinterpret_cast<const void *>(msbfs_kernel<W, true>);
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

// ---- the server's continuous BFS engine: host side ----
struct BfsEngine {
    apspie_serve_mailbox *mb = nullptr;  // host view
    apspie_serve_mailbox *d_mb = nullptr;  // device view of the same memory
    unsigned long long posted = 0;  // host copy of mb->tail
    unsigned long long seen = 0;    // completions consumed
};

namespace apspie {

// The engine's frontier lists can hold every vertex plus one level's admitted sources (a
// source may also be on the list already), so they get kServeSlots more entries.
size_t bfs_engine_scratch_need(int m, int W) {
    return batch_need(m, W) + Carver::need({sizeof(ServeState)}) + 5 * (kServeSlots * sizeof(int) + 256);
}

int bfs_engine_words(int slots) { return padded_words(slots < 32 ? 32 : slots > kServeSlots ? kServeSlots : slots); }

apspie_status bfs_engine_create(BfsEngine **out) {
    BfsEngine *e = new BfsEngine();
    void *h = nullptr, *d = nullptr;
    if (cudaHostAlloc(&h, sizeof(apspie_serve_mailbox), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
        (void)cudaGetLastError();
        if (h) cudaFreeHost(h);
        delete e;
        return APSPIE_ERR_OOM;
    }
    std::memset(h, 0, sizeof(apspie_serve_mailbox));
    e->mb = static_cast<apspie_serve_mailbox *>(h);
    e->d_mb = static_cast<apspie_serve_mailbox *>(d);
    *out = e;
    return APSPIE_OK;
}

void bfs_engine_destroy(BfsEngine *e) {
    if (!e) return;
    if (e->mb) cudaFreeHost(e->mb);
    delete e;
}

// Posts a request (source, output row, id); false when the ring is full.
bool bfs_engine_post(BfsEngine *e, int source, int *row, unsigned long long id) {
    if (e->posted - e->seen >= static_cast<unsigned long long>(kServeRing)) return false;
    ServeRequest &r = e->mb->req[e->posted % kServeRing];
    r.source = source;
    r.row = reinterpret_cast<unsigned long long>(row);
    r.id = id;
    std::atomic_thread_fence(std::memory_order_release);  // entry before the new tail
    ++e->posted;
    e->mb->tail = e->posted;
    return true;
}

// Completed request ids since the last call (at most cap).
int bfs_engine_completions(BfsEngine *e, unsigned long long *ids, int cap) {
    const unsigned long long ct = e->mb->ctail;
    std::atomic_thread_fence(std::memory_order_acquire);
    int n = 0;
    while (e->seen < ct && n < cap) ids[n++] = e->mb->comp[e->seen++ % kServeRing];
    return n;
}

// Requests posted that no launch has taken yet.
unsigned long long bfs_engine_waiting(const BfsEngine *e) { return e->posted - e->mb->head; }

void bfs_engine_set_accept(BfsEngine *e, int on) { e->mb->accept = on ? 1 : 0; }

// After a launch ended: the ids of the requests still waiting in the ring (posted, never
// taken), oldest first; the ring forgets them.
std::vector<unsigned long long> bfs_engine_take_back(BfsEngine *e) {
    std::vector<unsigned long long> ids;
    const unsigned long long head = e->mb->head;
    for (unsigned long long k = head; k < e->posted; ++k) ids.push_back(e->mb->req[k % kServeRing].id);
    e->posted = head;
    e->mb->tail = head;
    return ids;
}

// Launches the engine with 32 * W query slots on the context's stream (asynchronous);
// it runs until no request is in flight or waiting, or until admission is switched off.
apspie_status bfs_engine_launch(apspie_ctx *ctx, const apspie_csr *A, int W, BfsEngine *e) {
    cudaSetDevice(ctx->device);
    const int m = A->m;
    if (W != 1 && W != 2 && W != 4 && W != 8 && W != 16) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "engine words");
    void *base;
    apspie_status st = scratch_reserve(ctx, bfs_engine_scratch_need(m, W), &base);
    if (st != APSPIE_OK) return st;
    const size_t mi = static_cast<size_t>(m) + 1;
    const size_t ml = mi + kServeSlots;  // frontier lists and their per-entry arrays
    const size_t mw = static_cast<size_t>(m) * W;
    const size_t words = (static_cast<size_t>(m) + 31) / 32;
    Carver c(base);
    MsArgs a;
    std::memset(&a, 0, sizeof(a));
    a.vis = c.take<unsigned>(mw);
    a.fr[0] = c.take<unsigned>(mw);
    a.fr[1] = c.take<unsigned>(mw);
    a.touched = c.take<unsigned>(words);
    a.q[0] = c.take<int>(ml);
    a.q[1] = c.take<int>(ml);
    a.q[2] = c.take<int>(ml);
    a.tq = c.take<int>(mi);
    a.heavy = c.take<int>(mi);
    a.rs = c.take<int>(ml);
    a.loc_off = c.take<int>(ml);
    a.chunk_sum = c.take<int>(kMaxGrid);
    a.sv = c.take<ServeState>(1);
    a.mb = e->d_mb;
    a.rows = a.sv->rows;
    a.m = m;
    a.nnz = A->nnz;
    a.nq = 32 * W;
    a.depth_cap = 0;
    a.row_ptr = A->row_ptr;
    a.col_ind = A->col_ind;
    a.ctl = ctx->d_ctl;
    a.sticky = ctx->d_sticky_err;
    a.max_levels = 1LL << 40;
    a.push_frac = (A->flags & APSPIE_CSR_SYMMETRIC) ? effective_params(ctx, APSPIE_TUNE_BFS_BATCH, A).batch_push_frac
                                                     : 1e30f;
    e->mb->accept = 1;
    cudaError_t err = cudaMemsetAsync(a.sv, 0, sizeof(ServeState), ctx->stream);
    if (err != cudaSuccess) return cuda_error(ctx, err, "bfs engine reset");
    if ((st = reset_ctl(ctx)) != APSPIE_OK) return st;
    const void *fn = W == 1 ? msbfs_serve_fn<1>() : W == 2 ? msbfs_serve_fn<2>() : W == 4 ? msbfs_serve_fn<4>()
                     : W == 8 ? msbfs_serve_fn<8>() : msbfs_serve_fn<16>();
    void *args[] = {&a};
    return launch_persistent(ctx, fn, kMsBlock, args, 1LL << 40);
}

}  // namespace apspie

extern "C" apspie_status apspie_bfs_batch(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources,
                                          int32_t num_sources, int32_t depth_cap, int32_t *d_depths,
                                          apspie_run_stats *stats) {
    if (ctx && num_sources > 0 && !d_depths)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_bfs_batch: bad sources/output");
    return bfs_batch_impl(ctx, A, d_sources, num_sources, depth_cap, d_depths, nullptr, stats);
}
