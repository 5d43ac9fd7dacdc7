// Persistent SpMSpV traversal kernels: BFS (boolean OR-AND), SSSP (min-plus), MIS
// (priority max), and the one-hop boolean SpMSpV.
//
// Each algorithm is ONE cooperative launch whose blocks loop over levels/iterations with
// a bounded grid barrier between phases; the host never reads a count mid-run. This
// replaces the reference's host-driven level loops (src/bfs.cuh:87-110,
// src/spmspvBfs.cuh:174-222, src/sssp.cuh:79-98, src/spmspvMis.cuh:232-318), which issue
// ~10-14 launches, up to 3 device->host syncs and a cudaMalloc/cudaFree per level, and
// which stop after a caller-supplied `depth` taken from the CPU BFS.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "frontier.cuh"

namespace apspie {

namespace {

// Build-time knobs of the SSSP kernel (defaults are the tuned values).
#ifndef APSPIE_SSSP_VT
#define APSPIE_SSSP_VT 4
#endif
#ifndef APSPIE_SSSP_MINB
#define APSPIE_SSSP_MINB 4
#endif
#ifndef APSPIE_SSSP_RED
#define APSPIE_SSSP_RED 1
#endif
#ifndef APSPIE_SSSP_PREREAD
#define APSPIE_SSSP_PREREAD 1
#endif


constexpr int kBlock = 256;
constexpr int kVT = 4;
using BfsSmem = ExpandSmem<kBlock, kVT, false>;
using BfsSlice = BfsSmem::Warp;
constexpr int kSsspVT = APSPIE_SSSP_VT;
constexpr int kSsspPA = 4;  // frontier entries per thread per phase-A step
using SsspSmem = ExpandSmem<kBlock, kSsspVT, false>;
using SsspSlice = SsspSmem::Warp;
using WQ = WarpQueue<BfsSmem::QCAP>;

struct NoPost {
    template <class S>
    __device__ void operator()(int, S &) const {}
};

constexpr int kInf = 0x7fffffff;

// device error sites (reported as err_where)
enum : int {
    kSiteBfs = 100,
    kSiteSssp = 200,
    kSiteSsspNegWeight = 201,
    kSiteSsspOverflow = 202,
    kSiteSsspIterCap = 203,
    kSiteSsspBarA = 210,
    kSiteSsspBarB = 211,
    kSiteSsspBarF0 = 212,
    kSiteSsspBarF1 = 213,
    kSiteSsspGroup = 214,  // and 215
    kSiteSsspBadSource = 216,
    kSiteMis = 300,
    kSiteMisRoundCap = 301,
};

struct TravBuffers {
    int *q0, *q1, *q2, *q3, *rs, *loc_off, *chunk_sum, *aux, *aux2;
    unsigned *bits0, *bits1, *bits2;
};

size_t trav_scratch_bytes(int m) {
    const size_t words = (static_cast<size_t>(m) + 31) / 32;
    const size_t mi = static_cast<size_t>(m) + 1;
    return Carver::need({mi * 4, mi * 4, mi * 4, mi * 4, mi * 4, mi * 4, kMaxGrid * 4, mi * 4,
                         mi * 4, words * 4, words * 4, words * 4});
}

TravBuffers carve_trav(void *base, int m) {
    const size_t words = (static_cast<size_t>(m) + 31) / 32;
    const size_t mi = static_cast<size_t>(m) + 1;
    Carver c(base);
    TravBuffers b;
    b.q0 = c.take<int>(mi);
    b.q1 = c.take<int>(mi);
    b.q2 = c.take<int>(mi);
    b.q3 = c.take<int>(mi);
    b.rs = c.take<int>(mi);
    b.loc_off = c.take<int>(mi);
    b.chunk_sum = c.take<int>(kMaxGrid);
    b.aux = c.take<int>(mi);
    b.aux2 = c.take<int>(mi);
    b.bits0 = c.take<unsigned>(words);
    b.bits1 = c.take<unsigned>(words);
    b.bits2 = c.take<unsigned>(words);
    return b;
}

// ================================================================================
// BFS
// ================================================================================
struct BfsArgs {
    int m, nnz, src, depth_cap;
    const int *__restrict__ row_ptr;
    const int *__restrict__ col_ind;
    int *depth;
    TravBuffers buf;  // bits0 = visited, bits1/bits2 = frontier bitmaps (ping-pong)
    TravCtl *ctl;
    int *sticky;
    float alpha, beta;
    int allow_pull;  // pattern declared symmetric
};

// Level-synchronous BFS. Level L discovers the vertices at hop distance L.
//  push (top-down): merge-path expansion of the frontier queue; a neighbour is claimed by
//      an atomicOr test-and-set on the visited bitmap (the dedup that replaces the
//      reference's radix sort, src/spmspvBfs.cuh:195-197), its depth written, and it is
//      appended to the next queue by a warp-aggregated ballot.
//  pull (bottom-up): one warp per 32-vertex bitmap word; each unvisited vertex scans its
//      row until it meets a frontier vertex (frontier bitmap built in phase A).
// The direction follows Beamer's rule on the edges out of the frontier (m_f) against the
// edges still unexplored (m_u): push->pull when m_f > m_u/alpha, pull->push when the
// frontier holds fewer than m/beta vertices. Depth results do not depend on the choice.
__global__ void __launch_bounds__(kBlock) bfs_kernel(BfsArgs a) {
    __shared__ BfsSmem sm;
    timeline_mark(a.ctl, 0);
    const int G = gridDim.x;
    const int gtid = blockIdx.x * kBlock + threadIdx.x;
    const int gstride = G * kBlock;
    const int m = a.m;
    const int words = (m + 31) >> 5;
    unsigned *vis = a.buf.bits0;

    for (int i = gtid; i < m; i += gstride) a.depth[i] = (i == a.src) ? 0 : -1;
    for (int w = gtid; w < words; w += gstride) {
        vis[w] = (w == (a.src >> 5)) ? (1u << (a.src & 31)) : 0u;
        a.buf.bits1[w] = 0u;
        a.buf.bits2[w] = 0u;
    }
    if (gtid == 0) {
        a.buf.q0[0] = a.src;
        a.ctl->qlen[0] = 1;
        a.ctl->qlen[1] = 0;
    }
    if (!grid_barrier(a.ctl, a.sticky, kSiteBfs)) return;

    int cur = 0;
    bool pull = false;
    long long visited_edges = 0, reached = 0, expanded = 0;
    int levels = 0, npush = 0, npull = 0;
    for (int L = 1;; ++L) {
        const int nf = ld_volatile_i32(&a.ctl->qlen[cur]);
        if (nf == 0) break;
        if (a.depth_cap > 0 && L >= a.depth_cap) break;
        int *qc = cur ? a.buf.q1 : a.buf.q0;
        int *qn = cur ? a.buf.q0 : a.buf.q1;
        unsigned *fbc = cur ? a.buf.bits2 : a.buf.bits1;
        unsigned *fbn = cur ? a.buf.bits1 : a.buf.bits2;
        int *qlen_next = &a.ctl->qlen[cur ^ 1];

        // phase A: frontier degrees + frontier bitmap
        frontier_phase_a<kBlock>(qc, nf, a.row_ptr, a.buf.rs, a.buf.loc_off, a.buf.chunk_sum,
                                 sm.scan_tmp, [&](int, int v, int deg) {
                                     atomicOr(fbc + (v >> 5), 1u << (v & 31));
                                     return deg;
                                 });
        if (gtid == 0) *qlen_next = 0;
        if (!grid_barrier(a.ctl, a.sticky, kSiteBfs + 1)) return;

        const int E = frontier_chunk_bases<kBlock>(a.buf.chunk_sum, sm.base, sm.scan_tmp);
        visited_edges += E;
        reached += nf;
        expanded += E;
        const long long m_u = static_cast<long long>(a.nnz) - visited_edges;
        if (!pull) {
            if (a.allow_pull && a.alpha > 0.0f &&
                static_cast<double>(E) > static_cast<double>(m_u) / a.alpha)
                pull = true;
        } else if (static_cast<double>(nf) < static_cast<double>(m) / a.beta) {
            pull = false;
        }
        ++levels;

        // phase B
        const int wid = threadIdx.x >> 5;
        WQ wq(sm.qbuf[wid][0], qn, qlen_next);
        if (!pull) {
            ++npush;
            const int *col = a.col_ind;
            int *depth = a.depth;
            frontier_expand<kBlock, kVT, false>(
                nf, E, a.buf.loc_off, a.buf.rs, sm, [](int, int, BfsSlice &) {},
                [&](const bool (&valid)[kVT], const int (&kk)[kVT], const int (&idx)[kVT],
                    BfsSlice &) {
                    int v[kVT];
                    unsigned word[kVT];
#pragma unroll
                    for (int r = 0; r < kVT; ++r) v[r] = valid[r] ? __ldg(col + idx[r]) : 0;
#pragma unroll
                    for (int r = 0; r < kVT; ++r) word[r] = valid[r] ? __ldcg(vis + (v[r] >> 5)) : ~0u;
                    bool fresh[kVT];
#pragma unroll
                    for (int r = 0; r < kVT; ++r) {
                        const unsigned bit = 1u << (v[r] & 31);
                        fresh[r] = false;
                        if (valid[r] && !(word[r] & bit)) fresh[r] = !(atomicOr(vis + (v[r] >> 5), bit) & bit);
                    }
#pragma unroll
                    for (int r = 0; r < kVT; ++r) {
                        if (fresh[r]) depth[v[r]] = L;
                        wq.push(fresh[r], v[r]);
                    }
                },
                NoPost());
            wq.flush();
        } else {
            ++npull;
            const int lane = threadIdx.x & 31;
            const int nwarps = gstride >> 5;
            for (int w = gtid >> 5; w < words; w += nwarps) {
                const unsigned vw = __ldcg(vis + w);
                const int v = (w << 5) + lane;
                bool found = false;
                if (v < m && !(vw & (1u << lane))) {
                    const int r0 = __ldg(a.row_ptr + v), r1 = __ldg(a.row_ptr + v + 1);
                    for (int e = r0; e < r1; ++e) {
                        const int u = __ldg(a.col_ind + e);
                        if (__ldcg(fbc + (u >> 5)) & (1u << (u & 31))) {
                            found = true;
                            break;
                        }
                    }
                }
                const unsigned fm = __ballot_sync(0xffffffffu, found);
                if (fm) {
                    if (lane == 0) vis[w] = vw | fm;  // this warp owns word w in pull
                    if (found) a.depth[v] = L;
                    wq.push(found, v);
                }
            }
            wq.flush();
        }
        // the other frontier bitmap is idle this level: clear it for level L+1
        for (int w = gtid; w < words; w += gstride) fbn[w] = 0u;
        if (!grid_barrier(a.ctl, a.sticky, kSiteBfs + 2)) return;
        cur ^= 1;
    }
    if (gtid == 0) {
        a.ctl->iterations = levels;
        a.ctl->push_iterations = npush;
        a.ctl->pull_iterations = npull;
        a.ctl->edges_expanded = expanded;
        a.ctl->edges_component = visited_edges;
        a.ctl->vertices_reached = reached;
    }
}

// ================================================================================
// SSSP
// ================================================================================
struct SsspArgs {
    int m, nnz, src, delta_hint;
    int is_float;        // weights/distances are non-negative float32 held as their bit patterns
    int unreached_bits;  // written for unreached vertices (int -1, or a float's bits)
    long long band;      // edges per iteration of the distance band; <= 0: whole frontier
    const int *__restrict__ row_ptr;
    const int *__restrict__ col_ind;
    const int *__restrict__ w;
    int *dist;
    // bits0 = queued in the near frontier, bits1 = held in the far pile;
    // q0/q1 near queues, q2/q3 far piles, aux = distance snapshot of each near entry,
    // aux2 = distance each vertex was last expanded with
    TravBuffers buf;
    TravCtl *ctl;
    int *sticky;
};

// Histogram bin of distance d above the band base hb: 8 linear bins, then 8 bins per
// octave (three mantissa bits), 256 in all. Integer distances count in units of 1; float
// distances in units of 1/inv_unit.
__device__ __forceinline__ int band_bin(int d, int hb, int is_float, float inv_unit) {
    if (d <= hb) return 0;
    if (!is_float) {
        const unsigned x = static_cast<unsigned>(d) - static_cast<unsigned>(hb);
        if (x < 8u) return static_cast<int>(x);
        const int e = 31 - __clz(x);
        return 8 * (e - 2) + static_cast<int>((x >> (e - 3)) & 7u);
    }
    const float x = (__int_as_float(d) - __int_as_float(hb)) * inv_unit;
    if (x < 8.0f) return static_cast<int>(x);
    const unsigned b = __float_as_uint(x);
    const int e = static_cast<int>(b >> 23) - 127;
    const int bin = 8 * (e - 2) + static_cast<int>((b >> 20) & 7u);
    return bin < kBandBins - 1 ? bin : kBandBins - 1;
}

struct SsspShared {
    SsspSmem ex;
    unsigned long long hist[kBandBins];  // this block's share of the next band histogram
    unsigned long long scan[33];
    int hmin;                            // least distance this block queued
    int dbase;                           // where this block's deferred entries go
};

// Min-plus SpMSpV iterated to the fixed point with near/far buckets (delta-stepping in
// the near-far form): the frontier holds the vertices whose distance dropped below the
// current threshold T; a relaxation that lands at or above T parks the vertex on the far
// pile instead. When the near frontier empties, T advances by delta and the far pile is
// split into the new near frontier and what stays far. A vertex is expanded again only
// if its distance changed since its last expansion. Within the near frontier only the band
// of lowest distances carrying about a.band edges is expanded per iteration; the rest wait
// in the queue. The band's cut comes from a degree-weighted histogram of the distances
// queued during the previous iteration, taken relative to that queue's least distance,
// which is tracked exactly, and the vertices at that least distance always expand, so
// every iteration makes progress. The reference expands every finite
// vertex each iteration (src/spmspvSssp.cuh:31-36, sort + ReduceByKey(min) :220-232) and
// stops after the CPU BFS depth; here a relaxation is a plain read of dist[v] and, only
// if it improves, an atomicMin, and the loop ends when both piles are empty. The result is
// the exact fixed point for non-negative integer weights, independent of relaxation order.
__device__ __forceinline__ void sssp_body(SsspArgs a, VGrid vg) {
    static_assert(kBlock == kBandBins, "one histogram bin per thread");
    __shared__ SsspShared sh;
    SsspSmem &sm = sh.ex;
    timeline_mark(a.ctl, 0);
    const int G = vg.n;
    const int gtid = vg.id * kBlock + threadIdx.x;
    const int gstride = G * kBlock;
    const int m = a.m;
    const int words = (m + 31) >> 5;
    unsigned *inq = a.buf.bits0;
    unsigned *infar = a.buf.bits1;
    int *last = a.buf.aux2;

    // non-negative float32 values order like their int bit patterns, so one integer
    // atomicMin serves both weight types; +inf is the float "infinity"
    const int INF = a.is_float ? 0x7f800000 : kInf;
    for (int i = gtid; i < m; i += gstride) {
        a.dist[i] = (i == a.src) ? 0 : INF;
        last[i] = -1;
    }
    for (int w = gtid; w < words; w += gstride) {
        inq[w] = (w == (a.src >> 5)) ? (1u << (a.src & 31)) : 0u;
        infar[w] = 0u;
    }
    // sample the weights for the default bucket width
    constexpr int kSample = 1 << 16;
    const int nsamp = a.nnz < kSample ? a.nnz : kSample;
    {
        double ws = 0.0;
        for (int k = gtid; k < nsamp; k += gstride) {
            const int wb = __ldg(a.w + static_cast<long long>(k) * a.nnz / nsamp);
            ws += a.is_float ? static_cast<double>(__int_as_float(wb)) : static_cast<double>(wb);
        }
        for (int o = 16; o; o >>= 1) ws += __shfl_down_sync(0xffffffffu, ws, o);
        if ((threadIdx.x & 31) == 0 && ws != 0.0) atomicAdd(reinterpret_cast<double *>(&a.ctl->aux[0]), ws);
    }
    if (gtid == 0) {
        a.buf.q0[0] = a.src;
        a.ctl->qlen[0] = 1;
        a.ctl->qlen[1] = 0;
        a.ctl->flen[0] = 0;
        a.ctl->flen[1] = 0;
        a.ctl->sbase[0] = 0;  // the source's distance
        a.ctl->sbase[1] = INF;
    }
    sh.hist[threadIdx.x] = 0ull;
    if (threadIdx.x == 0) sh.hmin = INF;
    if (!grid_barrier(a.ctl, a.sticky, kSiteSssp, vg)) return;

    const bool banded = a.band > 0;
    const double sum_w = __longlong_as_double(__ldcg(&a.ctl->aux[0]));
    const double mean_w = nsamp ? sum_w / nsamp : 1.0;
    // float distances are binned in units of mean weight / 256
    const float inv_unit = (a.is_float && mean_w > 0.0) ? static_cast<float>(256.0 / mean_w) : 1.0f;
    double delta = a.delta_hint;
    if (delta <= 0 && banded) {
        delta = 1e300;  // the band orders the work: no far pile
    } else if (delta <= 0) {
        const double mean_deg = m ? static_cast<double>(a.nnz) / m : 1.0;
        delta = 32.0 * mean_w / (mean_deg > 1.0 ? mean_deg : 1.0);
        if (!a.is_float) delta = floor(delta);
        if (!(delta >= 1.0)) delta = a.is_float ? (delta > 0.0 ? delta : 1.0) : 1.0;
    }
    double thresh = delta;
    int hb = 0;  // base of the histogram in ctl->shist[cur] (the previous iteration's base)
    int cur = 0, fc = 0;
    long long expanded = 0;
    int iters = 0, steps = 0;
    const long long step_cap = 4LL * m + 4096;
    for (;;) {
        if (++steps > step_cap) {
            if (gtid == 0) raise_error(a.ctl, a.sticky, APSPIE_ERR_NOT_CONVERGED, kSiteSsspIterCap);
            break;
        }
        const int nf = ld_volatile_i32(&a.ctl->qlen[cur]);
        int *qc = cur ? a.buf.q1 : a.buf.q0;
        int *qn = cur ? a.buf.q0 : a.buf.q1;
        int *fcur = fc ? a.buf.q3 : a.buf.q2;
        int *fnext = fc ? a.buf.q2 : a.buf.q3;
        int *dist = a.dist;
        if (nf == 0) {
            // near frontier empty: advance the threshold and split the far pile
            const int nfar = ld_volatile_i32(&a.ctl->flen[fc]);
            if (nfar == 0) break;
            thresh += delta;
            // every block must have read qlen[cur] (== 0) before any block appends to it
            if (!grid_barrier(a.ctl, a.sticky, kSiteSsspBarF0, vg)) return;
            WQ wn(sm.qbuf[threadIdx.x >> 5][0], qc, &a.ctl->qlen[cur]);
            WQ wf(sm.qbuf[threadIdx.x >> 5][1], fnext, &a.ctl->flen[fc ^ 1]);
            for (int base = vg.id * kBlock; base < nfar; base += gstride) {
                const int i = base + threadIdx.x;
                bool to_near = false, stay = false;
                int v = 0;
                if (i < nfar) {
                    v = __ldcg(fcur + i);
                    const int d = __ldcg(dist + v);
                    const double dv = a.is_float ? static_cast<double>(__int_as_float(d)) : static_cast<double>(d);
                    if (dv < thresh) {
                        atomicAnd(infar + (v >> 5), ~(1u << (v & 31)));
                        const unsigned bit = 1u << (v & 31);
                        to_near = !(atomicOr(inq + (v >> 5), bit) & bit);
                        atomicMin(&a.ctl->sbase[cur], d);
                    } else {
                        stay = true;
                    }
                }
                wn.push(to_near, v);
                wf.push(stay, v);
            }
            wn.flush();
            wf.flush();
            if (!grid_barrier(a.ctl, a.sticky, kSiteSsspBarF1, vg)) return;
            if (gtid == 0) a.ctl->flen[fc] = 0;  // drained; every block read nfar above
            fc ^= 1;
            continue;
        }
        int *qlen_next = &a.ctl->qlen[cur ^ 1];  // zero: reset when that queue was last read
        int *snap = a.buf.aux;

        // the band: histogram bins up to the first where the running edge count reaches
        // a.band (kBandBins = every bin: band off, or too little queued work to cut)
        const int base_i = ld_volatile_i32(&a.ctl->sbase[cur]);
        int cut = kBandBins;
        if (banded) {
            const unsigned long long h = __ldcg(&a.ctl->shist[cur][threadIdx.x]);
            const unsigned long long incl = block_inclusive_scan_u64<kBlock>(h, sh.scan);
            const unsigned long long S = static_cast<unsigned long long>(a.band);
            const bool reach = sh.scan[32] >= S;
            const int below = __syncthreads_count(incl < S);
            if (reach && below < kBandBins - 1) cut = below;
        }
        const int hb_prev = hb;
        hb = base_i;
        const int is_float_a = a.is_float;

        // phase A: dequeue (clear queued bit), snapshot distance, skip unchanged vertices;
        // vertices above the band stay queued (re-appended to the next queue, bit kept)
        {
            // kSsspPA entries per thread per step, their loads issued together; the chunk
            // layout (chunk c = entries [c*C, (c+1)*C)) is the one frontier_expand reads
            constexpr int PA = kSsspPA;
            const int C = (nf + G - 1) / G;
            const int c0 = min(vg.id * C, nf);
            const int c1 = min(c0 + C, nf);
            const int *rpa = a.row_ptr;
            int carry = 0;
            for (int base = c0; base < c1; base += kBlock * PA) {
                const int i0 = base + static_cast<int>(threadIdx.x) * PA;
                int v[PA], r0[PA], r1[PA], d[PA], lst[PA], out[PA];
                bool valid[PA], defer[PA];
#pragma unroll
                for (int k = 0; k < PA; ++k) {
                    valid[k] = i0 + k < c1;
                    v[k] = valid[k] ? __ldcg(qc + i0 + k) : 0;
                }
#pragma unroll
                for (int k = 0; k < PA; ++k) {
                    r0[k] = valid[k] ? __ldg(rpa + v[k]) : 0;
                    r1[k] = valid[k] ? __ldg(rpa + v[k] + 1) : 0;
                    d[k] = valid[k] ? __ldcg(dist + v[k]) : 0;
                }
#pragma unroll
                for (int k = 0; k < PA; ++k) {
                    defer[k] = valid[k] && cut < kBandBins && d[k] != base_i &&
                               band_bin(d[k], hb_prev, is_float_a, inv_unit) > cut;
                    lst[k] = (valid[k] && !defer[k]) ? __ldcg(last + v[k]) : 0;
                }
                int sum = 0;
#pragma unroll
                for (int k = 0; k < PA; ++k) {
                    out[k] = 0;
                    if (valid[k]) {
                        snap[i0 + k] = d[k];
                        a.buf.rs[i0 + k] = r0[k];
                        if (!defer[k]) {
                            atomicAnd(inq + (v[k] >> 5), ~(1u << (v[k] & 31)));
                            if (lst[k] != d[k]) {
                                last[v[k]] = d[k];
                                out[k] = r1[k] - r0[k];
                            }
                        }
                    }
                    sum += out[k];
                }
                int ndef = 0;
#pragma unroll
                for (int k = 0; k < PA; ++k) {
                    // deferred entries of a warp mostly share one bin: one atomic then
                    const int bin = defer[k] ? band_bin(d[k], base_i, is_float_a, inv_unit) : -1;
                    const int bin0 = __shfl_sync(0xffffffffu, bin, 0);
                    if (__all_sync(0xffffffffu, bin == bin0)) {
                        const unsigned tot =
                            __reduce_add_sync(0xffffffffu, static_cast<unsigned>(min(r1[k] - r0[k], 1 << 26)));
                        if (bin0 >= 0 && (threadIdx.x & 31) == 0)
                            atomicAdd(&sh.hist[bin0], static_cast<unsigned long long>(tot));
                    } else if (defer[k]) {
                        atomicAdd(&sh.hist[bin], static_cast<unsigned long long>(r1[k] - r0[k]));
                    }
                    const int mn = __reduce_min_sync(0xffffffffu, defer[k] ? d[k] : 0x7fffffff);
                    if (mn != 0x7fffffff && (threadIdx.x & 31) == 0) atomicMin(&sh.hmin, mn);
                    ndef += defer[k] ? 1 : 0;
                }
                // one scan carries both the edge count (high half) and the deferred count
                // (low half, at most kBlock * PA per step, so it never carries over)
                const unsigned long long packed =
                    (static_cast<unsigned long long>(sum) << 32) | static_cast<unsigned>(ndef);
                const unsigned long long incl = block_inclusive_scan_u64<kBlock>(packed, sh.scan);
                const unsigned long long excl = incl - packed;
                const unsigned long long total = sh.scan[32];
                if (threadIdx.x == 0 && static_cast<unsigned>(total) != 0u)
                    sh.dbase = atomicAdd(qlen_next, static_cast<int>(static_cast<unsigned>(total)));
                __syncthreads();
                int run = carry + static_cast<int>(excl >> 32);
                int dpos = sh.dbase + static_cast<int>(static_cast<unsigned>(excl));
#pragma unroll
                for (int k = 0; k < PA; ++k) {
                    if (valid[k]) a.buf.loc_off[i0 + k] = run;
                    run += out[k];
                    if (defer[k]) qn[dpos++] = v[k];
                }
                carry += static_cast<int>(total >> 32);
                __syncthreads();  // sh.scan and sh.dbase are reused by the next step
            }
            if (threadIdx.x == 0) a.buf.chunk_sum[vg.id] = carry;
        }
        if (!grid_barrier(a.ctl, a.sticky, kSiteSsspBarA, vg)) return;
        // every block has read this queue's length, base and histogram: reset them for the
        // iteration that fills this queue next
        if (gtid < kBandBins) a.ctl->shist[cur][gtid] = 0ull;
        if (gtid == 0) {
            a.ctl->qlen[cur] = 0;
            a.ctl->sbase[cur] = INF;
        }

        const int E = frontier_chunk_bases<kBlock>(a.buf.chunk_sum, sm.base, sm.scan_tmp, vg);
        expanded += E;
        ++iters;
        const int *col = a.col_ind;
        const int *wt = a.w;
        const int *rp = a.row_ptr;
        TravCtl *ctl = a.ctl;
        int *sticky = a.sticky;
        int *flen = &a.ctl->flen[fc];
        const double T = thresh;
        const int is_float = a.is_float;
        WQ wn(sm.qbuf[threadIdx.x >> 5][0], qn, qlen_next);
        WQ wf(sm.qbuf[threadIdx.x >> 5][1], fcur, flen);
        auto relax = [&](const bool (&valid)[kSsspVT], const int (&kk)[kSsspVT], const int (&idx)[kSsspVT],
                         auto &ws) {
                constexpr int kVT = kSsspVT;
                int v[kVT], we[kVT], cd[kVT], nd[kVT];
                bool imp[kVT];
#pragma unroll
                for (int r = 0; r < kVT; ++r) {
                    v[r] = valid[r] ? __ldg(col + idx[r]) : 0;
                    we[r] = valid[r] ? __ldg(wt + idx[r]) : 0;
                }
                // plain (L1-cacheable) reads: a stale, larger value only costs an extra atomic
#pragma unroll
                for (int r = 0; r < kVT; ++r)
                    cd[r] = (valid[r] && APSPIE_SSSP_PREREAD) ? (APSPIE_SSSP_RED ? __ldcg(dist + v[r]) : dist[v[r]]) : INF;
#pragma unroll
                for (int r = 0; r < kVT; ++r) {
                    imp[r] = false;
                    nd[r] = 0;
                    if (!valid[r]) continue;
                    if (is_float) {
                        const float wf = __int_as_float(we[r]);
                        if (!(wf >= 0.0f)) {  // negative or NaN
                            raise_error(ctl, sticky, APSPIE_ERR_INVALID_ARG, kSiteSsspNegWeight);
                        } else {
                            nd[r] = __float_as_int(__fadd_rn(__int_as_float(ws.aux[kk[r]]), wf));
                            imp[r] = nd[r] < cd[r];
                        }
                        continue;
                    }
                    const long long d = static_cast<long long>(ws.aux[kk[r]]) + we[r];
                    if (we[r] < 0) {
                        raise_error(ctl, sticky, APSPIE_ERR_INVALID_ARG, kSiteSsspNegWeight);
                    } else if (d >= kInf) {
                        raise_error(ctl, sticky, APSPIE_ERR_INVALID_ARG, kSiteSsspOverflow);
                    } else {
                        nd[r] = static_cast<int>(d);
                        imp[r] = nd[r] < cd[r];
                    }
                }
                bool got[kVT];  // the relaxation lowered v's distance
#pragma unroll
                for (int r = 0; r < kVT; ++r) {
                    if (APSPIE_SSSP_RED) {
                        if (imp[r]) atomicMin(dist + v[r], nd[r]);
                        got[r] = imp[r];
                    } else {
                        got[r] = imp[r] && nd[r] < atomicMin(dist + v[r], nd[r]);
                    }
                }
                bool near[kVT], far[kVT];
#pragma unroll
                for (int r = 0; r < kVT; ++r) {
                    near[r] = far[r] = false;
                    if (got[r]) {
                        const unsigned bit = 1u << (v[r] & 31);
                        const double ndv = is_float ? static_cast<double>(__int_as_float(nd[r]))
                                                    : static_cast<double>(nd[r]);
                        if (ndv < T)
                            near[r] = !(atomicOr(inq + (v[r] >> 5), bit) & bit);
                        else
                            far[r] = !(atomicOr(infar + (v[r] >> 5), bit) & bit);
                    }
                }
                if (banded) {
                    // every improvement below T (queued now or already) enters the next
                    // band histogram at its new distance (improvements are a few percent of
                    // the relaxations, so plain shared-memory atomics rarely collide)
                    bool rec[kVT];
                    int dg[kVT];
#pragma unroll
                    for (int r = 0; r < kVT; ++r) {
                        rec[r] = got[r] &&
                                 (is_float ? static_cast<double>(__int_as_float(nd[r]))
                                           : static_cast<double>(nd[r])) < T;
                        dg[r] = rec[r] ? __ldg(rp + v[r] + 1) - __ldg(rp + v[r]) : 0;
                    }
#pragma unroll
                    for (int r = 0; r < kVT; ++r) {
                        if (!rec[r]) continue;
                        atomicAdd(&sh.hist[band_bin(nd[r], base_i, is_float, inv_unit)],
                                  static_cast<unsigned long long>(dg[r]));
                        atomicMin(&sh.hmin, nd[r]);
                    }
                }
#pragma unroll
                for (int r = 0; r < kVT; ++r) {
                    wn.push(near[r], v[r]);
                    wf.push(far[r], v[r]);
                }
            };
        frontier_expand<kBlock, kSsspVT, false>(
            nf, E, a.buf.loc_off, a.buf.rs, sm, [&](int jj, int k, SsspSlice &w) { w.aux[k] = __ldcg(snap + jj); },
            relax, NoPost(), vg);
        wn.flush();
        wf.flush();
        if (banded) {
            __syncthreads();
            const unsigned long long hv = sh.hist[threadIdx.x];
            if (hv) {
                atomicAdd(&a.ctl->shist[cur ^ 1][threadIdx.x], hv);
                sh.hist[threadIdx.x] = 0ull;
            }
            if (threadIdx.x == 0 && sh.hmin != INF) {
                atomicMin(&a.ctl->sbase[cur ^ 1], sh.hmin);
                sh.hmin = INF;
            }
        }
        if (!grid_barrier(a.ctl, a.sticky, kSiteSsspBarB, vg)) return;
        cur ^= 1;
    }
    // unreached -> -1, and the component statistics
    long long comp = 0, reached = 0;
    for (int i = gtid; i < m; i += gstride) {
        const int d = a.dist[i];
        if (d == INF) {
            a.dist[i] = a.unreached_bits;
        } else {
            comp += __ldg(a.row_ptr + i + 1) - __ldg(a.row_ptr + i);
            ++reached;
        }
    }
    for (int o = 16; o; o >>= 1) {
        comp += __shfl_down_sync(0xffffffffu, comp, o);
        reached += __shfl_down_sync(0xffffffffu, reached, o);
    }
    if ((threadIdx.x & 31) == 0 && (comp || reached)) {
        atomicAdd(reinterpret_cast<unsigned long long *>(&a.ctl->edges_component),
                  static_cast<unsigned long long>(comp));
        atomicAdd(reinterpret_cast<unsigned long long *>(&a.ctl->vertices_reached),
                  static_cast<unsigned long long>(reached));
    }
    if (gtid == 0) {
        a.ctl->iterations = iters;
        a.ctl->push_iterations = iters;
        a.ctl->pull_iterations = steps - 1 - iters;  // threshold advances
        a.ctl->edges_expanded = expanded;
        a.ctl->delta = delta < 2147483647.0 ? static_cast<int>(delta) : 0;  // 0: no far pile
    }
}

__global__ void __launch_bounds__(kBlock, APSPIE_SSSP_MINB) sssp_kernel(SsspArgs a) { sssp_body(a, hw_grid()); }

// Many sources in one launch: the grid splits into `groups` equal groups of blocks, each
// with its own control block and scratch, and each group runs the single-source SSSP
// above on queries grp, grp + groups, ... in turn, synchronising only among its own
// blocks. Every answer is the single-source kernel's answer; the queries of different
// groups run side by side, which pays because one query alone keeps the device
// latency-bound (few warps issue at a time).
struct SsspGroupArgs {
    SsspArgs base;       // graph, weights, band, sticky word; per query: src, dist, ctl, buf
    const int *srcs;
    int *out;            // nq x m, query-major
    int nq, groups, m;
    TravCtl *ctls;       // one control block per group
    size_t buf_stride;   // bytes between consecutive groups' scratch (base.buf is group 0's)
    TravCtl *main;       // the context's control block: errors and summed statistics
};

__device__ __forceinline__ TravBuffers shift_buffers(TravBuffers b, size_t off) {
    auto sh = [off](auto *p) { return reinterpret_cast<decltype(p)>(reinterpret_cast<char *>(p) + off); };
    b.q0 = sh(b.q0);
    b.q1 = sh(b.q1);
    b.q2 = sh(b.q2);
    b.q3 = sh(b.q3);
    b.rs = sh(b.rs);
    b.loc_off = sh(b.loc_off);
    b.chunk_sum = sh(b.chunk_sum);
    b.aux = sh(b.aux);
    b.aux2 = sh(b.aux2);
    b.bits0 = sh(b.bits0);
    b.bits1 = sh(b.bits1);
    b.bits2 = sh(b.bits2);
    return b;
}

__global__ void __launch_bounds__(kBlock, APSPIE_SSSP_MINB) sssp_group_kernel(SsspGroupArgs g) {
    const int bpg = static_cast<int>(gridDim.x) / g.groups;  // the host launches groups * bpg blocks
    const int grp = static_cast<int>(blockIdx.x) / bpg;
    const VGrid vg{static_cast<int>(blockIdx.x) - grp * bpg, bpg};
    TravCtl *ctl = g.ctls + grp;
    SsspArgs a = g.base;
    a.ctl = ctl;
    a.buf = shift_buffers(g.base.buf, g.buf_stride * grp);
    const int tid = vg.id * kBlock + static_cast<int>(threadIdx.x);
    for (int q = grp; q < g.nq; q += g.groups) {
        a.src = __ldg(g.srcs + q);
        if (a.src < 0 || a.src >= g.m) {
            // every block of the group reads the same source and skips the query alike
            if (tid == 0) raise_error(g.main, a.sticky, APSPIE_ERR_INVALID_ARG, kSiteSsspBadSource);
            continue;
        }
        a.dist = g.out + static_cast<size_t>(q) * g.m;
        sssp_body(a, vg);
        // every block of the group is done with the control block before it is reset
        if (!grid_barrier(ctl, a.sticky, kSiteSsspGroup, vg)) break;
        if (tid == 0) {
            atomicAdd(reinterpret_cast<unsigned long long *>(&g.main->edges_expanded),
                      static_cast<unsigned long long>(ctl->edges_expanded));
            atomicAdd(reinterpret_cast<unsigned long long *>(&g.main->edges_component),
                      static_cast<unsigned long long>(ctl->edges_component));
            atomicAdd(reinterpret_cast<unsigned long long *>(&g.main->vertices_reached),
                      static_cast<unsigned long long>(ctl->vertices_reached));
            atomicAdd(&g.main->iterations, ctl->iterations);
            atomicAdd(&g.main->push_iterations, ctl->push_iterations);
            ctl->edges_component = 0;
            ctl->vertices_reached = 0;
            for (int k = 0; k < 4; ++k) ctl->aux[k] = 0;
        }
        for (int k = tid; k < 2 * kBandBins; k += vg.n * kBlock) ctl->shist[k / kBandBins][k % kBandBins] = 0ull;
        if (!grid_barrier(ctl, a.sticky, kSiteSsspGroup + 1, vg)) break;
    }
    if (tid == 0 && ctl->err != 0) raise_error(g.main, a.sticky, ctl->err, ctl->err_where);
}

// ================================================================================
// MIS
// ================================================================================
enum : unsigned char { kUndecided = 0, kIn = 1, kOut = 2 };
#ifndef APSPIE_MIS_THREAD
#define APSPIE_MIS_THREAD 16
#endif
#ifndef APSPIE_MIS_WARP_CHUNKS
#define APSPIE_MIS_WARP_CHUNKS 8
#endif
constexpr int kMisThread = APSPIE_MIS_THREAD;          // neighbours one thread scans (phase S) before handing on
constexpr int kMisWarpChunks = APSPIE_MIS_WARP_CHUNKS;  // chunks of 32 neighbours a warp scans (phase L)
constexpr int kMisLightRow = 64;   // joiners with at most this many neighbours push by one thread

struct MisArgs {
    int m, nnz;
    const int *__restrict__ row_ptr;
    const int *__restrict__ col_ind;
    const unsigned *__restrict__ prio;
    unsigned char *member;
    int *member_i32;  // when set, the set is written here as int32 1/0 instead
    unsigned char *state;
    int *pos;          // CSR index of the outranking neighbour that blocks the vertex (row start - 1: none yet)
    int *queue[2];     // undecided vertices, by round parity
    int *longq;        // scans that go on past a thread's share (one warp each, phase L)
    int *longq2;       // scans that go on past a warp's share (one block each, phase L2)
    int *light;        // vertices that joined with rows of at most kMisLightRow (pushed next round)
    int *heavy_v;      // vertices that joined with longer rows,
    int *heavy_base;   // the offset of each one's row in the next round's flat range of pushes,
    int *heavy_delta;  // and row start - offset (push t of the range is CSR entry t + delta)
    int *unit_owner;   // the heavy entry holding the first push of each unit of the range
    int unit_shift;    // units of 1 << unit_shift pushes (one warp each)
    TravCtl *ctl;
    int *sticky;
};

__device__ __forceinline__ bool outranks(unsigned pu, int u, unsigned pv, int v) {
    return pu > pv || (pu == pv && u > v);
}

// A neighbour's state as a scan reads it: through L1, so the lines of high-degree
// neighbours (read by many scans at once) are not all fetched from L2. A stale value is
// safe: states only move from undecided to in or out, so a stale read can only make a scan
// stop early at a neighbour that is already out, and the next round's blocker check (a
// coherent read) sees it out and resumes the scan behind it.
#ifndef APSPIE_MIS_STATE_STRIDE
#define APSPIE_MIS_STATE_STRIDE 1
#endif
constexpr int kMisStateStride = APSPIE_MIS_STATE_STRIDE;  // bytes between consecutive vertices' states
__device__ __forceinline__ long long sx(int v) { return static_cast<long long>(v) * kMisStateStride; }
__device__ __forceinline__ unsigned char scan_state(const unsigned char *state, int u) { return state[sx(u)]; }

// One neighbour of a scanning vertex v: does it decide anything (an outranking neighbour
// that is not out: v's new blocker, or -- if in -- the vertex that knocks v out)?
__device__ __forceinline__ bool mis_stop(const MisArgs &a, int idx, int v, unsigned pv) {
    const int u = __ldg(a.col_ind + idx);
    const unsigned pu = __ldg(a.prio + u);
    const unsigned char su = scan_state(a.state, u);
    return u != v && su != kOut && outranks(pu, u, pv, v);
}

// Knock out neighbour u of a vertex that joined. Many joiners share their high-degree
// neighbours, and stores from many SMs into one line queue up in L2, so (check) a neighbour
// already seen out (through L1: a stale "undecided" only costs a redundant store) is
// skipped. In the first push round nothing is out yet.
__device__ __forceinline__ void mis_knock(const MisArgs &a, int u, bool check) {
    if (!check || scan_state(a.state, u) != kOut) a.state[sx(u)] = kOut;
}

// v joined with a row [r0, r0 + deg) longer than kMisLightRow: list it for the next
// round's pushes. One atomic on (entries << 32 | pushes) gives the entry index and the
// row's offset in the flat range, so offsets ascend with the index; the units starting
// inside the row record it.
__device__ __forceinline__ void mis_list_heavy(const MisArgs &a, unsigned long long *heavy, int v, int r0, int deg) {
    const unsigned long long old = atomicAdd(heavy, (1ull << 32) | static_cast<unsigned>(deg));
    const int idx = static_cast<int>(old >> 32);
    const int base = static_cast<int>(old & 0xffffffffull);
    a.heavy_v[idx] = v;
    a.heavy_base[idx] = base;
    a.heavy_delta[idx] = r0 - base;
    const int sh = a.unit_shift;
    for (int c = ((base - 1) >> sh) + 1; (c << sh) < base + deg; ++c) a.unit_owner[c] = idx;
}

// Greedy MIS in descending (priority, id) order -- the set spmspvMis converges to
// (src/spmspvMis.cuh:54-78: candidate if rand > threshold, select if rand > every
// candidate neighbour's, knock out the neighbours), with ties broken by id instead of
// left undecided. A vertex joins exactly when every neighbour that outranks it is out;
// it is out as soon as a neighbour joins.
//
// Only outranking neighbours can ever decide a vertex (a lower-ranked neighbour cannot
// join while the vertex is undecided), and a neighbour once seen out or lower-ranked
// stays so. So each undecided vertex keeps a scan position `pos`: every neighbour before
// it is settled, and the neighbour at it is its current blocker (undecided, outranking).
// Each scan stops at the first neighbour that decides anything, so rows are read about
// once over the whole run and mostly not to their end (about 6.8M of R-MAT scale 20's
// 31.4M entries). Round r, over the undecided vertices (round 0: all of them, which also
// sets every state; vertices without neighbours join there) and the vertices that joined
// in round r - 1:
//  phase P  (when anything joined) the joiners write out into their neighbours: rows of at
//           most kMisLightRow one thread each; longer rows, laid end to end in the order
//           they were listed, in equal units of 1 << unit_shift entries, one warp each.
//           Only stores (and L1 reads): on the B200 a phase in which many SMs both store
//           into and read the lines of high-degree vertices' states runs several times
//           slower, so the pushes are not made by the joining threads during the scans;
//  phase S  each undecided vertex, by one thread: out -> leaves; its blocker still
//           undecided (or in: its push comes next round) -> waits; else it scans on, four
//           neighbours a step, and stops at the first neighbour that outranks it and is not
//           out (its new blocker); no such neighbour -> it joins and is listed for the next
//           round's pushes. After kMisThread neighbours without an end the vertex goes to
//           the long list;
//  phase L  (only when that list is not empty) one warp per vertex goes on in chunks of
//           32, for up to kMisWarpChunks chunks; the rest (phase L2) one block each.
// The pushes of a round are complete before its scans start, so a scan sees every vertex
// knocked out so far; scans and joins of the same phase race only safely (a vertex joins
// only if every outranking neighbour was seen out, and out is final). The set is the
// greedy MIS whatever the timing.
//
// The lists a round fills (long lists and joiners in slot r mod 3 of the control block's
// round counters, the next queue in slot r + 1) are cleared by the round before: their
// last readers finished a full round earlier, so no block can still be reading them.
__global__ void __launch_bounds__(kBlock) mis_kernel(MisArgs a) {
    __shared__ int qbuf[kBlock / 32][3][BfsSmem::QCAP];
    __shared__ int s_stop;
    timeline_mark(a.ctl, 0);
    const int G = gridDim.x;
    const int gtid = blockIdx.x * kBlock + threadIdx.x;
    const int gstride = G * kBlock;
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int m = a.m;
    const int *col = a.col_ind;
    unsigned char *state = a.state;
    int *qlen = a.ctl->rcnt;                   // [3] undecided-queue lengths
    int *l1len = a.ctl->rcnt + 3;              // [3] long list (phase L)
    int *l2len = a.ctl->rcnt + 6;              // [3] longest list (phase L2)
    int *nlight = a.ctl->rcnt + 9;             // [3] light joiners
    unsigned long long *heavy = a.ctl->rcnt64;  // [3] (entries << 32) | pushes of heavy joiners
    long long pushed = 0, scanned = 0;
    int r = 0;
    for (;; ++r) {
        const int s0 = r % 3, s1 = (r + 1) % 3, s2 = (r + 2) % 3;
        const int sp = (r + 2) % 3;  // the joiner lists of round r - 1
        const int nf = r == 0 ? m : ld_volatile_i32(qlen + s0);  // round 0: every vertex
        const int nl = ld_volatile_i32(nlight + sp);
        const unsigned long long hh = __ldcg(reinterpret_cast<const unsigned long long *>(heavy + sp));
        const int nh = static_cast<int>(hh >> 32);
        const int H = static_cast<int>(hh & 0xffffffffull);
        const int sh = a.unit_shift;
        const int nu = H > 0 ? ((H - 1) >> sh) + 1 : 0;
        if (nf == 0 && nl == 0 && nu == 0) break;
        if (r > m + 1) {
            if (gtid == 0) raise_error(a.ctl, a.sticky, APSPIE_ERR_NOT_CONVERGED, kSiteMisRoundCap);
            break;
        }
        const int *qc = a.queue[r & 1];
        int *qn = a.queue[(r & 1) ^ 1];

        // phase P: the last round's joiners knock out their neighbours -- short rows one
        // thread each, long rows laid end to end and shared out in equal units, one warp
        // each. Plain byte stores: every neighbour of a vertex in the set is out.
        if (nl > 0 || nu > 0) {
            // skipping known outs pays when many joiners share neighbours; with few of them
            // the read before each store only lengthens the chain
            const bool check = r >= 2 && nl + nh >= 4096;
            // lanes per joiner: 1 when the joiners fill the grid, up to 8 when they are few,
            // so that a short round's rows are not walked one entry at a time by one thread
            int lpj = 1;
            while (lpj < 8 && static_cast<long long>(nl) * lpj * 2 <= gstride) lpj <<= 1;
            const int sub = gtid & (lpj - 1);
            for (int i = gtid / lpj; i < nl; i += gstride / lpj) {
                const int j = __ldcg(a.light + i);
                const int r0 = __ldg(a.row_ptr + j), r1 = __ldg(a.row_ptr + j + 1);
                if (sub == 0) pushed += r1 - r0;
                for (int e = r0 + sub; e < r1; e += 8 * lpj) {
                    int u[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) u[k] = e + k * lpj < r1 ? __ldg(col + e + k * lpj) : j;
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        if (u[k] != j) mis_knock(a, u[k], check);
                }
            }
            const int gw = gtid >> 5, nw = gstride >> 5;
            for (int c = gw; c < nu; c += nw) {
                // a unit spans the end of one row and the start of the next where rows meet in it
                const int t0 = c << sh, t1 = min(H, t0 + (1 << sh));
                int i = __ldcg(a.unit_owner + c);
                int hv = __ldcg(a.heavy_v + i), hd = __ldcg(a.heavy_delta + i);
                int nb = i + 1 < nh ? __ldcg(a.heavy_base + i + 1) : INT_MAX;
                if (lane == 0) pushed += t1 - t0;
                for (int tb = t0; tb < t1; tb += 128) {
                    int e[4], w[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int t = tb + 32 * q + lane;
                        while (t < t1 && t >= nb) {
                            ++i;
                            hv = __ldcg(a.heavy_v + i);
                            hd = __ldcg(a.heavy_delta + i);
                            nb = i + 1 < nh ? __ldcg(a.heavy_base + i + 1) : INT_MAX;
                        }
                        e[q] = t < t1 ? t + hd : -1;
                        w[q] = hv;
                    }
                    int u[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) u[q] = e[q] >= 0 ? __ldg(col + e[q]) : -1;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (u[q] >= 0 && u[q] != w[q]) mis_knock(a, u[q], check);
                }
            }
            if (!grid_barrier(a.ctl, a.sticky, kSiteMis + 2)) return;
        }
        // the lists this round fills start empty; their slots were last read a round ago
        if (gtid == 0) {
            qlen[s2] = 0;
            l1len[s1] = 0;
            l2len[s1] = 0;
            nlight[s1] = 0;
            heavy[s1] = 0ull;
        }

        // phase S: blocker checks, short scans and decisions, one thread per vertex; each
        // scan step loads four neighbours at once and takes the first that decides anything
        {
            WQ wq(qbuf[wid][0], qn, qlen + s1);
            WQ wj(qbuf[wid][1], a.light, nlight + s0);
            WQ wl(qbuf[wid][2], a.longq, l1len + s0);
            for (int base = blockIdx.x * kBlock; base < nf; base += gstride) {
                const int i = base + threadIdx.x;
                bool keep = false, light = false, along = false;
                int v = 0;
                if (i < nf) {
                    // round 0 takes every vertex and writes every state: vertices without
                    // neighbours join at once, the others start undecided with no blocker
                    v = r == 0 ? i : __ldcg(qc + i);
                    const int r0 = __ldg(a.row_ptr + v), r1 = __ldg(a.row_ptr + v + 1);
                    if (r == 0 && r1 == r0) {
                        state[sx(v)] = kIn;
                    } else if (r == 0 || __ldcg(state + sx(v)) == kUndecided) {
                        const int p = r == 0 ? r0 - 1 : __ldcg(a.pos + v);
                        if (r == 0) state[sx(v)] = kUndecided;
                        if (p >= r0 && __ldcg(state + sx(__ldg(col + p))) != kOut) {
                            keep = true;  // its blocker is undecided (or joined: its push comes next)
                        } else {
                            const unsigned pv = __ldg(a.prio + v);
                            const int start = p + 1, lim = min(r1, start + kMisThread);
                            int stop = -1, e = start;
                            for (; e < lim && stop < 0; e += 4) {
                                int u[4];
                                unsigned pu[4];
                                unsigned char su[4];
#pragma unroll
                                for (int k = 0; k < 4; ++k) u[k] = e + k < lim ? __ldg(col + e + k) : v;
#pragma unroll
                                for (int k = 0; k < 4; ++k) {
                                    pu[k] = __ldg(a.prio + u[k]);
                                    // in the first round every vertex with neighbours is undecided
                                    su[k] = r == 0 ? kUndecided : scan_state(state, u[k]);
                                }
#pragma unroll
                                for (int k = 0; k < 4; ++k)
                                    if (stop < 0 && u[k] != v && su[k] != kOut && outranks(pu[k], u[k], pv, v))
                                        stop = e + k;
                            }
                            scanned += (stop >= 0 ? stop + 1 : lim) - start;
                            if (stop >= 0) {
                                keep = true;
                                a.pos[v] = stop;
                            } else if (lim >= r1) {
                                state[sx(v)] = kIn;
                                light = r1 - r0 <= kMisLightRow;
                                if (!light) mis_list_heavy(a, heavy + s0, v, r0, r1 - r0);
                            } else {  // settled up to lim - 1: a warp goes on
                                a.pos[v] = lim - 1;
                                along = true;
                            }
                        }
                    }
                }
                wq.push(keep, v);
                wj.push(light, v);
                wl.push(along, v);
            }
            wq.flush();
            wj.flush();
            wl.flush();
        }
        if (!grid_barrier(a.ctl, a.sticky, kSiteMis + 3)) return;

        // phase L: longer scans, one warp per vertex (up to kMisWarpChunks chunks of 32)
        const int n1 = ld_volatile_i32(l1len + s0);
        if (n1 > 0) {
            WQ wq(qbuf[wid][0], qn, qlen + s1);
            WQ wj(qbuf[wid][1], a.light, nlight + s0);
            const int gw = gtid >> 5, nw = gstride >> 5;
            for (int k = gw; k < n1; k += nw) {
                const int v = __ldcg(a.longq + k);
                const int r1 = __ldg(a.row_ptr + v + 1);
                const int start = __ldcg(a.pos + v) + 1;
                const unsigned pv = __ldg(a.prio + v);
                int stop = -1, c = 0;
                for (; c < kMisWarpChunks && start + 32 * c < r1; ++c) {
                    const int idx = start + 32 * c + lane;
                    const unsigned b = __ballot_sync(0xffffffffu, idx < r1 && mis_stop(a, idx, v, pv));
                    if (b) {
                        stop = start + 32 * c + __ffs(b) - 1;
                        break;
                    }
                }
                const bool end = stop < 0 && start + 32 * c >= r1;
                bool light = false;
                if (lane == 0) {
                    scanned += min(r1, stop >= 0 ? stop + 1 : start + 32 * c) - start;
                    if (stop >= 0) {
                        a.pos[v] = stop;
                    } else if (end) {
                        state[sx(v)] = kIn;
                        const int r0 = __ldg(a.row_ptr + v);
                        light = r1 - r0 <= kMisLightRow;
                        if (!light) mis_list_heavy(a, heavy + s0, v, r0, r1 - r0);
                    } else {
                        a.pos[v] = start + 32 * kMisWarpChunks - 1;
                        a.longq2[atomicAdd(l2len + s0, 1)] = v;
                    }
                }
                wq.push(stop >= 0 && lane == 0, v);
                wj.push(light, v);
            }
            wq.flush();
            wj.flush();
            if (!grid_barrier(a.ctl, a.sticky, kSiteMis + 4)) return;
        }

        // phase L2: the longest scans, one block per vertex
        const int n2 = n1 > 0 ? ld_volatile_i32(l2len + s0) : 0;
        if (n2 > 0) {
            for (int k = blockIdx.x; k < n2; k += G) {
                const int v = __ldcg(a.longq2 + k);
                const int r1 = __ldg(a.row_ptr + v + 1);
                const int start = __ldcg(a.pos + v) + 1;
                const unsigned pv = __ldg(a.prio + v);
                if (threadIdx.x == 0) s_stop = kInf;
                __syncthreads();
                for (int b0 = start; b0 < r1; b0 += kBlock) {
                    const int idx = b0 + threadIdx.x;
                    const bool st = idx < r1 && mis_stop(a, idx, v, pv);
                    if (st) atomicMin(&s_stop, idx);
                    if (__syncthreads_or(st)) break;
                }
                if (threadIdx.x == 0) {
                    const int spos = s_stop;
                    scanned += (spos != kInf ? spos + 1 : r1) - start;
                    if (spos != kInf) {
                        a.pos[v] = spos;
                        qn[atomicAdd(qlen + s1, 1)] = v;
                    } else {
                        state[sx(v)] = kIn;
                        const int r0 = __ldg(a.row_ptr + v);
                        if (r1 - r0 <= kMisLightRow)
                            a.light[atomicAdd(nlight + s0, 1)] = v;
                        else
                            mis_list_heavy(a, heavy + s0, v, r0, r1 - r0);
                    }
                }
                __syncthreads();
            }
            if (!grid_barrier(a.ctl, a.sticky, kSiteMis + 5)) return;
        }
    }
    long long insz = 0;
    for (int i = gtid; i < m; i += gstride) {
        const unsigned char s = a.state[sx(i)];
        if (a.member_i32)
            a.member_i32[i] = (s == kIn) ? 1 : 0;
        else
            a.member[i] = (s == kIn) ? 1 : 0;
        insz += (s == kIn);
    }
    long long work = scanned + pushed;
    for (int o = 16; o; o >>= 1) {
        insz += __shfl_down_sync(0xffffffffu, insz, o);
        work += __shfl_down_sync(0xffffffffu, work, o);
    }
    if (lane == 0 && insz)
        atomicAdd(reinterpret_cast<unsigned long long *>(&a.ctl->vertices_reached),
                  static_cast<unsigned long long>(insz));
    if (lane == 0 && work)
        atomicAdd(reinterpret_cast<unsigned long long *>(&a.ctl->edges_expanded),
                  static_cast<unsigned long long>(work));
    if (gtid == 0) {
        a.ctl->iterations = r;
        a.ctl->push_iterations = r;
        a.ctl->edges_component = a.nnz;
    }
}

// ================================================================================
// one-hop boolean SpMSpV (MIS validity helper)
// ================================================================================
__global__ void spmspv_bool_kernel(int m, const int *__restrict__ row_ptr,
                                   const int *__restrict__ col_ind, const int *__restrict__ x,
                                   int *y) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int u = warp; u < m; u += nwarps) {
        if (__ldg(x + u) == 0) continue;
        const int r0 = __ldg(row_ptr + u), r1 = __ldg(row_ptr + u + 1);
        for (int e = r0 + lane; e < r1; e += 32) y[__ldg(col_ind + e)] = 1;
    }
}

apspie_status prepare_square(apspie_ctx *ctx, const apspie_csr *A, const char *who) {
    apspie_status st = check_csr_view(ctx, A, who);
    if (st != APSPIE_OK) return st;
    if (A->m != A->n)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": matrix must be square");
    if (A->m <= 0) return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string(who) + ": empty graph");
    if (ctx->validate) {
        st = validate_csr(ctx, A, true);
        if (st != APSPIE_OK) return st;
    }
    return APSPIE_OK;
}


}  // namespace

// ================================================================================
// Allocation-free BFS: scratch in a file-scope device array
// ================================================================================
namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kNaMaxV = APSPIE_NOALLOC_MAX_VERTICES;
constexpr size_t kNaQueueBytes = align256((kNaMaxV + 1) * sizeof(int));
constexpr size_t kNaWordsBytes = align256(((kNaMaxV + 31) / 32) * sizeof(unsigned));
constexpr size_t kNaCtlBytes = align256(sizeof(TravCtl)) + 256;  // control block + sticky error word
constexpr size_t kNaBytes =
    kNaCtlBytes + 4 * kNaQueueBytes + align256(kMaxGrid * sizeof(int)) + 3 * kNaWordsBytes;

// Shared by every apspie_bfs_noalloc call in the process (one copy per device). It keeps
// the last call's contents; the control block is cleared at the start of each call and the
// kernel initialises every queue and bitmap it reads.
static __device__ __align__(256) unsigned char g_bfs_noalloc_scratch[kNaBytes];

// A __device__ array has one address per CUDA context: the primary context of each device,
// any context a caller made with cuCtxCreate, and a primary context re-created after
// cudaDeviceReset each hold their own copy. The address is therefore looked up once per
// context and cached under the context's process-unique id (cuCtxGetId), never under a
// device number or a context handle, which a re-created context may reuse.
struct NaEntry {
    unsigned long long ctx_id;
    void *addr;
};
std::vector<NaEntry> g_na_cache;
std::mutex g_na_mu;

using CtxGetCurrentFn = int (*)(void **);              // cuCtxGetCurrent(CUcontext *)
using CtxGetIdFn = int (*)(void *, unsigned long long *);  // cuCtxGetId(CUcontext, id *)

// The id of the context current on this thread, or 0 when there is none or the driver
// cannot say (then the address is looked up on every call, which is always right).
unsigned long long current_ctx_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault) == cudaSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault) == cudaSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
        (void)cudaGetLastError();
    });
    void *c = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&c) != 0 || !c || get_id(c, &id) != 0) return 0;
    return id;
}

// Device address of g_bfs_noalloc_scratch in the current context, looked up (with
// cudaGetSymbolAddress, which also loads the library's device code into the context under
// lazy module loading) on the first call in each context.
cudaError_t noalloc_scratch(void **out) {
    std::lock_guard<std::mutex> lock(g_na_mu);
    unsigned long long id = current_ctx_id();
    if (id != 0)
        for (const NaEntry &e : g_na_cache)
            if (e.ctx_id == id) {
                *out = e.addr;
                return cudaSuccess;
            }
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_bfs_noalloc_scratch);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return e;
    }
    if (id == 0) id = current_ctx_id();  // the lookup may have made the primary context current
    if (id != 0) g_na_cache.push_back({id, p});
    *out = p;
    return cudaSuccess;
}

}  // namespace

size_t traversal_scratch_need(int m) { return trav_scratch_bytes(m); }

// what mis_common reserves: the traversal buffers, the state array, the push-unit owners
// and the list of light joiners
size_t mis_scratch_need(int m) {
    const size_t mi = static_cast<size_t>(m) + 1;
    return trav_scratch_bytes(m) + Carver::need({static_cast<size_t>(m) * kMisStateStride, mi * 4, mi * 4});
}

apspie_status trav_reserve(apspie_ctx *ctx, int m) {
    void *base;
    return scratch_reserve(ctx, std::max(trav_scratch_bytes(m) + static_cast<size_t>(m) * 5 + 512, mis_scratch_need(m)),
                           &base);
}

}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_ctx_reserve(apspie_ctx *ctx, int32_t m, int64_t nnz) {
    (void)nnz;
    if (!ctx || m < 0) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    return trav_reserve(ctx, m);
}

apspie_status apspie_bfs(apspie_ctx *ctx, const apspie_csr *A, int32_t source, int32_t depth_cap,
                         int32_t *d_depth, apspie_run_stats *stats) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = prepare_square(ctx, A, "apspie_bfs");
    if (st != APSPIE_OK) return st;
    if (source < 0 || source >= A->m)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_bfs: source out of range");
    if (!d_depth) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_bfs: NULL output");
    void *base;
    st = scratch_reserve(ctx, trav_scratch_bytes(A->m), &base);
    if (st != APSPIE_OK) return st;
    if ((st = reset_ctl(ctx)) != APSPIE_OK) return st;
    BfsArgs a;
    a.m = A->m;
    a.nnz = A->nnz;
    a.src = source;
    a.depth_cap = depth_cap;
    a.row_ptr = A->row_ptr;
    a.col_ind = A->col_ind;
    a.depth = d_depth;
    a.buf = carve_trav(base, A->m);
    a.ctl = ctx->d_ctl;
    a.sticky = ctx->d_sticky_err;
    const apspie_tune_params tp = effective_params(ctx, APSPIE_TUNE_BFS, A);
    a.alpha = tp.bfs_alpha;
    a.beta = tp.bfs_beta;
    a.allow_pull = (A->flags & APSPIE_CSR_SYMMETRIC) ? 1 : 0;
    void *args[] = {&a};
    st = launch_persistent(ctx, reinterpret_cast<const void *>(bfs_kernel), kBlock, args, A->nnz);
    if (st != APSPIE_OK) return st;
    return finish_call(ctx, stats, "apspie_bfs");
}

namespace apspie {
namespace {
apspie_status sssp_common(apspie_ctx *ctx, const apspie_csr *A, int32_t source, void *d_dist,
                          apspie_run_stats *stats, bool is_float, int unreached_bits);
}
}  // namespace apspie

apspie_status apspie_sssp(apspie_ctx *ctx, const apspie_csr *A, int32_t source, int32_t *d_dist,
                          apspie_run_stats *stats) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    if (A && A->val_type != APSPIE_VAL_I32)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp: int32 edge weights required");
    return sssp_common(ctx, A, source, d_dist, stats, false, -1);
}

apspie_status apspie_sssp_f32(apspie_ctx *ctx, const apspie_csr *A, int32_t source, float *d_dist,
                              float unreached, apspie_run_stats *stats) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    if (A && A->val_type != APSPIE_VAL_F32)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp_f32: float32 edge weights required");
    int bits;
    std::memcpy(&bits, &unreached, sizeof bits);
    return sssp_common(ctx, A, source, d_dist, stats, true, bits);
}

}  // extern "C"

namespace apspie {
namespace {
apspie_status sssp_common(apspie_ctx *ctx, const apspie_csr *A, int32_t source, void *d_dist,
                          apspie_run_stats *stats, bool is_float, int unreached_bits) {
    cudaSetDevice(ctx->device);
    apspie_status st = prepare_square(ctx, A, "apspie_sssp");
    if (st != APSPIE_OK) return st;
    if (A->nnz > 0 && !A->val) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp: NULL weights");
    if (source < 0 || source >= A->m)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp: source out of range");
    if (!d_dist) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_sssp: NULL output");
    void *base;
    st = scratch_reserve(ctx, trav_scratch_bytes(A->m), &base);
    if (st != APSPIE_OK) return st;
    if ((st = reset_ctl(ctx)) != APSPIE_OK) return st;
    SsspArgs a;
    a.m = A->m;
    a.nnz = A->nnz;
    a.src = source;
    a.row_ptr = A->row_ptr;
    a.col_ind = A->col_ind;
    a.w = static_cast<const int *>(A->val);
    a.dist = static_cast<int *>(d_dist);
    const apspie_tune_params tp = effective_params(ctx, APSPIE_TUNE_SSSP, A);
    a.delta_hint = tp.sssp_delta;
    if (tp.sssp_band > 0) {
        a.band = tp.sssp_band;
    } else if (tp.sssp_band == 0) {
        const long long b = A->nnz / 8;
        a.band = b < (1LL << 18) ? (1LL << 18) : (b > (1LL << 23) ? (1LL << 23) : b);
    } else {
        a.band = 0;
    }
    a.is_float = is_float ? 1 : 0;
    a.unreached_bits = unreached_bits;
    a.buf = carve_trav(base, A->m);
    a.ctl = ctx->d_ctl;
    a.sticky = ctx->d_sticky_err;
    void *args[] = {&a};
    st = launch_persistent(ctx, reinterpret_cast<const void *>(sssp_kernel), kBlock, args, A->nnz);
    if (st != APSPIE_OK) return st;
    return finish_call(ctx, stats, "apspie_sssp");
}
}  // namespace

size_t sssp_group_scratch_need(int m, int groups) {
    const size_t per = (trav_scratch_bytes(m) + 255) / 256 * 256;
    return per * static_cast<size_t>(groups) + static_cast<size_t>(groups) * ((sizeof(TravCtl) + 255) / 256 * 256);
}

int sssp_group_count(const apspie_ctx *ctx, int nq) {
    int g = ctx->sssp_batch_groups > 0 ? ctx->sssp_batch_groups : 4;
    return std::max(1, std::min(g, nq));
}

apspie_status sssp_batch_grouped(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources, int32_t nq,
                                 int32_t *d_dists, apspie_run_stats *stats) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (nq == 0) return APSPIE_OK;
    const int m = A->m;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, reinterpret_cast<const void *>(sssp_group_kernel), kBlock, 0);
    if (e != cudaSuccess || per_sm < 1) return cuda_error(ctx, e, "occupancy query");
    const int cap = persistent_cap(ctx, per_sm);
    const int groups = std::min(sssp_group_count(ctx, nq), cap);
    const int bpg = std::min(cap / groups, kMaxGrid);
    void *base;
    apspie_status st = scratch_reserve(ctx, sssp_group_scratch_need(m, groups), &base);
    if (st != APSPIE_OK) return st;
    if ((st = reset_ctl(ctx)) != APSPIE_OK) return st;
    const size_t per = (trav_scratch_bytes(m) + 255) / 256 * 256;
    TravCtl *ctls = reinterpret_cast<TravCtl *>(static_cast<char *>(base) + per * groups);
    if ((e = cudaMemsetAsync(ctls, 0, groups * ((sizeof(TravCtl) + 255) / 256 * 256), ctx->stream)) != cudaSuccess)
        return cuda_error(ctx, e, "apspie_sssp_batch reset");
    SsspGroupArgs g;
    SsspArgs &a = g.base;
    std::memset(&a, 0, sizeof(a));
    a.m = m;
    a.nnz = A->nnz;
    a.row_ptr = A->row_ptr;
    a.col_ind = A->col_ind;
    a.w = static_cast<const int *>(A->val);
    const apspie_tune_params tp = effective_params(ctx, APSPIE_TUNE_SSSP, A);
    a.delta_hint = tp.sssp_delta;
    if (tp.sssp_band > 0) {
        a.band = tp.sssp_band;
    } else if (tp.sssp_band == 0) {
        // the single-query default, scaled to the group's share of the device
        long long b = A->nnz / 8;
        b = b < (1LL << 18) ? (1LL << 18) : (b > (1LL << 23) ? (1LL << 23) : b);
        b = b * bpg / cap;
        a.band = b < (1LL << 16) ? (1LL << 16) : b;
    } else {
        a.band = 0;
    }
    a.is_float = 0;
    a.unreached_bits = -1;
    a.buf = carve_trav(base, m);
    a.sticky = ctx->d_sticky_err;
    g.srcs = d_sources;
    g.out = d_dists;
    g.nq = nq;
    g.groups = groups;
    g.m = m;
    g.ctls = ctls;
    g.buf_stride = per;
    g.main = ctx->d_ctl;
    void *args[] = {&g};
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(sssp_group_kernel), dim3(groups * bpg),
                                    dim3(kBlock), args, 0, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "cooperative launch");
    return finish_call(ctx, stats, "apspie_sssp_batch");
}

}  // namespace apspie

extern "C" {

static apspie_status mis_common(apspie_ctx *ctx, const apspie_csr *A, const uint32_t *d_priority,
                                uint8_t *d_member, int32_t *d_member_i32, apspie_run_stats *stats);

apspie_status apspie_mis(apspie_ctx *ctx, const apspie_csr *A, const uint32_t *d_priority,
                         uint8_t *d_member, apspie_run_stats *stats) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    if (!d_member) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_mis: NULL output");
    return mis_common(ctx, A, d_priority, d_member, nullptr, stats);
}

apspie_status apspie_mis_int32(apspie_ctx *ctx, const apspie_csr *A, const uint32_t *d_priority,
                               int32_t *d_mis_result, apspie_run_stats *stats) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    if (!d_mis_result) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_mis_int32: NULL output");
    return mis_common(ctx, A, d_priority, nullptr, d_mis_result, stats);
}

static apspie_status mis_common(apspie_ctx *ctx, const apspie_csr *A, const uint32_t *d_priority,
                                uint8_t *d_member, int32_t *d_member_i32, apspie_run_stats *stats) {
    cudaSetDevice(ctx->device);
    apspie_status st = prepare_square(ctx, A, "apspie_mis");
    if (st != APSPIE_OK) return st;
    if (!d_priority) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_mis: NULL priority");
    void *base;
    const size_t tb = trav_scratch_bytes(A->m);
    const size_t mi = static_cast<size_t>(A->m) + 1;
    st = scratch_reserve(ctx, mis_scratch_need(A->m), &base);
    if (st != APSPIE_OK) return st;
    if ((st = reset_ctl(ctx)) != APSPIE_OK) return st;
    MisArgs a;
    a.m = A->m;
    a.nnz = A->nnz;
    a.row_ptr = A->row_ptr;
    a.col_ind = A->col_ind;
    a.prio = d_priority;
    a.member = d_member;
    a.member_i32 = d_member_i32;
    const TravBuffers buf = carve_trav(base, A->m);
    a.pos = buf.aux;
    a.queue[0] = buf.q0;
    a.queue[1] = buf.q1;
    a.longq = buf.q2;
    a.longq2 = buf.aux2;
    a.heavy_v = buf.q3;
    a.heavy_base = buf.rs;
    a.heavy_delta = buf.loc_off;
    Carver c(static_cast<char *>(base) + tb);
    a.state = c.take<unsigned char>(static_cast<size_t>(A->m) * kMisStateStride);
    a.unit_owner = c.take<int>(mi);
    a.light = c.take<int>(mi);
    // push units hold at least 128 entries, and few enough that the units of a round's
    // pushes (at most nnz entries) fit the m + 1 slots of unit_owner
    a.unit_shift = 7;
    while ((static_cast<long long>(A->nnz) >> a.unit_shift) + 1 > static_cast<long long>(mi)) ++a.unit_shift;
    a.ctl = ctx->d_ctl;
    a.sticky = ctx->d_sticky_err;
    void *args[] = {&a};
    st = launch_persistent(ctx, reinterpret_cast<const void *>(mis_kernel), kBlock, args, A->nnz);
    if (st != APSPIE_OK) return st;
    return finish_call(ctx, stats, "apspie_mis");
}

apspie_status apspie_bfs_noalloc(const apspie_csr *A, int32_t source, int32_t depth_cap, int32_t *d_depth,
                                 void *cuda_stream, apspie_run_stats *stats) {
    if (!A || !d_depth || !A->row_ptr || (A->nnz > 0 && !A->col_ind) || A->m != A->n || A->m <= 0 ||
        A->nnz < 0)
        return APSPIE_ERR_INVALID_ARG;
    if (A->m > APSPIE_NOALLOC_MAX_VERTICES) return APSPIE_ERR_INVALID_ARG;  // beyond the static scratch
    if (source < 0 || source >= A->m) return APSPIE_ERR_INVALID_ARG;
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return APSPIE_ERR_CUDA;
    void *base = nullptr;
    if (noalloc_scratch(&base) != cudaSuccess) return APSPIE_ERR_CUDA;
    char *p = static_cast<char *>(base);
    TravCtl *ctl = reinterpret_cast<TravCtl *>(p);
    int *sticky = reinterpret_cast<int *>(p + align256(sizeof(TravCtl)));
    p += kNaCtlBytes;
    BfsArgs a;
    a.buf.q0 = reinterpret_cast<int *>(p);
    a.buf.q1 = reinterpret_cast<int *>(p + kNaQueueBytes);
    a.buf.rs = reinterpret_cast<int *>(p + 2 * kNaQueueBytes);
    a.buf.loc_off = reinterpret_cast<int *>(p + 3 * kNaQueueBytes);
    p += 4 * kNaQueueBytes;
    a.buf.chunk_sum = reinterpret_cast<int *>(p);
    p += align256(kMaxGrid * sizeof(int));
    a.buf.bits0 = reinterpret_cast<unsigned *>(p);
    a.buf.bits1 = reinterpret_cast<unsigned *>(p + kNaWordsBytes);
    a.buf.bits2 = reinterpret_cast<unsigned *>(p + 2 * kNaWordsBytes);
    a.buf.q2 = a.buf.q3 = a.buf.aux = a.buf.aux2 = nullptr;  // not used by BFS
    if (cudaMemsetAsync(ctl, 0, kNaCtlBytes, stream) != cudaSuccess) return APSPIE_ERR_CUDA;
    a.m = A->m;
    a.nnz = A->nnz;
    a.src = source;
    a.depth_cap = depth_cap;
    a.row_ptr = A->row_ptr;
    a.col_ind = A->col_ind;
    a.depth = d_depth;
    a.ctl = ctl;
    a.sticky = sticky;
    a.alpha = 14.0f;
    a.beta = 24.0f;
    a.allow_pull = (A->flags & APSPIE_CSR_SYMMETRIC) ? 1 : 0;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_kernel, kBlock, 0) != cudaSuccess ||
        per_sm < 1)
        return APSPIE_ERR_CUDA;
    long long grid = (static_cast<long long>(A->nnz) + kWorkPerBlock - 1) / kWorkPerBlock;
    if (grid < sms) grid = sms;
    if (grid > static_cast<long long>(per_sm) * sms) grid = static_cast<long long>(per_sm) * sms;
    if (grid > kMaxGrid) grid = kMaxGrid;
    void *args[] = {&a};
    if (cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(bfs_kernel), dim3(static_cast<int>(grid)),
                                    dim3(kBlock), args, 0, stream) != cudaSuccess) {
        (void)cudaGetLastError();
        return APSPIE_ERR_CUDA;
    }
    TravCtl h;
    if (cudaMemcpyAsync(&h, ctl, kCtlHostBytes, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return APSPIE_ERR_CUDA;
    if (stats) {
        stats->iterations = h.iterations;
        stats->push_iterations = h.push_iterations;
        stats->pull_iterations = h.pull_iterations;
        stats->reserved = 0;
        stats->edges_expanded = h.edges_expanded;
        stats->edges_component = h.edges_component;
        stats->vertices_reached = h.vertices_reached;
    }
    return h.err != 0 ? static_cast<apspie_status>(h.err) : APSPIE_OK;
}

apspie_status apspie_spmspv_bool(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_x,
                                 int32_t *d_y) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_csr_view(ctx, A, "apspie_spmspv_bool");
    if (st != APSPIE_OK) return st;
    if (!d_x || !d_y) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_spmspv_bool: NULL vector");
    if (ctx->validate && (st = validate_csr(ctx, A, false)) != APSPIE_OK) return st;
    cudaError_t e = cudaMemsetAsync(d_y, 0, static_cast<size_t>(A->n) * sizeof(int32_t), ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "spmspv_bool memset");
    if (A->m > 0) {
        spmspv_bool_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(A->m, A->row_ptr, A->col_ind,
                                                                      d_x, d_y);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_error(ctx, e, "spmspv_bool launch");
    }
    return APSPIE_OK;
}

}  // extern "C"
