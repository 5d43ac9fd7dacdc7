// Host-side graph construction: synthetic generators, Matrix Market loading, CSR helpers.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <thread>
#include <vector>

#include "../../../include/apspie_host.h"

namespace {

template <typename T>
T *host_alloc(size_t n) {
    return static_cast<T *>(std::malloc(std::max<size_t>(n, 1) * sizeof(T)));
}

// Stable LSD radix sort of (key, payload) pairs on the low `bits` bits of key.
void radix_sort_pairs(std::vector<uint64_t> &key, std::vector<int32_t> &pay, int bits) {
    const size_t n = key.size();
    std::vector<uint64_t> k2(n);
    std::vector<int32_t> p2(n);
    const int nt = std::max(1, omp_get_max_threads());
    std::vector<size_t> hist(static_cast<size_t>(nt) * 256);
    for (int shift = 0; shift < bits; shift += 8) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
        {
            const int t = omp_get_thread_num();
            const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
            size_t *h = &hist[static_cast<size_t>(t) * 256];
            for (size_t i = lo; i < hi; ++i) ++h[(key[i] >> shift) & 255];
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (int d = 0; d < 256; ++d)
                    for (int tt = 0; tt < nt; ++tt) {
                        size_t c = hist[static_cast<size_t>(tt) * 256 + d];
                        hist[static_cast<size_t>(tt) * 256 + d] = run;
                        run += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) {
                size_t pos = h[(key[i] >> shift) & 255]++;
                k2[pos] = key[i];
                p2[pos] = pay[i];
            }
        }
        key.swap(k2);
        pay.swap(p2);
    }
}

// Builds a symmetric CSR from unique canonical pairs (lo << 32 | hi, lo < hi) given in
// ascending (lo, hi) order: row r gets its lower neighbours first (pairs (lo, r), ascending
// lo), then its upper neighbours (pairs (r, hi), ascending hi) -- sorted rows without a
// sort. Threads take contiguous ranges of pairs; per-thread counts of each row's lower
// neighbours give every thread its own write offsets, so the rows come out in pair order
// exactly as a single pass would write them.
void build_symmetric(int m, const std::vector<uint64_t> &pairs, const std::vector<int32_t> *w,
                     apspie_host_csr *out) {
    const int64_t np = static_cast<int64_t>(pairs.size());
    out->m = out->n = m;
    out->nnz = static_cast<int32_t>(2 * np);
    out->row_ptr = host_alloc<int32_t>(static_cast<size_t>(m) + 1);
    out->col_ind = host_alloc<int32_t>(static_cast<size_t>(2 * np));
    int32_t *wv = nullptr;
    if (w) {
        wv = host_alloc<int32_t>(static_cast<size_t>(2 * np));
        out->val = wv;
        out->val_type = APSPIE_VAL_I32;
    } else {
        out->val = nullptr;
        out->val_type = APSPIE_VAL_NONE;
    }
    // per-thread count arrays: at most about 512 MB of them
    const int T = std::max(1, std::min<int>(omp_get_max_threads(),
                                            static_cast<int>((int64_t(1) << 27) / std::max(m, 1))));
    std::vector<int32_t> low(static_cast<size_t>(T) * m, 0);  // lower-neighbour counts, then offsets
    std::vector<int64_t> up(static_cast<size_t>(m), 0);       // first pair of row r's upper run
    std::vector<int32_t> nup(static_cast<size_t>(m), 0);      // length of that run
    auto lo_of = [&](int64_t i) { return static_cast<int32_t>(pairs[i] >> 32); };
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const int64_t i0 = np * t / T, i1 = np * (t + 1) / T;
        int32_t *h = &low[static_cast<size_t>(t) * m];
        for (int64_t i = i0; i < i1; ++i) {
            ++h[static_cast<int32_t>(pairs[i] & 0xffffffffu)];
            const int32_t lo = lo_of(i);
            if (i == 0 || lo_of(i - 1) != lo) {  // a run of pairs (lo, *) starts here
                int64_t j = i + 1;
                while (j < np && lo_of(j) == lo) ++j;
                up[lo] = i;
                nup[lo] = static_cast<int32_t>(j - i);
            }
        }
    }
    int64_t run = 0;
    for (int r = 0; r < m; ++r) {
        out->row_ptr[r] = static_cast<int32_t>(run);
        for (int t = 0; t < T; ++t) {
            int32_t &c = low[static_cast<size_t>(t) * m + r];
            const int32_t n = c;
            c = static_cast<int32_t>(run);
            run += n;
        }
        up[r] = run - up[r];  // pair i of row r's upper run lands at up[r] + i
        run += nup[r];
    }
    out->row_ptr[m] = static_cast<int32_t>(run);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const int64_t i0 = np * t / T, i1 = np * (t + 1) / T;
        int32_t *h = &low[static_cast<size_t>(t) * m];
        for (int64_t i = i0; i < i1; ++i) {
            const int32_t lo = lo_of(i);
            const int32_t hi = static_cast<int32_t>(pairs[i] & 0xffffffffu);
            const int64_t p = h[hi]++;  // lower neighbour lo of row hi
            const int64_t q = up[lo] + i;  // upper neighbour hi of row lo
            out->col_ind[p] = lo;
            out->col_ind[q] = hi;
            if (wv) wv[p] = wv[q] = (*w)[i];
        }
    }
}

// MT19937 (Matsumoto and Nishimura, ACM TOMACS 8(1), 1998), the generator std::mt19937
// implements, advanced one whole 624-word state block per call. The untempered block is
// handed out; mt_temper turns its words into the generator's outputs, in order.
class MtBlocks {
  public:
    static constexpr int kN = 624, kM = 397;
    explicit MtBlocks(uint32_t seed) {
        s_[0] = seed;
        for (int i = 1; i < kN; ++i) s_[i] = 1812433253u * (s_[i - 1] ^ (s_[i - 1] >> 30)) + static_cast<uint32_t>(i);
    }
    const uint32_t *next_block() {
        for (int i = 0; i < kN - kM; ++i) s_[i] = step(s_[i], s_[i + 1], s_[i + kM]);
        for (int i = kN - kM; i < kN - 1; ++i) s_[i] = step(s_[i], s_[i + 1], s_[i + kM - kN]);
        s_[kN - 1] = step(s_[kN - 1], s_[0], s_[kM - 1]);
        return s_;
    }

  private:
    static uint32_t step(uint32_t cur, uint32_t nxt, uint32_t far) {
        const uint32_t y = (cur & 0x80000000u) | (nxt & 0x7fffffffu);
        return far ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    uint32_t s_[kN];
};

inline uint32_t mt_temper(uint32_t y) {
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    return y ^ (y >> 18);
}

// Replays recorded untempered MT19937 words as the generator's outputs, so that a standard
// distribution draws from it exactly what it would draw from std::mt19937 itself.
struct MtReplay {
    using result_type = std::mt19937::result_type;
    const uint32_t *p;
    static constexpr result_type min() { return std::mt19937::min(); }
    static constexpr result_type max() { return std::mt19937::max(); }
    result_type operator()() { return mt_temper(*p++); }
};

// The R-MAT edge stream of std::mt19937(seed): edge k takes `scale` uniform doubles
// (std::uniform_real_distribution<double>(0, 1), two generator words each), one per bit
// level, u's bit then v's from the same draw. One thread advances the generator and
// copies its words into a ring of chunks; the other threads turn chunks into edges and
// call edge(k, u, v) for every edge of their chunk. The result is the serial stream's,
// edge for edge, whatever the thread count.
template <class Edge>
void rmat_edges(int scale, int64_t ne, uint32_t seed, double a, double b, double c, Edge edge) {
    const double ab = a + b, abc = a + b + c;
    const int64_t per_edge = 2LL * scale;  // generator words per edge
    const int64_t kChunk = 1 << 14;        // edges per chunk
    const int64_t nch = (ne + kChunk - 1) / kChunk;
    auto decode = [&](int64_t k0, int64_t k1, const uint32_t *words) {
        MtReplay g{words};
        std::uniform_real_distribution<double> U(0.0, 1.0);
        for (int64_t k = k0; k < k1; ++k) {
            uint32_t u = 0, v = 0;
            for (int l = 0; l < scale; ++l) {
                const double r = U(g);
                u = (u << 1) | ((r >= ab) ? 1u : 0u);
                v = (v << 1) | ((r < a) ? 0u : (r < ab ? 1u : (r < abc ? 0u : 1u)));
            }
            edge(k, u, v);
        }
    };
    const int workers = std::max(1, std::min<int>(omp_get_max_threads() - 1, static_cast<int>(nch)));
    const int ring = 2 * workers + 2;
    std::vector<std::vector<uint32_t>> slot(ring, std::vector<uint32_t>(static_cast<size_t>(kChunk * per_edge)));
    std::vector<std::atomic<int64_t>> filled(ring), done(ring);
    for (int i = 0; i < ring; ++i) {
        filled[i].store(-1);
        done[i].store(static_cast<int64_t>(i) - ring);  // slot i is free for chunk i
    }
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t ch = next.fetch_add(1);
            if (ch >= nch) return;
            const int sl = static_cast<int>(ch % ring);
            while (filled[sl].load(std::memory_order_acquire) != ch) std::this_thread::yield();
            decode(ch * kChunk, std::min(ne, (ch + 1) * kChunk), slot[sl].data());
            done[sl].store(ch, std::memory_order_release);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < workers; ++t) pool.emplace_back(worker);
    MtBlocks mt(seed);
    const uint32_t *blk = nullptr;
    int pos = MtBlocks::kN;
    for (int64_t ch = 0; ch < nch; ++ch) {
        const int sl = static_cast<int>(ch % ring);
        while (done[sl].load(std::memory_order_acquire) != ch - ring) std::this_thread::yield();
        uint32_t *dst = slot[sl].data();
        int64_t need = (std::min(ne, (ch + 1) * kChunk) - ch * kChunk) * per_edge;
        while (need > 0) {
            if (pos == MtBlocks::kN) {
                blk = mt.next_block();
                pos = 0;
            }
            const int take = static_cast<int>(std::min<int64_t>(need, MtBlocks::kN - pos));
            std::memcpy(dst, blk + pos, static_cast<size_t>(take) * sizeof(uint32_t));
            dst += take;
            pos += take;
            need -= take;
        }
        filled[sl].store(ch, std::memory_order_release);
    }
    for (auto &t : pool) t.join();
}

// The weight of generated edge k: the k-th draw of uniform_int_distribution<int>(1, 255)
// on std::mt19937(weight_seed), drawn for every generated edge in order.
void rmat_weights(int64_t ne, uint32_t weight_seed, int32_t *w) {
    std::mt19937 wrng(weight_seed);
    std::uniform_int_distribution<int> W(1, 255);
    for (int64_t k = 0; k < ne; ++k) w[k] = W(wrng);
}

}  // namespace

extern "C" {

void apspie_host_csr_free(apspie_host_csr *g) {
    if (!g) return;
    std::free(g->row_ptr);
    std::free(g->col_ind);
    std::free(g->val);
    g->row_ptr = g->col_ind = nullptr;
    g->val = nullptr;
}

apspie_status apspie_gen_rmat_coo(int scale, int edge_factor, uint32_t seed, uint32_t weight_seed, double a,
                                  double b, double c, int32_t *src, int32_t *dst, int32_t *weight) {
    if (!src || !dst || scale < 1 || scale > 30 || edge_factor < 1) return APSPIE_ERR_INVALID_ARG;
    const int64_t ne = (int64_t(1) << scale) * edge_factor;
    if (ne > INT32_MAX) return APSPIE_ERR_UNSUPPORTED;
    std::thread wthread;
    if (weight) wthread = std::thread(rmat_weights, ne, weight_seed, weight);
    rmat_edges(scale, ne, seed, a, b, c, [&](int64_t k, uint32_t u, uint32_t v) {
        src[k] = static_cast<int32_t>(u);
        dst[k] = static_cast<int32_t>(v);
    });
    if (wthread.joinable()) wthread.join();
    return APSPIE_OK;
}

apspie_status apspie_gen_rmat(int scale, int edge_factor, uint32_t seed, uint32_t weight_seed,
                              double a, double b, double c, int with_weights,
                              apspie_host_csr *out) {
    if (!out || scale < 1 || scale > 30 || edge_factor < 1) return APSPIE_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    const int64_t m = int64_t(1) << scale;
    const int64_t ne = m * edge_factor;
    if (2 * ne > INT32_MAX) return APSPIE_ERR_UNSUPPORTED;
    // key[k] = the canonical pair (lo << scale | hi) of generated edge k, or all ones for a
    // self-loop (it sorts after every pair and is dropped); wt[k] = its weight draw
    std::vector<uint64_t> key(static_cast<size_t>(ne));
    std::vector<int32_t> wt(static_cast<size_t>(ne));
    std::thread wthread(rmat_weights, ne, weight_seed, wt.data());
    rmat_edges(scale, ne, seed, a, b, c, [&](int64_t k, uint32_t u, uint32_t v) {
        const uint64_t lo = std::min(u, v), hi = std::max(u, v);
        key[k] = u == v ? ~0ull : ((lo << scale) | hi);
    });
    wthread.join();
    // stable sort by pair keeps generation order inside equal pairs: first copy wins
    radix_sort_pairs(key, wt, 2 * scale);
    // keep the first of every run of equal pairs (the self-loop marks sort last and go)
    int64_t nv = ne;
    while (nv > 0 && key[nv - 1] == ~0ull) --nv;
    const int T = std::max(1, omp_get_max_threads());
    std::vector<int64_t> kept(static_cast<size_t>(T) + 1, 0);
    auto first_of_run = [&](int64_t i) { return i == 0 || key[i] != key[i - 1]; };
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const int64_t i0 = nv * t / T, i1 = nv * (t + 1) / T;
        int64_t n = 0;
        for (int64_t i = i0; i < i1; ++i) n += first_of_run(i);
        kept[t + 1] = n;
    }
    for (int t = 0; t < T; ++t) kept[t + 1] += kept[t];
    std::vector<uint64_t> uniq(static_cast<size_t>(kept[T]));
    std::vector<int32_t> uw(static_cast<size_t>(kept[T]));
    const uint64_t mask = static_cast<uint64_t>(m - 1);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const int64_t i0 = nv * t / T, i1 = nv * (t + 1) / T;
        int64_t o = kept[t];
        for (int64_t i = i0; i < i1; ++i)
            if (first_of_run(i)) {
                uniq[o] = ((key[i] >> scale) << 32) | (key[i] & mask);
                uw[o++] = wt[i];
            }
    }
    build_symmetric(static_cast<int>(m), uniq, with_weights ? &uw : nullptr, out);
    return APSPIE_OK;
}

apspie_status apspie_gen_er(int n, int k, uint32_t seed, int val_type, apspie_host_csr *out) {
    if (!out || n < 1 || k < 0 || k > n) return APSPIE_ERR_INVALID_ARG;
    if (static_cast<int64_t>(n) * k > INT32_MAX) return APSPIE_ERR_UNSUPPORTED;
    std::memset(out, 0, sizeof(*out));
    const size_t nnz = static_cast<size_t>(n) * k;
    out->m = out->n = n;
    out->nnz = static_cast<int32_t>(nnz);
    out->row_ptr = host_alloc<int32_t>(static_cast<size_t>(n) + 1);
    out->col_ind = host_alloc<int32_t>(nnz);
    std::mt19937 rng(seed);
    std::uniform_int_distribution<int> C(0, n - 1);
    for (int i = 0; i <= n; ++i) out->row_ptr[i] = static_cast<int32_t>(static_cast<int64_t>(i) * k);
    for (int i = 0; i < n; ++i) {
        int32_t *row = out->col_ind + static_cast<size_t>(i) * k;
        int have = 0;
        while (have < k) {
            const int cnd = C(rng);
            bool dup = false;
            for (int t = 0; t < have; ++t) dup |= (row[t] == cnd);
            if (!dup) row[have++] = cnd;
        }
        std::sort(row, row + k);
    }
    out->val_type = val_type;
    if (val_type == APSPIE_VAL_F32) {
        float *v = host_alloc<float>(nnz);
        std::uniform_real_distribution<float> F(-1.0f, 1.0f);
        for (size_t e = 0; e < nnz; ++e) v[e] = F(rng);
        out->val = v;
    } else if (val_type == APSPIE_VAL_I32) {
        int32_t *v = host_alloc<int32_t>(nnz);
        std::uniform_int_distribution<int> I(1, 8);
        for (size_t e = 0; e < nnz; ++e) v[e] = I(rng);
        out->val = v;
    } else {
        out->val = nullptr;
        out->val_type = APSPIE_VAL_NONE;
    }
    return APSPIE_OK;
}

apspie_status apspie_mt19937_u32(uint32_t seed, int64_t count, uint32_t *out) {
    if (count < 0 || (count > 0 && !out)) return APSPIE_ERR_INVALID_ARG;
    std::mt19937 rng(seed);
    for (int64_t i = 0; i < count; ++i) out[i] = static_cast<uint32_t>(rng());
    return APSPIE_OK;
}

int32_t apspie_max_degree_vertex(const apspie_host_csr *g) {
    if (!g || g->m <= 0) return -1;
    int32_t best = 0, bd = -1;
    for (int32_t v = 0; v < g->m; ++v) {
        const int32_t d = g->row_ptr[v + 1] - g->row_ptr[v];
        if (d > bd) {
            bd = d;
            best = v;
        }
    }
    return best;
}

apspie_status apspie_lcc_sample(const apspie_host_csr *g, int32_t count, uint32_t seed,
                                int32_t *out) {
    if (!g || count < 0 || (count > 0 && !out) || g->m <= 0) return APSPIE_ERR_INVALID_ARG;
    const int32_t m = g->m;
    // connected components by lock-free union-find over all edges in parallel: a root is
    // only ever hooked under a smaller root, so each tree's root is its component's
    // smallest vertex, whatever the order of the unions
    std::vector<int32_t> parent(m);
    std::iota(parent.begin(), parent.end(), 0);
    int32_t *par = parent.data();
    auto find = [par](int32_t x) {
        for (;;) {
            const int32_t p = __atomic_load_n(par + x, __ATOMIC_RELAXED);
            if (p == x) return x;
            const int32_t gp = __atomic_load_n(par + p, __ATOMIC_RELAXED);
            if (gp != p) {
                int32_t expect = p;  // path halving; losing the race is harmless
                __atomic_compare_exchange_n(par + x, &expect, gp, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
            }
            x = gp;
        }
    };
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t u = 0; u < m; ++u)
        for (int32_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
            int32_t a = u, b = g->col_ind[e];
            for (;;) {
                a = find(a);
                b = find(b);
                if (a == b) break;
                if (a > b) std::swap(a, b);
                int32_t expect = b;  // hook the larger root under the smaller
                if (__atomic_compare_exchange_n(par + b, &expect, a, false, __ATOMIC_ACQ_REL, __ATOMIC_RELAXED))
                    break;
            }
        }
    std::vector<int32_t> comp(m);
    std::vector<int32_t> size(m, 0);
#pragma omp parallel for schedule(static)
    for (int32_t v = 0; v < m; ++v) {
        comp[v] = find(v);
        __atomic_fetch_add(&size[comp[v]], 1, __ATOMIC_RELAXED);
    }
    int32_t root = 0;
    for (int32_t v = 0; v < m; ++v)
        if (size[v] > size[root]) root = v;  // roots are component minima: ties -> smallest id
    std::vector<int32_t> lcc;
    lcc.reserve(size[root]);
    for (int32_t v = 0; v < m; ++v)
        if (comp[v] == root) lcc.push_back(v);
    if (count > static_cast<int32_t>(lcc.size())) return APSPIE_ERR_INVALID_ARG;
    std::mt19937 rng(seed);
    const int64_t sz = static_cast<int64_t>(lcc.size());
    for (int32_t i = 0; i < count; ++i) {
        std::uniform_int_distribution<int64_t> D(i, sz - 1);
        const int64_t j = D(rng);
        std::swap(lcc[i], lcc[j]);
        out[i] = lcc[i];
    }
    return APSPIE_OK;
}

apspie_status apspie_csr_strict_lower(const apspie_host_csr *A, apspie_host_csr *L) {
    if (!A || !L || A->m < 0) return APSPIE_ERR_INVALID_ARG;
    std::memset(L, 0, sizeof(*L));
    const int32_t m = A->m;
    L->m = m;
    L->n = A->n;
    L->row_ptr = host_alloc<int32_t>(static_cast<size_t>(m) + 1);
    int64_t cnt = 0;
    for (int32_t i = 0; i < m; ++i)
        for (int32_t e = A->row_ptr[i]; e < A->row_ptr[i + 1]; ++e) cnt += (A->col_ind[e] < i);
    L->col_ind = host_alloc<int32_t>(static_cast<size_t>(cnt));
    int64_t p = 0;
    for (int32_t i = 0; i < m; ++i) {
        L->row_ptr[i] = static_cast<int32_t>(p);
        for (int32_t e = A->row_ptr[i]; e < A->row_ptr[i + 1]; ++e)
            if (A->col_ind[e] < i) L->col_ind[p++] = A->col_ind[e];
    }
    L->row_ptr[m] = static_cast<int32_t>(p);
    L->nnz = static_cast<int32_t>(p);
    L->val = nullptr;
    L->val_type = APSPIE_VAL_NONE;
    return APSPIE_OK;
}

}  // extern "C"
