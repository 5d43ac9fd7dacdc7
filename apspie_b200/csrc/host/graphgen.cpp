// Host-side graph construction: synthetic generators, Matrix Market loading, CSR helpers.
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
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

// Builds a symmetric CSR from unique canonical pairs (lo < hi) given in ascending
// (lo, hi) order: row r gets its lower neighbours first (pairs (lo, r), ascending lo),
// then its upper neighbours (pairs (r, hi), ascending hi) -- sorted rows without a sort.
void build_symmetric(int m, const std::vector<uint64_t> &pairs, const std::vector<int32_t> *w,
                     apspie_host_csr *out) {
    const size_t np = pairs.size();
    out->m = out->n = m;
    out->nnz = static_cast<int32_t>(2 * np);
    out->row_ptr = host_alloc<int32_t>(static_cast<size_t>(m) + 1);
    out->col_ind = host_alloc<int32_t>(2 * np);
    int32_t *wv = nullptr;
    if (w) {
        wv = host_alloc<int32_t>(2 * np);
        out->val = wv;
        out->val_type = APSPIE_VAL_I32;
    } else {
        out->val = nullptr;
        out->val_type = APSPIE_VAL_NONE;
    }
    std::vector<int64_t> deg(static_cast<size_t>(m) + 1, 0);
    for (size_t i = 0; i < np; ++i) {
        ++deg[pairs[i] >> 32];
        ++deg[pairs[i] & 0xffffffffu];
    }
    int64_t run = 0;
    for (int r = 0; r < m; ++r) {
        out->row_ptr[r] = static_cast<int32_t>(run);
        run += deg[r];
    }
    out->row_ptr[m] = static_cast<int32_t>(run);
    std::vector<int64_t> cur(out->row_ptr, out->row_ptr + m);
    for (size_t i = 0; i < np; ++i) {  // lower neighbours
        const int32_t lo = static_cast<int32_t>(pairs[i] >> 32);
        const int32_t hi = static_cast<int32_t>(pairs[i] & 0xffffffffu);
        const int64_t p = cur[hi]++;
        out->col_ind[p] = lo;
        if (wv) wv[p] = (*w)[i];
    }
    for (size_t i = 0; i < np; ++i) {  // upper neighbours
        const int32_t lo = static_cast<int32_t>(pairs[i] >> 32);
        const int32_t hi = static_cast<int32_t>(pairs[i] & 0xffffffffu);
        const int64_t p = cur[lo]++;
        out->col_ind[p] = hi;
        if (wv) wv[p] = (*w)[i];
    }
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
    const double ab = a + b, abc = a + b + c;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::mt19937 wrng(weight_seed);
    std::uniform_int_distribution<int> W(1, 255);
    for (int64_t k = 0; k < ne; ++k) {
        uint32_t u = 0, v = 0;
        for (int l = 0; l < scale; ++l) {
            const double r = U(rng);
            u = (u << 1) | ((r >= ab) ? 1u : 0u);
            v = (v << 1) | ((r < a) ? 0u : (r < ab ? 1u : (r < abc ? 0u : 1u)));
        }
        const int wk = W(wrng);
        src[k] = static_cast<int32_t>(u);
        dst[k] = static_cast<int32_t>(v);
        if (weight) weight[k] = wk;
    }
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
    const double ab = a + b, abc = a + b + c;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::mt19937 wrng(weight_seed);
    std::uniform_int_distribution<int> W(1, 255);
    std::vector<uint64_t> key;
    std::vector<int32_t> wt;
    key.reserve(static_cast<size_t>(ne));
    wt.reserve(static_cast<size_t>(ne));
    for (int64_t k = 0; k < ne; ++k) {
        uint64_t u = 0, v = 0;
        for (int l = 0; l < scale; ++l) {
            const double r = U(rng);
            const unsigned ub = (r >= ab) ? 1u : 0u;
            const unsigned vb = (r < a) ? 0u : (r < ab ? 1u : (r < abc ? 0u : 1u));
            u = (u << 1) | ub;
            v = (v << 1) | vb;
        }
        const int wk = W(wrng);
        if (u == v) continue;
        const uint64_t lo = std::min(u, v), hi = std::max(u, v);
        key.push_back((lo << scale) | hi);
        wt.push_back(wk);
    }
    // stable sort by pair keeps generation order inside equal pairs: first copy wins
    radix_sort_pairs(key, wt, 2 * scale);
    std::vector<uint64_t> uniq;
    std::vector<int32_t> uw;
    uniq.reserve(key.size());
    uw.reserve(key.size());
    const uint64_t mask = static_cast<uint64_t>(m - 1);
    for (size_t i = 0; i < key.size(); ++i)
        if (i == 0 || key[i] != key[i - 1]) {
            uniq.push_back(((key[i] >> scale) << 32) | (key[i] & mask));
            uw.push_back(wt[i]);
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
    std::vector<int32_t> parent(m);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int32_t x) {
        while (parent[x] != x) {
            parent[x] = parent[parent[x]];
            x = parent[x];
        }
        return x;
    };
    for (int32_t u = 0; u < m; ++u)
        for (int32_t e = g->row_ptr[u]; e < g->row_ptr[u + 1]; ++e) {
            int32_t a = find(u), b = find(g->col_ind[e]);
            if (a != b) parent[std::max(a, b)] = std::min(a, b);
        }
    std::vector<int32_t> size(m, 0);
    for (int32_t v = 0; v < m; ++v) ++size[find(v)];
    int32_t root = 0;
    for (int32_t v = 0; v < m; ++v)
        if (size[v] > size[root]) root = v;  // roots are component minima: ties -> smallest id
    std::vector<int32_t> lcc;
    lcc.reserve(size[root]);
    for (int32_t v = 0; v < m; ++v)
        if (find(v) == root) lcc.push_back(v);
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
