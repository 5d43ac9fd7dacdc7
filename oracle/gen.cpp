// CPU oracle: serial restatement of the synthetic R-MAT input -- TEST INFRASTRUCTURE ONLY.
//
// Used by tests (to pin the product's parallel host generator) and by bench.py's reference
// arm (so that arm builds its input graph without loading the product library). The spec:
// edge k of 2^scale * edge_factor takes `scale` draws of std::mt19937(seed) through
// std::uniform_real_distribution<double>(0, 1), most significant bit first; a draw r picks
// the quadrant r < a: (0,0), r < a+b: (0,1), r < a+b+c: (1,0), else (1,1), whose first bit
// goes to u and second to v. Its weight is draw k of std::mt19937(weight_seed) through
// std::uniform_int_distribution<int>(1, 255), drawn for every generated edge. Self-loops
// are dropped, {u, v} is canonicalised and the first generated copy of each pair is kept;
// the pair is stored in both directions with that weight and rows are sorted by column.
// The reference itself benchmarks on downloaded Graph500 Kronecker graphs
// (test/bfs/run.sh:17-39); this synthetic stand-in has their a/b/c/d parameters.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <random>
#include <utility>
#include <vector>

extern "C" {

// Returns the number of directed entries (2 x unique pairs), or -1 on bad arguments.
// row_ptr must hold 2^scale + 1 ints; col_ind and w (may be NULL) must hold `cap` ints.
// With cap < the entry count only the count is returned (call again with room).
long long oracle_gen_rmat(int scale, int edge_factor, unsigned seed, unsigned weight_seed, double a, double b,
                          double c, long long cap, int *row_ptr, int *col_ind, int *w) {
    if (scale < 1 || scale > 30 || edge_factor < 1) return -1;
    const int64_t m = int64_t(1) << scale;
    const int64_t ne = m * edge_factor;
    const double ab = a + b, abc = a + b + c;
    std::mt19937 rng(seed), wrng(weight_seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::uniform_int_distribution<int> W(1, 255);
    // (canonical pair, generation index) for every non-loop edge; weights by index
    std::vector<std::pair<uint64_t, int64_t>> e;
    e.reserve(static_cast<size_t>(ne));
    std::vector<int> wk(static_cast<size_t>(ne));
    for (int64_t k = 0; k < ne; ++k) {
        uint64_t u = 0, v = 0;
        for (int l = 0; l < scale; ++l) {
            const double r = U(rng);
            u = (u << 1) | (r >= ab ? 1u : 0u);
            v = (v << 1) | (r < a ? 0u : r < ab ? 1u : r < abc ? 0u : 1u);
        }
        wk[static_cast<size_t>(k)] = W(wrng);
        if (u != v) e.emplace_back((std::min(u, v) << 32) | std::max(u, v), k);
    }
    std::sort(e.begin(), e.end());  // by pair, then generation order: the first copy leads
    std::vector<uint64_t> pair;
    std::vector<int> pw;
    for (size_t i = 0; i < e.size(); ++i)
        if (i == 0 || e[i].first != e[i - 1].first) {
            pair.push_back(e[i].first);
            pw.push_back(wk[static_cast<size_t>(e[i].second)]);
        }
    const long long nnz = 2LL * static_cast<long long>(pair.size());
    if (cap < nnz) return nnz;
    // Counting sort by row, stable, over the lower-neighbour entries (hi <- lo) in pair
    // order followed by the upper-neighbour entries (lo <- hi) in pair order: each row gets
    // its lower neighbours ascending, then its upper neighbours ascending.
    std::vector<int64_t> cnt(static_cast<size_t>(m) + 1, 0);
    for (uint64_t p : pair) {
        ++cnt[(p & 0xffffffffu) + 1];
        ++cnt[(p >> 32) + 1];
    }
    for (int64_t r = 0; r < m; ++r) cnt[r + 1] += cnt[r];
    for (int64_t r = 0; r <= m; ++r) row_ptr[r] = static_cast<int>(cnt[r]);
    for (size_t i = 0; i < pair.size(); ++i) {
        const int64_t lo = static_cast<int64_t>(pair[i] >> 32), hi = static_cast<int64_t>(pair[i] & 0xffffffffu);
        const int64_t at = cnt[hi]++;
        col_ind[at] = static_cast<int>(lo);
        if (w) w[at] = pw[i];
    }
    for (size_t i = 0; i < pair.size(); ++i) {
        const int64_t lo = static_cast<int64_t>(pair[i] >> 32), hi = static_cast<int64_t>(pair[i] & 0xffffffffu);
        const int64_t at = cnt[lo]++;
        col_ind[at] = static_cast<int>(hi);
        if (w) w[at] = pw[i];
    }
    return nnz;
}

}  // extern "C"
