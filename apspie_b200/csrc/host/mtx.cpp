// Matrix Market loader with the reference loader's semantics.
//
// Reference behaviour followed (src/util.cuh):
//  readEdge  :355-367  skip every line whose first character is '%', then read "m n nnz";
//  readMtx   :370-430  entry j is read as (first -> column, second -> row), both 1-based;
//                      the graph is weighted iff the character right after the two
//                      integers of the FIRST entry is a blank, and then every entry reads
//                      a float value; otherwise every value is 1.0;
//  makeSymmetric :572-643  append the mirror of every non-loop entry, sort by (row, col),
//                      drop repeated pairs (self-loops are kept);
//  buildMatrix (src/matrix.cpp:55-111): counting sort by row, keeping input order inside
//                      a row.
// Deliberate differences, both in the reference's bugs rather than its intent:
//  - the drivers pass the already-doubled entry count to makeSymmetric (e.g.
//    test/bfs/main.cu:111-112), which then mirrors uninitialised memory; this loader
//    mirrors exactly the entries read;
//  - makeSymmetric's compaction moves indices but not values (util.cuh:630-640); this
//    loader keeps every value with its entry (values of a repeated pair: the first in
//    (row, col, file order) order).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../../include/apspie_host.h"

extern "C" apspie_status apspie_load_mtx(const char *path, int undirected, apspie_host_csr *out) {
    if (!path || !out) return APSPIE_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    FILE *f = std::fopen(path, "r");
    if (!f) return APSPIE_ERR_INVALID_ARG;
    // header: skip comment lines (a line is a comment iff it starts with '%')
    int c = std::fgetc(f), prev = '\n';
    while (c != EOF) {
        if (prev == '\n' && c != '%') {
            std::ungetc(c, f);
            break;
        }
        prev = c;
        c = std::fgetc(f);
    }
    int m = 0, n = 0, nnz = 0;
    if (std::fscanf(f, "%d %d %d", &m, &n, &nnz) != 3 || m < 0 || n < 0 || nnz < 0) {
        std::fclose(f);
        return APSPIE_ERR_INVALID_ARG;
    }
    std::vector<int> row(nnz), col(nnz);
    std::vector<float> val(nnz, 1.0f);
    bool weighted = false;
    int got = 0;
    for (int j = 0; j < nnz; ++j) {
        int a = 0, b = 0;
        if (std::fscanf(f, "%d", &a) != 1) break;  // fewer entries than promised
        if (std::fscanf(f, "%d", &b) != 1) break;
        if (j == 0) weighted = (std::fgetc(f) == ' ');
        if (weighted) {
            float w = 0.0f;
            if (std::fscanf(f, "%f", &w) == 1) val[j] = w;
        }
        col[j] = a - 1;
        row[j] = b - 1;
        ++got;
    }
    std::fclose(f);
    nnz = got;
    row.resize(nnz);
    col.resize(nnz);
    val.resize(nnz);
    for (int j = 0; j < nnz; ++j)
        if (row[j] < 0 || row[j] >= m || col[j] < 0 || col[j] >= std::max(m, n))
            return APSPIE_ERR_INVALID_ARG;

    if (undirected) {
        std::vector<int> r2, c2;
        std::vector<float> v2;
        r2.reserve(2 * nnz);
        c2.reserve(2 * nnz);
        v2.reserve(2 * nnz);
        for (int j = 0; j < nnz; ++j) {
            r2.push_back(row[j]);
            c2.push_back(col[j]);
            v2.push_back(val[j]);
        }
        for (int j = 0; j < nnz; ++j)
            if (row[j] != col[j]) {
                r2.push_back(col[j]);
                c2.push_back(row[j]);
                v2.push_back(val[j]);
            }
        std::vector<int> order(r2.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int>(i);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return r2[x] != r2[y] ? r2[x] < r2[y] : c2[x] < c2[y];
        });
        row.clear();
        col.clear();
        val.clear();
        for (size_t i = 0; i < order.size(); ++i) {
            const int k = order[i];
            if (i > 0) {
                const int p = order[i - 1];
                if (r2[p] == r2[k] && c2[p] == c2[k]) continue;
            }
            row.push_back(r2[k]);
            col.push_back(c2[k]);
            val.push_back(v2[k]);
        }
        nnz = static_cast<int>(row.size());
        n = std::max(m, n);
    }
    out->m = m;
    out->n = undirected ? m : std::max(m, n);
    out->nnz = nnz;
    out->row_ptr = static_cast<int32_t *>(std::malloc((static_cast<size_t>(m) + 1) * sizeof(int32_t)));
    out->col_ind = static_cast<int32_t *>(std::malloc(std::max(nnz, 1) * sizeof(int32_t)));
    float *v = static_cast<float *>(std::malloc(std::max(nnz, 1) * sizeof(float)));
    out->val = v;
    out->val_type = APSPIE_VAL_F32;
    std::vector<int> cnt(static_cast<size_t>(m) + 1, 0);
    for (int j = 0; j < nnz; ++j) ++cnt[row[j]];
    int run = 0;
    for (int r = 0; r < m; ++r) {
        out->row_ptr[r] = run;
        run += cnt[r];
    }
    out->row_ptr[m] = run;
    std::vector<int> cur(out->row_ptr, out->row_ptr + m);
    for (int j = 0; j < nnz; ++j) {
        const int p = cur[row[j]]++;
        out->col_ind[p] = col[j];
        v[p] = val[j];
    }
    (void)weighted;
    return APSPIE_OK;
}
