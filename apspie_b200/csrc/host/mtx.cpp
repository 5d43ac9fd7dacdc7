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
//
// apspie_load_mtx_threads parses the entry lines in parallel (chunks cut at line ends, each
// parsed with strtol / strtof, which read numbers exactly as fscanf's %d / %f do) and sorts
// with the parallel stable sort; it assumes one entry per line, as every Matrix Market file
// has. Its result equals apspie_load_mtx's.
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <parallel/algorithm>
#include <vector>

#include "../../../include/apspie_host.h"

namespace {

struct Parsed {
    int m = 0, n = 0, nnz = 0;
    std::vector<int> row, col;
    std::vector<float> val;
};

apspie_status finish(Parsed &p, int undirected, int threads, apspie_host_csr *out);

apspie_status parse_serial(const char *path, Parsed &p) {
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
    row.resize(got);
    col.resize(got);
    val.resize(got);
    p.m = m;
    p.n = n;
    p.nnz = got;
    p.row = std::move(row);
    p.col = std::move(col);
    p.val = std::move(val);
    return APSPIE_OK;
}

// Parses one chunk [b, e) of entry lines: "a b" or "a b w" per line.
void parse_chunk(const char *b, const char *e, bool weighted, std::vector<int> &row, std::vector<int> &col,
                 std::vector<float> &val) {
    const char *q = b;
    while (q < e) {
        while (q < e && (*q == ' ' || *q == '\t' || *q == '\n' || *q == '\r')) ++q;
        if (q >= e) break;
        char *end = nullptr;
        const long a = std::strtol(q, &end, 10);
        if (end == q) break;
        q = end;
        const long c = std::strtol(q, &end, 10);
        if (end == q) break;
        q = end;
        float w = 1.0f;
        if (weighted) {
            const float x = std::strtof(q, &end);
            if (end != q) {
                w = x;
                q = end;
            }
        }
        while (q < e && *q != '\n') ++q;  // rest of the line
        col.push_back(static_cast<int>(a) - 1);
        row.push_back(static_cast<int>(c) - 1);
        val.push_back(w);
    }
}

apspie_status parse_parallel(const char *path, int threads, Parsed &p) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return APSPIE_ERR_INVALID_ARG;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> buf(static_cast<size_t>(size > 0 ? size : 0) + 1, '\0');
    const size_t rd = size > 0 ? std::fread(buf.data(), 1, static_cast<size_t>(size), f) : 0;
    std::fclose(f);
    const char *s = buf.data(), *end = s + rd;
    // header: skip lines that start with '%'
    const char *q = s;
    while (q < end && *q == '%') {
        while (q < end && *q != '\n') ++q;
        if (q < end) ++q;
    }
    char *e2 = nullptr;
    const long m = std::strtol(q, &e2, 10);
    if (e2 == q) return APSPIE_ERR_INVALID_ARG;
    q = e2;
    const long n = std::strtol(q, &e2, 10);
    if (e2 == q) return APSPIE_ERR_INVALID_ARG;
    q = e2;
    const long nnz = std::strtol(q, &e2, 10);
    if (e2 == q || m < 0 || n < 0 || nnz < 0) return APSPIE_ERR_INVALID_ARG;
    q = e2;
    // weighted iff the character right after the first entry's two integers is a blank
    bool weighted = false;
    {
        const char *t = q;
        std::strtol(t, &e2, 10);
        if (e2 != t) {
            t = e2;
            std::strtol(t, &e2, 10);
            if (e2 != t && e2 < end) weighted = (*e2 == ' ');
        }
    }
    const int T = std::max(1, threads);
    std::vector<const char *> cut(T + 1);
    cut[0] = q;
    cut[T] = end;
    for (int k = 1; k < T; ++k) {
        const char *c = q + (end - q) * static_cast<long long>(k) / T;
        while (c < end && *c != '\n') ++c;
        cut[k] = c < end ? c + 1 : end;
        if (cut[k] < cut[k - 1]) cut[k] = cut[k - 1];
    }
    std::vector<std::vector<int>> rows(T), cols(T);
    std::vector<std::vector<float>> vals(T);
#pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int k = 0; k < T; ++k) parse_chunk(cut[k], cut[k + 1], weighted, rows[k], cols[k], vals[k]);
    size_t total = 0;
    for (int k = 0; k < T; ++k) total += rows[k].size();
    const size_t keep = std::min(total, static_cast<size_t>(nnz));  // at most the promised count
    p.m = static_cast<int>(m);
    p.n = static_cast<int>(n);
    p.nnz = static_cast<int>(keep);
    p.row.resize(keep);
    p.col.resize(keep);
    p.val.resize(keep);
    size_t at = 0;
    for (int k = 0; k < T && at < keep; ++k) {
        const size_t c = std::min(rows[k].size(), keep - at);
        std::copy(rows[k].begin(), rows[k].begin() + c, p.row.begin() + at);
        std::copy(cols[k].begin(), cols[k].begin() + c, p.col.begin() + at);
        std::copy(vals[k].begin(), vals[k].begin() + c, p.val.begin() + at);
        at += c;
    }
    return APSPIE_OK;
}

apspie_status finish(Parsed &p, int undirected, int threads, apspie_host_csr *out) {
    const int m = p.m;
    int n = p.n, nnz = p.nnz;
    std::vector<int> &row = p.row, &col = p.col;
    std::vector<float> &val = p.val;
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
        const auto by_pair = [&](int x, int y) { return r2[x] != r2[y] ? r2[x] < r2[y] : c2[x] < c2[y]; };
        if (threads > 1)
            __gnu_parallel::stable_sort(order.begin(), order.end(), by_pair);
        else
            std::stable_sort(order.begin(), order.end(), by_pair);
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
    return APSPIE_OK;
}

}  // namespace

extern "C" apspie_status apspie_load_mtx(const char *path, int undirected, apspie_host_csr *out) {
    if (!path || !out) return APSPIE_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    Parsed p;
    apspie_status st = parse_serial(path, p);
    if (st != APSPIE_OK) return st;
    return finish(p, undirected, 1, out);
}

extern "C" apspie_status apspie_load_mtx_threads(const char *path, int undirected, int threads,
                                                 apspie_host_csr *out) {
    if (!path || !out || threads < 0) return APSPIE_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    const int T = threads > 0 ? threads : omp_get_max_threads();
    Parsed p;
    apspie_status st = parse_parallel(path, T, p);
    if (st != APSPIE_OK) return st;
    return finish(p, undirected, T, out);
}
