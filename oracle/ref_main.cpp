// Driver around the REFERENCE's own CPU code -- TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/Makefile into oracle/_ref/apspie_ref from the reference sources where
// they lie (REF_DIR/src: util.cuh loader + CompareResults/uncompareResults, testBfs.cpp
// bfsCPU, testSssp.cpp ssspCPU, mt19937ar.cpp; test/mis/main.cu's misCPU extracted at
// build time into oracle/_ref). Nothing of the reference is copied into this repository.
//
// Usage (binary CSR files: int32 {m, n, nnz, val_type}, row_ptr[m+1], col_ind[nnz],
// then nnz 4-byte values when val_type != 0):
//   apspie_ref load  <file.mtx> <undirected 0|1> <out.csr>
//   apspie_ref bfs   <in.csr> <source> <out.i32>        (bfsCPU, stop = 1<<30)
//   apspie_ref sssp  <in.csr> <source> <out.i32>        (ssspCPU on float(weight))
//   apspie_ref ssspf <in.csr f32> <source> <out.f32>    (ssspCPU, float distances)
//   apspie_ref mis   <in.csr> <source> <out.i32>        (misCPU, vertex order)
//   apspie_ref mischeck <in.csr> <member.u8>            (one-hop + uncompareResults)
//   apspie_ref mt    <seed> <count> <out.u32>           (init_genrand + genrand_int32)
// Each command prints one line "APSPIE_REF {json}" with its CPU time in ms
// (std::chrono::steady_clock around the reference call only).
#include <cuda_runtime.h>
#include <cusparse.h>

#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <util.cuh>
// testSssp.cpp calls a two-argument print_array that this util.cuh no longer has.
template <typename T>
void print_array(const T *, int) {}
#include <testBfs.cpp>
#include <testSssp.cpp>
#include <mt19937ar.h>
#include "mis_cpu.inc"

namespace {

struct Csr {
    int m = 0, n = 0, nnz = 0, vt = 0;
    std::vector<int> rp, ci;
    std::vector<float> vf;
    std::vector<int> vi;
};

bool read_csr(const char *path, Csr &g) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    int h[4];
    bool ok = std::fread(h, sizeof(int), 4, f) == 4;
    if (ok) {
        g.m = h[0]; g.n = h[1]; g.nnz = h[2]; g.vt = h[3];
        g.rp.resize(g.m + 1);
        g.ci.resize(g.nnz);
        ok = std::fread(g.rp.data(), sizeof(int), g.m + 1, f) == size_t(g.m + 1) &&
             std::fread(g.ci.data(), sizeof(int), g.nnz, f) == size_t(g.nnz);
        if (ok && g.vt == 1) {
            g.vf.resize(g.nnz);
            ok = std::fread(g.vf.data(), sizeof(float), g.nnz, f) == size_t(g.nnz);
        } else if (ok && g.vt == 2) {
            g.vi.resize(g.nnz);
            ok = std::fread(g.vi.data(), sizeof(int), g.nnz, f) == size_t(g.nnz);
        }
    }
    std::fclose(f);
    return ok;
}

template <typename T>
bool write_array(const char *path, const T *p, size_t n) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    bool ok = std::fwrite(p, sizeof(T), n, f) == n;
    std::fclose(f);
    return ok;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// COO -> CSR by counting sort keeping input order inside a row: buildMatrix's
// conversion (src/matrix.cpp:55-111), which needs cub/moderngpu headers to compile there.
void coo_to_csr(int m, int nnz, const int *row, const int *col, const float *val, Csr &g) {
    g.m = m;
    g.nnz = nnz;
    g.vt = 1;
    g.rp.assign(m + 1, 0);
    g.ci.resize(nnz);
    g.vf.resize(nnz);
    for (int i = 0; i < nnz; ++i) g.rp[row[i]]++;
    int cum = 0;
    for (int i = 0; i < m; ++i) {
        int t = g.rp[i];
        g.rp[i] = cum;
        cum += t;
    }
    g.rp[m] = nnz;
    std::vector<int> cur(g.rp.begin(), g.rp.end() - 1);
    for (int i = 0; i < nnz; ++i) {
        int d = cur[row[i]]++;
        g.ci[d] = col[i];
        g.vf[d] = val[i];
    }
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: apspie_ref <command> ...\n");
        return 2;
    }
    const std::string cmd = argv[1];
    if (cmd == "load" && argc == 5) {
        if (!std::freopen(argv[2], "r", stdin)) return 3;
        int m = 0, n = 0, edge = 0;
        readEdge(m, n, edge, stdin);
        const int undirected = std::atoi(argv[3]);
        // makeSymmetric writes the mirrors after the `edge` entries read and its compaction
        // may look one slot past the end: give it 2*edge entries plus zeroed slack.
        const size_t cap = 2 * size_t(edge) + 64;
        std::vector<int> col(cap, 0), row(cap, 0);
        std::vector<float> val(cap, 0.0f);
        readMtx<float>(edge, col.data(), row.data(), val.data());
        int nnz = edge;
        if (undirected) nnz = makeSymmetric(edge, col.data(), row.data(), val.data());
        Csr g;
        coo_to_csr(m, nnz, row.data(), col.data(), val.data(), g);
        g.n = n;
        FILE *f = std::fopen(argv[4], "wb");
        if (!f) return 3;
        int h[4] = {g.m, g.n, g.nnz, 1};
        std::fwrite(h, sizeof(int), 4, f);
        std::fwrite(g.rp.data(), sizeof(int), g.m + 1, f);
        std::fwrite(g.ci.data(), sizeof(int), g.nnz, f);
        std::fwrite(g.vf.data(), sizeof(float), g.nnz, f);
        std::fclose(f);
        std::printf("APSPIE_REF {\"cmd\": \"load\", \"m\": %d, \"nnz\": %d}\n", g.m, g.nnz);
        return 0;
    }
    if (cmd == "ssspf" && argc == 5) {  // ssspCPU on float weights, float distances out
        Csr g;
        if (!read_csr(argv[2], g)) return 3;
        const int src = std::atoi(argv[3]);
        if (src < 0 || src >= g.m || g.vt != 1) return 4;
        std::vector<float> w(std::max(g.nnz, g.m) + 1, 1.0f);
        for (int e = 0; e < g.nnz; ++e) w[e] = g.vf[e];
        std::vector<float> d(g.m);
        auto t0 = std::chrono::steady_clock::now();
        ssspCPU(src, g.m, g.rp.data(), g.ci.data(), w.data(), d.data(), 1 << 30);
        const double ms = ms_since(t0);
        if (!write_array(argv[4], d.data(), d.size())) return 3;
        std::printf("APSPIE_REF {\"cmd\": \"ssspf\", \"ms\": %.6f, \"m\": %d, \"nnz\": %d}\n", ms, g.m, g.nnz);
        return 0;
    }
    if ((cmd == "bfs" || cmd == "sssp" || cmd == "mis") && argc == 5) {
        Csr g;
        if (!read_csr(argv[2], g)) return 3;
        const int src = std::atoi(argv[3]);
        if (src < 0 || src >= g.m) return 4;
        std::vector<int> out(g.m);
        double ms = 0.0;
        if (cmd == "bfs") {
            auto t0 = std::chrono::steady_clock::now();
            bfsCPU<int>(src, g.m, g.rp.data(), g.ci.data(), out.data(), 1 << 30);
            ms = ms_since(t0);
        } else if (cmd == "sssp") {
            // SimpleReferenceSssp seeds its queue with h_csrValA[i] for i < m
            // (testSssp.cpp:49-54): keep at least m weights readable.
            std::vector<float> w(std::max(g.nnz, g.m) + 1, 1.0f);
            for (int e = 0; e < g.nnz; ++e)
                w[e] = g.vt == 2 ? float(g.vi[e]) : (g.vt == 1 ? g.vf[e] : 1.0f);
            std::vector<float> d(g.m);
            auto t0 = std::chrono::steady_clock::now();
            ssspCPU(src, g.m, g.rp.data(), g.ci.data(), w.data(), d.data(), 1 << 30);
            ms = ms_since(t0);
            for (int i = 0; i < g.m; ++i) out[i] = d[i] < 0 ? -1 : int(d[i]);
        } else {
            auto t0 = std::chrono::steady_clock::now();
            misCPU(src, g.m, g.rp.data(), g.ci.data(), out.data());
            ms = ms_since(t0);
        }
        if (!write_array(argv[4], out.data(), out.size())) return 3;
        std::printf("APSPIE_REF {\"cmd\": \"%s\", \"ms\": %.6f, \"m\": %d, \"nnz\": %d}\n",
                    cmd.c_str(), ms, g.m, g.nnz);
        return 0;
    }
    if (cmd == "mischeck" && argc == 4) {
        Csr g;
        if (!read_csr(argv[2], g)) return 3;
        std::vector<unsigned char> mem(g.m);
        FILE *f = std::fopen(argv[3], "rb");
        if (!f || std::fread(mem.data(), 1, g.m, f) != size_t(g.m)) return 3;
        std::fclose(f);
        std::vector<int> mis(g.m), hop(g.m, 0);
        for (int i = 0; i < g.m; ++i) mis[i] = mem[i];
        for (int v = 0; v < g.m; ++v)  // one-hop of the set (spmspvCsr semantics)
            if (mis[v])
                for (int e = g.rp[v]; e < g.rp[v + 1]; ++e) hop[g.ci[e]] = 1;
        int bad = uncompareResults(hop.data(), mis.data(), g.m, false);
        std::printf("APSPIE_REF {\"cmd\": \"mischeck\", \"errors\": %d}\n", bad);
        return 0;
    }
    if (cmd == "mt" && argc == 5) {
        const unsigned long seed = std::strtoul(argv[2], nullptr, 10);
        const long long count = std::atoll(argv[3]);
        std::vector<unsigned> out(count);
        init_genrand(seed);
        for (long long i = 0; i < count; ++i) out[i] = static_cast<unsigned>(genrand_int32());
        if (!write_array(argv[4], out.data(), out.size())) return 3;
        std::printf("APSPIE_REF {\"cmd\": \"mt\", \"count\": %lld}\n", count);
        return 0;
    }
    std::fprintf(stderr, "apspie_ref: bad command\n");
    return 2;
}
