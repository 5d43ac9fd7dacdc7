// Autotuner: times candidate knob settings of one kind of call on a given input, keeps
// the fastest per (kind, shape bucket) in the context's tuning table, and lets later
// calls on inputs of the same bucket use it. The table persists as a text file.
//
// The reference fixes these choices at compile time (the SpMSpV sort-based expansion has
// no push/pull switch, spgemm.cuh:131-342 takes its partition sizes from the caller, TC
// runs one thread per column); here they are the tiers and thresholds of this library's
// own kernels:
//   BFS        alpha, beta        push/pull switch (Beamer)
//   SSSP       band               edges expanded per iteration
//   BFS_BATCH  push_frac          batched push/pull switch
//   SPGEMM     reg_max, block_max rows sorted by a warp in registers / hashed in a
//                                 block's shared table / hashed in a global table
//   TC         task_work, orient  wedges per warp task, degree re-orientation
// A shape bucket is (kind, bit length of m, nearest integer log2 of nnz / m, symmetric).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "common.cuh"

namespace apspie {
namespace {

struct Bucket {
    int kind, log_m, log_deg, symmetric;
};

Bucket bucket_of(int kind, const apspie_csr *A) {
    Bucket b;
    b.kind = kind;
    unsigned m = A->m > 0 ? static_cast<unsigned>(A->m) : 1u;
    b.log_m = 32 - __builtin_clz(m);
    const double deg = A->m > 0 ? static_cast<double>(A->nnz) / A->m : 0.0;
    b.log_deg = deg >= 1.0 ? static_cast<int>(std::floor(std::log2(deg) + 0.5)) : 0;
    b.symmetric = (A->flags & APSPIE_CSR_SYMMETRIC) ? 1 : 0;
    return b;
}

apspie_tune_params own_params(const apspie_ctx *ctx) {
    apspie_tune_params p;
    std::memset(&p, 0, sizeof(p));
    p.bfs_alpha = ctx->bfs_alpha;
    p.bfs_beta = ctx->bfs_beta;
    p.batch_push_frac = ctx->batch_push_frac;
    p.sssp_delta = ctx->sssp_delta;
    p.sssp_band = ctx->sssp_band;
    p.spgemm_reg_max = ctx->spgemm_reg_max;
    p.spgemm_block_max = ctx->spgemm_block_max;
    p.tc_task_work = ctx->tc_task_work;
    p.tc_orient = ctx->tc_orient;
    return p;
}

bool params_valid(const apspie_tune_params &p) {
    const int r = p.spgemm_reg_max;
    return std::isfinite(p.bfs_alpha) && p.bfs_beta > 0.0f && p.batch_push_frac >= 0.0f &&
           (r == 0 || r == 32 || r == 64 || r == 128) && p.spgemm_block_max >= 0 && p.spgemm_block_max <= 1024 &&
           p.tc_task_work >= 256 && p.tc_task_work <= (1 << 24) && (p.tc_orient == 0 || p.tc_orient == 1);
}

void apply_params(apspie_ctx *ctx, const apspie_tune_params &p) {
    ctx->bfs_alpha = p.bfs_alpha;
    ctx->bfs_beta = p.bfs_beta;
    ctx->batch_push_frac = p.batch_push_frac;
    ctx->sssp_delta = p.sssp_delta;
    ctx->sssp_band = p.sssp_band;
    ctx->spgemm_reg_max = p.spgemm_reg_max;
    ctx->spgemm_block_max = p.spgemm_block_max;
    ctx->tc_task_work = p.tc_task_work;
    ctx->tc_orient = p.tc_orient;
}

// Copies the knobs of `kind` from src into dst (the other kinds' knobs stay).
void take_kind(apspie_tune_params &dst, const apspie_tune_params &src, int kind) {
    switch (kind) {
    case APSPIE_TUNE_BFS:
        dst.bfs_alpha = src.bfs_alpha;
        dst.bfs_beta = src.bfs_beta;
        break;
    case APSPIE_TUNE_SSSP:
        dst.sssp_delta = src.sssp_delta;
        dst.sssp_band = src.sssp_band;
        break;
    case APSPIE_TUNE_BFS_BATCH:
        dst.batch_push_frac = src.batch_push_frac;
        break;
    case APSPIE_TUNE_SPGEMM:
        dst.spgemm_reg_max = src.spgemm_reg_max;
        dst.spgemm_block_max = src.spgemm_block_max;
        break;
    case APSPIE_TUNE_TC:
        dst.tc_task_work = src.tc_task_work;
        dst.tc_orient = src.tc_orient;
        break;
    default:
        break;
    }
}

const apspie_tune_entry *find_entry(const apspie_ctx *ctx, const Bucket &b) {
    for (const apspie_tune_entry &e : ctx->tune_table)
        if (e.kind == b.kind && e.log_m == b.log_m && e.log_deg == b.log_deg && e.symmetric == b.symmetric)
            return &e;
    return nullptr;
}

void record(apspie_ctx *ctx, const Bucket &b, const apspie_tune_params &p, double ms) {
    for (apspie_tune_entry &e : ctx->tune_table)
        if (e.kind == b.kind && e.log_m == b.log_m && e.log_deg == b.log_deg && e.symmetric == b.symmetric) {
            e.p = p;
            e.ms = ms;
            return;
        }
    apspie_tune_entry e;
    e.kind = b.kind;
    e.log_m = b.log_m;
    e.log_deg = b.log_deg;
    e.symmetric = b.symmetric;
    e.p = p;
    e.ms = ms;
    ctx->tune_table.push_back(e);
}

// Device buffers the tuner owns for the duration of one autotune call.
struct TuneBuffers {
    std::vector<void *> ptrs;
    ~TuneBuffers() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <typename T>
    T *get(size_t n) {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
};

}  // namespace

apspie_tune_params effective_params(const apspie_ctx *ctx, int kind, const apspie_csr *A) {
    apspie_tune_params p = own_params(ctx);
    if (ctx->use_tuning && A && !ctx->tune_table.empty()) {
        const apspie_tune_entry *e = find_entry(ctx, bucket_of(kind, A));
        if (e) take_kind(p, e->p, kind);
    }
    return p;
}

}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_ctx_get_params(const apspie_ctx *ctx, apspie_tune_params *out) {
    if (!ctx || !out) return APSPIE_ERR_INVALID_ARG;
    *out = own_params(ctx);
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_params(apspie_ctx *ctx, const apspie_tune_params *p) {
    if (!ctx || !p) return APSPIE_ERR_INVALID_ARG;
    if (!params_valid(*p)) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_ctx_set_params: knob out of range");
    apply_params(ctx, *p);
    return APSPIE_OK;
}

apspie_status apspie_ctx_set_autotune(apspie_ctx *ctx, int32_t use) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    ctx->use_tuning = use ? 1 : 0;
    return APSPIE_OK;
}

int32_t apspie_tune_entries(const apspie_ctx *ctx) {
    return ctx ? static_cast<int32_t>(ctx->tune_table.size()) : 0;
}

apspie_status apspie_tune_lookup(const apspie_ctx *ctx, int32_t kind, const apspie_csr *A,
                                 apspie_tune_params *out, int32_t *found) {
    if (!ctx || !A || !out || kind < 0 || kind > APSPIE_TUNE_TC) return APSPIE_ERR_INVALID_ARG;
    const apspie_tune_entry *e = find_entry(ctx, bucket_of(kind, A));
    if (found) *found = e ? 1 : 0;
    *out = effective_params(ctx, kind, A);
    return APSPIE_OK;
}

apspie_status apspie_tune_save(const apspie_ctx *ctx, const char *path) {
    if (!ctx || !path) return APSPIE_ERR_INVALID_ARG;
    FILE *f = std::fopen(path, "w");
    if (!f) return APSPIE_ERR_INVALID_ARG;
    std::fprintf(f, "apspie-tune 1\n");
    std::fprintf(f, "# kind log2m log2deg symmetric alpha beta push_frac delta band reg_max block_max "
                    "task_work orient ms\n");
    for (const apspie_tune_entry &e : ctx->tune_table)
        std::fprintf(f, "%d %d %d %d %.9g %.9g %.9g %d %lld %d %d %d %d %.6f\n", e.kind, e.log_m, e.log_deg,
                     e.symmetric, e.p.bfs_alpha, e.p.bfs_beta, e.p.batch_push_frac, e.p.sssp_delta,
                     static_cast<long long>(e.p.sssp_band), e.p.spgemm_reg_max, e.p.spgemm_block_max,
                     e.p.tc_task_work, e.p.tc_orient, e.ms);
    const bool ok = std::fclose(f) == 0;
    return ok ? APSPIE_OK : APSPIE_ERR_INVALID_ARG;
}

apspie_status apspie_tune_load(apspie_ctx *ctx, const char *path) {
    if (!ctx || !path) return APSPIE_ERR_INVALID_ARG;
    FILE *f = std::fopen(path, "r");
    if (!f) return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string("apspie_tune_load: cannot open ") + path);
    char line[512];
    bool header = false;
    std::vector<apspie_tune_entry> got;
    while (std::fgets(line, sizeof(line), f)) {
        if (!header) {
            if (std::strncmp(line, "apspie-tune 1", 13) != 0) break;
            header = true;
            continue;
        }
        if (line[0] == '#' || line[0] == '\n') continue;
        apspie_tune_entry e;
        std::memset(&e, 0, sizeof(e));
        long long band = 0;
        const int n = std::sscanf(line, "%d %d %d %d %f %f %f %d %lld %d %d %d %d %lf", &e.kind, &e.log_m,
                                  &e.log_deg, &e.symmetric, &e.p.bfs_alpha, &e.p.bfs_beta, &e.p.batch_push_frac,
                                  &e.p.sssp_delta, &band, &e.p.spgemm_reg_max, &e.p.spgemm_block_max,
                                  &e.p.tc_task_work, &e.p.tc_orient, &e.ms);
        e.p.sssp_band = band;
        if (n != 14 || e.kind < 0 || e.kind > APSPIE_TUNE_TC || !params_valid(e.p)) {
            std::fclose(f);
            return set_error(ctx, APSPIE_ERR_INVALID_ARG, std::string("apspie_tune_load: bad line: ") + line);
        }
        got.push_back(e);
    }
    std::fclose(f);
    if (!header) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_tune_load: not a tuning file");
    for (const apspie_tune_entry &e : got) {
        Bucket b{e.kind, e.log_m, e.log_deg, e.symmetric};
        record(ctx, b, e.p, e.ms);
    }
    return APSPIE_OK;
}

apspie_status apspie_autotune(apspie_ctx *ctx, int32_t kind, const apspie_csr *A, const apspie_csr *B,
                              const int32_t *sources, int32_t nsources, int32_t reps,
                              apspie_tune_params *best, double *best_ms) {
    if (!ctx || !A || kind < 0 || kind > APSPIE_TUNE_TC) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (reps <= 0) reps = 3;
    const bool sym = (A->flags & APSPIE_CSR_SYMMETRIC) != 0;
    const apspie_tune_params saved = own_params(ctx);
    const int saved_use = ctx->use_tuning;
    std::vector<apspie_tune_params> cands;
    auto with = [&](auto edit) {
        apspie_tune_params p = saved;
        edit(p);
        cands.push_back(p);
    };
    TuneBuffers buf;
    // run(p) performs one call of `kind` with the context's knobs set to p
    std::function<apspie_status()> run;
    int32_t *d_out = nullptr, *d_src = nullptr, *crp = nullptr, *cci = nullptr;
    void *cval = nullptr;
    switch (kind) {
    case APSPIE_TUNE_BFS:
    case APSPIE_TUNE_SSSP: {
        if (!sources || nsources < 1 || sources[0] < 0 || sources[0] >= A->m)
            return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_autotune: need a source in range");
        if (!(d_out = buf.get<int32_t>(A->m))) return set_error(ctx, APSPIE_ERR_OOM, "apspie_autotune: output");
        const int src = sources[0];
        if (kind == APSPIE_TUNE_BFS) {
            with([](apspie_tune_params &p) { p.bfs_alpha = 0.0f; });  // push only
            if (sym)
                for (float a : {4.0f, 8.0f, 14.0f, 24.0f, 48.0f})
                    for (float b : {12.0f, 24.0f, 64.0f})
                        with([&](apspie_tune_params &p) {
                            p.bfs_alpha = a;
                            p.bfs_beta = b;
                        });
            run = [&, src]() { return apspie_bfs(ctx, A, src, 0, d_out, nullptr); };
        } else {
            with([](apspie_tune_params &p) {
                p.sssp_band = -1;
                p.sssp_delta = 0;
            });
            for (int sh : {6, 5, 4, 3, 2, 1})
                with([&](apspie_tune_params &p) {
                    p.sssp_band = std::max<long long>(static_cast<long long>(A->nnz) >> sh, 1LL << 14);
                    p.sssp_delta = 0;
                });
            run = [&, src]() { return apspie_sssp(ctx, A, src, d_out, nullptr); };
        }
        break;
    }
    case APSPIE_TUNE_BFS_BATCH: {
        if (!sources || nsources < 1)
            return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_autotune: need sources");
        for (int q = 0; q < nsources; ++q)
            if (sources[q] < 0 || sources[q] >= A->m)
                return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_autotune: source out of range");
        if (!(d_src = buf.get<int32_t>(nsources)) ||
            !(d_out = buf.get<int32_t>(static_cast<size_t>(nsources) * A->m)))
            return set_error(ctx, APSPIE_ERR_OOM, "apspie_autotune: batch buffers");
        if (cudaMemcpy(d_src, sources, nsources * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
            return set_error(ctx, APSPIE_ERR_CUDA, "apspie_autotune: source copy");
        if (sym)
            for (float f : {0.005f, 0.01f, 0.02f, 0.05f, 0.1f, 0.2f})
                with([&](apspie_tune_params &p) { p.batch_push_frac = f; });
        with([](apspie_tune_params &p) { p.batch_push_frac = 1e30f; });  // push only
        run = [&, nsources]() { return apspie_bfs_batch(ctx, A, d_src, nsources, 0, d_out, nullptr); };
        break;
    }
    case APSPIE_TUNE_SPGEMM: {
        if (!B) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_autotune: SpGEMM needs B");
        if (!(crp = buf.get<int32_t>(static_cast<size_t>(A->m) + 1)))
            return set_error(ctx, APSPIE_ERR_OOM, "apspie_autotune: row_ptr");
        int64_t nnz = 0;
        apspie_status st = apspie_spgemm_symbolic(ctx, A, B, crp, &nnz);
        if (st != APSPIE_OK) return st;
        if (!(cci = buf.get<int32_t>(static_cast<size_t>(nnz))) || !(cval = buf.get<int32_t>(static_cast<size_t>(nnz))))
            return set_error(ctx, APSPIE_ERR_OOM, "apspie_autotune: C");
        for (int r : {0, 32, 64, 128})
            for (int bm : {256, 1024})
                with([&](apspie_tune_params &p) {
                    p.spgemm_reg_max = r;
                    p.spgemm_block_max = bm;
                });
        run = [&]() {
            int64_t n2 = 0;
            apspie_status s2 = apspie_spgemm_symbolic(ctx, A, B, crp, &n2);
            if (s2 != APSPIE_OK) return s2;
            return apspie_spgemm_numeric(ctx, A, B, crp, cci, cval);
        };
        break;
    }
    case APSPIE_TUNE_TC: {
        for (int o : {1, 0})
            for (int tw : {1024, 2048, 4096, 8192, 16384})
                with([&](apspie_tune_params &p) {
                    p.tc_orient = o;
                    p.tc_task_work = tw;
                });
        run = [&]() {
            int64_t cnt = 0;
            return apspie_tc(ctx, A, &cnt);
        };
        break;
    }
    default:
        return APSPIE_ERR_INVALID_ARG;
    }

    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return set_error(ctx, APSPIE_ERR_CUDA, "apspie_autotune: events");
    ctx->use_tuning = 0;  // candidates run with exactly their own knobs
    apspie_status st = APSPIE_OK;
    double best_t = 1e300;
    apspie_tune_params best_p = saved;
    for (const apspie_tune_params &p : cands) {
        apply_params(ctx, p);
        if ((st = run()) != APSPIE_OK) break;  // warm-up (and plan / scratch sizing)
        std::vector<double> ts;
        for (int r = 0; r < reps && st == APSPIE_OK; ++r) {
            cudaEventRecord(e0, ctx->stream);
            st = run();
            cudaEventRecord(e1, ctx->stream);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            ts.push_back(ms);
        }
        if (st != APSPIE_OK) break;
        std::sort(ts.begin(), ts.end());
        const double med = ts[ts.size() / 2];
        if (med < best_t) {
            best_t = med;
            best_p = p;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply_params(ctx, saved);
    ctx->use_tuning = saved_use;
    if (st != APSPIE_OK) return st;
    // the table entry carries the chosen knobs of this kind; the rest are the context's
    apspie_tune_params rec = saved;
    take_kind(rec, best_p, kind);
    record(ctx, bucket_of(kind, A), rec, best_t);
    if (best) *best = rec;
    if (best_ms) *best_ms = best_t;
    return APSPIE_OK;
}

}  // extern "C"
