/*
 * apspie.h -- C ABI of the B200 (sm_100a) SpMSpV / hash-SpGEMM graph library.
 *
 * Every pointer named d_* is DEVICE memory on the context's GPU; h_* is host memory.
 * All CSR structures are int32 (row offsets and column indices), as in the reference's
 * d_matrix container (src/matrix.hpp:6-37: d_cscColPtr / d_cscRowInd / d_cscVal, which
 * hold CSR despite their names).
 *
 * Conventions shared by every entry point:
 *  - Calls never exit the process. They return an apspie_status; the message of the
 *    last failure on a context is apspie_ctx_last_error(ctx).
 *  - The caller owns input and output arrays. Scratch (frontier queues, bitmaps, hash
 *    tables) is owned by the context, reused across calls and grown on demand; there is
 *    no per-level or per-iteration allocation.
 *  - Calls are enqueued on the context's stream. Those that return a host scalar
 *    (triangle count, nnz(C), run statistics) synchronise that stream.
 *  - A context is not thread-safe; distinct contexts are independent.
 *  - Termination is decided on the device (empty frontier / no change). The reference's
 *    `depth` argument is kept as a level cap: depth <= 0 means unlimited.
 */
#ifndef APSPIE_H
#define APSPIE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum apspie_status {
    APSPIE_OK = 0,
    APSPIE_ERR_INVALID_ARG = 1,   /* bad pointer, size, source, or CSR contents */
    APSPIE_ERR_OOM = 2,           /* device allocation failed */
    APSPIE_ERR_HASH_OVERFLOW = 3, /* a hash table ran out of probes (spgemmKernel.cuh:335) */
    APSPIE_ERR_TIMEOUT = 4,       /* a bounded device-side wait ran out */
    APSPIE_ERR_CUDA = 5,          /* a CUDA runtime call failed */
    APSPIE_ERR_UNSUPPORTED = 6,   /* valid request this build does not serve */
    APSPIE_ERR_NOT_CONVERGED = 7  /* iteration cap reached before the fixed point */
} apspie_status;

typedef enum apspie_val_type {
    APSPIE_VAL_NONE = 0, /* pattern only (boolean semiring) */
    APSPIE_VAL_F32 = 1,
    APSPIE_VAL_I32 = 2
} apspie_val_type;

/* apspie_csr.flags */
enum {
    /* The caller asserts that the pattern is symmetric (an undirected graph, as built by
     * the reference's makeSymmetric). Enables bottom-up (pull) BFS levels, which scan a
     * vertex's own row for parents; without it BFS expands top-down only. */
    APSPIE_CSR_SYMMETRIC = 1u
};

/* Device-resident CSR matrix view (not owned). */
typedef struct apspie_csr {
    int32_t m;             /* rows */
    int32_t n;             /* columns */
    int32_t nnz;           /* stored entries */
    int32_t val_type;      /* apspie_val_type of `val` */
    const int32_t *row_ptr; /* d, m+1 */
    const int32_t *col_ind; /* d, nnz */
    const void *val;        /* d, nnz elements of val_type, or NULL */
    uint32_t flags;         /* APSPIE_CSR_* */
    uint32_t reserved;      /* 0 */
} apspie_csr;

/* Device-resident CSR matrix allocated by the library (spgemm output); release with
 * apspie_csr_free. Mirrors the callee-allocated C of spgemm.cuh:202-204 / tc.cuh:73,120. */
typedef struct apspie_csr_owned {
    int32_t m, n, nnz, val_type;
    int32_t *row_ptr;
    int32_t *col_ind;
    void *val;
} apspie_csr_owned;

/* Per-call statistics (filled only when a non-NULL pointer is passed; that call then
 * synchronises the stream). */
typedef struct apspie_run_stats {
    int32_t iterations;        /* BFS levels / SSSP iterations / MIS rounds executed */
    int32_t push_iterations;   /* iterations expanded top-down (push) */
    int32_t pull_iterations;   /* iterations expanded bottom-up (pull) */
    int32_t reserved;
    int64_t edges_expanded;    /* sum of deg(v) over every frontier expansion (re-expansions counted) */
    int64_t edges_component;   /* sum of deg(v) over reached vertices: the GTEPS numerator */
    int64_t vertices_reached;
} apspie_run_stats;

typedef struct apspie_ctx apspie_ctx;

/* ---- context ------------------------------------------------------------------ */

/* Creates a context on `device`, enqueuing on `cuda_stream` (a cudaStream_t; NULL = the
 * legacy default stream). Replaces the reference's mgpu::CudaContext (test/bfs/main.cu:27). */
apspie_status apspie_ctx_create(int device, void *cuda_stream, apspie_ctx **out);
void apspie_ctx_destroy(apspie_ctx *ctx);
const char *apspie_ctx_last_error(const apspie_ctx *ctx);
apspie_status apspie_ctx_synchronize(apspie_ctx *ctx);
/* Pre-sizes the scratch arena for graphs up to m vertices and nnz entries. */
apspie_status apspie_ctx_reserve(apspie_ctx *ctx, int32_t m, int64_t nnz);
/* When on (default off), every traversal entry point first checks its CSR on the device
 * (offsets monotone, first 0, last nnz, columns in range) and returns
 * APSPIE_ERR_INVALID_ARG instead of touching a malformed graph. */
apspie_status apspie_ctx_set_validate(apspie_ctx *ctx, int on);
/* Direction-switch thresholds for BFS (Beamer's alpha/beta; defaults 14 and 24).
 * alpha <= 0 forces push on every level. */
apspie_status apspie_ctx_set_bfs_tuning(apspie_ctx *ctx, float alpha, float beta);
/* SSSP far-pile threshold step (delta-stepping "near/far" buckets). delta <= 0 (default):
 * no far pile when the distance band is on (below), else 32 * mean weight / mean degree
 * from a sample of the weights. */
apspie_status apspie_ctx_set_sssp_delta(apspie_ctx *ctx, int32_t delta);
/* SSSP distance band: each iteration expands only the frontier vertices of lowest
 * distance whose edges add up to about `edges` (the rest wait in the frontier), chosen
 * from a degree-weighted distance histogram gathered on the device. edges == 0 (default):
 * nnz / 8 clamped to [2^18, 2^23]; edges < 0: off (expand the whole frontier). */
apspie_status apspie_ctx_set_sssp_band(apspie_ctx *ctx, int64_t edges);
/* Batched SSSP: <= 0 = the multi-query kernel (default); > 0 = that many query groups,
 * each running the single-source kernel on its share of the sources. */
apspie_status apspie_ctx_set_sssp_batch_groups(apspie_ctx *ctx, int32_t groups);
/* Batched BFS direction switch: a level expands top-down while (active vertices x mean
 * degree) < frac * nnz, else bottom-up (default 0.05; bottom-up only on symmetric graphs). */
apspie_status apspie_ctx_set_batch_push_frac(apspie_ctx *ctx, float frac);
/* Caps the number of co-resident blocks of the persistent traversal kernels
 * (0 = as many as fit). */
apspie_status apspie_ctx_set_max_grid(apspie_ctx *ctx, int32_t max_blocks);
/* Bound of every device-side wait of this context's persistent kernels (the grid barrier
 * between their phases), in nanoseconds; ns <= 0 restores the default of 4 s. A wait that
 * runs out raises APSPIE_ERR_TIMEOUT, every block of the launch leaves, and the call (or
 * the next apspie_ctx_synchronize) returns that status; the context stays usable. No
 * reference counterpart (the reference synchronises on the host every level). */
apspie_status apspie_ctx_set_wait_limit(apspie_ctx *ctx, int64_t ns);
/* Health check of the persistent-kernel machinery on this context's device and stream:
 * one cooperative grid as large as the traversal kernels use passes `rounds` grid
 * barriers. With absent_block >= 0 that block leaves before its first arrival, so the
 * others' wait runs out after the context's wait limit and the call returns
 * APSPIE_ERR_TIMEOUT -- the timeout path exercised without disturbing the GPU. *grid (may
 * be NULL) receives the number of blocks launched. Synchronous. */
apspie_status apspie_grid_barrier_check(apspie_ctx *ctx, int32_t rounds, int32_t absent_block, int32_t *grid);
/* Phase timeline of the last traversal call made with a stats pointer: for each grid
 * barrier block 0 passed (up to 128), the barrier's site code and the nanoseconds since the
 * kernel started (globaltimer). Site 0 is the kernel start. */
apspie_status apspie_ctx_timeline(const apspie_ctx *ctx, int32_t *sites, int64_t *ns, int32_t cap,
                                  int32_t *count);
/* Bytes of device scratch the context currently holds. */
int64_t apspie_ctx_scratch_bytes(const apspie_ctx *ctx);

/* ---- autotuner ------------------------------------------------------------------ */

/* The knobs the autotuner picks. A context holds one set of its own (the set_* calls
 * above and apspie_ctx_set_params) and a tuning table of sets recorded per (kind, shape
 * bucket); a call whose input falls in a recorded bucket uses the recorded set for the
 * knobs of its kind (unless apspie_ctx_set_autotune(ctx, 0)). No reference counterpart:
 * the reference's thresholds are compile-time constants. */
typedef struct apspie_tune_params {
    float bfs_alpha;          /* BFS push -> pull when frontier edges > unvisited edges / alpha */
    float bfs_beta;           /* BFS pull -> push when frontier < m / beta */
    float batch_push_frac;    /* batched BFS: push while frontier edges < frac * nnz */
    int32_t sssp_delta;       /* SSSP far-pile step (<= 0: none with the band, else device-chosen) */
    int64_t sssp_band;        /* SSSP edges per iteration (0 auto, < 0 whole frontier) */
    int32_t spgemm_reg_max;   /* SpGEMM rows with at most this many products (0, 32, 64 or 128)
                                 are sorted by one warp in registers */
    int32_t spgemm_block_max; /* larger rows up to this many products (<= 1024) use a block's
                                 shared-memory hash table; longer rows a global table */
    int32_t tc_task_work;     /* triangle counting: wedges per warp task (>= 256) */
    int32_t tc_orient;        /* triangle counting: 1 = re-orient L by degree first */
    int32_t reserved[4];
} apspie_tune_params;

enum {
    APSPIE_TUNE_BFS = 0,
    APSPIE_TUNE_SSSP = 1,
    APSPIE_TUNE_BFS_BATCH = 2,
    APSPIE_TUNE_SPGEMM = 3,
    APSPIE_TUNE_TC = 4
};

apspie_status apspie_ctx_get_params(const apspie_ctx *ctx, apspie_tune_params *out);
/* Replaces the context's own knobs (validated: APSPIE_ERR_INVALID_ARG if out of range). */
apspie_status apspie_ctx_set_params(apspie_ctx *ctx, const apspie_tune_params *p);
/* use != 0 (default): calls consult the tuning table; 0: only the context's own knobs. */
apspie_status apspie_ctx_set_autotune(apspie_ctx *ctx, int32_t use);
/* Times every candidate setting of `kind`'s knobs on this input (reps timed runs each,
 * after one warm-up; the median counts), records the fastest for the input's shape
 * bucket and returns it in *best (and its median milliseconds in *best_ms). Inputs:
 * BFS/SSSP: A and host `sources[0]`; BFS_BATCH: A and `nsources` host sources; SPGEMM:
 * A and B; TC: A = strict lower triangle. Output buffers are allocated for the duration
 * of the call. Candidates: BFS alpha x beta; SSSP band sizes; batched BFS push fraction;
 * SpGEMM register-tier limit x shared-table limit; TC task size x orientation. */
apspie_status apspie_autotune(apspie_ctx *ctx, int32_t kind, const apspie_csr *A, const apspie_csr *B,
                              const int32_t *sources, int32_t nsources, int32_t reps,
                              apspie_tune_params *best, double *best_ms);
/* The tuning table: entries, lookup of the set a call on A would use, and persistence as
 * a text file (one entry per line; load merges, replacing entries of the same bucket). */
int32_t apspie_tune_entries(const apspie_ctx *ctx);
apspie_status apspie_tune_lookup(const apspie_ctx *ctx, int32_t kind, const apspie_csr *A,
                                 apspie_tune_params *out, int32_t *found);
apspie_status apspie_tune_save(const apspie_ctx *ctx, const char *path);
apspie_status apspie_tune_load(apspie_ctx *ctx, const char *path);

/* Checks a CSR on the device; APSPIE_OK or APSPIE_ERR_INVALID_ARG. */
apspie_status apspie_csr_validate(apspie_ctx *ctx, const apspie_csr *A);

/* ---- traversal (SpMSpV) --------------------------------------------------------- */

/* Level-synchronous BFS by boolean OR-AND SpMSpV with a push/pull switch (pull only
 * when A->flags has APSPIE_CSR_SYMMETRIC).
 * d_depth[m] (int32, caller-allocated): hop count from `source`, -1 unreached.
 * Replaces spmspvBfs (src/spmspvBfs.cuh:96) and bfs<T> (src/bfs.cuh:33). */
apspie_status apspie_bfs(apspie_ctx *ctx, const apspie_csr *A, int32_t source,
                         int32_t depth_cap, int32_t *d_depth, apspie_run_stats *stats);

/* Single-source shortest paths by min-plus SpMSpV over int32 edge weights >= 0
 * (A->val_type == APSPIE_VAL_I32), iterated on the device to the fixed point, each
 * iteration expanding the frontier's lowest-distance band (apspie_ctx_set_sssp_band).
 * d_dist[m] (int32): distance, -1 unreached (the CPU check's convention,
 * src/testSssp.cpp:50). Replaces sssp<Value> (src/sssp.cuh:28) and
 * spmspvSssp (src/spmspvSssp.cuh:92). Returns APSPIE_ERR_INVALID_ARG when a path
 * length would exceed INT32_MAX - 1. */
apspie_status apspie_sssp(apspie_ctx *ctx, const apspie_csr *A, int32_t source,
                          int32_t *d_dist, apspie_run_stats *stats);

/* Maximal independent set with fixed priorities: the set a priority-thresholded Luby
 * loop converges to (src/spmspvMis.cuh:149-344), i.e. the greedy MIS in descending
 * (priority, vertex id) order. d_member[m] (uint8): 1 in the set, 0 not. A must be
 * symmetric; self-loops are ignored. */
apspie_status apspie_mis(apspie_ctx *ctx, const apspie_csr *A, const uint32_t *d_priority,
                         uint8_t *d_member, apspie_run_stats *stats);

/* Batched multi-source BFS: num_sources queries on one resident graph, up to 512 per
 * persistent launch (query-bit SpMSpM levels, push/pull by frontier size). d_depths is
 * num_sources x m int32, query-major (row q = the depth vector apspie_bfs returns for
 * d_sources[q]); -1 unreached. Sources may repeat. */
apspie_status apspie_bfs_batch(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources,
                               int32_t num_sources, int32_t depth_cap, int32_t *d_depths,
                               apspie_run_stats *stats);

/* Batched multi-source SSSP over int32 weights in one persistent launch. d_dists is
 * num_sources x m int32, query-major (row q = what apspie_sssp returns for d_sources[q]);
 * -1 unreached. By default a multi-query kernel relaxes all changed queries of a frontier
 * row together, one warp per edge with a lane per query over vertex-major labels
 * (32*W queries per launch with (nnz + m) * W < 2^31, W <= 16; device scratch about
 * 160 * m * W bytes). With apspie_ctx_set_sssp_batch_groups(ctx, g > 0) the launch's blocks
 * split into g query groups instead, each running the single-source kernel on its share. */
apspie_status apspie_sssp_batch(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_sources,
                                int32_t num_sources, int32_t *d_dists, apspie_run_stats *stats);

/* BFS that allocates nothing, for callers that cannot call cudaMalloc: code running where
 * device allocation is forbidden or unavailable (inside another allocator's memory budget,
 * a host that reserves all device memory up front, a plugin loaded into such a process).
 * No reference counterpart: the reference has only allocating entry points.
 * Same semantics and outputs as apspie_bfs, on the CURRENT device and the given stream,
 * with no context. Its scratch (frontier queues, bitmaps, control block, about 4.3 MB) is a
 * fixed device array inside the library that every GPU which loads the library holds until
 * the process exits; graphs above APSPIE_NOALLOC_MAX_VERTICES vertices are rejected with
 * APSPIE_ERR_INVALID_ARG. The first call in each CUDA context (the device's primary
 * context, a context made with cuCtxCreate, or a primary context re-created after
 * cudaDeviceReset) looks the array's address up with cudaGetSymbolAddress, so make that
 * first call before any stream capture. Under lazy module loading (CUDA_MODULE_LOADING=LAZY,
 * the default since CUDA 12.2) that first call is also what loads the library's device
 * code and the 4.3 MB array into the context: a host that reserves all free device memory
 * up front should make one call first (or run with CUDA_MODULE_LOADING=EAGER), else the
 * first call can fail with APSPIE_ERR_CUDA for want of memory. All calls share the one
 * array: calls that overlap on the GPU (other streams, other host threads) race and
 * corrupt each other; serialise them. Synchronises `cuda_stream` and returns any
 * device-side error; `stats` may be NULL. */
#define APSPIE_NOALLOC_MAX_VERTICES 262144
apspie_status apspie_bfs_noalloc(const apspie_csr *A, int32_t source, int32_t depth_cap,
                                 int32_t *d_depth, void *cuda_stream, apspie_run_stats *stats);

/* apspie_sssp over float32 weights >= 0 (A->val_type == APSPIE_VAL_F32): float32
 * distances, each the fixed point min over paths of float sums (independent of the order
 * relaxations land, as the reference's CPU ssspCPU computes it); unreached vertices get
 * `unreached` (the reference GPU path leaves 1.70141e+38, src/sssp.cuh:48; its CPU check
 * uses -1, src/testSssp.cpp:50). */
apspie_status apspie_sssp_f32(apspie_ctx *ctx, const apspie_csr *A, int32_t source, float *d_dist,
                              float unreached, apspie_run_stats *stats);

/* apspie_mis writing the reference's int32 result layout (1 in the set, 0 not;
 * d_misResult of spmspvMis, src/spmspvMis.cuh:150). */
apspie_status apspie_mis_int32(apspie_ctx *ctx, const apspie_csr *A, const uint32_t *d_priority,
                               int32_t *d_mis_result, apspie_run_stats *stats);

/* One-hop boolean SpMSpV y = A^T x over a dense 0/1 int32 vector: d_y[v] = 1 if some
 * u with d_x[u] != 0 has v in its row, else 0. Replaces spmspvCsr
 * (src/spmspvMis.cuh:81), the reference's MIS validity helper. */
apspie_status apspie_spmspv_bool(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_x,
                                 int32_t *d_y);

/* Valued sparse-in / sparse-out SpMSpV y = x^T A: x has x_nnz entries (row index
 * d_x_ind[j] of A, value d_x_val[j], in A's value type, F32 or I32; repeated indices add);
 * y gets one entry per column that some product lands in, d_y_ind ascending and d_y_val
 * the sum of that column's products (a column whose products cancel keeps a 0 entry), and
 * *y_nnz their number. d_y_ind / d_y_val must hold min(n, sum of x's row lengths)
 * entries. Each sum is taken in x's entry order, then A's row order, with correctly
 * rounded f32 multiplies and adds (no fused multiply-add; int32 wraps), so it is
 * bit-identical to that sequential loop. Synchronises the context's stream. Replaces
 * mXv<T> (src/mXv.cuh:249-389: IntervalGather of the vector's CSC columns, elementMult,
 * SortPairs, ReduceByKey). An index outside [0, m) is APSPIE_ERR_INVALID_ARG. */
apspie_status apspie_spmspv(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_x_ind, const void *d_x_val,
                            int32_t x_nnz, int32_t *d_y_ind, void *d_y_val, int32_t *y_nnz);

/* Checksums of result rows, to check many answers against a reference without copying
 * them to the host: for each k < nrows, d_out[h_slots[k]] += sum_i row_k[i] * d_coef[i]
 * over i < m, with row_k = h_rows[k] (device memory; int32 elements for elem_bytes 4,
 * uint8 for 1), int32 products (wrapping) and an exact int64 sum, so the value does not
 * depend on the order of the additions. h_rows / h_slots are host arrays; zero the d_out
 * slots first. Asynchronous on the context's stream. No reference counterpart (the
 * reference compares whole result vectors on the host, src/util.cuh:260-269). */
apspie_status apspie_row_checksums(apspie_ctx *ctx, const void *const *h_rows, const int32_t *h_slots,
                                   int32_t nrows, int32_t m, int32_t elem_bytes, const int32_t *d_coef,
                                   int64_t *d_out);

/* ---- SpGEMM and triangle counting ---------------------------------------------- */

/* C = A * B, row-binned hash Gustavson. A and B share val_type (F32 or I32). C's rows are
 * sorted by column; int32 values are exact; FP32 values of rows with at most 128 products
 * are summed in increasing position of A's row (deterministic), longer rows accumulate by
 * atomicAdd (summation order only). The library allocates C (release with
 * apspie_csr_free); synchronises. Replaces spgemm(d_matrix*, d_matrix*, d_matrix*, partSize,
 * partNum, ctx) (src/spgemm.cuh:132), spgemm<T>(d_matrix*...) (src/spgemm.cuh:346) and
 * spgemm<T>(edge, m, ..., T*&, int*&, int*&) (src/tc.cuh:63). */
apspie_status apspie_spgemm(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B,
                            apspie_csr_owned *C);
/* Two-step form with caller-owned C: symbolic fills d_row_ptr_c[A->m + 1] and *nnz_c
 * (synchronises); numeric fills d_col_c[nnz] and d_val_c[nnz] (A's val_type). */
apspie_status apspie_spgemm_symbolic(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B,
                                     int32_t *d_row_ptr_c, int64_t *nnz_c);
apspie_status apspie_spgemm_numeric(apspie_ctx *ctx, const apspie_csr *A, const apspie_csr *B,
                                    const int32_t *d_row_ptr_c, int32_t *d_col_c, void *d_val_c);
void apspie_csr_free(apspie_csr_owned *C);

/* ---- graph construction on the device ---------------------------------------------- */

enum {
    APSPIE_BUILD_SYMMETRIZE = 1,       /* store {u, v} in both rows (canonical pair lo < hi) */
    APSPIE_BUILD_DROP_SELF_LOOPS = 2,  /* drop edges u == v */
    APSPIE_BUILD_DEDUP = 4             /* keep the first occurrence of each pair (input order) */
};

/* Builds a CSR with sorted rows from nedges device COO edges (d_src[k], d_dst[k], optional
 * 32-bit values d_val[k] of val_type). With SYMMETRIZE | DROP_SELF_LOOPS | DEDUP it applies
 * the rules of the host R-MAT generator and makeSymmetric: self-loops dropped, each
 * unordered pair kept once with the value of its first occurrence, then mirrored; row r
 * lists its lower neighbours then its upper ones, ascending. The output is allocated by
 * the callee (apspie_csr_free). Replaces makeSymmetric + buildMatrix
 * (src/util.cuh:573-643, src/matrix.cpp:55-111) for graphs already in device memory.
 * Synchronises. */
apspie_status apspie_csr_build(apspie_ctx *ctx, int32_t m, int64_t nedges, const int32_t *d_src,
                               const int32_t *d_dst, const void *d_val, int32_t val_type, int32_t flags,
                               apspie_csr_owned *out);
/* CSR -> CSC (the transpose as a CSR of n rows), rows sorted; values follow their entries.
 * Replaces csr2csc (src/util.cuh:474) and extract_csr2csc (src/matrix.cpp:229).
 * Synchronises. */
apspie_status apspie_csr_transpose(apspie_ctx *ctx, const apspie_csr *A, apspie_csr_owned *out);

/* ---- dense-vector SpMV and PageRank -------------------------------------------------- */

/* y = alpha * A * x + beta * y (float32; A with float32 values, or a pattern of 1.0s).
 * Replaces SpmvCsrBinary (src/bfs.cuh:11-14) and cuspmv (src/tc.cuh:17-59). */
apspie_status apspie_spmv(apspie_ctx *ctx, const apspie_csr *A, const float *d_x, float *d_y, float alpha,
                          float beta);
/* PageRank of the directed graph A (row u lists u's out-edges): r = 1/n initially, then
 * r' = (1 - damping) / n + damping * (sum over in-edges (u, v) of r[u] / outdeg(u)
 * + (rank mass of vertices without out-edges) / n), until sum |r' - r| < tol or max_iter
 * iterations (*iterations reports how many ran). d_rank: float32[m], so a tol below what
 * float32 ranks resolve (about 1e-7 summed over the graph) runs all max_iter iterations.
 * Synchronises once per iteration. No reference counterpart (the reference ships
 * test_pr.mtx only). */
apspie_status apspie_pagerank(apspie_ctx *ctx, const apspie_csr *A, float damping, double tol, int32_t max_iter,
                              float *d_rank, int32_t *iterations);

/* Triangle count = sum((L*L) .* L) for L the strict lower triangle (column < row) of a
 * symmetric graph, rows sorted; masked hash SpGEMM, L*L never materialised; int64 result
 * (synchronises). Replaces the flow of test/tc/main.cu:243-249 (spgemm<T> tc.cuh:63 ->
 * ewiseMultTc tc.cuh:169 -> mgpu::Reduce). */
apspie_status apspie_tc(apspie_ctx *ctx, const apspie_csr *L, int64_t *count);
/* Strict lower triangle of a square CSR on the device (buildLower, test/tc/main.cu:39-55,
 * in CSR); library-allocated, release with apspie_csr_free. Values are dropped. */
apspie_status apspie_csr_strict_lower_device(apspie_ctx *ctx, const apspie_csr *A,
                                             apspie_csr_owned *L);

#ifdef __cplusplus
}
#endif

#endif /* APSPIE_H */
