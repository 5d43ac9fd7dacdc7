/*
 * apspie_host.h -- host-side (CPU) graph construction of the apspie B200 library:
 * Matrix Market loading with the reference's semantics, synthetic R-MAT / Erdos-Renyi
 * generators, and small CSR utilities. Arrays here are HOST memory, allocated by the
 * library and released with apspie_host_csr_free.
 */
#ifndef APSPIE_HOST_H
#define APSPIE_HOST_H

#include <stdint.h>

#include "apspie.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct apspie_host_csr {
    int32_t m, n, nnz, val_type; /* val_type: apspie_val_type */
    int32_t *row_ptr;            /* m+1 */
    int32_t *col_ind;            /* nnz */
    void *val;                   /* nnz elements of val_type, or NULL */
} apspie_host_csr;

void apspie_host_csr_free(apspie_host_csr *g);

/* Loads a Matrix Market file with the reference loader's semantics (src/util.cuh:355-430
 * readEdge/readMtx, :572-643 makeSymmetric, src/matrix.cpp:55-111 buildMatrix):
 * lines starting with '%' are skipped; header "m n nnz"; each entry is read as
 * (column, row) 1-based, so CSR row r holds the entries whose SECOND number is r+1;
 * an entry is weighted (float) iff the first entry line has a blank after its two
 * integers, else every value is 1.0. undirected != 0 mirrors every non-loop entry,
 * sorts by (row, col) and drops repeated pairs (self-loops kept), as makeSymmetric does;
 * otherwise rows keep file order. Values are returned as float (val_type F32). */
apspie_status apspie_load_mtx(const char *path, int undirected, apspie_host_csr *out);
/* The same loader with the entry lines parsed and the pairs sorted on `threads` host
 * threads (0 = all); one entry per line assumed, as in every Matrix Market file. Same
 * result as apspie_load_mtx. No reference counterpart (the reference parses with fscanf on
 * one thread, src/util.cuh:370-430). */
apspie_status apspie_load_mtx_threads(const char *path, int undirected, int threads, apspie_host_csr *out);

/* Undirected R-MAT graph: 2^scale vertices, edge_factor * 2^scale generated edges.
 * Edge k (k = 0, 1, ...) takes `scale` draws of std::mt19937(seed) through
 * std::uniform_real_distribution<double>(0,1), most significant bit first; each draw
 * picks the quadrant (r < a: 00, r < a+b: 01, r < a+b+c: 10, else 11) whose first bit
 * goes to the row u and second to the column v. Self-loops are dropped, {u,v} is
 * canonicalised and the first generated copy of each pair kept; its weight is draw k of
 * std::mt19937(weight_seed) through std::uniform_int_distribution<int>(1,255) (one draw
 * per generated edge, self-loops included). The pair is stored in both directions with
 * the same weight; rows are sorted by column. with_weights = 0 returns no values. */
apspie_status apspie_gen_rmat(int scale, int edge_factor, uint32_t seed, uint32_t weight_seed,
                              double a, double b, double c, int with_weights,
                              apspie_host_csr *out);
/* The generated edge list itself, in generation order, before self-loops are dropped and
 * pairs deduplicated: src/dst/weight[k] for k < 2^scale * edge_factor (weight may be NULL).
 * apspie_csr_build with SYMMETRIZE | DROP_SELF_LOOPS | DEDUP turns it into exactly the CSR
 * apspie_gen_rmat returns. */
apspie_status apspie_gen_rmat_coo(int scale, int edge_factor, uint32_t seed, uint32_t weight_seed, double a,
                                  double b, double c, int32_t *src, int32_t *dst, int32_t *weight);

/* Erdos-Renyi matrix with exactly k distinct uniformly random columns per row: row by row,
 * draws of std::mt19937(seed) through std::uniform_int_distribution<int>(0, n-1), repeats
 * rejected, then sorted. Values continue the same engine in CSR order:
 * F32 -> std::uniform_real_distribution<float>(-1,1), I32 -> uniform_int_distribution<int>(1,8),
 * NONE -> no values. */
apspie_status apspie_gen_er(int n, int k, uint32_t seed, int val_type, apspie_host_csr *out);

/* count outputs of std::mt19937(seed) (identical to the reference's init_genrand(seed) +
 * genrand_int32(), src/mt19937ar.cpp:57,102). */
apspie_status apspie_mt19937_u32(uint32_t seed, int64_t count, uint32_t *out);

/* Vertex of maximum degree, smallest id on ties. */
int32_t apspie_max_degree_vertex(const apspie_host_csr *g);

/* `count` distinct vertices of the largest connected component (ties: the component with
 * the smallest vertex id), drawn without replacement from its sorted vertex list by a
 * partial Fisher-Yates shuffle driven by std::mt19937(seed) through
 * std::uniform_int_distribution<int64_t>(i, size-1). */
apspie_status apspie_lcc_sample(const apspie_host_csr *g, int32_t count, uint32_t seed,
                                int32_t *out);

/* Strict lower triangle L = {(i,j) in A : j < i} (the matrix B of buildLower,
 * test/tc/main.cu:39-55, in CSR). Values are dropped. */
apspie_status apspie_csr_strict_lower(const apspie_host_csr *A, apspie_host_csr *L);

#ifdef __cplusplus
}
#endif

#endif /* APSPIE_HOST_H */
