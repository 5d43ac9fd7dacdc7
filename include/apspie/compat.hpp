// compat.hpp -- the reference's C++ entry points, names and argument orders, forwarding to
// the apspie_b200 C ABI. A program written against apspie's headers (bfs.cuh,
// spmspvBfs.cuh, sssp.cuh, spmspvMis.cuh, spgemm.cuh, tc.cuh, matrix.hpp) compiles against
// this header instead and runs on the sm_100a kernels of libapspie.so.
//
// Differences a caller may notice (all deliberate, see the reference lines cited):
//  - results are exact: SSSP iterates to the fixed point rather than the CPU BFS depth
//    (src/sssp.cuh:79-98), MIS ties break by vertex id (src/spmspvMis.cuh:66);
//  - `depth` is a level cap (the reference's loop bound), <= 0 meaning unlimited;
//  - errors print one line to stderr and the call returns, as the reference's printf
//    style does, but nothing exits the process.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

#include "../apspie.h"
#include "../apspie_host.h"

namespace mgpu {

// Stand-in for moderngpu's CudaContext (test/bfs/main.cu:27): one apspie context on a
// device and stream. set_symmetric(true) tells the traversals the graph is undirected
// (what the drivers' -undirected flag produces), enabling bottom-up BFS levels.
class CudaContext {
   public:
    explicit CudaContext(int device = 0, cudaStream_t stream = nullptr) {
        if (apspie_ctx_create(device, stream, &ctx_) != APSPIE_OK) {
            std::fprintf(stderr, "apspie: cannot create a context on device %d\n", device);
            ctx_ = nullptr;
        }
    }
    ~CudaContext() { apspie_ctx_destroy(ctx_); }
    CudaContext(const CudaContext &) = delete;
    CudaContext &operator=(const CudaContext &) = delete;
    apspie_ctx *get() const { return ctx_; }
    void set_symmetric(bool s) { symmetric_ = s; }
    bool symmetric() const { return symmetric_; }

   private:
    apspie_ctx *ctx_ = nullptr;
    bool symmetric_ = false;
};

typedef std::shared_ptr<CudaContext> ContextPtr;
inline ContextPtr CreateCudaDevice(int ordinal) { return std::make_shared<CudaContext>(ordinal); }

}  // namespace mgpu

namespace apspie_compat {

inline bool report(apspie_status st, mgpu::CudaContext &c, const char *who) {
    if (st == APSPIE_OK) return true;
    std::fprintf(stderr, "%s: %s\n", who, apspie_ctx_last_error(c.get()));
    return false;
}

inline apspie_csr view(int m, int n, int nnz, const int *rp, const int *ci, const void *val, int vt,
                       bool symmetric) {
    apspie_csr a;
    a.m = m;
    a.n = n;
    a.nnz = nnz;
    a.val_type = vt;
    a.row_ptr = rp;
    a.col_ind = ci;
    a.val = val;
    a.flags = symmetric ? APSPIE_CSR_SYMMETRIC : 0u;
    a.reserved = 0u;
    return a;
}

template <typename T>
struct ValType;
template <>
struct ValType<float> {
    static const int value = APSPIE_VAL_F32;
};
template <>
struct ValType<int> {
    static const int value = APSPIE_VAL_I32;
};

inline mgpu::CudaContext &default_context() {
    static mgpu::CudaContext ctx(0);
    return ctx;
}

}  // namespace apspie_compat

// ---------------------------------------------------------------------------------
// Sparse container (src/matrix.hpp:6-37): same field names. The d_csc* arrays hold CSR
// (row offsets, column indices, values) exactly as the reference uses them.
// ---------------------------------------------------------------------------------
typedef struct matrix {
    static const int DCSC = 32;
    int *d_dcscPartPtr;
    int *d_dcscColPtr_ind;
    int *d_dcscColPtr_off;
    int *d_dcscRowInd;
    float *d_dcscVal;
    int *d_cscColInd;
    int *d_cscColPtr;
    int *d_cscRowInd;
    float *d_cscVal;
    int *h_dcscPartPtr;
    int *h_cscColPtr;
    int *h_cscRowInd;
    float *h_cscVal;
    int m;
    int n;
    int nnz;
    int part;
    int col_length;
} d_matrix;

// src/matrix.cpp:8 (the DCSC buffers of the outer-product design are not used here).
inline void matrix_new(d_matrix *A, int m, int n) {
    std::memset(A, 0, sizeof(*A));
    A->m = m;
    A->n = n;
    A->h_cscColPtr = static_cast<int *>(std::malloc((m + 1) * sizeof(int)));
    cudaMalloc(&A->d_cscColPtr, (m + 1) * sizeof(int));
}

// src/matrix.cpp:55-111: COO -> CSR by a counting sort that keeps input order in a row.
template <typename typeVal>
void buildMatrix(d_matrix *A, int numEdge, int *h_cooRowInd, int *h_cooColInd, typeVal *h_cooVal) {
    A->nnz = numEdge;
    A->h_cscRowInd = static_cast<int *>(std::malloc(std::max(numEdge, 1) * sizeof(int)));
    A->h_cscVal = static_cast<float *>(std::malloc(std::max(numEdge, 1) * sizeof(float)));
    std::vector<int> cnt(A->m + 1, 0);
    for (int i = 0; i < numEdge; ++i) ++cnt[h_cooRowInd[i]];
    int run = 0;
    for (int r = 0; r < A->m; ++r) {
        A->h_cscColPtr[r] = run;
        run += cnt[r];
    }
    A->h_cscColPtr[A->m] = run;
    std::vector<int> cur(A->h_cscColPtr, A->h_cscColPtr + A->m);
    for (int i = 0; i < numEdge; ++i) {
        const int d = cur[h_cooRowInd[i]]++;
        A->h_cscRowInd[d] = h_cooColInd[i];
        A->h_cscVal[d] = static_cast<float>(h_cooVal[i]);
    }
    cudaMalloc(&A->d_cscRowInd, std::max(numEdge, 1) * sizeof(int));
    cudaMalloc(&A->d_cscVal, std::max(numEdge, 1) * sizeof(float));
    cudaMemcpy(A->d_cscColPtr, A->h_cscColPtr, (A->m + 1) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(A->d_cscRowInd, A->h_cscRowInd, numEdge * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(A->d_cscVal, A->h_cscVal, numEdge * sizeof(float), cudaMemcpyHostToDevice);
}

inline void matrix_delete(d_matrix *A) {
    cudaFree(A->d_cscColPtr);
    if (A->d_cscRowInd) cudaFree(A->d_cscRowInd);
    if (A->d_cscVal) cudaFree(A->d_cscVal);
    std::free(A->h_cscColPtr);
    std::free(A->h_cscRowInd);
    std::free(A->h_cscVal);
    A->d_cscColPtr = A->d_cscRowInd = nullptr;
    A->d_cscVal = nullptr;
}

// ---------------------------------------------------------------------------------
// Traversals
// ---------------------------------------------------------------------------------

// src/bfs.cuh:33 (float-semiring BFS over CSC arrays; d_cscValA unused).
template <typename T>
void bfs(const int vertex, const int edge, const int m, const T *d_cscValA, const int *d_cscColPtrA,
         const int *d_cscRowIndA, int *d_bfsResult, const int depth, mgpu::CudaContext &context) {
    (void)d_cscValA;
    apspie_csr a = apspie_compat::view(m, m, edge, d_cscColPtrA, d_cscRowIndA, nullptr, APSPIE_VAL_NONE,
                                       context.symmetric());
    apspie_compat::report(apspie_bfs(context.get(), &a, vertex, depth, d_bfsResult, nullptr), context, "bfs");
}

// src/spmspvBfs.cuh:96 (boolean SpMSpV BFS; h_csrRowPtr unused).
inline void spmspvBfs(const int vertex, const int edge, const int m, const int *h_csrRowPtr,
                      const int *d_csrRowPtr, const int *d_csrColInd, int *d_bfsResult, const int depth,
                      mgpu::CudaContext &context) {
    (void)h_csrRowPtr;
    apspie_csr a = apspie_compat::view(m, m, edge, d_csrRowPtr, d_csrColInd, nullptr, APSPIE_VAL_NONE,
                                       context.symmetric());
    apspie_compat::report(apspie_bfs(context.get(), &a, vertex, depth, d_bfsResult, nullptr), context,
                          "spmspvBfs");
}

// src/sssp.cuh:28. Value = int: exact int32 distances, -1 unreached. Value = float:
// float32 distances, 1.70141e+38 unreached (the value the reference GPU path leaves).
template <typename Value>
void sssp(const int vertex, const int edge, const int m, const Value *d_csrValA, const int *d_csrRowPtrA,
          const int *d_csrColIndA, Value *d_ssspResult, const int depth, mgpu::CudaContext &context) {
    (void)depth;  // iterated to the fixed point
    apspie_csr a = apspie_compat::view(m, m, edge, d_csrRowPtrA, d_csrColIndA, d_csrValA,
                                       apspie_compat::ValType<Value>::value, context.symmetric());
    apspie_status st;
    if (apspie_compat::ValType<Value>::value == APSPIE_VAL_F32)
        st = apspie_sssp_f32(context.get(), &a, vertex, reinterpret_cast<float *>(d_ssspResult), 1.70141e+38f,
                             nullptr);
    else
        st = apspie_sssp(context.get(), &a, vertex, reinterpret_cast<int32_t *>(d_ssspResult), nullptr);
    apspie_compat::report(st, context, "sssp");
}

// src/spmspvMis.cuh:150. T = float priorities in [0, 1] (cuRAND uniform): non-negative
// floats order like their bit patterns, which are used as uint32 keys; T = unsigned: as is.
// `delta` (the threshold step) does not change the fixed point and is ignored.
template <typename T>
void spmspvMis(const int edge, const int m, const int *h_csrRowPtr, const int *d_csrRowPtr,
               const int *d_csrColInd, const T *d_randVec, int *d_misResult, const float delta,
               mgpu::CudaContext &context) {
    static_assert(sizeof(T) == 4, "32-bit priorities");
    (void)h_csrRowPtr;
    (void)delta;
    apspie_csr a = apspie_compat::view(m, m, edge, d_csrRowPtr, d_csrColInd, nullptr, APSPIE_VAL_NONE, true);
    apspie_compat::report(apspie_mis_int32(context.get(), &a, reinterpret_cast<const uint32_t *>(d_randVec),
                                           d_misResult, nullptr),
                          context, "spmspvMis");
}

// src/spmspvMis.cuh:81: one-hop boolean SpMSpV (the MIS validity helper).
template <typename T>
void spmspvCsr(const T *d_inputVector, const int edge, const int m, const int *d_csrRowPtr,
               const int *d_csrColInd, T *d_spmspvResult, mgpu::CudaContext &context) {
    static_assert(sizeof(T) == 4, "int vectors");
    apspie_csr a = apspie_compat::view(m, m, edge, d_csrRowPtr, d_csrColInd, nullptr, APSPIE_VAL_NONE, false);
    apspie_compat::report(apspie_spmspv_bool(context.get(), &a, reinterpret_cast<const int32_t *>(d_inputVector),
                                             reinterpret_cast<int32_t *>(d_spmspvResult)),
                          context, "spmspvCsr");
}

// src/scratch.hpp:5-31 / src/util.cuh:646-672: the reference's per-call scratch block. The
// context owns all scratch here, so the block carries nothing; allocScratch / freeScratch
// keep programs that create and pass one compiling.
struct d_scratch {};
inline void allocScratch(d_scratch **d, const int edge, const int m) {
    (void)edge;
    (void)m;
    *d = new d_scratch();
}
inline void freeScratch(d_scratch *d) { delete d; }

// src/mXv.cuh:249: sparse vector (d_randVecInd, d_randVecVal, nnz entries) times the CSC
// matrix (column j = d_cscRowInd[d_cscColPtr[j] ..]); the result's indices go to d_resultInd
// ascending with summed values in d_resultVal, and nnz becomes their number. Over the same
// arrays read as CSR this is y = x^T A.
template <typename T>
void mXv(const int *d_randVecInd, const T *d_randVecVal, const int edge, const int m, int &nnz, const T *d_cscVal,
         const int *d_cscColPtr, const int *d_cscRowInd, int *d_resultInd, T *d_resultVal, d_scratch *d,
         mgpu::CudaContext &context) {
    (void)d;
    apspie_csr a = apspie_compat::view(m, m, edge, d_cscColPtr, d_cscRowInd, d_cscVal,
                                       apspie_compat::ValType<T>::value, false);
    int32_t ny = 0;
    if (apspie_compat::report(apspie_spmspv(context.get(), &a, d_randVecInd, d_randVecVal, nnz, d_resultInd,
                                            d_resultVal, &ny),
                              context, "mXv"))
        nnz = ny;
}

// ---------------------------------------------------------------------------------
// SpGEMM and triangle counting
// ---------------------------------------------------------------------------------

// src/spgemm.cuh:132 (hash SpGEMM; partSize/partNum of the outer-product design unused).
// C's arrays are allocated here, as the reference does (src/spgemm.cuh:202-204).
inline void spgemm(d_matrix *C, d_matrix *A, d_matrix *B, const int partSize, const int partNum,
                   mgpu::CudaContext &context) {
    (void)partSize;
    (void)partNum;
    apspie_csr a = apspie_compat::view(A->m, A->n, A->nnz, A->d_cscColPtr, A->d_cscRowInd, A->d_cscVal,
                                       APSPIE_VAL_F32, false);
    apspie_csr b = apspie_compat::view(B->m, B->n, B->nnz, B->d_cscColPtr, B->d_cscRowInd, B->d_cscVal,
                                       APSPIE_VAL_F32, false);
    apspie_csr_owned c;
    if (!apspie_compat::report(apspie_spgemm(context.get(), &a, &b, &c), context, "spgemm")) return;
    if (C->d_cscColPtr) cudaFree(C->d_cscColPtr);
    C->m = c.m;
    C->n = c.n;
    C->nnz = c.nnz;
    C->d_cscColPtr = c.row_ptr;
    C->d_cscRowInd = c.col_ind;
    C->d_cscVal = static_cast<float *>(c.val);
}

// src/spgemm.cuh:346 (the cuSPARSE csrgemm wrapper).
template <typename T>
void spgemm(d_matrix *C, d_matrix *A, d_matrix *B) {
    spgemm(C, A, B, 0, 0, apspie_compat::default_context());
}

// src/tc.cuh:63: C = A*B over raw CSR arrays; allocates C and returns nnz(C).
template <typename T>
int spgemm(const int edge, const int m, const T *d_cscValA, const int *d_cscColPtrA, const int *d_cscRowIndA,
           const T *d_cscValB, const int *d_cscColPtrB, const int *d_cscRowIndB, T *&d_cscValC, int *&d_cscColPtrC,
           int *&d_cscRowIndC) {
    mgpu::CudaContext &ctx = apspie_compat::default_context();
    const int nnz_a = edge;
    int nnz_b = 0;
    cudaMemcpy(&nnz_b, d_cscColPtrB + m, sizeof(int), cudaMemcpyDeviceToHost);
    apspie_csr a = apspie_compat::view(m, m, nnz_a, d_cscColPtrA, d_cscRowIndA, d_cscValA,
                                       apspie_compat::ValType<T>::value, false);
    apspie_csr b = apspie_compat::view(m, m, nnz_b, d_cscColPtrB, d_cscRowIndB, d_cscValB,
                                       apspie_compat::ValType<T>::value, false);
    apspie_csr_owned c;
    if (!apspie_compat::report(apspie_spgemm(ctx.get(), &a, &b, &c), ctx, "spgemm")) return 0;
    d_cscColPtrC = c.row_ptr;
    d_cscRowIndC = c.col_ind;
    d_cscValC = static_cast<T *>(c.val);
    return c.nnz;
}

// src/tc.cuh:315: C = A*B column by column over CSC arrays, written into caller buffers
// (the reference sizes them 16*edge); returns nnz(C). As CSR of the transposes,
// C^T = B^T * A^T, which is what is computed.
template <typename T>
int mXm(const int edge, const int m, const T *d_cscValA, const int *d_cscColPtrA, const int *d_cscRowIndA,
        const T *d_cscValB, const int *h_cscColPtrB, const int *d_cscColPtrB, const int *d_cscRowIndB, T *d_cscValC,
        int *d_cscColPtrC, int *d_cscRowIndC, mgpu::CudaContext &context) {
    apspie_csr at = apspie_compat::view(m, m, edge, d_cscColPtrA, d_cscRowIndA, d_cscValA,
                                        apspie_compat::ValType<T>::value, false);
    apspie_csr bt = apspie_compat::view(m, m, h_cscColPtrB[m], d_cscColPtrB, d_cscRowIndB, d_cscValB,
                                        apspie_compat::ValType<T>::value, false);
    int64_t nnz = 0;
    if (!apspie_compat::report(apspie_spgemm_symbolic(context.get(), &bt, &at, d_cscColPtrC, &nnz), context, "mXm"))
        return 0;
    if (!apspie_compat::report(apspie_spgemm_numeric(context.get(), &bt, &at, d_cscColPtrC, d_cscRowIndC, d_cscValC),
                               context, "mXm"))
        return 0;
    return static_cast<int>(nnz);
}

// The TC flow of test/tc/main.cu:243-249 on a symmetric graph (CSR arrays): strict lower
// triangle on the device, then the masked count. Returns the exact count.
inline long long triangleCount(const int edge, const int m, const int *d_csrRowPtr, const int *d_csrColInd,
                               mgpu::CudaContext &context) {
    apspie_csr a = apspie_compat::view(m, m, edge, d_csrRowPtr, d_csrColInd, nullptr, APSPIE_VAL_NONE, true);
    apspie_csr_owned l;
    if (!apspie_compat::report(apspie_csr_strict_lower_device(context.get(), &a, &l), context, "triangleCount"))
        return -1;
    apspie_csr lv = apspie_compat::view(l.m, l.n, l.nnz, l.row_ptr, l.col_ind, nullptr, APSPIE_VAL_NONE, false);
    int64_t count = -1;
    apspie_compat::report(apspie_tc(context.get(), &lv, &count), context, "triangleCount");
    apspie_csr_free(&l);
    return count;
}
