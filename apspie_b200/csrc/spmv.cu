// Dense-vector SpMV and PageRank: the dense-frontier end of the push/pull spectrum.
//
// The reference multiplies by a dense vector through moderngpu's SpmvCsrBinary
// (src/bfs.cuh:11-14) and a cuSPARSE csrmv wrapper (cuspmv, src/tc.cuh:17-59); it ships
// test_pr.mtx but no PageRank. Here:
//   * apspie_spmv: y = alpha * A * x + beta * y in FP32, a group of G lanes per row (G from
//     the mean row length: 4, 8, 16 or 32), lane-strided partial sums reduced by shuffles
//     (fixed order, so repeated calls give identical bits);
//   * apspie_pagerank: power iteration r' = (1 - d) / n + d * (A^T (r / outdeg) + dangling
//     mass / n) on the transposed graph (pull: no atomics), stopping when the L1 change is
//     below tol or after max_iter iterations.
#include <algorithm>
#include <cstring>

#include "common.cuh"

namespace apspie {
namespace {

template <int G>
__global__ void spmv_kernel(int m, const int *__restrict__ rp, const int *__restrict__ ci,
                            const float *__restrict__ val, const float *__restrict__ x, float *y, float alpha,
                            float beta) {
    const int lane = threadIdx.x % G;
    const long long grp = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) / G;
    const long long ngrp = static_cast<long long>(gridDim.x) * blockDim.x / G;
    for (long long r0 = grp - grp % (32 / G); r0 < m; r0 += ngrp) {  // a warp's groups move together
        const long long r = r0 + grp % (32 / G);
        float s = 0.0f;
        if (r < m) {
            const int e1 = __ldg(rp + r + 1);
            for (int e = __ldg(rp + r) + lane; e < e1; e += G) {
                const float a = val ? __ldg(val + e) : 1.0f;
                s = __fmaf_rn(a, __ldg(x + __ldg(ci + e)), s);
            }
        }
#pragma unroll
        for (int o = G / 2; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, G);
        if (r < m && lane == 0) y[r] = beta == 0.0f ? alpha * s : alpha * s + beta * y[r];
    }
}

apspie_status launch_spmv(apspie_ctx *ctx, const apspie_csr *A, const float *x, float *y, float alpha,
                          float beta) {
    const float *val = A->val_type == APSPIE_VAL_F32 ? static_cast<const float *>(A->val) : nullptr;
    const double mean = A->m > 0 ? static_cast<double>(A->nnz) / A->m : 0.0;
    const int blocks = static_cast<int>(std::max<long long>(
        1, std::min<long long>((static_cast<long long>(A->m) * 32 + 255) / 256, ctx->num_sms * 16LL)));
    if (mean <= 6)
        spmv_kernel<4><<<blocks, 256, 0, ctx->stream>>>(A->m, A->row_ptr, A->col_ind, val, x, y, alpha, beta);
    else if (mean <= 12)
        spmv_kernel<8><<<blocks, 256, 0, ctx->stream>>>(A->m, A->row_ptr, A->col_ind, val, x, y, alpha, beta);
    else if (mean <= 24)
        spmv_kernel<16><<<blocks, 256, 0, ctx->stream>>>(A->m, A->row_ptr, A->col_ind, val, x, y, alpha, beta);
    else
        spmv_kernel<32><<<blocks, 256, 0, ctx->stream>>>(A->m, A->row_ptr, A->col_ind, val, x, y, alpha, beta);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? APSPIE_OK : cuda_error(ctx, e, "spmv launch");
}

// x[u] = r[u] / outdeg(u); dangling mass (outdeg 0) summed into acc[0] (double)
__global__ void pr_scale(int n, const int *__restrict__ rp, const float *__restrict__ r, float *x, double *acc) {
    double dang = 0.0;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        const int d = __ldg(rp + u + 1) - __ldg(rp + u);
        x[u] = d > 0 ? r[u] / static_cast<float>(d) : 0.0f;
        if (d == 0) dang += r[u];
    }
    for (int o = 16; o; o >>= 1) dang += __shfl_down_sync(0xffffffffu, dang, o);
    if ((threadIdx.x & 31) == 0 && dang != 0.0) atomicAdd(acc, dang);
}

// r'[v] = (1 - d) / n + d * (y[v] + dangling / n); acc[1] += |r'[v] - r[v]|
__global__ void pr_update(int n, float damping, const float *__restrict__ y, float *r, double *acc) {
    const float base = static_cast<float>((1.0 - damping) / n + damping * acc[0] / n);
    double diff = 0.0;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float nr = __fmaf_rn(damping, y[v], base);
        diff += fabs(static_cast<double>(nr) - static_cast<double>(r[v]));
        r[v] = nr;
    }
    for (int o = 16; o; o >>= 1) diff += __shfl_down_sync(0xffffffffu, diff, o);
    if ((threadIdx.x & 31) == 0 && diff != 0.0) atomicAdd(acc + 1, diff);
}

__global__ void pr_init(int n, float *r) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) r[v] = 1.0f / n;
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_spmv(apspie_ctx *ctx, const apspie_csr *A, const float *d_x, float *d_y, float alpha,
                          float beta) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_csr_view(ctx, A, "apspie_spmv");
    if (st != APSPIE_OK) return st;
    if (A->val_type == APSPIE_VAL_I32)
        return set_error(ctx, APSPIE_ERR_UNSUPPORTED, "apspie_spmv: float32 values or a pattern required");
    if (A->m > 0 && (!d_y || (A->nnz > 0 && !d_x)))
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_spmv: NULL vector");
    if (ctx->validate && (st = validate_csr(ctx, A, false)) != APSPIE_OK) return st;
    if (A->m == 0) return APSPIE_OK;
    return launch_spmv(ctx, A, d_x, d_y, alpha, beta);
}

apspie_status apspie_pagerank(apspie_ctx *ctx, const apspie_csr *A, float damping, double tol, int32_t max_iter,
                              float *d_rank, int32_t *iterations) {
    if (!ctx || !d_rank || max_iter < 1 || !(damping >= 0.0f && damping < 1.0f) || !(tol >= 0.0))
        return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_csr_view(ctx, A, "apspie_pagerank");
    if (st != APSPIE_OK) return st;
    if (A->m != A->n || A->m == 0)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_pagerank: square, non-empty graph required");
    if (ctx->validate && (st = validate_csr(ctx, A, true)) != APSPIE_OK) return st;
    const int n = A->m;
    // pull over in-edges: A^T, or A itself when the pattern is symmetric
    apspie_csr_owned T;
    std::memset(&T, 0, sizeof(T));
    apspie_csr at = *A;
    at.val_type = APSPIE_VAL_NONE;
    at.val = nullptr;
    if (!(A->flags & APSPIE_CSR_SYMMETRIC)) {
        if ((st = apspie_csr_transpose(ctx, &at, &T)) != APSPIE_OK) return st;
        at.row_ptr = T.row_ptr;
        at.col_ind = T.col_ind;
        at.nnz = T.nnz;
    }
    void *base;
    st = scratch_reserve(ctx, Carver::need({static_cast<size_t>(n) * 4, static_cast<size_t>(n) * 4, 64}), &base);
    if (st != APSPIE_OK) {
        apspie_csr_free(&T);
        return st;
    }
    Carver c(base);
    float *x = c.take<float>(n);
    float *y = c.take<float>(n);
    double *acc = c.take<double>(4);
    const int blocks = std::max(1, std::min((n + 255) / 256, ctx->num_sms * 8));
    pr_init<<<blocks, 256, 0, ctx->stream>>>(n, d_rank);
    int it = 0;
    double h_acc[2] = {0.0, 0.0};
    cudaError_t e = cudaSuccess;
    while (it < max_iter) {
        if ((e = cudaMemsetAsync(acc, 0, 2 * sizeof(double), ctx->stream)) != cudaSuccess) break;
        pr_scale<<<blocks, 256, 0, ctx->stream>>>(n, A->row_ptr, d_rank, x, acc);
        if ((st = launch_spmv(ctx, &at, x, y, 1.0f, 0.0f)) != APSPIE_OK) break;
        pr_update<<<blocks, 256, 0, ctx->stream>>>(n, damping, y, d_rank, acc);
        ++it;
        if ((e = cudaMemcpyAsync(h_acc, acc, sizeof(h_acc), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
            break;
        if (h_acc[1] < tol) break;
    }
    apspie_csr_free(&T);
    if (st != APSPIE_OK) return st;
    if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_pagerank");
    if (iterations) *iterations = it;
    return APSPIE_OK;
}

}  // extern "C"
