// Valued sparse-vector times sparse-matrix product with a sparse result: y = x^T A.
//
// The reference's mXv<T> (src/mXv.cuh:249-389) gathers the CSC columns named by the sparse
// vector's indices (IntervalGather / Scan / IntervalExpand), multiplies every gathered
// matrix value by its vector entry (elementMult), sorts the (row index, product) pairs
// (cub SortPairs) and sums runs of equal indices (mgpu ReduceByKey). Over CSR this is the
// combination of A's rows x_ind[j] with weights x_val[j]. Here:
//   1. one thread per vector entry reads its row length (indices out of range are an
//      error, counted as empty rows); a device scan gives each entry's first product;
//   2. one thread per product finds its entry by binary search over those offsets and
//      writes the product x_val[j] * A(x_ind[j], c) and the sort key c, with the product's
//      own index as the value, so products of one column stay in (entry, edge) order;
//   3. the stable radix sort of build.cu's construction path orders them by column;
//   4. one thread per run of equal columns sums its products in that order (int32:
//      wrapping adds; f32: correctly rounded multiply and add, no fused multiply-add),
//      exactly the order a sequential loop over the entries and their rows would use, so
//      the result is bit-exact against such a loop.
#include <algorithm>
#include <cstring>

#include "sort.cuh"

namespace apspie {
namespace {

__global__ void sv_degrees(int nx, const int *__restrict__ x_ind, int m, const int *__restrict__ row_ptr, int *deg,
                           int *bad) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nx; j += gridDim.x * blockDim.x) {
        const int r = __ldg(x_ind + j);
        int d = 0;
        if (r < 0 || r >= m)
            atomicOr(bad, 1);
        else
            d = __ldg(row_ptr + r + 1) - __ldg(row_ptr + r);
        deg[j] = d;
    }
}

template <typename T>
__device__ __forceinline__ unsigned sv_mul(unsigned a, unsigned b);
template <>
__device__ __forceinline__ unsigned sv_mul<float>(unsigned a, unsigned b) {
    return __float_as_uint(__fmul_rn(__uint_as_float(a), __uint_as_float(b)));
}
template <>
__device__ __forceinline__ unsigned sv_mul<int>(unsigned a, unsigned b) {
    return a * b;  // int32 product, wrapping
}
template <typename T>
__device__ __forceinline__ unsigned sv_add(unsigned a, unsigned b);
template <>
__device__ __forceinline__ unsigned sv_add<float>(unsigned a, unsigned b) {
    return __float_as_uint(__fadd_rn(__uint_as_float(a), __uint_as_float(b)));
}
template <>
__device__ __forceinline__ unsigned sv_add<int>(unsigned a, unsigned b) {
    return a + b;
}

// Product p of [0, total): entry j with off[j] <= p < off[j + 1].
template <typename T>
__global__ void sv_expand(long long total, int nx, const int *__restrict__ off, const int *__restrict__ x_ind,
                          const unsigned *__restrict__ x_val, const int *__restrict__ row_ptr,
                          const int *__restrict__ col_ind, const unsigned *__restrict__ a_val,
                          unsigned long long *key, unsigned *idx, unsigned *prod) {
    for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < total;
         p += static_cast<long long>(gridDim.x) * blockDim.x) {
        int lo = 0, hi = nx - 1;  // last j with off[j] <= p
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(off + mid) <= p)
                lo = mid;
            else
                hi = mid - 1;
        }
        const long long e = __ldg(row_ptr + __ldg(x_ind + lo)) + (p - __ldg(off + lo));
        key[p] = static_cast<unsigned>(__ldg(col_ind + e));
        idx[p] = static_cast<unsigned>(p);
        prod[p] = sv_mul<T>(__ldg(x_val + lo), __ldg(a_val + e));
    }
}

__global__ void sv_run_flags(long long n, const unsigned long long *__restrict__ key, int *flag) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

template <typename T>
__global__ void sv_reduce(long long n, const unsigned long long *__restrict__ key, const unsigned *__restrict__ idx,
                          const unsigned *__restrict__ prod, const int *__restrict__ run, int *y_ind, unsigned *y_val) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const unsigned long long k = key[i];
        if (i > 0 && key[i - 1] == k) continue;  // not the first of its run
        unsigned acc = 0u;                       // +0.0f and int 0 share the bit pattern
        for (long long t = i; t < n && key[t] == k; ++t) acc = sv_add<T>(acc, __ldg(prod + idx[t]));
        const int r = run[i];
        y_ind[r] = static_cast<int>(k);
        y_val[r] = acc;
    }
}

int sv_grid(const apspie_ctx *ctx, long long n) {
    const long long g = (n + 255) / 256;
    const long long cap = static_cast<long long>(ctx->num_sms) * 16;
    return static_cast<int>(std::max(1LL, std::min(g, cap)));
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" apspie_status apspie_spmspv(apspie_ctx *ctx, const apspie_csr *A, const int32_t *d_x_ind,
                                       const void *d_x_val, int32_t x_nnz, int32_t *d_y_ind, void *d_y_val,
                                       int32_t *y_nnz) {
    if (!ctx || !y_nnz) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    apspie_status st = check_csr_view(ctx, A, "apspie_spmspv");
    if (st != APSPIE_OK) return st;
    if (A->val_type != APSPIE_VAL_F32 && A->val_type != APSPIE_VAL_I32)
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_spmspv: A needs F32 or I32 values");
    if (x_nnz < 0 || (x_nnz > 0 && (!d_x_ind || !d_x_val || !d_y_ind || !d_y_val)))
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_spmspv: bad vector arguments");
    if (ctx->validate && (st = validate_csr(ctx, A, false)) != APSPIE_OK) return st;
    *y_nnz = 0;
    if (x_nnz == 0) return APSPIE_OK;
    // degrees and their scan (off[x_nnz] = number of products)
    void *base;
    const size_t head = Carver::need({static_cast<size_t>(x_nnz) * 4, static_cast<size_t>(x_nnz + 1) * 4,
                                      scan_scratch_bytes(x_nnz) + 64, 64});
    if ((st = scratch_reserve(ctx, head, &base)) != APSPIE_OK) return st;
    Carver c0(base);
    int *deg = c0.take<int>(x_nnz);
    int *off = c0.take<int>(x_nnz + 1);
    void *stmp = c0.take<char>(scan_scratch_bytes(x_nnz) + 64);
    int *flags = c0.take<int>(16);
    cudaError_t e = cudaMemsetAsync(flags, 0, 64, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_spmspv reset");
    sv_degrees<<<sv_grid(ctx, x_nnz), 256, 0, ctx->stream>>>(x_nnz, d_x_ind, A->m, A->row_ptr, deg, flags);
    if ((st = device_exclusive_scan(ctx, deg, x_nnz, off, stmp, flags + 4)) != APSPIE_OK) return st;
    int h[16] = {0}, total_i = 0;
    if ((e = cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&total_i, off + x_nnz, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return cuda_error(ctx, e, "apspie_spmspv count");
    if (h[0]) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_spmspv: vector index out of range");
    if (h[4]) return set_error(ctx, APSPIE_ERR_UNSUPPORTED, "apspie_spmspv: more than 2^31 - 1 products");
    const long long total = total_i;
    if (total == 0) return APSPIE_OK;
    // the products, sorted by column (the head buffers move to the front of a larger arena)
    const size_t need = head + sort_need(total) +
                        Carver::need({static_cast<size_t>(total) * 4, static_cast<size_t>(total + 1) * 4});
    std::vector<int> h_off;
    if (need > ctx->scratch_bytes) {
        // growing the arena drops its contents: keep the offsets on the host meanwhile
        h_off.resize(static_cast<size_t>(x_nnz) + 1);
        if ((e = cudaMemcpy(h_off.data(), off, h_off.size() * 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cuda_error(ctx, e, "apspie_spmspv offsets");
        if ((st = scratch_reserve(ctx, need, &base)) != APSPIE_OK) return st;
    }
    Carver c(base);
    deg = c.take<int>(x_nnz);
    off = c.take<int>(x_nnz + 1);
    stmp = c.take<char>(scan_scratch_bytes(x_nnz) + 64);
    flags = c.take<int>(16);
    if (!h_off.empty() &&
        (e = cudaMemcpyAsync(off, h_off.data(), h_off.size() * 4, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return cuda_error(ctx, e, "apspie_spmspv offsets");
    SortBufs s = carve_sort(c, total);
    unsigned *prod = c.take<unsigned>(total);
    int *run = c.take<int>(total + 1);
    if ((e = cudaMemsetAsync(s.ovf, 0, 64, ctx->stream)) != cudaSuccess) return cuda_error(ctx, e, "apspie_spmspv reset");
    const int g = sv_grid(ctx, total);
    const bool f32 = A->val_type == APSPIE_VAL_F32;
    const unsigned *xv = static_cast<const unsigned *>(d_x_val);
    const unsigned *av = static_cast<const unsigned *>(A->val);
    if (f32)
        sv_expand<float><<<g, 256, 0, ctx->stream>>>(total, x_nnz, off, d_x_ind, xv, A->row_ptr, A->col_ind, av,
                                                      s.k[0], s.v[0], prod);
    else
        sv_expand<int><<<g, 256, 0, ctx->stream>>>(total, x_nnz, off, d_x_ind, xv, A->row_ptr, A->col_ind, av,
                                                    s.k[0], s.v[0], prod);
    int which = 0;
    if ((st = radix_sort(ctx, s, total, bit_length(A->n), &which)) != APSPIE_OK) return st;
    // run numbers: exclusive scan of run-start flags (held in the sort's spare value buffer)
    int *rflag = reinterpret_cast<int *>(s.v[which ^ 1]);
    sv_run_flags<<<g, 256, 0, ctx->stream>>>(total, s.k[which], rflag);
    if ((st = device_exclusive_scan(ctx, rflag, total, run, s.scan_tmp, s.ovf)) != APSPIE_OK) return st;
    if (f32)
        sv_reduce<float><<<g, 256, 0, ctx->stream>>>(total, s.k[which], s.v[which], prod, run, d_y_ind,
                                                      static_cast<unsigned *>(d_y_val));
    else
        sv_reduce<int><<<g, 256, 0, ctx->stream>>>(total, s.k[which], s.v[which], prod, run, d_y_ind,
                                                    static_cast<unsigned *>(d_y_val));
    int ny = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&ny, run + total, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return cuda_error(ctx, e, "apspie_spmspv");
    *y_nnz = ny;
    return APSPIE_OK;
}
