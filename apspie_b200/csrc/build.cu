// Device-side graph construction: COO -> CSR (optionally symmetrised and deduplicated with
// the generator's rules) and CSR transpose, on a stable LSD radix sort of this file's own.
//
// The reference builds graphs on the host: readMtx + makeSymmetric (src/util.cuh:371-643,
// a qsort of every edge and its mirror, then a compaction) and buildMatrix
// (src/matrix.cpp:55-111, a COO -> CSR conversion through cuSPARSE), and transposes with
// csr2csc (src/util.cuh:474). Here the same results come from device kernels:
//   * keys (a << B) | b of B = bit length of m bits each; symmetrising canonicalises
//     {u, v} to a = min, b = max; dropped self-loops get a sentinel key that sorts last;
//   * a stable radix sort (8-bit digits; per pass: per-tile digit counts, one device scan,
//     then a scatter that ranks each tile's keys in input order with warp match masks), so
//     equal keys keep their input order and deduplication keeps the first occurrence;
//   * symmetric CSR rows: lower neighbours (pairs (lo, r)) then upper ones ((r, hi)), each
//     ascending, so rows come out sorted without a per-row sort: row_ptr[r] is the number
//     of pairs with lo < r plus the number with hi < r, read off the two sorted orders.
#include <algorithm>
#include <cstring>

#include "sort.cuh"

namespace apspie {
namespace {

// start[r] = first index i with (key[i] >> shift) >= r, for r in [0, m]; keys ascending
// in that field.
__global__ void run_starts(long long n, const unsigned long long *__restrict__ keys, int shift,
                           unsigned long long fmask, int m, int *start) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i <= n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int r = i < n ? static_cast<int>((keys[i] >> shift) & fmask) : m;
        const int rp = i > 0 ? static_cast<int>((keys[i - 1] >> shift) & fmask) : -1;
        for (int x = rp + 1; x <= r; ++x) start[x] = static_cast<int>(i);
    }
}

__global__ void plain_fill(long long n, const unsigned long long *__restrict__ keys, const unsigned *__restrict__ vals,
                           unsigned long long cmask, int *col, unsigned *val) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        col[i] = static_cast<int>(keys[i] & cmask);
        if (val) val[i] = vals[i];
    }
}

__global__ void sym_row_ptr(int m, const int *__restrict__ up, const int *__restrict__ low, int *row_ptr) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= m; r += gridDim.x * blockDim.x)
        row_ptr[r] = up[r] + low[r];
}

// Upper neighbours: pair i (ascending (lo, hi)) lands after row lo's lower neighbours.
__global__ void sym_fill_upper(long long np, const unsigned long long *__restrict__ keys,
                               const unsigned *__restrict__ vals, int B, const int *__restrict__ row_ptr,
                               const int *__restrict__ up, const int *__restrict__ low, int *col, unsigned *val) {
    const unsigned long long mask = (1ull << B) - 1ull;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < np;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int lo = static_cast<int>(keys[i] >> B), hi = static_cast<int>(keys[i] & mask);
        const long long p = row_ptr[lo] + (low[lo + 1] - low[lo]) + (i - up[lo]);
        col[p] = hi;
        if (val) val[p] = vals[i];
    }
}

// Lower neighbours: position j of the pairs re-sorted by hi (payload: index in (lo, hi)
// order) lands at row hi's start, in ascending lo.
__global__ void sym_fill_lower(long long np, const unsigned long long *__restrict__ hkeys,
                               const unsigned *__restrict__ idx, const unsigned long long *__restrict__ keys,
                               const unsigned *__restrict__ vals, int B, const int *__restrict__ row_ptr,
                               const int *__restrict__ low, int *col, unsigned *val) {
    for (long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; j < np;
         j += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int hi = static_cast<int>(hkeys[j]);
        const unsigned i = idx[j];
        const long long p = row_ptr[hi] + (j - low[hi]);
        col[p] = static_cast<int>(keys[i] >> B);
        if (val) val[p] = vals[i];
    }
}

__global__ void hi_keys(long long np, const unsigned long long *__restrict__ keys, int B, unsigned long long *hk,
                        unsigned *idx) {
    const unsigned long long mask = (1ull << B) - 1ull;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < np;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        hk[i] = keys[i] & mask;
        idx[i] = static_cast<unsigned>(i);
    }
}

__global__ void entry_rows(int m, const int *__restrict__ rp, int *row_of) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < m; r += nwarps)
        for (int e = rp[r] + lane; e < rp[r + 1]; e += 32) row_of[e] = r;
}

__global__ void col_keys(long long nnz, const int *__restrict__ ci, unsigned long long *keys, unsigned *idx) {
    for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < nnz;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        keys[e] = static_cast<unsigned>(ci[e]);
        idx[e] = static_cast<unsigned>(e);
    }
}

__global__ void transpose_fill(long long nnz, const unsigned *__restrict__ idx, const int *__restrict__ row_of,
                               const unsigned *__restrict__ val_in, int *col, unsigned *val) {
    for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < nnz;
         p += static_cast<long long>(gridDim.x) * blockDim.x) {
        const unsigned e = idx[p];
        col[p] = row_of[e];
        if (val) val[p] = val_in[e];
    }
}

int grid_for(const apspie_ctx *ctx, long long n) {
    return static_cast<int>(std::max<long long>(1, std::min<long long>((n + 255) / 256, ctx->num_sms * 16LL)));
}

apspie_status alloc_owned(apspie_ctx *ctx, int m, int n, long long nnz, int val_type, apspie_csr_owned *out) {
    std::memset(out, 0, sizeof(*out));
    cudaError_t e = cudaMalloc(&out->row_ptr, (static_cast<size_t>(m) + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&out->col_ind, static_cast<size_t>(std::max(nnz, 1LL)) * 4);
    if (e == cudaSuccess && val_type != APSPIE_VAL_NONE)
        e = cudaMalloc(&out->val, static_cast<size_t>(std::max(nnz, 1LL)) * 4);
    if (e != cudaSuccess) {
        apspie_csr_free(out);
        return cuda_error(ctx, e, "csr allocation");
    }
    out->m = m;
    out->n = n;
    out->nnz = static_cast<int32_t>(nnz);
    out->val_type = val_type;
    return APSPIE_OK;
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

apspie_status apspie_csr_build(apspie_ctx *ctx, int32_t m, int64_t nedges, const int32_t *d_src,
                               const int32_t *d_dst, const void *d_val, int32_t val_type, int32_t flags,
                               apspie_csr_owned *out) {
    if (!ctx || !out || m < 1 || nedges < 0 || (nedges > 0 && (!d_src || !d_dst))) return APSPIE_ERR_INVALID_ARG;
    if (val_type != APSPIE_VAL_NONE && val_type != APSPIE_VAL_I32 && val_type != APSPIE_VAL_F32)
        return APSPIE_ERR_INVALID_ARG;
    if (val_type != APSPIE_VAL_NONE && nedges > 0 && !d_val) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    std::memset(out, 0, sizeof(*out));
    const bool sym = (flags & APSPIE_BUILD_SYMMETRIZE) != 0;
    const bool dedup = (flags & APSPIE_BUILD_DEDUP) != 0;
    const bool loops = (flags & APSPIE_BUILD_DROP_SELF_LOOPS) != 0;
    if (nedges > 0x7fffffffLL || (sym && 2 * nedges > 0x7fffffffLL))
        return set_error(ctx, APSPIE_ERR_UNSUPPORTED, "apspie_csr_build: more than 2^31 - 1 entries");
    // m + 1 values per field, so the all-ones sentinel is never a real (u, u) key
    const int B = bit_length(static_cast<long long>(m) + 1);
    const long long n = nedges;
    void *base;
    const size_t need = sort_need(n) + Carver::need({static_cast<size_t>(n + 1) * 4, static_cast<size_t>(n + 1) * 4,
                                                     static_cast<size_t>(m + 1) * 4, static_cast<size_t>(m + 1) * 4,
                                                     64, static_cast<size_t>(n + 1) * 8,
                                                     static_cast<size_t>(n + 1) * 4});
    apspie_status st = scratch_reserve(ctx, need, &base);
    if (st != APSPIE_OK) return st;
    Carver c(base);
    SortBufs s = carve_sort(c, n);
    int *keep = c.take<int>(n + 1);
    int *pos = c.take<int>(n + 1);
    int *up = c.take<int>(static_cast<size_t>(m) + 1);
    int *low = c.take<int>(static_cast<size_t>(m) + 1);
    int *flag = c.take<int>(16);
    unsigned long long *hk = c.take<unsigned long long>(n + 1);  // the hi-ordered copy (symmetric)
    unsigned *hv = c.take<unsigned>(n + 1);
    cudaError_t e = cudaMemsetAsync(flag, 0, 64, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.ovf, 0, 64, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_csr_build reset");
    const int g = grid_for(ctx, n);
    if (n > 0)
        coo_keys<<<g, 256, 0, ctx->stream>>>(n, m, d_src, d_dst, static_cast<const unsigned *>(d_val), B, sym ? 1 : 0,
                                             loops ? 1 : 0, s.k[0], s.v[0], flag);
    int which = 0;
    if ((st = radix_sort(ctx, s, n, 2 * B, &which)) != APSPIE_OK) return st;
    // drop sentinels (and duplicates): compact into the other buffer pair
    const unsigned long long sentinel = (1ull << (2 * B)) - 1ull;
    if (n > 0) mark_keep<<<g, 256, 0, ctx->stream>>>(n, s.k[which], sentinel, dedup ? 1 : 0, keep);
    if ((st = device_exclusive_scan(ctx, keep, n, pos, s.scan_tmp, s.ovf)) != APSPIE_OK) return st;
    int kept = 0, bad = 0;
    if ((e = cudaMemcpyAsync(&kept, pos + n, 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&bad, flag, 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return cuda_error(ctx, e, "apspie_csr_build count");
    if (bad) return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_csr_build: vertex id out of range");
    const int o = which ^ 1;
    if (n > 0) compact_kv<<<g, 256, 0, ctx->stream>>>(n, s.k[which], s.v[which], keep, pos, s.k[o], s.v[o]);
    const long long np = kept;
    const long long nnz = sym ? 2 * np : np;
    if ((st = alloc_owned(ctx, m, m, nnz, val_type, out)) != APSPIE_OK) return st;
    unsigned *oval = static_cast<unsigned *>(out->val);
    const int gp = grid_for(ctx, np + 1);
    run_starts<<<gp, 256, 0, ctx->stream>>>(np, s.k[o], B, (1ull << B) - 1ull, m, up);
    if (!sym) {
        run_starts<<<gp, 256, 0, ctx->stream>>>(np, s.k[o], B, (1ull << B) - 1ull, m, out->row_ptr);
        if (np > 0) plain_fill<<<gp, 256, 0, ctx->stream>>>(np, s.k[o], s.v[o], (1ull << B) - 1ull, out->col_ind, oval);
    } else {
        // the pairs again, ordered by hi (stably, so ascending lo within each hi); the sort
        // ping-pongs between the free pre-compaction buffers and the hi copy
        const int w = o ^ 1;
        if (np > 0) hi_keys<<<gp, 256, 0, ctx->stream>>>(np, s.k[o], B, s.k[w], s.v[w]);
        SortBufs h = s;
        h.k[0] = s.k[w];
        h.v[0] = s.v[w];
        h.k[1] = hk;
        h.v[1] = hv;
        int hw = 0;
        if ((st = radix_sort(ctx, h, np, B, &hw)) != APSPIE_OK) {
            apspie_csr_free(out);
            return st;
        }
        run_starts<<<gp, 256, 0, ctx->stream>>>(np, h.k[hw], 0, (1ull << B) - 1ull, m, low);
        sym_row_ptr<<<grid_for(ctx, m + 1), 256, 0, ctx->stream>>>(m, up, low, out->row_ptr);
        if (np > 0) {
            sym_fill_upper<<<gp, 256, 0, ctx->stream>>>(np, s.k[o], s.v[o], B, out->row_ptr, up, low, out->col_ind,
                                                        oval);
            sym_fill_lower<<<gp, 256, 0, ctx->stream>>>(np, h.k[hw], h.v[hw], s.k[o], s.v[o], B, out->row_ptr, low,
                                                        out->col_ind, oval);
        }
    }
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
        apspie_csr_free(out);
        return cuda_error(ctx, e, "apspie_csr_build");
    }
    return APSPIE_OK;
}

apspie_status apspie_csr_transpose(apspie_ctx *ctx, const apspie_csr *A, apspie_csr_owned *out) {
    if (!ctx || !out) return APSPIE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    std::memset(out, 0, sizeof(*out));
    apspie_status st = check_csr_view(ctx, A, "apspie_csr_transpose");
    if (st != APSPIE_OK) return st;
    if (ctx->validate && (st = validate_csr(ctx, A, false)) != APSPIE_OK) return st;
    const long long nnz = A->nnz;
    const int n = A->n;
    void *base;
    st = scratch_reserve(ctx, sort_need(nnz) + Carver::need({static_cast<size_t>(nnz + 1) * 4}), &base);
    if (st != APSPIE_OK) return st;
    Carver c(base);
    SortBufs s = carve_sort(c, nnz);
    int *row_of = c.take<int>(nnz + 1);
    cudaError_t e = cudaMemsetAsync(s.ovf, 0, 64, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "apspie_csr_transpose reset");
    if ((st = alloc_owned(ctx, n, A->m, nnz, A->val ? A->val_type : APSPIE_VAL_NONE, out)) != APSPIE_OK) return st;
    const int g = grid_for(ctx, nnz);
    if (A->m > 0) entry_rows<<<grid_for(ctx, A->m * 32LL), 256, 0, ctx->stream>>>(A->m, A->row_ptr, row_of);
    if (nnz > 0) col_keys<<<g, 256, 0, ctx->stream>>>(nnz, A->col_ind, s.k[0], s.v[0]);
    int which = 0;
    if ((st = radix_sort(ctx, s, nnz, bit_length(n), &which)) != APSPIE_OK) {
        apspie_csr_free(out);
        return st;
    }
    run_starts<<<grid_for(ctx, nnz + 1), 256, 0, ctx->stream>>>(nnz, s.k[which], 0, ~0ull, n, out->row_ptr);
    if (nnz > 0)
        transpose_fill<<<g, 256, 0, ctx->stream>>>(nnz, s.v[which], row_of, static_cast<const unsigned *>(A->val),
                                                   out->col_ind, static_cast<unsigned *>(out->val));
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
        apspie_csr_free(out);
        return cuda_error(ctx, e, "apspie_csr_transpose");
    }
    return APSPIE_OK;
}

}  // extern "C"
