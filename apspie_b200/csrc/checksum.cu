// Checksums of result rows: for each row, sum_i row[i] * coef[i] with int32 products
// (wrapping) summed in int64 (exact, so independent of the summation order). Used to check
// every answer of a long query stream against a reference without copying rows to the
// host. No reference counterpart (the reference compares whole result vectors on the host,
// src/util.cuh:260-269).
#include <algorithm>

#include "common.cuh"

namespace apspie {
namespace {

constexpr int kSumRows = 128;  // rows per launch (the pointer table travels as a kernel parameter)

struct SumArgs {
    int n, m, elem_bytes;
    const void *row[kSumRows];
    int slot[kSumRows];
};

// 64-thread blocks, so that the checksums also run beside a persistent grid that leaves
// only a little room on each SM
constexpr int kSumBlock = 64;

__device__ __forceinline__ long long dot_term(int x, int c) {
    return static_cast<int>(static_cast<unsigned>(x) * static_cast<unsigned>(c));
}

// Row blockIdx.y, split over gridDim.x blocks. 32-bit rows whose start is 16-byte aligned
// (and the coefficients, which are) are read four entries per load, four loads in flight
// per thread, so that the few warps a persistent grid leaves room for still stream.
__global__ void __launch_bounds__(kSumBlock) row_checksums(SumArgs a, const int *__restrict__ coef,
                                                           unsigned long long *out) {
    const int k = blockIdx.y;
    if (k >= a.n) return;
    long long s = 0;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    if (a.elem_bytes == 4) {
        const int *r = static_cast<const int *>(a.row[k]);
        int done = 0;
        if ((reinterpret_cast<uintptr_t>(r) & 15u) == 0 && (reinterpret_cast<uintptr_t>(coef) & 15u) == 0) {
            const int n4 = a.m >> 2;
            const int4 *r4 = reinterpret_cast<const int4 *>(r);
            const int4 *c4 = reinterpret_cast<const int4 *>(coef);
            for (int i = tid; i < n4; i += 4 * stride) {
                int4 x[4], c[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int j = i + u * stride;
                    x[u] = j < n4 ? __ldcs(r4 + j) : make_int4(0, 0, 0, 0);
                    c[u] = j < n4 ? __ldg(c4 + j) : make_int4(0, 0, 0, 0);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    s += dot_term(x[u].x, c[u].x) + dot_term(x[u].y, c[u].y) + dot_term(x[u].z, c[u].z) +
                         dot_term(x[u].w, c[u].w);
            }
            done = n4 << 2;
        }
        for (int i = done + tid; i < a.m; i += stride) s += dot_term(__ldcs(r + i), __ldg(coef + i));
    } else {
        const unsigned char *r = static_cast<const unsigned char *>(a.row[k]);
        for (int i = tid; i < a.m; i += stride) s += dot_term(r[i], __ldg(coef + i));
    }
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s != 0) atomicAdd(out + a.slot[k], static_cast<unsigned long long>(s));
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" apspie_status apspie_row_checksums(apspie_ctx *ctx, const void *const *h_rows, const int32_t *h_slots,
                                              int32_t nrows, int32_t m, int32_t elem_bytes, const int32_t *d_coef,
                                              int64_t *d_out) {
    if (!ctx) return APSPIE_ERR_INVALID_ARG;
    if (nrows < 0 || m < 0 || (elem_bytes != 1 && elem_bytes != 4) ||
        (nrows > 0 && (!h_rows || !h_slots || !d_coef || !d_out)))
        return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_row_checksums: bad arguments");
    cudaSetDevice(ctx->device);
    const int bx = std::max(1, std::min((m + kSumBlock - 1) / kSumBlock,
                                        std::max(1, 16 * ctx->num_sms / std::max(1, nrows) + 1)));
    for (int r0 = 0; r0 < nrows; r0 += kSumRows) {
        SumArgs a;
        a.n = std::min(kSumRows, nrows - r0);
        a.m = m;
        a.elem_bytes = elem_bytes;
        for (int k = 0; k < a.n; ++k) {
            if (!h_rows[r0 + k] || h_slots[r0 + k] < 0)
                return set_error(ctx, APSPIE_ERR_INVALID_ARG, "apspie_row_checksums: NULL row or negative slot");
            a.row[k] = h_rows[r0 + k];
            a.slot[k] = h_slots[r0 + k];
        }
        if (m > 0)
            row_checksums<<<dim3(bx, a.n), kSumBlock, 0, ctx->stream>>>(a, d_coef,
                                                                  reinterpret_cast<unsigned long long *>(d_out));
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? APSPIE_OK : cuda_error(ctx, e, "apspie_row_checksums");
}
