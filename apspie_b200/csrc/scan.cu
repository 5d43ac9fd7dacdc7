// Device-wide exclusive scan of int32 counts into int32 offsets (plus the total at
// out[n]), the project's own replacement for mgpu::Scan (used by the reference at
// src/mXv.cuh:142,160 and src/spmspvBfs.cuh:178,184 with a D2H count read each time).
// Three short launches: per-block sums, a single-block scan of those sums, and the
// per-block rescan with its base. Totals above INT32_MAX raise APSPIE_ERR_UNSUPPORTED.
#include "common.cuh"

namespace apspie {
namespace {

constexpr int kScanBlock = 512;
constexpr int kScanItems = 4;  // per thread
constexpr int kScanTile = kScanBlock * kScanItems;

__global__ void __launch_bounds__(kScanBlock) scan_block_sums(const int *__restrict__ in, long long n,
                                                              long long *sums) {
    __shared__ int tmp[33];
    const long long base = static_cast<long long>(blockIdx.x) * kScanTile;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const long long i = base + static_cast<long long>(k) * kScanBlock + threadIdx.x;
        if (i < n) s += in[i];
    }
    int tot;
    block_exclusive_scan<kScanBlock>(s, tot, tmp);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) scan_sums(long long *sums, int nb, int *overflow) {
    // one block: sequential chunks of 1024 with carry
    __shared__ long long wsum[32];
    __shared__ long long carry_s;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        long long x = i < nb ? sums[i] : 0;
        long long incl = x;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            long long w = wsum[lane];
            long long wi = w;
            for (int o = 1; o < 32; o <<= 1) {
                long long y = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += y;
            }
            wsum[lane] = wi - w;
        }
        __syncthreads();
        const long long c = carry_s;
        if (i < nb) sums[i] = c + wsum[wid] + incl - x;
        __syncthreads();
        if (threadIdx.x == 1023) carry_s = c + wsum[wid] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[nb] = carry_s;
        if (carry_s > 0x7fffffffLL) *overflow = 1;
    }
}

__global__ void __launch_bounds__(kScanBlock) scan_apply(const int *__restrict__ in, long long n,
                                                         const long long *__restrict__ sums, int *out) {
    __shared__ int tmp[33];
    const long long base = static_cast<long long>(blockIdx.x) * kScanTile;
    // each thread owns kScanItems consecutive elements
    const long long first = base + static_cast<long long>(threadIdx.x) * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (first + k < n) ? in[first + k] : 0;
        s += v[k];
    }
    int tot;
    int run = block_exclusive_scan<kScanBlock>(s, tot, tmp) + static_cast<int>(sums[blockIdx.x]);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (first + k < n) out[first + k] = run;
        run += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = static_cast<int>(sums[gridDim.x]);
}

}  // namespace

size_t scan_scratch_bytes(long long n) {
    const long long nb = (n + kScanTile - 1) / kScanTile;
    return static_cast<size_t>(nb + 2) * sizeof(long long) + 64;
}

// out[0..n) = exclusive prefix of in[0..n), out[n] = total. `tmp` holds scan_scratch_bytes(n).
apspie_status device_exclusive_scan(apspie_ctx *ctx, const int *in, long long n, int *out, void *tmp,
                                    int *overflow_flag) {
    if (n <= 0) {
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(int), ctx->stream);
        return e == cudaSuccess ? APSPIE_OK : cuda_error(ctx, e, "scan memset");
    }
    const long long nb = (n + kScanTile - 1) / kScanTile;
    if (nb > 0x7fffffffLL) return set_error(ctx, APSPIE_ERR_UNSUPPORTED, "scan too long");
    long long *sums = static_cast<long long *>(tmp);
    scan_block_sums<<<static_cast<int>(nb), kScanBlock, 0, ctx->stream>>>(in, n, sums);
    scan_sums<<<1, 1024, 0, ctx->stream>>>(sums, static_cast<int>(nb), overflow_flag);
    scan_apply<<<static_cast<int>(nb), kScanBlock, 0, ctx->stream>>>(in, n, sums, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? APSPIE_OK : cuda_error(ctx, e, "scan launch");
}

}  // namespace apspie
