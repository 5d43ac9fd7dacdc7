// Stable LSD radix sort of (64-bit key, 32-bit value) pairs on the device, shared by the
// graph construction (build.cu) and the sparse-vector product (spmspv.cu). 8-bit digits;
// per pass: per-tile digit counts, one device scan, then a scatter that ranks each tile's
// keys in input order with warp match masks, so equal keys keep their input order.
#pragma once

#include "common.cuh"

namespace apspie {
namespace {

constexpr int kRsBlock = 256;
constexpr int kRsItems = 8;
constexpr int kRsTile = kRsBlock * kRsItems;
constexpr int kRsWarps = kRsBlock / 32;

__global__ void __launch_bounds__(kRsBlock) rs_hist(const unsigned long long *__restrict__ keys, long long n,
                                                    int shift, int *counts, int nblocks) {
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const long long t0 = static_cast<long long>(blockIdx.x) * kRsTile;
#pragma unroll
    for (int j = 0; j < kRsItems; ++j) {
        const long long i = t0 + j * kRsBlock + threadIdx.x;
        if (i < n) atomicAdd(&h[(__ldg(keys + i) >> shift) & 255u], 1);
    }
    __syncthreads();
    counts[static_cast<long long>(threadIdx.x) * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: keys are taken in input order (round j, thread t handles
// element j * 256 + t); a key's place is its digit's global offset for this tile, plus the
// keys of that digit in earlier rounds, in earlier warps of this round, and in earlier
// lanes of its warp (match mask).
__global__ void __launch_bounds__(kRsBlock) rs_scatter(const unsigned long long *__restrict__ kin,
                                                       const unsigned *__restrict__ vin,
                                                       unsigned long long *kout, unsigned *vout, long long n,
                                                       int shift, const int *__restrict__ offs, int nblocks) {
    __shared__ int base[256];
    __shared__ int wh[kRsWarps][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    base[tid] = offs[static_cast<long long>(tid) * nblocks + blockIdx.x];
    const long long t0 = static_cast<long long>(blockIdx.x) * kRsTile;
#pragma unroll 1
    for (int j = 0; j < kRsItems; ++j) {
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) wh[w][tid] = 0;
        __syncthreads();
        const long long i = t0 + j * kRsBlock + tid;
        const bool valid = i < n;
        const unsigned long long key = valid ? kin[i] : 0ull;
        const unsigned val = valid ? vin[i] : 0u;
        const int d = valid ? static_cast<int>((key >> shift) & 255u) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0) wh[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int pos = base[d] + rank;
            for (int w = 0; w < warp; ++w) pos += wh[w][d];
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        int add = 0;
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) add += wh[w][tid];
        base[tid] += add;
        __syncthreads();
    }
}

struct SortBufs {
    unsigned long long *k[2];
    unsigned *v[2];
    int *counts, *offs;
    void *scan_tmp;
    int *ovf;
};

// The scan scratch serves the digit-count scans (nc entries) and the callers' scans of up
// to n + 1 entries.
size_t sort_need(long long n) {
    const long long nb = (n + kRsTile - 1) / kRsTile;
    const long long nc = 256 * (nb > 0 ? nb : 1);
    const long long ns = nc > n + 1 ? nc : n + 1;
    return Carver::need({static_cast<size_t>(n) * 8, static_cast<size_t>(n) * 8, static_cast<size_t>(n) * 4,
                         static_cast<size_t>(n) * 4, static_cast<size_t>(nc) * 4, static_cast<size_t>(nc + 1) * 4,
                         scan_scratch_bytes(ns) + 64, 64});
}

SortBufs carve_sort(Carver &c, long long n) {
    const long long nb = (n + kRsTile - 1) / kRsTile;
    const long long nc = 256 * (nb > 0 ? nb : 1);
    const long long ns = nc > n + 1 ? nc : n + 1;
    SortBufs s;
    s.k[0] = c.take<unsigned long long>(n);
    s.k[1] = c.take<unsigned long long>(n);
    s.v[0] = c.take<unsigned>(n);
    s.v[1] = c.take<unsigned>(n);
    s.counts = c.take<int>(nc);
    s.offs = c.take<int>(nc + 1);
    s.scan_tmp = c.take<char>(scan_scratch_bytes(ns) + 64);
    s.ovf = c.take<int>(16);
    return s;
}

// Sorts (k[0], v[0]) by the low `bits` bits of the keys, stably; returns which buffer
// pair holds the result.
apspie_status radix_sort(apspie_ctx *ctx, SortBufs &s, long long n, int bits, int *which) {
    int cur = 0;
    const long long nb = (n + kRsTile - 1) / kRsTile;
    for (int shift = 0; shift < bits && n > 1; shift += 8) {
        rs_hist<<<static_cast<int>(nb), kRsBlock, 0, ctx->stream>>>(s.k[cur], n, shift, s.counts,
                                                                    static_cast<int>(nb));
        apspie_status st = device_exclusive_scan(ctx, s.counts, 256 * nb, s.offs, s.scan_tmp, s.ovf);
        if (st != APSPIE_OK) return st;
        rs_scatter<<<static_cast<int>(nb), kRsBlock, 0, ctx->stream>>>(s.k[cur], s.v[cur], s.k[cur ^ 1],
                                                                       s.v[cur ^ 1], n, shift, s.offs,
                                                                       static_cast<int>(nb));
        cur ^= 1;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(ctx, e, "radix sort");
    *which = cur;
    return APSPIE_OK;
}

int bit_length(long long x) {  // bits needed for values 0 .. x-1 (at least 1)
    int b = 1;
    while ((1LL << b) < x) ++b;
    return b;
}

__global__ void coo_keys(long long ne, int m, const int *__restrict__ src, const int *__restrict__ dst,
                         const unsigned *__restrict__ w, int B, int symmetrize, int drop_loops,
                         unsigned long long *keys, unsigned *vals, int *bad) {
    const unsigned long long sentinel = (1ull << (2 * B)) - 1ull;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < ne;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        int u = __ldg(src + k), v = __ldg(dst + k);
        if (u < 0 || u >= m || v < 0 || v >= m) {
            atomicOr(bad, 1);
            u = v = 0;
        }
        if (symmetrize && u > v) {
            const int t = u;
            u = v;
            v = t;
        }
        keys[k] = (drop_loops && u == v) ? sentinel
                                         : ((static_cast<unsigned long long>(u) << B) | static_cast<unsigned>(v));
        vals[k] = w ? __ldg(w + k) : 0u;
    }
}

// keep[i]: key i is not the sentinel and (without dedup, or) differs from key i - 1.
__global__ void mark_keep(long long n, const unsigned long long *__restrict__ keys, unsigned long long sentinel,
                          int dedup, int *keep) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const unsigned long long k = keys[i];
        keep[i] = (k != sentinel && (!dedup || i == 0 || keys[i - 1] != k)) ? 1 : 0;
    }
}

__global__ void compact_kv(long long n, const unsigned long long *__restrict__ kin, const unsigned *__restrict__ vin,
                           const int *__restrict__ keep, const int *__restrict__ pos, unsigned long long *kout,
                           unsigned *vout) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        if (keep[i]) {
            kout[pos[i]] = kin[i];
            vout[pos[i]] = vin[i];
        }
}

}  // namespace
}  // namespace apspie
