// ccs_scan.cuh -- exclusive prefix sums on the device (three launches:
// per-tile scans, one block over the tile sums, per-element offsets).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ccs {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 4;                                // per thread
constexpr int kScanTile = kScanBlock * kScanItems;           // per block

// tile sums needed for n elements
inline int64_t scan_tiles(int64_t n) { return n / kScanTile + 2; }

template <class T>
__device__ __forceinline__ T scan_block_exclusive(T x, T* warpSums, T& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) warpSums[w] = incl;
    __syncthreads();
    if (w == 0) {
        T s = lane < kScanBlock / 32 ? warpSums[lane] : T(0);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += y;
        }
        if (lane < kScanBlock / 32) warpSums[lane] = s;      // inclusive over warps
    }
    __syncthreads();
    total = warpSums[kScanBlock / 32 - 1];
    const T before = w > 0 ? warpSums[w - 1] : T(0);
    __syncthreads();
    return before + incl - x;
}

template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(const T* __restrict__ in, T* __restrict__ out,
                                                           T* __restrict__ tileSums, int64_t n) {
    __shared__ T warpSums[kScanBlock / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    T v[kScanItems], sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? in[base + i] : T(0);
        sum += v[i];
    }
    T total;
    T run = scan_block_exclusive<T>(sum, warpSums, total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0) tileSums[blockIdx.x] = total;
}

// one block: exclusive scan of the tile sums in place, grand total to *total
template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(T* __restrict__ sums, int64_t nt, T* __restrict__ total) {
    __shared__ T warpSums[kScanBlock / 32];
    T carry = 0;
    for (int64_t c = 0; c < nt; c += kScanBlock) {
        const int64_t i = c + threadIdx.x;
        const T x = i < nt ? sums[i] : T(0);
        T chunk;
        const T ex = scan_block_exclusive<T>(x, warpSums, chunk);
        if (i < nt) sums[i] = carry + ex;
        carry += chunk;
    }
    if (threadIdx.x == 0) *total = carry;
}

template <class T>
__global__ void __launch_bounds__(kScanBlock) k_scan_add(T* __restrict__ out, const T* __restrict__ tileSums,
                                                         int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) out[i] += tileSums[i / kScanTile];
}

// out[0..n) = exclusive scan of in[0..n) (in place allowed); *total = the
// sum (device); `tiles` holds scan_tiles(n) elements
template <class T>
cudaError_t exclusive_scan(const T* in, T* out, int64_t n, T* tiles, T* total, cudaStream_t s) {
    const int64_t nt = (n + kScanTile - 1) / kScanTile;
    if (nt > 0) k_scan_tiles<T><<<(unsigned)nt, kScanBlock, 0, s>>>(in, out, tiles, n);
    k_scan_sums<T><<<1, kScanBlock, 0, s>>>(tiles, nt, total);
    if (n > 0) k_scan_add<T><<<(unsigned)((n + kScanBlock - 1) / kScanBlock), kScanBlock, 0, s>>>(out, tiles, n);
    return cudaGetLastError();
}

}  // namespace ccs
