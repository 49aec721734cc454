// cvl_scan.cuh -- exclusive prefix sums for the CSR offsets, hash-bucket
// starts and output positions (reduce-then-scan: per-tile sums, a scan of the
// tile sums, then a tile scan that adds its offset). No spin waits.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cvl {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total in *total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *total) {
    __shared__ T warp_tot[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const T inc = warp_incl_scan(v, lane);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T t = (lane < SCAN_THREADS / 32) ? warp_tot[lane] : T(0);
        t = warp_incl_scan(t, lane);
        if (lane < SCAN_THREADS / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    const T before = (wid > 0) ? warp_tot[wid - 1] : T(0);
    *total = warp_tot[SCAN_THREADS / 32 - 1];
    __syncthreads();
    return before + inc - v;
}

template <typename TIn, typename TOut>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const TIn *__restrict__ in, size_t n,
                                                               TOut *__restrict__ tile_sums) {
    const size_t base = (size_t)blockIdx.x * SCAN_TILE;
    TOut s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const size_t idx = base + (size_t)k * SCAN_THREADS + threadIdx.x;
        if (idx < n) s += (TOut)in[idx];
    }
    TOut tot;
    (void)block_excl_scan<TOut>(s, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// out[0..n] = exclusive scan of in (out[n] = total), plus tile_offsets[blockIdx] if given.
template <typename TIn, typename TOut>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const TIn *__restrict__ in, size_t n,
                                                              const TOut *__restrict__ tile_offsets,
                                                              TOut *__restrict__ out) {
    const size_t base = (size_t)blockIdx.x * SCAN_TILE;
    TOut v[SCAN_ITEMS];
    TOut s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const size_t idx = base + (size_t)threadIdx.x * SCAN_ITEMS + k;
        v[k] = (idx < n) ? (TOut)in[idx] : TOut(0);
        s += v[k];
    }
    TOut tot;
    TOut run = block_excl_scan<TOut>(s, &tot);
    if (tile_offsets) run += tile_offsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const size_t idx = base + (size_t)threadIdx.x * SCAN_ITEMS + k;
        if (idx < n) out[idx] = run;
        run += v[k];
        if (idx + 1 == n) out[n] = run;
    }
}

}  // namespace cvl
