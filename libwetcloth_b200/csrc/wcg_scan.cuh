// Device-wide exclusive prefix sum and deterministic reductions.
// Three-pass scan: per-tile sums, a single-block scan of the tile sums, then a
// per-tile scan with the tile offset.  Deterministic (fixed summation order).
#pragma once

#include <cuda_runtime.h>

namespace wcg {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ inline T block_exclusive_scan(T v, T* smem, T& total) {
  // smem: kScanThreads / 32 + 1 entries
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    T w = lane < nw ? smem[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) smem[lane] = w;
  }
  __syncthreads();
  const T warp_prefix = warp ? smem[warp - 1] : T(0);
  total = smem[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

template <typename TIn, typename TOut>
__global__ void scan_tile_sums(const TIn* __restrict__ in, long long n,
                               TOut* __restrict__ tile_sums) {
  __shared__ TOut sm[kScanThreads / 32 + 1];
  const long long base = (long long)blockIdx.x * kScanTile;
  TOut s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long long i = base + (long long)k * kScanThreads + threadIdx.x;
    if (i < n) s += (TOut)in[i];
  }
  TOut total;
  block_exclusive_scan<TOut>(s, sm, total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

template <typename TOut>
__global__ void scan_tile_offsets(TOut* __restrict__ tile_sums, long long ntiles,
                                  TOut* __restrict__ grand_total) {
  __shared__ TOut sm[kScanThreads / 32 + 1];
  TOut carry = 0;
  for (long long b = 0; b < ntiles; b += kScanThreads) {
    const long long i = b + threadIdx.x;
    const TOut v = i < ntiles ? tile_sums[i] : TOut(0);
    TOut total;
    const TOut ex = block_exclusive_scan<TOut>(v, sm, total);
    if (i < ntiles) tile_sums[i] = ex + carry;
    carry += total;
  }
  if (threadIdx.x == 0 && grand_total) *grand_total = carry;
}

// out[i] = sum_{j<i} in[j]; out may alias in.  Items of a thread are strided
// by kScanThreads so loads stay coalesced; the scan order is item-major.
template <typename TIn, typename TOut>
__global__ void scan_tiles(const TIn* __restrict__ in, long long n,
                           const TOut* __restrict__ tile_offsets,
                           TOut* __restrict__ out) {
  __shared__ TOut sm[kScanThreads / 32 + 1];
  const long long base = (long long)blockIdx.x * kScanTile;
  TOut carry = tile_offsets[blockIdx.x];
  for (int k = 0; k < kScanItems; ++k) {
    const long long i = base + (long long)k * kScanThreads + threadIdx.x;
    const TOut v = i < n ? (TOut)in[i] : TOut(0);
    TOut total;
    const TOut ex = block_exclusive_scan<TOut>(v, sm, total);
    if (i < n) out[i] = carry + ex;
    carry += total;
  }
}

// Host helper: exclusive scan of n items into out (out[n] = total if
// total_out != nullptr).  tmp must hold ceil(n/kScanTile) TOut.
template <typename TIn, typename TOut>
inline void exclusive_scan(const TIn* in, long long n, TOut* out, TOut* tmp,
                           TOut* total_out, cudaStream_t st) {
  const long long ntiles = (n + kScanTile - 1) / kScanTile;
  if (ntiles == 0) {
    if (total_out) cudaMemsetAsync(total_out, 0, sizeof(TOut), st);
    return;
  }
  scan_tile_sums<TIn, TOut><<<(unsigned)ntiles, kScanThreads, 0, st>>>(in, n, tmp);
  scan_tile_offsets<TOut><<<1, kScanThreads, 0, st>>>(tmp, ntiles, total_out);
  scan_tiles<TIn, TOut><<<(unsigned)ntiles, kScanThreads, 0, st>>>(in, n, tmp, out);
}

}  // namespace wcg
