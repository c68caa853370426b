// Device-wide exclusive scan in three steps fused into the kernels around it (used by the
// hierarchy builders for the per-round and per-level compactions):
//
//   producer kernel   writes its values and, per block of kScanBlock threads, their sum
//                     (block_total)
//   k_scan_totals     one block scans the block sums in place (exclusive) and appends
//                     the grand total
//   consumer kernel   recomputes its block's exclusive scan of the same values in shared
//                     memory and adds the block's scanned sum (block_exclusive_scan)
//
// Producer and consumer use the same block size and grid (block b covers values
// [b * kScanBlock, (b + 1) * kScanBlock)); both call the block helpers from every thread.
#pragma once
#include <cuda_runtime.h>

namespace eos {

constexpr int kScanBlock = 256;

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T u = __shfl_up_sync(0xffffffffu, v, off);
    if (lane >= off) v += u;
  }
  return v;
}

// Exclusive scan of one value per thread over the block (blockDim.x a multiple of 32, at
// most 1024); every thread gets its exclusive prefix and the block's total.
template <class T>
__device__ __forceinline__ T block_exclusive_scan(T v, T& total) {
  __shared__ T warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
  const T inc = warp_inclusive_scan(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const T s = lane < n_warps ? warp_sums[lane] : T(0);
    warp_sums[lane] = warp_inclusive_scan(s);  // inclusive prefix of the warp sums
  }
  __syncthreads();
  total = warp_sums[n_warps - 1];
  const T ex = inc - v + (warp > 0 ? warp_sums[warp - 1] : T(0));
  __syncthreads();  // warp_sums is reused by the next call
  return ex;
}

// Sum of one value per thread over the block, written to totals[blockIdx.x].
template <class T>
__device__ __forceinline__ void block_total(T v, T* totals) {
  T total;
  block_exclusive_scan(v, total);
  if (threadIdx.x == 0) totals[blockIdx.x] = total;
}

// In-place exclusive scan of totals[0, n_blocks) by one block of 1024 threads;
// totals[n_blocks] = the grand total.
template <class T>
__global__ void __launch_bounds__(1024) k_scan_totals(T* __restrict__ totals, int n_blocks) {
  T carry = T(0);
  for (int base = 0; base < n_blocks; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const T v = i < n_blocks ? totals[i] : T(0);
    T chunk;
    const T ex = block_exclusive_scan(v, chunk);
    if (i < n_blocks) totals[i] = carry + ex;
    carry += chunk;
  }
  if (threadIdx.x == 0) totals[n_blocks] = carry;
}

inline int scan_blocks(long long n) { return (int)((n + kScanBlock - 1) / kScanBlock); }

}  // namespace eos
