// Exclusive prefix sum of int32 counts into int64 offsets (three passes:
// per-block sums, scan of the block sums in one block, block-local scan).
// Writes out[0..n] with out[n] = total and returns the total on the host.
#pragma once

#include "problem.cuh"

namespace sphgpu {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS*SCAN_ITEMS;

__device__ __forceinline__ int64_t warp_incl_scan(int64_t v) {
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan; returns the exclusive prefix of `v`, sets *total.
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* total) {
  __shared__ int64_t wsum[SCAN_THREADS/32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t inc = warp_incl_scan(v);
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    int64_t s = lane < SCAN_THREADS/32 ? wsum[lane] : 0;
    s = warp_incl_scan(s);
    if (lane < SCAN_THREADS/32) wsum[lane] = s;
  }
  __syncthreads();
  const int64_t before = (w > 0 ? wsum[w - 1] : 0) + inc - v;
  *total = wsum[SCAN_THREADS/32 - 1];
  __syncthreads();
  return before;
}

__global__ void scan_tile_sums_kernel(const int32_t* in, int64_t n, int64_t* tileSums) {
  const int64_t base = (int64_t)blockIdx.x*SCAN_TILE;
  int64_t s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int64_t idx = base + (int64_t)k*SCAN_THREADS + threadIdx.x;
    if (idx < n) s += in[idx];
  }
  int64_t total;
  block_excl_scan(s, &total);
  if (threadIdx.x == 0) tileSums[blockIdx.x] = total;
}

__global__ void scan_sums_kernel(int64_t* tileSums, int64_t ntiles, int64_t* totalOut) {
  int64_t carry = 0;
  for (int64_t base = 0; base < ntiles; base += SCAN_THREADS) {
    const int64_t idx = base + threadIdx.x;
    const int64_t v = idx < ntiles ? tileSums[idx] : 0;
    int64_t total;
    const int64_t ex = block_excl_scan(v, &total);
    if (idx < ntiles) tileSums[idx] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *totalOut = carry;
}

__global__ void scan_apply_kernel(const int32_t* in, int64_t n, const int64_t* tileSums, int64_t* out,
                                  const int64_t* totalIn) {
  const int64_t base = (int64_t)blockIdx.x*SCAN_TILE;
  // each thread owns SCAN_ITEMS consecutive elements
  int32_t v[SCAN_ITEMS];
  int64_t s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int64_t idx = base + (int64_t)threadIdx.x*SCAN_ITEMS + k;
    v[k] = idx < n ? in[idx] : 0;
    s += v[k];
  }
  int64_t total;
  int64_t run = block_excl_scan(s, &total) + tileSums[blockIdx.x];
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int64_t idx = base + (int64_t)threadIdx.x*SCAN_ITEMS + k;
    if (idx < n) out[idx] = run;
    run += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = *totalIn;
}

}  // namespace sphgpu
