// Device-side helpers shared by the SpGEMM kernels: warp scans, the
// column hash, compensated-arithmetic primitives and the status word.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sg {

constexpr unsigned FULL = 0xffffffffu;
constexpr unsigned EMPTY_KEY = 0xffffffffu;

// Bits of the device status word (atomicOr'ed by kernels, read by the host
// at each synchronisation point). Kernels never trap: a failed check records
// its bit and skips the access.
enum StatusBits : unsigned {
  ST_TABLE_FULL = 1u << 0,      // hash probe ran past the table size
  ST_COUNT_MISMATCH = 1u << 1,  // numeric pass found a different nnz than symbolic
  ST_ROW_TOO_LONG = 1u << 2,    // a row has >= 2^31 partial products
  ST_SLICE_OVERFLOW = 1u << 3,  // long-row slice list capacity exceeded
  ST_BAD_INDEX = 1u << 4,       // an input index was outside its dimension
  ST_UNSORTED = 1u << 5         // a row of B is not sorted by column
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int t = __shfl_up_sync(FULL, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

__device__ __forceinline__ long long warp_incl_scan64(long long v) {
  const int lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    long long t = __shfl_up_sync(FULL, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
  return v;
}

// Multiplicative (Fibonacci) hashing of a column index into 2^log2n slots.
__device__ __forceinline__ unsigned hash_col(unsigned c, int log2n) {
  return (c * 2654435769u) >> (32 - log2n);
}

// Error of s = fl(a + b) (Knuth's TwoSum): a + b == s + err exactly.
// Explicit _rn intrinsics keep the compiler from contracting or
// reassociating the sequence.
__device__ __forceinline__ float two_sum_err(float a, float b, float s) {
  float bb = __fsub_rn(s, a);
  float aa = __fsub_rn(s, bb);
  return __fadd_rn(__fsub_rn(a, aa), __fsub_rn(b, bb));
}

// Lower bound of `key` in the sorted array v[lo, hi).
__device__ __forceinline__ int lower_bound_i32(const int* __restrict__ v, int lo,
                                               int hi, int key) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(v + mid) < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

}  // namespace sg
