// Device-side building blocks shared by the screen kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cee {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr uint64_t kEmptyKey = ~uint64_t{0};

// Exact TSPLIB distance between two points whose coordinates are stored relative to the
// snapshot's bounding-box corner, so 0 <= x, y < 2^30 and the result fits int32.
//
// The reference computes floor(sqrt(s)) with an integer restoring square root
// (src/common/distance.cpp:9-27) and then rounds: EUC_2D adds 1 when s - q^2 > q (nearest
// integer, ties impossible for integer s), CEIL_2D adds 1 when q^2 != s (:44-52). Here the
// root estimate is the correctly rounded FP64 sqrt of s (s < 2^61, so double(s) carries a
// relative error <= 2^-53 and the estimate lies within 2^-21 of sqrt(s)); truncating it can
// therefore only be one too high (sqrt(s) just below an integer) or one too low (s a
// perfect square just above the estimate), which the two integer comparisons correct, so q
// equals floor(sqrt(s)) exactly and the rounding below is the reference's, bit for bit.
__device__ __forceinline__ uint32_t exact_distance(int2 p, int2 q, int dist_type) {
  const int64_t dx = static_cast<int64_t>(p.x) - q.x;
  const int64_t dy = static_cast<int64_t>(p.y) - q.y;
  const uint64_t s = static_cast<uint64_t>(dx * dx + dy * dy);
  uint64_t r = static_cast<uint64_t>(sqrt(static_cast<double>(s)));
  if (r * r > s) {
    --r;
  } else if ((r + 1) * (r + 1) <= s) {
    ++r;
  }
  const uint64_t rem = s - r * r;
  const uint64_t up = dist_type == 0 ? (rem > r ? 1u : 0u) : (rem != 0 ? 1u : 0u);
  return static_cast<uint32_t>(r + up);
}

// Ascending bitonic sort of one 64-bit key per lane across a full warp.
__device__ __forceinline__ uint64_t warp_sort_asc(uint64_t key, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const uint64_t other = __shfl_xor_sync(kFullMask, key, j);
      const bool ascending = (lane & k) == 0;
      const bool lower = (lane & j) == 0;
      key = (lower == ascending) ? min(key, other) : max(key, other);
    }
  }
  return key;
}

// Given two ascending warp-wide lists, returns the 32 smallest keys of their union,
// ascending (min against the reversed second list yields a bitonic sequence holding them;
// one bitonic merge pass sorts it).
__device__ __forceinline__ uint64_t warp_merge_smallest(uint64_t top, uint64_t batch, int lane) {
  const uint64_t reversed = __shfl_sync(kFullMask, batch, 31 - lane);
  uint64_t key = min(top, reversed);
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) {
    const uint64_t other = __shfl_xor_sync(kFullMask, key, j);
    key = (lane & j) == 0 ? min(key, other) : max(key, other);
  }
  return key;
}

// Inclusive warp prefix sum.
__device__ __forceinline__ int warp_inclusive_sum(int value, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int other = __shfl_up_sync(kFullMask, value, d);
    if (lane >= d) value += other;
  }
  return value;
}

// Binary search for `needle` in the ascending slice nbr[lo, hi).
__device__ __forceinline__ bool row_contains(const int32_t* __restrict__ nbr, int32_t lo,
                                             int32_t end, int32_t needle) {
  int32_t hi = end;
  while (lo < hi) {
    const int32_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(nbr + mid) < needle) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  return lo < end && __ldg(nbr + lo) == needle;
}

}  // namespace cee
