// Device-side building blocks shared by the screen kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cee {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr uint64_t kEmptyKey = ~uint64_t{0};

// Exact TSPLIB distance between two points whose coordinates are stored relative to the
// snapshot's bounding-box corner (0 <= x, y < 2^30, so the result fits int32).
//
// The reference computes q = floor(sqrt(s)) of the squared distance s with an integer
// restoring square root (src/common/distance.cpp:9-27) and rounds: EUC_2D adds 1 when
// s - q^2 > q (nearest integer; s is an integer so there are no ties), CEIL_2D adds 1 when
// q^2 != s (:44-52). Both variants below return exactly that value.
//
// kWide = false (coordinate span < 2^26, so s < 2^53): everything in FP64. dx, dy, s and
// q^2 - s are exact in double below 2^53; q = trunc(sqrt(s)) with the correctly rounded FP64
// square root; the two fma residuals then move q by one step if the root landed on the wrong
// side of an integer (provably never for s < 2^52, kept as a check), and give s - q^2 exactly
// for the rounding decision.
// kWide = true (span up to 2^30, s < 2^61): s in uint64, FP64 root estimate within 2^-21 of
// sqrt(s) (double(s) has relative error <= 2^-53), integer fix-up by one step either way.
template <bool kWide>
__device__ __forceinline__ uint32_t exact_distance(int2 p, int2 q, int dist_type) {
  if constexpr (kWide) {
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
  } else {
    const double dx = static_cast<double>(p.x - q.x);
    const double dy = static_cast<double>(p.y - q.y);
    const double s = fma(dx, dx, dy * dy);
    double r = trunc(sqrt(s));
    double below = fma(r, r, -s);  // r^2 - s
    if (below > 0.0) {
      r -= 1.0;
      below = fma(r, r, -s);
    } else if (fma(r + 1.0, r + 1.0, -s) <= 0.0) {
      r += 1.0;
      below = fma(r, r, -s);
    }
    const double rem = -below;  // s - r^2 >= 0
    const bool up = dist_type == 0 ? rem > r : rem != 0.0;
    return static_cast<uint32_t>(r) + (up ? 1u : 0u);
  }
}

// Distances with a span below this bound are evaluated with exact_distance<false>.
constexpr int64_t kNarrowSpan = int64_t{1} << 26;

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

// The same network on 32-bit keys.
__device__ __forceinline__ uint32_t warp_sort_asc32(uint32_t key, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const uint32_t other = __shfl_xor_sync(kFullMask, key, j);
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
