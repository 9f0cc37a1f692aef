// Device-side building blocks shared by the screen kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cee {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr uint64_t kEmptyKey = ~uint64_t{0};

// Coordinate span classes: the larger of a snapshot's x and y spans selects the exact-distance
// routine (a template parameter of every kernel that evaluates distances).
constexpr int kSpanSmall = 0;   // span < 2^21: FP32 root estimate, int32 residual
constexpr int kSpanNarrow = 1;  // span < 2^26: FP64
constexpr int kSpanWide = 2;    // span < 2^30: int64 residual
constexpr int kSpanClasses = 3;
constexpr int64_t kSmallSpan = int64_t{1} << 21;
constexpr int64_t kNarrowSpan = int64_t{1} << 26;

// The span class of coordinate spans sx, sy (both < 2^30).
__host__ __device__ constexpr int span_class(int64_t sx, int64_t sy) {
  return (sx < kSmallSpan && sy < kSmallSpan) ? kSpanSmall
         : (sx < kNarrowSpan && sy < kNarrowSpan) ? kSpanNarrow
                                                  : kSpanWide;
}

// sqrt.approx.f32: the SM's one-instruction square-root approximation.
__device__ __forceinline__ float sqrt_estimate(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Exact TSPLIB distance between two points whose coordinates are stored relative to the
// snapshot's bounding-box corner (0 <= x, y < 2^30, so the result fits int32).
//
// The reference computes q = floor(sqrt(s)) of the squared distance s with an integer
// restoring square root (src/common/distance.cpp:9-27) and rounds: EUC_2D adds 1 when
// s - q^2 > q, i.e. returns the nearest integer to sqrt(s) (s is an integer, so there are no
// ties), CEIL_2D adds 1 when q^2 != s, i.e. returns ceil(sqrt(s)) (:44-52). All three variants
// return exactly that value; they differ only in how they reach it.
//
// kSpanSmall (|dx|, |dy| < 2^21, s < 2^43): an FP32 estimate f of sqrt(s), rounded to the
// candidate answer r (nearest for EUC_2D, up for CEIL_2D), then checked and corrected with the
// exact residual t = s - r^2. dx and dy are exact in FP32; the FP32 sum of squares carries a
// relative error of at most 2u + u^2 (u = 2^-24), which the root halves; sqrt.approx.f32 adds
// at most 2^-23.25 (its largest relative error over every float in [1, 2^44), the range the
// FP32 sums of squares of this class fall in, measured exhaustively on the B200 by
// cee_sqrt_estimate_error). So |f - sqrt(s)| <= sqrt(s) * 2^-22.58 <
// 2^21.5 * 2^-22.58 < 0.48, the candidate is within one of the answer, and t lies well inside
// int32, so it is exact when computed modulo 2^32 from wrapped 32-bit products. The answer is r
// iff -r < t <= r (EUC_2D: (r - 1/2)^2 < s < (r + 1/2)^2) or -(2r - 1) < t <= 0 (CEIL_2D:
// (r - 1)^2 < s <= r^2), for r > 0 (r = 0 iff s = 0); one step up or down fixes r otherwise.
// The fix-up makes the routine exact for any estimate within one of sqrt(s), twice the bound.
// kSpanNarrow (span < 2^26, so s < 2^53): everything in FP64. dx, dy, s and q^2 - s are exact
// in double below 2^53; q = trunc(sqrt(s)) with the correctly rounded FP64 square root; the
// two fma residuals then move q by one step if the root landed on the wrong side of an
// integer (provably never for s < 2^52, kept as a check), and give s - q^2 exactly for the
// rounding decision.
// kSpanWide (span up to 2^30, s < 2^61): s in uint64, FP64 root estimate within 2^-21 of
// sqrt(s) (double(s) has relative error <= 2^-53), integer fix-up by one step either way.
template <int kSpan>
__device__ __forceinline__ uint32_t exact_distance(int2 p, int2 q, int dist_type) {
  if constexpr (kSpan == kSpanSmall) {
    const int32_t dx = p.x - q.x, dy = p.y - q.y;
    const float fx = static_cast<float>(dx), fy = static_cast<float>(dy);
    const float f = sqrt_estimate(__fmaf_rn(fx, fx, __fmul_rn(fy, fy)));
    const uint32_t ux = static_cast<uint32_t>(dx), uy = static_cast<uint32_t>(dy);
    const uint32_t s_lo = ux * ux + uy * uy;  // s modulo 2^32
    if (dist_type == 0) {
      uint32_t r = __float2uint_rn(f);
      const int32_t t = static_cast<int32_t>(s_lo - r * r);
      if (t > static_cast<int32_t>(r)) {
        ++r;
      } else if (t <= -static_cast<int32_t>(r) && r > 0) {
        --r;
      }
      return r;
    } else {
      uint32_t r = __float2uint_ru(f);
      const int32_t t = static_cast<int32_t>(s_lo - r * r);
      if (t > 0) {
        ++r;
      } else if (t <= 1 - 2 * static_cast<int32_t>(r) && r > 0) {
        --r;
      }
      return r;
    }
  } else if constexpr (kSpan == kSpanWide) {
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

// The kCount smallest of the warp's 32-bit keys, ascending: lane i < kCount ends with the i-th
// smallest, every other lane with 0xffffffff. Keys other than 0xffffffff (the empty key) must be
// distinct. kCount warp min-reductions, each knocking its key out, cost fewer instructions than
// the 15-stage bitonic network when only the head of the order is wanted.
template <int kCount>
__device__ __forceinline__ uint32_t warp_smallest_asc32(uint32_t key, int lane) {
  uint32_t out = 0xffffffffu;
#pragma unroll
  for (int r = 0; r < kCount; ++r) {
    const uint32_t smallest = __reduce_min_sync(kFullMask, key);
    if (lane == r) out = smallest;
    if (key == smallest) key = 0xffffffffu;
  }
  return out;
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
