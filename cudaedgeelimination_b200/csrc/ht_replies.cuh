// Hamilton and end replies of the HT prover's OR moves (src/cuda/ht_replies.cu:406-520 in the
// reference; semantics src/cpu/hamilton_tutte.cpp:230-282).
//
// Each list is built in two passes over the same device routine, so that the counts and the lists
// cannot disagree: a count pass (replies per center / task), the offsets (an exclusive prefix sum on
// the host, which returns them to the caller anyway), then a write pass that stores each reply at
// its place. One warp per center: the center's neighbour pairs (a, b), a < b in CSR order, are
// flattened a-major (the reference's nested-loop order) and tested 32 at a time; a ballot gives the
// replies of a round, and each lane writes its own at the running offset plus the replies of lower
// lanes, so the list comes out in the reference's order without a sort. Rows of up to 32 neighbours
// keep each neighbour's coordinates, center edge cost and 2-opt survival in its lane; longer rows
// recompute them per pair. End replies: one warp per task, lanes over the endpoint's row.
#pragma once

#include "device_common.cuh"

namespace cee {

constexpr int kReplyWarps = 8;

struct ReplyArgs {
  const int2* __restrict__ xy;  // coordinates relative to the bounding-box corner
  int32_t dist_type;
  const int32_t* __restrict__ row_offsets;
  const int32_t* __restrict__ nbr;
  int32_t tu, tv;  // target, tu < tv
  const int32_t* __restrict__ centers;
  int64_t count;
  unsigned long long* counts;         // count pass: replies per center
  const unsigned long long* offsets;  // write pass: [count + 1]
  int32_t* out;                       // write pass: (center, first, second) per reply
  int32_t* error;                     // 2: a write past the counted range, 4: count and write disagree
};

struct EndReplyArgs {
  const int32_t* __restrict__ row_offsets;
  const int32_t* __restrict__ nbr;
  const int2* __restrict__ tasks;  // (endpoint, internal neighbour)
  int64_t count;
  unsigned long long* counts;
  const unsigned long long* offsets;
  int2* out;       // (lower, higher)
  int32_t* error;  // 1: the internal neighbour is not in the endpoint's row, 2 and 4 as above
};

// (a, b), a < b, of index p of the a-major order of a row of d neighbours:
// p = a (2d - a - 1) / 2 + (b - a - 1). An FP32 estimate of a, then exact integer steps.
__device__ __forceinline__ void reply_pair_of_index(int64_t p, int d, int& a, int& b) {
  const float twod = 2.0f * static_cast<float>(d) - 1.0f;
  a = static_cast<int>((twod - sqrtf(fmaxf(twod * twod - 8.0f * static_cast<float>(p), 0.0f))) * 0.5f);
  a = max(0, min(a, d - 2));
  while (a > 0 && static_cast<int64_t>(a) * (2 * d - a - 1) / 2 > p) --a;
  while (a < d - 2 && static_cast<int64_t>(a + 1) * (2 * d - a - 2) / 2 <= p) ++a;
  b = static_cast<int>(p - static_cast<int64_t>(a) * (2 * d - a - 1) / 2) + a + 1;
}

template <int kSpan, bool kWrite>
static __global__ void __launch_bounds__(kReplyWarps * 32) ht_reply_kernel(ReplyArgs A) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kReplyWarps;
  const int2 pu = __ldg(A.xy + A.tu), pv = __ldg(A.xy + A.tv);
  const uint32_t cuv = exact_distance<kSpan>(pu, pv, A.dist_type);
  const unsigned below = (1u << lane) - 1u;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kReplyWarps + (threadIdx.x >> 5); i < A.count; i += warps) {
    const int32_t center = __ldg(A.centers + i);
    const int32_t r0 = __ldg(A.row_offsets + center), deg = __ldg(A.row_offsets + center + 1) - r0;
    const int2 pc = __ldg(A.xy + center);
    const uint32_t cuc = exact_distance<kSpan>(pu, pc, A.dist_type), cvc = exact_distance<kSpan>(pv, pc, A.dist_type);
    const uint64_t center_target = static_cast<uint64_t>(cuc) + cvc;
    // neighbour j: node, coordinates, C(center, j), and whether edge (center, j) survives 2-opt
    // against the target (EdgesSurviveTwoOpt, src/cpu/hamilton_tutte.cpp:79-87, on the canonical edge)
    auto neighbour = [&](int j, int32_t& node, int2& p, uint32_t& cost, bool& survives) {
      node = __ldg(A.nbr + r0 + j);
      p = __ldg(A.xy + node);
      cost = exact_distance<kSpan>(pc, p, A.dist_type);
      const bool center_low = center < node;
      const uint32_t cu_o = exact_distance<kSpan>(pu, p, A.dist_type), cv_o = exact_distance<kSpan>(pv, p, A.dist_type);
      const uint64_t original = static_cast<uint64_t>(cuv) + cost;
      const uint64_t first = center_low ? static_cast<uint64_t>(cu_o) + cvc : static_cast<uint64_t>(cuc) + cv_o;
      const uint64_t second = center_low ? static_cast<uint64_t>(cuc) + cv_o : static_cast<uint64_t>(cu_o) + cvc;
      survives = first >= original || second >= original;
    };
    int32_t my_node = -1;
    int2 my_p = make_int2(0, 0);
    uint32_t my_cost = 0;
    bool my_survives = false;
    if (deg <= 32 && lane < deg) neighbour(lane, my_node, my_p, my_cost, my_survives);
    const int64_t pairs = deg < 2 ? 0 : static_cast<int64_t>(deg) * (deg - 1) / 2;
    unsigned long long at = 0, end = 0;
    if constexpr (kWrite) {
      at = A.offsets[i];
      end = A.offsets[i + 1];
    }
    unsigned long long count = 0;
    for (int64_t base = 0; base < pairs; base += 32) {
      const int64_t p = base + lane;
      int a = 0, b = 1;
      if (p < pairs) reply_pair_of_index(p, deg, a, b);
      int32_t na = -1, nb = -1;
      int2 qa = make_int2(0, 0), qb = make_int2(0, 0);
      uint32_t ca = 0, cb = 0;
      bool sa = false, sb = false;
      if (deg <= 32) {
        na = __shfl_sync(kFullMask, my_node, a);
        nb = __shfl_sync(kFullMask, my_node, b);
        qa = make_int2(__shfl_sync(kFullMask, my_p.x, a), __shfl_sync(kFullMask, my_p.y, a));
        qb = make_int2(__shfl_sync(kFullMask, my_p.x, b), __shfl_sync(kFullMask, my_p.y, b));
        ca = __shfl_sync(kFullMask, my_cost, a);
        cb = __shfl_sync(kFullMask, my_cost, b);
        sa = __shfl_sync(kFullMask, my_survives, a);
        sb = __shfl_sync(kFullMask, my_survives, b);
      } else if (p < pairs) {
        neighbour(a, na, qa, ca, sa);
        neighbour(b, nb, qb, cb, sb);
      }
      bool reply = false;
      if (p < pairs && sa && sb && !(min(na, nb) == A.tu && max(na, nb) == A.tv)) {
        const uint64_t original = static_cast<uint64_t>(cuv) + ca + cb;
        const uint64_t replacement = static_cast<uint64_t>(exact_distance<kSpan>(qa, qb, A.dist_type)) + center_target;
        reply = original <= replacement;
      }
      const unsigned mask = __ballot_sync(kFullMask, reply);
      if constexpr (kWrite) {
        if (reply) {
          const unsigned long long pos = at + static_cast<unsigned>(__popc(mask & below));
          if (pos < end) {
            A.out[3 * pos] = center;
            A.out[3 * pos + 1] = na;
            A.out[3 * pos + 2] = nb;
          } else {
            atomicOr(A.error, 2);
          }
        }
        at += static_cast<unsigned>(__popc(mask));
      } else {
        count += static_cast<unsigned>(__popc(mask));
      }
    }
    if (lane == 0) {
      if constexpr (kWrite) {
        if (at != end) atomicOr(A.error, 4);
      } else {
        A.counts[i] = count;
      }
    }
    __syncwarp();
  }
}

template <bool kWrite>
static __global__ void __launch_bounds__(kReplyWarps * 32) ht_end_reply_kernel(EndReplyArgs A) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kReplyWarps;
  const unsigned below = (1u << lane) - 1u;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * kReplyWarps + (threadIdx.x >> 5); i < A.count; i += warps) {
    const int2 task = __ldg(A.tasks + i);
    const int32_t e = task.x, w = task.y;
    const int32_t r0 = __ldg(A.row_offsets + e), r1 = __ldg(A.row_offsets + e + 1);
    unsigned long long at = 0, end = 0, count = 0;
    if constexpr (kWrite) {
      at = A.offsets[i];
      end = A.offsets[i + 1];
    }
    bool found = false;
    for (int32_t s0 = r0; s0 < r1; s0 += 32) {
      const int32_t s = s0 + lane;
      const int32_t nb = s < r1 ? __ldg(A.nbr + s) : -1;
      found = found || __any_sync(kFullMask, s < r1 && nb == w);
      const bool keep = s < r1 && nb != w;
      const unsigned mask = __ballot_sync(kFullMask, keep);
      if constexpr (kWrite) {
        if (keep) {
          const unsigned long long pos = at + static_cast<unsigned>(__popc(mask & below));
          if (pos < end) {
            A.out[pos] = make_int2(min(e, nb), max(e, nb));
          } else {
            atomicOr(A.error, 2);
          }
        }
        at += static_cast<unsigned>(__popc(mask));
      } else {
        count += static_cast<unsigned>(__popc(mask));
      }
    }
    if (lane == 0) {
      if constexpr (kWrite) {
        if (at != end) atomicOr(A.error, 4);
      } else {
        if (!found) atomicOr(A.error, 1);
        A.counts[i] = count;
      }
    }
    __syncwarp();
  }
}

}  // namespace cee
