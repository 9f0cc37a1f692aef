// Hamilton-Tutte c,d root screen over caller-built tasks.
//
// Semantics (src/cpu/hamilton_tutte.cpp:79-101, src/cuda/ht_cd.cu:157-178): for target (u,v)
// and task (c,d), incompatible = C(u,d)+C(v,c) < C(u,v)+C(c,d) and C(u,c)+C(v,d) < C(u,v)+C(c,d)
// (neither 2-opt orientation survives); flag = active && incompatible in mode
// kActiveIncompatible, !active || incompatible in mode kMissingOrIncompatible.
#pragma once

#include "device_common.cuh"

namespace cee {

// One task in the reference's HtCdScreenTask layout: int32 c, int32 d, uint8 active (+3 pad).
struct CdTask {
  int32_t c;
  int32_t d;
  uint32_t active_word;  // low byte = active
};

template <int kSpan>
__device__ __forceinline__ uint8_t cd_flag(int2 pu, int2 pv, uint32_t cuv, int2 pc, int2 pd,
                                           bool active, int mode, int dist_type) {
  const uint64_t original = static_cast<uint64_t>(cuv) + exact_distance<kSpan>(pc, pd, dist_type);
  const uint64_t orient0 =
      static_cast<uint64_t>(exact_distance<kSpan>(pu, pd, dist_type)) + exact_distance<kSpan>(pv, pc, dist_type);
  const uint64_t orient1 =
      static_cast<uint64_t>(exact_distance<kSpan>(pu, pc, dist_type)) + exact_distance<kSpan>(pv, pd, dist_type);
  const bool incompatible = orient0 < original && orient1 < original;
  return static_cast<uint8_t>(mode == 0 ? (active && incompatible) : (!active || incompatible));
}

template <int kSpan>
static __global__ void cd_screen_kernel(int32_t u, int32_t v, const CdTask* __restrict__ tasks,
                                 int64_t count, const int2* __restrict__ xy, int32_t n,
                                 int32_t dist_type, int32_t mode, uint8_t* __restrict__ flags,
                                 int32_t* __restrict__ error) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const CdTask t = tasks[i];
  if (static_cast<uint32_t>(t.c) >= static_cast<uint32_t>(n) ||
      static_cast<uint32_t>(t.d) >= static_cast<uint32_t>(n)) {
    atomicOr(error, 1);
    flags[i] = 0;
    return;
  }
  const int2 pu = __ldg(xy + u), pv = __ldg(xy + v);
  flags[i] = cd_flag<kSpan>(pu, pv, exact_distance<kSpan>(pu, pv, dist_type), __ldg(xy + t.c), __ldg(xy + t.d),
                     (t.active_word & 0xffu) != 0, mode, dist_type);
}

}  // namespace cee
