// Batched screen: many instances (disjoint snapshots packed into one union snapshot with
// global ids) screened by one persistent kernel. Warps pull work items from an atomic counter:
//
//   [0, I)            target selection of instance i: the first T edges of
//                     SelectHtTargetEdgeIds (src/cpu/ht_scan.cpp:316-345) -- active edges with
//                     both degrees > 2, weight descending, then (u, v, id) ascending;
//   [I, I + J)        JV tiles: `jv_tile` consecutive union edges screened one warp per edge
//                     (jv_screen_edge_warp, same semantics as the single-snapshot screen);
//   [I + J, I + J + I*T)  one HT c,d root screen per target (u, v): BuildCdScreenTasks
//                     (src/cpu/hamilton_tutte.cpp:168-216) -- the `nb` nodes of the instance
//                     other than u, v with degree <= max_degree (0 = no cap) nearest to the
//                     doubled midpoint 2p - p_u - p_v, ties by node -- then every pair i < j of
//                     that neighbourhood as (c, d) = (min, max) screened as ScreenHtCdKernel
//                     (src/cuda/ht_cd.cu:157-178); with max_cd > 0 the item then ranks the
//                     flagged pairs as FinalizeCdCandidates (src/cpu/hamilton_tutte.cpp:283-327):
//                     Hamilton reply count of every neighbourhood node (pairs of its CSR
//                     neighbours, AppendHtHamiltonRepliesUnchecked :230-269), product per pair,
//                     the max_cd smallest (product, c, d).
//
// Spatial chunks: at upload, every instance of at most kSpatialMaxNodes nodes gets its nodes in
// Morton order of their coordinates (perm) cut into chunks of 32 with their bounding boxes. A c,d
// item then visits chunks in increasing order of the smallest doubled-midpoint distance their box
// allows and stops once that bound exceeds the current 25th-best score: every skipped node scores
// above it, so the neighbourhood (the NB smallest (score, node) pairs) is exactly the full scan's,
// from a few chunks instead of the whole instance. Larger instances keep the full scan.
//
// The c,d items of an instance wait (bounded, with an error on timeout) for that instance's
// target-selection item; those items come first in the queue and take a few microseconds, so
// the wait is normally never observed. All CTAs of the grid are resident (the grid is sized
// from the occupancy), so every claimed item runs to completion.
#pragma once

#include "cd_screen.cuh"
#include "jv_screen.cuh"

namespace cee {

constexpr int kBatchWarps = 8;
constexpr int kBatchMaxTargets = 64;
constexpr int kBatchMaxNeighborhood = 32;
constexpr int kBatchMaxPairs = kBatchMaxNeighborhood * (kBatchMaxNeighborhood - 1) / 2;  // 496
constexpr int kBatchFlagWords = (kBatchMaxPairs + 31) / 32;                              // 16
constexpr int32_t kBatchWaitError = 8;
constexpr int32_t kBatchRangeError = 128;  // finalisation: instance > 65536 nodes or a product too large
constexpr int kBatchMaxCd = 32;
constexpr int kSpatialChunk = 32;        // nodes per spatial chunk (one warp pass)
constexpr int kSpatialMaxNodes = 8192;   // larger instances keep the full neighbourhood scan
constexpr int kSpatialMaxChunks = kSpatialMaxNodes / kSpatialChunk;
static_assert(kSpatialMaxNodes <= (1 << 13), "spatial sort keys hold a 13-bit node index");

struct BatchArgs {
  JvGraph g;                          // the union snapshot (global node and edge ids)
  const int64_t* __restrict__ node_begin;  // [instances + 1]
  const int64_t* __restrict__ edge_begin;  // [instances + 1]
  int32_t first_instance, instances;  // this launch covers instances [first, first + instances)
  int32_t targets;                    // T <= 64
  int32_t nb;                         // neighbourhood size, 2..32
  int32_t max_degree;                 // 0 = no cap
  int32_t mode;                       // HtCdMode
  int32_t jv_tile;                    // edges per JV work item
  int32_t flag_words;                 // ceil(nb (nb - 1) / 2 / 32)
  int64_t jv_first, jv_items;         // JV tiles cover union edges [jv_first, jv_first + items * tile) clipped
  int64_t jv_last;
  int32_t* __restrict__ witness;      // [m]
  int32_t* __restrict__ target_ids;   // [I * T] global edge ids, -1 padding
  int32_t* __restrict__ target_count; // [I]
  int32_t* __restrict__ nbhd;         // [I * T * nb] global node ids, -1 padding
  uint32_t* __restrict__ flags;       // [I * T * flag_words] bit p = flag of pair p
  int32_t max_cd;                     // 0: flags only; else finalised candidates per target
  int32_t* __restrict__ cand_c;       // [I * T * max_cd] global node ids
  int32_t* __restrict__ cand_d;
  int64_t* __restrict__ cand_product; // reply products
  int32_t* __restrict__ cand_count;   // [I * T]
  unsigned long long* __restrict__ counter;  // work counter, zero at launch
  int32_t* __restrict__ ready;        // [I] set when the instance's targets are written, zero at launch
  int32_t* __restrict__ error;
  long long wait_limit;               // spin iterations before an item gives up
  const int32_t* __restrict__ perm;        // [n] instance nodes in Morton order (global ids)
  const int4* __restrict__ chunk_box;      // per chunk {min x, max x, min y, max y}
  const int64_t* __restrict__ chunk_begin; // [I + 1]; an instance without chunks has none
};

struct BatchWarpScratch {
  JvWarpScratch jv;
  unsigned long long chunk_bound[kSpatialMaxChunks];  // c,d items: per-chunk score bounds
};

// Spatial chunks of instances [first, first + gridDim.x): one block per instance (kSpatialThreads
// threads, dynamic shared memory for the padded key count), skipping instances without chunks.
constexpr int kSpatialThreads = 512;
static __global__ void __launch_bounds__(kSpatialThreads) batch_spatial(const int2* __restrict__ xy,
                                                                         const int64_t* __restrict__ node_begin,
                                                                         const int64_t* __restrict__ chunk_begin,
                                                                         int32_t first, int32_t* __restrict__ perm,
                                                                         int4* __restrict__ chunk_box) {
  extern __shared__ uint32_t keys[];  // Morton code << 13 | node (n <= kSpatialMaxNodes = 2^13)
  __shared__ int bounds[4];
  const int32_t inst = first + static_cast<int32_t>(blockIdx.x);
  const int64_t c0 = chunk_begin[inst], c1 = chunk_begin[inst + 1];
  if (c1 == c0) return;
  const int64_t n0 = node_begin[inst];
  const int n = static_cast<int>(node_begin[inst + 1] - n0);
  int N = 1;
  while (N < n) N <<= 1;
  if (threadIdx.x == 0) {
    bounds[0] = bounds[2] = INT32_MAX;
    bounds[1] = bounds[3] = INT32_MIN;
  }
  __syncthreads();
  {  // the instance's box: per-thread, per-warp, then one shared atomic per warp
    int lx = INT32_MAX, hx = INT32_MIN, ly = INT32_MAX, hy = INT32_MIN;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      const int2 p = xy[n0 + j];
      lx = min(lx, p.x);
      hx = max(hx, p.x);
      ly = min(ly, p.y);
      hy = max(hy, p.y);
    }
    lx = __reduce_min_sync(kFullMask, lx);
    hx = __reduce_max_sync(kFullMask, hx);
    ly = __reduce_min_sync(kFullMask, ly);
    hy = __reduce_max_sync(kFullMask, hy);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&bounds[0], lx);
      atomicMax(&bounds[1], hx);
      atomicMin(&bounds[2], ly);
      atomicMax(&bounds[3], hy);
    }
  }
  __syncthreads();
  // 9-bit coordinates in the instance's box, bit-interleaved (any order of the nodes gives the same
  // results; a compact one prunes more, and a 512 x 512 grid is finer than 32-node chunks need)
  const float scale_x = 511.0f / static_cast<float>(max(1, bounds[1] - bounds[0]));
  const float scale_y = 511.0f / static_cast<float>(max(1, bounds[3] - bounds[2]));
  auto spread = [](uint32_t v) {  // bit b of v (b < 9) to bit 2b
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    return (v | (v << 1)) & 0x55555555u;
  };
  for (int j = threadIdx.x; j < N; j += blockDim.x) {
    uint32_t key = 0xffffffffu;  // padding sorts last: real keys are below 2^31
    if (j < n) {
      const int2 p = xy[n0 + j];
      const uint32_t qx = min(511u, static_cast<uint32_t>(static_cast<float>(p.x - bounds[0]) * scale_x));
      const uint32_t qy = min(511u, static_cast<uint32_t>(static_cast<float>(p.y - bounds[2]) * scale_y));
      key = ((spread(qx) | (spread(qy) << 1)) << 13) | static_cast<uint32_t>(j);
    }
    keys[j] = key;
  }
  __syncthreads();
  // bitonic sort of the N keys, ascending. Thread t takes pair (j, j + h), j = 2t - (t mod h); for
  // h <= 32 the pairs of a warp's threads stay inside its own 64-key segments, so a stage whose
  // neighbours are also that small needs only a warp barrier
  for (int k = 2; k <= N; k <<= 1) {
    for (int h = k >> 1; h > 0; h >>= 1) {
      for (int t = threadIdx.x; t < (N >> 1); t += blockDim.x) {
        const int j = 2 * t - (t & (h - 1)), o = j + h;
        const uint32_t a = keys[j], b = keys[o];
        if (((j & k) == 0) == (a > b)) {
          keys[j] = b;
          keys[o] = a;
        }
      }
      const int next_h = h > 1 ? h >> 1 : k;
      if (h > 32 || next_h > 32) {
        __syncthreads();
      } else {
        __syncwarp();
      }
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    perm[n0 + j] = static_cast<int32_t>(n0 + static_cast<int64_t>(keys[j] & 0x1fffu));
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int64_t c = c0 + (threadIdx.x >> 5); c < c1; c += blockDim.x >> 5) {  // one warp per chunk
    const int j = static_cast<int>(c - c0) * kSpatialChunk + lane;
    int2 p = make_int2(INT32_MAX, INT32_MAX), q = make_int2(INT32_MIN, INT32_MIN);
    if (j < n) {
      p = xy[n0 + static_cast<int64_t>(keys[j] & 0x1fffu)];
      q = p;
    }
    const int4 box = make_int4(__reduce_min_sync(kFullMask, p.x), __reduce_max_sync(kFullMask, q.x),
                               __reduce_min_sync(kFullMask, p.y), __reduce_max_sync(kFullMask, q.y));
    if (lane == 0) chunk_box[c] = box;
  }
}

// Smallest (2x - mx)^2 + (2y - my)^2 over the chunk's box.
__device__ __forceinline__ unsigned long long chunk_bound(int4 box, int64_t mx, int64_t my) {
  const int64_t dx = max(max(2 * static_cast<int64_t>(box.x) - mx, mx - 2 * static_cast<int64_t>(box.y)), int64_t{0});
  const int64_t dy = max(max(2 * static_cast<int64_t>(box.z) - my, my - 2 * static_cast<int64_t>(box.w)), int64_t{0});
  return static_cast<unsigned long long>(dx * dx) + static_cast<unsigned long long>(dy * dy);
}

// ---- warp top lists ------------------------------------------------------------------

__device__ __forceinline__ uint64_t warp_bitonic_clean(uint64_t key, int lane) {
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) {
    const uint64_t other = __shfl_xor_sync(kFullMask, key, j);
    key = (lane & j) == 0 ? min(key, other) : max(key, other);
  }
  return key;
}

// (score, node) pairs ordered lexicographically.
__device__ __forceinline__ bool pair_less(uint64_t sa, int32_t na, uint64_t sb, int32_t nb) {
  return sa < sb || (sa == sb && na < nb);
}

__device__ __forceinline__ void warp_sort_pairs(uint64_t& score, int32_t& node, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const uint64_t os = __shfl_xor_sync(kFullMask, score, j);
      const int32_t on = __shfl_xor_sync(kFullMask, node, j);
      const bool ascending = (lane & k) == 0;
      const bool lower = (lane & j) == 0;
      const bool other_smaller = pair_less(os, on, score, node);
      if ((lower == ascending) == other_smaller) {
        score = os;
        node = on;
      }
    }
  }
}

// The 32 smallest pairs of two ascending lists, ascending.
__device__ __forceinline__ void warp_merge_pairs(uint64_t& score, int32_t& node, uint64_t bs, int32_t bn, int lane) {
  const uint64_t rs = __shfl_sync(kFullMask, bs, 31 - lane);
  const int32_t rn = __shfl_sync(kFullMask, bn, 31 - lane);
  if (pair_less(rs, rn, score, node)) {
    score = rs;
    node = rn;
  }
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) {
    const uint64_t os = __shfl_xor_sync(kFullMask, score, j);
    const int32_t on = __shfl_xor_sync(kFullMask, node, j);
    const bool other_smaller = pair_less(os, on, score, node);
    if (((lane & j) == 0) == other_smaller) {
      score = os;
      node = on;
    }
  }
}

// ---- work items ----------------------------------------------------------------------

template <int kSpan>
__device__ void batch_select_targets(const BatchArgs& A, int32_t inst, int lane) {
  const JvGraph& g = A.g;
  const int64_t e0 = A.edge_begin[inst], e1 = A.edge_begin[inst + 1];
  const int K = A.targets;
  uint64_t l1 = kEmptyKey, l2 = kEmptyKey;  // ascending ranks 0..31 and 32..63
  for (int64_t base = e0; base < e1; base += 32) {
    const int64_t e = base + lane;
    uint64_t key = kEmptyKey;
    const int4 er = e < e1 ? __ldg(g.edge4 + e) : make_int4(0, 0, 0, 0);
    if (er.w != 0) {
      const int4 nu = __ldg(g.node4 + er.x), nv = __ldg(g.node4 + er.y);
      const int32_t du = nu.w - nu.z, dv = nv.w - nv.z;
      if (du > 2 && dv > 2) {
        // weight descending, then the instance's edge order (= (u, v) order, edges canonical)
        key = (static_cast<uint64_t>(0x7fffffffu - static_cast<uint32_t>(er.z)) << 32) |
              static_cast<uint32_t>(e - e0);
      }
    }
    const uint64_t threshold = K <= 32 ? __shfl_sync(kFullMask, l1, K - 1) : __shfl_sync(kFullMask, l2, K - 33);
    if (!__any_sync(kFullMask, key < threshold)) continue;
    const uint64_t batch = warp_sort_asc(key, lane);
    const uint64_t reversed = __shfl_sync(kFullMask, batch, 31 - lane);
    const uint64_t lo = min(l1, reversed), hi = max(l1, reversed);
    l1 = warp_bitonic_clean(lo, lane);
    if (K > 32) l2 = warp_merge_smallest(l2, warp_bitonic_clean(hi, lane), lane);
  }
  int32_t* out = A.target_ids + static_cast<int64_t>(inst) * K;
  const int32_t id1 = l1 == kEmptyKey ? -1 : static_cast<int32_t>(e0 + (l1 & 0xffffffffu));
  const int32_t id2 = l2 == kEmptyKey ? -1 : static_cast<int32_t>(e0 + (l2 & 0xffffffffu));
  if (lane < K) out[lane] = id1;
  if (lane + 32 < K) out[lane + 32] = id2;
  const int count = __popc(__ballot_sync(kFullMask, lane < K && id1 >= 0)) +
                    __popc(__ballot_sync(kFullMask, lane + 32 < K && id2 >= 0));
  __syncwarp();
  if (lane == 0) {
    A.target_count[inst] = count;
    __threadfence();
    atomicExch(A.ready + inst, 1);
  }
}

// Neighbour pairs (a, b), a < b, in b-major order (b(b-1)/2 + a): the first d(d-1)/2 entries are the
// pairs of a row of d neighbours, for every d <= kReplyTableDegree.
constexpr int kReplyTableDegree = 64;
constexpr int kReplyTablePairs = kReplyTableDegree * (kReplyTableDegree - 1) / 2;

// Number of Hamilton replies at `center` for target (u, v) (AppendHtHamiltonRepliesUnchecked,
// src/cpu/hamilton_tutte.cpp:230-269): pairs first < second of the center's CSR neighbours whose
// edges to the center both survive 2-opt against the target, whose node pair is not the target,
// and with C(u,v) + C(c,first) + C(c,second) <= C(first,second) + C(u,c) + C(v,c). Whole warp; rows
// of up to 32 neighbours keep them one per lane, longer rows re-read both neighbours per pair.
// Pairs come from `reply_pairs` (the table above) for rows of up to kReplyTableDegree neighbours.
template <int kSpan>
__device__ int32_t ht_reply_count(const JvGraph& g, int32_t u, int32_t v, int2 pu, int2 pv, uint32_t cuv,
                                  int32_t center, int2 pc, uint32_t cuc, uint32_t cvc, const uint16_t* reply_pairs,
                                  int lane) {
  const int4 c4 = __ldg(g.node4 + center);
  const int32_t r0 = c4.z, deg = c4.w - c4.z;
  if (deg < 2) return 0;
  const uint64_t center_target = static_cast<uint64_t>(cuc) + cvc;
  // neighbour j: node, C(center, j), 2-opt survival of edge (center, j) against the target
  auto neighbour = [&](int j, int32_t& node, int2& p, uint32_t& cost, bool& survives) {
    const int4 s4 = __ldg(g.slot4 + r0 + j);
    node = s4.x;
    p = make_int2(s4.z, s4.w);
    cost = exact_distance<kSpan>(pc, p, g.dist_type);
    const bool center_low = center < node;  // canonical edge (ou, ov)
    const uint32_t cu_o = exact_distance<kSpan>(pu, p, g.dist_type), cv_o = exact_distance<kSpan>(pv, p, g.dist_type);
    const uint64_t original = static_cast<uint64_t>(cuv) + cost;
    // first = C(u, ov) + C(v, ou), second = C(u, ou) + C(v, ov)
    const uint64_t first = center_low ? static_cast<uint64_t>(cu_o) + cvc : static_cast<uint64_t>(cuc) + cv_o;
    const uint64_t second = center_low ? static_cast<uint64_t>(cuc) + cv_o : static_cast<uint64_t>(cu_o) + cvc;
    survives = first >= original || second >= original;
  };
  int32_t my_node = -1;
  int2 my_p = make_int2(0, 0);
  uint32_t my_cost = 0;
  bool my_survives = false;
  if (deg <= 32 && lane < deg) neighbour(lane, my_node, my_p, my_cost, my_survives);
  const int64_t pairs = static_cast<int64_t>(deg) * (deg - 1) / 2;
  const int tu = min(u, v), tv = max(u, v);
  int32_t count = 0;
  for (int64_t base = 0; base < pairs; base += 32) {
    const int64_t p = base + lane;
    int a = 0, b = 1;
    if (p < pairs && deg <= kReplyTableDegree) {  // the count is a sum: any pair order will do
      const uint16_t ab = reply_pairs[p];
      a = ab & 0xff;
      b = ab >> 8;
    } else if (p < pairs) {  // invert p = a (2 deg - a - 1) / 2 + (b - a - 1)
      const float twod = 2.0f * deg - 1.0f;
      a = static_cast<int>((twod - sqrtf(twod * twod - 8.0f * static_cast<float>(p))) * 0.5f);
      a = max(0, min(a, deg - 2));
      while (a > 0 && static_cast<int64_t>(a) * (2 * deg - a - 1) / 2 > p) --a;
      while (static_cast<int64_t>(a + 1) * (2 * deg - a - 2) / 2 <= p) ++a;
      b = static_cast<int>(p - static_cast<int64_t>(a) * (2 * deg - a - 1) / 2) + a + 1;
    }
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
    if (p < pairs && sa && sb && !(min(na, nb) == tu && max(na, nb) == tv)) {
      const uint64_t original = static_cast<uint64_t>(cuv) + ca + cb;
      const uint64_t replacement = static_cast<uint64_t>(exact_distance<kSpan>(qa, qb, g.dist_type)) + center_target;
      reply = original <= replacement;
    }
    count += __popc(__ballot_sync(kFullMask, reply));
  }
  return count;
}

template <int kSpan>
__device__ void batch_cd_target(const BatchArgs& A, int32_t inst, int32_t t, const uint8_t* pair_i,
                                 const uint8_t* pair_j, unsigned long long* bound, int lane) {
  const JvGraph& g = A.g;
  const int64_t slot = static_cast<int64_t>(inst) * A.targets + t;
  int32_t* nbhd_out = A.nbhd + slot * A.nb;
  uint32_t* flags_out = A.flags + slot * A.flag_words;
  // wait for the instance's targets (bounded)
  if (lane == 0) {
    long long spins = 0;
    while (atomicAdd(A.ready + inst, 0) == 0 && spins < A.wait_limit) {
      __nanosleep(64);
      ++spins;
    }
    if (spins >= A.wait_limit) atomicOr(A.error, kBatchWaitError);
  }
  __syncwarp();
  const int32_t count = *reinterpret_cast<volatile int32_t*>(A.target_count + inst);
  const int32_t target = t < count ? *reinterpret_cast<volatile int32_t*>(A.target_ids + slot) : -1;
  if (target < 0) {
    for (int r = lane; r < A.nb; r += 32) nbhd_out[r] = -1;
    for (int w = lane; w < A.flag_words; w += 32) flags_out[w] = 0;
    return;
  }
  const int2 uv = g.edge_uv[target];
  const int32_t u = uv.x, v = uv.y;
  const int2 pu = __ldg(g.xy + u), pv = __ldg(g.xy + v);
  const int64_t n0 = A.node_begin[inst], n1 = A.node_begin[inst + 1];
  const int64_t mx = static_cast<int64_t>(pu.x) + pv.x, my = static_cast<int64_t>(pu.y) + pv.y;
  const int NB = A.nb;

  // neighbourhood: the NB smallest (doubled-midpoint squared distance, node)
  uint64_t ls = kEmptyKey;
  int32_t ln = INT32_MAX;
  const int64_t c0 = A.chunk_begin[inst], chunks = A.chunk_begin[inst + 1] - c0;
  if (chunks > 0) {  // spatial chunks, best bound first, until the bound exceeds the NB-th best score
    for (int64_t c = lane; c < chunks; c += 32) bound[c] = chunk_bound(__ldg(A.chunk_box + c0 + c), mx, my);
    __syncwarp();
    while (true) {
      unsigned long long best = ~0ull;
      int bc = -1;
      for (int c = lane; c < chunks; c += 32) {
        if (bound[c] < best) {
          best = bound[c];
          bc = c;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long ob = __shfl_xor_sync(kFullMask, best, off);
        const int oc = __shfl_xor_sync(kFullMask, bc, off);
        if (ob < best || (ob == best && static_cast<unsigned>(oc) < static_cast<unsigned>(bc))) {
          best = ob;
          bc = oc;
        }
      }
      const uint64_t ts = __shfl_sync(kFullMask, ls, NB - 1);
      if (bc < 0 || best > ts) break;  // every chunk left scores above the NB-th best (ties included)
      __syncwarp();
      if (lane == 0) bound[bc] = ~0ull;  // visited (real bounds stay below 2^63)
      __syncwarp();
      const int j = bc * kSpatialChunk + lane;
      uint64_t s = kEmptyKey;
      int32_t node = INT32_MAX;
      if (n0 + j < n1) {
        const int32_t x = __ldg(A.perm + n0 + j);
        if (x != u && x != v) {
          const int4 x4 = __ldg(g.node4 + x);
          if (A.max_degree == 0 || x4.w - x4.z <= A.max_degree) {
            const int2 p = make_int2(x4.x, x4.y);
            const int64_t dx = 2 * static_cast<int64_t>(p.x) - mx, dy = 2 * static_cast<int64_t>(p.y) - my;
            s = static_cast<uint64_t>(dx * dx) + static_cast<uint64_t>(dy * dy);
            node = x;
          }
        }
      }
      const int32_t tn = __shfl_sync(kFullMask, ln, NB - 1);
      if (!__any_sync(kFullMask, pair_less(s, node, ts, tn))) continue;
      warp_sort_pairs(s, node, lane);
      warp_merge_pairs(ls, ln, s, node, lane);
    }
  }
  for (int64_t base = chunks > 0 ? n1 : n0; base < n1; base += 32) {
    const int64_t x = base + lane;
    uint64_t s = kEmptyKey;
    int32_t node = INT32_MAX;
    if (x < n1 && x != u && x != v) {
      const int4 x4 = __ldg(g.node4 + x);
      if (A.max_degree == 0 || x4.w - x4.z <= A.max_degree) {
        const int2 p = make_int2(x4.x, x4.y);
        const int64_t dx = 2 * static_cast<int64_t>(p.x) - mx, dy = 2 * static_cast<int64_t>(p.y) - my;
        s = static_cast<uint64_t>(dx * dx) + static_cast<uint64_t>(dy * dy);
        node = static_cast<int32_t>(x);
      }
    }
    const uint64_t ts = __shfl_sync(kFullMask, ls, NB - 1);
    const int32_t tn = __shfl_sync(kFullMask, ln, NB - 1);
    if (!__any_sync(kFullMask, pair_less(s, node, ts, tn))) continue;
    warp_sort_pairs(s, node, lane);
    warp_merge_pairs(ls, ln, s, node, lane);
  }
  const bool have = lane < NB && ln != INT32_MAX;
  if (lane < NB) nbhd_out[lane] = have ? ln : -1;
  const int size = __popc(__ballot_sync(kFullMask, have));
  // C(u, x) and C(v, x) of every neighbourhood node
  uint32_t cu = 0, cv = 0;
  int2 px = make_int2(0, 0);
  if (have) {
    px = __ldg(g.xy + ln);
    cu = exact_distance<kSpan>(pu, px, g.dist_type);
    cv = exact_distance<kSpan>(pv, px, g.dist_type);
  }
  const uint32_t cuv = exact_distance<kSpan>(pu, pv, g.dist_type);
  const int pairs = size * (size - 1) / 2;
  // pair p of the neighbourhood is (i, j), i < j, in the reference's order (i major); the smem
  // table holds that order for the full size NB, a smaller neighbourhood (a small instance)
  // inverts p for its own size
  for (int base = 0; base < A.flag_words * 32; base += 32) {
    const int p = base + lane;
    bool flag = false;
    int i = 0, j = 1;
    if (p < pairs) {
      if (size == NB) {
        i = pair_i[p];
        j = pair_j[p];
      } else {
        i = 0;
        int rest = p;
        while (rest >= size - 1 - i) {
          rest -= size - 1 - i;
          ++i;
        }
        j = i + 1 + rest;
      }
    }
    const int32_t ni = __shfl_sync(kFullMask, ln, i), nj = __shfl_sync(kFullMask, ln, j);
    const uint32_t cui = __shfl_sync(kFullMask, cu, i), cuj = __shfl_sync(kFullMask, cu, j);
    const uint32_t cvi = __shfl_sync(kFullMask, cv, i), cvj = __shfl_sync(kFullMask, cv, j);
    const int2 pi = make_int2(__shfl_sync(kFullMask, px.x, i), __shfl_sync(kFullMask, px.y, i));
    const int2 pj = make_int2(__shfl_sync(kFullMask, px.x, j), __shfl_sync(kFullMask, px.y, j));
    if (p < pairs) {
      const bool i_is_c = ni < nj;
      const int32_t c = i_is_c ? ni : nj, d = i_is_c ? nj : ni;
      const uint32_t cuc = i_is_c ? cui : cuj, cud = i_is_c ? cuj : cui;
      const uint32_t cvc = i_is_c ? cvi : cvj, cvd = i_is_c ? cvj : cvi;
      const int4 c4 = __ldg(g.node4 + c);
      const bool active = row_contains(g.nbr, c4.z, c4.w, d);
      const uint64_t original = static_cast<uint64_t>(cuv) + exact_distance<kSpan>(pi, pj, g.dist_type);
      const uint64_t orient0 = static_cast<uint64_t>(cud) + cvc;
      const uint64_t orient1 = static_cast<uint64_t>(cuc) + cvd;
      const bool incompatible = orient0 < original && orient1 < original;
      flag = A.mode == 0 ? (active && incompatible) : (!active || incompatible);
    }
    const uint32_t word = __ballot_sync(kFullMask, flag);
    if (lane == 0) flags_out[base >> 5] = word;
  }
}

// Eight blocks of eight warps per SM (32 registers, a few spilled): a full SM of warps hides the screen's
// dependent loads and shuffle latencies better than six blocks at 40 registers (18.22 vs 18.70 ms per step)
// or five at 48 (19.7 vs 21.8 ms before the instance-relative keys).
// kLocal: every instance has at most kJvLocalSpan nodes (the JV screen's instance-relative keys).
template <int kSpan, bool kLocal>
static __global__ void __launch_bounds__(kBatchWarps * 32, 8) batch_screen_kernel(BatchArgs A) {
  __shared__ BatchWarpScratch scratch[kBatchWarps];
  __shared__ uint8_t pair_i[kBatchMaxPairs], pair_j[kBatchMaxPairs];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int p = threadIdx.x; p < A.nb * (A.nb - 1) / 2; p += blockDim.x) {
    int i = 0, rest = p;
    while (rest >= A.nb - 1 - i) {
      rest -= A.nb - 1 - i;
      ++i;
    }
    pair_i[p] = static_cast<uint8_t>(i);
    pair_j[p] = static_cast<uint8_t>(i + 1 + rest);
  }
  __syncthreads();
  const int64_t n_select = A.instances;
  const int64_t n_jv = A.jv_items;
  const int64_t n_cd = static_cast<int64_t>(A.instances) * A.targets;
  const int64_t total = n_select + n_jv + n_cd;
  while (true) {
    unsigned long long item = 0;
    if (lane == 0) item = atomicAdd(A.counter, 1ull);
    item = __shfl_sync(kFullMask, item, 0);
    if (static_cast<int64_t>(item) >= total) break;
    const int64_t q = static_cast<int64_t>(item);
    if (q < n_select) {
      batch_select_targets<kSpan>(A, A.first_instance + static_cast<int32_t>(q), lane);
    } else if (q < n_select + n_jv) {
      const int64_t e0 = A.jv_first + (q - n_select) * A.jv_tile;
      const int64_t e1 = min(e0 + A.jv_tile, A.jv_last);
      for (int64_t e = e0; e < e1; ++e) {
        const int32_t w = jv_screen_edge_warp<kSpan, true, kLocal, true>(A.g, e, scratch[warp].jv, lane, A.error);
        if (lane == 0) A.witness[e] = w;
        __syncwarp();
      }
    } else {
      const int64_t s = q - n_select - n_jv;
      batch_cd_target<kSpan>(A, A.first_instance + static_cast<int32_t>(s / A.targets),
                             static_cast<int32_t>(s % A.targets), pair_i, pair_j, scratch[warp].chunk_bound, lane);
    }
    __syncwarp();
  }
}

// FinalizeCdCandidates (src/cpu/hamilton_tutte.cpp:283-327) for one (instance, target) slot, after
// the screen: the Hamilton reply count of every neighbourhood node, the reply product of every
// flagged pair, and the max_cd smallest (product, c, d) as 64-bit keys
// product << 32 | (c - n0) << 16 | (d - n0). A separate launch, so that the screen keeps its
// registers.
template <int kSpan>
__device__ void batch_finalize_target(const BatchArgs& A, int32_t inst, int32_t t, const uint8_t* pair_i,
                                      const uint8_t* pair_j, const uint16_t* reply_pairs, int lane) {
  const JvGraph& g = A.g;
  const int64_t slot = static_cast<int64_t>(inst) * A.targets + t;
  const int32_t count = A.target_count[inst];
  if (t >= count) {
    if (lane == 0) A.cand_count[slot] = 0;
    return;
  }
  const int2 uv = g.edge_uv[A.target_ids[slot]];
  const int32_t u = uv.x, v = uv.y;
  const int2 pu = __ldg(g.xy + u), pv = __ldg(g.xy + v);
  const int64_t n0 = A.node_begin[inst], n1 = A.node_begin[inst + 1];
  const int NB = A.nb;
  const int32_t ln = lane < NB ? A.nbhd[slot * NB + lane] : -1;
  const bool have = ln >= 0;
  const int size = __popc(__ballot_sync(kFullMask, have));
  const int pairs = size * (size - 1) / 2;
  uint32_t cu = 0, cv = 0;
  int2 px = make_int2(0, 0);
  if (have) {
    px = __ldg(g.xy + ln);
    cu = exact_distance<kSpan>(pu, px, g.dist_type);
    cv = exact_distance<kSpan>(pv, px, g.dist_type);
  }
  const uint32_t cuv = exact_distance<kSpan>(pu, pv, g.dist_type);
  const uint32_t my_word = lane < A.flag_words ? A.flags[slot * A.flag_words + lane] : 0u;  // lane w: word w
  const bool any_flag = __any_sync(kFullMask, my_word != 0);
  int32_t* cc_out = A.cand_c + slot * A.max_cd;
  int32_t* cd_out = A.cand_d + slot * A.max_cd;
  int64_t* cp_out = A.cand_product + slot * A.max_cd;
  // FinalizeCdCandidates: the reply count of every neighbourhood node that is an end of a flagged
  // pair (lane k keeps node k's; the products need no other count)
  uint32_t need = 0;
  for (int base = 0; base < A.flag_words * 32 && any_flag; base += 32) {
    const int p = base + lane;
    const uint32_t word = __shfl_sync(kFullMask, my_word, base >> 5);
    if (p < pairs && ((word >> lane) & 1u) != 0) {
      int i = 0, j = 1;
      if (size == NB) {
        i = pair_i[p];
        j = pair_j[p];
      } else {
        int rest = p;
        while (rest >= size - 1 - i) {
          rest -= size - 1 - i;
          ++i;
        }
        j = i + 1 + rest;
      }
      need |= (1u << i) | (1u << j);
    }
  }
  need = __reduce_or_sync(kFullMask, need);
  int32_t my_replies = 0;
  if (any_flag) {
    for (uint32_t rest = need; rest != 0; rest &= rest - 1) {
      const int k = __ffs(rest) - 1;
      const int32_t x = __shfl_sync(kFullMask, ln, k);
      const int2 pxk = make_int2(__shfl_sync(kFullMask, px.x, k), __shfl_sync(kFullMask, px.y, k));
      const uint32_t cuk = __shfl_sync(kFullMask, cu, k), cvk = __shfl_sync(kFullMask, cv, k);
      const int32_t r = ht_reply_count<kSpan>(g, u, v, pu, pv, cuv, x, pxk, cuk, cvk, reply_pairs, lane);
      if (lane == k) my_replies = r;
    }
  }
  // the max_cd smallest (product, c, d) among the flagged pairs, as 64-bit keys
  // product << 32 | (c - n0) << 16 | (d - n0)
  uint64_t top = kEmptyKey;
  for (int base = 0; base < A.flag_words * 32 && any_flag; base += 32) {
    const int p = base + lane;
    const uint32_t word = __shfl_sync(kFullMask, my_word, base >> 5);
    const bool flagged = p < pairs && ((word >> lane) & 1u) != 0;
    int i = 0, j = 1;
    if (flagged) {
      if (size == NB) {
        i = pair_i[p];
        j = pair_j[p];
      } else {
        int rest = p;
        while (rest >= size - 1 - i) {
          rest -= size - 1 - i;
          ++i;
        }
        j = i + 1 + rest;
      }
    }
    const int32_t ni = __shfl_sync(kFullMask, ln, i), nj = __shfl_sync(kFullMask, ln, j);
    const int32_t ri = __shfl_sync(kFullMask, my_replies, i), rj = __shfl_sync(kFullMask, my_replies, j);
    uint64_t key = kEmptyKey;
    if (flagged) {
      const int32_t c = min(ni, nj), d = max(ni, nj);
      const uint64_t product = static_cast<uint64_t>(ri) * static_cast<uint64_t>(rj);
      if (n1 - n0 > 65536 || product >= 0xfffffffeull) atomicOr(A.error, kBatchRangeError);
      key = (min(product, static_cast<uint64_t>(0xfffffffeull)) << 32) |
            (static_cast<uint64_t>(c - n0) << 16) | static_cast<uint64_t>((d - n0) & 0xffff);
    }
    if (!__any_sync(kFullMask, key != kEmptyKey)) continue;
    key = warp_sort_asc(key, lane);
    top = warp_merge_smallest(top, key, lane);
  }
  const int kept = min(A.max_cd, __popc(__ballot_sync(kFullMask, top != kEmptyKey)));
  if (lane < kept) {
    cc_out[lane] = static_cast<int32_t>(n0 + ((top >> 16) & 0xffff));
    cd_out[lane] = static_cast<int32_t>(n0 + (top & 0xffff));
    cp_out[lane] = static_cast<int64_t>(top >> 32);
  }
  if (lane == 0) A.cand_count[slot] = kept;
}

template <int kSpan>
static __global__ void __launch_bounds__(kBatchWarps * 32) batch_finalize_kernel(BatchArgs A) {
  __shared__ uint8_t pair_i[kBatchMaxPairs], pair_j[kBatchMaxPairs];
  __shared__ uint16_t reply_pairs[kReplyTablePairs];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int p = threadIdx.x; p < A.nb * (A.nb - 1) / 2; p += blockDim.x) {
    int i = 0, rest = p;
    while (rest >= A.nb - 1 - i) {
      rest -= A.nb - 1 - i;
      ++i;
    }
    pair_i[p] = static_cast<uint8_t>(i);
    pair_j[p] = static_cast<uint8_t>(i + 1 + rest);
  }
  for (int b = 1 + static_cast<int>(threadIdx.x); b < kReplyTableDegree; b += blockDim.x) {
    for (int a = 0; a < b; ++a) reply_pairs[b * (b - 1) / 2 + a] = static_cast<uint16_t>(a | (b << 8));
  }
  __syncthreads();
  const int64_t slots = static_cast<int64_t>(A.instances) * A.targets;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kBatchWarps;
  for (int64_t q = static_cast<int64_t>(blockIdx.x) * kBatchWarps + warp; q < slots; q += warps) {
    batch_finalize_target<kSpan>(A, A.first_instance + static_cast<int32_t>(q / A.targets),
                                 static_cast<int32_t>(q % A.targets), pair_i, pair_j, reply_pairs, lane);
    __syncwarp();
  }
}

}  // namespace cee
