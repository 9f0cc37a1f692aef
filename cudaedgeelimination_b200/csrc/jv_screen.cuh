// Jonker-Volgenant fast-elimination screen.
//
// Semantics (the reference's CPU oracle, src/cpu/jv_elimination.cpp:45-117, 209-224):
//   for every active edge (a,b) with deg(a) > 2 and deg(b) > 2
//     candidates = the 10 smallest (score, node) over
//                    c in N(a)\{a,b}:                 score = w(a,c) + C(c,b)
//                    c in N(b)\{a,b}, c not in N(a):  score = w(b,c) + C(c,a)
//     witness    = the first candidate c (in that order) such that every
//                  d in N(c)\{a,b} is incompatible:  w(a,b) + w(c,d) > C(a,c) + C(d,b)
//                                                and w(a,b) + w(c,d) > C(a,d) + C(b,c)
// where w are the snapshot's CSR slot weights and C the exact TSPLIB distance. Scores and the
// comparison sums fit 33 bits here (int32 weights and distances) and are kept in 64 bits.
//
// Two mappings of the same screen, chosen per launch:
//   * jv_screen_thread_kernel, one thread per edge: the top-10 list lives in ten 64-bit
//     registers (key = score << 32 | node) and takes new keys through a branch-free
//     compare-exchange chain; N(b) is filtered against N(a) by a merge walk over the two
//     sorted rows; the witness scan is the sequential early-exit loop. Few instructions per
//     edge; lanes of a warp diverge on loop lengths.
//   * jv_screen_warp_kernel, one warp per edge: the lanes score up to 32 candidates at once (when
//     N(a) and N(b) fit one round, a node of N(b) already in N(a) is found by matching lane
//     values, otherwise by a binary search of row a) and keep the top-10 (one round of 32-bit keys:
//     ten warp min-reductions; otherwise a warp-wide bitonic-sorted list merged round by round);
//     the witness search tests the first
//     three neighbours of all ten candidates at once, then flattens the remaining pairs of the
//     still-open candidates over the lanes, accepting a candidate only once all of its pairs
//     are tested and every earlier candidate is closed (so the sequential choice is kept).
#pragma once

#include "device_common.cuh"

namespace cee {

constexpr int kJvMaxCandidates = 10;  // src/cpu/jv_elimination.cpp:28
// Components (instances) of at most kJvLocalSpan nodes with consecutive ids let the warp screen
// key candidates by node id relative to the edge's endpoint (the kLocal screens).
constexpr int kJvLocalSpan = 8192;
constexpr int kJvWarpsPerBlock = 8;
constexpr int kJvThreadBlock = 128;

// Device view of a snapshot (coordinates relative to the bounding-box corner).
struct JvGraph {
  int32_t n;
  int32_t dist_type;
  int64_t m;
  const int2* __restrict__ xy;              // [n]
  const int2* __restrict__ edge_uv;         // [m] (u, v) of the stable edge list
  const int32_t* __restrict__ edge_w;       // [m]
  const uint8_t* __restrict__ active;       // [m]
  const int32_t* __restrict__ row_offsets;  // [n + 1]
  const int32_t* __restrict__ nbr;          // [adjacency], rows ascending
  const int32_t* __restrict__ slot_w;       // [adjacency], weight of the CSR slot's edge
  const int4* __restrict__ slot4;           // [adjacency] {neighbour, slot weight, x, y} (batched screen)
  const int4* __restrict__ node4;           // [n] {x, y, row_offsets[x], row_offsets[x + 1]} (batched screen)
  const int4* __restrict__ edge4;           // [m] {u, v, weight, active} (batched screen)
};

// ------------------------------------------------------------------ thread per edge -----

// Keeps list[0..9] the ten smallest keys seen, ascending: each slot keeps the smaller of
// (slot, carried key) and passes the larger on; the key left after slot 9 is dropped.
__device__ __forceinline__ void top10_insert(uint64_t (&list)[kJvMaxCandidates], uint64_t key) {
#pragma unroll
  for (int i = 0; i < kJvMaxCandidates; ++i) {
    const uint64_t lo = min(list[i], key);
    key = max(list[i], key);
    list[i] = lo;
  }
}

template <int kSpan>
__device__ __forceinline__ int32_t jv_screen_edge_thread(const JvGraph& g, int64_t e,
                                                         int32_t* __restrict__ error) {
  if (g.active[e] == 0) return -1;
  const int2 uv = __ldg(g.edge_uv + e);
  const int32_t a = uv.x, b = uv.y;
  const int32_t ra0 = __ldg(g.row_offsets + a), ra1 = __ldg(g.row_offsets + a + 1);
  const int32_t rb0 = __ldg(g.row_offsets + b), rb1 = __ldg(g.row_offsets + b + 1);
  if (ra1 - ra0 <= 2 || rb1 - rb0 <= 2) return -1;
  const int2 pa = __ldg(g.xy + a), pb = __ldg(g.xy + b);
  const int64_t cab = __ldg(g.edge_w + e);
  const uint32_t n = static_cast<uint32_t>(g.n);

  uint64_t top[kJvMaxCandidates];
#pragma unroll
  for (int i = 0; i < kJvMaxCandidates; ++i) top[i] = kEmptyKey;
  for (int32_t off = ra0; off < ra1; ++off) {
    const int32_t c = __ldg(g.nbr + off);
    if (c == a || c == b) continue;
    if (static_cast<uint32_t>(c) >= n) {
      atomicOr(error, 1);
      continue;
    }
    const uint64_t score = static_cast<uint64_t>(static_cast<uint32_t>(__ldg(g.slot_w + off))) +
                           exact_distance<kSpan>(__ldg(g.xy + c), pb, g.dist_type);
    top10_insert(top, (score << 32) | static_cast<uint32_t>(c));
  }
  // N(b) ascending, skipping nodes already reached through N(a) (merge walk over N(a))
  int32_t walk = ra0;
  int32_t next_a = walk < ra1 ? __ldg(g.nbr + walk) : INT32_MAX;
  for (int32_t off = rb0; off < rb1; ++off) {
    const int32_t c = __ldg(g.nbr + off);
    while (next_a < c) {
      ++walk;
      next_a = walk < ra1 ? __ldg(g.nbr + walk) : INT32_MAX;
    }
    if (c == a || c == b || next_a == c) continue;
    if (static_cast<uint32_t>(c) >= n) {
      atomicOr(error, 1);
      continue;
    }
    const uint64_t score = static_cast<uint64_t>(static_cast<uint32_t>(__ldg(g.slot_w + off))) +
                           exact_distance<kSpan>(__ldg(g.xy + c), pa, g.dist_type);
    top10_insert(top, (score << 32) | static_cast<uint32_t>(c));
  }

#pragma unroll
  for (int i = 0; i < kJvMaxCandidates; ++i) {
    if (top[i] == kEmptyKey) return -1;
    const int32_t c = static_cast<int32_t>(top[i] & 0xffffffffu);
    const int2 pc = __ldg(g.xy + c);
    const int64_t cac = exact_distance<kSpan>(pa, pc, g.dist_type);
    const int64_t cbc = exact_distance<kSpan>(pb, pc, g.dist_type);
    const int32_t rc1 = __ldg(g.row_offsets + c + 1);
    bool witness = true;
    for (int32_t off = __ldg(g.row_offsets + c); off < rc1; ++off) {
      const int32_t d = __ldg(g.nbr + off);
      if (d == a || d == b) continue;
      if (static_cast<uint32_t>(d) >= n) {
        atomicOr(error, 1);
        continue;
      }
      const int2 pd = __ldg(g.xy + d);
      const int64_t left = cab + __ldg(g.slot_w + off);
      if (left <= cac + exact_distance<kSpan>(pd, pb, g.dist_type) ||
          left <= exact_distance<kSpan>(pa, pd, g.dist_type) + cbc) {
        witness = false;  // d is compatible with (a,b)
        break;
      }
    }
    if (witness) return c;
  }
  return -1;
}

template <int kSpan>
static __global__ void __launch_bounds__(kJvThreadBlock)
    jv_screen_thread_kernel(JvGraph g, int64_t first, int64_t last, int32_t* __restrict__ witness,
                            int32_t* __restrict__ error) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = first + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < last; e += stride) {
    witness[e] = jv_screen_edge_thread<kSpan>(g, e, error);
  }
}

// ------------------------------------------------------------------ warp per edge -------

struct JvWarpScratch {
  int32_t c[kJvMaxCandidates];
  int32_t row[kJvMaxCandidates];    // first CSR slot of N(c)
  int32_t begin[kJvMaxCandidates];  // first flattened index of candidate i's remaining pairs
  int32_t end[kJvMaxCandidates];    // one past its last one (row end while the table is built)
  uint32_t cac[kJvMaxCandidates];   // C(a, c)
  uint32_t cbc[kJvMaxCandidates];   // C(b, c)
};

// Screens edge e with the calling (full) warp; returns the witness or -1 on every lane. With
// kSlot4 a CSR slot's neighbour, weight and neighbour coordinates come from one 16-byte load; with
// kLocal the caller guarantees that every neighbour of a or b has an id within kJvLocalSpan - 1 of a
// (the snapshot, or each instance of a batch union, has at most kJvLocalSpan nodes); with kRecords
// an edge's ends, weight and active flag, and a node's coordinates and CSR row, each come from one
// 16-byte load.
template <int kSpan, bool kSlot4 = false, bool kLocal = false, bool kRecords = false>
__device__ __forceinline__ int32_t jv_screen_edge_warp(const JvGraph& g, int64_t e, JvWarpScratch& s,
                                                       int lane, int32_t* __restrict__ error) {
  int32_t a, b;
  int64_t cab;
  if constexpr (kRecords) {
    const int4 er = __ldg(g.edge4 + e);
    if (er.w == 0) return -1;
    a = er.x;
    b = er.y;
    cab = er.z;
  } else {
    if (__ldg(g.active + e) == 0) return -1;
    const int2 uv = __ldg(g.edge_uv + e);
    a = uv.x;
    b = uv.y;
  }
  int32_t ra0, ra1, rb0, rb1;
  int2 pa, pb;
  if constexpr (kRecords) {
    const int4 na = __ldg(g.node4 + a), nb = __ldg(g.node4 + b);
    pa = make_int2(na.x, na.y);
    pb = make_int2(nb.x, nb.y);
    ra0 = na.z;
    ra1 = na.w;
    rb0 = nb.z;
    rb1 = nb.w;
  } else {
    ra0 = __ldg(g.row_offsets + a);
    ra1 = __ldg(g.row_offsets + a + 1);
    rb0 = __ldg(g.row_offsets + b);
    rb1 = __ldg(g.row_offsets + b + 1);
  }
  const int32_t da = ra1 - ra0, db = rb1 - rb0;
  if (da <= 2 || db <= 2) return -1;
  if constexpr (!kRecords) {
    pa = __ldg(g.xy + a);
    pb = __ldg(g.xy + b);
    cab = __ldg(g.edge_w + e);
  }
  // neighbours must lie in [lo, lo + range): the snapshot's ids, or with kLocal also within
  // kJvLocalSpan - 1 of a (the one test bounds both the gathers and the instance-relative keys)
  const int32_t lo = kLocal ? max(a - (kJvLocalSpan - 1), 0) : 0;
  const uint32_t range = static_cast<uint32_t>(kLocal ? min(g.n, a + kJvLocalSpan) - lo : g.n);

  uint64_t top = kEmptyKey;
  const int total = da + db;
  for (int base = 0; base < total; base += 32) {
    const int i = base + lane;
    uint64_t key = kEmptyKey;
    const bool second = i >= da;
    const int32_t slot = second ? rb0 + (i - da) : ra0 + i;
    int32_t c = -1, sw = 0;
    int2 pc = make_int2(0, 0);
    bool ok = false;
    if (i < total) {
      if constexpr (kSlot4) {
        const int4 si = __ldg(g.slot4 + slot);
        c = si.x;
        sw = si.y;
        pc = make_int2(si.z, si.w);
      } else {
        c = __ldg(g.nbr + slot);
      }
      ok = c != a && c != b;
      if (ok && static_cast<uint32_t>(c - lo) >= range) {
        atomicOr(error, 1);
        ok = false;
      }
    }
    if (total <= 32) {
      // one round: N(a) sits on lanes [0, da), so a node of N(b) already scored through N(a)
      // is found by matching lane values (other lanes hold distinct negative placeholders)
      const unsigned same = __match_any_sync(kFullMask, ok ? c : -1 - lane);
      if (ok && second) ok = (same & ((1u << da) - 1u)) == 0;
    } else if (ok && second) {
      ok = !row_contains(g.nbr, ra0, ra1, c);
    }
    uint64_t score = 0;
    if (ok) {
      if constexpr (!kSlot4) {
        sw = __ldg(g.slot_w + slot);
        pc = __ldg(g.xy + c);
      }
      score = static_cast<uint64_t>(static_cast<uint32_t>(sw)) + exact_distance<kSpan>(pc, second ? pa : pb, g.dist_type);
      key = (score << 32) | static_cast<uint32_t>(c);
    }
    if (kLocal && total <= 32) {
      // kLocal: every node of the edge's component has an id within kJvLocalSpan - 1 of a, so
      // (score, c - a + kJvLocalSpan) in 32 bits keeps the order of the 64-bit keys whenever every
      // score fits 18 bits -- one vote instead of the three warp reductions below (a neighbour
      // outside that range, a CSR row that leaves its instance, failed the bounds test above)
      if (__all_sync(kFullMask, !ok || score < (1u << 18) - 1u)) {
        uint32_t k32 = ok ? (static_cast<uint32_t>(score) << 14) | static_cast<uint32_t>(c - a + kJvLocalSpan)
                          : 0xffffffffu;
        k32 = warp_smallest_asc32<kJvMaxCandidates>(k32, lane);  // keys are distinct: distinct nodes
        top = k32 == 0xffffffffu ? kEmptyKey
                                 : (static_cast<uint64_t>(k32 >> 14) << 32) |
                                       static_cast<uint32_t>(static_cast<int32_t>(k32 & 0x3fffu) - kJvLocalSpan + a);
        break;
      }
    } else if (total <= 32) {
      // compact keys: (score, node - min node) in 32 bits sort in half the shuffles; used when
      // every score and the node spread fit (the order is the same as the 64-bit keys')
      const uint32_t cmin = __reduce_min_sync(kFullMask, ok ? static_cast<uint32_t>(c) : 0xffffffffu);
      const uint32_t cmax = __reduce_max_sync(kFullMask, ok ? static_cast<uint32_t>(c) : 0u);
      const uint32_t smax = __reduce_max_sync(kFullMask, ok ? static_cast<uint32_t>(score) : 0u);
      const bool narrow_scores = __all_sync(kFullMask, (score >> 32) == 0);
      const uint32_t span = cmax >= cmin ? cmax - cmin : 0u;
      const int node_bits = span == 0 ? 1 : 32 - __clz(span);
      if (narrow_scores && node_bits < 31 && smax < (1u << (32 - node_bits)) - 1u) {
        uint32_t k32 = ok ? (static_cast<uint32_t>(score) << node_bits) | (static_cast<uint32_t>(c) - cmin) : 0xffffffffu;
        k32 = warp_smallest_asc32<kJvMaxCandidates>(k32, lane);
        top = k32 == 0xffffffffu ? kEmptyKey
                                 : (static_cast<uint64_t>(k32 >> node_bits) << 32) |
                                       (cmin + (k32 & ((1u << node_bits) - 1u)));
        break;  // total <= 32: this was the only round
      }
    }
    key = warp_sort_asc(key, lane);
    top = base == 0 ? key : warp_merge_smallest(top, key, lane);
  }
  const int nc = __popc(__ballot_sync(kFullMask, lane < kJvMaxCandidates && top != kEmptyKey));
  if (nc == 0) return -1;

  {  // candidate table: C(a,c) on lanes 0..9, C(b,c) on lanes 10..19
    const int ci = lane < kJvMaxCandidates ? lane : lane - kJvMaxCandidates;
    const uint64_t key = __shfl_sync(kFullMask, top, ci);
    if (lane < 2 * kJvMaxCandidates && ci < nc) {
      const int32_t c = static_cast<int32_t>(key & 0xffffffffu);
      int2 pc;
      int32_t row0 = 0, row1 = 0;
      if constexpr (kRecords) {
        const int4 nc4 = __ldg(g.node4 + c);
        pc = make_int2(nc4.x, nc4.y);
        row0 = nc4.z;
        row1 = nc4.w;
      } else {
        pc = __ldg(g.xy + c);
        if (lane < kJvMaxCandidates) {
          row0 = __ldg(g.row_offsets + c);
          row1 = __ldg(g.row_offsets + c + 1);
        }
      }
      const uint32_t dist = exact_distance<kSpan>(lane < kJvMaxCandidates ? pa : pb, pc, g.dist_type);
      if (lane < kJvMaxCandidates) {
        s.c[ci] = c;
        s.row[ci] = row0;
        s.end[ci] = row1;
        s.cac[ci] = dist;
      } else {
        s.cbc[ci] = dist;
      }
    }
  }
  __syncwarp();

  auto compatible_pair = [&](int ci, int32_t slot) -> bool {
    int32_t d, dw;
    int2 pd;
    if constexpr (kSlot4) {
      const int4 si = __ldg(g.slot4 + slot);
      d = si.x;
      dw = si.y;
      pd = make_int2(si.z, si.w);
    } else {
      d = __ldg(g.nbr + slot);
    }
    if (d == a || d == b) return false;
    if (static_cast<uint32_t>(d) >= static_cast<uint32_t>(g.n)) {
      atomicOr(error, 1);
      return false;
    }
    if constexpr (!kSlot4) {
      pd = __ldg(g.xy + d);
      dw = __ldg(g.slot_w + slot);
    }
    const int64_t left = cab + dw;
    return left <= static_cast<int64_t>(s.cac[ci]) + exact_distance<kSpan>(pd, pb, g.dist_type) ||
           left <= static_cast<int64_t>(exact_distance<kSpan>(pa, pd, g.dist_type)) + s.cbc[ci];
  };

  constexpr int kHead = 3;
  const int deg = lane < nc ? s.end[lane] - s.row[lane] : 0;
  uint32_t compatible = 0;
  {
    const int hi = lane / kHead, hj = lane - hi * kHead;
    bool hit = false;
    if (hi < nc) {
      const int32_t row = s.row[hi];
      if (hj < s.end[hi] - row) hit = compatible_pair(hi, row + hj);
    }
    compatible = __reduce_or_sync(kFullMask, hit ? 1u << hi : 0u);
  }
  const uint32_t all = (1u << nc) - 1u;
  uint32_t open = all & ~compatible;
  if (open == 0) return -1;

  const int rest = ((open >> lane) & 1u) != 0 ? max(deg - kHead, 0) : 0;
  const int incl = warp_inclusive_sum(rest, lane);
  __syncwarp();
  if (lane < nc) {
    s.begin[lane] = incl - rest;
    s.end[lane] = incl;
  }
  const int pairs = __shfl_sync(kFullMask, incl, nc - 1);
  __syncwarp();
  int first_open = __ffs(open) - 1;
  if (s.end[first_open] == s.begin[first_open]) return s.c[first_open];
  int base = s.begin[first_open];
  while (true) {
    const int p = base + lane;
    uint32_t bit = 0;
    if (p < pairs) {
      int ci = 0;  // last candidate whose run starts at or before p (begin[] is non-decreasing)
#pragma unroll
      for (int step = 8; step > 0; step >>= 1) {
        if (ci + step < nc && s.begin[ci + step] <= p) ci += step;
      }
      if (((compatible >> ci) & 1u) == 0 && compatible_pair(ci, s.row[ci] + kHead + (p - s.begin[ci]))) {
        bit = 1u << ci;
      }
    }
    compatible |= __reduce_or_sync(kFullMask, bit);
    open = all & ~compatible;
    if (open == 0) return -1;
    first_open = __ffs(open) - 1;
    const int chunk_end = base + 32;
    if (s.end[first_open] <= chunk_end) return s.c[first_open];
    base = max(chunk_end, s.begin[first_open]);
  }
}

template <int kSpan>
static __global__ void __launch_bounds__(kJvWarpsPerBlock * 32)
    jv_screen_warp_kernel(JvGraph g, int64_t first, int64_t last, int32_t* __restrict__ witness,
                          int32_t* __restrict__ error) {
  __shared__ JvWarpScratch scratch[kJvWarpsPerBlock];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kJvWarpsPerBlock;
  for (int64_t e = first + static_cast<int64_t>(blockIdx.x) * kJvWarpsPerBlock + warp; e < last; e += warps) {
    const int32_t w = jv_screen_edge_warp<kSpan>(g, e, scratch[warp], lane, error);
    if (lane == 0) witness[e] = w;
    __syncwarp();
  }
}

}  // namespace cee
