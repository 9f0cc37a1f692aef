// Exact k-opt leaf cost matrix: costs[row][template] = sum of the k added-edge distances.
//
// Semantics (src/cpu/kopt_search.cpp:962-1042, tests/unit/test_kopt.cpp:48-74): a template
// pairs the 2k ports of a row; its added edges are canon(port p, port mate[p]) for p < mate[p]
// in ascending p. The cell is INT64_MAX when an added edge is a self loop, equals one of the k
// deleted edges canon(port 2e, port 2e+1), repeats an earlier added edge, or the sum overflows
// (impossible here: k <= 5 int32 distances). Otherwise it is the int64 sum.
//
// B200 mapping: a block owns a tile of consecutive rows of one segment (one k). It stages the
// tile's ports in shared memory, evaluates each distinct port pair's exact distance once per
// row (k(2k-1) pairs, at most 45, instead of k distances per cell), then writes the tile's
// cells in row-major order with 16-byte streaming stores: consecutive threads own
// consecutive cell pairs, so every warp store covers 512 contiguous bytes. Rows whose 2k
// port nodes are pairwise distinct cannot produce an invalid cell (a template never pairs
// 2e with 2e+1), so their cells are plain sums; the remaining rows take the checked path.
#pragma once

#include "device_common.cuh"

namespace cee {

constexpr int kKoptThreads = 256;
constexpr int kKoptMaxPorts = 10;
constexpr int kKoptMaxPairs = 45;          // k(2k-1) for k = 5
constexpr int kKoptMaxTemplates = 208;     // proper 5-opt templates
constexpr int kKoptSmemBytes = 48 * 1024;  // dynamic shared memory per block
constexpr int kKoptMaxSegments = 8;

// pair index of ports p < q among 2k ports (row-major upper triangle)
__host__ __device__ __forceinline__ int kopt_pair_index(int p, int q, int ports) {
  return p * ports - (p * (p + 1)) / 2 + (q - p - 1);
}

struct KoptSegment {
  const int32_t* __restrict__ tasks;  // rows x 12 int32 (48-byte rows: 10 ports + int64)
  int64_t* __restrict__ costs;        // rows x T
  int64_t rows;
  const uint8_t* __restrict__ pairs;  // T x k pair indices (device)
  int32_t k;
  int32_t templates;
  int32_t rows_per_tile;
  int32_t tile_begin;                 // first block index of this segment
};

struct KoptLaunch {
  KoptSegment seg[kKoptMaxSegments];
  int32_t segments;
  int32_t dist_type;
  int32_t n;
  const int2* __restrict__ xy;
};

__device__ __forceinline__ uint64_t kopt_canon_key(int32_t a, int32_t b) {
  const uint32_t lo = static_cast<uint32_t>(min(a, b)), hi = static_cast<uint32_t>(max(a, b));
  return (static_cast<uint64_t>(lo) << 32) | hi;
}

// Checked cell for rows with repeated port nodes (the reference's full rule set).
static __device__ __noinline__ int64_t kopt_checked_cell(const int32_t* ports, int k,
                                                  const uint8_t* tpairs, const int32_t* dist,
                                                  const uint8_t* pair_p, const uint8_t* pair_q) {
  uint64_t added[5];
  int64_t total = 0;
  for (int i = 0; i < k; ++i) {
    const int pid = tpairs[i];
    const int32_t a = ports[pair_p[pid]], b = ports[pair_q[pid]];
    if (a == b) return INT64_MAX;
    const uint64_t key = kopt_canon_key(a, b);
    for (int e = 0; e < k; ++e) {
      if (key == kopt_canon_key(ports[2 * e], ports[2 * e + 1])) return INT64_MAX;
    }
    for (int j = 0; j < i; ++j) {
      if (key == added[j]) return INT64_MAX;
    }
    added[i] = key;
    total += dist[pid];
  }
  return total;
}

static __global__ void __launch_bounds__(kKoptThreads) kopt_cost_kernel(KoptLaunch L,
                                                                  int32_t* __restrict__ error) {
  extern __shared__ __align__(16) unsigned char smem[];
  // locate segment
  int si = 0;
  while (si + 1 < L.segments && static_cast<int32_t>(blockIdx.x) >= L.seg[si + 1].tile_begin) ++si;
  const KoptSegment S = L.seg[si];
  const int k = S.k, ports = 2 * k, T = S.templates;
  const int npairs = k * (ports - 1);
  const int64_t row0 = static_cast<int64_t>(blockIdx.x - S.tile_begin) * S.rows_per_tile;
  if (row0 >= S.rows) return;
  const int rows = static_cast<int>(min(static_cast<int64_t>(S.rows_per_tile), S.rows - row0));

  // shared layout: template pairs | pair ports | row ports | row distinct flags | distances
  uint8_t* s_tpairs = smem;                                   // T * k
  uint8_t* s_pp = s_tpairs + kKoptMaxTemplates * 5;           // 45
  uint8_t* s_pq = s_pp + 48;                                  // 45
  int32_t* s_ports = reinterpret_cast<int32_t*>(s_pq + 48);   // rows * ports  (aligned: 1040+96)
  uint8_t* s_distinct = reinterpret_cast<uint8_t*>(s_ports + S.rows_per_tile * ports);
  int32_t* s_dist = reinterpret_cast<int32_t*>(
      s_distinct + ((S.rows_per_tile + 15) & ~15));           // rows * npairs

  for (int i = threadIdx.x; i < T * k; i += blockDim.x) s_tpairs[i] = S.pairs[i];
  if (threadIdx.x < npairs) {
    // invert kopt_pair_index
    int p = 0, idx = threadIdx.x;
    while (idx >= ports - 1 - p) {
      idx -= ports - 1 - p;
      ++p;
    }
    s_pp[threadIdx.x] = static_cast<uint8_t>(p);
    s_pq[threadIdx.x] = static_cast<uint8_t>(p + 1 + idx);
  }
  for (int i = threadIdx.x; i < rows * ports; i += blockDim.x) {
    const int r = i / ports, p = i - r * ports;
    int32_t node = __ldg(S.tasks + (row0 + r) * 12 + p);
    if (static_cast<uint32_t>(node) >= static_cast<uint32_t>(L.n)) {
      atomicOr(error, 1);
      node = 0;
    }
    s_ports[i] = node;
  }
  __syncthreads();

  // per-row distinct-port flag and per-pair exact distances
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const int32_t* pr = s_ports + r * ports;
    bool distinct = true;
    for (int p = 0; p < ports; ++p) {
      for (int q = p + 1; q < ports; ++q) distinct = distinct && pr[p] != pr[q];
    }
    s_distinct[r] = distinct ? 1 : 0;
  }
  for (int i = threadIdx.x; i < rows * npairs; i += blockDim.x) {
    const int r = i / npairs, pid = i - r * npairs;
    const int32_t* pr = s_ports + r * ports;
    const int32_t a = pr[s_pp[pid]], b = pr[s_pq[pid]];
    s_dist[i] = static_cast<int32_t>(exact_distance(__ldg(L.xy + a), __ldg(L.xy + b), L.dist_type));
  }
  __syncthreads();

  // cells: thread owns cell pairs (2j, 2j+1) of the tile, tile start is 16-byte aligned
  const int64_t cells = static_cast<int64_t>(rows) * T;
  int64_t* out = S.costs + row0 * T;
  for (int64_t j = 2 * static_cast<int64_t>(threadIdx.x); j < cells; j += 2 * blockDim.x) {
    int64_t v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t cell = j + h;
      v[h] = 0;
      if (cell < cells) {
        const int r = static_cast<int>(cell / T), t = static_cast<int>(cell - static_cast<int64_t>(r) * T);
        const int32_t* dr = s_dist + r * npairs;
        const uint8_t* tp = s_tpairs + t * k;
        if (s_distinct[r]) {
          int64_t sum = 0;
          for (int i = 0; i < k; ++i) sum += dr[tp[i]];
          v[h] = sum;
        } else {
          v[h] = kopt_checked_cell(s_ports + r * ports, k, tp, dr, s_pp, s_pq);
        }
      }
    }
    if (j + 1 < cells) {
      __stcs(reinterpret_cast<longlong2*>(out + j), make_longlong2(v[0], v[1]));
    } else {
      __stcs(reinterpret_cast<long long*>(out + j), static_cast<long long>(v[0]));
    }
  }
}

// Shared bytes a tile of `rows` rows needs for k.
__host__ __forceinline__ int kopt_tile_smem(int k, int rows) {
  const int ports = 2 * k, npairs = k * (ports - 1);
  return kKoptMaxTemplates * 5 + 96 + rows * ports * 4 + ((rows + 15) & ~15) + rows * npairs * 4;
}

}  // namespace cee
