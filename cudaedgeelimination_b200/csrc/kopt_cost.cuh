// Exact k-opt leaf cost matrix: costs[row][template] = sum of the k added-edge distances.
//
// Semantics (src/cpu/kopt_search.cpp:962-1042, tests/unit/test_kopt.cpp:48-74): a template
// pairs the 2k ports of a row; its added edges are canon(port p, port mate[p]) for p < mate[p]
// in ascending p. The cell is INT64_MAX when an added edge is a self loop, equals one of the k
// deleted edges canon(port 2e, port 2e+1), repeats an earlier added edge, or the sum overflows
// (impossible here: k <= 5 int32 distances). Otherwise it is the int64 sum.
//
// B200 mapping: a block owns a tile of consecutive rows of one segment (one k).
//   1. the tile's ports are staged in shared memory;
//   2. every port pair p < q of every row gets its exact distance once (k(2k-1) pairs, at
//      most 45, instead of k distances per cell), plus, for rows whose 2k port nodes are not
//      pairwise distinct, a code byte: 0xff when the pair is a self loop or re-adds a deleted
//      edge, else the index of the first pair with the same node pair (to detect duplicates);
//   3. thread j owns template t = j mod T, keeps its k pair indices in registers and walks
//      rows j / T, j / T + 256 / T, ...; the threads of one step write 256/T consecutive rows,
//      i.e. one contiguous run of row-major cells, with streaming stores.
// Rows with pairwise-distinct ports cannot produce an invalid cell (a template never pairs 2e
// with 2e+1), so their cells are plain sums.
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

struct KoptSmem {
  int32_t* ports;   // rows * ports
  int32_t* dist;    // rows * npairs
  uint8_t* code;    // rows * npairs
  uint8_t* ok;      // rows
  uint8_t* pp;      // npairs: first port of pair
  uint8_t* pq;      // npairs: second port of pair
};

__host__ __device__ __forceinline__ int kopt_tile_smem(int k, int rows) {
  const int ports = 2 * k, npairs = k * (ports - 1);
  const int a = rows * ports * 4, b = rows * npairs * 4, c = (rows * npairs + 15) & ~15;
  return a + b + c + ((rows + 15) & ~15) + 96;
}

__device__ __forceinline__ KoptSmem kopt_carve(unsigned char* base, int k, int rows) {
  const int ports = 2 * k, npairs = k * (ports - 1);
  KoptSmem s;
  s.ports = reinterpret_cast<int32_t*>(base);
  s.dist = s.ports + rows * ports;
  s.code = reinterpret_cast<uint8_t*>(s.dist + rows * npairs);
  s.ok = s.code + ((rows * npairs + 15) & ~15);
  s.pp = s.ok + ((rows + 15) & ~15);
  s.pq = s.pp + 48;
  return s;
}

static __global__ void __launch_bounds__(kKoptThreads) kopt_cost_kernel(KoptLaunch L,
                                                                        int32_t* __restrict__ error) {
  extern __shared__ __align__(16) unsigned char smem[];
  int si = 0;
  while (si + 1 < L.segments && static_cast<int32_t>(blockIdx.x) >= L.seg[si + 1].tile_begin) ++si;
  const KoptSegment& S = L.seg[si];
  const int k = S.k, ports = 2 * k, T = S.templates;
  const int npairs = k * (ports - 1);
  const int64_t row0 = static_cast<int64_t>(blockIdx.x - S.tile_begin) * S.rows_per_tile;
  if (row0 >= S.rows) return;
  const int rows = static_cast<int>(min(static_cast<int64_t>(S.rows_per_tile), S.rows - row0));
  const KoptSmem sm = kopt_carve(smem, k, S.rows_per_tile);
  const int tid = threadIdx.x;

  if (tid < npairs) {  // invert the pair numbering p < q
    int p = 0, idx = tid;
    while (idx >= ports - 1 - p) {
      idx -= ports - 1 - p;
      ++p;
    }
    sm.pp[tid] = static_cast<uint8_t>(p);
    sm.pq[tid] = static_cast<uint8_t>(p + 1 + idx);
  }
  for (int i = tid; i < rows * ports; i += kKoptThreads) {
    const int r = i / ports, p = i - r * ports;
    int32_t node = __ldg(S.tasks + (row0 + r) * 12 + p);
    if (static_cast<uint32_t>(node) >= static_cast<uint32_t>(L.n)) {
      atomicOr(error, 1);
      node = 0;
    }
    sm.ports[i] = node;
  }
  __syncthreads();
  for (int r = tid; r < rows; r += kKoptThreads) {
    const int32_t* pr = sm.ports + r * ports;
    bool distinct = true;
    for (int p = 0; p < ports; ++p) {
      for (int q = p + 1; q < ports; ++q) distinct = distinct && pr[p] != pr[q];
    }
    sm.ok[r] = distinct ? 1 : 0;
  }
  __syncthreads();
  for (int i = tid; i < rows * npairs; i += kKoptThreads) {
    const int r = i / npairs, pid = i - r * npairs;
    const int32_t* pr = sm.ports + r * ports;
    const int32_t a = pr[sm.pp[pid]], b = pr[sm.pq[pid]];
    sm.dist[i] = static_cast<int32_t>(exact_distance(__ldg(L.xy + a), __ldg(L.xy + b), L.dist_type));
    if (!sm.ok[r]) {
      uint8_t code = static_cast<uint8_t>(pid);
      const uint64_t key = kopt_canon_key(a, b);
      if (a == b) code = 0xff;
      for (int e = 0; e < k && code != 0xff; ++e) {
        if (key == kopt_canon_key(pr[2 * e], pr[2 * e + 1])) code = 0xff;
      }
      for (int o = 0; o < pid && code == pid; ++o) {
        if (key == kopt_canon_key(pr[sm.pp[o]], pr[sm.pq[o]])) code = static_cast<uint8_t>(o);
      }
      sm.code[i] = code;
    }
  }
  __syncthreads();

  const int per_step = kKoptThreads / T;  // rows written per step
  const int rr = tid / T, t = tid - rr * T;
  if (rr >= per_step) return;
  int pid[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) pid[i] = i < k ? __ldg(S.pairs + t * k + i) : 0;
  int64_t* out = S.costs + row0 * T;
  for (int r = rr; r < rows; r += per_step) {
    const int32_t* dr = sm.dist + r * npairs;
    int64_t v = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      if (i < k) v += dr[pid[i]];
    }
    if (!sm.ok[r]) {
      const uint8_t* cr = sm.code + r * npairs;
      uint64_t used = 0;
      bool bad = false;
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        if (i < k) {
          const uint8_t c = cr[pid[i]];
          bad = bad || c == 0xff || ((used >> c) & 1u);
          used |= uint64_t{1} << (c & 63);
        }
      }
      if (bad) v = INT64_MAX;
    }
    __stcs(reinterpret_cast<long long*>(out + static_cast<int64_t>(r) * T + t), static_cast<long long>(v));
  }
}

}  // namespace cee
