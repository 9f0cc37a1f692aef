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
//   2. every port is mapped to the first port of the row holding the same node (its class);
//      every port pair p < q gets its exact distance once (k(2k-1) pairs, at most 45, instead
//      of k distances per cell); rows that repeat a node get a validity summary (KoptRowInfo);
//   3. thread j owns template t = j mod T, keeps its k pair indices and its 64-bit pair mask in
//      registers and walks rows j / T, j / T + 256 / T, ...; the threads of one step write
//      256/T consecutive rows, i.e. one contiguous run of row-major cells, with streaming stores.
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

// Per-row validity summary. A cell is invalid iff its template uses a pair marked in `bad`
// (self loop or a re-added deleted edge) or uses two pairs adding the same node pair. Each
// pair's code is the pair index of its node pair in port-class space; the port pairs sharing a
// code form a duplicate set, and a template contains two of them iff the popcount of its pair
// mask restricted to the set is >= 2. Only codes whose two classes both hold two or more ports
// need a set (otherwise all members share the single port and no matching holds two), so a row
// of 10 ports has at most C(5,2) = 10 sets.
constexpr int kKoptMaxDupSets = 10;

struct KoptRowInfo {
  uint32_t bad_lo, bad_hi;  // 64-bit mask over pair indices
  uint32_t dup_count;
  uint32_t repeats;          // number of repeated nodes (0 = all ports distinct)
  uint64_t dup[kKoptMaxDupSets];
};

struct KoptSmem {
  int32_t* ports;     // rows * ports: node ids
  int32_t* dist;      // rows * npairs
  uint8_t* cls;       // rows * ports: first port holding the same node
  uint8_t* code;      // rows * npairs: class-pair index, 0xff when bad (rows with repeats only)
  KoptRowInfo* info;  // rows
  uint8_t* pp;        // npairs: first port of pair
  uint8_t* pq;        // npairs: second port of pair
};

__host__ __device__ __forceinline__ int kopt_tile_smem(int k, int rows) {
  const int ports = 2 * k, npairs = k * (ports - 1);
  return rows * ports * 4 + rows * npairs * 4 + ((rows * ports + 15) & ~15) + ((rows * npairs + 15) & ~15) +
         rows * static_cast<int>(sizeof(KoptRowInfo)) + 96;
}

__device__ __forceinline__ KoptSmem kopt_carve(unsigned char* base, int k, int rows) {
  const int ports = 2 * k, npairs = k * (ports - 1);
  KoptSmem s;
  s.ports = reinterpret_cast<int32_t*>(base);
  s.dist = s.ports + rows * ports;
  s.cls = reinterpret_cast<uint8_t*>(s.dist + rows * npairs);
  s.code = s.cls + ((rows * ports + 15) & ~15);
  s.info = reinterpret_cast<KoptRowInfo*>(s.code + ((rows * npairs + 15) & ~15));
  s.pp = reinterpret_cast<uint8_t*>(s.info + rows);
  s.pq = s.pp + 48;
  return s;
}

// q = i / d for i * d < 2^32, with magic = ceil(2^32 / d).
__device__ __forceinline__ int kopt_div(int i, uint32_t magic) {
  return static_cast<int>(__umulhi(static_cast<uint32_t>(i), magic));
}

template <bool kWide>
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
  const uint32_t magic_ports = static_cast<uint32_t>((0x100000000ull + ports - 1) / ports);
  const uint32_t magic_pairs = static_cast<uint32_t>((0x100000000ull + npairs - 1) / npairs);

  if (tid < npairs) {  // invert the pair numbering p < q
    int p = 0, idx = tid;
    while (idx >= ports - 1 - p) {
      idx -= ports - 1 - p;
      ++p;
    }
    sm.pp[tid] = static_cast<uint8_t>(p);
    sm.pq[tid] = static_cast<uint8_t>(p + 1 + idx);
  }
  for (int r = tid; r < rows; r += kKoptThreads) {
    sm.info[r].bad_lo = sm.info[r].bad_hi = 0;
    sm.info[r].dup_count = sm.info[r].repeats = 0;
  }
  for (int i = tid; i < rows * ports; i += kKoptThreads) {
    const int r = kopt_div(i, magic_ports), p = i - r * ports;
    int32_t node = __ldg(S.tasks + (row0 + r) * 12 + p);
    if (static_cast<uint32_t>(node) >= static_cast<uint32_t>(L.n)) {
      atomicOr(error, 1);
      node = 0;
    }
    sm.ports[i] = node;
  }
  __syncthreads();
  // port classes: the first port of the row holding the same node
  for (int i = tid; i < rows * ports; i += kKoptThreads) {
    const int r = kopt_div(i, magic_ports), p = i - r * ports;
    const int32_t* pr = sm.ports + r * ports;
    int c = p;
    for (int q = p - 1; q >= 0; --q) c = pr[q] == pr[p] ? q : c;
    sm.cls[i] = static_cast<uint8_t>(c);
    if (c != p) atomicAdd(&sm.info[r].repeats, 1u);
  }
  __syncthreads();
  // exact distance of every port pair; pairs that are self loops or re-add a deleted edge
  // (compared in port-class space) are marked in the row's bad mask
  for (int i = tid; i < rows * npairs; i += kKoptThreads) {
    const int r = kopt_div(i, magic_pairs), pid = i - r * npairs;
    const int p = sm.pp[pid], q = sm.pq[pid];
    const int32_t* pr = sm.ports + r * ports;
    sm.dist[i] = static_cast<int32_t>(exact_distance<kWide>(__ldg(L.xy + pr[p]), __ldg(L.xy + pr[q]), L.dist_type));
    if (sm.info[r].repeats != 0) {
      const uint8_t* cr = sm.cls + r * ports;
      const int cp = cr[p], cq = cr[q];
      bool bad = cp == cq;
      const int code = kopt_pair_index(min(cp, cq), max(cp, cq), ports);
      for (int e = 0; e < k && !bad; ++e) {
        const int d0 = cr[2 * e], d1 = cr[2 * e + 1];
        bad = d0 != d1 && code == kopt_pair_index(min(d0, d1), max(d0, d1), ports);
      }
      if (bad) atomicOr(pid < 32 ? &sm.info[r].bad_lo : &sm.info[r].bad_hi, 1u << (pid & 31));
      sm.code[i] = bad ? 0xff : static_cast<uint8_t>(code);
    }
  }
  __syncthreads();
  // duplicate sets: the pairs sharing a class-pair code (the representative pair, whose code
  // is its own index, plus every pair mapped onto it)
  for (int r = tid; r < rows; r += kKoptThreads) {
    if (sm.info[r].repeats == 0) continue;
    const uint8_t* cr = sm.code + r * npairs;
    const uint8_t* cl = sm.cls + r * ports;
    uint32_t multi = 0;  // classes holding two or more ports
    for (int p = 0; p < ports; ++p) {
      if (cl[p] != p) multi |= 1u << cl[p];
    }
    uint32_t sets = 0;
    for (int a = 0; a < npairs; ++a) {
      const int c = cr[a];
      if (c == 0xff || c == a) continue;
      // pairs through a single-port class all share that port: never two in one template
      if (((multi >> cl[sm.pp[a]]) & (multi >> cl[sm.pq[a]]) & 1u) == 0) continue;
      const uint64_t rep = uint64_t{1} << c;
      uint32_t j = 0;
      while (j < sets && (sm.info[r].dup[j] & rep) == 0) ++j;
      if (j == sets) {
        if (sets == kKoptMaxDupSets) {  // cannot happen (see kKoptMaxDupSets); fail loudly
          atomicOr(error, 4);
          break;
        }
        sm.info[r].dup[sets++] = rep;
      }
      sm.info[r].dup[j] |= uint64_t{1} << a;
    }
    sm.info[r].dup_count = sets;
  }
  __syncthreads();

  // cells: thread owns template t for rows rr, rr + per_step, ...
  const int per_step = kKoptThreads / T;
  const int rr = tid / T, t = tid - rr * T;
  if (rr >= per_step) return;
  int pid[5];
  uint64_t tmask = 0;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    pid[i] = i < k ? __ldg(S.pairs + t * k + i) : 0;
    if (i < k) tmask |= uint64_t{1} << pid[i];
  }
  long long* out = reinterpret_cast<long long*>(S.costs + row0 * T) + static_cast<int64_t>(rr) * T + t;
  const int64_t out_step = static_cast<int64_t>(per_step) * T;
  for (int r = rr; r < rows; r += per_step, out += out_step) {
    const int32_t* dr = sm.dist + r * npairs;
    int64_t v = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      if (i < k) v += dr[pid[i]];
    }
    const KoptRowInfo& info = sm.info[r];
    if (info.repeats != 0) {
      const uint64_t bad = (static_cast<uint64_t>(info.bad_hi) << 32) | info.bad_lo;
      bool invalid = (bad & tmask) != 0;
      for (uint32_t j = 0; j < info.dup_count; ++j) invalid = invalid || __popcll(info.dup[j] & tmask) >= 2;
      if (invalid) v = INT64_MAX;
    }
    __stcs(out, static_cast<long long>(v));
  }
}

}  // namespace cee
