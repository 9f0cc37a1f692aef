// Exact k-opt leaf cost matrix: costs[row][template] = sum of the k added-edge distances.
//
// Semantics (src/cpu/kopt_search.cpp:962-1042, tests/unit/test_kopt.cpp:48-74): a template
// pairs the 2k ports of a row; its added edges are canon(port p, port mate[p]) for p < mate[p]
// in ascending p. The cell is INT64_MAX when an added edge is a self loop, equals one of the k
// deleted edges canon(port 2e, port 2e+1), repeats an earlier added edge, or the sum overflows
// (impossible here: k <= 5 int32 distances). Otherwise it is the int64 sum.
//
// Validity in port-class space: every port is mapped to its class, the first port of the row
// holding the same node, and every port pair p < q to the pair index of its class pair
// (min, max), its code. Two added edges are the same node pair iff their codes are equal; an
// added edge is a self loop iff its two classes are equal and re-adds a deleted edge iff its
// code is a deleted edge's code ("bad" pairs). Two pairs of one template can share a code only
// if both classes of that code hold two or more ports (pairs through a one-port class share that
// port, and a matching uses each port once): with 2k <= 10 ports there are at most C(5,2) = 10
// such "multi" codes. Rows whose 2k ports are distinct nodes have no bad pair and no shared code
// (a proper template never pairs 2e with 2e+1; a caller template that does is marked in its
// pair table and yields invalid cells).
//
// Small and narrow span classes (span < 2^26, each distance < 2^26.5): a pair's entry is one 64-bit word,
// low half = its distance, or 2^29 when the pair is bad; high half = 1 << 3f when its code is
// the f-th multi code of the row, else 0. A cell adds its k entries: the low half is the cost
// (< 5 * 2^26.5 < 2^29 unless a bad pair is present; < 2^32 always), each 3-bit field of the
// high half counts the template's pairs on one multi code (<= 5), and the cell is invalid iff
// low >= 2^29 or some field is >= 2. The wide span class keeps int32 distances and a one-hot 64-bit
// mask per pair (bit = code, bit 63 = bad): invalid iff the OR of the k masks has bit 63 set or
// fewer than k bits.
//
// B200 mapping: a block owns a tile of consecutive rows of one segment (one k; the tile
// routine is compiled per k so the per-row work is fully unrolled).
//   A. the tile's ports are staged in shared memory (one thread per port);
//   B. one thread per row finds the port classes, whether the row repeats a node, the rank of
//      each port's class among the multi classes and the row's deleted-code set;
//   C. one thread per (row, port pair) computes the pair's exact distance (k(2k-1) pairs, at
//      most 45, instead of k distances per cell) and its entry (narrow) or mask (wide);
//   D. thread j owns template t = j mod T with its k pair indices in registers and walks rows
//      j / T, j / T + B / T, ... (B = 224 threads: 56 rows of k = 3, 8 rows of k = 4, one
//      row of k = 5 per step); the threads of a step write one contiguous run of row-major
//      cells with streaming stores. Small blocks (7 warps, nine per SM) keep the stages'
//      barriers and load latencies of one tile overlapped with other tiles' work.
// Gap-pattern rows. Rows built from a tour (the reference's leaf rows, BuildKOptCostTask,
// src/cpu/kopt_search.cpp:561-584) repeat a node only where two deleted edges are adjacent in the
// tour: port 2e+1 and port (2e+2) mod 2k hold the same node ("gap" e closed), and all other ports
// are distinct. Such a row's class structure is fixed by its gap pattern g (bit e = gap e closed,
// < 2^k <= 32 patterns), so whether a template is invalid on it depends on (template, g) only: the
// host precomputes per template a 32-bit mask over the patterns (KoptSegment::patterns). Stage B
// recognises these rows (the equal port pairs are exactly the closed gaps), stage C then stores only
// the pair distances, and stage D sums k int32 distances and tests one bit; every other row keeps
// the general class-code path above.
// Fused leaf consume (mask_words > 0): stage D also marks, per row, the templates whose cost is
// below the row's deleted cost — the templates the reference's leaf consumer tries, in order — in a
// shared bit mask; the tile then writes the masks and each row's first improving template, and the
// cost matrix itself becomes optional (write_costs).
#pragma once

#include "device_common.cuh"

namespace cee {

constexpr int kKoptThreads = 224;          // 7 warps: 56 x 4 cells per step, 8 x 25 + 24, 208 + 16
constexpr int kKoptMaxPorts = 10;
constexpr int kKoptMaxPairs = 45;          // k(2k-1) for k = 5
constexpr int kKoptMaxTemplates = 208;     // proper 5-opt templates
constexpr int kKoptSmemBytes = 96 * 1024;  // dynamic shared memory cap per block (opted in above 48 KB)
constexpr int kKoptMaxSegments = 8;
constexpr uint64_t kKoptBadPair = uint64_t{1} << 63;     // wide masks
constexpr uint32_t kKoptBadCost = uint32_t{1} << 29;      // narrow entries: cost of a bad pair
constexpr uint32_t kKoptSharedCode = 0x36DB6DB6u;         // bits 1 and 2 of ten 3-bit fields
// First pair index of a template that pairs some port 2e with 2e + 1 (re-adds deleted edge e,
// so every cell is invalid); proper templates never do.
constexpr uint8_t kKoptReaddsDeleted = 0xff;
constexpr uint8_t kKoptGeneralRow = 0xff;  // fastpat of a row that is not a gap-pattern row

// pair index of ports p < q among 2k ports (row-major upper triangle)
__host__ __device__ constexpr int kopt_pair_index(int p, int q, int ports) {
  return p * ports - (p * (p + 1)) / 2 + (q - p - 1);
}

struct KoptSegment {
  const int32_t* __restrict__ tasks;  // rows x 12 int32 (48-byte rows: 10 ports + int64)
  int64_t* __restrict__ costs;        // rows x T
  int64_t rows;
  const uint8_t* __restrict__ pairs;  // T x k pair indices (device)
  const uint32_t* __restrict__ patterns;  // T: bit g = the template is invalid on rows of gap pattern g
  const uint32_t* __restrict__ validity;  // 32 x ceil(T/32): bit t % 32 of word [g][t / 32] = patterns[t] bit g
  int32_t canonical;                      // 1: the table is the proper one (kopt_rows.cuh may serve it)
  uint32_t* __restrict__ improving;   // rows x mask_words: bit t = template t improves the row
  int32_t* __restrict__ first;        // rows: first improving template, or -1
  int32_t k;
  int32_t templates;
  int32_t rows_per_tile;
  int32_t tile_begin;                 // first block index of this segment
  int32_t mask_words;                 // 0: no improving sets (the plain cost matrix)
  int32_t write_costs;                // 0: improving sets only
};

struct KoptLaunch {
  KoptSegment seg[kKoptMaxSegments];
  int32_t segments;
  int32_t dist_type;
  int32_t n;
  const int2* __restrict__ xy;
};

// Shared-memory tile: 8-byte arrays first, then 4-byte, then bytes.
struct KoptSmem {
  uint64_t* mask;     // rows * npairs: packed entries (narrow) or one-hot masks (wide, repeating rows)
  uint64_t* delmask;  // rows: one-hot codes of the deleted edges
  int32_t* ports;     // rows * ports: node ids
  int32_t* dist;      // rows * npairs (wide)
  uint8_t* cls;       // rows * ports
  uint8_t* mrank;     // rows * ports: rank of the port's class among the multi classes, or 0xff
  uint8_t* repeats;   // rows: 1 when the row repeats a node
  uint8_t* fastpat;   // rows: gap pattern of a gap-pattern row, else kKoptGeneralRow
  uint8_t* pp;        // npairs: first port of each pair
  uint8_t* pq;        // npairs: second port
  uint8_t* ctab;      // ports * ports: code of a class pair, 0xff on the diagonal
  int64_t* deleted;   // rows: deleted cost (improving sets only)
  uint32_t* imask;    // rows * mask words: improving templates (improving sets only)
};

__host__ __device__ constexpr int kopt_tile_smem(int k, int rows, int mask_words = 0) {
  const int ports = 2 * k, npairs = k * (ports - 1);
  const int bytes = 2 * rows * ports + 2 * rows + 2 * npairs + ports * ports;
  return rows * npairs * 8 + rows * 8 + rows * ports * 4 + rows * npairs * 4 + ((bytes + 15) & ~15) +
         (mask_words > 0 ? rows * 8 + rows * mask_words * 4 : 0);
}

__device__ __forceinline__ KoptSmem kopt_carve(unsigned char* base, int k, int rows, int mask_words = 0) {
  const int ports = 2 * k, npairs = k * (ports - 1);
  KoptSmem s;
  s.mask = reinterpret_cast<uint64_t*>(base);
  s.delmask = s.mask + rows * npairs;
  s.ports = reinterpret_cast<int32_t*>(s.delmask + rows);
  s.dist = s.ports + rows * ports;
  s.cls = reinterpret_cast<uint8_t*>(s.dist + rows * npairs);
  s.mrank = s.cls + rows * ports;
  s.repeats = s.mrank + rows * ports;
  s.fastpat = s.repeats + rows;
  s.pp = s.fastpat + rows;
  s.pq = s.pp + npairs;
  s.ctab = s.pq + npairs;
  const int bytes = 2 * rows * ports + 2 * rows + 2 * npairs + ports * ports;
  s.deleted = reinterpret_cast<int64_t*>(reinterpret_cast<unsigned char*>(s.cls) + ((bytes + 15) & ~15));
  s.imask = reinterpret_cast<uint32_t*>(s.deleted + (mask_words > 0 ? rows : 0));
  return s;
}

// Pair decode and class-pair code tables for k (any group of threads; callers synchronise).
template <int K>
__device__ __forceinline__ void kopt_tables(uint8_t* pp, uint8_t* pq, uint8_t* ctab, int tid, int threads) {
  constexpr int P = 2 * K, NP = K * (P - 1);
  for (int i = tid; i < NP; i += threads) {
    int p = 0, rest = i;
    while (rest >= P - 1 - p) {
      rest -= P - 1 - p;
      ++p;
    }
    pp[i] = static_cast<uint8_t>(p);
    pq[i] = static_cast<uint8_t>(p + 1 + rest);
  }
  for (int i = tid; i < P * P; i += threads) {
    const int a = i / P, b = i - (i / P) * P;
    ctab[i] = a == b ? 0xff : static_cast<uint8_t>(kopt_pair_index(min(a, b), max(a, b), P));
  }
}

// Stage B for one row: port classes (first port with the same node), the repeat flag, the rank
// of each port's class among the multi classes (classes of two or more ports) and the one-hot
// codes of the deleted edges.
template <int K>
__device__ __forceinline__ void kopt_row_classes(const int32_t* nodes, const uint8_t* ctab, uint8_t* cls, uint8_t* mrank,
                                                 uint8_t* repeats, uint64_t* delmask) {
  constexpr int P = 2 * K;
  int32_t nd[P];
#pragma unroll
  for (int p = 0; p < P; ++p) nd[p] = nodes[p];
  int c[P];
  bool multi[P];
  bool rep = false;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    int cp = p;
    bool shared = false;
#pragma unroll
    for (int q = P - 1; q >= 0; --q) {
      if (q != p && nd[q] == nd[p]) {
        shared = true;
        if (q < p) cp = q;
      }
    }
    c[p] = cp;
    multi[p] = shared;
    rep = rep || shared;
    cls[p] = static_cast<uint8_t>(cp);
  }
  uint64_t dm = 0;
  if (rep) {
#pragma unroll
    for (int p = 0; p < P; ++p) {
      int rank = 0;  // multi classes whose first port precedes this port's class
#pragma unroll
      for (int q = 0; q < P; ++q) rank += (q < c[p] && c[q] == q && multi[q]) ? 1 : 0;
      mrank[p] = multi[p] ? static_cast<uint8_t>(rank) : 0xff;
    }
#pragma unroll
    for (int e = 0; e < K; ++e) {
      const int code = ctab[c[2 * e] * P + c[2 * e + 1]];
      if (code != 0xff) dm |= uint64_t{1} << code;
    }
  }
  *repeats = rep ? 1 : 0;
  *delmask = dm;
}

// Stage B's test for a gap-pattern row: its gap pattern, or kKoptGeneralRow when some equal port
// pair is not a closed gap.
template <int K>
__device__ __forceinline__ uint8_t kopt_gap_pattern(const int32_t* nodes) {
  constexpr int P = 2 * K;
  int32_t nd[P];
#pragma unroll
  for (int p = 0; p < P; ++p) nd[p] = nodes[p];
  int equal = 0;
#pragma unroll
  for (int p = 0; p < P; ++p) {
#pragma unroll
    for (int q = p + 1; q < P; ++q) equal += nd[p] == nd[q] ? 1 : 0;
  }
  uint32_t g = 0;
#pragma unroll
  for (int e = 0; e < K; ++e) g |= (nd[2 * e + 1] == nd[(2 * e + 2) % P] ? 1u : 0u) << e;
  return equal == __popc(g) ? static_cast<uint8_t>(g) : kKoptGeneralRow;
}

// Stage C for one (row, pair): the exact distance and the pair's entry (narrow) or mask (wide).
template <int K, int kSpan>
__device__ __forceinline__ void kopt_pair_entry(const KoptSmem& sm, int r, int pid, const int2* xy, int32_t dist_type) {
  constexpr int P = 2 * K, NP = K * (P - 1);
  const int p = sm.pp[pid], q = sm.pq[pid];
  const int32_t* pr = sm.ports + r * P;
  const int2 a = __ldg(xy + pr[p]);
  const int2 b = __ldg(xy + pr[q]);
  const uint32_t d = exact_distance<kSpan>(a, b, dist_type);
  if constexpr (kSpan == kSpanWide) {
    sm.dist[r * NP + pid] = static_cast<int32_t>(d);
    if (sm.repeats[r] != 0) {
      const uint8_t* cr = sm.cls + r * P;
      const int code = sm.ctab[cr[p] * P + cr[q]];
      const bool bad = code == 0xff || ((sm.delmask[r] >> code) & 1u) != 0;
      sm.mask[r * NP + pid] = bad ? kKoptBadPair : uint64_t{1} << code;
    }
  } else {
    uint32_t lo = d, hi = 0;
    if (sm.repeats[r] != 0) {
      const uint8_t* cr = sm.cls + r * P;
      const int code = sm.ctab[cr[p] * P + cr[q]];
      if (code == 0xff || ((sm.delmask[r] >> code) & 1u) != 0) {
        lo = kKoptBadCost;
      } else {
        const int ra = sm.mrank[r * P + p], rb = sm.mrank[r * P + q];
        if (ra != 0xff && rb != 0xff) hi = 1u << (3 * kopt_pair_index(min(ra, rb), max(ra, rb), 5));
      }
    }
    sm.mask[r * NP + pid] = (static_cast<uint64_t>(hi) << 32) | lo;
  }
}

// Stage D for one cell.
template <int K, int kSpan>
__device__ __forceinline__ int64_t kopt_cell(const KoptSmem& sm, int r, const int (&pid)[K]) {
  constexpr int NP = K * (2 * K - 1);
  if constexpr (kSpan == kSpanWide) {
    const int32_t* dr = sm.dist + r * NP;
    int64_t v = 0;
#pragma unroll
    for (int i = 0; i < K; ++i) v += dr[pid[i]];
    if (sm.repeats[r] != 0) {
      const uint64_t* mr = sm.mask + r * NP;
      uint64_t m = 0;
#pragma unroll
      for (int i = 0; i < K; ++i) m |= mr[pid[i]];
      if ((m & kKoptBadPair) != 0 || __popcll(m) != K) v = INT64_MAX;
    }
    return v;
  } else {
    const uint64_t* er = sm.mask + r * NP;
    uint64_t acc = 0;
#pragma unroll
    for (int i = 0; i < K; ++i) acc += er[pid[i]];
    const uint32_t lo = static_cast<uint32_t>(acc), hi = static_cast<uint32_t>(acc >> 32);
    return (lo >= kKoptBadCost || (hi & kKoptSharedCode) != 0) ? INT64_MAX : static_cast<int64_t>(lo);
  }
}

template <int K, int kSpan>
__device__ __forceinline__ void kopt_tile(const KoptLaunch& L, const KoptSegment& S, int64_t row0, int rows,
                                          unsigned char* smem, int32_t* error) {
  constexpr int P = 2 * K, NP = K * (P - 1);
  const KoptSmem sm = kopt_carve(smem, K, S.rows_per_tile, S.mask_words);
  const int tid = threadIdx.x;
  const int W = S.mask_words;
  kopt_tables<K>(sm.pp, sm.pq, sm.ctab, tid, kKoptThreads);
  if (W > 0) {
    for (int r = tid; r < rows; r += kKoptThreads) {
      sm.deleted[r] = __ldg(reinterpret_cast<const long long*>(S.tasks + (row0 + r) * 12 + 10));
    }
    for (int i = tid; i < rows * W; i += kKoptThreads) sm.imask[i] = 0;
  }
  for (int i = tid; i < rows * P; i += kKoptThreads) {
    const int r = i / P, p = i - (i / P) * P;
    int32_t node = __ldg(S.tasks + (row0 + r) * 12 + p);
    if (static_cast<uint32_t>(node) >= static_cast<uint32_t>(L.n)) {
      atomicOr(error, 1);
      node = 0;
    }
    sm.ports[i] = node;
  }
  __syncthreads();
  for (int r = tid; r < rows; r += kKoptThreads) {
    const uint8_t g = kopt_gap_pattern<K>(sm.ports + r * P);
    sm.fastpat[r] = g;
    if (g == kKoptGeneralRow) {
      kopt_row_classes<K>(sm.ports + r * P, sm.ctab, sm.cls + r * P, sm.mrank + r * P, sm.repeats + r, sm.delmask + r);
    }
  }
  __syncthreads();
  for (int i = tid; i < rows * NP; i += kKoptThreads) {
    const int r = i / NP, pid = i - r * NP;
    if (sm.fastpat[r] != kKoptGeneralRow) {  // gap-pattern row: the distance alone
      const int32_t* pr = sm.ports + r * P;
      sm.dist[i] = static_cast<int32_t>(
          exact_distance<kSpan>(__ldg(L.xy + pr[sm.pp[pid]]), __ldg(L.xy + pr[sm.pq[pid]]), L.dist_type));
    } else {
      kopt_pair_entry<K, kSpan>(sm, r, pid, L.xy, L.dist_type);
    }
  }
  __syncthreads();
  const int T = S.templates;
  const int per_step = kKoptThreads / T;
  const int rr = tid / T, t = tid - rr * T;
  if (rr < per_step) {
    int pid[K];
#pragma unroll
    for (int i = 0; i < K; ++i) pid[i] = __ldg(S.pairs + t * K + i);
    const bool readds_deleted = pid[0] == kKoptReaddsDeleted;
    if (readds_deleted) pid[0] = 0;
    const uint32_t invalid_on = __ldg(S.patterns + t);
    long long* out = reinterpret_cast<long long*>(S.costs + row0 * T) + static_cast<int64_t>(rr) * T + t;
    const int64_t out_step = static_cast<int64_t>(per_step) * T;
    for (int r = rr; r < rows; r += per_step, out += out_step) {
      const uint32_t g = sm.fastpat[r];
      int64_t v;
      if (g != kKoptGeneralRow) {
        const int32_t* dr = sm.dist + r * NP;
        if constexpr (kSpan == kSpanWide) {
          int64_t sum = 0;
#pragma unroll
          for (int i = 0; i < K; ++i) sum += dr[pid[i]];
          v = sum;
        } else {  // k distances < 2^26.5 each: the sum fits 32 bits
          uint32_t sum = 0;
#pragma unroll
          for (int i = 0; i < K; ++i) sum += static_cast<uint32_t>(dr[pid[i]]);
          v = sum;
        }
        if (((invalid_on >> g) & 1u) != 0 || readds_deleted) v = INT64_MAX;
      } else {
        v = readds_deleted ? INT64_MAX : kopt_cell<K, kSpan>(sm, r, pid);
      }
      if (S.write_costs != 0) __stcs(out, static_cast<long long>(v));
      // the leaf consumer tries templates with added cost < deleted cost (src/cpu/kopt_search.cpp:697)
      if (W > 0 && v < sm.deleted[r]) atomicOr(sm.imask + r * W + (t >> 5), 1u << (t & 31));
    }
  }
  if (W == 0) return;
  __syncthreads();
  for (int i = tid; i < rows * W; i += kKoptThreads) S.improving[row0 * W + i] = sm.imask[i];
  for (int r = tid; r < rows; r += kKoptThreads) {
    int f = -1;
    for (int w = W - 1; w >= 0; --w) {
      const uint32_t bits = sm.imask[r * W + w];
      if (bits != 0) f = w * 32 + __ffs(bits) - 1;
    }
    S.first[row0 + r] = f;
  }
}

template <int kSpan>
static __global__ void __launch_bounds__(kKoptThreads, 9) kopt_cost_kernel(KoptLaunch L,
                                                                        int32_t* __restrict__ error) {
  extern __shared__ __align__(16) unsigned char smem[];
  int si = 0;
  while (si + 1 < L.segments && static_cast<int32_t>(blockIdx.x) >= L.seg[si + 1].tile_begin) ++si;
  const KoptSegment& S = L.seg[si];
  const int64_t row0 = static_cast<int64_t>(blockIdx.x - S.tile_begin) * S.rows_per_tile;
  if (row0 >= S.rows) return;
  const int rows = static_cast<int>(min(static_cast<int64_t>(S.rows_per_tile), S.rows - row0));
  switch (S.k) {
    case 3:
      kopt_tile<3, kSpan>(L, S, row0, rows, smem, error);
      break;
    case 4:
      kopt_tile<4, kSpan>(L, S, row0, rows, smem, error);
      break;
    default:
      kopt_tile<5, kSpan>(L, S, row0, rows, smem, error);
      break;
  }
}

}  // namespace cee
