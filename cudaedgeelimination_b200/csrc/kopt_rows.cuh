// Exact k-opt leaf cost matrix for the proper templates: one thread per row, the templates
// compiled in.
//
// Same cells as kopt_cost.cuh (src/cpu/kopt_search.cpp:962-1042): costs[row][t] = the sum of the k
// added-edge distances of template t, or INT64_MAX when an added edge is a self loop, re-adds a
// deleted edge or repeats another added edge. This kernel serves the case that dominates the
// reference's use -- the library's own proper templates (BuildKOptReconnectTable,
// src/cpu/kopt_search.cpp:1143-1193) on coordinates of span < 2^26 -- and is chosen by the host
// when a segment's template table is byte-identical to the proper one; any other table, and wide
// coordinates, take kopt_cost_kernel.
//
// The proper templates are generated at compile time (kopt_canon_table, the same lexicographic
// enumeration and single-cycle test as the reference) and pinned by static_asserts to the
// reference's generator hashes (configs/kopt_reconnect_hashes_v1.txt). With the templates known
// to the compiler, a thread keeps its row's k(2k-1) pair distances in registers and every cell is
// k-1 register adds with compile-time operands, a validity bit and a store:
//   * a row cut from a tour repeats a node only where two deleted edges are adjacent in the tour
//     (a closed gap, kopt_cost.cuh); its validity depends on (template, gap pattern g) alone. The
//     host's table valid[g][w] (bit t mod 32 of word t / 32 = template t invalid on pattern g, 896
//     bytes, cached in L1) gives a thread its row's words.
//   * any other row (a "general" row: repeats that are not closed gaps) is rare in the reference's
//     leaf batches; a warp holding one scores all its rows cooperatively with kopt_cost.cuh's
//     class-code entries.
// Stores: the cells are HBM-bound writes (8 T bytes per row against 48 read), so each warp stages
// its rows' cells in shared memory and leaves the writing to the bulk-copy engine (no multicast):
//   * k = 5 (1,664 B per row = 13 lines): 13 boxes of one line x the warp's 32 rows, each one 2-D
//     tensor store through the segment's tensor map (rows past the segment's end are clipped by the
//     engine); a box writes whole lines, so none reaches DRAM partly written (which costs a read);
//   * k = 4 (200 B per row): the warp's 32 rows are one contiguous 6,400 B run of the output,
//     written by one bulk copy (an odd last row of a segment is stored directly);
//   * k = 3 (32 B per row): two 16-byte streaming stores per row.
// Fused leaf consume (kMasks): the improving-template masks (cost < the row's deleted cost, the
// templates the reference's consumer tries, src/cpu/kopt_search.cpp:694-715) are accumulated in
// registers and written per row with the first improving template; the cost matrix is optional.
#pragma once

#include <cuda.h>  // CUtensorMap (the type only; the library does not link the driver API)

#include <type_traits>
#include <utility>

#include "kopt_cost.cuh"

namespace cee {

// f(integral_constant<int, i>) for i = Begin, ..., End - 1, unrolled at compile time.
template <int Begin, typename F, int... I>
__device__ __forceinline__ void static_for_seq(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, Begin + I>{}), ...);
}
template <int Begin, int End, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_seq<Begin>(f, std::make_integer_sequence<int, End - Begin>{});
}

// ---------------------------------------------------------------- compile-time templates -----

template <int K>
struct KoptCanonTable {
  static constexpr int P = 2 * K;
  static constexpr int T = K == 3 ? 4 : (K == 4 ? 25 : 208);
  static constexpr int NP = K * (P - 1);
  static constexpr int W = (T + 31) / 32;
  uint8_t mate[T][P] = {};
  uint8_t pair[T][K] = {};       // kopt_pair_index of the added edges, ascending first port
  uint32_t invalid_on[T] = {};   // bit g: invalid on gap-pattern rows of pattern g
  int count = 0;
  uint64_t hash = 0;
};

// The alternating walk mate, component, mate, ... from port 0 closes after all 2k ports iff the
// template and the component matching 1-2, 3-4, ..., (2k-1)-0 form one Hamiltonian cycle.
template <int K>
constexpr bool kopt_single_cycle(const uint8_t (&mate)[2 * K]) {
  constexpr int P = 2 * K;
  int p = 0, steps = 0;
  do {
    if (steps % 2 == 0) {
      p = mate[p];
    } else {
      p = p == 0 ? P - 1 : (p == P - 1 ? 0 : (p % 2 == 1 ? p + 1 : p - 1));
    }
    ++steps;
  } while (p != 0 && steps <= P);
  return steps == P;
}

// Perfect matchings in lexicographic order (the lowest unmatched port takes each higher unmatched
// port in turn), kept when proper: no port 2e paired with 2e+1, one alternating cycle.
template <int K>
constexpr void kopt_extend(KoptCanonTable<K>& tab, uint8_t (&mate)[2 * K]) {
  constexpr int P = 2 * K;
  int first = -1;
  for (int p = 0; p < P && first < 0; ++p) {
    if (mate[p] == 0xff) first = p;
  }
  if (first < 0) {
    for (int e = 0; e < K; ++e) {
      if (mate[2 * e] == 2 * e + 1) return;
    }
    if (!kopt_single_cycle<K>(mate)) return;
    for (int p = 0; p < P; ++p) tab.mate[tab.count][p] = mate[p];
    ++tab.count;
    return;
  }
  for (int q = first + 1; q < P; ++q) {
    if (mate[q] != 0xff) continue;
    mate[first] = static_cast<uint8_t>(q);
    mate[q] = static_cast<uint8_t>(first);
    kopt_extend<K>(tab, mate);
    mate[first] = 0xff;
    mate[q] = 0xff;
  }
}

// FNV-1a over "CUDAEE_KOPT_RECONNECT_TEMPLATES_V1", k and the count (little endian), then each
// template's 2k mates: the reference's generator hash of the table.
template <int K>
constexpr uint64_t kopt_table_hash(const KoptCanonTable<K>& tab) {
  uint64_t h = 14695981039346656037ull;
  const char tag[] = "CUDAEE_KOPT_RECONNECT_TEMPLATES_V1";
  for (int i = 0; tag[i] != '\0'; ++i) h = (h ^ static_cast<uint8_t>(tag[i])) * 1099511628211ull;
  for (int s = 0; s < 32; s += 8) h = (h ^ ((static_cast<uint32_t>(K) >> s) & 0xffu)) * 1099511628211ull;
  for (int s = 0; s < 32; s += 8) h = (h ^ ((static_cast<uint32_t>(tab.count) >> s) & 0xffu)) * 1099511628211ull;
  for (int t = 0; t < tab.count; ++t) {
    for (int p = 0; p < 2 * K; ++p) h = (h ^ tab.mate[t][p]) * 1099511628211ull;
  }
  return h;
}

template <int K>
constexpr KoptCanonTable<K> kopt_canon_table() {
  constexpr int P = 2 * K;
  KoptCanonTable<K> tab{};
  uint8_t mate[P] = {};
  for (int p = 0; p < P; ++p) mate[p] = 0xff;
  kopt_extend<K>(tab, mate);
  for (int t = 0; t < tab.count; ++t) {
    int found = 0;
    for (int p = 0; p < P; ++p) {
      if (p < tab.mate[t][p]) tab.pair[t][found++] = static_cast<uint8_t>(kopt_pair_index(p, tab.mate[t][p], P));
    }
  }
  // validity on gap-pattern rows: ports 2e+1 and (2e+2) mod 2k merge when gap e is closed
  for (int g = 0; g < (1 << K); ++g) {
    int cls[P] = {};
    for (int p = 0; p < P; ++p) cls[p] = p;
    for (int e = 0; e < K; ++e) {
      if ((g >> e) & 1) {
        const int a = cls[2 * e + 1], b = cls[(2 * e + 2) % P];
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        for (int p = 0; p < P; ++p) {
          if (cls[p] == hi) cls[p] = lo;
        }
      }
    }
    for (int t = 0; t < tab.count; ++t) {
      int codes[K] = {};
      bool invalid = false;
      for (int i = 0; i < K && !invalid; ++i) {
        int p = 0, rest = tab.pair[t][i];
        while (rest >= P - 1 - p) {
          rest -= P - 1 - p;
          ++p;
        }
        const int q = p + 1 + rest;
        const int a = cls[p] < cls[q] ? cls[p] : cls[q], b = cls[p] < cls[q] ? cls[q] : cls[p];
        const int code = a * P + b;
        invalid = a == b;
        for (int e = 0; e < K && !invalid; ++e) {
          const int da = cls[2 * e] < cls[2 * e + 1] ? cls[2 * e] : cls[2 * e + 1];
          const int db = cls[2 * e] < cls[2 * e + 1] ? cls[2 * e + 1] : cls[2 * e];
          invalid = code == da * P + db;
        }
        for (int j = 0; j < i && !invalid; ++j) invalid = codes[j] == code;
        codes[i] = code;
      }
      if (invalid) tab.invalid_on[t] |= 1u << g;
    }
  }
  tab.hash = kopt_table_hash<K>(tab);
  return tab;
}

template <int K>
struct KoptCanon {
  static constexpr KoptCanonTable<K> value = kopt_canon_table<K>();
};

// Pair index i of proper template t, as a compile-time scalar.
template <int K, int t, int i>
constexpr int kKoptCanonPair = KoptCanon<K>::value.pair[t][i];

// The reference's pinned generator hashes (configs/kopt_reconnect_hashes_v1.txt:3-5).
static_assert(KoptCanon<3>::value.count == 4 && KoptCanon<3>::value.hash == 0xe58af5e08d290d04ull,
              "proper 3-opt templates");
static_assert(KoptCanon<4>::value.count == 25 && KoptCanon<4>::value.hash == 0x03179e3ca191ce82ull,
              "proper 4-opt templates");
static_assert(KoptCanon<5>::value.count == 208 && KoptCanon<5>::value.hash == 0x6696dde548591bceull,
              "proper 5-opt templates");

// ---------------------------------------------------------------- the kernel -----------------
//
// A block is 4 independent warps; a warp owns 32 consecutive rows of one segment, one row per
// lane, and needs no block barrier. All of a block's rows have the same k, and so does the layout
// of its staging areas in shared memory: per warp two k = 5 box buffers (1 KB aligned, so a box is
// written while the engine still reads the previous one), or the k = 4 tile, or the general-row
// scratch. Six blocks per SM (80 registers a thread, 33 KB of shared memory a block). Measured on
// the 1,000,000-row matrix: 4-warp blocks 0.168 ms, 8-warp blocks 0.172 ms; one box buffer (more
// blocks per SM, 64 registers) 0.179 ms; an L2 prefetch of the task rows a wave ahead, no gain.

constexpr int kKoptRowWarps = 4;
constexpr int kKoptRowThreads = 32 * kKoptRowWarps;  // also the rows of a block
constexpr int kKopt5Box = 16;                         // k = 5: cells per box (one 128-byte line of a row)
constexpr int kKopt5BoxBytes = 32 * kKopt5Box * 8;   // a box: the warp's 32 rows x 16 cells
constexpr int kKopt5Buffers = 2;
constexpr int kKopt4TileBytes = 32 * 25 * 8;          // k = 4: the warp's 32 rows (contiguous in the output)
constexpr int kKoptWarpStage = 13 * 512;              // k = 3 / 4 staging per warp (tile, or general scratch)
constexpr int kKoptRowsSmem =
    (kKoptRowWarps * kKopt5Buffers * kKopt5BoxBytes > kKoptRowWarps * kKoptWarpStage
         ? kKoptRowWarps * kKopt5Buffers * kKopt5BoxBytes
         : kKoptRowWarps * kKoptWarpStage) +
    1024;  // + slack to align the base to 1 KB
static_assert(kKopt4TileBytes <= kKoptWarpStage, "k = 4 tile");
static_assert(kopt_tile_smem(5, 1) <= kKopt5BoxBytes && kopt_tile_smem(4, 1) <= kKoptWarpStage, "general-row scratch");
static_assert(KoptCanonTable<5>::T % kKopt5Box == 0, "k = 5 boxes tile the row");

// The warp's staging area for rows of k.
__device__ __forceinline__ unsigned char* kopt_rows_stage(unsigned char* smem, int k, int warp) {
  return smem + warp * (k == 5 ? kKopt5Buffers * kKopt5BoxBytes : kKoptWarpStage);
}

// Kernel parameters: the launch, and per k = 5 segment that writes costs the tensor map of its
// output ([rows][208] int64; {16 cells, 32 rows} boxes; 128-byte swizzle).
struct KoptRowsParams {
  CUtensorMap box5[kKoptMaxSegments];
  KoptLaunch L;
};

__device__ __forceinline__ void bulk_fence_shared() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// One bulk copy shared -> global of `bytes` (16-byte aligned addresses, a multiple of 16 bytes).
__device__ __forceinline__ void bulk_store(void* global, const void* shared, uint32_t bytes) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(shared));
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n"
               :: "l"(global), "r"(s), "r"(bytes) : "memory");
}
// One 2-D tensor store of the box at `shared` to coordinates {c0, c1} (no multicast).
__device__ __forceinline__ void tensor_store_2d(const CUtensorMap* map, const void* shared, int32_t c0, int32_t c1) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(shared));
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];\n"
               :: "l"(reinterpret_cast<uint64_t>(map)), "r"(s), "r"(c0), "r"(c1) : "memory");
}
// Waits until at most N of this thread's bulk copies still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;\n" :: "n"(N) : "memory");
}
// Waits until every bulk copy of this thread has completed.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

// A cell of a gap-pattern row: the sum, or INT64_MAX when `bad`.
__device__ __forceinline__ uint2 kopt_cell_word(uint32_t sum, bool bad) {
  return make_uint2(bad ? 0xffffffffu : sum, bad ? 0x7fffffffu : 0u);
}

// The rows `rows_mask` of the warp whose first row is warp_row0, one at a time, with kopt_cost.cuh's
// class-code entries (any row, repeated ports included): cells go straight to the output and, with
// kMasks, the improving masks and first improving template. `scratch` holds one row's tile.
template <int K, int kSpan, bool kMasks>
__device__ void kopt_general_rows(const KoptLaunch& L, const KoptSegment& S, int64_t warp_row0, unsigned rows_mask,
                                  unsigned char* scratch, int lane, int32_t* error) {
  constexpr int P = 2 * K, NP = K * (P - 1), T = KoptCanonTable<K>::T, W = KoptCanonTable<K>::W;
  const KoptSmem sm = kopt_carve(scratch, K, 1);
  kopt_tables<K>(sm.pp, sm.pq, sm.ctab, lane, 32);
  while (rows_mask != 0) {
    const int r = __ffs(rows_mask) - 1;
    rows_mask &= rows_mask - 1;
    const int64_t row = warp_row0 + r;
    __syncwarp();
    if (lane < P) {
      int32_t node = __ldg(S.tasks + row * 12 + lane);
      if (static_cast<uint32_t>(node) >= static_cast<uint32_t>(L.n)) {
        atomicOr(error, 1);
        node = 0;
      }
      sm.ports[lane] = node;
    }
    __syncwarp();
    if (lane == 0) kopt_row_classes<K>(sm.ports, sm.ctab, sm.cls, sm.mrank, sm.repeats, sm.delmask);
    __syncwarp();
    for (int pid = lane; pid < NP; pid += 32) kopt_pair_entry<K, kSpan>(sm, 0, pid, L.xy, L.dist_type);
    __syncwarp();
    const int64_t deleted = kMasks ? __ldg(reinterpret_cast<const long long*>(S.tasks + row * 12 + 10)) : 0;
    int64_t* out = S.costs + row * T;
    int first = -1;
    for (int t0 = 0; t0 < T; t0 += 32) {
      const int t = t0 + lane;
      int64_t v = INT64_MAX;
      if (t < T) {
        int pid[K];
#pragma unroll
        for (int i = 0; i < K; ++i) pid[i] = __ldg(S.pairs + t * K + i);
        v = kopt_cell<K, kSpan>(sm, 0, pid);
        if (S.write_costs != 0) out[t] = v;
      }
      if constexpr (kMasks) {
        const unsigned word = __ballot_sync(kFullMask, t < T && v < deleted);
        if (lane == 0) S.improving[row * W + t0 / 32] = word;
        if (first < 0 && word != 0) first = t0 + __ffs(word) - 1;
      }
    }
    if (kMasks && lane == 0) S.first[row] = first;
  }
  __syncwarp();
}

// The warp's rows row0 .. row0 + rows - 1 (rows <= 32) of segment S, row row0 + lane on this lane.
template <int K, int kSpan, bool kMasks>
__device__ __forceinline__ void kopt_proper_rows_warp(const KoptLaunch& L, const KoptSegment& S, const CUtensorMap* box5,
                                               int64_t row0, int rows, unsigned char* stage, int32_t* error) {
  using Tab = KoptCanonTable<K>;
  constexpr int P = Tab::P, NP = Tab::NP, T = Tab::T, W = Tab::W;
  const int lane = threadIdx.x & 31;
  const bool live = lane < rows;
  const int64_t row = row0 + lane;
  int32_t nd[P];
  int64_t deleted = 0;
  {
    int4 q[3] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
    if (live) {
      const int4* src = reinterpret_cast<const int4*>(S.tasks + row * 12);
      q[0] = __ldg(src);
      q[1] = __ldg(src + 1);
      q[2] = __ldg(src + 2);
    }
    const int32_t words[12] = {q[0].x, q[0].y, q[0].z, q[0].w, q[1].x, q[1].y, q[1].z, q[1].w,
                               q[2].x, q[2].y, q[2].z, q[2].w};
#pragma unroll
    for (int p = 0; p < P; ++p) {
      nd[p] = words[p];
      if (static_cast<uint32_t>(nd[p]) >= static_cast<uint32_t>(L.n)) {
        atomicOr(error, 1);
        nd[p] = 0;
      }
    }
    deleted = static_cast<int64_t>((static_cast<uint64_t>(static_cast<uint32_t>(words[11])) << 32) |
                                   static_cast<uint32_t>(words[10]));
  }
  // gap pattern: a gap-pattern row's equal port pairs are exactly its closed gaps
  int equal = 0;
  uint32_t g = 0;
#pragma unroll
  for (int p = 0; p < P; ++p) {
#pragma unroll
    for (int q = p + 1; q < P; ++q) equal += nd[p] == nd[q] ? 1 : 0;
  }
#pragma unroll
  for (int e = 0; e < K; ++e) g |= (nd[2 * e + 1] == nd[(2 * e + 2) % P] ? 1u : 0u) << e;
  if (__ballot_sync(kFullMask, live && equal != __popc(g)) != 0) {
    // a warp holding any other row scores all of its rows with the class-code path
    kopt_general_rows<K, kSpan, kMasks>(L, S, row0, __ballot_sync(kFullMask, live), stage, lane, error);
    return;
  }

  // the k(2k-1) pair distances in registers (compile-time indices; pairs no template uses are dropped)
  uint32_t d[NP];
  {
    int2 c[P];
    static_for<0, P>([&](auto pc) { c[decltype(pc)::value] = __ldg(L.xy + nd[decltype(pc)::value]); });
    static_for<0, P>([&](auto pc) {
      constexpr int p = decltype(pc)::value;
      static_for<p + 1, P>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        d[kopt_pair_index(p, q, P)] = exact_distance<kSpan>(c[p], c[q], L.dist_type);
      });
    });
  }
  // the leaf consumer tries templates with added cost < deleted cost (src/cpu/kopt_search.cpp:697);
  // valid sums are < 2^29, so the comparison runs in 32 bits with the deleted cost clamped
  const uint32_t dl = deleted <= 0 ? 0u : (deleted >= 0xffffffffll ? 0xffffffffu : static_cast<uint32_t>(deleted));
  const bool write = S.write_costs != 0;
  // per 32 templates: the row's validity word (read from L1 as the cells reach it) and, with
  // kMasks, the improving word, written once complete; first = the first improving template
  uint32_t valid_word = 0, improving_word = 0;
  int first = -1;

  // cell t of this row (compile-time t, in increasing order): its word, and its improving bit
  auto cell = [&](auto tc) -> uint2 {
    constexpr int t = decltype(tc)::value;
    if constexpr (t % 32 == 0) valid_word = __ldg(S.validity + g * W + t / 32);
    uint32_t sum = d[kKoptCanonPair<K, t, 0>];
    static_for<1, K>([&](auto ic) { sum += d[kKoptCanonPair<K, t, decltype(ic)::value>]; });
    const bool bad = ((valid_word >> (t % 32)) & 1u) != 0;
    if constexpr (kMasks) {
      improving_word |= static_cast<uint32_t>(!bad && sum < dl) << (t % 32);
      if constexpr (t % 32 == 31 || t == T - 1) {
        if (live) S.improving[row * W + t / 32] = improving_word;
        if (first < 0 && improving_word != 0) first = (t & ~31) + __ffs(improving_word) - 1;
        improving_word = 0;
      }
    }
    return kopt_cell_word(sum, bad);
  };

  if constexpr (K == 5) {
    if (write) {
      // 13 boxes of 16 cells, each one whole 128-byte line of every row of the warp (segments
      // start on a line), so that no line reaches DRAM partly written. Lane r's 128 bytes sit at
      // row r of the box with their 16-byte units swizzled by bits 7-9 of the offset (the tensor
      // map's 128-byte swizzle), so the lanes' 16-byte stores are conflict-free.
      const int swz = lane & 7;
      static_for<0, T / kKopt5Box>([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        unsigned char* box = stage + (j % kKopt5Buffers) * kKopt5BoxBytes;
        if constexpr (j >= kKopt5Buffers) {
          if (lane == 0) bulk_wait_read<kKopt5Buffers - 1>();
          __syncwarp();
        }
        static_for<0, kKopt5Box / 2>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          const uint2 a = cell(std::integral_constant<int, j * kKopt5Box + 2 * i>{});
          const uint2 b = cell(std::integral_constant<int, j * kKopt5Box + 2 * i + 1>{});
          *reinterpret_cast<uint4*>(box + lane * 128 + ((i ^ swz) << 4)) = make_uint4(a.x, a.y, b.x, b.y);
        });
        bulk_fence_shared();
        __syncwarp();
        if (lane == 0) {
          tensor_store_2d(box5, box, j * kKopt5Box, static_cast<int32_t>(row0));
          bulk_commit();
        }
      });
    } else {
      static_for<0, T>([&](auto tc) { (void)cell(tc); });
    }
  } else if constexpr (K == 4) {
    if (write) {
      // the warp's rows are contiguous in the output: stage them (row stride 200 bytes, so the
      // lanes' 8-byte stores are conflict-free) and write them with one bulk copy
      uint2* mine = reinterpret_cast<uint2*>(stage + lane * T * 8);
      static_for<0, T>([&](auto tc) { mine[decltype(tc)::value] = cell(tc); });
      bulk_fence_shared();
      __syncwarp();
      const int bulk_rows = rows & ~1;  // 200-byte rows: an even count is a multiple of 16 bytes
      if (lane == 0 && bulk_rows > 0) {
        bulk_store(S.costs + row0 * T, stage, static_cast<uint32_t>(bulk_rows) * T * 8);
        bulk_commit();
      }
      if (lane == rows - 1 && (rows & 1) != 0) {  // an odd last row: direct stores
        uint2* dst = reinterpret_cast<uint2*>(S.costs + row * T);
#pragma unroll
        for (int t = 0; t < T; ++t) dst[t] = mine[t];
      }
    } else {
      static_for<0, T>([&](auto tc) { (void)cell(tc); });
    }
  } else {
    uint2 v[T];
    static_for<0, T>([&](auto tc) { v[decltype(tc)::value] = cell(tc); });
    if (write && live) {
      uint4* out = reinterpret_cast<uint4*>(S.costs + row * T);
      static_for<0, T / 2>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        __stcs(out + i, make_uint4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y));
      });
    }
  }
  if constexpr (kMasks) {
    if (live) S.first[row] = first;
  }
  // the staging area stays in use until the bulk copies have read it, and the block's shared
  // memory must outlive them
  if (lane == 0) bulk_wait_all();
  __syncwarp();
}

template <int kSpan, bool kMasks>
static __global__ void __launch_bounds__(kKoptRowThreads, 6)
    kopt_rows_kernel(const __grid_constant__ KoptRowsParams P, int32_t* __restrict__ error) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const KoptLaunch& L = P.L;
  int si = 0;
  while (si + 1 < L.segments && static_cast<int32_t>(blockIdx.x) >= L.seg[si + 1].tile_begin) ++si;
  const KoptSegment& S = L.seg[si];
  const int warp = threadIdx.x >> 5;
  const int64_t row0 = static_cast<int64_t>(blockIdx.x - S.tile_begin) * kKoptRowThreads + warp * 32;
  if (row0 >= S.rows) return;  // warp-uniform; the kernel has no block barrier
  const int rows = static_cast<int>(min(static_cast<int64_t>(32), S.rows - row0));
  unsigned char* stage = kopt_rows_stage(smem, S.k, warp);
  switch (S.k) {
    case 3:
      kopt_proper_rows_warp<3, kSpan, kMasks>(L, S, &P.box5[si], row0, rows, stage, error);
      break;
    case 4:
      kopt_proper_rows_warp<4, kSpan, kMasks>(L, S, &P.box5[si], row0, rows, stage, error);
      break;
    default:
      kopt_proper_rows_warp<5, kSpan, kMasks>(L, S, &P.box5[si], row0, rows, stage, error);
      break;
  }
}

}  // namespace cee
