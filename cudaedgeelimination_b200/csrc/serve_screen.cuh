// Device side of the serving loop: one persistent kernel runs every admitted job.
//
// The host posts a job into a host-mapped mailbox (the descriptor, then its generation) with plain
// stores: no copy or other CUDA call per job, so a submission does not queue behind the copy
// engines' result downloads (while those fill the link, each small host-to-device copy waits tens of
// microseconds). One dispatcher warp (the last warp of block 0) polls the mailbox over PCIe and
// installs each posted job into the device slot table in seqlock order: state word = 0, the job's
// descriptor, the slot's ticket and done counters = generation << 32, state word = generation (see
// serve_read_job). A k-opt job's rows go up by one bulk copy per segment followed by the slot's
// rows-ready word (= generation), and the dispatcher installs the job only once that word shows its
// generation. Every other warp is a worker. Work is claimed with one atomicAdd on the slot's
// ticket, whose high half names the generation the item belongs to and whose low half the item
// index, so claims never retry however many warps contend. A warp keeps claiming from the job it
// holds while that job has items left; otherwise it scans the slots for the oldest published job
// with items left (jobs only get younger, so this keeps oldest-first order). A claim may land on
// a newer generation than the warp expected (the dispatcher republished the slot between the
// warp's check and its atomicAdd): the warp then reads that generation's descriptor and runs the item,
// so no item is ever lost; indices past a job's item count are simply dropped. The warp that
// finishes a job's last item (done counter) makes the job's outputs visible and writes the
// job's error word, then the generation, into the slot's words of a host-mapped array; the host
// then copies the results back. Jobs that arrive while others run share the warps item by item
// (continuous batching). Every wait is bounded: a warp that finds no work for `idle_limit`
// scans, or sees the stop word, leaves after its current item; the host relaunches the kernel
// when work arrives.
//
// Memory: snapshot arrays are read through the non-coherent L1 path (__ldg). That is safe
// because the host never writes snapshot memory while a launch runs: a snapshot upload first
// stops the kernel (stop word, wait for it to end) and the next launch starts with a clean L1.
// Per-job inputs (k-opt rows) are written into reused arena memory while the kernel runs, so
// they are read L2-coherently (__ldcg); the control table and the mailbox are read with volatile
// loads.
#pragma once

#include "jv_screen.cuh"
#include "kopt_cost.cuh"
#include "kopt_rows.cuh"

namespace cee {

constexpr int kServeWarps = 8;
constexpr int kServeMaxSlots = 256;
constexpr int kServeJv = 1;
constexpr int kServeKopt = 2;
constexpr int kServeJvTile = 32;          // JV edges per item
constexpr int kServeKoptRowsPerItem = 64; // k-opt rows per item, processed in chunks

struct ServeSegment {
  const int32_t* tasks;  // 48-byte rows
  int64_t* costs;        // rows x T, or null (improving sets only)
  int64_t rows;
  int64_t item_begin;    // first item (relative to the job) of this segment
  int32_t k, T, pad0, pad1;
  uint32_t* improving;   // rows x ceil(T / 32): bit t = template t improves the row, or null
  int32_t* first;        // rows: the first improving template, or -1
};

struct ServeJob {
  uint32_t generation;
  int32_t type;
  int32_t span;  // span class of the snapshot's coordinates (kSpanSmall / kSpanNarrow / kSpanWide)
  int32_t segments;
  uint32_t items;
  uint32_t rows_gate;  // 1: install only once the slot's rows-ready word equals the generation
  uint32_t host_outputs;  // 1: the outputs are page-locked host memory, written in place
  uint32_t pad;
  JvGraph g;  // JV jobs; k-opt jobs use g.xy / g.n / g.dist_type
  int32_t* witness;
  ServeSegment seg[3];
};

struct ServeControl {
  ServeJob jobs[kServeMaxSlots];
  unsigned long long ticket[kServeMaxSlots];  // generation << 32 | next item
  unsigned long long done[kServeMaxSlots];    // generation << 32 | items finished
  uint32_t state[kServeMaxSlots];
  // per job slot: the device bounds checks of the job now in the slot (1); reset when a job is
  // published there, so one job's bad index is reported for that job alone
  int32_t slot_error[kServeMaxSlots];
  uint32_t rows_ready[kServeMaxSlots];  // generation whose k-opt rows have landed in the arena
  uint32_t stop;
  int32_t error;  // loop-wide, sticky: a descriptor that never appeared (8)
};

// Host-mapped: the host writes a job's descriptor into desc[slot] and then its generation into
// posted[slot]; a slot is posted again only after its previous job has been reported, long after
// the dispatcher installed that one.
struct ServeMailbox {
  ServeJob desc[kServeMaxSlots];
  uint32_t posted[kServeMaxSlots];
};

// Bounded wait (about a second) for the descriptor of a generation whose item a claim returned.
constexpr int kServeDescriptorWaits = 1 << 22;
// Word of the host-mapped `finished` array that mirrors a lost item (error bit 8), so the host
// can fail the loop's pending jobs instead of waiting for them.
constexpr int kServeLostWord = 2 * kServeMaxSlots;

// k-opt rows per warp chunk: 8 rows of k = 3, 4 of k = 4, 2 of k = 5 (32..416 cells).
__host__ __device__ constexpr int serve_rows_per_chunk(int k) { return k == 3 ? 8 : (k == 4 ? 4 : 2); }

// One warp's k-opt tile (kopt_cost.cuh's layout), sized for the largest chunk of any k.
// (also the staging buffer of kopt_serve_proper32: one box of 16 cells x 32 rows)
constexpr int kServeKoptScratch = 4096;
static_assert(kopt_tile_smem(3, serve_rows_per_chunk(3)) <= kServeKoptScratch, "k = 3 chunk tile");
static_assert(kopt_tile_smem(4, serve_rows_per_chunk(4)) <= kServeKoptScratch, "k = 4 chunk tile");
static_assert(kopt_tile_smem(5, serve_rows_per_chunk(5)) <= kServeKoptScratch, "k = 5 chunk tile");

// The k-opt cells of rows [row_begin, row_end) of a segment, one warp, chunk by chunk
// (kopt_cost_kernel's stages at warp size).
template <int K, int kSpan>
__device__ void kopt_rows_warp(const ServeSegment& S, int64_t row_begin, int64_t row_end, const uint8_t* tpairs,
                               const int2* xy, int32_t n, int32_t dist_type, unsigned char* scratch, int lane,
                               int32_t* error) {
  constexpr int P = 2 * K, NP = K * (P - 1), C = serve_rows_per_chunk(K);
  constexpr int T = K == 3 ? 4 : (K == 4 ? 25 : 208);
  const KoptSmem sm = kopt_carve(scratch, K, C);
  kopt_tables<K>(sm.pp, sm.pq, sm.ctab, lane, 32);
  for (int64_t row0 = row_begin; row0 < row_end; row0 += C) {
    const int rows = static_cast<int>(min(static_cast<int64_t>(C), row_end - row0));
    __syncwarp();
    for (int i = lane; i < rows * P; i += 32) {
      const int r = i / P, p = i - (i / P) * P;
      int32_t node = __ldcg(S.tasks + (row0 + r) * 12 + p);
      if (static_cast<uint32_t>(node) >= static_cast<uint32_t>(n)) {
        atomicOr(error, 1);
        node = 0;
      }
      sm.ports[i] = node;
    }
    __syncwarp();
    if (lane < rows) {
      kopt_row_classes<K>(sm.ports + lane * P, sm.ctab, sm.cls + lane * P, sm.mrank + lane * P, sm.repeats + lane,
                          sm.delmask + lane);
    }
    __syncwarp();
    for (int i = lane; i < rows * NP; i += 32) {
      const int r = i / NP;
      kopt_pair_entry<K, kSpan>(sm, r, i - r * NP, xy, dist_type);
    }
    __syncwarp();
    if (S.costs != nullptr) {
      long long* out = reinterpret_cast<long long*>(S.costs + row0 * T);
      for (int j = lane; j < rows * T; j += 32) {
        const int r = j / T, t = j - (j / T) * T;
        int pid[K];
#pragma unroll
        for (int i = 0; i < K; ++i) pid[i] = tpairs[t * K + i];
        __stcs(out + j, static_cast<long long>(kopt_cell<K, kSpan>(sm, r, pid)));
      }
    }
    if (S.improving != nullptr) {
      // the fused leaf consume: templates whose cost is below the row's deleted cost, the ones the
      // reference's consumer tries (src/cpu/kopt_search.cpp:694-715), 32 per ballot
      constexpr int W = (T + 31) / 32;
      for (int r = 0; r < rows; ++r) {
        const int64_t row = row0 + r;
        const long long deleted = __ldcg(reinterpret_cast<const long long*>(S.tasks + row * 12 + 10));
        int first = -1;
        for (int t0 = 0; t0 < T; t0 += 32) {
          const int t = t0 + lane;
          long long v = INT64_MAX;
          if (t < T) {
            int pid[K];
#pragma unroll
            for (int i = 0; i < K; ++i) pid[i] = tpairs[t * K + i];
            v = static_cast<long long>(kopt_cell<K, kSpan>(sm, r, pid));
          }
          const unsigned word = __ballot_sync(kFullMask, t < T && v < deleted);
          if (lane == 0) S.improving[row * W + t0 / 32] = word;
          if (first < 0 && word != 0) first = t0 + __ffs(word) - 1;
        }
        if (lane == 0) S.first[row] = first;
      }
    }
  }
  __syncwarp();
}

// Canonical template pair tables for k = 3, 4, 5 packed back to back (4*3 + 25*4 + 208*5 bytes).
constexpr int kServeTemplateBytes = 4 * 3 + 25 * 4 + 208 * 5;
__host__ __device__ __forceinline__ int serve_template_offset(int k) { return k == 3 ? 0 : (k == 4 ? 12 : 112); }
// After them, the proper templates' validity words by gap pattern (kopt_rows.cuh): word [g][w] of k
// holds bit t mod 32 for template t = 32 w + ... invalid on gap-pattern rows of pattern g; 32 x 1,
// 32 x 1 and 32 x 7 words for k = 3, 4, 5.
constexpr int kServeValidityWords = 32 * (1 + 1 + 7);
static_assert(kServeTemplateBytes % 16 == 0, "validity words start 16-byte aligned");
__host__ __device__ __forceinline__ int serve_validity_offset(int k) { return k == 3 ? 0 : (k == 4 ? 32 : 64); }

// 32 rows [row0, row0 + rows) of a segment, one per lane, with the proper templates compiled in
// (kopt_rows.cuh's row routine at warp size): the k(2k-1) pair distances in registers, each cell k-1
// adds, a validity bit and its store. k = 5 cells go out a box of 16 cells x 32 rows at a time
// through the warp's shared buffer, as whole 128-byte lines of each row with coalesced stores;
// k = 4 and 3 rows are stored from registers. A warp holding a row that is not a gap-pattern row
// scores its rows with the chunked class-code routine instead.
template <int K, int kSpan>
__device__ void kopt_serve_proper32(const ServeJob& job, const ServeSegment& S, int64_t row0, int rows,
                                    const uint32_t* __restrict__ valid, const uint8_t* tpairs,
                                    unsigned char* scratch, int lane, int32_t* error) {
  using Tab = KoptCanonTable<K>;
  constexpr int P = Tab::P, NP = Tab::NP, T = Tab::T, W = Tab::W;
  const bool live = lane < rows;
  const int64_t row = row0 + lane;
  int32_t nd[P];
  int64_t deleted = 0;
  {
    int4 q[3] = {make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0), make_int4(0, 0, 0, 0)};
    if (live) {
      const int4* src = reinterpret_cast<const int4*>(S.tasks + row * 12);
      q[0] = __ldcg(src);
      q[1] = __ldcg(src + 1);
      q[2] = __ldcg(src + 2);
    }
    const int32_t words[12] = {q[0].x, q[0].y, q[0].z, q[0].w, q[1].x, q[1].y, q[1].z, q[1].w,
                               q[2].x, q[2].y, q[2].z, q[2].w};
#pragma unroll
    for (int p = 0; p < P; ++p) {
      nd[p] = words[p];
      if (static_cast<uint32_t>(nd[p]) >= static_cast<uint32_t>(job.g.n)) {
        atomicOr(error, 1);
        nd[p] = 0;
      }
    }
    deleted = static_cast<int64_t>((static_cast<uint64_t>(static_cast<uint32_t>(words[11])) << 32) |
                                   static_cast<uint32_t>(words[10]));
  }
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
    kopt_rows_warp<K, kSpan>(S, row0, row0 + rows, tpairs, job.g.xy, job.g.n, job.g.dist_type, scratch, lane, error);
    return;
  }
  uint32_t d[NP];
  {
    int2 c[P];
    static_for<0, P>([&](auto pc) { c[decltype(pc)::value] = __ldg(job.g.xy + nd[decltype(pc)::value]); });
    static_for<0, P>([&](auto pc) {
      constexpr int p = decltype(pc)::value;
      static_for<p + 1, P>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        d[kopt_pair_index(p, q, P)] = exact_distance<kSpan>(c[p], c[q], job.g.dist_type);
      });
    });
  }
  const uint32_t dl = deleted <= 0 ? 0u : (deleted >= 0xffffffffll ? 0xffffffffu : static_cast<uint32_t>(deleted));
  const uint32_t* vrow = valid + serve_validity_offset(K) + g * W;
  const bool sets = S.improving != nullptr;
  uint32_t valid_word = 0, improving_word = 0;
  int first = -1;
  auto cell = [&](auto tc) -> uint2 {
    constexpr int t = decltype(tc)::value;
    if constexpr (t % 32 == 0) valid_word = __ldg(vrow + t / 32);
    uint32_t sum = d[kKoptCanonPair<K, t, 0>];
    static_for<1, K>([&](auto ic) { sum += d[kKoptCanonPair<K, t, decltype(ic)::value>]; });
    const bool bad = ((valid_word >> (t % 32)) & 1u) != 0;
    improving_word |= static_cast<uint32_t>(!bad && sum < dl) << (t % 32);
    if constexpr (t % 32 == 31 || t == T - 1) {
      if (sets && live) S.improving[row * W + t / 32] = improving_word;
      if (first < 0 && improving_word != 0) first = (t & ~31) + __ffs(improving_word) - 1;
      improving_word = 0;
    }
    return kopt_cell_word(sum, bad);
  };
  if (S.costs == nullptr) {
    static_for<0, T>([&](auto tc) { (void)cell(tc); });
  } else if constexpr (K == 5) {
    const int swz = lane & 7;
    static_for<0, T / 16>([&](auto jc) {
      constexpr int j = decltype(jc)::value;
      __syncwarp();  // the previous box has been read out
      static_for<0, 8>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const uint2 a = cell(std::integral_constant<int, 16 * j + 2 * i>{});
        const uint2 b = cell(std::integral_constant<int, 16 * j + 2 * i + 1>{});
        *reinterpret_cast<uint4*>(scratch + lane * 128 + ((i ^ swz) << 4)) = make_uint4(a.x, a.y, b.x, b.y);
      });
      __syncwarp();
#pragma unroll
      for (int v = 0; v < 8; ++v) {  // 16-byte unit u = lane + 32 v: part u & 7 of row u >> 3
        const int u = lane + 32 * v, r = u >> 3, part = u & 7;
        if (r < rows) {
          const uint4 x = *reinterpret_cast<const uint4*>(scratch + r * 128 + ((part ^ (r & 7)) << 4));
          __stcs(reinterpret_cast<uint4*>(S.costs + (row0 + r) * T + 16 * j) + part, x);
        }
      }
    });
  } else if constexpr (K == 4) {
    uint2* out = reinterpret_cast<uint2*>(S.costs + row * T);
    static_for<0, T>([&](auto tc) {
      const uint2 v = cell(tc);
      if (live) __stcs(out + decltype(tc)::value, v);
    });
  } else {
    uint2 v[T];
    static_for<0, T>([&](auto tc) { v[decltype(tc)::value] = cell(tc); });
    if (live) {
      uint4* out = reinterpret_cast<uint4*>(S.costs + row * T);
      __stcs(out, make_uint4(v[0].x, v[0].y, v[1].x, v[1].y));
      __stcs(out + 1, make_uint4(v[2].x, v[2].y, v[3].x, v[3].y));
    }
  }
  if (sets && live) S.first[row] = first;
  __syncwarp();
}

__device__ __forceinline__ uint32_t volatile_load(const uint32_t* p) { return *reinterpret_cast<const volatile uint32_t*>(p); }
__device__ __forceinline__ unsigned long long volatile_load(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}

// Copies slot `slot`'s descriptor into `out` (all lanes) and returns true when it is the
// published, complete descriptor: state read before and after the copy (with fences) equals the
// copy's generation. The dispatcher warp unpublishes a slot (state = 0) before rewriting its
// descriptor and republishes it after, with fences between the steps (serve_install), so a torn copy
// always fails this check.
__device__ __forceinline__ bool serve_read_job(const ServeControl* ctl, int slot, ServeJob& out, int lane) {
  const uint32_t s1 = volatile_load(&ctl->state[slot]);
  __threadfence();
  constexpr int kWords = static_cast<int>(sizeof(ServeJob) / 4);
  const volatile uint32_t* src = reinterpret_cast<const volatile uint32_t*>(&ctl->jobs[slot]);
  uint32_t* dst = reinterpret_cast<uint32_t*>(&out);
  for (int i = lane; i < kWords; i += 32) dst[i] = src[i];
  __threadfence();
  const uint32_t s2 = volatile_load(&ctl->state[slot]);
  __syncwarp();
  return s1 != 0 && s1 == s2 && out.generation == s1;
}

// One atomicAdd on the slot's ticket (lane 0); returns the ticket value on every lane.
__device__ __forceinline__ unsigned long long serve_take(ServeControl* ctl, int slot, int lane) {
  unsigned long long t = 0;
  if (lane == 0) t = atomicAdd(&ctl->ticket[slot], 1ull);
  return __shfl_sync(kFullMask, t, 0);
}

__device__ __forceinline__ uint32_t acquire_load_sys(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Installs the job posted in `slot` with generation `gen` (all lanes): the descriptor is read from
// the mailbox after the posted word (acquire) and checked against `gen`, then written into the
// slot table in seqlock order. Returns false (nothing written) when the mailbox still shows an
// older descriptor or the job's rows have not landed yet; the dispatcher tries again on its next
// pass.
__device__ __forceinline__ bool serve_install(ServeControl* ctl, const ServeMailbox* mb, int slot, uint32_t gen,
                                              int lane) {
  constexpr int kWords = static_cast<int>(sizeof(ServeJob) / 4);
  constexpr int kPerLane = (kWords + 31) / 32;
  static_assert(sizeof(ServeJob) % 4 == 0, "descriptor copied as 32-bit words");
  __threadfence_system();
  const volatile uint32_t* src = reinterpret_cast<const volatile uint32_t*>(&mb->desc[slot]);
  uint32_t w[kPerLane];
#pragma unroll
  for (int j = 0; j < kPerLane; ++j) w[j] = lane + 32 * j < kWords ? src[lane + 32 * j] : 0u;
  if (__shfl_sync(kFullMask, w[0], 0) != gen) return false;  // word 0 is the descriptor's generation
  constexpr int kGateWord = static_cast<int>(offsetof(ServeJob, rows_gate) / 4);
  static_assert(kGateWord < 32, "the gate word is in the first 32 words");
  if (__shfl_sync(kFullMask, w[0], kGateWord) != 0) {
    if (volatile_load(&ctl->rows_ready[slot]) != gen) return false;
    __threadfence();  // the rows before the install that lets workers read them
  }
  if (lane == 0) {
    reinterpret_cast<volatile uint32_t*>(ctl->state)[slot] = 0u;
    reinterpret_cast<volatile int32_t*>(ctl->slot_error)[slot] = 0;
  }
  __threadfence();
  __syncwarp();
  volatile uint32_t* dst = reinterpret_cast<volatile uint32_t*>(&ctl->jobs[slot]);
#pragma unroll
  for (int j = 0; j < kPerLane; ++j) {
    if (lane + 32 * j < kWords) dst[lane + 32 * j] = w[j];
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    atomicExch(&ctl->ticket[slot], static_cast<unsigned long long>(gen) << 32);
    atomicExch(&ctl->done[slot], static_cast<unsigned long long>(gen) << 32);
    __threadfence();
    reinterpret_cast<volatile uint32_t*>(ctl->state)[slot] = gen;
  }
  __syncwarp();
  return true;
}

// The dispatcher warp: installs every posted job whose generation the slot table does not hold
// yet. It stays while any installed job has unclaimed items or it installed a job within
// `idle_limit` passes (about 2 us each: a PCIe read of the posted words and a 1 us sleep), or until
// the stop word. A post it cannot install yet (rows not landed) counts as an idle pass, so the wait
// for it is bounded too: if the warp leaves, the host relaunches the kernel for the waiting job.
__device__ void serve_dispatch(ServeControl* ctl, const ServeMailbox* mb, int32_t slots, long long idle_limit,
                               int lane) {
  long long idle = 0;
  while (idle < idle_limit) {
    if (volatile_load(&ctl->stop) != 0) return;
    bool active = false;
    for (int base = 0; base < slots; base += 32) {
      const int s = base + lane;
      uint32_t posted = 0, cur = 0;
      bool open = false;
      if (s < slots) {
        posted = acquire_load_sys(&mb->posted[s]);
        cur = volatile_load(&ctl->state[s]);
        if (cur != 0) {
          const unsigned long long t = volatile_load(&ctl->ticket[s]);
          open = static_cast<uint32_t>(t >> 32) == cur && static_cast<uint32_t>(t) < volatile_load(&ctl->jobs[s].items);
        }
      }
      unsigned fresh = __ballot_sync(kFullMask, posted != 0 && posted != cur);
      active = active || __any_sync(kFullMask, open);
      while (fresh != 0) {
        const int b = __ffs(fresh) - 1;
        fresh &= fresh - 1;
        if (serve_install(ctl, mb, base + b, __shfl_sync(kFullMask, posted, b), lane)) active = true;
      }
    }
    if (active) {
      idle = 0;
    } else {
      ++idle;
      __nanosleep(1000);
    }
  }
}

// Rows [r0, r1) of a segment: the proper-template row routine 32 rows at a time (coordinates of span
// < 2^26), else the chunked class-code routine.
template <int K>
__device__ __forceinline__ void serve_kopt_item(const ServeJob& job, const ServeSegment& S, int64_t r0, int64_t r1,
                                                const uint8_t* tpairs, const uint32_t* valid, unsigned char* scratch,
                                                int lane, int32_t* error) {
  if (job.span == kSpanWide) {
    kopt_rows_warp<K, kSpanWide>(S, r0, r1, tpairs, job.g.xy, job.g.n, job.g.dist_type, scratch, lane, error);
    return;
  }
  for (int64_t g0 = r0; g0 < r1; g0 += 32) {
    const int rows = static_cast<int>(min(static_cast<int64_t>(32), r1 - g0));
    if (job.span == kSpanSmall) {
      kopt_serve_proper32<K, kSpanSmall>(job, S, g0, rows, valid, tpairs, scratch, lane, error);
    } else {
      kopt_serve_proper32<K, kSpanNarrow>(job, S, g0, rows, valid, tpairs, scratch, lane, error);
    }
  }
}

// Four blocks per SM (64 registers): JV items want the warps; the k-opt row routine spills some of its
// 45 pair distances at this budget, and 3 or 2 blocks (80 / 128 registers) measured no faster for
// k-opt jobs, whose results are bound by the PCIe download, and slower for JV jobs.
static __global__ void __launch_bounds__(kServeWarps * 32, 4)
    serve_kernel(ServeControl* ctl, const ServeMailbox* mailbox, uint32_t* finished, const uint8_t* templates,
                 int32_t slots, long long idle_limit) {
  __shared__ JvWarpScratch jv_scratch[kServeWarps];
  __shared__ __align__(16) unsigned char kopt_scratch[kServeWarps][kServeKoptScratch];
  __shared__ ServeJob job_copy[kServeWarps];
  __shared__ uint8_t tpairs[kServeTemplateBytes];
  for (int i = threadIdx.x; i < kServeTemplateBytes; i += blockDim.x) tpairs[i] = templates[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (blockIdx.x == 0 && warp == kServeWarps - 1) {  // no block-wide barrier follows
    serve_dispatch(ctl, mailbox, slots, idle_limit, lane);
    return;
  }
  ServeJob& job = job_copy[warp];
  int held = -1;  // slot whose descriptor `job` holds
  long long idle = 0;
  while (idle < idle_limit) {
    if (volatile_load(&ctl->stop) != 0) break;
    int slot = held;
    if (held < 0) {
      // the oldest published job with items left
      uint32_t best_gen = 0xffffffffu;
      int best_slot = -1;
      for (int s = lane; s < slots; s += 32) {
        const uint32_t gen = volatile_load(&ctl->state[s]);
        if (gen == 0 || gen >= best_gen) continue;
        const unsigned long long t = volatile_load(&ctl->ticket[s]);
        if (static_cast<uint32_t>(t >> 32) == gen && static_cast<uint32_t>(t) < volatile_load(&ctl->jobs[s].items)) {
          best_gen = gen;
          best_slot = s;
        }
      }
      const uint32_t oldest = __reduce_min_sync(kFullMask, best_gen);
      const unsigned owner = __ballot_sync(kFullMask, best_slot >= 0 && best_gen == oldest);
      if (owner == 0) {
        ++idle;
        __nanosleep(2000);
        continue;
      }
      slot = __shfl_sync(kFullMask, best_slot, __ffs(owner) - 1);
      if (!serve_read_job(ctl, slot, job, lane)) {  // torn by a concurrent publication: rescan
        ++idle;
        continue;
      }
      held = slot;
    }
    const unsigned long long t = serve_take(ctl, slot, lane);
    const uint32_t gen = static_cast<uint32_t>(t >> 32);
    const uint32_t index = static_cast<uint32_t>(t);
    if (gen != job.generation) {
      // the slot was republished after this warp read it: the claimed item belongs to the newer
      // job, whose descriptor was written before its ticket (serve_install); read it, bounded
      bool found = false;
      for (int w = 0; w < kServeDescriptorWaits && !found; ++w) {
        const uint32_t state = __shfl_sync(kFullMask, lane == 0 ? volatile_load(&ctl->state[slot]) : 0u, 0);
        if (state == gen) {
          found = serve_read_job(ctl, slot, job, lane) && job.generation == gen;
        } else if (state != 0) {
          break;  // an even newer job: generation `gen` already finished, so `index` was past its end
        } else {
          __nanosleep(256);
        }
      }
      if (!found) {
        if (lane == 0 && volatile_load(&ctl->state[slot]) == 0) {  // the publication never completed
          atomicOr(&ctl->error, 8);
          __threadfence_system();
          reinterpret_cast<volatile uint32_t*>(finished)[kServeLostWord] = 1u;
        }
        held = -1;
        ++idle;
        continue;
      }
    }
    if (index >= job.items) {  // every item of the held job is taken
      held = -1;
      ++idle;
      continue;
    }
    held = slot;
    idle = 0;
    int32_t* error = &ctl->slot_error[slot];
    const long long local = index;
    if (job.type == kServeJv) {
      const int64_t e0 = local * kServeJvTile;
      const int64_t e1 = min(e0 + kServeJvTile, job.g.m);
      int32_t mine = -1;  // the witness of edge e0 + lane
      for (int64_t e = e0; e < e1; ++e) {
        const int32_t wv =
            job.span == kSpanSmall    ? jv_screen_edge_warp<kSpanSmall, true>(job.g, e, jv_scratch[warp], lane, error)
            : job.span == kSpanNarrow ? jv_screen_edge_warp<kSpanNarrow, true>(job.g, e, jv_scratch[warp], lane, error)
                                      : jv_screen_edge_warp<kSpanWide, true>(job.g, e, jv_scratch[warp], lane, error);
        const int32_t w0 = __shfl_sync(kFullMask, wv, 0);
        if (lane == static_cast<int>(e - e0)) mine = w0;
        __syncwarp();
      }
      if (e0 + lane < e1) job.witness[e0 + lane] = mine;  // one 128-byte store per item
    } else {
      int si = 0;
      while (si + 1 < job.segments && local >= job.seg[si + 1].item_begin) ++si;
      const ServeSegment& S = job.seg[si];
      const int64_t r0 = (local - S.item_begin) * kServeKoptRowsPerItem;
      const int64_t r1 = min(r0 + kServeKoptRowsPerItem, S.rows);
      const uint8_t* tp = tpairs + serve_template_offset(S.k);
      unsigned char* ks = kopt_scratch[warp];
      const uint32_t* valid = reinterpret_cast<const uint32_t*>(templates + kServeTemplateBytes);
      if (S.k == 3) {
        serve_kopt_item<3>(job, S, r0, r1, tp, valid, ks, lane, error);
      } else if (S.k == 4) {
        serve_kopt_item<4>(job, S, r0, r1, tp, valid, ks, lane, error);
      } else {
        serve_kopt_item<5>(job, S, r0, r1, tp, valid, ks, lane, error);
      }
    }
    // this warp's outputs before its done count (a release at GPU scope). Outputs in page-locked host
    // memory need no system-scope fence here: the warp finishing the job acquires every done count
    // and then releases at system scope (fence + finished word), and causality order is transitive
    // across those synchronizations, so the host that acquires the finished word sees every warp's
    // writes.
    __threadfence();
    __syncwarp();
    if (lane == 0) {
      const unsigned long long d = atomicAdd(&ctl->done[slot], 1ull);
      // the job's last item: finished[kServeMaxSlots + slot] = the job's error word, then
      // finished[slot] = generation
      if (static_cast<uint32_t>(d >> 32) == job.generation && static_cast<uint32_t>(d) + 1 == job.items) {
        __threadfence_system();
        reinterpret_cast<volatile uint32_t*>(finished)[kServeMaxSlots + slot] =
            volatile_load(reinterpret_cast<uint32_t*>(&ctl->slot_error[slot]));
        __threadfence_system();
        reinterpret_cast<volatile uint32_t*>(finished)[slot] = job.generation;
      }
    }
    __syncwarp();
  }
}

}  // namespace cee
