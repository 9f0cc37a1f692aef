// Device-resident JV elimination to a fixed point: every epoch (screen, commit gate, CSR
// compaction) runs on the GPU; the host only reads two counters per epoch.
//
// Semantics follow RunJvElimination's epoch loop (src/cpu/jv_elimination.cpp:250-322) with the
// commit of CommitVerifiedCandidates (src/cpu/elimination_commit.cpp:13-76) and the CSR rebuild of
// GraphSnapshot::RebuildCsr (src/common/graph.cpp:230-282):
//   epoch: screen every active edge; candidates = edges with a witness, in (u, v) order; walk the
//   candidates in that order and commit one when both endpoints still have degree > 2 (then
//   decrement both); deactivate the committed edges and rebuild the CSR; stop after an epoch that
//   commits nothing or after max_rounds epochs.
//
// The walk is sequential in the reference. Here it runs in rounds: a candidate is decided once it
// is the first undecided candidate at both of its endpoints (per-node atomicMin over the undecided
// candidates' indices), which makes every decision see exactly the degrees the sequential walk
// would; the globally first undecided candidate is always decidable, so rounds <= candidates.
// Candidate order comes from a (u, v) ranking of the edges computed once on the host (edges must be
// unique undirected pairs, as the reference's edge files are). Rows of the compacted CSR keep their
// ascending neighbour order, which is the order the reference's rebuild produces.
#include "cee.h"
#include "cee_internal.h"

#include "jv_screen.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>
#include <vector>

namespace cee {

int ValidateView(cee_ctx* ctx, const cee_graph_view* g);

namespace {

constexpr int kScanBlock = 1024;
constexpr int kGateRoundsPerCheck = 8;

// ---- exclusive scan of int32 (three passes) --------------------------------------------------

__device__ __forceinline__ int32_t block_inclusive_scan(int32_t v, int32_t* warp_sums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_inclusive_sum(v, lane);
  if (lane == 31) warp_sums[warp] = v;
  __syncthreads();
  if (warp == 0) {
    int32_t w = lane < static_cast<int>(blockDim.x >> 5) ? warp_sums[lane] : 0;
    w = warp_inclusive_sum(w, lane);
    warp_sums[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += warp_sums[warp - 1];
  return v;
}

static __global__ void __launch_bounds__(kScanBlock) scan_blocks(const int32_t* __restrict__ in, int64_t count,
                                                                 int32_t* __restrict__ out, int32_t* __restrict__ sums) {
  __shared__ int32_t warp_sums[32];
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kScanBlock + threadIdx.x;
  const int32_t v = i < count ? in[i] : 0;
  const int32_t incl = block_inclusive_scan(v, warp_sums);
  if (i < count) out[i] = incl - v;
  if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = incl;
}

// Exclusive scan of the block sums in one block; sums[blocks] receives the total.
static __global__ void __launch_bounds__(kScanBlock) scan_sums(int32_t* __restrict__ sums, int32_t blocks) {
  __shared__ int32_t warp_sums[32];
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int32_t base = 0; base < blocks; base += kScanBlock) {
    const int32_t i = base + threadIdx.x;
    const int32_t v = i < blocks ? sums[i] : 0;
    const int32_t incl = block_inclusive_scan(v, warp_sums);
    const int32_t c = carry;
    __syncthreads();
    if (i < blocks) sums[i] = c + incl - v;
    if (threadIdx.x == kScanBlock - 1) carry = c + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blocks] = carry;
}

static __global__ void scan_add(int32_t* __restrict__ out, int64_t count, const int32_t* __restrict__ sums) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * kScanBlock + threadIdx.x;
  if (i < count) out[i] += sums[blockIdx.x];
}

// ---- epoch kernels ---------------------------------------------------------------------------

// JV screen of every edge with one 16-byte load per CSR slot.
template <int kSpan>
static __global__ void __launch_bounds__(kJvWarpsPerBlock * 32)
    epoch_screen(JvGraph g, int32_t* __restrict__ witness, int32_t* __restrict__ error) {
  __shared__ JvWarpScratch scratch[kJvWarpsPerBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kJvWarpsPerBlock;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * kJvWarpsPerBlock + warp; e < g.m; e += warps) {
    const int32_t w = jv_screen_edge_warp<kSpan, true>(g, e, scratch[warp], lane, error);
    if (lane == 0) witness[e] = w;
    __syncwarp();
  }
}

// slot4[s] = {nbr[s], edge_w[ids[s]], xy[nbr[s]]}; bad ids or neighbours are recorded and read as zeros.
static __global__ void epoch_slots(const int32_t* __restrict__ ids, const int32_t* __restrict__ nbr,
                                   const int2* __restrict__ xy, const int32_t* __restrict__ w32, int64_t count,
                                   int64_t m, int32_t n, int4* __restrict__ slot4, int32_t* __restrict__ error) {
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < count;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = ids[s], c = nbr[s];
    const bool id_ok = static_cast<uint64_t>(static_cast<uint32_t>(id)) < static_cast<uint64_t>(m);
    const bool c_ok = static_cast<uint32_t>(c) < static_cast<uint32_t>(n);
    if (!id_ok || !c_ok) atomicOr(error, 2);
    const int2 p = c_ok ? xy[c] : make_int2(0, 0);
    slot4[s] = make_int4(c_ok ? c : 0, id_ok ? __ldg(w32 + id) : 0, p.x, p.y);
  }
}

// flag[i] = 1 when edge order[i] has a witness.
static __global__ void epoch_flags(const int32_t* __restrict__ order, int64_t m, const int32_t* __restrict__ witness,
                                   int32_t* __restrict__ flag) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    flag[i] = witness[order[i]] >= 0 ? 1 : 0;
  }
}

// cand[pos[i]] = order[i] for flagged i: the candidates in (u, v) order; resets their state.
static __global__ void epoch_fill(const int32_t* __restrict__ order, const int32_t* __restrict__ flag,
                                  const int32_t* __restrict__ pos, int64_t m, int32_t* __restrict__ cand,
                                  uint8_t* __restrict__ decided, uint8_t* __restrict__ commit) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (flag[i] != 0) {
      const int32_t p = pos[i];
      cand[p] = order[i];
      decided[p] = 0;
      commit[p] = 0;
    }
  }
}

// Round part 1: every undecided candidate offers its index to both endpoints.
static __global__ void gate_offer(const int32_t* __restrict__ cand, int32_t count, const int2* __restrict__ uv,
                                  const uint8_t* __restrict__ decided, int32_t* __restrict__ node_min) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    if (decided[i] != 0) continue;
    const int2 e = uv[cand[i]];
    atomicMin(node_min + e.x, i);
    atomicMin(node_min + e.y, i);
  }
}

// Round part 2: a candidate first at both endpoints is decided with the degrees the sequential
// walk would see (no other candidate of this round touches its endpoints).
static __global__ void gate_decide(const int32_t* __restrict__ cand, int32_t count, const int2* __restrict__ uv,
                                   const int32_t* __restrict__ node_min, uint8_t* __restrict__ decided,
                                   uint8_t* __restrict__ commit, int32_t* __restrict__ degree,
                                   int32_t* __restrict__ undecided) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    if (decided[i] != 0) continue;
    const int2 e = uv[cand[i]];
    if (node_min[e.x] == i && node_min[e.y] == i) {
      const bool ok = degree[e.x] > 2 && degree[e.y] > 2;
      if (ok) {
        degree[e.x] -= 1;
        degree[e.y] -= 1;
      }
      commit[i] = ok ? 1 : 0;
      decided[i] = 1;
    } else {
      atomicAdd(undecided, 1);
    }
  }
}

// Round part 3: clear the offers for the next round.
static __global__ void gate_clear(const int32_t* __restrict__ cand, int32_t count, const int2* __restrict__ uv,
                                  int32_t* __restrict__ node_min) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int2 e = uv[cand[i]];
    node_min[e.x] = INT32_MAX;
    node_min[e.y] = INT32_MAX;
  }
}

// Deactivates the committed candidates and records their epoch and witness.
static __global__ void epoch_apply(const int32_t* __restrict__ cand, int32_t count, const uint8_t* __restrict__ commit,
                                   const int32_t* __restrict__ witness, int32_t epoch, uint8_t* __restrict__ active,
                                   int32_t* __restrict__ epoch_of, int32_t* __restrict__ witness_of,
                                   int32_t* __restrict__ committed) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    if (commit[i] == 0) continue;
    const int32_t e = cand[i];
    active[e] = 0;
    epoch_of[e] = epoch;
    witness_of[e] = witness[e];
    atomicAdd(committed, 1);
  }
}

// New row lengths: the slots whose edge is still active.
static __global__ void csr_count(const int32_t* __restrict__ ro, int32_t n, const int32_t* __restrict__ ids,
                                 const uint8_t* __restrict__ active, int32_t* __restrict__ len) {
  for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    int32_t c = 0;
    for (int32_t s = ro[v]; s < ro[v + 1]; ++s) c += active[ids[s]] != 0 ? 1 : 0;
    len[v] = c;
  }
}

// Copies the kept slots of every row, in order, to the new CSR.
static __global__ void csr_fill(const int32_t* __restrict__ ro, int32_t n, const int32_t* __restrict__ new_ro,
                                const int32_t* __restrict__ ids, const int32_t* __restrict__ nbr,
                                const int4* __restrict__ slot4, const uint8_t* __restrict__ active,
                                int32_t* __restrict__ ids2, int32_t* __restrict__ nbr2, int4* __restrict__ slot42) {
  for (int32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    int32_t j = new_ro[v];
    for (int32_t s = ro[v]; s < ro[v + 1]; ++s) {
      const int32_t id = ids[s];
      if (active[id] == 0) continue;
      ids2[j] = id;
      nbr2[j] = nbr[s];
      slot42[j] = slot4[s];
      ++j;
    }
  }
}

}  // namespace

struct EpochState {
  DevBuf xy, uv, w32, active, ro[2], nbr[2], ids[2], slot4[2], order, witness, flag, pos, sums, cand, decided, commit,
      node_min, degree, epoch_of, witness_of, counters;
  // per epoch of the last call: candidates found, wall time of the screen and commit gate
  std::vector<int64_t> proposed;
  std::vector<double> screen_ms;
  bool ran = false;
  void Release() {
    for (DevBuf* b : {&xy, &uv, &w32, &active, &order, &witness, &flag, &pos, &sums, &cand, &decided, &commit, &node_min,
                      &degree, &epoch_of, &witness_of, &counters}) {
      b->Release();
    }
    for (int i = 0; i < 2; ++i) {
      ro[i].Release();
      nbr[i].Release();
      ids[i].Release();
      slot4[i].Release();
    }
  }
};

namespace {

// Exclusive scan of `count` int32 values; the total lands in sums[blocks].
cudaError_t Scan(EpochState& s, const int32_t* in, int32_t* out, int64_t count, cudaStream_t st, int32_t** total) {
  const int32_t blocks = static_cast<int32_t>(std::max<int64_t>(1, (count + kScanBlock - 1) / kScanBlock));
  int32_t* sums = static_cast<int32_t*>(s.sums.ptr);
  scan_blocks<<<blocks, kScanBlock, 0, st>>>(in, count, out, sums);
  scan_sums<<<1, kScanBlock, 0, st>>>(sums, blocks);
  scan_add<<<blocks, kScanBlock, 0, st>>>(out, count, sums);
  *total = sums + blocks;
  return cudaGetLastError();
}

}  // namespace

void ReleaseEpoch(cee_ctx* ctx) {
  if (ctx->epoch == nullptr) return;
  ctx->epoch->Release();
  delete ctx->epoch;
  ctx->epoch = nullptr;
}

uint64_t EpochResident(const cee_ctx* ctx) {
  const EpochState* s = ctx->epoch;
  if (s == nullptr) return 0;
  uint64_t bytes = 0;
  for (const DevBuf* b : {&s->xy, &s->uv, &s->w32, &s->active, &s->order, &s->witness, &s->flag, &s->pos, &s->sums,
                          &s->cand, &s->decided, &s->commit, &s->node_min, &s->degree, &s->epoch_of, &s->witness_of,
                          &s->counters}) {
    bytes += b->capacity;
  }
  for (int i = 0; i < 2; ++i) {
    bytes += s->ro[i].capacity + s->nbr[i].capacity + s->ids[i].capacity + s->slot4[i].capacity;
  }
  return bytes;
}

}  // namespace cee

using namespace cee;

extern "C" int cee_jv_eliminate(cee_ctx* ctx, const cee_graph_view* g, uint32_t max_rounds, uint8_t* active_out,
                                int32_t* witness_out, int32_t* epoch_out, int64_t* epoch_edges_before,
                                int64_t* epoch_committed, cee_jv_elim_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (stats != nullptr) *stats = cee_jv_elim_stats{};
  rc = ValidateView(ctx, g);
  if (rc != CEE_OK) return rc;
  if (max_rounds == 0) return Fail(ctx, CEE_ERR_INVALID, "max_rounds must be greater than 0");
  const int64_t m = g->m;
  const int32_t n = g->n;
  if (m > 0 && (active_out == nullptr || witness_out == nullptr || epoch_out == nullptr)) {
    return Fail(ctx, CEE_ERR_INVALID, "null output arrays");
  }
  const auto t_start = std::chrono::steady_clock::now();
  // commit order: edge ids by (u, v); the edges must be unique undirected pairs
  std::vector<int32_t> order(static_cast<size_t>(m));
  std::iota(order.begin(), order.end(), 0);
  for (int64_t e = 0; e < m; ++e) {
    if (g->edge_u[e] < 0 || g->edge_v[e] < 0 || g->edge_u[e] >= n || g->edge_v[e] >= n || g->edge_u[e] >= g->edge_v[e]) {
      return Fail(ctx, CEE_ERR_INVALID, "edges must be canonical (u < v) and in range");
    }
    if (g->edge_w[e] < 0 || g->edge_w[e] > INT32_MAX) return Fail(ctx, CEE_ERR_RANGE, "edge weight outside [0, 2^31)");
  }
  std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return g->edge_u[a] != g->edge_u[b] ? g->edge_u[a] < g->edge_u[b] : g->edge_v[a] < g->edge_v[b];
  });
  for (int64_t i = 1; i < m; ++i) {
    if (g->edge_u[order[i]] == g->edge_u[order[i - 1]] && g->edge_v[order[i]] == g->edge_v[order[i - 1]]) {
      return Fail(ctx, CEE_ERR_INVALID, "duplicate undirected edge");
    }
  }
  std::vector<int2> xy;
  int span = kSpanSmall;
  rc = PackCoordinates(ctx, n, g->x, g->y, &xy, &span);
  if (rc != CEE_OK) return rc;
  std::vector<int2> uv(static_cast<size_t>(m));
  std::vector<int32_t> w32(static_cast<size_t>(m)), degree(static_cast<size_t>(n));
  for (int64_t e = 0; e < m; ++e) {
    uv[e] = make_int2(g->edge_u[e], g->edge_v[e]);
    w32[e] = static_cast<int32_t>(g->edge_w[e]);
  }
  const int64_t adj = m > 0 ? g->adjacency : 0;
  for (int32_t v = 0; v < n; ++v) degree[v] = m > 0 ? g->row_offsets[v + 1] - g->row_offsets[v] : 0;
  int64_t active_edges = 0;
  for (int64_t e = 0; e < m; ++e) active_edges += g->active[e] != 0 ? 1 : 0;

  if (ctx->epoch == nullptr) ctx->epoch = new EpochState();
  EpochState& s = *ctx->epoch;
  s.ran = false;
  s.proposed.clear();
  s.screen_ms.clear();
  const size_t mm = static_cast<size_t>(std::max<int64_t>(m, 1)), nn = static_cast<size_t>(std::max<int32_t>(n, 1));
  const size_t aa = static_cast<size_t>(std::max<int64_t>(adj, 1));
  const size_t scan_blocks_max = (std::max(mm, nn + 1) + kScanBlock - 1) / kScanBlock + 2;
  cudaError_t status = cudaSuccess;
  for (auto [buf, bytes] : std::initializer_list<std::pair<DevBuf*, size_t>>{
           {&s.xy, nn * 8}, {&s.uv, mm * 8}, {&s.w32, mm * 4}, {&s.active, mm}, {&s.ro[0], (nn + 1) * 4},
           {&s.ro[1], (nn + 1) * 4}, {&s.nbr[0], aa * 4}, {&s.nbr[1], aa * 4}, {&s.ids[0], aa * 4}, {&s.ids[1], aa * 4},
           {&s.slot4[0], aa * 16}, {&s.slot4[1], aa * 16}, {&s.order, mm * 4}, {&s.witness, mm * 4},
           {&s.flag, std::max(mm, nn + 1) * 4}, {&s.pos, std::max(mm, nn + 1) * 4}, {&s.sums, scan_blocks_max * 4}, {&s.cand, mm * 4},
           {&s.decided, mm}, {&s.commit, mm}, {&s.node_min, nn * 4}, {&s.degree, nn * 4}, {&s.epoch_of, mm * 4},
           {&s.witness_of, mm * 4}, {&s.counters, 64}}) {
    if (status == cudaSuccess) status = buf->Reserve(bytes, nullptr);
  }
  if (status != cudaSuccess) return CudaFail(ctx, status, "epoch workspace allocation");
  cudaStream_t st = ctx->stream;
  if (n > 0) cudaMemcpyAsync(s.xy.ptr, xy.data(), static_cast<size_t>(n) * 8, cudaMemcpyHostToDevice, st);
  if (m > 0) {
    cudaMemcpyAsync(s.uv.ptr, uv.data(), mm * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.w32.ptr, w32.data(), mm * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.active.ptr, g->active, mm, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.order.ptr, order.data(), mm * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.ro[0].ptr, g->row_offsets, (static_cast<size_t>(n) + 1) * 4, cudaMemcpyHostToDevice, st);
    if (adj > 0) {
      cudaMemcpyAsync(s.nbr[0].ptr, g->neighbors, static_cast<size_t>(adj) * 4, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(s.ids[0].ptr, g->csr_edge_ids, static_cast<size_t>(adj) * 4, cudaMemcpyHostToDevice, st);
    }
    cudaMemsetAsync(s.epoch_of.ptr, 0xff, mm * 4, st);
    cudaMemsetAsync(s.witness_of.ptr, 0xff, mm * 4, st);
  }
  if (n > 0) {
    cudaMemcpyAsync(s.degree.ptr, degree.data(), static_cast<size_t>(n) * 4, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(s.node_min.ptr, 0x7f, static_cast<size_t>(n) * 4, st);  // 0x7f7f7f7f: above any index
  }
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), st);
  const int grid = ctx->sm_count * 8;
  if (adj > 0) {
    epoch_slots<<<GridFor(adj, 256, grid), 256, 0, st>>>(
        static_cast<const int32_t*>(s.ids[0].ptr), static_cast<const int32_t*>(s.nbr[0].ptr),
        static_cast<const int2*>(s.xy.ptr), static_cast<const int32_t*>(s.w32.ptr), adj, m, n,
        static_cast<int4*>(s.slot4[0].ptr), ctx->d_error);
  }
  int occ = 1;
  WithSpan(span, [&](auto S) {
    status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, epoch_screen<S.value>, kJvWarpsPerBlock * 32, 0);
  });
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "epoch occupancy"));
  const int screen_blocks = GridFor(m, kJvWarpsPerBlock, ctx->sm_count * std::max(1, occ));
  int32_t* counters = static_cast<int32_t*>(s.counters.ptr);  // [0] committed, [1] undecided
  int cur = 0;
  uint32_t epochs = 0;
  int64_t total_committed = 0;
  int32_t host[2] = {0, 0};
  if (m == 0) {  // one epoch that commits nothing, as the reference's loop reports
    if (epoch_edges_before != nullptr) epoch_edges_before[0] = 0;
    if (epoch_committed != nullptr) epoch_committed[0] = 0;
    epochs = 1;
    s.proposed.push_back(0);
    s.screen_ms.push_back(0.0);
  }
  for (uint32_t epoch = 0; epoch < max_rounds && m > 0; ++epoch) {
    const auto epoch_start = std::chrono::steady_clock::now();
    JvGraph jg{};
    jg.n = n;
    jg.dist_type = g->dist_type;
    jg.m = m;
    jg.xy = static_cast<const int2*>(s.xy.ptr);
    jg.edge_uv = static_cast<const int2*>(s.uv.ptr);
    jg.edge_w = static_cast<const int32_t*>(s.w32.ptr);
    jg.active = static_cast<const uint8_t*>(s.active.ptr);
    jg.row_offsets = static_cast<const int32_t*>(s.ro[cur].ptr);
    jg.nbr = static_cast<const int32_t*>(s.nbr[cur].ptr);
    jg.slot4 = static_cast<const int4*>(s.slot4[cur].ptr);
    int32_t* witness = static_cast<int32_t*>(s.witness.ptr);
    WithSpan(span, [&](auto S) {
      epoch_screen<S.value><<<screen_blocks, kJvWarpsPerBlock * 32, 0, st>>>(jg, witness, ctx->d_error);
    });
    // candidates in (u, v) order
    epoch_flags<<<GridFor(m, 256, grid), 256, 0, st>>>(static_cast<const int32_t*>(s.order.ptr), m, witness,
                                                          static_cast<int32_t*>(s.flag.ptr));
    int32_t* total = nullptr;
    status = Scan(s, static_cast<const int32_t*>(s.flag.ptr), static_cast<int32_t*>(s.pos.ptr), m, st, &total);
    if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "epoch scan"));
    epoch_fill<<<GridFor(m, 256, grid), 256, 0, st>>>(
        static_cast<const int32_t*>(s.order.ptr), static_cast<const int32_t*>(s.flag.ptr),
        static_cast<const int32_t*>(s.pos.ptr), m, static_cast<int32_t*>(s.cand.ptr),
        static_cast<uint8_t*>(s.decided.ptr), static_cast<uint8_t*>(s.commit.ptr));
    int32_t candidates = 0;
    cudaMemcpyAsync(&candidates, total, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    status = cudaStreamSynchronize(st);
    if (status != cudaSuccess) return CudaFail(ctx, status, "epoch screen");
    if (epoch_edges_before != nullptr) epoch_edges_before[epoch] = active_edges;
    ++epochs;
    int32_t committed = 0;
    if (candidates > 0) {
      // commit gate in rounds
      const int gate_grid = GridFor(candidates, 256, grid);
      const int2* duv = static_cast<const int2*>(s.uv.ptr);
      const int32_t* cand = static_cast<const int32_t*>(s.cand.ptr);
      uint8_t* decided = static_cast<uint8_t*>(s.decided.ptr);
      uint8_t* commit = static_cast<uint8_t*>(s.commit.ptr);
      int32_t* node_min = static_cast<int32_t*>(s.node_min.ptr);
      int32_t* deg = static_cast<int32_t*>(s.degree.ptr);
      for (int64_t round = 0;;) {
        for (int r = 0; r < kGateRoundsPerCheck; ++r, ++round) {
          cudaMemsetAsync(counters + 1, 0, sizeof(int32_t), st);
          gate_offer<<<gate_grid, 256, 0, st>>>(cand, candidates, duv, decided, node_min);
          gate_decide<<<gate_grid, 256, 0, st>>>(cand, candidates, duv, node_min, decided, commit, deg, counters + 1);
          gate_clear<<<gate_grid, 256, 0, st>>>(cand, candidates, duv, node_min);
        }
        cudaMemcpyAsync(&host[1], counters + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        status = cudaStreamSynchronize(st);
        if (status != cudaSuccess) return CudaFail(ctx, status, "epoch commit gate");
        if (host[1] == 0) break;
        if (round > static_cast<int64_t>(candidates) + kGateRoundsPerCheck) {
          return Fail(ctx, CEE_ERR_STATE, "commit gate did not converge");  // each round decides at least one
        }
      }
      cudaMemsetAsync(counters, 0, sizeof(int32_t), st);
      epoch_apply<<<gate_grid, 256, 0, st>>>(cand, candidates, commit, witness, static_cast<int32_t>(epoch),
                                             static_cast<uint8_t*>(s.active.ptr), static_cast<int32_t*>(s.epoch_of.ptr),
                                             static_cast<int32_t*>(s.witness_of.ptr), counters);
      cudaMemcpyAsync(&host[0], counters, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
      status = cudaStreamSynchronize(st);
      if (status != cudaSuccess) return CudaFail(ctx, status, "epoch apply");
      committed = host[0];
    }
    if (epoch_committed != nullptr) epoch_committed[epoch] = committed;
    s.proposed.push_back(candidates);
    s.screen_ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - epoch_start).count());
    total_committed += committed;
    active_edges -= committed;
    if (committed == 0) break;
    // CSR compaction into the other buffer set
    const int nxt = 1 - cur;
    int32_t* len = static_cast<int32_t*>(s.flag.ptr);  // n + 1 entries (the flag buffer is free here)
    csr_count<<<GridFor(n, 256, grid), 256, 0, st>>>(static_cast<const int32_t*>(s.ro[cur].ptr), n,
                                                        static_cast<const int32_t*>(s.ids[cur].ptr),
                                                        static_cast<const uint8_t*>(s.active.ptr), len);
    cudaMemsetAsync(len + n, 0, sizeof(int32_t), st);
    status = Scan(s, len, static_cast<int32_t*>(s.ro[nxt].ptr), static_cast<int64_t>(n) + 1, st, &total);
    if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "epoch CSR scan"));
    csr_fill<<<GridFor(n, 256, grid), 256, 0, st>>>(
        static_cast<const int32_t*>(s.ro[cur].ptr), n, static_cast<const int32_t*>(s.ro[nxt].ptr),
        static_cast<const int32_t*>(s.ids[cur].ptr), static_cast<const int32_t*>(s.nbr[cur].ptr),
        static_cast<const int4*>(s.slot4[cur].ptr), static_cast<const uint8_t*>(s.active.ptr),
        static_cast<int32_t*>(s.ids[nxt].ptr), static_cast<int32_t*>(s.nbr[nxt].ptr), static_cast<int4*>(s.slot4[nxt].ptr));
    status = cudaGetLastError();
    if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "epoch CSR compaction"));
    cur = nxt;
  }
  if (m > 0) {
    cudaMemcpyAsync(active_out, s.active.ptr, mm, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(epoch_out, s.epoch_of.ptr, mm * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(witness_out, s.witness_of.ptr, mm * 4, cudaMemcpyDeviceToHost, st);
  }
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  status = cudaStreamSynchronize(st);
  if (status != cudaSuccess) return CudaFail(ctx, status, "epoch results");
  rc = CheckDeviceError(ctx, "JV epoch loop");
  if (rc != CEE_OK) return rc;
  if (stats != nullptr) {
    stats->epochs = static_cast<int32_t>(epochs);
    stats->committed = total_committed;
    stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    stats->resident_bytes = EpochResident(ctx);
  }
  s.ran = true;
  return CEE_OK;
}

extern "C" int cee_jv_eliminate_metrics(const cee_ctx* ctx, int64_t* proposed, double* screen_ms, int32_t capacity) {
  using namespace cee;
  if (ctx == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null context");
  const EpochState* s = ctx->epoch;
  if (s == nullptr || !s->ran) return Fail(nullptr, CEE_ERR_STATE, "cee_jv_eliminate_metrics before cee_jv_eliminate");
  const int32_t epochs = static_cast<int32_t>(s->proposed.size());
  if (capacity < epochs) return Fail(nullptr, CEE_ERR_INVALID, "capacity below the epoch count");
  for (int32_t e = 0; e < epochs; ++e) {
    if (proposed != nullptr) proposed[e] = s->proposed[static_cast<size_t>(e)];
    if (screen_ms != nullptr) screen_ms[e] = s->screen_ms[static_cast<size_t>(e)];
  }
  return CEE_OK;
}
