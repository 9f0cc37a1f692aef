// Batched screen runtime: many instances in one persistent, CUDA-graph-captured launch
// (batch_screen.cuh), the one-launch-per-instance comparison path, the chunked end-to-end call
// with copy/compute overlap, and the launch-shape autotuner. Contract in include/cee.h.
#include "cee.h"
#include "cee_internal.h"

#include "batch_screen.cuh"

#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace cee {

// Runs body(begin, end) over [0, count) split across host threads (one range when small).
template <typename Body>
void ParallelRanges(int64_t count, Body body) {
  const int64_t kMinPerThread = int64_t{1} << 18;
  const int threads = static_cast<int>(std::min<int64_t>(
      std::max(1u, std::min(16u, std::thread::hardware_concurrency())), std::max<int64_t>(1, count / kMinPerThread)));
  if (threads <= 1) {
    body(0, count, 0);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(static_cast<size_t>(threads));
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([=] { body(count * t / threads, count * (t + 1) / threads, t); });
  }
  for (std::thread& th : pool) th.join();
}

constexpr int kMaxChunks = 64;

struct BatchState {
  cee_batch_options opt{};
  cee_batch_tuning tune{64, 0, 8};
  int32_t instances = 0;
  int64_t n = 0, m = 0, adj = 0;
  int32_t dist_type = 0;
  int span = kSpanSmall;  // span class of the union's coordinates
  int32_t flag_words = 0;
  std::vector<int64_t> node_begin, edge_begin;
  std::vector<int64_t> chunk_begin;  // spatial chunks per instance (batch_screen.cuh)
  int spatial_keys = 0;               // padded key count of the largest chunked instance
  bool local = false;                 // every instance has at most kJvLocalSpan nodes
  // the union snapshot in the kernels' layout
  DevBuf d_node_begin, d_edge_begin, xy, uv, w32, active, ro, nbr, ids, slot4, node4, edge4;
  // raw uploads of the end-to-end call (converted on the device)
  DevBuf raw_x, raw_y, raw_v, estart;  // estart[x]: the first edge whose lower end is x or above
  int32_t* stage_host = nullptr;  // pinned int32 staging of the end-to-end call: weights [m], edge starts [n + 1]
  size_t stage_count = 0;
  // outputs and work-queue state
  DevBuf witness, target_ids, target_count, nbhd, flags, counter, ready;
  DevBuf perm, chunk_box, d_chunk_begin;  // spatial chunks of the instances
  DevBuf cand_c, cand_d, cand_product, cand_count;  // finalised c,d candidates (max_cd_candidates > 0)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t h2d = nullptr, d2h = nullptr, prep = nullptr;
  cudaEvent_t up[kMaxChunks] = {}, done[kMaxChunks] = {}, prepped[kMaxChunks] = {};
  int occupancy[kSpanClasses] = {1, 1, 1};  // resident screen blocks per SM, per span class
  bool prepared = false;

  void ReleaseGraph() {
    if (exec != nullptr) cudaGraphExecDestroy(exec);
    if (graph != nullptr) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void Release() {
    ReleaseGraph();
    for (DevBuf* b : {&d_node_begin, &d_edge_begin, &xy, &uv, &w32, &active, &ro, &nbr, &ids, &slot4, &node4, &edge4, &raw_x, &raw_y,
                      &raw_v, &estart, &witness, &target_ids, &target_count, &nbhd, &flags, &counter, &ready,
                      &cand_c, &cand_d, &cand_product, &cand_count, &perm, &chunk_box, &d_chunk_begin}) {
      b->Release();
    }
    for (int i = 0; i < kMaxChunks; ++i) {
      if (up[i] != nullptr) cudaEventDestroy(up[i]);
      if (done[i] != nullptr) cudaEventDestroy(done[i]);
      if (prepped[i] != nullptr) cudaEventDestroy(prepped[i]);
      up[i] = done[i] = prepped[i] = nullptr;
    }
    if (stage_host != nullptr) cudaFreeHost(stage_host);
    stage_host = nullptr;
    stage_count = 0;
    if (h2d != nullptr) cudaStreamDestroy(h2d);
    if (prep != nullptr) cudaStreamDestroy(prep);
    prep = nullptr;
    if (d2h != nullptr) cudaStreamDestroy(d2h);
    h2d = d2h = nullptr;
    prepared = false;
  }
};

void ReleaseBatch(cee_ctx* ctx) {
  if (ctx->batch != nullptr) {
    ctx->batch->Release();
    delete ctx->batch;
    ctx->batch = nullptr;
  }
}

uint64_t BatchResident(const cee_ctx* ctx) {
  const BatchState* s = ctx->batch;
  if (s == nullptr) return 0;
  uint64_t bytes = 0;
  for (const DevBuf* b : {&s->d_node_begin, &s->d_edge_begin, &s->xy, &s->uv, &s->w32, &s->active, &s->ro, &s->nbr,
                          &s->ids, &s->slot4, &s->node4, &s->edge4, &s->raw_x, &s->raw_y, &s->raw_v, &s->estart, &s->witness,
                          &s->target_ids, &s->target_count, &s->nbhd, &s->flags, &s->counter, &s->ready, &s->perm,
                          &s->chunk_box, &s->d_chunk_begin}) {
    bytes += b->capacity;
  }
  return bytes;
}

namespace {

BatchState* State(cee_ctx* ctx) {
  if (ctx->batch == nullptr) ctx->batch = new BatchState();
  return ctx->batch;
}

int ValidateOptions(cee_ctx* ctx, const cee_batch_options* o) {
  if (o == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null batch options");
  if (o->targets < 1 || o->targets > kBatchMaxTargets) return Fail(ctx, CEE_ERR_INVALID, "targets must lie in [1,64]");
  if (o->max_neighborhood < 2 || o->max_neighborhood > kBatchMaxNeighborhood) {
    return Fail(ctx, CEE_ERR_INVALID, "max_neighborhood must lie in [2,32] for the batched screen");
  }
  if (o->max_candidate_degree < 0) return Fail(ctx, CEE_ERR_INVALID, "negative degree cap");
  if (o->cd_mode != CEE_CD_ACTIVE_INCOMPATIBLE && o->cd_mode != CEE_CD_MISSING_OR_INCOMPATIBLE) {
    return Fail(ctx, CEE_ERR_INVALID, "unknown c,d mode");
  }
  if (o->max_cd_candidates < 0 || o->max_cd_candidates > kBatchMaxCd) {
    return Fail(ctx, CEE_ERR_INVALID, "max_cd_candidates must lie in [0,32]");
  }
  return CEE_OK;
}

// Structural checks in O(instances): sizes, instance offsets, the CSR's end points, null arrays.
int ValidateShape(cee_ctx* ctx, const cee_batch_view* b) {
  if (b == nullptr || b->instances < 1 || b->node_begin == nullptr || b->edge_begin == nullptr) {
    return Fail(ctx, CEE_ERR_INVALID, "bad batch description");
  }
  const cee_graph_view& g = b->graph;
  if (g.n < 0 || g.m < 0 || g.m > INT32_MAX || (g.dist_type != CEE_EUC_2D && g.dist_type != CEE_CEIL_2D)) {
    return Fail(ctx, CEE_ERR_INVALID, "bad union snapshot");
  }
  if (b->node_begin[0] != 0 || b->edge_begin[0] != 0 || b->node_begin[b->instances] != g.n ||
      b->edge_begin[b->instances] != g.m) {
    return Fail(ctx, CEE_ERR_INVALID, "instance offsets must cover the union exactly");
  }
  for (int32_t i = 0; i < b->instances; ++i) {
    if (b->node_begin[i + 1] < b->node_begin[i] || b->edge_begin[i + 1] < b->edge_begin[i]) {
      return Fail(ctx, CEE_ERR_INVALID, "instance offsets must be non-decreasing");
    }
  }
  if (g.adjacency < 0 || g.adjacency > INT32_MAX || g.row_offsets == nullptr || g.row_offsets[0] != 0 ||
      g.row_offsets[g.n] != g.adjacency) {
    return Fail(ctx, CEE_ERR_INVALID, "bad union CSR");
  }
  if (g.n > 0 && (g.x == nullptr || g.y == nullptr)) return Fail(ctx, CEE_ERR_INVALID, "null union coordinates");
  if (g.m > 0 && (g.edge_u == nullptr || g.edge_v == nullptr || g.edge_w == nullptr || g.active == nullptr)) {
    return Fail(ctx, CEE_ERR_INVALID, "null union arrays");
  }
  if (g.adjacency > 0 && (g.neighbors == nullptr || g.csr_edge_ids == nullptr)) {
    return Fail(ctx, CEE_ERR_INVALID, "null union CSR arrays");
  }
  return CEE_OK;
}

// The O(n) checks, one pass on host threads: row offsets non-decreasing (so that every row lies
// inside [0, adjacency)) and the coordinate bounding box (box = {min x, max x, min y, max y}).
int ScanNodes(cee_ctx* ctx, const cee_graph_view& g, int64_t box[4]) {
  std::vector<int64_t> part(16 * 4);
  std::vector<uint8_t> bad(16, 0);
  for (int t = 0; t < 16; ++t) {
    part[4 * t] = part[4 * t + 2] = INT64_MAX;
    part[4 * t + 1] = part[4 * t + 3] = INT64_MIN;
  }
  ParallelRanges(g.n, [&](int64_t i0, int64_t i1, int t) {
    int64_t lx = INT64_MAX, hx = INT64_MIN, ly = INT64_MAX, hy = INT64_MIN;
    bool decreasing = false;
    for (int64_t i = i0; i < i1; ++i) {
      decreasing |= g.row_offsets[i + 1] < g.row_offsets[i];
      lx = std::min(lx, g.x[i]);
      hx = std::max(hx, g.x[i]);
      ly = std::min(ly, g.y[i]);
      hy = std::max(hy, g.y[i]);
    }
    bad[t] = decreasing ? 1 : 0;
    part[4 * t] = lx;
    part[4 * t + 1] = hx;
    part[4 * t + 2] = ly;
    part[4 * t + 3] = hy;
  });
  if (std::any_of(bad.begin(), bad.end(), [](uint8_t b) { return b != 0; })) {
    return Fail(ctx, CEE_ERR_INVALID, "row_offsets not non-decreasing");
  }
  box[0] = box[2] = INT64_MAX;
  box[1] = box[3] = INT64_MIN;
  for (int t = 0; t < 16; ++t) {
    box[0] = std::min(box[0], part[4 * t]);
    box[1] = std::max(box[1], part[4 * t + 1]);
    box[2] = std::min(box[2], part[4 * t + 2]);
    box[3] = std::max(box[3], part[4 * t + 3]);
  }
  if (g.n == 0) box[0] = box[1] = box[2] = box[3] = 0;
  if (static_cast<__int128>(box[1]) - box[0] >= (__int128{1} << 30) ||
      static_cast<__int128>(box[3]) - box[2] >= (__int128{1} << 30)) {
    return Fail(ctx, CEE_ERR_RANGE, "coordinate span >= 2^30: outside the exact int32 distance range of the kernels");
  }
  return CEE_OK;
}

int Reserve(cee_ctx* ctx, DevBuf& buf, size_t bytes) {
  const cudaError_t status = buf.Reserve(bytes + 16, nullptr);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch allocation");
  return CEE_OK;
}

int ReserveAll(cee_ctx* ctx, BatchState& s) {
  const size_t I = static_cast<size_t>(s.instances), T = static_cast<size_t>(s.opt.targets);
  const size_t n = static_cast<size_t>(s.n), m = static_cast<size_t>(s.m), adj = static_cast<size_t>(s.adj);
  const size_t NB = static_cast<size_t>(s.opt.max_neighborhood);
  int rc = CEE_OK;
  const std::pair<DevBuf*, size_t> wants[] = {
      {&s.d_node_begin, (I + 1) * 8}, {&s.d_edge_begin, (I + 1) * 8}, {&s.xy, n * 8}, {&s.uv, m * 8},
      {&s.w32, m * 4}, {&s.active, m}, {&s.ro, (n + 1) * 4}, {&s.nbr, adj * 4}, {&s.ids, adj * 4},
      {&s.slot4, adj * 16}, {&s.node4, n * 16}, {&s.edge4, m * 16}, {&s.witness, m * 4}, {&s.target_ids, I * T * 4}, {&s.target_count, I * 4},
      {&s.nbhd, I * T * NB * 4}, {&s.flags, I * T * static_cast<size_t>(s.flag_words) * 4},
      {&s.counter, kMaxChunks * 8}, {&s.ready, I * 4}, {&s.perm, n * 4},
      {&s.chunk_box, static_cast<size_t>(s.chunk_begin.back()) * 16}, {&s.d_chunk_begin, (I + 1) * 8}};
  const size_t K = static_cast<size_t>(s.opt.max_cd_candidates);
  for (const auto& [buf, bytes] : wants) {
    rc = Reserve(ctx, *buf, bytes);
    if (rc != CEE_OK) return rc;
  }
  if (K > 0) {
    const std::pair<DevBuf*, size_t> cands[] = {
        {&s.cand_c, I * T * K * 4}, {&s.cand_d, I * T * K * 4}, {&s.cand_product, I * T * K * 8}, {&s.cand_count, I * T * 4}};
    for (const auto& [buf, bytes] : cands) {
      rc = Reserve(ctx, *buf, bytes);
      if (rc != CEE_OK) return rc;
    }
  }
  return CEE_OK;
}

// Device error word of the batched screen: bounds checks and the bounded wait are malformed-input
// or scheduling errors, the finalisation's range limits are CEE_ERR_RANGE.
int BatchCheck(cee_ctx* ctx) {
  if ((*ctx->h_error & kBatchRangeError) != 0) {
    return Fail(ctx, CEE_ERR_RANGE, "batched c,d finalisation: an instance has more than 65536 nodes or a reply "
                                    "product reached 2^32 - 2");
  }
  return CheckDeviceError(ctx, "batched screen");
}

void SetShape(BatchState& s, const cee_batch_view* b, const cee_batch_options* o) {
  s.opt = *o;
  s.instances = b->instances;
  s.n = b->graph.n;
  s.m = b->graph.m;
  s.adj = b->graph.adjacency;
  s.dist_type = b->graph.dist_type;
  const int pairs = o->max_neighborhood * (o->max_neighborhood - 1) / 2;
  s.flag_words = (pairs + 31) / 32;
  s.node_begin.assign(b->node_begin, b->node_begin + b->instances + 1);
  s.edge_begin.assign(b->edge_begin, b->edge_begin + b->instances + 1);
  s.chunk_begin.assign(static_cast<size_t>(b->instances) + 1, 0);
  s.spatial_keys = 0;
  s.local = true;
  for (int32_t i = 0; i < b->instances; ++i) {
    const int64_t n = b->node_begin[i + 1] - b->node_begin[i];
    s.local = s.local && n <= kJvLocalSpan;
    const int64_t chunks = n <= kSpatialMaxNodes ? (n + kSpatialChunk - 1) / kSpatialChunk : 0;
    s.chunk_begin[i + 1] = s.chunk_begin[i] + chunks;
    if (chunks > 0) {
      int keys = 1;
      while (keys < n) keys <<= 1;
      s.spatial_keys = std::max(s.spatial_keys, keys);
    }
  }
}

BatchArgs MakeArgs(cee_ctx* ctx, BatchState& s, int32_t first, int32_t count, int chunk) {
  BatchArgs A{};
  A.g.n = static_cast<int32_t>(s.n);
  A.g.dist_type = s.dist_type;
  A.g.m = s.m;
  A.g.xy = static_cast<const int2*>(s.xy.ptr);
  A.g.edge_uv = static_cast<const int2*>(s.uv.ptr);
  A.g.edge_w = static_cast<const int32_t*>(s.w32.ptr);
  A.g.active = static_cast<const uint8_t*>(s.active.ptr);
  A.g.row_offsets = static_cast<const int32_t*>(s.ro.ptr);
  A.g.nbr = static_cast<const int32_t*>(s.nbr.ptr);
  A.g.slot_w = nullptr;
  A.g.slot4 = static_cast<const int4*>(s.slot4.ptr);
  A.g.node4 = static_cast<const int4*>(s.node4.ptr);
  A.g.edge4 = static_cast<const int4*>(s.edge4.ptr);
  A.node_begin = static_cast<const int64_t*>(s.d_node_begin.ptr);
  A.edge_begin = static_cast<const int64_t*>(s.d_edge_begin.ptr);
  A.first_instance = first;
  A.instances = count;
  A.targets = s.opt.targets;
  A.nb = s.opt.max_neighborhood;
  A.max_degree = s.opt.max_candidate_degree;
  A.mode = s.opt.cd_mode;
  A.jv_tile = s.tune.jv_tile;
  A.flag_words = s.flag_words;
  A.jv_first = s.edge_begin[first];
  A.jv_last = s.edge_begin[first + count];
  A.jv_items = (A.jv_last - A.jv_first + A.jv_tile - 1) / A.jv_tile;
  A.witness = static_cast<int32_t*>(s.witness.ptr);
  A.target_ids = static_cast<int32_t*>(s.target_ids.ptr);
  A.target_count = static_cast<int32_t*>(s.target_count.ptr);
  A.nbhd = static_cast<int32_t*>(s.nbhd.ptr);
  A.flags = static_cast<uint32_t*>(s.flags.ptr);
  A.max_cd = s.opt.max_cd_candidates;
  A.cand_c = static_cast<int32_t*>(s.cand_c.ptr);
  A.cand_d = static_cast<int32_t*>(s.cand_d.ptr);
  A.cand_product = static_cast<int64_t*>(s.cand_product.ptr);
  A.cand_count = static_cast<int32_t*>(s.cand_count.ptr);
  A.counter = static_cast<unsigned long long*>(s.counter.ptr) + chunk;
  A.ready = static_cast<int32_t*>(s.ready.ptr);
  A.error = ctx->d_error;
  A.wait_limit = 1ll << 24;  // ~1 s of 64 ns naps
  A.perm = static_cast<const int32_t*>(s.perm.ptr);
  A.chunk_box = static_cast<const int4*>(s.chunk_box.ptr);
  A.chunk_begin = static_cast<const int64_t*>(s.d_chunk_begin.ptr);
  return A;
}

// Spatial chunks of instances [first, first + count) (their coordinates must be on the device).
cudaError_t LaunchSpatial(const BatchState& s, int32_t first, int32_t count, cudaStream_t stream) {
  if (count <= 0 || s.spatial_keys == 0) return cudaSuccess;
  const int smem = s.spatial_keys * 4;
  if (smem > 48 * 1024) {
    const cudaError_t status = cudaFuncSetAttribute(batch_spatial, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (status != cudaSuccess) return status;
  }
  batch_spatial<<<count, kSpatialThreads, smem, stream>>>(
      static_cast<const int2*>(s.xy.ptr), static_cast<const int64_t*>(s.d_node_begin.ptr),
      static_cast<const int64_t*>(s.d_chunk_begin.ptr), first, static_cast<int32_t*>(s.perm.ptr),
      static_cast<int4*>(s.chunk_box.ptr));
  return cudaGetLastError();
}

cudaError_t QueryBatchOccupancy(BatchState& s) {
  cudaError_t status = cudaSuccess;
  for (int span = 0; span < kSpanClasses && status == cudaSuccess; ++span) {
    WithSpan(span, [&](auto S) {
      int blocks = 0;
      status = s.local ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, batch_screen_kernel<S.value, true>,
                                                                       kBatchWarps * 32, 0)
                       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, batch_screen_kernel<S.value, false>,
                                                                       kBatchWarps * 32, 0);
      s.occupancy[span] = std::max(1, blocks);
    });
  }
  return status;
}

int Grid(cee_ctx* ctx, const BatchState& s, int64_t items) {
  const int per_sm = std::max(1, std::min(s.tune.blocks_per_sm > 0 ? s.tune.blocks_per_sm : 64,
                                          s.occupancy[s.span]));
  const int64_t want = (items + kBatchWarps - 1) / kBatchWarps;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, static_cast<int64_t>(ctx->sm_count) * per_sm)));
}

int LaunchRange(cee_ctx* ctx, BatchState& s, int32_t first, int32_t count, int chunk, cudaStream_t stream) {
  const BatchArgs A = MakeArgs(ctx, s, first, count, chunk);
  const int64_t items = static_cast<int64_t>(count) * (1 + s.opt.targets) + A.jv_items;
  cudaMemsetAsync(A.counter, 0, sizeof(unsigned long long), stream);
  cudaMemsetAsync(A.ready + first, 0, static_cast<size_t>(count) * 4, stream);
  const int blocks = Grid(ctx, s, items);
  WithSpan(s.span, [&](auto S) {
    if (s.local) {
      batch_screen_kernel<S.value, true><<<blocks, kBatchWarps * 32, 0, stream>>>(A);
    } else {
      batch_screen_kernel<S.value, false><<<blocks, kBatchWarps * 32, 0, stream>>>(A);
    }
  });
  if (A.max_cd > 0) {  // FinalizeCdCandidates for every target of the range
    const int fin_blocks = GridFor(static_cast<int64_t>(count) * s.opt.targets, kBatchWarps, ctx->sm_count * 8);
    WithSpan(s.span, [&](auto S) { batch_finalize_kernel<S.value><<<fin_blocks, kBatchWarps * 32, 0, stream>>>(A); });
  }
  const cudaError_t status = cudaGetLastError();
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch_screen_kernel launch");
  return CEE_OK;
}

int Capture(cee_ctx* ctx, BatchState& s) {
  s.ReleaseGraph();
  cudaError_t status = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch graph capture");
  const int rc = LaunchRange(ctx, s, 0, s.instances, 0, ctx->stream);
  status = cudaStreamEndCapture(ctx->stream, &s.graph);
  if (rc != CEE_OK) return rc;
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch graph capture");
  status = cudaGraphInstantiate(&s.exec, s.graph, 0);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch graph instantiate");
  return CEE_OK;
}

// slot4[s] = {nbr[s], edge_w[ids[s]], xy[nbr[s]]} over slots [s0, s1) (the JV screen's one-load
// view of a CSR slot); bad ids or neighbours are recorded and read as zeros.
__global__ void batch_gather(const int32_t* __restrict__ ids, const int32_t* __restrict__ nbr, const int2* __restrict__ xy,
                             int64_t s0, int64_t s1, const int32_t* __restrict__ w32, int64_t m, int64_t n,
                             int4* __restrict__ slot4, int32_t* __restrict__ error) {
  for (int64_t s = s0 + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < s1;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = ids[s], c = nbr[s];
    const bool id_ok = static_cast<uint64_t>(static_cast<uint32_t>(id)) < static_cast<uint64_t>(m);
    const bool c_ok = static_cast<uint64_t>(static_cast<uint32_t>(c)) < static_cast<uint64_t>(n);
    if (!id_ok || !c_ok) atomicOr(error, 2);
    const int2 p = c_ok ? xy[c] : make_int2(0, 0);
    slot4[s] = make_int4(c_ok ? c : 0, id_ok ? __ldg(w32 + id) : 0, p.x, p.y);
  }
}

// node4[x] = {xy[x], row_offsets[x], row_offsets[x + 1]} over nodes [n0, n1) and edge4[e] =
// {uv[e], w32[e], active[e]} over edges [e0, e1): the batched screen's one-load views of a node
// (coordinates and CSR row) and of an edge (ends, weight, active flag).
__global__ void batch_records(const int2* __restrict__ xy, const int32_t* __restrict__ ro, int64_t n0, int64_t n1,
                              int4* __restrict__ node4, const int2* __restrict__ uv, const int32_t* __restrict__ w32,
                              const uint8_t* __restrict__ active, int64_t e0, int64_t e1, int4* __restrict__ edge4) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int64_t i = n0 + first; i < n1; i += stride) {
    const int2 p = xy[i];
    node4[i] = make_int4(p.x, p.y, ro[i], ro[i + 1]);
  }
  for (int64_t e = e0 + first; e < e1; e += stride) {
    const int2 q = uv[e];
    edge4[e] = make_int4(q.x, q.y, w32[e], active[e]);
  }
}

// Raw host layout -> kernel layout for nodes [n0, n1) and their edges [e0, e1): coordinates relative
// to (min_x, min_y), and each edge's ends (u, v) with u from estart (estart[x], x in [n0, n1], is the
// first edge whose lower end is x or above; the host builds it from the checked, (u, v)-sorted edge
// list). A warp takes 32 consecutive nodes and walks their edges with coalesced loads, finding each
// edge's lower end by a binary search over the lanes' estart values. Out-of-range values are
// recorded in *error and replaced by harmless ones ((0, 0)) so that no later access leaves its array.
__global__ void batch_pack(const int64_t* __restrict__ x, const int64_t* __restrict__ y, int64_t n0, int64_t n1,
                           int64_t min_x, int64_t min_y, int2* __restrict__ xy, const int32_t* __restrict__ estart,
                           const int32_t* __restrict__ v, int64_t e0, int64_t e1, int2* __restrict__ uv,
                           int32_t* __restrict__ error) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int64_t i = n0 + first; i < n1; i += stride) {
    const int64_t dx = x[i] - min_x, dy = y[i] - min_y;
    if (dx < 0 || dy < 0 || dx >= (int64_t{1} << 30) || dy >= (int64_t{1} << 30)) {
      atomicOr(error, 16);
      xy[i] = make_int2(0, 0);
    } else {
      xy[i] = make_int2(static_cast<int32_t>(dx), static_cast<int32_t>(dy));
    }
  }
  const int lane = static_cast<int>(threadIdx.x & 31);
  const int64_t warps = stride >> 5;
  for (int64_t g0 = n0 + (first >> 5) * 32; g0 < n1; g0 += warps * 32) {
    const int64_t node = g0 + lane;
    const int32_t start = node < n1 ? estart[node] : INT32_MAX;
    const int32_t begin = __shfl_sync(kFullMask, start, 0);
    const int32_t end = estart[min(g0 + 32, n1)];
    if (begin < e0 || end > e1 || begin > end) {  // estart is built on the host; checked all the same
      if (lane == 0) atomicOr(error, 32);
      continue;
    }
    for (int64_t base = begin; base < end; base += 32) {
      const int64_t e = base + lane;
      int lo = 0;  // the last lane whose first edge is at or before e (starts are non-decreasing)
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        if (__shfl_sync(kFullMask, start, lo + step) <= e) lo += step;
      }
      const int32_t first_of_a = __shfl_sync(kFullMask, start, lo);
      if (e < end) {
        const int32_t a = static_cast<int32_t>(g0 + lo), b = v[e];
        // canonical, inside the chunk, and v ascending among the edges of lower end a
        const bool sorted = e == first_of_a || v[e - 1] < b;
        if (b <= a || b >= n1 || !sorted) {
          atomicOr(error, 32);
          uv[e] = make_int2(0, 0);
        } else {
          uv[e] = make_int2(a, b);
        }
      }
    }
  }
}

}  // namespace
}  // namespace cee

using namespace cee;

extern "C" {

int cee_batch_prepare(cee_ctx* ctx, const cee_batch_view* b, const cee_batch_options* options, cee_batch_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  rc = ValidateOptions(ctx, options);
  if (rc == CEE_OK) rc = ValidateShape(ctx, b);
  int64_t box[4];
  if (rc == CEE_OK) rc = ScanNodes(ctx, b->graph, box);
  if (rc != CEE_OK) return rc;
  const cee_graph_view& g = b->graph;
  // every edge canonical, inside its own instance, instance-sorted by (u, v)
  for (int32_t i = 0; i < b->instances; ++i) {
    const int64_t n0 = b->node_begin[i], n1 = b->node_begin[i + 1];
    for (int64_t e = b->edge_begin[i]; e < b->edge_begin[i + 1]; ++e) {
      const int32_t u = g.edge_u[e], v = g.edge_v[e];
      if (u < n0 || v >= n1 || u >= v) return Fail(ctx, CEE_ERR_INVALID, "edge outside its instance or not canonical");
      if (e > b->edge_begin[i] && (g.edge_u[e - 1] > u || (g.edge_u[e - 1] == u && g.edge_v[e - 1] >= v))) {
        return Fail(ctx, CEE_ERR_INVALID, "instance edges must be sorted by (u, v)");
      }
      if (g.edge_w[e] < 0 || g.edge_w[e] > INT32_MAX) return Fail(ctx, CEE_ERR_RANGE, "edge weight outside [0, 2^31)");
    }
  }
  BatchState& s = *State(ctx);
  s.prepared = false;
  std::vector<int2> xy;
  rc = PackCoordinates(ctx, g.n, g.x, g.y, &xy, &s.span);
  if (rc != CEE_OK) return rc;
  SetShape(s, b, options);
  rc = ReserveAll(ctx, s);
  if (rc != CEE_OK) return rc;
  std::vector<int2> uv(static_cast<size_t>(g.m));
  std::vector<int32_t> w32(static_cast<size_t>(g.m));
  for (int64_t e = 0; e < g.m; ++e) {
    uv[e] = make_int2(g.edge_u[e], g.edge_v[e]);
    w32[e] = static_cast<int32_t>(g.edge_w[e]);
  }
  cudaStream_t st = ctx->stream;
  cudaEventRecord(ctx->ev[0], st);
  cudaMemcpyAsync(s.d_node_begin.ptr, b->node_begin, (b->instances + 1) * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.d_edge_begin.ptr, b->edge_begin, (b->instances + 1) * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.d_chunk_begin.ptr, s.chunk_begin.data(), (b->instances + 1) * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.xy.ptr, xy.data(), xy.size() * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.uv.ptr, uv.data(), uv.size() * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.w32.ptr, w32.data(), w32.size() * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.active.ptr, g.active, static_cast<size_t>(g.m), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s.ro.ptr, g.row_offsets, (static_cast<size_t>(g.n) + 1) * 4, cudaMemcpyHostToDevice, st);
  if (g.adjacency > 0) {
    cudaMemcpyAsync(s.nbr.ptr, g.neighbors, static_cast<size_t>(g.adjacency) * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.ids.ptr, g.csr_edge_ids, static_cast<size_t>(g.adjacency) * 4, cudaMemcpyHostToDevice, st);
  }
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), st);
  if (g.adjacency > 0) {
    batch_gather<<<GridFor(g.adjacency, 256, ctx->sm_count * 8), 256, 0, st>>>(
        static_cast<const int32_t*>(s.ids.ptr), static_cast<const int32_t*>(s.nbr.ptr), static_cast<const int2*>(s.xy.ptr),
        0, g.adjacency, static_cast<const int32_t*>(s.w32.ptr), g.m, g.n, static_cast<int4*>(s.slot4.ptr), ctx->d_error);
  }
  if (g.n > 0 || g.m > 0) {
    batch_records<<<GridFor(std::max<int64_t>(g.n, g.m), 256, ctx->sm_count * 8), 256, 0, st>>>(
        static_cast<const int2*>(s.xy.ptr), static_cast<const int32_t*>(s.ro.ptr), 0, g.n, static_cast<int4*>(s.node4.ptr),
        static_cast<const int2*>(s.uv.ptr), static_cast<const int32_t*>(s.w32.ptr),
        static_cast<const uint8_t*>(s.active.ptr), 0, g.m, static_cast<int4*>(s.edge4.ptr));
  }
  cudaError_t status = LaunchSpatial(s, 0, b->instances, st);
  if (status == cudaSuccess) {
    status = cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  }
  if (status == cudaSuccess) status = cudaStreamSynchronize(st);  // host staging vectors die at return
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch upload");
  rc = BatchCheck(ctx);  // the upload kernels' checks (edge ids, neighbours)
  if (rc != CEE_OK) return rc;
  cudaEventRecord(ctx->ev[1], st);
  status = QueryBatchOccupancy(s);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch occupancy");
  rc = Capture(ctx, s);
  if (rc != CEE_OK) return rc;
  s.prepared = true;
  if (stats != nullptr) {
    *stats = cee_batch_stats{};
    stats->nodes = s.n;
    stats->edges = s.m;
    stats->adjacency = s.adj;
    stats->targets = static_cast<int64_t>(s.instances) * s.opt.targets;
    stats->flag_words = s.flag_words;
    stats->resident_bytes = BatchResident(ctx);
    stats->h2d_bytes = static_cast<int64_t>((b->instances + 1) * 24 + xy.size() * 8 + uv.size() * 12 + g.m +
                                            (g.n + 1) * 4 + g.adjacency * 8);
  }
  return CEE_OK;
}

int cee_batch_launch(cee_ctx* ctx) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  BatchState* s = ctx->batch;
  if (s == nullptr || !s->prepared) return Fail(ctx, CEE_ERR_STATE, "batch not prepared");
  if (s->exec == nullptr) {  // first resident launch after cee_batch_screen
    rc = Capture(ctx, *s);
    if (rc != CEE_OK) return rc;
  }
  const cudaError_t status = cudaGraphLaunch(s->exec, ctx->stream);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch graph launch");
  return CEE_OK;
}

int cee_batch_launch_plain(cee_ctx* ctx) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  BatchState* s = ctx->batch;
  if (s == nullptr || !s->prepared) return Fail(ctx, CEE_ERR_STATE, "batch not prepared");
  for (int32_t i = 0; i < s->instances; ++i) {
    rc = LaunchRange(ctx, *s, i, 1, 0, ctx->stream);
    if (rc != CEE_OK) return rc;
    const cudaError_t status = cudaStreamSynchronize(ctx->stream);
    if (status != cudaSuccess) return CudaFail(ctx, status, "plain batch launch");
  }
  return CEE_OK;
}

int cee_batch_fetch(cee_ctx* ctx, int32_t* witness, int32_t* target_ids, int32_t* target_count, int32_t* nbhd,
                    uint32_t* flags) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  BatchState* s = ctx->batch;
  if (s == nullptr || !s->prepared) return Fail(ctx, CEE_ERR_STATE, "batch not prepared");
  const size_t IT = static_cast<size_t>(s->instances) * s->opt.targets;
  cudaStream_t st = ctx->stream;
  if (witness != nullptr) cudaMemcpyAsync(witness, s->witness.ptr, s->m * 4, cudaMemcpyDeviceToHost, st);
  if (target_ids != nullptr) cudaMemcpyAsync(target_ids, s->target_ids.ptr, IT * 4, cudaMemcpyDeviceToHost, st);
  if (target_count != nullptr) {
    cudaMemcpyAsync(target_count, s->target_count.ptr, s->instances * 4, cudaMemcpyDeviceToHost, st);
  }
  if (nbhd != nullptr) {
    cudaMemcpyAsync(nbhd, s->nbhd.ptr, IT * s->opt.max_neighborhood * 4, cudaMemcpyDeviceToHost, st);
  }
  if (flags != nullptr) cudaMemcpyAsync(flags, s->flags.ptr, IT * s->flag_words * 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  const cudaError_t status = cudaStreamSynchronize(st);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch fetch");
  return BatchCheck(ctx);
}

int cee_batch_fetch_candidates(cee_ctx* ctx, int32_t* c, int32_t* d, int64_t* product, int32_t* count) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  BatchState* s = ctx->batch;
  if (s == nullptr || !s->prepared) return Fail(ctx, CEE_ERR_STATE, "batch not prepared");
  if (s->opt.max_cd_candidates == 0) return Fail(ctx, CEE_ERR_STATE, "the batch was prepared without c,d finalisation");
  const size_t IT = static_cast<size_t>(s->instances) * s->opt.targets;
  const size_t K = static_cast<size_t>(s->opt.max_cd_candidates);
  cudaStream_t st = ctx->stream;
  if (c != nullptr) cudaMemcpyAsync(c, s->cand_c.ptr, IT * K * 4, cudaMemcpyDeviceToHost, st);
  if (d != nullptr) cudaMemcpyAsync(d, s->cand_d.ptr, IT * K * 4, cudaMemcpyDeviceToHost, st);
  if (product != nullptr) cudaMemcpyAsync(product, s->cand_product.ptr, IT * K * 8, cudaMemcpyDeviceToHost, st);
  if (count != nullptr) cudaMemcpyAsync(count, s->cand_count.ptr, IT * 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  const cudaError_t status = cudaStreamSynchronize(st);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch candidate fetch");
  return BatchCheck(ctx);
}

int cee_batch_set_tuning(cee_ctx* ctx, const cee_batch_tuning* t) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (t == nullptr || t->jv_tile < 1 || t->jv_tile > 4096 || t->blocks_per_sm < 0 || t->blocks_per_sm > 64 ||
      t->chunks < 1 || t->chunks > kMaxChunks) {
    return Fail(ctx, CEE_ERR_INVALID, "bad batch tuning");
  }
  BatchState& s = *State(ctx);
  s.tune = *t;
  if (s.prepared) return Capture(ctx, s);
  return CEE_OK;
}

int cee_batch_get_tuning(const cee_ctx* ctx, cee_batch_tuning* t) {
  if (ctx == nullptr || t == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null argument");
  *t = ctx->batch != nullptr ? ctx->batch->tune : cee_batch_tuning{64, 0, 8};
  return CEE_OK;
}

int cee_batch_autotune(cee_ctx* ctx, int32_t reps, cee_batch_tuning* chosen) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  BatchState* s = ctx->batch;
  if (s == nullptr || !s->prepared) return Fail(ctx, CEE_ERR_STATE, "batch not prepared");
  reps = std::max(1, reps);
  const cee_batch_tuning start = s->tune;
  cee_batch_tuning best = start;
  float best_ms = 1e30f;
  const int occ = s->occupancy[s->span];
  for (const int tile : {16, 32, 64, 128, 256}) {
    for (const int per_sm : {occ, std::max(1, occ / 2)}) {
      cee_batch_tuning t = start;
      t.jv_tile = tile;
      t.blocks_per_sm = per_sm;
      rc = cee_batch_set_tuning(ctx, &t);
      if (rc != CEE_OK) return rc;
      rc = cee_batch_launch(ctx);  // warm-up
      if (rc != CEE_OK) return rc;
      cudaEventRecord(ctx->ev[2], ctx->stream);
      for (int r = 0; r < reps; ++r) {
        rc = cee_batch_launch(ctx);
        if (rc != CEE_OK) return rc;
      }
      cudaEventRecord(ctx->ev[3], ctx->stream);
      const cudaError_t status = cudaEventSynchronize(ctx->ev[3]);
      if (status != cudaSuccess) return CudaFail(ctx, status, "batch autotune");
      const float ms = EventMs(ctx->ev[2], ctx->ev[3]) / reps;
      if (ms < best_ms) {
        best_ms = ms;
        best = t;
      }
    }
  }
  rc = cee_batch_set_tuning(ctx, &best);
  if (rc != CEE_OK) return rc;
  if (chosen != nullptr) *chosen = best;
  return CEE_OK;
}

int cee_batch_screen(cee_ctx* ctx, const cee_batch_view* b, const cee_batch_options* options, int32_t* witness,
                     int32_t* target_ids, int32_t* target_count, int32_t* nbhd, uint32_t* flags,
                     cee_batch_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  rc = ValidateOptions(ctx, options);
  if (rc == CEE_OK) rc = ValidateShape(ctx, b);
  if (rc != CEE_OK) return rc;
  const cee_graph_view& g = b->graph;
  BatchState& s = *State(ctx);
  s.prepared = false;
  s.ReleaseGraph();
  SetShape(s, b, options);
  rc = ReserveAll(ctx, s);
  for (const auto& [buf, bytes] : {std::pair<DevBuf*, size_t>{&s.raw_x, g.n * 8ull}, {&s.raw_y, g.n * 8ull},
                                   {&s.raw_v, g.m * 4ull}, {&s.estart, (g.n + 1) * 4ull}}) {
    if (rc == CEE_OK) rc = Reserve(ctx, *buf, bytes);
  }
  if (rc != CEE_OK) return rc;
  const size_t stage_need = static_cast<size_t>(g.m) + static_cast<size_t>(g.n) + 1;
  if (s.stage_count < stage_need) {  // pinned int32 staging, reallocated when it grows
    if (s.stage_host != nullptr) cudaFreeHost(s.stage_host);
    s.stage_host = nullptr;
    s.stage_count = 0;
    const size_t count = stage_need;
    if (cudaHostAlloc(reinterpret_cast<void**>(&s.stage_host), count * sizeof(int32_t), cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      s.stage_host = nullptr;
      return Fail(ctx, CEE_ERR_NOMEM, "pinned weight staging");
    }
    s.stage_count = count;
  }
  cudaError_t status = cudaSuccess;
  if (s.h2d == nullptr) status = cudaStreamCreateWithFlags(&s.h2d, cudaStreamNonBlocking);
  if (status == cudaSuccess && s.d2h == nullptr) status = cudaStreamCreateWithFlags(&s.d2h, cudaStreamNonBlocking);
  if (status == cudaSuccess && s.prep == nullptr) status = cudaStreamCreateWithFlags(&s.prep, cudaStreamNonBlocking);
  for (int i = 0; i < kMaxChunks && status == cudaSuccess; ++i) {
    if (s.up[i] == nullptr) status = cudaEventCreateWithFlags(&s.up[i], cudaEventDisableTiming);
    if (status == cudaSuccess && s.done[i] == nullptr) status = cudaEventCreateWithFlags(&s.done[i], cudaEventDisableTiming);
    if (status == cudaSuccess && s.prepped[i] == nullptr) {
      status = cudaEventCreateWithFlags(&s.prepped[i], cudaEventDisableTiming);
    }
  }
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch streams");
  status = QueryBatchOccupancy(s);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batch occupancy");
  const int chunks = std::max(1, std::min<int>(s.tune.chunks, b->instances));
  cudaStream_t cs = ctx->stream;
  // every early return after the first queued copy: the caller's buffers stay borrowed until all queued
  // copies (uploads, and downloads of finished chunks) have ended
  auto drain = [&] {
    cudaStreamSynchronize(s.h2d);
    cudaStreamSynchronize(s.prep);
    cudaStreamSynchronize(cs);
    cudaStreamSynchronize(s.d2h);
  };
  // ev[0] follows the error-word reset and the offset copies, so that the copy stream, and through it the
  // preparation stream, starts behind them (and behind earlier work on the context's stream)
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), cs);
  cudaMemcpyAsync(s.d_node_begin.ptr, b->node_begin, (b->instances + 1) * 8, cudaMemcpyHostToDevice, cs);
  cudaMemcpyAsync(s.d_edge_begin.ptr, b->edge_begin, (b->instances + 1) * 8, cudaMemcpyHostToDevice, cs);
  cudaMemcpyAsync(s.d_chunk_begin.ptr, s.chunk_begin.data(), (b->instances + 1) * 8, cudaMemcpyHostToDevice, cs);
  cudaEventRecord(ctx->ev[0], cs);
  cudaStreamWaitEvent(s.h2d, ctx->ev[0], 0);
  const size_t T = static_cast<size_t>(s.opt.targets), NB = static_cast<size_t>(s.opt.max_neighborhood);
  const size_t FW = static_cast<size_t>(s.flag_words);
  int64_t h2d_bytes = (b->instances + 1) * 24, d2h_bytes = 0;
  std::vector<int32_t> bounds(static_cast<size_t>(chunks) + 1, 0);
  for (int c = 0; c <= chunks; ++c) {
    bounds[static_cast<size_t>(c)] = static_cast<int32_t>(static_cast<int64_t>(b->instances) * c / chunks);
    // the chunks' CSR slices are copied before the full row-offset check: their end points first
    const int32_t slot = g.row_offsets[b->node_begin[bounds[static_cast<size_t>(c)]]];
    if (slot < 0 || slot > g.adjacency || (c > 0 && slot < g.row_offsets[b->node_begin[bounds[c - 1]]])) {
      drain();
      return Fail(ctx, CEE_ERR_INVALID, "row_offsets not non-decreasing");
    }
  }
  // Per chunk: the chunk's arrays go up on the copy stream while its weights are narrowed to int32 on
  // host threads (range-checked) into pinned staging, which follows them; its screen is queued behind
  // them. The O(n) host checks run once, after the first chunk's copies are queued and before any
  // kernel reads them.
  int64_t min_x = 0, min_y = 0;
  for (int c = 0; c < chunks; ++c) {
    const int32_t i0 = bounds[c], i1 = bounds[c + 1];
    if (i1 == i0) continue;
    const int64_t n0 = b->node_begin[i0], n1 = b->node_begin[i1], e0 = b->edge_begin[i0], e1 = b->edge_begin[i1];
    const int64_t s0 = g.row_offsets[n0], s1 = g.row_offsets[n1];
    cudaMemcpyAsync(static_cast<int64_t*>(s.raw_x.ptr) + n0, g.x + n0, (n1 - n0) * 8, cudaMemcpyHostToDevice, s.h2d);
    cudaMemcpyAsync(static_cast<int64_t*>(s.raw_y.ptr) + n0, g.y + n0, (n1 - n0) * 8, cudaMemcpyHostToDevice, s.h2d);
    cudaMemcpyAsync(static_cast<int32_t*>(s.ro.ptr) + n0, g.row_offsets + n0, (n1 - n0 + 1) * 4, cudaMemcpyHostToDevice, s.h2d);
    cudaMemcpyAsync(static_cast<int32_t*>(s.raw_v.ptr) + e0, g.edge_v + e0, (e1 - e0) * 4, cudaMemcpyHostToDevice, s.h2d);
    cudaMemcpyAsync(static_cast<uint8_t*>(s.active.ptr) + e0, g.active + e0, e1 - e0, cudaMemcpyHostToDevice, s.h2d);
    if (s1 > s0) {
      cudaMemcpyAsync(static_cast<int32_t*>(s.nbr.ptr) + s0, g.neighbors + s0, (s1 - s0) * 4, cudaMemcpyHostToDevice, s.h2d);
      cudaMemcpyAsync(static_cast<int32_t*>(s.ids.ptr) + s0, g.csr_edge_ids + s0, (s1 - s0) * 4, cudaMemcpyHostToDevice, s.h2d);
    }
    // On host threads: the weights narrowed to int32, and the lower ends checked (inside this
    // chunk's nodes, ascending) while estart is built from them: estart[x], x in [n0, n1], is the
    // first edge whose lower end is x or above. The device rebuilds each u from estart, so the lower
    // ends never cross PCIe, and checks the upper ends (batch_pack).
    std::vector<uint8_t> bad_weight(16, 0), bad_edge(16, 0);
    int32_t* const estart_host = s.stage_host + g.m;
    ParallelRanges(e1 - e0, [&](int64_t a0, int64_t a1, int t) {
      int64_t pu = n0 - 1;
      if (a0 > 0) pu = std::min<int64_t>(std::max<int64_t>(g.edge_u[e0 + a0 - 1], n0 - 1), n1);
      for (int64_t e = e0 + a0; e < e0 + a1; ++e) {
        const int64_t w = g.edge_w[e];
        if (w < 0 || w > INT32_MAX) bad_weight[t] = 1;
        s.stage_host[e] = static_cast<int32_t>(w);
        const int64_t u = g.edge_u[e];
        if (u < n0 || u < pu || u >= n1) {
          bad_edge[t] = 1;
          return;
        }
        for (int64_t node = pu + 1; node <= u; ++node) estart_host[node] = static_cast<int32_t>(e);
        pu = u;
      }
      if (a1 == e1 - e0) {
        for (int64_t node = pu + 1; node <= n1; ++node) estart_host[node] = static_cast<int32_t>(e1);
      }
    });
    if (std::any_of(bad_weight.begin(), bad_weight.end(), [](uint8_t v) { return v != 0; })) {
      drain();
      return Fail(ctx, CEE_ERR_RANGE, "edge weight outside [0, 2^31)");
    }
    if (std::any_of(bad_edge.begin(), bad_edge.end(), [](uint8_t v) { return v != 0; })) {
      drain();
      return Fail(ctx, CEE_ERR_INVALID, "edges must be canonical, inside their instance and sorted by (u, v)");
    }
    cudaMemcpyAsync(static_cast<int32_t*>(s.w32.ptr) + e0, s.stage_host + e0, (e1 - e0) * 4, cudaMemcpyHostToDevice, s.h2d);
    cudaMemcpyAsync(static_cast<int32_t*>(s.estart.ptr) + n0, estart_host + n0, (n1 - n0 + 1) * 4, cudaMemcpyHostToDevice,
                    s.h2d);
    h2d_bytes += (n1 - n0) * 24 + 8 + (e1 - e0) * 9 + (s1 - s0) * 8;
    cudaEventRecord(s.up[c], s.h2d);
    if (c == 0) {  // row offsets and the bounding box on host threads, while the first copies run
      int64_t box[4];
      rc = ScanNodes(ctx, g, box);
      if (rc != CEE_OK) {
        drain();
        return rc;
      }
      min_x = box[0];
      min_y = box[2];
      s.span = span_class(box[1] - box[0], box[3] - box[2]);
    }
    // convert (preparation stream: its blocks take the SMs that the previous chunk's screen frees as
    // it drains), screen (compute stream), download (second copy stream)
    cudaStreamWaitEvent(s.prep, s.up[c], 0);
    batch_pack<<<GridFor(std::max(n1 - n0, e1 - e0), 256, ctx->sm_count * 8), 256, 0, s.prep>>>(
        static_cast<const int64_t*>(s.raw_x.ptr), static_cast<const int64_t*>(s.raw_y.ptr), n0, n1, min_x, min_y,
        static_cast<int2*>(s.xy.ptr), static_cast<const int32_t*>(s.estart.ptr), static_cast<const int32_t*>(s.raw_v.ptr),
        e0, e1, static_cast<int2*>(s.uv.ptr), ctx->d_error);
    batch_records<<<GridFor(std::max(n1 - n0, e1 - e0), 256, ctx->sm_count * 8), 256, 0, s.prep>>>(
        static_cast<const int2*>(s.xy.ptr), static_cast<const int32_t*>(s.ro.ptr), n0, n1, static_cast<int4*>(s.node4.ptr),
        static_cast<const int2*>(s.uv.ptr), static_cast<const int32_t*>(s.w32.ptr),
        static_cast<const uint8_t*>(s.active.ptr), e0, e1, static_cast<int4*>(s.edge4.ptr));
    if (s1 > s0) {
      batch_gather<<<GridFor(s1 - s0, 256, ctx->sm_count * 8), 256, 0, s.prep>>>(
          static_cast<const int32_t*>(s.ids.ptr), static_cast<const int32_t*>(s.nbr.ptr), static_cast<const int2*>(s.xy.ptr),
          s0, s1, static_cast<const int32_t*>(s.w32.ptr), g.m, g.n, static_cast<int4*>(s.slot4.ptr), ctx->d_error);
    }
    status = LaunchSpatial(s, i0, i1 - i0, s.prep);
    if (status != cudaSuccess) {
      drain();
      return CudaFail(ctx, status, "batch spatial chunks");
    }
    cudaEventRecord(s.prepped[c], s.prep);
    cudaStreamWaitEvent(cs, s.prepped[c], 0);
    rc = LaunchRange(ctx, s, i0, i1 - i0, c, cs);
    if (rc != CEE_OK) {
      drain();
      return rc;
    }
    cudaEventRecord(s.done[c], cs);
    // download the chunk's results (second copy stream)
    cudaStreamWaitEvent(s.d2h, s.done[c], 0);
    const size_t t0 = static_cast<size_t>(i0) * T, t1 = static_cast<size_t>(i1) * T;
    if (witness != nullptr) {
      cudaMemcpyAsync(witness + e0, static_cast<int32_t*>(s.witness.ptr) + e0, (e1 - e0) * 4, cudaMemcpyDeviceToHost, s.d2h);
      d2h_bytes += (e1 - e0) * 4;
    }
    if (target_ids != nullptr) {
      cudaMemcpyAsync(target_ids + t0, static_cast<int32_t*>(s.target_ids.ptr) + t0, (t1 - t0) * 4,
                      cudaMemcpyDeviceToHost, s.d2h);
      d2h_bytes += (t1 - t0) * 4;
    }
    if (target_count != nullptr) {
      cudaMemcpyAsync(target_count + i0, static_cast<int32_t*>(s.target_count.ptr) + i0, (i1 - i0) * 4,
                      cudaMemcpyDeviceToHost, s.d2h);
      d2h_bytes += (i1 - i0) * 4;
    }
    if (nbhd != nullptr) {
      cudaMemcpyAsync(nbhd + t0 * NB, static_cast<int32_t*>(s.nbhd.ptr) + t0 * NB, (t1 - t0) * NB * 4,
                      cudaMemcpyDeviceToHost, s.d2h);
      d2h_bytes += (t1 - t0) * NB * 4;
    }
    if (flags != nullptr) {
      cudaMemcpyAsync(flags + t0 * FW, static_cast<uint32_t*>(s.flags.ptr) + t0 * FW, (t1 - t0) * FW * 4,
                      cudaMemcpyDeviceToHost, s.d2h);
      d2h_bytes += (t1 - t0) * FW * 4;
    }
  }
  cudaEventRecord(ctx->ev[4], s.d2h);
  cudaStreamWaitEvent(cs, ctx->ev[4], 0);
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, cs);
  cudaEventRecord(ctx->ev[5], cs);
  status = cudaStreamSynchronize(cs);
  if (status != cudaSuccess) return CudaFail(ctx, status, "batched screen");
  rc = BatchCheck(ctx);
  if (rc != CEE_OK) return rc;
  s.prepared = true;  // the resident copy now holds this batch; its graph is captured by the next cee_batch_launch
  if (stats != nullptr) {
    *stats = cee_batch_stats{};
    stats->nodes = s.n;
    stats->edges = s.m;
    stats->adjacency = s.adj;
    stats->targets = static_cast<int64_t>(s.instances) * s.opt.targets;
    stats->flag_words = s.flag_words;
    stats->resident_bytes = BatchResident(ctx);
    stats->h2d_bytes = h2d_bytes;
    stats->d2h_bytes = d2h_bytes;
    stats->total_ms = EventMs(ctx->ev[0], ctx->ev[5]);
  }
  return CEE_OK;
}

}  // extern "C"
