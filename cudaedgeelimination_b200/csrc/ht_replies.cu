// Host side of the HT reply lists (ht_replies.cuh): validation as the reference's seam does it
// (src/cuda/ht_replies.cu:521-581), the snapshot kept on the device while it does not change, the
// count pass, the offsets, the write pass, and the copy-out.
#include "cee.h"
#include "cee_internal.h"

#include "ht_replies.cuh"

#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace cee {

struct ReplyState {
  // snapshot key: coordinates and CSR of the last upload
  bool has_graph = false;
  int32_t n = 0, dist_type = 0;
  int span = kSpanSmall;
  std::vector<int64_t> hx, hy;
  std::vector<int32_t> hro, hnbr;
  std::vector<uint8_t> hactive;  // with the CSR: the content the last validation passed on
  DevBuf xy, ro, nbr;
  // per call
  DevBuf items, counts, offsets, out;
  int kind = 0;  // 1: Hamilton replies (cee_ht_pair), 2: end replies (cee_node_edge)
  uint64_t total = 0;
};

void ReleaseReplies(cee_ctx* ctx) {
  if (ctx->replies == nullptr) return;
  ReplyState* s = ctx->replies;
  for (DevBuf* b : {&s->xy, &s->ro, &s->nbr, &s->items, &s->counts, &s->offsets, &s->out}) b->Release();
  delete s;
  ctx->replies = nullptr;
}

uint64_t RepliesResident(const cee_ctx* ctx) {
  const ReplyState* s = ctx->replies;
  if (s == nullptr) return 0;
  return s->xy.capacity + s->ro.capacity + s->nbr.capacity + s->items.capacity + s->counts.capacity +
         s->offsets.capacity + s->out.capacity;
}

namespace {

template <typename T>
bool Same(const std::vector<T>& kept, const T* data, size_t count) {
  return kept.size() == count && (count == 0 || std::memcmp(kept.data(), data, count * sizeof(T)) == 0);
}

// ValidateGraphShape (src/cuda/ht_replies.cu:521-553): a Euclidean or ceiling snapshot of at least 4
// nodes whose CSR rows are strictly ascending, in range, free of self loops and symmetric, and hold
// exactly the active edges (two slots each).
int ValidateReplyGraph(cee_ctx* ctx, const cee_graph_view* g) {
  int rc = ValidateView(ctx, g);
  if (rc != CEE_OK) return rc;
  if (g->n < 4) return Fail(ctx, CEE_ERR_INVALID, "HT replies need a snapshot of at least 4 nodes");
  int64_t active = 0;
  for (int64_t e = 0; e < g->m; ++e) active += g->active[e] != 0 ? 1 : 0;
  if (g->adjacency != 2 * active) return Fail(ctx, CEE_ERR_INVALID, "HT replies: the CSR must hold exactly the active edges");
  for (int32_t node = 0; node < g->n; ++node) {
    int32_t previous = -1;
    for (int32_t s = g->row_offsets[node]; s < g->row_offsets[node + 1]; ++s) {
      const int32_t nb = g->neighbors[s];
      if (nb <= previous || nb < 0 || nb >= g->n || nb == node) {
        return Fail(ctx, CEE_ERR_INVALID, "HT replies: CSR rows must ascend strictly, in range, without self loops");
      }
      previous = nb;
    }
  }
  for (int32_t node = 0; node < g->n; ++node) {
    for (int32_t s = g->row_offsets[node]; s < g->row_offsets[node + 1]; ++s) {
      if (!HostHasActiveEdge(g, g->neighbors[s], node)) {
        return Fail(ctx, CEE_ERR_INVALID, "HT replies: the CSR is not symmetric");
      }
    }
  }
  return CEE_OK;
}

// Whether the snapshot equals the last one validated and uploaded: coordinates, CSR and active flags
// (ValidateReplyGraph's outcome is a function of exactly these and of the sizes, so it need not run
// again).
bool SameReplyGraph(const ReplyState* s, const cee_graph_view* g) {
  if (s == nullptr || !s->has_graph || s->n != g->n || s->dist_type != g->dist_type) return false;
  const size_t n = static_cast<size_t>(g->n), adj = static_cast<size_t>(g->adjacency), m = static_cast<size_t>(g->m);
  return g->adjacency >= 0 && g->m >= 0 && Same(s->hro, g->row_offsets, n + 1) && Same(s->hnbr, g->neighbors, adj) &&
         Same(s->hactive, g->active, m) && Same(s->hx, g->x, n) && Same(s->hy, g->y, n);
}

// Uploads coordinates and CSR of a validated snapshot unless `same` (it equals the last upload).
int PrepareReplyGraph(cee_ctx* ctx, const cee_graph_view* g, bool same, bool* grew) {
  if (ctx->replies == nullptr) ctx->replies = new ReplyState();
  ReplyState& s = *ctx->replies;
  const size_t n = static_cast<size_t>(g->n), adj = static_cast<size_t>(g->adjacency);
  if (same) return CEE_OK;
  s.has_graph = false;
  std::vector<int2> xy;
  const int rc = PackCoordinates(ctx, g->n, g->x, g->y, &xy, &s.span);
  if (rc != CEE_OK) return rc;
  bool g1 = false, g2 = false, g3 = false;
  cudaError_t status = s.xy.Reserve(n * sizeof(int2) + 16, &g1);
  if (status == cudaSuccess) status = s.ro.Reserve((n + 1) * 4 + 16, &g2);
  if (status == cudaSuccess) status = s.nbr.Reserve(adj * 4 + 16, &g3);
  if (status != cudaSuccess) return CudaFail(ctx, status, "HT reply snapshot allocation");
  *grew = *grew || g1 || g2 || g3;
  status = CopyFromHost(ctx, s.xy.ptr, xy.data(), n * sizeof(int2));
  if (status == cudaSuccess) status = CopyFromHost(ctx, s.ro.ptr, g->row_offsets, (n + 1) * 4);
  if (status == cudaSuccess && adj > 0) status = CopyFromHost(ctx, s.nbr.ptr, g->neighbors, adj * 4);
  if (status != cudaSuccess) return CudaFail(ctx, status, "HT reply snapshot upload");
  s.hx.assign(g->x, g->x + n);
  s.hy.assign(g->y, g->y + n);
  s.hro.assign(g->row_offsets, g->row_offsets + n + 1);
  s.hnbr.assign(g->neighbors, g->neighbors + adj);
  s.hactive.assign(g->active, g->active + g->m);
  s.n = g->n;
  s.dist_type = g->dist_type;
  s.has_graph = true;
  return CEE_OK;
}

int ReplyGrid(cee_ctx* ctx, int64_t items) {
  return GridFor(items, kReplyWarps, ctx->sm_count * 8);
}

// After the count pass: the offsets (exclusive prefix sum of the counts) into offsets_out and up to
// the device for the write pass; the reply total into s.total.
int ReplyOffsets(cee_ctx* ctx, ReplyState& s, int64_t count, uint64_t* offsets_out, bool* grew) {
  std::vector<unsigned long long> counts(static_cast<size_t>(count));
  cudaStream_t st = ctx->stream;
  cudaMemcpyAsync(counts.data(), s.counts.ptr, static_cast<size_t>(count) * 8, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  cudaError_t status = cudaStreamSynchronize(st);
  if (status != cudaSuccess) return CudaFail(ctx, status, "HT reply count pass");
  offsets_out[0] = 0;
  for (int64_t i = 0; i < count; ++i) {
    if (counts[static_cast<size_t>(i)] > std::numeric_limits<uint64_t>::max() - offsets_out[i]) {
      return Fail(ctx, CEE_ERR_RANGE, "HT reply total overflows 64 bits");
    }
    offsets_out[i + 1] = offsets_out[i] + counts[static_cast<size_t>(i)];
  }
  s.total = offsets_out[count];
  bool g1 = false;
  status = s.offsets.Reserve(static_cast<size_t>(count + 1) * 8, &g1);
  *grew = *grew || g1;
  if (status != cudaSuccess) return CudaFail(ctx, status, "HT reply offsets allocation");
  cudaMemcpyAsync(s.offsets.ptr, offsets_out, static_cast<size_t>(count + 1) * 8, cudaMemcpyHostToDevice, st);
  return CEE_OK;
}

void FillStats(const cee_ctx* ctx, bool hit, bool grew, cee_ht_reply_stats* stats) {
  if (stats == nullptr) return;
  stats->graph_hit = hit ? 1 : 0;
  stats->workspace_hit = grew ? 0 : 1;
  stats->resident_bytes = RepliesResident(ctx);
}

}  // namespace
}  // namespace cee

using namespace cee;

extern "C" {

int cee_ht_replies(cee_ctx* ctx, const cee_graph_view* graph, int32_t u, int32_t v, const int32_t* centers,
                   int64_t count, uint64_t* offsets_out, cee_ht_reply_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (stats != nullptr) *stats = cee_ht_reply_stats{};
  if (graph == nullptr || count < 0 || offsets_out == nullptr || (count > 0 && centers == nullptr)) {
    return Fail(ctx, CEE_ERR_INVALID, "bad HT reply arguments");
  }
  rc = ValidateView(ctx, graph);
  if (rc != CEE_OK) return rc;
  const bool same = SameReplyGraph(ctx->replies, graph);  // validated and uploaded last time
  if (!same) {
    rc = ValidateReplyGraph(ctx, graph);
    if (rc != CEE_OK) return rc;
  }
  // ValidateInputs (src/cuda/ht_replies.cu:555-566)
  if (u < 0 || v >= graph->n || u >= v || !HostHasActiveEdge(graph, u, v)) {
    return Fail(ctx, CEE_ERR_INVALID, "HT replies: the target must be an active edge (u < v)");
  }
  for (int64_t i = 0; i < count; ++i) {
    if (centers[i] < 0 || centers[i] >= graph->n || centers[i] == u || centers[i] == v) {
      return Fail(ctx, CEE_ERR_INVALID, "HT replies: a center is out of range or a target endpoint");
    }
  }
  offsets_out[0] = 0;
  if (ctx->replies == nullptr) ctx->replies = new ReplyState();
  ctx->replies->kind = 1;
  ctx->replies->total = 0;
  if (count == 0) return CEE_OK;
  const bool hit = same;
  bool grew = false;
  rc = PrepareReplyGraph(ctx, graph, same, &grew);
  if (rc != CEE_OK) return Drained(ctx, rc);
  ReplyState& s = *ctx->replies;
  s.kind = 1;
  s.total = 0;
  bool g1 = false, g2 = false;
  cudaError_t status = s.items.Reserve(static_cast<size_t>(count) * 4, &g1);
  if (status == cudaSuccess) status = s.counts.Reserve(static_cast<size_t>(count) * 8, &g2);
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT reply workspace allocation"));
  grew = grew || g1 || g2;
  cudaStream_t st = ctx->stream;
  status = CopyFromHost(ctx, s.items.ptr, centers, static_cast<size_t>(count) * 4);
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT reply center upload"));
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), st);
  ReplyArgs A{};
  A.xy = static_cast<const int2*>(s.xy.ptr);
  A.dist_type = s.dist_type;
  A.row_offsets = static_cast<const int32_t*>(s.ro.ptr);
  A.nbr = static_cast<const int32_t*>(s.nbr.ptr);
  A.tu = u;
  A.tv = v;
  A.centers = static_cast<const int32_t*>(s.items.ptr);
  A.count = count;
  A.counts = static_cast<unsigned long long*>(s.counts.ptr);
  A.error = ctx->d_error;
  const int grid = ReplyGrid(ctx, count);
  WithSpan(s.span, [&](auto S) { ht_reply_kernel<S.value, false><<<grid, kReplyWarps * 32, 0, st>>>(A); });
  status = cudaGetLastError();
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT reply count launch"));
  rc = ReplyOffsets(ctx, s, count, offsets_out, &grew);
  if (rc != CEE_OK) return Drained(ctx, rc);
  if (*ctx->h_error != 0) return CheckDeviceError(ctx, "HT reply count pass");
  if (s.total > 0) {
    bool g3 = false;
    status = s.out.Reserve(static_cast<size_t>(s.total) * sizeof(cee_ht_pair), &g3);
    if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT reply list allocation"));
    grew = grew || g3;
    A.offsets = static_cast<const unsigned long long*>(s.offsets.ptr);
    A.out = static_cast<int32_t*>(s.out.ptr);
    WithSpan(s.span, [&](auto S) { ht_reply_kernel<S.value, true><<<grid, kReplyWarps * 32, 0, st>>>(A); });
    status = cudaGetLastError();
    if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT reply write launch"));
  }
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  status = cudaStreamSynchronize(st);
  if (status != cudaSuccess) return CudaFail(ctx, status, "HT reply write pass");
  if (*ctx->h_error != 0) {
    s.total = 0;
    return Fail(ctx, CEE_ERR_STATE, "HT replies: the write pass disagreed with the count pass (code " +
                                        std::to_string(*ctx->h_error) + ")");
  }
  FillStats(ctx, hit, grew, stats);
  return CEE_OK;
}

int cee_ht_end_replies(cee_ctx* ctx, const cee_graph_view* graph, const cee_ht_end_task* tasks, int64_t count,
                       uint64_t* offsets_out, cee_ht_reply_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (stats != nullptr) *stats = cee_ht_reply_stats{};
  if (graph == nullptr || count < 0 || offsets_out == nullptr || (count > 0 && tasks == nullptr)) {
    return Fail(ctx, CEE_ERR_INVALID, "bad HT end reply arguments");
  }
  rc = ValidateView(ctx, graph);
  if (rc != CEE_OK) return rc;
  const bool same = SameReplyGraph(ctx->replies, graph);
  if (!same) {
    rc = ValidateReplyGraph(ctx, graph);
    if (rc != CEE_OK) return rc;
  }
  // ValidateEndInputs (src/cuda/ht_replies.cu:568-581)
  for (int64_t i = 0; i < count; ++i) {
    const cee_ht_end_task t = tasks[i];
    if (t.endpoint < 0 || t.endpoint >= graph->n || t.internal_neighbor < 0 || t.internal_neighbor >= graph->n ||
        t.endpoint == t.internal_neighbor || !HostHasActiveEdge(graph, t.endpoint, t.internal_neighbor)) {
      return Fail(ctx, CEE_ERR_INVALID, "HT end replies: a task's edge must be active");
    }
  }
  offsets_out[0] = 0;
  if (ctx->replies == nullptr) ctx->replies = new ReplyState();
  ctx->replies->kind = 2;
  ctx->replies->total = 0;
  if (count == 0) return CEE_OK;
  const bool hit = same;
  bool grew = false;
  rc = PrepareReplyGraph(ctx, graph, same, &grew);
  if (rc != CEE_OK) return Drained(ctx, rc);
  ReplyState& s = *ctx->replies;
  s.kind = 2;
  s.total = 0;
  bool g1 = false, g2 = false;
  cudaError_t status = s.items.Reserve(static_cast<size_t>(count) * sizeof(cee_ht_end_task), &g1);
  if (status == cudaSuccess) status = s.counts.Reserve(static_cast<size_t>(count) * 8, &g2);
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT end reply workspace allocation"));
  grew = grew || g1 || g2;
  cudaStream_t st = ctx->stream;
  status = CopyFromHost(ctx, s.items.ptr, tasks, static_cast<size_t>(count) * sizeof(cee_ht_end_task));
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT end reply task upload"));
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), st);
  EndReplyArgs A{};
  A.row_offsets = static_cast<const int32_t*>(s.ro.ptr);
  A.nbr = static_cast<const int32_t*>(s.nbr.ptr);
  A.tasks = static_cast<const int2*>(s.items.ptr);
  A.count = count;
  A.counts = static_cast<unsigned long long*>(s.counts.ptr);
  A.error = ctx->d_error;
  const int grid = ReplyGrid(ctx, count);
  ht_end_reply_kernel<false><<<grid, kReplyWarps * 32, 0, st>>>(A);
  status = cudaGetLastError();
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT end reply count launch"));
  rc = ReplyOffsets(ctx, s, count, offsets_out, &grew);
  if (rc != CEE_OK) return Drained(ctx, rc);
  if (*ctx->h_error != 0) {
    s.total = 0;
    return Fail(ctx, CEE_ERR_INVALID, "HT end replies: a task's internal neighbour is not in its endpoint's row");
  }
  if (s.total > 0) {
    bool g3 = false;
    status = s.out.Reserve(static_cast<size_t>(s.total) * sizeof(cee_node_edge), &g3);
    if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT end reply list allocation"));
    grew = grew || g3;
    A.offsets = static_cast<const unsigned long long*>(s.offsets.ptr);
    A.out = static_cast<int2*>(s.out.ptr);
    ht_end_reply_kernel<true><<<grid, kReplyWarps * 32, 0, st>>>(A);
    status = cudaGetLastError();
    if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "HT end reply write launch"));
  }
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  status = cudaStreamSynchronize(st);
  if (status != cudaSuccess) return CudaFail(ctx, status, "HT end reply write pass");
  if (*ctx->h_error != 0) {
    s.total = 0;
    return Fail(ctx, CEE_ERR_STATE, "HT end replies: the write pass disagreed with the count pass (code " +
                                        std::to_string(*ctx->h_error) + ")");
  }
  FillStats(ctx, hit, grew, stats);
  return CEE_OK;
}

int cee_ht_replies_fetch(cee_ctx* ctx, void* replies_out) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  const ReplyState* s = ctx->replies;
  if (s == nullptr || s->kind == 0) return Fail(ctx, CEE_ERR_STATE, "no HT reply call to fetch from");
  if (s->total == 0) return CEE_OK;
  if (replies_out == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null reply output");
  const size_t record = s->kind == 1 ? sizeof(cee_ht_pair) : sizeof(cee_node_edge);
  const cudaError_t status = CopyToHost(ctx, replies_out, s->out.ptr, static_cast<size_t>(s->total) * record);
  if (status != cudaSuccess) return CudaFail(ctx, status, "HT reply download");
  return CEE_OK;
}

}  // extern "C"
