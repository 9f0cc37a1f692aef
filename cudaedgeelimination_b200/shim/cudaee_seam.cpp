// The reference's CUDA-backend seam, implemented on the B200 C ABI (include/cee.h).
//
// Linking this translation unit in place of the reference's src/cuda/jv_cuda.cu,
// src/cuda/kopt_cost.cu and src/cuda/ht_cd.cu (or their *_stub.cpp twins, selected by
// CMakeLists.txt:43-67) makes RunJvElimination, EvaluateKOptTemplateCosts and
// EvaluateHtCdCandidates drive the sm_100a kernels unchanged; their in-situ CPU checks
// (candidate re-verification, full-matrix certification, flag comparison) stay in force.
//
// Contract kept from the reference:
//   * one cache per (host thread, device): a thread-local cee_ctx per device
//     (src/cuda/jv_cuda.cu:138-139, src/cuda/kopt_cost.cu:133-134);
//   * device choice: the thread's forced device (cuda_device_affinity.hpp), else the device
//     this thread used last, else the device with the most free memory
//     (src/cuda/jv_cuda.cu:290-346);
//   * input validation before any launch, errors as exceptions: invalid input ->
//     std::invalid_argument, out of the exact range -> std::overflow_error, everything else ->
//     std::runtime_error; *Available() returns false with a reason instead of throwing;
//   * the HT wavefront propagation entry points keep the stub behaviour
//     (src/cuda/ht_cd_stub.cpp:20-33): unavailable, and throwing when called;
//   * the HT reply seam (src/cuda/ht_replies.cu:583-758) replaces the reference's stub
//     (src/cuda/ht_replies_stub.cpp) as well.
#include "cee.h"

#include "cuda_edge_elimination/cuda_device_affinity.hpp"
#include "cuda_edge_elimination/elimination.hpp"
#include "cuda_edge_elimination/hamilton_tutte.hpp"
#include "cuda_edge_elimination/local_search.hpp"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <omp.h>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace cudaee {
namespace {

struct ThreadContexts {
  std::vector<std::pair<int, cee_ctx*>> contexts;
  int preferred = -1;
  ~ThreadContexts() {
    for (auto& entry : contexts) cee_destroy(entry.second);
  }
};

thread_local ThreadContexts g_threads;

[[noreturn]] void Raise(int status, const cee_ctx* ctx, const std::string& what) {
  const std::string message = what + ": " + cee_last_error(ctx);
  if (status == CEE_ERR_INVALID) throw std::invalid_argument(message);
  if (status == CEE_ERR_RANGE) throw std::overflow_error(message);
  throw std::runtime_error(message);
}

int SelectDevice(std::string* reason) {
  int count = 0;
  cee_device_count(&count);
  if (count == 0) {
    if (reason != nullptr) *reason = "no visible CUDA device";
    return -1;
  }
  const int forced = detail::CudaDevicePreferenceForCurrentThread();
  if (forced >= 0) {
    if (forced >= count) {
      if (reason != nullptr) *reason = "forced CUDA device ordinal is not visible";
      return -1;
    }
    g_threads.preferred = forced;
    return forced;
  }
  if (g_threads.preferred >= 0 && g_threads.preferred < count) return g_threads.preferred;
  int device = -1;
  if (cee_select_device(&device) != CEE_OK) {
    if (reason != nullptr) *reason = cee_last_error(nullptr);
    return -1;
  }
  g_threads.preferred = device;
  return device;
}

cee_ctx* ContextFor(int device) {
  for (auto& entry : g_threads.contexts) {
    if (entry.first == device) return entry.second;
  }
  cee_ctx* ctx = nullptr;
  const int status = cee_create(device, &ctx);
  if (status != CEE_OK) Raise(status, nullptr, "B200 context creation");
  g_threads.contexts.emplace_back(device, ctx);
  return ctx;
}

cee_ctx* RequireContext(int* selected_device, const char* what) {
  std::string reason;
  const int device = SelectDevice(&reason);
  if (device < 0) throw std::runtime_error(std::string(what) + " unavailable: " + reason);
  if (selected_device != nullptr) *selected_device = device;
  return ContextFor(device);
}

// Flat host arrays behind a cee_graph_view of a GraphSnapshot (Point and Edge are structs), kept
// across calls. Bind refreshes them in one pass that compares each static value (coordinates,
// edge endpoints and weights: the reference's resident-cache key, src/cuda/jv_cuda.cu:360-382)
// with the kept one and writes only what differs, so that it knows whether the static content
// changed. `jv_ctx` is the context whose JV static cache was last loaded from this content.
constexpr int64_t kParallelElements = 1 << 16;

struct SnapshotArrays {
  std::vector<int64_t> x, y, w;
  std::vector<int32_t> u, v;
  std::vector<uint8_t> active;
  std::vector<int32_t> witness;
  int32_t dimension = -1, distance_type = -1;
  cee_ctx* jv_ctx = nullptr;
  cee_graph_view view{};

  // Returns true when the static content equals the previous Bind's. Each element is compared
  // and stored in the same pass (an OR of XORs), on the OpenMP team for large snapshots.
  bool Bind(const GraphSnapshot& graph, bool with_edges) {
    const int64_t n = static_cast<int64_t>(graph.points.size());
    const int64_t m = with_edges ? static_cast<int64_t>(graph.edges.size()) : 0;
    const bool sized = static_cast<int64_t>(x.size()) == n && static_cast<int64_t>(u.size()) == m &&
                       dimension == graph.dimension && distance_type == static_cast<int32_t>(graph.distance_type);
    x.resize(static_cast<size_t>(n));
    y.resize(static_cast<size_t>(n));
    u.resize(static_cast<size_t>(m));
    v.resize(static_cast<size_t>(m));
    w.resize(static_cast<size_t>(m));
    active.resize(static_cast<size_t>(m));
    const Point* pts = graph.points.data();
    const Edge* eds = graph.edges.data();
    int64_t* px = x.data();
    int64_t* py = y.data();
    int32_t* pu = u.data();
    int32_t* pv = v.data();
    int64_t* pw = w.data();
    uint8_t* pa = active.data();
    uint64_t diff = 0;
#pragma omp parallel for schedule(static) reduction(| : diff) if (n + m > kParallelElements)
    for (int64_t i = 0; i < n + m; ++i) {
      if (i < n) {
        const int64_t a = pts[i].integer_x, b = pts[i].integer_y;
        diff |= static_cast<uint64_t>(px[i] ^ a) | static_cast<uint64_t>(py[i] ^ b);
        px[i] = a;
        py[i] = b;
      } else {
        const int64_t e = i - n;
        const Edge& edge = eds[e];
        diff |= static_cast<uint64_t>(static_cast<uint32_t>(pu[e] ^ edge.u) | static_cast<uint32_t>(pv[e] ^ edge.v)) |
                static_cast<uint64_t>(pw[e] ^ edge.weight);
        pu[e] = edge.u;
        pv[e] = edge.v;
        pw[e] = edge.weight;
        pa[e] = edge.active ? 1 : 0;
      }
    }
    const bool same = sized && diff == 0;
    dimension = graph.dimension;
    distance_type = static_cast<int32_t>(graph.distance_type);
    if (!same) jv_ctx = nullptr;
    view = cee_graph_view{};
    view.n = graph.dimension;
    view.dist_type = static_cast<int32_t>(graph.distance_type);
    view.x = x.data();
    view.y = y.data();
    view.m = static_cast<int64_t>(m);
    view.edge_u = u.data();
    view.edge_v = v.data();
    view.edge_w = w.data();
    view.active = active.data();
    view.adjacency = static_cast<int64_t>(graph.neighbors.size());
    view.row_offsets = graph.row_offsets.data();
    view.neighbors = graph.neighbors.data();
    view.csr_edge_ids = graph.csr_edge_ids.data();
    return same;
  }
};

thread_local SnapshotArrays g_arrays;

}  // namespace

bool CudaBackendAvailable(std::string* const reason) { return SelectDevice(reason) >= 0; }

std::vector<Candidate> FindJvCandidatesCuda(const GraphSnapshot& graph, int* const selected_device,
                                            JvCudaCacheUsage* const cache_usage) {
  if (cache_usage != nullptr) *cache_usage = {};
  if (!graph.integer_coordinates || !graph.integer_distance_safe) {
    throw std::runtime_error("CUDA JV needs integer coordinates whose squared distances fit uint64");
  }
  if (graph.edges.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
    throw std::overflow_error("CUDA JV edge count exceeds the int32 edge-id range");
  }
  cee_ctx* ctx = RequireContext(selected_device, "CUDA JV backend");
  if (graph.edges.empty()) return {};
  const bool same = g_arrays.Bind(graph, true);
  // this context's static cache holds exactly the kept content: skip its second comparison
  const uint32_t hint = same && g_arrays.jv_ctx == ctx ? CEE_JV_STATIC_UNCHANGED : 0u;
  std::vector<int32_t>& witness = g_arrays.witness;
  witness.resize(graph.edges.size());
  cee_jv_stats stats{};
  g_arrays.jv_ctx = nullptr;
  const int status =
      cee_jv_screen_ex(ctx, &g_arrays.view, witness.data(), cache_usage != nullptr ? &stats : nullptr, hint);
  if (status != CEE_OK) Raise(status, ctx, "B200 JV screen");
  g_arrays.jv_ctx = ctx;
  if (cache_usage != nullptr) {
    cache_usage->static_hit = stats.static_hit != 0;
    cache_usage->workspace_hit = stats.workspace_hit != 0;
    // resident_bytes is the figure the reference's callers print and its tests pin: the device
    // bytes of its own layout for this snapshot -- 24 B per edge, 20 B per node plus 4, and 8 B per
    // CSR slot (tests/unit/test_core.cpp:186-192). This build's layout is smaller (int32
    // coordinates and weights); its own allocation is cee_jv_stats.resident_bytes.
    cache_usage->resident_bytes = 24u * static_cast<uint64_t>(graph.edges.size()) +
                                  20u * static_cast<uint64_t>(graph.points.size()) + 4u +
                                  8u * static_cast<uint64_t>(graph.neighbors.size());
    cache_usage->h2d_ms = stats.h2d_ms;
    cache_usage->kernel_ms = stats.kernel_ms;
    cache_usage->d2h_ms = stats.d2h_ms;
  }
  // the edges with a witness, ascending: counted per block of edges, then written at each block's
  // offset (on the OpenMP team for large snapshots)
  const int64_t m = static_cast<int64_t>(witness.size());
  const int64_t blocks = m > kParallelElements ? std::min<int64_t>(4 * omp_get_max_threads(), m / 4096 + 1) : 1;
  std::vector<int64_t> at(static_cast<size_t>(blocks) + 1, 0);
  const int32_t* wit = witness.data();
#pragma omp parallel for schedule(static) if (blocks > 1)
  for (int64_t b = 0; b < blocks; ++b) {
    int64_t count = 0;
    for (int64_t e = m * b / blocks; e < m * (b + 1) / blocks; ++e) count += wit[e] >= 0 ? 1 : 0;
    at[static_cast<size_t>(b) + 1] = count;
  }
  for (int64_t b = 0; b < blocks; ++b) at[static_cast<size_t>(b) + 1] += at[static_cast<size_t>(b)];
  std::vector<Candidate> candidates(static_cast<size_t>(at[static_cast<size_t>(blocks)]));
  Candidate* out = candidates.data();
#pragma omp parallel for schedule(static) if (blocks > 1)
  for (int64_t b = 0; b < blocks; ++b) {
    int64_t k = at[static_cast<size_t>(b)];
    for (int64_t e = m * b / blocks; e < m * (b + 1) / blocks; ++e) {
      if (wit[e] >= 0) out[k++] = Candidate{static_cast<int32_t>(e), wit[e], EliminationMethod::kJv};
    }
  }
  return candidates;
}

void ClearJvCudaCache() {
  for (auto& entry : g_threads.contexts) cee_ctx_clear(entry.second, 1u);
  g_threads.preferred = -1;
  g_arrays.jv_ctx = nullptr;
}

namespace detail {

bool KOptCostCudaAvailable(std::string* const reason) { return SelectDevice(reason) >= 0; }

std::vector<std::int64_t> EvaluateKOptTemplateCostsCuda(const GraphSnapshot& graph,
                                                        const KOptReconnectTable& table,
                                                        const std::vector<KOptCostTask>& tasks,
                                                        int* const selected_device,
                                                        KOptCudaCacheUsage* const cache_usage) {
  static_assert(sizeof(KOptCostTask) == sizeof(cee_kopt_task), "KOptCostTask layout");
  if (cache_usage != nullptr) *cache_usage = {};
  cee_ctx* ctx = RequireContext(selected_device, "CUDA k-opt cost backend");
  if (tasks.empty()) return {};
  if (table.k < 3U || table.k > 5U || table.templates.empty()) {
    throw std::invalid_argument("CUDA k-opt reconnect table is invalid");
  }
  std::vector<uint8_t> mates(table.templates.size() * 14, 0xff);
  for (size_t t = 0; t < table.templates.size(); ++t) {
    std::memcpy(mates.data() + 14 * t, table.templates[t].mate.data(), 14);
  }
  g_arrays.Bind(graph, false);
  std::vector<int64_t> costs(tasks.size() * table.templates.size());
  cee_kopt_stats stats{};
  const int status = cee_kopt_costs(ctx, graph.dimension, static_cast<int32_t>(graph.distance_type),
                                    g_arrays.x.data(), g_arrays.y.data(), table.k, mates.data(),
                                    static_cast<int32_t>(table.templates.size()), table.generator_hash,
                                    reinterpret_cast<const cee_kopt_task*>(tasks.data()),
                                    static_cast<int64_t>(tasks.size()), costs.data(), &stats);
  if (status != CEE_OK) Raise(status, ctx, "B200 k-opt cost matrix");
  if (cache_usage != nullptr) {
    cache_usage->snapshot_hit = stats.snapshot_hit != 0;
    cache_usage->template_hit = stats.template_hit != 0;
    cache_usage->workspace_hit = stats.workspace_hit != 0;
    cache_usage->resident_bytes = stats.resident_bytes;
  }
  return costs;
}

void ClearKOptCostCudaCache() {
  for (auto& entry : g_threads.contexts) cee_ctx_clear(entry.second, 2u);
}

bool HtCdCudaAvailable(std::string* const reason) { return SelectDevice(reason) >= 0; }

std::vector<std::uint8_t> ScreenHtCdCandidatesCuda(const GraphSnapshot& graph, const NodeEdge target_edge,
                                                   const std::vector<HtCdScreenTask>& tasks,
                                                   const HtCdMode mode, int* const selected_device) {
  static_assert(sizeof(HtCdScreenTask) == sizeof(cee_cd_task), "HtCdScreenTask layout");
  if (target_edge.u < 0 || target_edge.v >= graph.dimension || target_edge.u >= target_edge.v ||
      (mode != HtCdMode::kActiveIncompatible && mode != HtCdMode::kMissingOrIncompatible)) {
    throw std::invalid_argument("CUDA HT c,d input is invalid");
  }
  cee_ctx* ctx = RequireContext(selected_device, "CUDA HT c,d backend");
  if (tasks.empty()) return {};
  g_arrays.Bind(graph, true);
  std::vector<uint8_t> flags(tasks.size());
  const int status = cee_cd_screen(ctx, &g_arrays.view, target_edge.u, target_edge.v,
                                   reinterpret_cast<const cee_cd_task*>(tasks.data()),
                                   static_cast<int64_t>(tasks.size()), static_cast<int32_t>(mode), flags.data());
  if (status != CEE_OK) Raise(status, ctx, "B200 HT c,d screen");
  return flags;
}

bool HtHamiltonReplyCudaAvailable(std::string* const reason) { return SelectDevice(reason) >= 0; }

HtHamiltonReplyDeviceBatch EvaluateHtHamiltonRepliesCuda(const GraphSnapshot& graph, const NodeEdge target_edge,
                                                         const std::vector<std::int32_t>& centers,
                                                         int* const selected_device,
                                                         HtReplyCudaCacheUsage* const cache_usage) {
  static_assert(sizeof(HtNeighborPair) == sizeof(cee_ht_pair), "HtNeighborPair layout");
  if (cache_usage != nullptr) *cache_usage = {};
  cee_ctx* ctx = RequireContext(selected_device, "CUDA HT reply backend");
  g_arrays.Bind(graph, true);
  HtHamiltonReplyDeviceBatch result;
  result.offsets.assign(centers.size() + 1U, 0U);
  cee_ht_reply_stats stats{};
  int status = cee_ht_replies(ctx, &g_arrays.view, target_edge.u, target_edge.v, centers.data(),
                              static_cast<int64_t>(centers.size()), result.offsets.data(), &stats);
  if (status != CEE_OK) Raise(status, ctx, "B200 HT Hamilton replies");
  result.replies.resize(static_cast<size_t>(result.offsets.back()));
  status = cee_ht_replies_fetch(ctx, result.replies.data());
  if (status != CEE_OK) Raise(status, ctx, "B200 HT Hamilton reply download");
  if (cache_usage != nullptr) {
    cache_usage->graph_hit = stats.graph_hit != 0;
    cache_usage->workspace_hit = stats.workspace_hit != 0;
    cache_usage->resident_bytes = stats.resident_bytes;
  }
  return result;
}

bool HtEndReplyCudaAvailable(std::string* const reason) { return SelectDevice(reason) >= 0; }

HtEndReplyDeviceBatch EvaluateHtEndRepliesCuda(const GraphSnapshot& graph, const std::vector<HtEndReplyTask>& tasks,
                                               int* const selected_device, HtReplyCudaCacheUsage* const cache_usage) {
  static_assert(sizeof(HtEndReplyTask) == sizeof(cee_ht_end_task), "HtEndReplyTask layout");
  static_assert(sizeof(NodeEdge) == sizeof(cee_node_edge), "NodeEdge layout");
  if (cache_usage != nullptr) *cache_usage = {};
  cee_ctx* ctx = RequireContext(selected_device, "CUDA HT end reply backend");
  g_arrays.Bind(graph, true);
  HtEndReplyDeviceBatch result;
  result.offsets.assign(tasks.size() + 1U, 0U);
  cee_ht_reply_stats stats{};
  int status = cee_ht_end_replies(ctx, &g_arrays.view, reinterpret_cast<const cee_ht_end_task*>(tasks.data()),
                                  static_cast<int64_t>(tasks.size()), result.offsets.data(), &stats);
  if (status != CEE_OK) Raise(status, ctx, "B200 HT end replies");
  result.replies.resize(static_cast<size_t>(result.offsets.back()));
  status = cee_ht_replies_fetch(ctx, result.replies.data());
  if (status != CEE_OK) Raise(status, ctx, "B200 HT end reply download");
  if (cache_usage != nullptr) {
    cache_usage->graph_hit = stats.graph_hit != 0;
    cache_usage->workspace_hit = stats.workspace_hit != 0;
    cache_usage->resident_bytes = stats.resident_bytes;
  }
  return result;
}

void ClearHtReplyCudaCache() {
  for (auto& entry : g_threads.contexts) cee_ctx_clear(entry.second, 64u);
}

bool HtWavefrontCudaAvailable(std::string* const reason) {
  if (reason != nullptr) *reason = "HT wavefront propagation is not part of the B200 screen backend";
  return false;
}

HtWavefrontDeviceResult EvaluateHtWavefrontCuda(const std::vector<HtWavefrontStateTask>&,
                                                const std::vector<HtWavefrontMoveTask>&,
                                                const std::vector<HtWavefrontReplyTask>&,
                                                const std::vector<std::uint32_t>&, std::uint32_t, int*) {
  throw std::runtime_error("HT wavefront propagation is not part of the B200 screen backend");
}

}  // namespace detail
}  // namespace cudaee
