// Test infrastructure (oracle). A flat extern "C" view of the reference library's own CPU
// entry points, so that pytest can drive the reference through ctypes. Linked into
// oracle/_ref/libcudaee_ref.so (reference CUDA seam = the reference's stubs), into
// oracle/_ref/libcudaee_dropin.so (reference CUDA seam = this project's shim) and into
// oracle/_ref/libcudaee_refcuda.so (reference CUDA seam = the reference's own CUDA units).
//
// Every function returns 0 on success and a negative value when the reference threw; the
// message is then available from ref_last_error().
#include "cuda_edge_elimination/distance.hpp"
#include "cuda_edge_elimination/elimination.hpp"
#include "cuda_edge_elimination/graph.hpp"
#include "cuda_edge_elimination/hamilton_tutte.hpp"
#include "cuda_edge_elimination/local_search.hpp"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <limits>
#include <string>
#include <vector>

#include <omp.h>

namespace {

thread_local std::string g_error;

template <typename F> int Guard(F&& body) {
  try {
    return body();
  } catch (const std::exception& error) {
    g_error = error.what();
    return -1;
  } catch (...) {
    g_error = "unknown exception";
    return -1;
  }
}

cudaee::GraphSnapshot* AsGraph(void* handle) { return static_cast<cudaee::GraphSnapshot*>(handle); }

static_assert(sizeof(cudaee::KOptCostTask) == 48, "KOptCostTask layout");
static_assert(sizeof(cudaee::HtCdScreenTask) == 12, "HtCdScreenTask layout");

} // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

uint64_t ref_isqrt(uint64_t value) { return cudaee::IntegerSqrtFloor(value); }

// Exact TSPLIB distance between two integer points (src/common/distance.cpp:29-68).
int ref_exact_distance(int64_t x1, int64_t y1, int64_t x2, int64_t y2, int type, int64_t* out) {
  cudaee::Point a{static_cast<double>(x1), static_cast<double>(y1), x1, y1};
  cudaee::Point b{static_cast<double>(x2), static_cast<double>(y2), x2, y2};
  std::string error;
  if (!cudaee::ExactIntegerDistance(a, b, static_cast<cudaee::DistanceType>(type), out, &error)) {
    g_error = error;
    return -1;
  }
  return 0;
}

// Builds a GraphSnapshot the way GraphSnapshot::Load does after parsing
// (src/common/graph.cpp:98-228): integer coordinates, integer_distance_safe from the
// bounding box, edges kept in the caller's order (so unsorted snapshots exercise the CSR
// sort fallback), weights = exact distance when w is null, then RebuildCsr().
int ref_graph_new(int32_t n, int dist_type, const int64_t* x, const int64_t* y, int64_t m,
                  const int32_t* eu, const int32_t* ev, const int64_t* w, const uint8_t* active,
                  void** out) {
  return Guard([&] {
    auto graph = std::make_unique<cudaee::GraphSnapshot>();
    graph->dimension = n;
    graph->distance_type = static_cast<cudaee::DistanceType>(dist_type);
    graph->integer_coordinates = true;
    graph->points.resize(static_cast<std::size_t>(n));
    int64_t min_x = 0, max_x = 0, min_y = 0, max_y = 0;
    for (int32_t i = 0; i < n; ++i) {
      graph->points[i] = {static_cast<double>(x[i]), static_cast<double>(y[i]), x[i], y[i]};
      if (i == 0 || x[i] < min_x) min_x = x[i];
      if (i == 0 || x[i] > max_x) max_x = x[i];
      if (i == 0 || y[i] < min_y) min_y = y[i];
      if (i == 0 || y[i] > max_y) max_y = y[i];
    }
    const __int128 dx = static_cast<__int128>(max_x) - min_x;
    const __int128 dy = static_cast<__int128>(max_y) - min_y;
    graph->integer_distance_safe = dx * dx + dy * dy <= std::numeric_limits<uint64_t>::max();
    graph->edges.resize(static_cast<std::size_t>(m));
    for (int64_t e = 0; e < m; ++e) {
      cudaee::Edge& edge = graph->edges[e];
      edge.u = eu[e];
      edge.v = ev[e];
      edge.weight = w != nullptr ? w[e] : graph->Distance(edge.u, edge.v);
      edge.active = active == nullptr || active[e] != 0;
    }
    graph->RebuildCsr();
    *out = graph.release();
    return 0;
  });
}

void ref_graph_free(void* handle) { delete AsGraph(handle); }

int ref_graph_set_active(void* handle, const uint8_t* active) {
  return Guard([&] {
    cudaee::GraphSnapshot* graph = AsGraph(handle);
    for (std::size_t e = 0; e < graph->edges.size(); ++e) graph->edges[e].active = active[e] != 0;
    graph->RebuildCsr();
    return 0;
  });
}

void ref_graph_sizes(void* handle, int64_t* m, int64_t* adjacency) {
  *m = static_cast<int64_t>(AsGraph(handle)->edges.size());
  *adjacency = static_cast<int64_t>(AsGraph(handle)->neighbors.size());
}

void ref_graph_csr(void* handle, int32_t* row_offsets, int32_t* neighbors, int32_t* csr_edge_ids,
                   int64_t* csr_weights) {
  const cudaee::GraphSnapshot* graph = AsGraph(handle);
  std::copy(graph->row_offsets.begin(), graph->row_offsets.end(), row_offsets);
  std::copy(graph->neighbors.begin(), graph->neighbors.end(), neighbors);
  std::copy(graph->csr_edge_ids.begin(), graph->csr_edge_ids.end(), csr_edge_ids);
  std::copy(graph->csr_weights.begin(), graph->csr_weights.end(), csr_weights);
}

void ref_graph_active(void* handle, uint8_t* active) {
  const cudaee::GraphSnapshot* graph = AsGraph(handle);
  for (std::size_t e = 0; e < graph->edges.size(); ++e) active[e] = graph->edges[e].active ? 1 : 0;
}

uint64_t ref_graph_hash(void* handle) { return AsGraph(handle)->ContentHash(); }

// FindJvCandidatesCpu (src/cpu/jv_elimination.cpp:209-224) as a per-edge witness array.
int ref_jv_cpu(void* handle, int32_t* witness_per_edge) {
  return Guard([&] {
    const cudaee::GraphSnapshot* graph = AsGraph(handle);
    std::fill(witness_per_edge, witness_per_edge + graph->edges.size(), -1);
    const auto candidates = cudaee::FindJvCandidatesCpu(*graph);
    for (const auto& c : candidates) witness_per_edge[c.edge_id] = c.witness;
    return static_cast<int>(candidates.size());
  });
}

// FindJvCandidatesCuda through whatever CUDA seam this library was linked with
// (stubs throw; the drop-in shim calls the B200 kernels). Candidates must come back in
// ascending edge id, which is checked here as the reference's callers rely on it.
int ref_jv_cuda(void* handle, int32_t* witness_per_edge, int32_t* usage /*[3] static,ws,-*/,
                uint64_t* resident_bytes) {
  return Guard([&] {
    const cudaee::GraphSnapshot* graph = AsGraph(handle);
    std::fill(witness_per_edge, witness_per_edge + graph->edges.size(), -1);
    int device = -1;
    cudaee::JvCudaCacheUsage cache;
    const auto candidates = cudaee::FindJvCandidatesCuda(*graph, &device, &cache);
    int32_t previous = -1;
    for (const auto& c : candidates) {
      if (c.edge_id <= previous || c.method != cudaee::EliminationMethod::kJv) {
        g_error = "CUDA JV candidates are not in strictly ascending edge id";
        return -2;
      }
      previous = c.edge_id;
      witness_per_edge[c.edge_id] = c.witness;
    }
    if (usage != nullptr) {
      usage[0] = cache.static_hit ? 1 : 0;
      usage[1] = cache.workspace_hit ? 1 : 0;
      usage[2] = device;
    }
    if (resident_bytes != nullptr) *resident_bytes = cache.resident_bytes;
    return static_cast<int>(candidates.size());
  });
}

void ref_jv_clear_cuda_cache() { cudaee::ClearJvCudaCache(); }

int ref_cuda_available(char* reason, int reason_capacity) {
  std::string why;
  const bool ok = cudaee::CudaBackendAvailable(&why);
  if (reason != nullptr && reason_capacity > 0) {
    std::snprintf(reason, static_cast<std::size_t>(reason_capacity), "%s", why.c_str());
  }
  return ok ? 1 : 0;
}

int ref_jv_verify(void* handle, int32_t edge_id, int32_t witness) {
  std::string reason;
  return cudaee::VerifyJvCandidate(*AsGraph(handle), {edge_id, witness, cudaee::EliminationMethod::kJv},
                                   &reason)
             ? 1
             : 0;
}

// RunJvElimination (src/cpu/jv_elimination.cpp:250-322) on the snapshot in place.
// backend: 1 = kCpu, 2 = kCuda. Per-epoch edges_before/proposed/committed go to
// epoch_stats[3*e..3*e+2]; proof records (epoch, edge_id, witness) to records[3*r..].
int ref_run_jv(void* handle, int backend, uint32_t max_rounds, int64_t* epoch_stats,
               int32_t epoch_capacity, int32_t* records, int64_t record_capacity,
               int64_t* record_count, uint64_t* initial_hash, uint64_t* final_hash) {
  return Guard([&] {
    const cudaee::Backend b = backend == 2 ? cudaee::Backend::kCuda : cudaee::Backend::kCpu;
    const cudaee::EliminationResult result = cudaee::RunJvElimination(AsGraph(handle), b, max_rounds);
    const int32_t epochs = static_cast<int32_t>(result.epochs.size());
    for (int32_t e = 0; e < epochs && e < epoch_capacity; ++e) {
      epoch_stats[3 * e] = static_cast<int64_t>(result.epochs[e].edges_before);
      epoch_stats[3 * e + 1] = static_cast<int64_t>(result.epochs[e].proposed);
      epoch_stats[3 * e + 2] = static_cast<int64_t>(result.epochs[e].committed);
    }
    *record_count = static_cast<int64_t>(result.proof.size());
    for (std::size_t r = 0; r < result.proof.size() && static_cast<int64_t>(r) < record_capacity; ++r) {
      records[3 * r] = static_cast<int32_t>(result.proof[r].epoch);
      records[3 * r + 1] = result.proof[r].edge_id;
      records[3 * r + 2] = result.proof[r].witness;
    }
    *initial_hash = result.initial_hash;
    *final_hash = result.final_hash;
    return epochs;
  });
}

// RunJvElimination(kCpu) on the snapshot in place, then WriteProof (src/cpu/jv_elimination.cpp:324-368)
// of the run to `path`. Returns the epoch count.
int ref_write_proof_cpu(void* handle, uint32_t max_rounds, const char* path) {
  return Guard([&] {
    const cudaee::EliminationResult result =
        cudaee::RunJvElimination(AsGraph(handle), cudaee::Backend::kCpu, max_rounds);
    cudaee::WriteProof(path, result);
    return static_cast<int>(result.epochs.size());
  });
}

// GraphSnapshot::WriteActiveEdges (src/common/graph.cpp:284-298) of the snapshot as it stands.
int ref_write_active_edges(void* handle, const char* path) {
  return Guard([&] {
    AsGraph(handle)->WriteActiveEdges(path);
    return 0;
  });
}

// ReadProof(path), then ReplayProof (src/cpu/jv_elimination.cpp:525-600) on a copy of the snapshot:
// the number of records replayed, or -1 with the reference's reason when it rejects the proof.
int ref_replay_proof_file(void* handle, const char* path) {
  return Guard([&] {
    cudaee::GraphSnapshot working = *AsGraph(handle);
    const cudaee::EliminationResult expected = cudaee::ReadProof(path);
    const cudaee::EliminationResult replayed = cudaee::ReplayProof(&working, expected);
    return static_cast<int>(replayed.proof.size());
  });
}

// BuildKOptReconnectTable (src/cpu/kopt_search.cpp:1143-1193): mates[t*14 + p].
int ref_kopt_table(uint32_t k, uint8_t* mates, uint64_t* hash) {
  return Guard([&] {
    const cudaee::KOptReconnectTable table = cudaee::BuildKOptReconnectTable(k);
    for (std::size_t t = 0; t < table.templates.size(); ++t) {
      std::memcpy(mates + 14 * t, table.templates[t].mate.data(), 14);
    }
    *hash = table.generator_hash;
    return static_cast<int>(table.templates.size());
  });
}

// EvaluateKOptTemplateCosts (src/cpu/kopt_search.cpp:1435-1488). backend: 1 = kCpu,
// 2 = kCuda (drop-in only; the reference then certifies every cell against its CPU matrix).
// meta[0] = cpu threads used, meta[1] = selected device, meta[2..4] = snapshot/template/
// workspace cache hits.
int ref_kopt_costs(void* handle, uint32_t k, const void* tasks, int64_t rows, int backend,
                   int64_t* costs, int64_t* meta) {
  return Guard([&] {
    std::vector<cudaee::KOptCostTask> list(static_cast<std::size_t>(rows));
    std::memcpy(list.data(), tasks, sizeof(cudaee::KOptCostTask) * list.size());
    const auto b = backend == 2 ? cudaee::PathCompatibilityBackend::kCuda
                                : cudaee::PathCompatibilityBackend::kCpu;
    const cudaee::KOptCostBatchResult result =
        cudaee::EvaluateKOptTemplateCosts(*AsGraph(handle), k, list, b);
    std::copy(result.added_costs.begin(), result.added_costs.end(), costs);
    if (meta != nullptr) {
      meta[0] = result.cpu_threads_used;
      meta[1] = result.selected_device;
      meta[2] = result.cuda_cache.snapshot_hit;
      meta[3] = result.cuda_cache.template_hit;
      meta[4] = result.cuda_cache.workspace_hit;
    }
    return static_cast<int>(result.template_count);
  });
}

void ref_kopt_clear_cuda_cache() { cudaee::detail::ClearKOptCostCudaCache(); }

// The CUDA seam calls themselves, timed on the host (steady clock around each call; each call
// returns its results to host memory, so it includes its uploads, launch and download). With
// libcudaee_refcuda.so they run the reference's own kernels, with libcudaee_dropin.so this
// project's: the same reference API either way. ms[i] = duration of call i; the first call (its
// caches cold) is reported too.

// FindJvCandidatesCuda (include/cuda_edge_elimination/elimination.hpp:333-338), `reps` calls on
// one snapshot; the last call's witnesses per edge.
int ref_seam_jv_timed(void* handle, int32_t reps, double* ms, int32_t* witness_per_edge) {
  return Guard([&] {
    const cudaee::GraphSnapshot* graph = AsGraph(handle);
    std::vector<cudaee::Candidate> candidates;
    for (int32_t i = 0; i < reps; ++i) {
      int device = -1;
      const auto t0 = std::chrono::steady_clock::now();
      candidates = cudaee::FindJvCandidatesCuda(*graph, &device, nullptr);
      ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    std::fill(witness_per_edge, witness_per_edge + graph->edges.size(), -1);
    for (const auto& c : candidates) witness_per_edge[c.edge_id] = c.witness;
    return static_cast<int>(candidates.size());
  });
}

// detail::EvaluateKOptTemplateCostsCuda (local_search.hpp:235-242) with the proper templates of
// k, `reps` calls (no CPU certification: that belongs to the dispatcher around the seam); the
// last call's cost matrix.
int ref_seam_kopt_timed(void* handle, uint32_t k, const void* tasks, int64_t rows, int32_t reps, double* ms,
                        int64_t* costs) {
  return Guard([&] {
    std::vector<cudaee::KOptCostTask> list(static_cast<std::size_t>(rows));
    std::memcpy(list.data(), tasks, sizeof(cudaee::KOptCostTask) * list.size());
    const cudaee::KOptReconnectTable table = cudaee::BuildKOptReconnectTable(k);
    std::vector<std::int64_t> out;
    for (int32_t i = 0; i < reps; ++i) {
      int device = -1;
      cudaee::KOptCudaCacheUsage cache;
      const auto t0 = std::chrono::steady_clock::now();
      out = cudaee::detail::EvaluateKOptTemplateCostsCuda(*AsGraph(handle), table, list, &device, &cache);
      ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    std::copy(out.begin(), out.end(), costs);
    return static_cast<int>(table.templates.size());
  });
}

// The OpenMP thread count of the calling thread's next parallel regions (omp_set_num_threads):
// EvaluateKOptTemplateCosts(kCpu) uses min(kKOptCpuMaxThreads = 8, this, the processor count)
// threads (src/cpu/kopt_search.cpp:37-40, 1069-1089).
void ref_set_omp_threads(int threads) { omp_set_num_threads(threads > 0 ? threads : 1); }

// Snapshots of every instance of a disjoint union (instance i owns nodes [node_begin[i],
// node_begin[i+1]) and edges [edge_begin[i], edge_begin[i+1]), global ids), each built through
// ref_graph_new with local ids, for callers that build every snapshot before a timed region.
int ref_graph_new_many(int32_t count, int dist_type, const int64_t* node_begin, const int64_t* edge_begin,
                       const int64_t* x, const int64_t* y, const int32_t* eu, const int32_t* ev,
                       const int64_t* w, const uint8_t* active, void** out) {
  std::vector<int32_t> local_u, local_v;
  for (int32_t i = 0; i < count; ++i) {
    const int64_t n0 = node_begin[i], e0 = edge_begin[i], m = edge_begin[i + 1] - e0;
    local_u.resize(static_cast<std::size_t>(m));
    local_v.resize(static_cast<std::size_t>(m));
    for (int64_t e = 0; e < m; ++e) {
      local_u[e] = static_cast<int32_t>(eu[e0 + e] - n0);
      local_v[e] = static_cast<int32_t>(ev[e0 + e] - n0);
    }
    const int rc = ref_graph_new(static_cast<int32_t>(node_begin[i + 1] - n0), dist_type, x + n0, y + n0, m,
                                 local_u.data(), local_v.data(), w + e0, active + e0, &out[i]);
    if (rc != 0) {
      for (int32_t j = 0; j < i; ++j) delete AsGraph(out[j]);
      return rc;
    }
  }
  return 0;
}

// EvaluateHtCdCandidates (src/cpu/hamilton_tutte.cpp:662-704). backend: 1 = kCpu, 2 = kCuda.
// out[3*i..] = (c, d, reply_product clipped to int64).
int ref_cd_candidates(void* handle, int32_t u, int32_t v, uint32_t max_neighborhood,
                      uint32_t max_cd_candidates, uint32_t max_candidate_degree, int mode,
                      int backend, int64_t* out, int32_t capacity) {
  return Guard([&] {
    cudaee::HtShallowOptions options;
    options.max_neighborhood = max_neighborhood;
    options.max_cd_candidates = max_cd_candidates;
    options.max_candidate_degree = max_candidate_degree;
    options.cd_mode = static_cast<cudaee::HtCdMode>(mode);
    options.candidate_backend = backend == 2 ? cudaee::PathCompatibilityBackend::kCuda
                                             : cudaee::PathCompatibilityBackend::kCpu;
    const cudaee::HtCdBatchResult result =
        cudaee::EvaluateHtCdCandidates(*AsGraph(handle), {u, v}, options);
    const int32_t count = static_cast<int32_t>(result.candidates.size());
    for (int32_t i = 0; i < count && i < capacity; ++i) {
      out[3 * i] = result.candidates[i].c;
      out[3 * i + 1] = result.candidates[i].d;
      out[3 * i + 2] = static_cast<int64_t>(
          std::min<uint64_t>(result.candidates[i].reply_product, INT64_MAX));
    }
    return count;
  });
}

// EvaluateHtHamiltonReplies (src/cpu/hamilton_tutte.cpp:604-611; backend 1 = kCpu, 2 = kCuda: its
// CUDA seam, whose lists the reference compares with its CPU lists before returning) for target
// (u, v) and `count` centers: offsets[count + 1], replies[3 i ..] = (center, first, second) for the
// first `capacity` replies, *total = their number, *used = 2 when the result came from the CUDA
// seam, 1 from the CPU, 0 from the CPU fallback.
int ref_ht_hamilton_replies(void* handle, int32_t u, int32_t v, const int32_t* centers, int64_t count, int backend,
                            int dedup, uint64_t* offsets, int32_t* replies, int64_t capacity, int64_t* total,
                            int32_t* used) {
  return Guard([&] {
    const std::vector<std::int32_t> list(centers, centers + count);
    const auto b = backend == 2 ? cudaee::PathCompatibilityBackend::kCuda : cudaee::PathCompatibilityBackend::kCpu;
    const cudaee::HtHamiltonReplyBatchResult result =
        cudaee::EvaluateHtHamiltonReplies(*AsGraph(handle), {u, v}, list, b, dedup != 0);
    std::copy(result.offsets.begin(), result.offsets.end(), offsets);
    const int64_t n = static_cast<int64_t>(result.replies.size());
    for (int64_t i = 0; i < n && i < capacity; ++i) {
      replies[3 * i] = result.replies[i].center;
      replies[3 * i + 1] = result.replies[i].first;
      replies[3 * i + 2] = result.replies[i].second;
    }
    *total = n;
    *used = result.backend == "cuda" ? 2 : (result.backend == "cpu" ? 1 : 0);
    return 0;
  });
}

// EvaluateHtEndReplies (src/cpu/hamilton_tutte.cpp:625-631), as ref_ht_hamilton_replies; tasks are
// (endpoint, internal neighbour) pairs and replies (lower, higher) node pairs.
int ref_ht_end_replies(void* handle, const int32_t* tasks, int64_t count, int backend, int dedup, uint64_t* offsets,
                       int32_t* replies, int64_t capacity, int64_t* total, int32_t* used) {
  return Guard([&] {
    std::vector<cudaee::HtEndReplyTask> list(static_cast<std::size_t>(count));
    for (int64_t i = 0; i < count; ++i) list[static_cast<std::size_t>(i)] = {tasks[2 * i], tasks[2 * i + 1]};
    const auto b = backend == 2 ? cudaee::PathCompatibilityBackend::kCuda : cudaee::PathCompatibilityBackend::kCpu;
    const cudaee::HtEndReplyBatchResult result = cudaee::EvaluateHtEndReplies(*AsGraph(handle), list, b, dedup != 0);
    std::copy(result.offsets.begin(), result.offsets.end(), offsets);
    const int64_t n = static_cast<int64_t>(result.replies.size());
    for (int64_t i = 0; i < n && i < capacity; ++i) {
      replies[2 * i] = result.replies[i].u;
      replies[2 * i + 1] = result.replies[i].v;
    }
    *total = n;
    *used = result.backend == "cuda" ? 2 : (result.backend == "cpu" ? 1 : 0);
    return 0;
  });
}

// detail::EvaluateHtHamiltonRepliesCuda (include/cuda_edge_elimination/hamilton_tutte.hpp:533-537),
// `reps` calls on the host clock; returns the reply total of the last call.
int ref_seam_ht_replies_timed(void* handle, int32_t u, int32_t v, const int32_t* centers, int64_t count, int32_t reps,
                              double* ms, int64_t* total) {
  return Guard([&] {
    const std::vector<std::int32_t> list(centers, centers + count);
    cudaee::detail::HtHamiltonReplyDeviceBatch batch;
    for (int32_t i = 0; i < reps; ++i) {
      int device = -1;
      const auto t0 = std::chrono::steady_clock::now();
      batch = cudaee::detail::EvaluateHtHamiltonRepliesCuda(*AsGraph(handle), {u, v}, list, &device, nullptr);
      ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    *total = static_cast<int64_t>(batch.replies.size());
    return 0;
  });
}

// SelectHtTargetEdgeIds (src/cpu/ht_scan.cpp:316-345), order 1 = weight descending.
int ref_ht_targets(void* handle, int order, int32_t* out, int32_t capacity) {
  return Guard([&] {
    const auto targets = cudaee::SelectHtTargetEdgeIds(
        *AsGraph(handle),
        order == 1 ? cudaee::HtTargetOrder::kWeightDescending : cudaee::HtTargetOrder::kCanonical);
    const int32_t count = static_cast<int32_t>(targets.size());
    for (int32_t i = 0; i < count && i < capacity; ++i) out[i] = targets[i];
    return count;
  });
}

} // extern "C"
