// Test infrastructure (oracle). The reference keeps its c,d task builder and CPU screen in
// an anonymous namespace of src/cpu/hamilton_tutte.cpp (BuildCdScreenTasks :168-216,
// ScreenCdTasksCpu :218-228). This translation unit compiles that reference source file
// itself (included from the reference tree at build time, not copied) and exposes the two
// functions to ctypes. It replaces hamilton_tutte.cpp in the oracle link, so every other
// symbol of that file is still provided exactly once.
#include "src/cpu/hamilton_tutte.cpp"

#include "cuda_edge_elimination/elimination.hpp"

#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>

extern "C" {

// Tasks for target (u,v): c[i], d[i], active[i]; returns the task count (<= capacity) or -1.
int ref_cd_tasks(void* handle, int32_t u, int32_t v, uint32_t max_neighborhood,
                 uint32_t max_candidate_degree, int32_t* c, int32_t* d, uint8_t* active,
                 int64_t capacity) {
  try {
    const auto* graph = static_cast<const cudaee::GraphSnapshot*>(handle);
    cudaee::HtShallowOptions options;
    options.max_neighborhood = max_neighborhood;
    options.max_candidate_degree = max_candidate_degree;
    const auto tasks = cudaee::BuildCdScreenTasks(*graph, cudaee::NodeEdge{u, v}, options);
    if (static_cast<int64_t>(tasks.size()) > capacity) return -1;
    for (std::size_t i = 0; i < tasks.size(); ++i) {
      c[i] = tasks[i].c;
      d[i] = tasks[i].d;
      active[i] = tasks[i].active;
    }
    return static_cast<int>(tasks.size());
  } catch (...) {
    return -1;
  }
}

// ScreenCdTasksCpu over caller-given tasks; flags[i] in {0,1}.
int ref_cd_screen_cpu(void* handle, int32_t u, int32_t v, const int32_t* c, const int32_t* d,
                      const uint8_t* active, int64_t count, int mode, uint8_t* flags) {
  try {
    const auto* graph = static_cast<const cudaee::GraphSnapshot*>(handle);
    std::vector<cudaee::HtCdScreenTask> tasks(static_cast<std::size_t>(count));
    for (int64_t i = 0; i < count; ++i) tasks[i] = {c[i], d[i], active[i]};
    const auto result = cudaee::ScreenCdTasksCpu(*graph, cudaee::NodeEdge{u, v}, tasks,
                                                 static_cast<cudaee::HtCdMode>(mode));
    std::memcpy(flags, result.data(), result.size());
    return 0;
  } catch (...) {
    return -1;
  }
}

// The reference's CPU code for one step of the batching workload, over prebuilt snapshots (the
// timed CPU baseline; nothing is built or marshalled inside it): per snapshot FindJvCandidatesCpu
// (src/cpu/jv_elimination.cpp:209-224), SelectHtTargetEdgeIds in weight order
// (src/cpu/ht_scan.cpp:316-345) and, for its first `targets` targets, BuildCdScreenTasks +
// ScreenCdTasksCpu (:168-228). Snapshots are taken by `threads` host threads from a shared
// counter. Writes the active edges screened and the c,d tasks screened; returns 0, or -1 when
// the reference threw.
int ref_batch_step(void* const* handles, int32_t count, uint32_t targets, uint32_t max_neighborhood,
                   uint32_t max_candidate_degree, int mode, int32_t threads, int64_t* edges_out,
                   int64_t* cd_tasks_out) {
  std::atomic<int32_t> next{0};
  std::atomic<int64_t> edges{0}, tasks_screened{0};
  std::atomic<bool> failed{false};
  cudaee::HtShallowOptions options;
  options.max_neighborhood = max_neighborhood;
  options.max_candidate_degree = max_candidate_degree;
  const auto work = [&] {
    try {
      int64_t local_edges = 0, local_tasks = 0;
      for (int32_t i = next++; i < count && !failed; i = next++) {
        const auto* graph = static_cast<const cudaee::GraphSnapshot*>(handles[i]);
        const auto candidates = cudaee::FindJvCandidatesCpu(*graph);
        (void)candidates;
        for (const auto& edge : graph->edges) local_edges += edge.active ? 1 : 0;
        const auto ids = cudaee::SelectHtTargetEdgeIds(*graph, cudaee::HtTargetOrder::kWeightDescending);
        const std::size_t used = std::min<std::size_t>(ids.size(), targets);
        for (std::size_t t = 0; t < used; ++t) {
          const cudaee::Edge& e = graph->edges[static_cast<std::size_t>(ids[t])];
          const cudaee::NodeEdge target{e.u, e.v};
          const auto tasks = cudaee::BuildCdScreenTasks(*graph, target, options);
          const auto flags = cudaee::ScreenCdTasksCpu(*graph, target, tasks, static_cast<cudaee::HtCdMode>(mode));
          local_tasks += static_cast<int64_t>(flags.size());
        }
      }
      edges += local_edges;
      tasks_screened += local_tasks;
    } catch (...) {
      failed = true;
    }
  };
  std::vector<std::thread> pool;
  for (int32_t t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  *edges_out = edges;
  *cd_tasks_out = tasks_screened;
  return failed ? -1 : 0;
}

// The same work as ref_batch_step on the calling thread alone, with the two parts timed apart
// (steady clock, accumulated per instance): FindJvCandidatesCpu, and SelectHtTargetEdgeIds +
// BuildCdScreenTasks + ScreenCdTasksCpu. Writes the seconds of each part and what each screened.
int ref_batch_parts_1core(void* const* handles, int32_t count, uint32_t targets, uint32_t max_neighborhood,
                          uint32_t max_candidate_degree, int mode, double* jv_seconds, double* cd_seconds,
                          int64_t* edges_out, int64_t* cd_tasks_out) {
  try {
    cudaee::HtShallowOptions options;
    options.max_neighborhood = max_neighborhood;
    options.max_candidate_degree = max_candidate_degree;
    double jv = 0.0, cd = 0.0;
    int64_t edges = 0, tasks_screened = 0;
    for (int32_t i = 0; i < count; ++i) {
      const auto* graph = static_cast<const cudaee::GraphSnapshot*>(handles[i]);
      const auto t0 = std::chrono::steady_clock::now();
      const auto candidates = cudaee::FindJvCandidatesCpu(*graph);
      const auto t1 = std::chrono::steady_clock::now();
      (void)candidates;
      for (const auto& edge : graph->edges) edges += edge.active ? 1 : 0;
      const auto t2 = std::chrono::steady_clock::now();
      const auto ids = cudaee::SelectHtTargetEdgeIds(*graph, cudaee::HtTargetOrder::kWeightDescending);
      const std::size_t used = std::min<std::size_t>(ids.size(), targets);
      for (std::size_t t = 0; t < used; ++t) {
        const cudaee::Edge& e = graph->edges[static_cast<std::size_t>(ids[t])];
        const cudaee::NodeEdge target{e.u, e.v};
        const auto tasks = cudaee::BuildCdScreenTasks(*graph, target, options);
        const auto flags = cudaee::ScreenCdTasksCpu(*graph, target, tasks, static_cast<cudaee::HtCdMode>(mode));
        tasks_screened += static_cast<int64_t>(flags.size());
      }
      const auto t3 = std::chrono::steady_clock::now();
      jv += std::chrono::duration<double>(t1 - t0).count();
      cd += std::chrono::duration<double>(t3 - t2).count();
    }
    *jv_seconds = jv;
    *cd_seconds = cd;
    *edges_out = edges;
    *cd_tasks_out = tasks_screened;
    return 0;
  } catch (...) {
    return -1;
  }
}

// detail::ScreenHtCdCandidatesCuda (include/cuda_edge_elimination/hamilton_tutte.hpp:527-531)
// over prebuilt snapshots: for each snapshot its first `targets` SelectHtTargetEdgeIds targets,
// their BuildCdScreenTasks lists built before the clock starts, then every (snapshot, target)
// screened through the seam, timed on the host (steady clock around all the calls). Writes the
// seconds, the tasks screened and the flags set (a checksum for comparing two seams).
int ref_seam_cd_timed(void* const* handles, int32_t count, uint32_t targets, uint32_t max_neighborhood,
                      uint32_t max_candidate_degree, int mode, double* seconds, int64_t* tasks_out,
                      int64_t* flags_set) {
  try {
    cudaee::HtShallowOptions options;
    options.max_neighborhood = max_neighborhood;
    options.max_candidate_degree = max_candidate_degree;
    struct Item {
      const cudaee::GraphSnapshot* graph;
      cudaee::NodeEdge target;
      std::vector<cudaee::HtCdScreenTask> tasks;
    };
    std::vector<Item> items;
    for (int32_t i = 0; i < count; ++i) {
      const auto* graph = static_cast<const cudaee::GraphSnapshot*>(handles[i]);
      const auto ids = cudaee::SelectHtTargetEdgeIds(*graph, cudaee::HtTargetOrder::kWeightDescending);
      const std::size_t used = std::min<std::size_t>(ids.size(), targets);
      for (std::size_t t = 0; t < used; ++t) {
        const cudaee::Edge& e = graph->edges[static_cast<std::size_t>(ids[t])];
        const cudaee::NodeEdge target{e.u, e.v};
        items.push_back({graph, target, cudaee::BuildCdScreenTasks(*graph, target, options)});
      }
    }
    int64_t screened = 0, set = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (const Item& item : items) {
      int device = -1;
      const auto flags = cudaee::detail::ScreenHtCdCandidatesCuda(*item.graph, item.target, item.tasks,
                                                                  static_cast<cudaee::HtCdMode>(mode), &device);
      screened += static_cast<int64_t>(flags.size());
      for (const std::uint8_t f : flags) set += f;
    }
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *tasks_out = screened;
    *flags_set = set;
    return 0;
  } catch (...) {
    return -1;
  }
}

} // extern "C"
