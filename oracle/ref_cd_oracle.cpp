// Test infrastructure (oracle). The reference keeps its c,d task builder and CPU screen in
// an anonymous namespace of src/cpu/hamilton_tutte.cpp (BuildCdScreenTasks :168-216,
// ScreenCdTasksCpu :218-228). This translation unit compiles that reference source file
// itself (included from the reference tree at build time, not copied) and exposes the two
// functions to ctypes. It replaces hamilton_tutte.cpp in the oracle link, so every other
// symbol of that file is still provided exactly once.
#include "src/cpu/hamilton_tutte.cpp"

#include <cstring>

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

} // extern "C"
