// Host-side state behind the C ABI (shared by the translation units of libcee.so).
#pragma once

#include "cee.h"
#include "kopt_cost.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <type_traits>
#include <vector>

namespace cee {

// A device allocation that only grows.
struct DevBuf {
  void* ptr = nullptr;
  size_t capacity = 0;
  cudaError_t Reserve(size_t bytes, bool* grew);
  void Release();
};

struct JvState {
  // static key, compared element-wise like the reference (src/cuda/jv_cuda.cu:360-382)
  bool has_static = false;
  int32_t n = 0, dist_type = 0;
  int64_t m = 0;
  std::vector<int64_t> hx, hy, hw;
  std::vector<int32_t> heu, hev;
  DevBuf xy, uv, w32;
  int span = kSpanSmall;  // span class of the coordinates (exact-distance routine)
  // dynamic workspace, refreshed every call
  DevBuf active, ro, nbr, ids, slotw, witness;
  int64_t adjacency = 0;
  int64_t edges_screened = 0;
  int64_t last_h2d_bytes = 0;
  bool prepared = false;
  void Release() {
    for (DevBuf* b : {&xy, &uv, &w32, &active, &ro, &nbr, &ids, &slotw, &witness}) b->Release();
    has_static = false;
    prepared = false;
    hx.clear();
    hy.clear();
    hw.clear();
    heu.clear();
    hev.clear();
  }
};

struct KoptTable {
  uint32_t k = 0;
  uint64_t hash = 0;
  int32_t T = 0;
  std::vector<uint8_t> mates;
  DevBuf pairs;     // T x k pair indices
  DevBuf patterns;  // T: gap patterns on which the template is invalid (kopt_cost.cuh)
  DevBuf validity;  // 32 x ceil(T/32): the same bits by pattern (kopt_rows.cuh)
  bool canonical = false;  // the proper templates of k, byte for byte
  void Release() {
    pairs.Release();
    patterns.Release();
    validity.Release();
    canonical = false;
    k = 0;
    T = 0;
    mates.clear();
  }
};

struct KoptState {
  bool has_coords = false;
  int32_t n = 0, dist_type = 0;
  std::vector<int64_t> hx, hy;
  DevBuf xy;
  int span = kSpanSmall;
  KoptTable user[3];   // caller templates per k (the reference's template cache)
  KoptTable canon[3];  // this library's proper templates per k
  DevBuf tasks, costs;
  DevBuf masks, firsts;  // improving-template sets of the fused leaf consume
  KoptLaunch launch{};
  int32_t segments = 0, tiles = 0;
  int64_t seg_rows[kKoptMaxSegments] = {};
  int32_t seg_T[kKoptMaxSegments] = {};
  int64_t last_h2d_bytes = 0, last_d2h_bytes = 0;
  bool prepared = false;
  void Release() {
    xy.Release();
    tasks.Release();
    costs.Release();
    masks.Release();
    firsts.Release();
    for (KoptTable& t : user) t.Release();
    for (KoptTable& t : canon) t.Release();
    has_coords = false;
    prepared = false;
    hx.clear();
    hy.clear();
  }
};

struct CdState {
  bool has_coords = false;
  int32_t n = 0, dist_type = 0;
  std::vector<int64_t> hx, hy;
  DevBuf xy, tasks, flags;
  int span = kSpanSmall;
  void Release() {
    xy.Release();
    tasks.Release();
    flags.Release();
    has_coords = false;
    hx.clear();
    hy.clear();
  }
};

struct BatchState;
struct ServeState;
struct EpochState;
struct ReplyState;

}  // namespace cee

namespace cee {
// Pinned staging buffers of a context for copies to and from pageable caller memory (host_copy.cu).
constexpr int kStageBuffers = 3;
struct HostStage {
  uint8_t* buf[kStageBuffers] = {};
  cudaEvent_t ev[kStageBuffers] = {};  // the last copy that used each buffer
  bool ready = false;
  void Release();
};
// Device -> caller memory on the context's stream; returns after the data is in `dst`.
cudaError_t CopyToHost(cee_ctx* ctx, void* dst, const void* src, size_t bytes);
// Caller memory -> device on the context's stream; returns once `src` may be reused (the copy to
// the device may still be queued on the stream).
cudaError_t CopyFromHost(cee_ctx* ctx, void* dst, const void* src, size_t bytes);
}  // namespace cee

struct cee_ctx {
  int device = -1;
  int sm_count = 148;
  int jv_kernel = 1;                  // 0 = thread per edge, 1 = warp per edge (default)
  int jv_waves = 4;                   // grid = SMs x resident blocks x waves (thread kernel)
  int occ_jv_thread[cee::kSpanClasses] = {1, 1, 1};  // resident blocks per SM, per span class
  int occ_jv_warp[cee::kSpanClasses] = {1, 1, 1};
  int kopt_rows_per_tile[3] = {0, 0, 0};  // 0 = default tile for k = 3, 4, 5
  int kopt_kernel = 1;                    // 1 = the one-thread-per-row kernel where it applies, 0 = tiled
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[6] = {};
  int32_t* d_error = nullptr;  // device bounds-check word
  int32_t* h_error = nullptr;  // pinned copy
  std::string error;
  cee::JvState jv;
  cee::KoptState kopt;
  cee::CdState cd;
  cee::BatchState* batch = nullptr;
  cee::ServeState* serve = nullptr;
  cee::EpochState* epoch = nullptr;
  cee::ReplyState* replies = nullptr;
  cee::HostStage stage;
};

namespace cee {

// Calls f(std::integral_constant<int, S>{}) with S the span class `span`, so that one call site
// launches the kernel instantiation for that class.
template <typename F>
decltype(auto) WithSpan(int span, F&& f) {
  switch (span) {
    case kSpanSmall:
      return f(std::integral_constant<int, kSpanSmall>{});
    case kSpanNarrow:
      return f(std::integral_constant<int, kSpanNarrow>{});
    default:
      return f(std::integral_constant<int, kSpanWide>{});
  }
}

int Fail(cee_ctx* ctx, int code, const std::string& message);
int CudaFail(cee_ctx* ctx, cudaError_t status, const char* what);
int Activate(cee_ctx* ctx);
int PackCoordinates(cee_ctx* ctx, int32_t n, const int64_t* x, const int64_t* y, std::vector<int2>* out,
                    int* span);
int GridFor(int64_t work, int per_block, int max_blocks);
float EventMs(cudaEvent_t a, cudaEvent_t b);
int CheckDeviceError(cee_ctx* ctx, const char* what);
// Returns rc after the context stream has finished: for error returns once copies from or to caller
// buffers are queued, so that none of them runs after the call returns.
int Drained(cee_ctx* ctx, int rc);
void ReleaseBatch(cee_ctx* ctx);
uint64_t BatchResident(const cee_ctx* ctx);
void ReleaseServe(cee_ctx* ctx, int32_t* error_word = nullptr);
uint64_t ServeResident(const cee_ctx* ctx);
void ReleaseEpoch(cee_ctx* ctx);
uint64_t EpochResident(const cee_ctx* ctx);
void ReleaseReplies(cee_ctx* ctx);
uint64_t RepliesResident(const cee_ctx* ctx);
// Snapshot view checks shared by the entry points (sizes, distance type, edge arrays, CSR offsets).
int ValidateView(cee_ctx* ctx, const cee_graph_view* g);
// Whether v is in u's CSR row (rows ascending by neighbour).
bool HostHasActiveEdge(const cee_graph_view* g, int32_t u, int32_t v);

}  // namespace cee
