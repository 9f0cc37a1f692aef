// JV screen that allocates no memory: cee_jv_screen_noalloc (see include/cee.h).
//
// Some callers cannot call cudaMalloc: a host that hands every byte of device memory to its
// own pool or arena and forbids allocation from libraries, and paths that must not allocate
// while they run (a latency-critical loop that has reserved its memory up front, or a process
// working under a hard device-memory quota). For them this entry point screens a snapshot the
// caller already holds in device memory, writes the witnesses into the caller's device buffer,
// and keeps its own working memory in file-scope device arrays of fixed size, so the call
// itself allocates nothing on the device or the host.
//
// Working memory: the CSR slot weights (one int32 per adjacency slot, at most
// kNoAllocMaxSlots) and a status word. Every GPU that loads the library holds these arrays
// (16 MiB + 256 B) until the process exits. Every call shares them and they keep the last
// call's contents: the slot weights are rewritten in full for [0, adjacency) and the status
// words are cleared at the start of each call. Calls whose work overlaps on the GPU (different
// streams, or different host threads on the same device) race on these arrays and must be
// serialised by the caller.
#include "cee.h"
#include "cee_internal.h"
#include "jv_screen.cuh"

#include <algorithm>
#include <mutex>
#include <string>

namespace cee {
namespace {

constexpr int64_t kNoAllocMaxSlots = int64_t{1} << 22;  // 16 MiB of int32 slot weights
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) int32_t g_noalloc_slot_w[kNoAllocMaxSlots];
static __device__ __align__(256) int32_t g_noalloc_status[64];

struct NoAllocDevice {
  bool ready = false;
  int32_t* slot_w = nullptr;
  int32_t* status = nullptr;
  int sms = 0;
  int warp_blocks_per_sm = 1;
};

std::mutex g_noalloc_mutex;
NoAllocDevice g_noalloc_devices[kNoAllocMaxDevices];

// Status bits written by the kernels (0 = valid input).
enum : int32_t {
  kBadCoordinate = 1,
  kBadEdge = 2,
  kBadRowOffsets = 4,
  kBadNeighbor = 8,
  kBadEdgeId = 16,
  kBadRowOrder = 32,  // a CSR row not strictly ascending by neighbour
};

// Validates the caller's device snapshot and builds the slot weights in the scratch array;
// status[1], status[2] receive the largest x and y (the coordinates are >= 0, so these bound the
// spans and select the exact-distance routine).
__global__ void noalloc_prepare(cee_device_graph g, int32_t* __restrict__ slot_w, int32_t* __restrict__ status) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint32_t limit = 1u << 30;
  uint32_t max_x = 0, max_y = 0;
  for (int64_t i = first; i < g.n; i += stride) {
    const uint32_t x = static_cast<uint32_t>(g.xy[2 * i]), y = static_cast<uint32_t>(g.xy[2 * i + 1]);
    if (x >= limit || y >= limit) {
      atomicOr(status, kBadCoordinate);
    } else {
      max_x = max(max_x, x);
      max_y = max(max_y, y);
    }
  }
  max_x = __reduce_max_sync(kFullMask, max_x);
  max_y = __reduce_max_sync(kFullMask, max_y);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(status + 1, static_cast<int32_t>(max_x));
    atomicMax(status + 2, static_cast<int32_t>(max_y));
  }
  for (int64_t i = first; i <= g.n; i += stride) {
    const int32_t here = g.row_offsets[i];
    const bool bad = here < 0 || here > g.adjacency || (i == 0 && here != 0) || (i == g.n && here != g.adjacency) ||
                     (i < g.n && g.row_offsets[i + 1] < here);
    if (bad) atomicOr(status, kBadRowOffsets);
    // rows must ascend by neighbour (the warp screen finds N(a) members by search or lane match);
    // only rows whose bounds are in range are read
    if (i < g.n) {
      const int32_t next = g.row_offsets[i + 1];
      if (here >= 0 && here <= next && next <= g.adjacency) {
        for (int32_t s = here + 1; s < next; ++s) {
          if (g.neighbors[s - 1] >= g.neighbors[s]) {
            atomicOr(status, kBadRowOrder);
            break;
          }
        }
      }
    }
  }
  for (int64_t e = first; e < g.m; e += stride) {
    const int32_t u = g.edge_uv[2 * e], v = g.edge_uv[2 * e + 1];
    if (static_cast<uint32_t>(u) >= static_cast<uint32_t>(g.n) || static_cast<uint32_t>(v) >= static_cast<uint32_t>(g.n) ||
        g.edge_w[e] < 0) {
      atomicOr(status, kBadEdge);
    }
  }
  for (int64_t s = first; s < g.adjacency; s += stride) {
    if (static_cast<uint32_t>(g.neighbors[s]) >= static_cast<uint32_t>(g.n)) atomicOr(status, kBadNeighbor);
    const int32_t id = g.csr_edge_ids[s];
    if (static_cast<uint64_t>(static_cast<uint32_t>(id)) >= static_cast<uint64_t>(g.m)) {
      atomicOr(status, kBadEdgeId);
      slot_w[s] = 0;
    } else {
      slot_w[s] = g.edge_w[id];
    }
  }
}

int NoAllocFail(int code, const std::string& message) { return Fail(nullptr, code, "cee_jv_screen_noalloc: " + message); }

// Once per device, with that device current: the device addresses of the scratch arrays.
// (In host code the arrays' names are host-side stand-ins, not device addresses.)
int NoAllocSetup(int device, NoAllocDevice** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return NoAllocFail(CEE_ERR_NODEVICE, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocDevice& d = g_noalloc_devices[device];
  if (!d.ready) {
    void* slot = nullptr;
    void* status = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&slot, g_noalloc_slot_w);
    if (rc == cudaSuccess) rc = cudaGetSymbolAddress(&status, g_noalloc_status);
    if (rc == cudaSuccess) rc = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device);
    if (rc == cudaSuccess) {
      // the smallest occupancy of the three span classes' instantiations sizes every launch
      d.warp_blocks_per_sm = 1 << 20;
      for (int span = 0; span < kSpanClasses && rc == cudaSuccess; ++span) {
        WithSpan(span, [&](auto S) {
          int blocks = 0;
          rc = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, jv_screen_warp_kernel<S.value>,
                                                             kJvWarpsPerBlock * 32, 0);
          d.warp_blocks_per_sm = std::min(d.warp_blocks_per_sm, blocks);
        });
      }
    }
    if (rc != cudaSuccess) {
      cudaGetLastError();
      return NoAllocFail(CEE_ERR_CUDA, std::string("device set-up: ") + cudaGetErrorString(rc));
    }
    d.slot_w = static_cast<int32_t*>(slot);
    d.status = static_cast<int32_t*>(status);
    d.warp_blocks_per_sm = d.warp_blocks_per_sm < 1 ? 1 : d.warp_blocks_per_sm;
    d.ready = true;
  }
  *out = &d;
  return CEE_OK;
}

// Reads the status word (and, with `bounds`, the two coordinate maxima after it).
int ReadStatus(const NoAllocDevice& d, cudaStream_t stream, const char* stage, int32_t* bounds = nullptr) {
  int32_t words[3] = {0, 0, 0};
  cudaError_t rc = cudaMemcpyAsync(words, d.status, (bounds != nullptr ? 3 : 1) * sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, stream);
  const int32_t& status = words[0];
  if (rc == cudaSuccess) rc = cudaStreamSynchronize(stream);
  if (rc != cudaSuccess) {
    cudaGetLastError();
    return NoAllocFail(CEE_ERR_CUDA, std::string(stage) + ": " + cudaGetErrorString(rc));
  }
  if (status != 0) {
    return NoAllocFail(CEE_ERR_INVALID, std::string(stage) + ": the device snapshot failed validation (status bits " +
                                            std::to_string(status) + ")");
  }
  if (bounds != nullptr) {
    bounds[0] = words[1];
    bounds[1] = words[2];
  }
  return CEE_OK;
}

}  // namespace
}  // namespace cee

extern "C" int cee_jv_screen_noalloc(const cee_device_graph* graph, int32_t* witness_out, void* stream_handle) {
  using namespace cee;
  if (graph == nullptr || (graph->m > 0 && witness_out == nullptr)) return NoAllocFail(CEE_ERR_INVALID, "null argument");
  const cee_device_graph& g = *graph;
  if (g.n < 0 || g.m < 0 || g.adjacency < 0 || (g.dist_type != CEE_EUC_2D && g.dist_type != CEE_CEIL_2D)) {
    return NoAllocFail(CEE_ERR_INVALID, "bad sizes or distance type");
  }
  if (g.m > INT32_MAX || g.n >= INT32_MAX) return NoAllocFail(CEE_ERR_RANGE, "snapshot exceeds the int32 id range");
  if (g.adjacency > kNoAllocMaxSlots) {
    return NoAllocFail(CEE_ERR_RANGE, "adjacency " + std::to_string(g.adjacency) + " exceeds the no-alloc scratch of " +
                                          std::to_string(kNoAllocMaxSlots) + " CSR slots");
  }
  if (g.m == 0) return CEE_OK;
  if (g.xy == nullptr || g.edge_uv == nullptr || g.edge_w == nullptr || g.active == nullptr || g.row_offsets == nullptr ||
      (g.adjacency > 0 && (g.neighbors == nullptr || g.csr_edge_ids == nullptr))) {
    return NoAllocFail(CEE_ERR_INVALID, "null device array");
  }
  if ((reinterpret_cast<uintptr_t>(g.xy) | reinterpret_cast<uintptr_t>(g.edge_uv)) % 8 != 0) {
    return NoAllocFail(CEE_ERR_INVALID, "xy and edge_uv must be 8-byte aligned (int32 pairs)");
  }
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return NoAllocFail(CEE_ERR_NODEVICE, "no current CUDA device");
  }
  NoAllocDevice* d = nullptr;
  int rc = NoAllocSetup(device, &d);
  if (rc != CEE_OK) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);

  cudaError_t status = cudaMemsetAsync(d->status, 0, 3 * sizeof(int32_t), stream);
  if (status == cudaSuccess) {
    const int64_t work = g.adjacency > g.m ? g.adjacency : (g.m > g.n ? g.m : g.n + 1);
    const int blocks = static_cast<int>(std::min<int64_t>((work + 255) / 256, static_cast<int64_t>(d->sms) * 8));
    noalloc_prepare<<<blocks < 1 ? 1 : blocks, 256, 0, stream>>>(g, d->slot_w, d->status);
    status = cudaGetLastError();
  }
  if (status != cudaSuccess) {
    cudaGetLastError();
    return NoAllocFail(CEE_ERR_CUDA, std::string("validation launch: ") + cudaGetErrorString(status));
  }
  int32_t bounds[2] = {0, 0};
  rc = ReadStatus(*d, stream, "validation", bounds);
  if (rc != CEE_OK) return rc;
  const int span = span_class(bounds[0], bounds[1]);

  JvGraph jg{};
  jg.n = g.n;
  jg.dist_type = g.dist_type;
  jg.m = g.m;
  jg.xy = reinterpret_cast<const int2*>(g.xy);
  jg.edge_uv = reinterpret_cast<const int2*>(g.edge_uv);
  jg.edge_w = g.edge_w;
  jg.active = g.active;
  jg.row_offsets = g.row_offsets;
  jg.nbr = g.neighbors;
  jg.slot_w = d->slot_w;
  const int64_t max_blocks = static_cast<int64_t>(d->sms) * d->warp_blocks_per_sm;
  const int blocks = static_cast<int>(std::min<int64_t>((g.m + kJvWarpsPerBlock - 1) / kJvWarpsPerBlock, max_blocks));
  WithSpan(span, [&](auto S) {
    jv_screen_warp_kernel<S.value><<<blocks, kJvWarpsPerBlock * 32, 0, stream>>>(jg, 0, g.m, witness_out, d->status);
  });
  status = cudaGetLastError();
  if (status != cudaSuccess) return NoAllocFail(CEE_ERR_CUDA, std::string("screen launch: ") + cudaGetErrorString(status));
  return ReadStatus(*d, stream, "screen");
}
