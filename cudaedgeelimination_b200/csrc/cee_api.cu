// C ABI of the B200 edge-elimination screen: contexts, resident caches, input validation and
// the launches of the JV, k-opt and c,d kernels. See include/cee.h for the contract.
#include "cee.h"
#include "cee_internal.h"

#include "cd_screen.cuh"
#include "jv_screen.cuh"
#include "kopt_cost.cuh"
#include "kopt_rows.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace cee {

thread_local std::string g_global_error;

int Fail(cee_ctx* ctx, int code, const std::string& message) {
  if (ctx != nullptr) {
    ctx->error = message;
  } else {
    g_global_error = message;
  }
  return code;
}

int CudaFail(cee_ctx* ctx, cudaError_t status, const char* what) {
  cudaGetLastError();  // clear a sticky launch error so the context stays usable
  const int code = status == cudaErrorMemoryAllocation ? CEE_ERR_NOMEM : CEE_ERR_CUDA;
  return Fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(status));
}

cudaError_t DevBuf::Reserve(size_t bytes, bool* grew) {
  if (bytes <= capacity) return cudaSuccess;
  if (grew != nullptr) *grew = true;
  // geometric growth like the reference's workspaces (src/cuda/jv_cuda.cu:432-440)
  const size_t target = std::max(bytes, capacity * 2);
  Release();
  cudaError_t status = cudaMalloc(&ptr, target);
  if (status != cudaSuccess) {
    ptr = nullptr;
    status = cudaMalloc(&ptr, bytes);  // retry without the growth slack
    if (status != cudaSuccess) {
      ptr = nullptr;
      return status;
    }
    capacity = bytes;
    return cudaSuccess;
  }
  capacity = target;
  return cudaSuccess;
}

void DevBuf::Release() {
  if (ptr != nullptr) cudaFree(ptr);
  ptr = nullptr;
  capacity = 0;
}

int Activate(cee_ctx* ctx) {
  if (ctx == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null context");
  const cudaError_t status = cudaSetDevice(ctx->device);
  if (status != cudaSuccess) return CudaFail(ctx, status, "cudaSetDevice");
  return CEE_OK;
}

// Coordinates as int32 offsets from the bounding-box corner; rejects spans >= 2^30.
int PackCoordinates(cee_ctx* ctx, int32_t n, const int64_t* x, const int64_t* y,
                    std::vector<int2>* out, int* span) {
  *span = kSpanSmall;
  if (n <= 0) {
    out->clear();
    return CEE_OK;
  }
  if (x == nullptr || y == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null coordinates");
  int64_t min_x = x[0], max_x = x[0], min_y = y[0], max_y = y[0];
  for (int32_t i = 1; i < n; ++i) {
    min_x = std::min(min_x, x[i]);
    max_x = std::max(max_x, x[i]);
    min_y = std::min(min_y, y[i]);
    max_y = std::max(max_y, y[i]);
  }
  const __int128 span_x = static_cast<__int128>(max_x) - min_x;
  const __int128 span_y = static_cast<__int128>(max_y) - min_y;
  if (span_x >= (__int128{1} << 30) || span_y >= (__int128{1} << 30)) {
    return Fail(ctx, CEE_ERR_RANGE,
                "coordinate span >= 2^30: outside the exact int32 distance range of the kernels");
  }
  *span = span_class(static_cast<int64_t>(span_x), static_cast<int64_t>(span_y));
  out->resize(static_cast<size_t>(n));
  for (int32_t i = 0; i < n; ++i) {
    (*out)[i] = make_int2(static_cast<int32_t>(x[i] - min_x), static_cast<int32_t>(y[i] - min_y));
  }
  return CEE_OK;
}

int ValidateCsr(cee_ctx* ctx, const cee_graph_view* g) {
  if (g->adjacency < 0 || g->adjacency > INT32_MAX) {
    return Fail(ctx, CEE_ERR_RANGE, "CSR adjacency exceeds the int32 slot range");
  }
  if (g->row_offsets == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null row_offsets");
  if (g->adjacency > 0 && (g->neighbors == nullptr || g->csr_edge_ids == nullptr)) {
    return Fail(ctx, CEE_ERR_INVALID, "null CSR arrays");
  }
  if (g->row_offsets[0] != 0 || g->row_offsets[g->n] != g->adjacency) {
    return Fail(ctx, CEE_ERR_INVALID, "row_offsets must start at 0 and end at adjacency");
  }
  for (int32_t i = 0; i < g->n; ++i) {
    if (g->row_offsets[i + 1] < g->row_offsets[i]) {
      return Fail(ctx, CEE_ERR_INVALID, "row_offsets are not non-decreasing");
    }
  }
  return CEE_OK;
}

int ValidateView(cee_ctx* ctx, const cee_graph_view* g) {
  if (g == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null graph view");
  if (g->n < 0 || g->m < 0) return Fail(ctx, CEE_ERR_INVALID, "negative graph size");
  if (g->m > INT32_MAX) return Fail(ctx, CEE_ERR_RANGE, "edge count exceeds the int32 edge-id range");
  if (g->dist_type != CEE_EUC_2D && g->dist_type != CEE_CEIL_2D) {
    return Fail(ctx, CEE_ERR_INVALID, "unknown distance type");
  }
  if (g->m > 0 && (g->edge_u == nullptr || g->edge_v == nullptr || g->edge_w == nullptr ||
                   g->active == nullptr)) {
    return Fail(ctx, CEE_ERR_INVALID, "null edge arrays");
  }
  return ValidateCsr(ctx, g);
}

template <typename T> bool SameArray(const std::vector<T>& cached, const T* data, int64_t count) {
  return static_cast<int64_t>(cached.size()) == count &&
         (count == 0 || std::memcmp(cached.data(), data, sizeof(T) * static_cast<size_t>(count)) == 0);
}

// slot_w[s] = edge_w[ids[s]]; bad ids are recorded and read as 0.
__global__ void gather_slot_weights(const int32_t* __restrict__ ids, int64_t count,
                                    const int32_t* __restrict__ edge_w, int64_t m,
                                    int32_t* __restrict__ slot_w, int32_t* __restrict__ error) {
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s < count;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t id = ids[s];
    if (static_cast<uint64_t>(static_cast<uint32_t>(id)) >= static_cast<uint64_t>(m)) {
      atomicOr(error, 2);
      slot_w[s] = 0;
    } else {
      slot_w[s] = __ldg(edge_w + id);
    }
  }
}

int GridFor(int64_t work, int per_block, int max_blocks) {
  const int64_t blocks = (work + per_block - 1) / per_block;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(blocks, max_blocks)));
}

uint64_t JvResident(const JvState& s) {
  return s.xy.capacity + s.uv.capacity + s.w32.capacity + s.active.capacity + s.ro.capacity +
         s.nbr.capacity + s.ids.capacity + s.slotw.capacity + s.witness.capacity;
}

uint64_t KoptResident(const KoptState& s) {
  uint64_t bytes = s.xy.capacity + s.tasks.capacity + s.costs.capacity + s.masks.capacity + s.firsts.capacity;
  for (const KoptTable& t : s.user) bytes += t.pairs.capacity + t.patterns.capacity;
  for (const KoptTable& t : s.canon) bytes += t.pairs.capacity + t.patterns.capacity;
  return bytes;
}

float EventMs(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    cudaGetLastError();
    return 0.0f;
  }
  return ms;
}

// Resident blocks per SM of every kernel variant (grid sizing).
int QueryOccupancyOne(const void* kernel, int threads, int smem, int* out) {
  int blocks = 0;
  const cudaError_t status = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem);
  *out = std::max(1, blocks);
  return status;
}

cudaError_t QueryOccupancy(cee_ctx* ctx) {
  int bad = 0;
  for (int span = 0; span < kSpanClasses; ++span) {
    WithSpan(span, [&](auto S) {
      bad |= QueryOccupancyOne(reinterpret_cast<const void*>(jv_screen_thread_kernel<S.value>), kJvThreadBlock, 0,
                               &ctx->occ_jv_thread[span]);
      bad |= QueryOccupancyOne(reinterpret_cast<const void*>(jv_screen_warp_kernel<S.value>), kJvWarpsPerBlock * 32,
                               0, &ctx->occ_jv_warp[span]);
    });
  }
  return bad ? cudaErrorInvalidValue : cudaSuccess;
}

// ---------------------------------------------------------------- exact distance --------

template <int kSpan>
static __global__ void distance_pairs_kernel(const int2* __restrict__ xy, const int2* __restrict__ pairs, int64_t count,
                                             int32_t dist_type, int32_t* __restrict__ out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < count; k += stride) {
    const int2 p = __ldg(pairs + k);
    out[k] = static_cast<int32_t>(exact_distance<kSpan>(__ldg(xy + p.x), __ldg(xy + p.y), dist_type));
  }
}

// Largest relative error of sqrt_estimate over the float bit patterns [lo, hi), as the bits of
// a non-negative double (ordered like the value).
static __global__ void root_error_kernel(uint32_t lo, uint32_t hi, unsigned long long* __restrict__ out) {
  double worst = 0.0;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t b = lo + static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < hi; b += stride) {
    const float x = __uint_as_float(static_cast<uint32_t>(b));
    const double root = sqrt(static_cast<double>(x));
    worst = fmax(worst, fabs(static_cast<double>(sqrt_estimate(x)) - root) / root);
  }
  atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(worst)));
}

// ---------------------------------------------------------------- JV --------------------

// flags: CEE_JV_STATIC_UNCHANGED skips the element-wise comparison of the static arrays with the
// cached ones (the caller vouches for them); the sizes and the distance type are compared always.
int JvPrepare(cee_ctx* ctx, const cee_graph_view* g, cee_jv_stats* stats, uint32_t flags = 0) {
  int rc = ValidateView(ctx, g);
  if (rc != CEE_OK) return rc;
  JvState& s = ctx->jv;
  s.prepared = false;
  cudaStream_t st = ctx->stream;
  const bool vouched = (flags & CEE_JV_STATIC_UNCHANGED) != 0;
  const bool static_hit = s.has_static && s.n == g->n && s.dist_type == g->dist_type && s.m == g->m &&
                          (vouched || (SameArray(s.hx, g->x, g->n) && SameArray(s.hy, g->y, g->n) &&
                                       SameArray(s.heu, g->edge_u, g->m) && SameArray(s.hev, g->edge_v, g->m) &&
                                       SameArray(s.hw, g->edge_w, g->m)));
  cudaEventRecord(ctx->ev[0], st);
  int64_t h2d = 0;
  if (!static_hit) {
    s.has_static = false;
    std::vector<int2> xy;
    rc = PackCoordinates(ctx, g->n, g->x, g->y, &xy, &s.span);
    if (rc != CEE_OK) return rc;
    std::vector<int2> uv(static_cast<size_t>(g->m));
    std::vector<int32_t> w32(static_cast<size_t>(g->m));
    for (int64_t e = 0; e < g->m; ++e) {
      if (g->edge_u[e] < 0 || g->edge_u[e] >= g->n || g->edge_v[e] < 0 || g->edge_v[e] >= g->n) {
        return Fail(ctx, CEE_ERR_INVALID, "edge endpoint out of range");
      }
      if (g->edge_w[e] < 0 || g->edge_w[e] > INT32_MAX) {
        return Fail(ctx, CEE_ERR_RANGE, "edge weight outside [0, 2^31)");
      }
      uv[e] = make_int2(g->edge_u[e], g->edge_v[e]);
      w32[e] = static_cast<int32_t>(g->edge_w[e]);
    }
    cudaError_t e1 = s.xy.Reserve(xy.size() * sizeof(int2) + 16, nullptr);
    cudaError_t e2 = s.uv.Reserve(uv.size() * sizeof(int2) + 16, nullptr);
    cudaError_t e3 = s.w32.Reserve(w32.size() * sizeof(int32_t) + 16, nullptr);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      return CudaFail(ctx, e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3), "JV static allocation");
    }
    cudaMemcpyAsync(s.xy.ptr, xy.data(), xy.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.uv.ptr, uv.data(), uv.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.w32.ptr, w32.data(), w32.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st);
    const cudaError_t copy = cudaStreamSynchronize(st);  // host staging vectors die here
    if (copy != cudaSuccess) return CudaFail(ctx, copy, "JV static upload");
    h2d += static_cast<int64_t>(xy.size() * sizeof(int2) + uv.size() * sizeof(int2) + w32.size() * 4);
    s.hx.assign(g->x, g->x + g->n);
    s.hy.assign(g->y, g->y + g->n);
    s.heu.assign(g->edge_u, g->edge_u + g->m);
    s.hev.assign(g->edge_v, g->edge_v + g->m);
    s.hw.assign(g->edge_w, g->edge_w + g->m);
    s.n = g->n;
    s.dist_type = g->dist_type;
    s.m = g->m;
    s.has_static = true;
  }
  bool grew = false;
  const size_t m = static_cast<size_t>(g->m), adj = static_cast<size_t>(g->adjacency);
  cudaError_t status = cudaSuccess;
  for (auto [buf, bytes] : {std::pair<DevBuf*, size_t>{&s.active, m + 16},
                            {&s.ro, (static_cast<size_t>(g->n) + 1) * 4},
                            {&s.nbr, adj * 4 + 16}, {&s.ids, adj * 4 + 16},
                            {&s.slotw, adj * 4 + 16}, {&s.witness, m * 4 + 16}}) {
    status = buf->Reserve(bytes, &grew);
    if (status != cudaSuccess) return CudaFail(ctx, status, "JV workspace allocation");
  }
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), st);
  status = CopyFromHost(ctx, s.active.ptr, g->active, m);
  if (status == cudaSuccess) status = CopyFromHost(ctx, s.ro.ptr, g->row_offsets, (static_cast<size_t>(g->n) + 1) * 4);
  if (status == cudaSuccess) status = CopyFromHost(ctx, s.nbr.ptr, g->neighbors, adj * 4);
  if (status == cudaSuccess) status = CopyFromHost(ctx, s.ids.ptr, g->csr_edge_ids, adj * 4);
  if (status != cudaSuccess) return CudaFail(ctx, status, "JV snapshot upload");
  h2d += static_cast<int64_t>(m + (static_cast<size_t>(g->n) + 1) * 4 + adj * 8);
  cudaEventRecord(ctx->ev[1], st);
  if (adj > 0) {
    gather_slot_weights<<<GridFor(static_cast<int64_t>(adj), 256, ctx->sm_count * 8), 256, 0, st>>>(
        static_cast<const int32_t*>(s.ids.ptr), static_cast<int64_t>(adj),
        static_cast<const int32_t*>(s.w32.ptr), g->m, static_cast<int32_t*>(s.slotw.ptr), ctx->d_error);
  }
  status = cudaGetLastError();
  if (status != cudaSuccess) return CudaFail(ctx, status, "slot weight gather launch");
  s.adjacency = g->adjacency;
  s.prepared = true;
  s.last_h2d_bytes = h2d;
  s.edges_screened = 0;
  if (stats != nullptr) {
    for (int64_t e = 0; e < g->m; ++e) s.edges_screened += g->active[e] != 0;
    stats->static_hit = static_hit ? 1 : 0;
    stats->workspace_hit = grew ? 0 : 1;
    stats->resident_bytes = JvResident(s);
    stats->h2d_bytes = h2d;
    stats->edges_screened = s.edges_screened;
  }
  return CEE_OK;
}

int JvLaunch(cee_ctx* ctx) {
  JvState& s = ctx->jv;
  if (!s.prepared) return Fail(ctx, CEE_ERR_STATE, "cee_jv_launch before cee_jv_prepare");
  if (s.m == 0) return CEE_OK;
  JvGraph graph{};
  graph.n = s.n;
  graph.dist_type = s.dist_type;
  graph.m = s.m;
  graph.xy = static_cast<const int2*>(s.xy.ptr);
  graph.edge_uv = static_cast<const int2*>(s.uv.ptr);
  graph.edge_w = static_cast<const int32_t*>(s.w32.ptr);
  graph.active = static_cast<const uint8_t*>(s.active.ptr);
  graph.row_offsets = static_cast<const int32_t*>(s.ro.ptr);
  graph.nbr = static_cast<const int32_t*>(s.nbr.ptr);
  graph.slot_w = static_cast<const int32_t*>(s.slotw.ptr);
  int32_t* witness = static_cast<int32_t*>(s.witness.ptr);
  if (ctx->jv_kernel == 1) {
    const int blocks = GridFor(s.m, kJvWarpsPerBlock, ctx->sm_count * ctx->occ_jv_warp[s.span]);
    WithSpan(s.span, [&](auto S) {
      jv_screen_warp_kernel<S.value><<<blocks, kJvWarpsPerBlock * 32, 0, ctx->stream>>>(graph, 0, s.m, witness,
                                                                                         ctx->d_error);
    });
  } else {
    const int blocks = GridFor(s.m, kJvThreadBlock, ctx->sm_count * ctx->occ_jv_thread[s.span] * ctx->jv_waves);
    WithSpan(s.span, [&](auto S) {
      jv_screen_thread_kernel<S.value><<<blocks, kJvThreadBlock, 0, ctx->stream>>>(graph, 0, s.m, witness,
                                                                                   ctx->d_error);
    });
  }
  const cudaError_t status = cudaGetLastError();
  if (status != cudaSuccess) return CudaFail(ctx, status, "jv_screen_kernel launch");
  return CEE_OK;
}

int CheckDeviceError(cee_ctx* ctx, const char* what) {
  if (*ctx->h_error != 0) {
    return Fail(ctx, CEE_ERR_INVALID,
                std::string(what) + ": device bounds check rejected an out-of-range index (code " +
                    std::to_string(*ctx->h_error) + ")");
  }
  return CEE_OK;
}

int Drained(cee_ctx* ctx, int rc) {
  cudaStreamSynchronize(ctx->stream);
  return rc;
}

int JvFetch(cee_ctx* ctx, int32_t* witness_out) {
  JvState& s = ctx->jv;
  if (!s.prepared) return Fail(ctx, CEE_ERR_STATE, "cee_jv_fetch before cee_jv_prepare");
  if (s.m > 0 && witness_out == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null witness output");
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
  const cudaError_t status = CopyToHost(ctx, witness_out, s.witness.ptr, static_cast<size_t>(s.m) * 4);
  if (status != cudaSuccess) return CudaFail(ctx, status, "JV screen");
  return CheckDeviceError(ctx, "JV screen");
}

// ---------------------------------------------------------------- k-opt -----------------

// Proper k-opt reconnect templates. The table is the reference's: perfect matchings of the
// 2k ports in lexicographic order (the lowest unmatched port takes each higher unmatched port
// in turn), kept when, alternated with the component matching 1-2, 3-4, ..., (2k-1)-0, they
// close a single cycle through all ports and re-add no deleted edge 2e-(2e+1).
struct TemplateBuilder {
  uint32_t k;
  uint8_t mate[14];
  std::vector<uint8_t> out;
  int count = 0;

  bool SingleCycle() const {
    const uint32_t ports = 2 * k;
    auto component = [&](uint32_t p) -> uint32_t {
      if (p == 0) return ports - 1;
      if (p == ports - 1) return 0;
      return (p % 2 == 1) ? p + 1 : p - 1;
    };
    uint32_t p = 0, steps = 0;
    do {
      p = (steps % 2 == 0) ? mate[p] : component(p);
      ++steps;
    } while (p != 0 && steps <= ports);
    return steps == ports;
  }

  void Extend() {
    const uint32_t ports = 2 * k;
    uint32_t first = ports;
    for (uint32_t p = 0; p < ports; ++p) {
      if (mate[p] == 0xff) {
        first = p;
        break;
      }
    }
    if (first == ports) {
      for (uint32_t e = 0; e < k; ++e) {
        if (mate[2 * e] == 2 * e + 1) return;
      }
      if (!SingleCycle()) return;
      out.insert(out.end(), mate, mate + 14);
      ++count;
      return;
    }
    for (uint32_t q = first + 1; q < ports; ++q) {
      if (mate[q] != 0xff) continue;
      mate[first] = static_cast<uint8_t>(q);
      mate[q] = static_cast<uint8_t>(first);
      Extend();
      mate[first] = mate[q] = 0xff;
    }
  }
};

uint64_t TemplateHash(uint32_t k, int count, const uint8_t* mates) {
  uint64_t hash = 14695981039346656037ULL;
  auto byte = [&](uint8_t v) {
    hash ^= v;
    hash *= 1099511628211ULL;
  };
  for (const char* p = "CUDAEE_KOPT_RECONNECT_TEMPLATES_V1"; *p != '\0'; ++p) byte(static_cast<uint8_t>(*p));
  for (int shift = 0; shift < 32; shift += 8) byte(static_cast<uint8_t>((k >> shift) & 0xff));
  for (int shift = 0; shift < 32; shift += 8) byte(static_cast<uint8_t>((static_cast<uint32_t>(count) >> shift) & 0xff));
  for (int t = 0; t < count; ++t) {
    for (uint32_t p = 0; p < 2 * k; ++p) byte(mates[14 * t + p]);
  }
  return hash;
}

// Converts caller template mates into per-template pair indices (ascending port order).
int PairTable(cee_ctx* ctx, uint32_t k, const uint8_t* mates, int32_t count, std::vector<uint8_t>* pairs) {
  const uint32_t ports = 2 * k;
  pairs->assign(static_cast<size_t>(count) * k, 0);
  for (int32_t t = 0; t < count; ++t) {
    const uint8_t* mate = mates + 14 * t;
    uint32_t found = 0;
    for (uint32_t p = 0; p < ports; ++p) {
      const uint32_t q = mate[p];
      if (q >= ports || q == p || mate[q] != p) {
        return Fail(ctx, CEE_ERR_INVALID, "k-opt template is not a perfect matching of the 2k ports");
      }
      if (p < q) (*pairs)[static_cast<size_t>(t) * k + found++] = static_cast<uint8_t>(kopt_pair_index(p, q, ports));
    }
    // a template that pairs 2e with 2e + 1 re-adds deleted edge e on every row
    for (uint32_t e = 0; e < k; ++e) {
      if (mate[2 * e] == 2 * e + 1) (*pairs)[static_cast<size_t>(t) * k] = kKoptReaddsDeleted;
    }
  }
  return CEE_OK;
}

// For each template (k pair indices, or the re-adds-deleted marker): bit g is set when the template's
// cell is invalid on every gap-pattern row of pattern g (kopt_cost.cuh). Such a row's ports fall into
// classes that merge port 2e+1 with port (2e+2) mod 2k for each closed gap e; a cell is invalid when
// an added edge joins two ports of one class (a self loop), equals a deleted edge's class pair, or
// repeats another added edge's class pair (src/cpu/kopt_search.cpp:962-1042).
std::vector<uint32_t> GapPatternMasks(uint32_t k, const std::vector<uint8_t>& pairs, int32_t count) {
  const int P = static_cast<int>(2 * k);
  std::vector<int> pp, pq;
  for (int p = 0; p < P; ++p) {
    for (int q = p + 1; q < P; ++q) {
      pp.push_back(p);
      pq.push_back(q);
    }
  }
  std::vector<uint32_t> masks(static_cast<size_t>(count), 0);
  for (uint32_t g = 0; g < (1u << k); ++g) {
    int cls[kKoptMaxPorts];
    for (int p = 0; p < P; ++p) cls[p] = p;
    for (uint32_t e = 0; e < k; ++e) {
      if ((g >> e) & 1u) {  // the two ports share a node; the class is its lower port
        const int a = static_cast<int>(2 * e + 1), b = static_cast<int>((2 * e + 2) % P);
        const int lo = std::min(cls[a], cls[b]), hi = std::max(cls[a], cls[b]);
        for (int p = 0; p < P; ++p) {
          if (cls[p] == hi) cls[p] = lo;
        }
      }
    }
    std::vector<std::pair<int, int>> deleted;
    for (uint32_t e = 0; e < k; ++e) {
      deleted.emplace_back(std::min(cls[2 * e], cls[2 * e + 1]), std::max(cls[2 * e], cls[2 * e + 1]));
    }
    for (int32_t t = 0; t < count; ++t) {
      const uint8_t* tp = pairs.data() + static_cast<size_t>(t) * k;
      bool invalid = tp[0] == kKoptReaddsDeleted;
      std::vector<std::pair<int, int>> added;
      for (uint32_t i = 0; i < k && !invalid; ++i) {
        const int a = cls[pp[tp[i]]], b = cls[pq[tp[i]]];
        const std::pair<int, int> code{std::min(a, b), std::max(a, b)};
        invalid = a == b || std::find(deleted.begin(), deleted.end(), code) != deleted.end() ||
                  std::find(added.begin(), added.end(), code) != added.end();
        added.push_back(code);
      }
      if (invalid) masks[static_cast<size_t>(t)] |= 1u << g;
    }
  }
  return masks;
}

// Whether `mates` is the proper table of k byte for byte (the one kopt_rows.cuh compiles in).
template <int K>
bool SameAsCanon(const uint8_t* mates, int32_t count) {
  const KoptCanonTable<K>& tab = KoptCanon<K>::value;
  if (count != tab.count) return false;
  for (int t = 0; t < count; ++t) {
    for (int p = 0; p < 14; ++p) {
      const uint8_t want = p < 2 * K ? tab.mate[t][p] : 0xff;
      if (mates[14 * t + p] != want && p < 2 * K) return false;
    }
  }
  return true;
}

bool IsCanonicalTable(uint32_t k, const uint8_t* mates, int32_t count) {
  return k == 3 ? SameAsCanon<3>(mates, count) : (k == 4 ? SameAsCanon<4>(mates, count) : SameAsCanon<5>(mates, count));
}

int EnsureTable(cee_ctx* ctx, KoptTable* table, uint32_t k, const uint8_t* mates, int32_t count,
                uint64_t hash, bool* hit) {
  const size_t bytes = static_cast<size_t>(count) * 14;
  if (table->k == k && table->hash == hash && table->T == count && table->mates.size() == bytes &&
      std::memcmp(table->mates.data(), mates, bytes) == 0) {
    *hit = true;
    return CEE_OK;
  }
  *hit = false;
  std::vector<uint8_t> pairs;
  const int rc = PairTable(ctx, k, mates, count, &pairs);
  if (rc != CEE_OK) return rc;
  cudaError_t status = table->pairs.Reserve(pairs.size() + 16, nullptr);
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt template allocation");
  status = cudaMemcpy(table->pairs.ptr, pairs.data(), pairs.size(), cudaMemcpyHostToDevice);
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt template upload");
  const std::vector<uint32_t> masks = GapPatternMasks(k, pairs, count);
  status = table->patterns.Reserve(masks.size() * sizeof(uint32_t) + 16, nullptr);
  if (status == cudaSuccess) {
    status = cudaMemcpy(table->patterns.ptr, masks.data(), masks.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
  }
  // the same bits by pattern: word [g][w] holds bit (t mod 32) for templates t of word w
  const int words = (count + 31) / 32;
  std::vector<uint32_t> by_pattern(static_cast<size_t>(32) * words, 0);
  for (int g = 0; g < 32; ++g) {
    for (int t = 0; t < count; ++t) by_pattern[g * words + t / 32] |= ((masks[t] >> g) & 1u) << (t % 32);
  }
  if (status == cudaSuccess) status = table->validity.Reserve(by_pattern.size() * sizeof(uint32_t) + 16, nullptr);
  if (status == cudaSuccess) {
    status = cudaMemcpy(table->validity.ptr, by_pattern.data(), by_pattern.size() * sizeof(uint32_t),
                        cudaMemcpyHostToDevice);
  }
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt template pattern upload");
  table->canonical = IsCanonicalTable(k, mates, count);
  table->k = k;
  table->hash = hash;
  table->T = count;
  table->mates.assign(mates, mates + bytes);
  return CEE_OK;
}

int KoptCoords(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y, bool* hit) {
  KoptState& s = ctx->kopt;
  if (n <= 0) return Fail(ctx, CEE_ERR_INVALID, "k-opt snapshot has no nodes");
  if (dist_type != CEE_EUC_2D && dist_type != CEE_CEIL_2D) {
    return Fail(ctx, CEE_ERR_INVALID, "unknown distance type");
  }
  if (s.has_coords && s.n == n && s.dist_type == dist_type && SameArray(s.hx, x, n) && SameArray(s.hy, y, n)) {
    *hit = true;
    return CEE_OK;
  }
  *hit = false;
  s.has_coords = false;
  std::vector<int2> xy;
  int rc = PackCoordinates(ctx, n, x, y, &xy, &s.span);
  if (rc != CEE_OK) return rc;
  cudaError_t status = s.xy.Reserve(xy.size() * sizeof(int2) + 16, nullptr);
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt coordinate allocation");
  status = cudaMemcpy(s.xy.ptr, xy.data(), xy.size() * sizeof(int2), cudaMemcpyHostToDevice);
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt coordinate upload");
  s.hx.assign(x, x + n);
  s.hy.assign(y, y + n);
  s.n = n;
  s.dist_type = dist_type;
  s.has_coords = true;
  return CEE_OK;
}

int KoptTemplatesFor(int k) { return k == 3 ? 4 : (k == 4 ? 25 : 208); }

int DefaultRowsPerTile(uint32_t k) { return k == 3 ? 96 : (k == 4 ? 56 : 32); }  // ~22 KB tiles: nine blocks per SM

// The tiled kernel's tiles of the prepared segments, from the context's rows-per-tile options.
void KoptRetile(cee_ctx* ctx) {
  KoptState& s = ctx->kopt;
  int32_t tile = 0;
  for (int32_t i = 0; i < s.launch.segments; ++i) {
    KoptSegment& seg = s.launch.seg[i];
    const int option = ctx->kopt_rows_per_tile[seg.k - 3];
    seg.rows_per_tile = option > 0 ? option : DefaultRowsPerTile(static_cast<uint32_t>(seg.k));
    seg.tile_begin = tile;
    tile += static_cast<int32_t>((seg.rows + seg.rows_per_tile - 1) / seg.rows_per_tile);
  }
  s.tiles = tile;
}

// Uploads the rows of every segment and records the launch description.
int KoptPrepareSegments(cee_ctx* ctx, int32_t segments, const uint32_t* ks, const KoptTable* const* tables,
                        const cee_kopt_task* const* tasks, const int64_t* rows, cee_kopt_stats* stats,
                        bool snapshot_hit, bool template_hit) {
  KoptState& s = ctx->kopt;
  s.prepared = false;
  if (segments < 1 || segments > kKoptMaxSegments) return Fail(ctx, CEE_ERR_INVALID, "bad k-opt segment count");
  int64_t total_rows = 0, total_cells = 0;
  std::vector<int64_t> cost_offset(static_cast<size_t>(segments));
  for (int32_t i = 0; i < segments; ++i) {
    if (rows[i] < 0) return Fail(ctx, CEE_ERR_INVALID, "negative k-opt row count");
    if (rows[i] > 0 && tasks[i] == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null k-opt tasks");
    cost_offset[i] = total_cells;
    total_rows += rows[i];
    total_cells += (rows[i] * tables[i]->T + 15) & ~int64_t{15};  // each segment starts on a 128-byte line
  }
  bool grew = false;
  cudaError_t status = s.tasks.Reserve(static_cast<size_t>(total_rows) * sizeof(cee_kopt_task) + 16, &grew);
  if (status == cudaSuccess) status = s.costs.Reserve(static_cast<size_t>(total_cells) * 8 + 16, &grew);
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt workspace allocation");
  cudaStream_t st = ctx->stream;
  cudaEventRecord(ctx->ev[0], st);
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), st);
  int64_t row_offset = 0;
  KoptLaunch& L = s.launch;
  L = KoptLaunch{};
  L.segments = segments;
  L.dist_type = s.dist_type;
  L.n = s.n;
  L.xy = static_cast<const int2*>(s.xy.ptr);
  for (int32_t i = 0; i < segments; ++i) {
    const size_t bytes = static_cast<size_t>(rows[i]) * sizeof(cee_kopt_task);
    cee_kopt_task* dst = static_cast<cee_kopt_task*>(s.tasks.ptr) + row_offset;
    status = CopyFromHost(ctx, dst, tasks[i], bytes);
    if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt task upload");
    KoptSegment& seg = L.seg[i];
    seg.tasks = reinterpret_cast<const int32_t*>(dst);
    seg.costs = static_cast<int64_t*>(s.costs.ptr) + cost_offset[i];
    seg.rows = rows[i];
    seg.pairs = static_cast<const uint8_t*>(tables[i]->pairs.ptr);
    seg.patterns = static_cast<const uint32_t*>(tables[i]->patterns.ptr);
    seg.validity = static_cast<const uint32_t*>(tables[i]->validity.ptr);
    seg.canonical = tables[i]->canonical ? 1 : 0;
    seg.k = static_cast<int32_t>(ks[i]);
    seg.templates = tables[i]->T;
    seg.write_costs = 1;
    row_offset += rows[i];
    s.seg_rows[i] = rows[i];
    s.seg_T[i] = tables[i]->T;
  }
  s.segments = segments;
  KoptRetile(ctx);
  cudaEventRecord(ctx->ev[1], st);
  s.prepared = true;
  s.last_h2d_bytes = total_rows * static_cast<int64_t>(sizeof(cee_kopt_task));
  if (stats != nullptr) {
    stats->snapshot_hit = snapshot_hit ? 1 : 0;
    stats->template_hit = template_hit ? 1 : 0;
    stats->workspace_hit = grew ? 0 : 1;
    stats->resident_bytes = KoptResident(s);
    stats->h2d_bytes = s.last_h2d_bytes;
  }
  return CEE_OK;
}

// cuTensorMapEncodeTiled, from the driver through the runtime (the library links only cudart).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn TensorMapEncoder() {
  static const EncodeTiledFn fn = [] {
    void* entry = nullptr;
    cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &entry, 12000, cudaEnableDefault, &found) !=
            cudaSuccess ||
        found != cudaDriverEntryPointSuccess) {
      return static_cast<EncodeTiledFn>(nullptr);
    }
    return reinterpret_cast<EncodeTiledFn>(entry);
  }();
  return fn;
}

// The tensor map of a k = 5 segment's cost matrix: [rows][208] int64, boxes of 16 cells x 32 rows,
// 128-byte swizzle (the layout kopt_proper_rows_warp stages).
bool EncodeKopt5Map(CUtensorMap* map, int64_t* costs, int64_t rows) {
  const EncodeTiledFn encode = TensorMapEncoder();
  if (encode == nullptr) return false;
  const cuuint64_t dims[2] = {208, static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {208 * sizeof(int64_t)};
  const cuuint32_t box[2] = {kKopt5Box, 32};
  const cuuint32_t step[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_INT64, 2, costs, dims, strides, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The one-thread-per-row kernel (kopt_rows.cuh) when every segment uses the proper templates and
// the coordinates are not of the wide span class: 256 rows per block, 32 per warp. Returns false
// when it does not apply; *status carries a launch error.
bool KoptRowsLaunch(cee_ctx* ctx, cudaError_t* status) {
  KoptState& s = ctx->kopt;
  if (ctx->kopt_kernel == 0 || s.span == kSpanWide) return false;
  bool masks = false;
  for (int32_t i = 0; i < s.segments; ++i) {
    if (s.launch.seg[i].canonical == 0 || s.launch.seg[i].rows >= (int64_t{1} << 31)) return false;
    masks = masks || s.launch.seg[i].mask_words > 0;
  }
  // blocks of the heavier rows first (k = 5, then 4, then 3), so that the light tiles fill the tail;
  // the kernel maps a block to its segment by tile_begin, so the segments are listed in that order
  KoptRowsParams P{};  // about 2 KB; the launch copies it
  KoptLaunch& L = P.L;
  L = s.launch;
  std::stable_sort(L.seg, L.seg + L.segments, [](const KoptSegment& a, const KoptSegment& b) { return a.k > b.k; });
  int32_t tile = 0;
  for (int32_t i = 0; i < L.segments; ++i) {
    KoptSegment& seg = L.seg[i];
    seg.tile_begin = tile;
    tile += static_cast<int32_t>((seg.rows + kKoptRowThreads - 1) / kKoptRowThreads);
    if (seg.k == 5 && seg.write_costs != 0 && seg.rows > 0 && !EncodeKopt5Map(&P.box5[i], seg.costs, seg.rows)) {
      *status = cudaErrorInvalidValue;
      return true;
    }
  }
  if (tile == 0) return true;
  WithSpan(s.span, [&](auto S) {
    if constexpr (S.value != kSpanWide) {
      auto launch = [&](auto kernel) {
        *status = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kKoptRowsSmem);
        if (*status == cudaSuccess) kernel<<<tile, kKoptRowThreads, kKoptRowsSmem, ctx->stream>>>(P, ctx->d_error);
      };
      if (masks) {
        launch(kopt_rows_kernel<S.value, true>);
      } else {
        launch(kopt_rows_kernel<S.value, false>);
      }
    }
  });
  return true;
}

int KoptLaunchPrepared(cee_ctx* ctx) {
  KoptState& s = ctx->kopt;
  if (!s.prepared) return Fail(ctx, CEE_ERR_STATE, "cee_kopt_launch before prepare");
  if (s.tiles == 0) return CEE_OK;
  {
    cudaError_t status = cudaSuccess;
    if (KoptRowsLaunch(ctx, &status)) {
      if (status == cudaSuccess) status = cudaGetLastError();
      if (status != cudaSuccess) return CudaFail(ctx, status, "kopt_rows_kernel launch (tensor map or launch)");
      return CEE_OK;
    }
  }
  int smem = 0;
  for (int32_t i = 0; i < s.segments; ++i) {
    smem = std::max(smem, kopt_tile_smem(s.launch.seg[i].k, s.launch.seg[i].rows_per_tile, s.launch.seg[i].mask_words));
  }
  if (smem > kKoptSmemBytes) return Fail(ctx, CEE_ERR_INVALID, "k-opt tile exceeds shared memory");
  cudaError_t status = cudaSuccess;
  WithSpan(s.span, [&](auto S) {
    if (smem > 48 * 1024) {
      status = cudaFuncSetAttribute(kopt_cost_kernel<S.value>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    }
    if (status == cudaSuccess) kopt_cost_kernel<S.value><<<s.tiles, kKoptThreads, smem, ctx->stream>>>(s.launch, ctx->d_error);
  });
  if (status == cudaSuccess) status = cudaGetLastError();
  if (status != cudaSuccess) return CudaFail(ctx, status, "kopt_cost_kernel launch");
  return CEE_OK;
}

int KoptFetch(cee_ctx* ctx, int64_t* const* costs_out) {
  KoptState& s = ctx->kopt;
  if (!s.prepared) return Fail(ctx, CEE_ERR_STATE, "cee_kopt_fetch before prepare");
  int64_t bytes = 0;
  for (int32_t i = 0; i < s.segments; ++i) {
    const size_t n = static_cast<size_t>(s.seg_rows[i]) * static_cast<size_t>(s.seg_T[i]) * 8;
    if (n > 0 && costs_out[i] == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null k-opt cost output");
  }
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t status = cudaSuccess;
  for (int32_t i = 0; i < s.segments && status == cudaSuccess; ++i) {
    const size_t n = static_cast<size_t>(s.seg_rows[i]) * static_cast<size_t>(s.seg_T[i]) * 8;
    status = CopyToHost(ctx, costs_out[i], s.launch.seg[i].costs, n);
    bytes += static_cast<int64_t>(n);
  }
  if (status == cudaSuccess) status = cudaStreamSynchronize(ctx->stream);
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt cost matrix");
  s.last_d2h_bytes = bytes;
  return CheckDeviceError(ctx, "k-opt cost matrix");
}

int CanonicalTable(cee_ctx* ctx, uint32_t k, const KoptTable** out) {
  KoptTable& table = ctx->kopt.canon[k - 3];
  if (table.T == 0) {
    std::vector<uint8_t> mates(14 * kKoptMaxTemplates, 0xff);
    uint64_t hash = 0;
    const int count = cee_kopt_templates(k, mates.data(), &hash);
    if (count <= 0) return Fail(ctx, CEE_ERR_INVALID, "k-opt template generation failed");
    bool hit = false;
    const int rc = EnsureTable(ctx, &table, k, mates.data(), count, hash, &hit);
    if (rc != CEE_OK) return rc;
  }
  *out = &table;
  return CEE_OK;
}

// cee_kopt_prepare_multi without the final wait: its copies stay queued for the calls that launch next.
int KoptPrepareMulti(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y, int32_t segments,
                     const uint32_t* ks, const cee_kopt_task* const* tasks, const int64_t* rows,
                     cee_kopt_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (stats != nullptr) *stats = cee_kopt_stats{};
  if (segments < 1 || segments > kKoptMaxSegments || ks == nullptr || tasks == nullptr || rows == nullptr) {
    return Fail(ctx, CEE_ERR_INVALID, "bad k-opt segment description");
  }
  bool snapshot_hit = false;
  rc = KoptCoords(ctx, n, dist_type, x, y, &snapshot_hit);
  if (rc != CEE_OK) return rc;
  const KoptTable* tables[kKoptMaxSegments];
  for (int32_t i = 0; i < segments; ++i) {
    if (ks[i] < 3 || ks[i] > 5) return Fail(ctx, CEE_ERR_INVALID, "k must lie in [3,5]");
    rc = CanonicalTable(ctx, ks[i], &tables[i]);
    if (rc != CEE_OK) return rc;
  }
  return KoptPrepareSegments(ctx, segments, ks, tables, tasks, rows, stats, snapshot_hit, true);
}

// ---------------------------------------------------------------- c,d -------------------

bool HostHasActiveEdge(const cee_graph_view* g, int32_t u, int32_t v) {
  if (u < 0 || v < 0 || u >= g->n || v >= g->n) return false;
  const int32_t* begin = g->neighbors + g->row_offsets[u];
  const int32_t* end = g->neighbors + g->row_offsets[u + 1];
  return std::binary_search(begin, end, v);
}

}  // namespace cee

using namespace cee;

// ====================================================================== C ABI ===========

extern "C" {

int cee_abi_version(void) { return CEE_ABI_VERSION; }

int cee_device_count(int* count) {
  if (count == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null count");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return CEE_OK;
}

int cee_select_device(int* device) {
  if (device == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null device");
  int count = 0;
  cee_device_count(&count);
  if (count == 0) return Fail(nullptr, CEE_ERR_NODEVICE, "no visible CUDA device");
  int best = -1;
  size_t best_free = 0;
  for (int d = 0; d < count; ++d) {
    if (cudaSetDevice(d) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    size_t free_bytes = 0, total = 0;
    if (cudaMemGetInfo(&free_bytes, &total) == cudaSuccess && (best < 0 || free_bytes > best_free)) {
      best = d;
      best_free = free_bytes;
    }
  }
  if (best < 0) return Fail(nullptr, CEE_ERR_NODEVICE, "no visible CUDA device answered cudaMemGetInfo");
  *device = best;
  return CEE_OK;
}

int cee_create(int device, cee_ctx** out) {
  if (out == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null output");
  *out = nullptr;
  int count = 0;
  cee_device_count(&count);
  if (count == 0) return Fail(nullptr, CEE_ERR_NODEVICE, "no visible CUDA device");
  if (device < 0) {
    const int rc = cee_select_device(&device);
    if (rc != CEE_OK) return rc;
  }
  if (device >= count) return Fail(nullptr, CEE_ERR_NODEVICE, "device ordinal out of range");
  auto* ctx = new cee_ctx();
  ctx->device = device;
  cudaError_t status = cudaSetDevice(device);
  if (status == cudaSuccess) status = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  for (auto& ev : ctx->ev) {
    if (status == cudaSuccess) status = cudaEventCreate(&ev);
  }
  if (status == cudaSuccess) status = cudaMalloc(&ctx->d_error, sizeof(int32_t));
  if (status == cudaSuccess) status = cudaHostAlloc(&ctx->h_error, sizeof(int32_t), cudaHostAllocDefault);
  if (status == cudaSuccess) status = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (status == cudaSuccess) status = QueryOccupancy(ctx);
  if (status != cudaSuccess) {
    const std::string message = std::string("context creation: ") + cudaGetErrorString(status);
    cudaGetLastError();
    cee_destroy(ctx);
    return Fail(nullptr, status == cudaErrorMemoryAllocation ? CEE_ERR_NOMEM : CEE_ERR_CUDA, message);
  }
  *ctx->h_error = 0;
  *out = ctx;
  return CEE_OK;
}

void cee_destroy(cee_ctx* ctx) {
  if (ctx == nullptr) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream != nullptr) cudaStreamSynchronize(ctx->stream);
  ReleaseServe(ctx);
  ReleaseBatch(ctx);
  ReleaseEpoch(ctx);
  ReleaseReplies(ctx);
  ctx->jv.Release();
  ctx->kopt.Release();
  ctx->cd.Release();
  ctx->stage.Release();
  if (ctx->d_error != nullptr) cudaFree(ctx->d_error);
  if (ctx->h_error != nullptr) cudaFreeHost(ctx->h_error);
  for (auto& ev : ctx->ev) {
    if (ev != nullptr) cudaEventDestroy(ev);
  }
  if (ctx->stream != nullptr) cudaStreamDestroy(ctx->stream);
  cudaGetLastError();
  delete ctx;
}

const char* cee_last_error(const cee_ctx* ctx) {
  return ctx != nullptr ? ctx->error.c_str() : g_global_error.c_str();
}

int cee_ctx_device(const cee_ctx* ctx) { return ctx != nullptr ? ctx->device : -1; }

void* cee_ctx_stream(cee_ctx* ctx) { return ctx != nullptr ? static_cast<void*>(ctx->stream) : nullptr; }

int cee_ctx_sm_count(const cee_ctx* ctx) { return ctx != nullptr ? ctx->sm_count : 0; }

int cee_ctx_synchronize(cee_ctx* ctx) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  const cudaError_t status = cudaStreamSynchronize(ctx->stream);
  if (status != cudaSuccess) return CudaFail(ctx, status, "stream synchronize");
  return CEE_OK;
}

uint64_t cee_ctx_resident_bytes(const cee_ctx* ctx) {
  if (ctx == nullptr) return 0;
  return JvResident(ctx->jv) + KoptResident(ctx->kopt) + ctx->cd.xy.capacity + ctx->cd.tasks.capacity +
         ctx->cd.flags.capacity + BatchResident(ctx) + ServeResident(ctx) + EpochResident(ctx) +
         RepliesResident(ctx);
}

int cee_ctx_clear(cee_ctx* ctx, unsigned what) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  cudaStreamSynchronize(ctx->stream);
  if (what & 1u) ctx->jv.Release();
  if (what & 2u) ctx->kopt.Release();
  if (what & 4u) ctx->cd.Release();
  if (what & 8u) ReleaseBatch(ctx);
  if (what & 16u) ReleaseServe(ctx);
  if (what & 32u) ReleaseEpoch(ctx);
  if (what & 64u) ReleaseReplies(ctx);
  return CEE_OK;
}

int cee_ctx_set_option(cee_ctx* ctx, int32_t option, int64_t value) {
  if (ctx == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null context");
  switch (option) {
    case CEE_OPT_JV_KERNEL:
      if (value != 0 && value != 1) return Fail(ctx, CEE_ERR_INVALID, "JV kernel must be 0 (thread) or 1 (warp)");
      ctx->jv_kernel = static_cast<int>(value);
      return CEE_OK;
    case CEE_OPT_JV_WAVES:
      if (value < 1 || value > 64) return Fail(ctx, CEE_ERR_INVALID, "JV waves must lie in [1,64]");
      ctx->jv_waves = static_cast<int>(value);
      return CEE_OK;
    case CEE_OPT_KOPT_ROWS_K3:
    case CEE_OPT_KOPT_ROWS_K4:
    case CEE_OPT_KOPT_ROWS_K5: {
      const int k = option - CEE_OPT_KOPT_ROWS_K3 + 3;
      if (value != 0 && (value < 2 || value % 2 != 0 || kopt_tile_smem(k, static_cast<int>(value)) > kKoptSmemBytes ||
                         value * KoptTemplatesFor(k) > (int64_t{1} << 20))) {
        return Fail(ctx, CEE_ERR_INVALID, "k-opt rows per tile must be even and fit the shared-memory tile");
      }
      ctx->kopt_rows_per_tile[k - 3] = static_cast<int>(value);
      if (ctx->kopt.prepared) KoptRetile(ctx);
      return CEE_OK;
    }
    case CEE_OPT_KOPT_KERNEL:
      if (value != 0 && value != 1) return Fail(ctx, CEE_ERR_INVALID, "k-opt kernel must be 0 (tiled) or 1 (rows)");
      ctx->kopt_kernel = static_cast<int>(value);
      return CEE_OK;
    default:
      return Fail(ctx, CEE_ERR_INVALID, "unknown option");
  }
}

// ---- JV ----

int cee_jv_prepare(cee_ctx* ctx, const cee_graph_view* graph, cee_jv_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (stats != nullptr) *stats = cee_jv_stats{};
  rc = JvPrepare(ctx, graph, stats);
  const cudaError_t status = cudaStreamSynchronize(ctx->stream);  // the graph's arrays are released on return
  if (rc != CEE_OK) return rc;
  if (status != cudaSuccess) return CudaFail(ctx, status, "JV upload");
  return CEE_OK;
}

int cee_jv_launch(cee_ctx* ctx) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  return JvLaunch(ctx);
}

int cee_jv_fetch(cee_ctx* ctx, int32_t* witness_out) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  return JvFetch(ctx, witness_out);
}

int cee_jv_screen(cee_ctx* ctx, const cee_graph_view* graph, int32_t* witness_out, cee_jv_stats* stats) {
  return cee_jv_screen_ex(ctx, graph, witness_out, stats, 0u);
}

int cee_jv_screen_ex(cee_ctx* ctx, const cee_graph_view* graph, int32_t* witness_out, cee_jv_stats* stats,
                     uint32_t flags) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if ((flags & ~CEE_JV_STATIC_UNCHANGED) != 0) return Fail(ctx, CEE_ERR_INVALID, "unknown JV screen flags");
  cee_jv_stats local{};
  rc = JvPrepare(ctx, graph, stats != nullptr ? &local : nullptr, flags);
  if (rc != CEE_OK) return Drained(ctx, rc);
  cudaEventRecord(ctx->ev[2], ctx->stream);
  rc = JvLaunch(ctx);
  if (rc != CEE_OK) return Drained(ctx, rc);
  cudaEventRecord(ctx->ev[3], ctx->stream);
  rc = JvFetch(ctx, witness_out);
  cudaEventRecord(ctx->ev[4], ctx->stream);
  cudaEventSynchronize(ctx->ev[4]);
  if (rc != CEE_OK) return rc;
  local.h2d_ms = EventMs(ctx->ev[0], ctx->ev[1]);
  local.kernel_ms = EventMs(ctx->ev[1], ctx->ev[3]);
  local.d2h_ms = EventMs(ctx->ev[3], ctx->ev[4]);
  local.d2h_bytes = ctx->jv.m * 4;
  if (stats != nullptr) *stats = local;
  return CEE_OK;
}

// ---- k-opt ----

int cee_kopt_templates(uint32_t k, uint8_t* mates, uint64_t* generator_hash) {
  if (k < 3 || k > 5) return Fail(nullptr, CEE_ERR_INVALID, "k must lie in [3,5]");
  TemplateBuilder builder;
  builder.k = k;
  std::memset(builder.mate, 0xff, sizeof(builder.mate));
  builder.Extend();
  if (mates != nullptr) std::memcpy(mates, builder.out.data(), builder.out.size());
  if (generator_hash != nullptr) *generator_hash = TemplateHash(k, builder.count, builder.out.data());
  return builder.count;
}

int cee_kopt_costs(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y,
                   uint32_t k, const uint8_t* mates, int32_t template_count, uint64_t template_hash,
                   const cee_kopt_task* tasks, int64_t rows, int64_t* costs_out, cee_kopt_stats* stats) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (stats != nullptr) *stats = cee_kopt_stats{};
  if (k < 3 || k > 5) return Fail(ctx, CEE_ERR_INVALID, "CUDA k-opt reconnect table k must lie in [3,5]");
  if (template_count <= 0 || template_count > kKoptMaxTemplates || mates == nullptr) {
    return Fail(ctx, CEE_ERR_INVALID, "CUDA k-opt reconnect table is empty or too large");
  }
  bool snapshot_hit = false, template_hit = false;
  rc = KoptCoords(ctx, n, dist_type, x, y, &snapshot_hit);
  if (rc != CEE_OK) return rc;
  KoptTable* table = &ctx->kopt.user[k - 3];
  rc = EnsureTable(ctx, table, k, mates, template_count, template_hash, &template_hit);
  if (rc != CEE_OK) return rc;
  const KoptTable* tables[1] = {table};
  const cee_kopt_task* task_list[1] = {tasks};
  cee_kopt_stats local{};
  rc = KoptPrepareSegments(ctx, 1, &k, tables, task_list, &rows, &local, snapshot_hit, template_hit);
  if (rc != CEE_OK) return Drained(ctx, rc);
  cudaEventRecord(ctx->ev[2], ctx->stream);
  rc = KoptLaunchPrepared(ctx);
  if (rc != CEE_OK) return Drained(ctx, rc);
  cudaEventRecord(ctx->ev[3], ctx->stream);
  int64_t* outs[1] = {costs_out};
  rc = KoptFetch(ctx, outs);
  cudaEventRecord(ctx->ev[4], ctx->stream);
  cudaEventSynchronize(ctx->ev[4]);
  if (rc != CEE_OK) return rc;
  local.h2d_ms = EventMs(ctx->ev[0], ctx->ev[1]);
  local.kernel_ms = EventMs(ctx->ev[2], ctx->ev[3]);
  local.d2h_ms = EventMs(ctx->ev[3], ctx->ev[4]);
  local.d2h_bytes = ctx->kopt.last_d2h_bytes;
  if (stats != nullptr) *stats = local;
  return CEE_OK;
}

int cee_kopt_prepare_multi(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y,
                           int32_t segments, const uint32_t* ks, const cee_kopt_task* const* tasks,
                           const int64_t* rows, cee_kopt_stats* stats) {
  const int rc = KoptPrepareMulti(ctx, n, dist_type, x, y, segments, ks, tasks, rows, stats);
  if (ctx == nullptr) return rc;
  const cudaError_t status = cudaStreamSynchronize(ctx->stream);  // the task arrays are released on return
  if (rc != CEE_OK) return rc;
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt upload");
  return CEE_OK;
}

int cee_kopt_launch(cee_ctx* ctx) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  return KoptLaunchPrepared(ctx);
}

int cee_kopt_set_tuning(cee_ctx* ctx, const cee_kopt_tuning* tuning) {
  if (ctx == nullptr || tuning == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null k-opt tuning");
  int rc = cee_ctx_set_option(ctx, CEE_OPT_KOPT_KERNEL, tuning->kernel);
  for (int k = 0; k < 3 && rc == CEE_OK; ++k) {
    rc = cee_ctx_set_option(ctx, CEE_OPT_KOPT_ROWS_K3 + k, tuning->rows_per_tile[k]);
  }
  return rc;
}

int cee_kopt_get_tuning(const cee_ctx* ctx, cee_kopt_tuning* tuning) {
  if (ctx == nullptr || tuning == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null k-opt tuning");
  tuning->kernel = ctx->kopt_kernel;
  for (int k = 0; k < 3; ++k) tuning->rows_per_tile[k] = ctx->kopt_rows_per_tile[k];
  tuning->ms = 0.0f;
  return CEE_OK;
}

int cee_kopt_autotune(cee_ctx* ctx, int32_t reps, cee_kopt_tuning* chosen) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (!ctx->kopt.prepared) return Fail(ctx, CEE_ERR_STATE, "cee_kopt_autotune before prepare");
  reps = std::max(1, reps);
  std::vector<cee_kopt_tuning> candidates;
  candidates.push_back({1, {0, 0, 0}, 0.0f});
  for (const int scale : {1, 2, 4}) {  // half, default and double tiles (even row counts)
    cee_kopt_tuning t{0, {0, 0, 0}, 0.0f};
    for (int k = 3; k <= 5; ++k) t.rows_per_tile[k - 3] = std::max(2, DefaultRowsPerTile(k) * scale / 2) & ~1;
    candidates.push_back(t);
  }
  cee_kopt_tuning best{};
  float best_ms = 1e30f;
  for (cee_kopt_tuning& t : candidates) {
    rc = cee_kopt_set_tuning(ctx, &t);
    if (rc == CEE_OK) rc = KoptLaunchPrepared(ctx);  // warm-up
    if (rc != CEE_OK) return rc;
    cudaEventRecord(ctx->ev[4], ctx->stream);
    for (int r = 0; r < reps && rc == CEE_OK; ++r) rc = KoptLaunchPrepared(ctx);
    if (rc != CEE_OK) return rc;
    cudaEventRecord(ctx->ev[5], ctx->stream);
    const cudaError_t status = cudaEventSynchronize(ctx->ev[5]);
    if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt autotune");
    t.ms = EventMs(ctx->ev[4], ctx->ev[5]) / reps;
    if (t.ms < best_ms) {
      best_ms = t.ms;
      best = t;
    }
  }
  rc = cee_kopt_set_tuning(ctx, &best);
  if (rc != CEE_OK) return rc;
  if (chosen != nullptr) *chosen = best;
  return CEE_OK;
}

int cee_kopt_fetch(cee_ctx* ctx, int64_t* const* costs_out) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (costs_out == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null k-opt outputs");
  return KoptFetch(ctx, costs_out);
}

int cee_kopt_improving_multi(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y,
                             int32_t segments, const uint32_t* ks, const cee_kopt_task* const* tasks,
                             const int64_t* rows, uint32_t* const* masks_out, int32_t* const* first_out,
                             int64_t* const* costs_out, cee_kopt_stats* stats) {
  cee_kopt_stats local{};
  if (masks_out == nullptr || first_out == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null improving-set outputs");
  int rc = KoptPrepareMulti(ctx, n, dist_type, x, y, segments, ks, tasks, rows, &local);
  if (rc != CEE_OK) return ctx != nullptr ? Drained(ctx, rc) : rc;
  KoptState& s = ctx->kopt;
  int64_t words = 0, total_rows = 0;
  for (int32_t i = 0; i < segments; ++i) {
    words += rows[i] * ((s.launch.seg[i].templates + 31) / 32);
    total_rows += rows[i];
  }
  cudaError_t status = s.masks.Reserve(static_cast<size_t>(words) * 4 + 16, nullptr);
  if (status == cudaSuccess) status = s.firsts.Reserve(static_cast<size_t>(total_rows) * 4 + 16, nullptr);
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "k-opt improving-set allocation"));
  int64_t word_at = 0, row_at = 0;
  for (int32_t i = 0; i < segments; ++i) {
    KoptSegment& seg = s.launch.seg[i];
    seg.mask_words = (seg.templates + 31) / 32;
    seg.improving = static_cast<uint32_t*>(s.masks.ptr) + word_at;
    seg.first = static_cast<int32_t*>(s.firsts.ptr) + row_at;
    seg.write_costs = costs_out != nullptr && costs_out[i] != nullptr ? 1 : 0;
    word_at += rows[i] * seg.mask_words;
    row_at += rows[i];
  }
  cudaEventRecord(ctx->ev[2], ctx->stream);
  rc = KoptLaunchPrepared(ctx);
  if (rc != CEE_OK) return Drained(ctx, rc);
  cudaEventRecord(ctx->ev[3], ctx->stream);
  int64_t d2h = 0;
  for (int32_t i = 0; i < segments; ++i) {
    const KoptSegment& seg = s.launch.seg[i];
    if (rows[i] == 0) continue;
    if (masks_out[i] == nullptr || first_out[i] == nullptr) {
      return Drained(ctx, Fail(ctx, CEE_ERR_INVALID, "null improving-set output"));
    }
    const size_t mb = static_cast<size_t>(rows[i]) * seg.mask_words * 4;
    cudaMemcpyAsync(masks_out[i], seg.improving, mb, cudaMemcpyDeviceToHost, ctx->stream);
    cudaMemcpyAsync(first_out[i], seg.first, static_cast<size_t>(rows[i]) * 4, cudaMemcpyDeviceToHost, ctx->stream);
    d2h += static_cast<int64_t>(mb) + rows[i] * 4;
    if (seg.write_costs != 0) {
      const size_t cb = static_cast<size_t>(rows[i]) * seg.templates * 8;
      cudaMemcpyAsync(costs_out[i], seg.costs, cb, cudaMemcpyDeviceToHost, ctx->stream);
      d2h += static_cast<int64_t>(cb);
    }
  }
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
  cudaEventRecord(ctx->ev[4], ctx->stream);
  status = cudaEventSynchronize(ctx->ev[4]);
  if (status != cudaSuccess) return CudaFail(ctx, status, "k-opt improving sets");
  rc = CheckDeviceError(ctx, "k-opt improving sets");
  if (rc != CEE_OK) return rc;
  local.h2d_ms = EventMs(ctx->ev[0], ctx->ev[1]);
  local.kernel_ms = EventMs(ctx->ev[2], ctx->ev[3]);
  local.d2h_ms = EventMs(ctx->ev[3], ctx->ev[4]);
  local.d2h_bytes = d2h;
  if (stats != nullptr) *stats = local;
  return CEE_OK;
}

int cee_kopt_costs_multi(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y,
                         int32_t segments, const uint32_t* ks, const cee_kopt_task* const* tasks,
                         const int64_t* rows, int64_t* const* costs_out, cee_kopt_stats* stats) {
  cee_kopt_stats local{};
  int rc = KoptPrepareMulti(ctx, n, dist_type, x, y, segments, ks, tasks, rows, &local);
  if (rc != CEE_OK) return ctx != nullptr ? Drained(ctx, rc) : rc;
  cudaEventRecord(ctx->ev[2], ctx->stream);
  rc = KoptLaunchPrepared(ctx);
  if (rc != CEE_OK) return Drained(ctx, rc);
  cudaEventRecord(ctx->ev[3], ctx->stream);
  rc = cee_kopt_fetch(ctx, costs_out);
  cudaEventRecord(ctx->ev[4], ctx->stream);
  cudaEventSynchronize(ctx->ev[4]);
  if (rc != CEE_OK) return rc;
  local.h2d_ms = EventMs(ctx->ev[0], ctx->ev[1]);
  local.kernel_ms = EventMs(ctx->ev[2], ctx->ev[3]);
  local.d2h_ms = EventMs(ctx->ev[3], ctx->ev[4]);
  local.d2h_bytes = ctx->kopt.last_d2h_bytes;
  if (stats != nullptr) *stats = local;
  return CEE_OK;
}

// ---- c,d ----

int cee_cd_screen(cee_ctx* ctx, const cee_graph_view* graph, int32_t u, int32_t v, const cee_cd_task* tasks,
                  int64_t count, int32_t mode, uint8_t* flags_out) {
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  rc = ValidateView(ctx, graph);
  if (rc != CEE_OK) return rc;
  if (u < 0 || v >= graph->n || u >= v ||
      (mode != CEE_CD_ACTIVE_INCOMPATIBLE && mode != CEE_CD_MISSING_OR_INCOMPATIBLE)) {
    return Fail(ctx, CEE_ERR_INVALID, "CUDA HT c,d input is invalid");
  }
  if (count < 0 || (count > 0 && (tasks == nullptr || flags_out == nullptr))) {
    return Fail(ctx, CEE_ERR_INVALID, "bad c,d task buffers");
  }
  for (int64_t i = 0; i < count; ++i) {
    const cee_cd_task& t = tasks[i];
    if (t.c < 0 || t.d >= graph->n || t.c >= t.d || t.c == u || t.c == v || t.d == u || t.d == v ||
        t.active > 1 || (t.active != 0) != HostHasActiveEdge(graph, t.c, t.d)) {
      return Fail(ctx, CEE_ERR_INVALID, "CUDA HT c,d task is invalid or its active bit disagrees with the CSR");
    }
  }
  if (count == 0) return CEE_OK;
  CdState& s = ctx->cd;
  if (!(s.has_coords && s.n == graph->n && s.dist_type == graph->dist_type && SameArray(s.hx, graph->x, graph->n) &&
        SameArray(s.hy, graph->y, graph->n))) {
    s.has_coords = false;
    std::vector<int2> xy;
    rc = PackCoordinates(ctx, graph->n, graph->x, graph->y, &xy, &s.span);
    if (rc != CEE_OK) return rc;
    cudaError_t status = s.xy.Reserve(xy.size() * sizeof(int2) + 16, nullptr);
    if (status == cudaSuccess) status = cudaMemcpy(s.xy.ptr, xy.data(), xy.size() * sizeof(int2), cudaMemcpyHostToDevice);
    if (status != cudaSuccess) return CudaFail(ctx, status, "c,d coordinate upload");
    s.hx.assign(graph->x, graph->x + graph->n);
    s.hy.assign(graph->y, graph->y + graph->n);
    s.n = graph->n;
    s.dist_type = graph->dist_type;
    s.has_coords = true;
  }
  cudaError_t status = s.tasks.Reserve(static_cast<size_t>(count) * sizeof(cee_cd_task) + 16, nullptr);
  if (status == cudaSuccess) status = s.flags.Reserve(static_cast<size_t>(count) + 16, nullptr);
  if (status != cudaSuccess) return CudaFail(ctx, status, "c,d workspace allocation");
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(ctx->d_error, 0, sizeof(int32_t), st);
  cudaMemcpyAsync(s.tasks.ptr, tasks, static_cast<size_t>(count) * sizeof(cee_cd_task), cudaMemcpyHostToDevice, st);
  WithSpan(s.span, [&](auto S) {
    cd_screen_kernel<S.value><<<GridFor(count, 256, 1 << 30), 256, 0, st>>>(
        u, v, static_cast<const CdTask*>(s.tasks.ptr), count, static_cast<const int2*>(s.xy.ptr), s.n,
        s.dist_type, mode, static_cast<uint8_t*>(s.flags.ptr), ctx->d_error);
  });
  status = cudaGetLastError();
  if (status != cudaSuccess) return Drained(ctx, CudaFail(ctx, status, "cd_screen_kernel launch"));
  cudaMemcpyAsync(flags_out, s.flags.ptr, static_cast<size_t>(count), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ctx->h_error, ctx->d_error, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  status = cudaStreamSynchronize(st);
  if (status != cudaSuccess) return CudaFail(ctx, status, "c,d screen");
  return CheckDeviceError(ctx, "c,d screen");
}

int cee_sqrt_estimate_error(cee_ctx* ctx, double* max_relative_error) {
  if (ctx == nullptr || max_relative_error == nullptr) return Fail(ctx, CEE_ERR_INVALID, "null argument");
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  DevBuf word;
  cudaError_t status = word.Reserve(sizeof(unsigned long long), nullptr);
  unsigned long long bits = 0;
  if (status == cudaSuccess) status = cudaMemsetAsync(word.ptr, 0, sizeof(unsigned long long), ctx->stream);
  if (status == cudaSuccess) {
    const uint32_t lo = 0x3f800000u, hi = 0x55800000u;  // the floats in [1, 2^44)
    root_error_kernel<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(lo, hi, static_cast<unsigned long long*>(word.ptr));
    status = cudaGetLastError();
  }
  if (status == cudaSuccess) {
    status = cudaMemcpyAsync(&bits, word.ptr, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream);
  }
  if (status == cudaSuccess) status = cudaStreamSynchronize(ctx->stream);
  word.Release();
  if (status != cudaSuccess) return CudaFail(ctx, status, "square-root estimate check");
  std::memcpy(max_relative_error, &bits, sizeof(double));
  return CEE_OK;
}

int cee_exact_distances(cee_ctx* ctx, int32_t n, const int64_t* x, const int64_t* y, int32_t dist_type,
                        int64_t count, const int32_t* pair_i, const int32_t* pair_j, int32_t* out,
                        int32_t* span_class) {
  if (ctx == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null context");
  int rc = Activate(ctx);
  if (rc != CEE_OK) return rc;
  if (n < 0 || count < 0 || (dist_type != CEE_EUC_2D && dist_type != CEE_CEIL_2D) ||
      (count > 0 && (pair_i == nullptr || pair_j == nullptr || out == nullptr))) {
    return Fail(ctx, CEE_ERR_INVALID, "exact distances: bad arguments");
  }
  std::vector<int2> pairs(static_cast<size_t>(count));
  for (int64_t k = 0; k < count; ++k) {
    if (pair_i[k] < 0 || pair_i[k] >= n || pair_j[k] < 0 || pair_j[k] >= n) {
      return Fail(ctx, CEE_ERR_INVALID, "exact distances: point index out of range");
    }
    pairs[static_cast<size_t>(k)] = make_int2(pair_i[k], pair_j[k]);
  }
  std::vector<int2> xy;
  int span = kSpanSmall;
  rc = PackCoordinates(ctx, n, x, y, &xy, &span);
  if (rc != CEE_OK) return rc;
  if (span_class != nullptr) *span_class = span;
  if (count == 0) return CEE_OK;
  DevBuf d_xy, d_pairs, d_out;
  cudaError_t status = d_xy.Reserve(xy.size() * sizeof(int2), nullptr);
  if (status == cudaSuccess) status = d_pairs.Reserve(pairs.size() * sizeof(int2), nullptr);
  if (status == cudaSuccess) status = d_out.Reserve(static_cast<size_t>(count) * sizeof(int32_t), nullptr);
  cudaStream_t st = ctx->stream;
  if (status == cudaSuccess) {
    cudaMemcpyAsync(d_xy.ptr, xy.data(), xy.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_pairs.ptr, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
    WithSpan(span, [&](auto S) {
      distance_pairs_kernel<S.value><<<GridFor(count, 256, ctx->sm_count * 8), 256, 0, st>>>(
          static_cast<const int2*>(d_xy.ptr), static_cast<const int2*>(d_pairs.ptr), count, dist_type,
          static_cast<int32_t*>(d_out.ptr));
    });
    status = cudaGetLastError();
  }
  if (status == cudaSuccess) {
    cudaMemcpyAsync(out, d_out.ptr, static_cast<size_t>(count) * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    status = cudaStreamSynchronize(st);
  }
  d_xy.Release();
  d_pairs.Release();
  d_out.Release();
  if (status != cudaSuccess) return CudaFail(ctx, status, "exact distances");
  return CEE_OK;
}

}  // extern "C"
