// The JV proof log of a device elimination, on the host: snapshot content hashes
// (GraphSnapshot::ContentHash, src/common/graph.cpp:323-346), the proof records RunJvElimination
// appends (src/cpu/jv_elimination.cpp:304-312) rebuilt from cee_jv_eliminate's per-edge epochs and
// witnesses, a CUDAEE_PROOF_V1 writer (WriteProof, src/cpu/jv_elimination.cpp:324-368) and the
// active-edge file writer (GraphSnapshot::WriteActiveEdges, src/common/graph.cpp:284-298).
//
// The content hash is 64-bit FNV-1a over the snapshot's bytes: a strictly sequential chain, so it
// runs on host threads (one per epoch snapshot), not on the device.
#include "cee.h"
#include "cee_internal.h"

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

namespace cee {
namespace {

constexpr uint64_t kFnvOffset = 14695981039346656037ull;  // FNV-1a 64-bit offset basis
constexpr uint64_t kFnvPrime = 1099511628211ull;          // FNV-1a 64-bit prime

// FNV-1a over the little-endian bytes of an integer value (the in-memory bytes on the hosts the
// reference runs on).
template <typename T>
inline void HashInt(uint64_t& hash, T value) {
  const uint64_t bits = static_cast<uint64_t>(value);
  for (size_t i = 0; i < sizeof(T); ++i) {
    hash ^= (bits >> (8 * i)) & 0xffu;
    hash *= kFnvPrime;
  }
}

// ContentHash of `g` with edge e active iff active(e).
template <typename Active>
uint64_t SnapshotHash(const cee_graph_view& g, Active active) {
  uint64_t hash = kFnvOffset;
  HashInt<int32_t>(hash, g.n);                                  // dimension
  HashInt<uint8_t>(hash, static_cast<uint8_t>(g.dist_type));   // DistanceType (uint8)
  HashInt<uint8_t>(hash, 1);                                    // integer_coordinates
  for (int32_t i = 0; i < g.n; ++i) {
    HashInt<int64_t>(hash, g.x[i]);
    HashInt<int64_t>(hash, g.y[i]);
  }
  for (int64_t e = 0; e < g.m; ++e) {
    HashInt<int32_t>(hash, g.edge_u[e]);
    HashInt<int32_t>(hash, g.edge_v[e]);
    HashInt<int64_t>(hash, g.edge_w[e]);
    HashInt<uint8_t>(hash, active(e) ? 1 : 0);
  }
  return hash;
}

int CheckView(const cee_graph_view* g) {
  if (g == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null graph view");
  if (g->n < 0 || g->m < 0) return Fail(nullptr, CEE_ERR_INVALID, "negative graph size");
  if (g->n > 0 && (g->x == nullptr || g->y == nullptr)) return Fail(nullptr, CEE_ERR_INVALID, "null coordinates");
  if (g->m > 0 && (g->edge_u == nullptr || g->edge_v == nullptr || g->edge_w == nullptr || g->active == nullptr)) {
    return Fail(nullptr, CEE_ERR_INVALID, "null edge arrays");
  }
  if (g->dist_type != CEE_EUC_2D && g->dist_type != CEE_CEIL_2D) {
    return Fail(nullptr, CEE_ERR_INVALID, "unknown distance type");
  }
  return CEE_OK;
}

// Runs body(i) for i in [0, count) on up to `count` host threads.
template <typename Body>
void ParallelFor(int64_t count, Body body) {
  const int threads = static_cast<int>(
      std::max<int64_t>(1, std::min<int64_t>(count, std::max(1u, std::thread::hardware_concurrency()))));
  if (threads <= 1) {
    for (int64_t i = 0; i < count; ++i) body(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  pool.reserve(static_cast<size_t>(threads));
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&] {
      for (int64_t i = next++; i < count; i = next++) body(i);
    });
  }
  for (std::thread& th : pool) th.join();
}

}  // namespace
}  // namespace cee

extern "C" {

int cee_content_hash(const cee_graph_view* graph, uint64_t* hash) {
  using namespace cee;
  if (hash == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null hash output");
  const int rc = CheckView(graph);
  if (rc != CEE_OK) return rc;
  *hash = SnapshotHash(*graph, [&](int64_t e) { return graph->active[e] != 0; });
  return CEE_OK;
}

int cee_jv_proof(const cee_graph_view* graph, uint32_t epochs, const int32_t* edge_epoch, const int32_t* witness,
                 cee_jv_proof_record* records, int64_t capacity, int64_t* count, uint64_t* hashes) {
  using namespace cee;
  int rc = CheckView(graph);
  if (rc != CEE_OK) return rc;
  const cee_graph_view& g = *graph;
  if (count == nullptr || capacity < 0 || (capacity > 0 && records == nullptr) ||
      (g.m > 0 && (edge_epoch == nullptr || witness == nullptr))) {
    return Fail(nullptr, CEE_ERR_INVALID, "bad proof buffers");
  }
  // the eliminated edges, in the proof's order: epoch, then commit order (u, v), then edge id
  std::vector<std::tuple<uint32_t, int32_t, int32_t, int32_t>> order;
  for (int64_t e = 0; e < g.m; ++e) {
    const int32_t ep = edge_epoch[e];
    if (ep < 0) continue;
    if (static_cast<uint32_t>(ep) >= epochs || g.active[e] == 0 || witness[e] < 0 || witness[e] >= g.n) {
      return Fail(nullptr, CEE_ERR_INVALID,
                  "edge " + std::to_string(e) + ": eliminated outside [0, epochs), while inactive, or without a witness node");
    }
    order.emplace_back(static_cast<uint32_t>(ep), g.edge_u[e], g.edge_v[e], static_cast<int32_t>(e));
  }
  std::sort(order.begin(), order.end());
  // hashes of the snapshot before each epoch (edges eliminated in earlier epochs inactive) and the final one
  std::vector<uint64_t> epoch_hash(static_cast<size_t>(epochs) + 1, 0);
  ParallelFor(static_cast<int64_t>(epochs) + 1, [&](int64_t k) {
    epoch_hash[static_cast<size_t>(k)] = SnapshotHash(g, [&](int64_t e) {
      return g.active[e] != 0 && !(edge_epoch[e] >= 0 && edge_epoch[e] < k);
    });
  });
  *count = static_cast<int64_t>(order.size());
  for (size_t r = 0; r < order.size() && static_cast<int64_t>(r) < capacity; ++r) {
    const auto& [ep, u, v, e] = order[r];
    cee_jv_proof_record& out = records[r];
    out.epoch = ep;
    out.edge_id = e;
    out.u = u;
    out.v = v;
    out.witness = witness[e];
    out.reserved = 0;
    out.snapshot_hash = epoch_hash[ep];
  }
  if (hashes != nullptr) std::copy(epoch_hash.begin(), epoch_hash.end(), hashes);
  return CEE_OK;
}

int cee_write_active_edges(const char* path, const cee_graph_view* graph, const uint8_t* active) {
  using namespace cee;
  if (path == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null path");
  const int rc = CheckView(graph);
  if (rc != CEE_OK) return rc;
  const cee_graph_view& g = *graph;
  const uint8_t* flags = active != nullptr ? active : g.active;
  if (g.m > 0 && flags == nullptr) return Fail(nullptr, CEE_ERR_INVALID, "null active flags");
  int64_t count = 0;
  for (int64_t e = 0; e < g.m; ++e) count += flags[e] != 0 ? 1 : 0;
  FILE* out = std::fopen(path, "wb");
  if (out == nullptr) return Fail(nullptr, CEE_ERR_INVALID, std::string("cannot create edge file ") + path);
  std::vector<char> buffer(1 << 20);
  std::setvbuf(out, buffer.data(), _IOFBF, buffer.size());
  std::fprintf(out, "%d %lld\n", g.n, static_cast<long long>(count));
  for (int64_t e = 0; e < g.m; ++e) {
    if (flags[e] != 0) {
      std::fprintf(out, "%d %d %lld\n", g.edge_u[e], g.edge_v[e], static_cast<long long>(g.edge_w[e]));
    }
  }
  const bool failed = std::ferror(out) != 0;
  if (std::fclose(out) != 0 || failed) return Fail(nullptr, CEE_ERR_INVALID, std::string("writing edge file ") + path);
  return CEE_OK;
}

int cee_jv_write_proof(const char* path, const char* backend, uint64_t initial_hash, uint64_t final_hash,
                       const cee_jv_proof_record* records, int64_t count, const cee_jv_epoch_metrics* metrics,
                       int32_t epochs) {
  using namespace cee;
  if (path == nullptr || backend == nullptr || count < 0 || epochs < 0 || (count > 0 && records == nullptr) ||
      (epochs > 0 && metrics == nullptr)) {
    return Fail(nullptr, CEE_ERR_INVALID, "bad proof arguments");
  }
  const size_t backend_len = std::strlen(backend);
  if (backend_len == 0 || std::any_of(backend, backend + backend_len, [](char c) {
        return std::isspace(static_cast<unsigned char>(c)) != 0;
      })) {
    return Fail(nullptr, CEE_ERR_INVALID, "backend must be one non-empty token");
  }
  for (int32_t e = 0; e < epochs; ++e) {
    if (!(metrics[e].propose_ms >= 0.0) || !(metrics[e].verify_ms >= 0.0)) {
      return Fail(nullptr, CEE_ERR_INVALID, "metrics times must be finite and non-negative");
    }
  }
  FILE* out = std::fopen(path, "wb");
  if (out == nullptr) return Fail(nullptr, CEE_ERR_INVALID, std::string("cannot create proof file ") + path);
  // WriteProof's lines; hashes as 16 lower-case hex digits, times in iostream's default (%g) form
  std::fprintf(out, "CUDAEE_PROOF_V1\nbackend %s\ninitial_hash %016llx\n", backend,
               static_cast<unsigned long long>(initial_hash));
  for (int64_t r = 0; r < count; ++r) {
    const cee_jv_proof_record& rec = records[r];
    std::fprintf(out, "record %u %016llx %d %d %d JV %d\n", rec.epoch, static_cast<unsigned long long>(rec.snapshot_hash),
                 rec.edge_id, rec.u, rec.v, rec.witness);
  }
  for (int32_t e = 0; e < epochs; ++e) {
    const cee_jv_epoch_metrics& mt = metrics[e];
    std::fprintf(out, "metrics %u %lld %lld %lld %lld %lld %g %g\n", mt.epoch, static_cast<long long>(mt.edges_before),
                 static_cast<long long>(mt.proposed), static_cast<long long>(mt.verified),
                 static_cast<long long>(mt.rejected), static_cast<long long>(mt.committed), mt.propose_ms, mt.verify_ms);
  }
  std::fprintf(out, "final_hash %016llx\nEND\n", static_cast<unsigned long long>(final_hash));
  const bool failed = std::ferror(out) != 0;
  if (std::fclose(out) != 0 || failed) return Fail(nullptr, CEE_ERR_INVALID, std::string("writing proof file ") + path);
  return CEE_OK;
}

}  // extern "C"
