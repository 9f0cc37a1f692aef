// Seeded synthetic snapshots and k-opt leaf rows for the benchmark workloads and tests.
//
// The reference measures on TSPLIB pcb3038 / rl5915 / d15112 with ElimTSP sparse edge sets,
// none of which ship with it; these generators stand in with the shapes the workloads name:
//   * uniform or Gaussian-clustered integer coordinates, de-duplicated by resampling
//     (as tests/exhaustive/check_small_instances.py:78-81 does for its instances);
//   * k-nearest-neighbour edge sets ranked by exact squared distance, ties by node id,
//     optionally with the 2 nearest neighbours per quadrant;
//   * canonical edges u < v sorted by (u, v) with weight = exact TSPLIB distance, all active
//     (the form GraphSnapshot::Load produces, src/common/graph.cpp:98-228);
//   * k-opt rows built like BuildKOptCostTask (src/cpu/kopt_search.cpp:561-584) from
//     self-avoiding walks on the kNN graph closed into a local tour.
// Everything is driven by std::mt19937_64 so that a (generator, seed) pair reproduces the
// same instance on any host with the same C++ standard library.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <unordered_set>
#include <utility>
#include <vector>

namespace {

struct Instance {
  int32_t n{};
  int32_t dist_type{};
  std::vector<int64_t> x, y;
  std::vector<int32_t> eu, ev;
  std::vector<int64_t> w;
};

int64_t IntegerSqrtFloor(uint64_t value) {
  // restoring bit-pair square root (the same published method the reference uses)
  uint64_t remainder = value, root = 0, bit = uint64_t{1} << 62;
  while (bit > remainder) bit >>= 2;
  while (bit != 0) {
    if (remainder >= root + bit) {
      remainder -= root + bit;
      root = (root >> 1) + bit;
    } else {
      root >>= 1;
    }
    bit >>= 2;
  }
  return static_cast<int64_t>(root);
}

int64_t ExactDistance(int64_t x1, int64_t y1, int64_t x2, int64_t y2, int32_t type) {
  const uint64_t dx = static_cast<uint64_t>(x1 > x2 ? x1 - x2 : x2 - x1);
  const uint64_t dy = static_cast<uint64_t>(y1 > y2 ? y1 - y2 : y2 - y1);
  const uint64_t s = dx * dx + dy * dy;
  const uint64_t r = static_cast<uint64_t>(IntegerSqrtFloor(s));
  if (type == 0) return static_cast<int64_t>(r + (s - r * r > r ? 1 : 0));
  return static_cast<int64_t>(r + (r * r != s ? 1 : 0));
}

struct PointSet {
  std::unordered_set<uint64_t> used;
  bool Insert(int64_t x, int64_t y) {
    return used.insert((static_cast<uint64_t>(x) << 32) ^ static_cast<uint64_t>(y)).second;
  }
};

// Uniform integer points in [0, range)^2, appended to (x, y).
void AddUniform(std::mt19937_64& rng, int64_t range, int32_t count, PointSet& set,
                std::vector<int64_t>& x, std::vector<int64_t>& y) {
  std::uniform_int_distribution<int64_t> coord(0, range - 1);
  for (int32_t i = 0; i < count;) {
    const int64_t px = coord(rng), py = coord(rng);
    if (set.Insert(px, py)) {
      x.push_back(px);
      y.push_back(py);
      ++i;
    }
  }
}

// Gaussian clusters: centers ~ U[0, range)^2, each point picks a center uniformly and is
// round(N(center, sigma^2)) clamped to [0, range-1].
void AddClustered(std::mt19937_64& rng, int64_t range, int32_t centers, double sigma,
                  int32_t count, PointSet& set, std::vector<int64_t>& x,
                  std::vector<int64_t>& y) {
  std::uniform_real_distribution<double> center_coord(0.0, static_cast<double>(range));
  std::vector<double> cx(static_cast<size_t>(centers)), cy(static_cast<size_t>(centers));
  for (int32_t c = 0; c < centers; ++c) {
    cx[c] = center_coord(rng);
    cy[c] = center_coord(rng);
  }
  std::uniform_int_distribution<int32_t> pick(0, centers - 1);
  std::normal_distribution<double> noise(0.0, sigma);
  for (int32_t i = 0; i < count;) {
    const int32_t c = pick(rng);
    int64_t px = std::llround(cx[c] + noise(rng));
    int64_t py = std::llround(cy[c] + noise(rng));
    px = std::clamp<int64_t>(px, 0, range - 1);
    py = std::clamp<int64_t>(py, 0, range - 1);
    if (set.Insert(px, py)) {
      x.push_back(px);
      y.push_back(py);
      ++i;
    }
  }
}

uint64_t Sq(const Instance& g, int32_t a, int32_t b) {
  const int64_t dx = g.x[a] - g.x[b], dy = g.y[a] - g.y[b];
  return static_cast<uint64_t>(dx * dx + dy * dy);
}

// Exact k nearest neighbours by (squared distance, node id) with a uniform grid.
std::vector<std::vector<int32_t>> KNearest(const Instance& g, int32_t k) {
  const int32_t n = g.n;
  int64_t min_x = g.x[0], max_x = g.x[0], min_y = g.y[0], max_y = g.y[0];
  for (int32_t i = 1; i < n; ++i) {
    min_x = std::min(min_x, g.x[i]);
    max_x = std::max(max_x, g.x[i]);
    min_y = std::min(min_y, g.y[i]);
    max_y = std::max(max_y, g.y[i]);
  }
  const double span = static_cast<double>(std::max(max_x - min_x, max_y - min_y) + 1);
  const int32_t cells = std::max(1, static_cast<int32_t>(std::sqrt(static_cast<double>(n) / 2.0)));
  const int64_t cell = static_cast<int64_t>(std::ceil(span / cells)) + 1;
  auto cell_of = [&](int64_t v, int64_t lo) { return static_cast<int32_t>((v - lo) / cell); };
  std::vector<std::vector<int32_t>> grid(static_cast<size_t>(cells) * cells);
  for (int32_t i = 0; i < n; ++i) {
    grid[static_cast<size_t>(cell_of(g.y[i], min_y)) * cells + cell_of(g.x[i], min_x)].push_back(i);
  }
  std::vector<std::vector<int32_t>> result(static_cast<size_t>(n));
  const int32_t want = std::min(k, n - 1);
  std::vector<std::pair<uint64_t, int32_t>> found;
  for (int32_t q = 0; q < n; ++q) {
    const int32_t qx = cell_of(g.x[q], min_x), qy = cell_of(g.y[q], min_y);
    found.clear();
    for (int32_t r = 0;; ++r) {
      for (int32_t gy = qy - r; gy <= qy + r; ++gy) {
        if (gy < 0 || gy >= cells) continue;
        for (int32_t gx = qx - r; gx <= qx + r; ++gx) {
          if (gx < 0 || gx >= cells) continue;
          if (std::max(std::abs(gx - qx), std::abs(gy - qy)) != r) continue;
          for (int32_t p : grid[static_cast<size_t>(gy) * cells + gx]) {
            if (p != q) found.emplace_back(Sq(g, q, p), p);
          }
        }
      }
      const bool exhausted = r >= cells;
      if (want == 0 || exhausted) break;
      if (static_cast<int32_t>(found.size()) >= want) {
        std::nth_element(found.begin(), found.begin() + (want - 1), found.end());
        // every point outside ring r is at least r * cell away along one axis
        const uint64_t bound = static_cast<uint64_t>(r) * static_cast<uint64_t>(cell);
        if (found[want - 1].first < bound * bound) break;
      }
    }
    std::partial_sort(found.begin(), found.begin() + want, found.end());
    for (int32_t i = 0; i < want; ++i) result[q].push_back(found[i].second);
  }
  return result;
}

// Nearest `per` nodes in each of the four half-open quadrants around every node
// (dx>0,dy>=0), (dx<=0,dy>0), (dx<0,dy<=0), (dx>=0,dy<0); brute force.
std::vector<std::vector<int32_t>> QuadrantNearest(const Instance& g, int32_t per) {
  std::vector<std::vector<int32_t>> result(static_cast<size_t>(g.n));
  std::vector<std::pair<uint64_t, int32_t>> quad[4];
  for (int32_t q = 0; q < g.n; ++q) {
    for (auto& list : quad) list.clear();
    for (int32_t p = 0; p < g.n; ++p) {
      if (p == q) continue;
      const int64_t dx = g.x[p] - g.x[q], dy = g.y[p] - g.y[q];
      int which = -1;
      if (dx > 0 && dy >= 0) which = 0;
      else if (dx <= 0 && dy > 0) which = 1;
      else if (dx < 0 && dy <= 0) which = 2;
      else if (dx >= 0 && dy < 0) which = 3;
      if (which >= 0) quad[which].emplace_back(Sq(g, q, p), p);
    }
    for (auto& list : quad) {
      const size_t take = std::min<size_t>(static_cast<size_t>(per), list.size());
      std::partial_sort(list.begin(), list.begin() + static_cast<std::ptrdiff_t>(take), list.end());
      for (size_t i = 0; i < take; ++i) result[q].push_back(list[i].second);
    }
  }
  return result;
}

void BuildEdges(Instance& g, const std::vector<std::vector<int32_t>>& lists) {
  std::vector<std::pair<int32_t, int32_t>> pairs;
  for (int32_t u = 0; u < g.n; ++u) {
    for (int32_t v : lists[u]) pairs.emplace_back(std::min(u, v), std::max(u, v));
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  g.eu.resize(pairs.size());
  g.ev.resize(pairs.size());
  g.w.resize(pairs.size());
  for (size_t e = 0; e < pairs.size(); ++e) {
    g.eu[e] = pairs[e].first;
    g.ev[e] = pairs[e].second;
    g.w[e] = ExactDistance(g.x[pairs[e].first], g.y[pairs[e].first], g.x[pairs[e].second],
                           g.y[pairs[e].second], g.dist_type);
  }
}

void MergeLists(std::vector<std::vector<int32_t>>& into, const std::vector<std::vector<int32_t>>& more) {
  for (size_t i = 0; i < into.size(); ++i) into[i].insert(into[i].end(), more[i].begin(), more[i].end());
}

}  // namespace

extern "C" {

// Uniform instance: n points in [0, range)^2, edges = union of k-NN.
void* cees_uniform_knn(int32_t n, int64_t range, int32_t k, int32_t dist_type, uint64_t seed) {
  auto g = std::make_unique<Instance>();
  g->n = n;
  g->dist_type = dist_type;
  std::mt19937_64 rng(seed);
  PointSet set;
  AddUniform(rng, range, n, set, g->x, g->y);
  BuildEdges(*g, KNearest(*g, k));
  return g.release();
}

// Clustered instance: `centers` Gaussian clusters (sigma) holding n - uniform points plus
// `uniform` uniform points, in [0, range)^2; edges = k-NN, plus the `quadrant` nearest per
// quadrant when quadrant > 0.
void* cees_clustered_knn(int32_t n, int64_t range, int32_t centers, double sigma,
                         int32_t uniform, int32_t k, int32_t quadrant, int32_t dist_type,
                         uint64_t seed) {
  auto g = std::make_unique<Instance>();
  g->n = n;
  g->dist_type = dist_type;
  std::mt19937_64 rng(seed);
  PointSet set;
  AddClustered(rng, range, centers, sigma, n - uniform, set, g->x, g->y);
  AddUniform(rng, range, uniform, set, g->x, g->y);
  auto lists = KNearest(*g, k);
  if (quadrant > 0) MergeLists(lists, QuadrantNearest(*g, quadrant));
  BuildEdges(*g, lists);
  return g.release();
}

// Instance `index` of the batching mix: n = floor(exp(U[ln n_lo, ln n_hi])) (100..5000 for
// the 4,096-instance batch), then a fair coin picks uniform in [0,1e5)^2 or clustered
// (ceil(n/100) centers, sigma 300, 20% uniform); 10-NN, EUC_2D; seed = base + index.
// The serving mix draws its JV jobs the same way with n in [200, 20000].
void* cees_batch_instance(uint64_t base_seed, uint64_t index, double n_lo, double n_hi) {
  std::mt19937_64 rng(base_seed + index);
  std::uniform_real_distribution<double> log_n(std::log(n_lo), std::log(n_hi));
  const int32_t n = static_cast<int32_t>(std::floor(std::exp(log_n(rng))));
  std::uniform_int_distribution<int32_t> coin(0, 1);
  const bool clustered = coin(rng) == 1;
  const uint64_t seed = rng();
  if (!clustered) return cees_uniform_knn(n, 100000, 10, 0, seed);
  const int32_t centers = (n + 99) / 100;
  const int32_t uniform = n / 5;
  return cees_clustered_knn(n, 100000, centers, 300.0, uniform, 10, 0, 0, seed);
}

void cees_free(void* handle) { delete static_cast<Instance*>(handle); }
int32_t cees_n(void* handle) { return static_cast<Instance*>(handle)->n; }
int64_t cees_m(void* handle) { return static_cast<int64_t>(static_cast<Instance*>(handle)->eu.size()); }
int32_t cees_dist_type(void* handle) { return static_cast<Instance*>(handle)->dist_type; }

void cees_copy(void* handle, int64_t* x, int64_t* y, int32_t* eu, int32_t* ev, int64_t* w) {
  const Instance& g = *static_cast<Instance*>(handle);
  std::memcpy(x, g.x.data(), g.x.size() * 8);
  std::memcpy(y, g.y.data(), g.y.size() * 8);
  std::memcpy(eu, g.eu.data(), g.eu.size() * 4);
  std::memcpy(ev, g.ev.data(), g.ev.size() * 4);
  std::memcpy(w, g.w.data(), g.w.size() * 8);
}

// k-opt leaf rows (48-byte KOptCostTask layout) on instance `handle`: row r uses k_of[r].
// A self-avoiding random walk of L = 2k + 4 distinct nodes on the instance's edge graph
// (restarted from a fresh random node when stuck) is closed into a local tour; k distinct
// tour positions are drawn uniformly and sorted; position p deletes the tour edge
// (tour[p], tour[(p + 1) mod L]), contributing its two ports and its exact distance.
int32_t cees_kopt_rows(void* handle, int64_t rows, const uint8_t* k_of, uint64_t seed, void* out) {
  const Instance& g = *static_cast<Instance*>(handle);
  std::vector<std::vector<int32_t>> adj(static_cast<size_t>(g.n));
  for (size_t e = 0; e < g.eu.size(); ++e) {
    adj[g.eu[e]].push_back(g.ev[e]);
    adj[g.ev[e]].push_back(g.eu[e]);
  }
  struct Row {
    int32_t port[10];
    int64_t deleted;
  };
  static_assert(sizeof(Row) == 48, "task layout");
  Row* rows_out = static_cast<Row*>(out);
  std::mt19937_64 rng(seed);
  std::uniform_int_distribution<int32_t> start_node(0, g.n - 1);
  std::vector<int32_t> tour;
  std::vector<char> on_tour(static_cast<size_t>(g.n), 0);
  std::vector<int32_t> options;
  for (int64_t r = 0; r < rows; ++r) {
    const int32_t k = k_of[r];
    if (k < 3 || k > 5) return -1;
    const int32_t length = 2 * k + 4;
    for (int attempts = 0;; ++attempts) {
      if (attempts > 100000) return -2;
      for (int32_t v : tour) on_tour[v] = 0;
      tour.clear();
      int32_t current = start_node(rng);
      tour.push_back(current);
      on_tour[current] = 1;
      while (static_cast<int32_t>(tour.size()) < length) {
        options.clear();
        for (int32_t next : adj[current]) {
          if (!on_tour[next]) options.push_back(next);
        }
        if (options.empty()) break;
        std::uniform_int_distribution<size_t> pick(0, options.size() - 1);
        current = options[pick(rng)];
        tour.push_back(current);
        on_tour[current] = 1;
      }
      if (static_cast<int32_t>(tour.size()) == length) break;
    }
    std::vector<int32_t> positions(static_cast<size_t>(length));
    for (int32_t i = 0; i < length; ++i) positions[i] = i;
    for (int32_t i = 0; i < k; ++i) {  // partial Fisher-Yates: k distinct positions
      std::uniform_int_distribution<int32_t> pick(i, length - 1);
      std::swap(positions[i], positions[pick(rng)]);
    }
    std::sort(positions.begin(), positions.begin() + k);
    Row& row = rows_out[r];
    std::memset(&row, 0, sizeof(Row));
    for (int32_t e = 0; e < k; ++e) {
      const int32_t p = positions[e];
      const int32_t a = tour[p], b = tour[(p + 1) % length];
      row.port[2 * e] = a;
      row.port[2 * e + 1] = b;
      row.deleted += ExactDistance(g.x[a], g.y[a], g.x[b], g.y[b], g.dist_type);
    }
  }
  for (int32_t v : tour) on_tour[v] = 0;
  return 0;
}

// ---- the disjoint union of many batch instances, with its CSR ---------------------------

struct Batch {
  std::vector<Instance*> parts;
  std::vector<int64_t> node_begin, edge_begin;
  ~Batch() {
    for (Instance* p : parts) delete p;
  }
};

// Builds instances [0, count) of the batching mix in parallel (OpenMP over instances).
void* cees_batch_build(uint64_t base_seed, int32_t count, double n_lo, double n_hi) {
  auto batch = std::make_unique<Batch>();
  batch->parts.assign(static_cast<size_t>(count), nullptr);
#pragma omp parallel for schedule(dynamic, 4)
  for (int32_t i = 0; i < count; ++i) {
    batch->parts[i] = static_cast<Instance*>(cees_batch_instance(base_seed, static_cast<uint64_t>(i), n_lo, n_hi));
  }
  batch->node_begin.assign(static_cast<size_t>(count) + 1, 0);
  batch->edge_begin.assign(static_cast<size_t>(count) + 1, 0);
  for (int32_t i = 0; i < count; ++i) {
    batch->node_begin[i + 1] = batch->node_begin[i] + batch->parts[i]->n;
    batch->edge_begin[i + 1] = batch->edge_begin[i] + static_cast<int64_t>(batch->parts[i]->eu.size());
  }
  return batch.release();
}

void cees_batch_free(void* handle) { delete static_cast<Batch*>(handle); }

void cees_batch_sizes(void* handle, int64_t* nodes, int64_t* edges) {
  const Batch& b = *static_cast<Batch*>(handle);
  *nodes = b.node_begin.back();
  *edges = b.edge_begin.back();
}

// Union arrays with global node ids and edge ids; the union edge list stays sorted by (u, v),
// so its CSR (rows ascending) is the per-instance CSR shifted by the offsets.
void cees_batch_copy(void* handle, int64_t* node_begin, int64_t* edge_begin, int64_t* x, int64_t* y,
                     int32_t* eu, int32_t* ev, int64_t* w, int32_t* row_offsets, int32_t* neighbors,
                     int32_t* csr_edge_ids) {
  const Batch& b = *static_cast<Batch*>(handle);
  const int32_t count = static_cast<int32_t>(b.parts.size());
  std::memcpy(node_begin, b.node_begin.data(), b.node_begin.size() * 8);
  std::memcpy(edge_begin, b.edge_begin.data(), b.edge_begin.size() * 8);
  row_offsets[0] = 0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int32_t i = 0; i < count; ++i) {
    const Instance& g = *b.parts[i];
    const int64_t n0 = b.node_begin[i], e0 = b.edge_begin[i];
    const int64_t m = static_cast<int64_t>(g.eu.size());
    std::vector<int32_t> degree(static_cast<size_t>(g.n) + 1, 0);
    for (int64_t e = 0; e < m; ++e) {
      eu[e0 + e] = static_cast<int32_t>(g.eu[e] + n0);
      ev[e0 + e] = static_cast<int32_t>(g.ev[e] + n0);
      w[e0 + e] = g.w[e];
      ++degree[g.eu[e] + 1];
      ++degree[g.ev[e] + 1];
    }
    for (int32_t v = 0; v < g.n; ++v) {
      x[n0 + v] = g.x[v];
      y[n0 + v] = g.y[v];
      degree[v + 1] += degree[v];
    }
    // slot base of this instance = 2 * (edges before it): every edge is active
    const int64_t s0 = 2 * e0;
    for (int32_t v = 0; v < g.n; ++v) row_offsets[n0 + v + 1] = static_cast<int32_t>(s0 + degree[v + 1]);
    std::vector<int32_t> cursor(degree.begin(), degree.end() - 1);
    for (int64_t e = 0; e < m; ++e) {  // edge-id order, u-row then v-row (rows come out ascending)
      int64_t slot = s0 + cursor[g.eu[e]]++;
      neighbors[slot] = static_cast<int32_t>(g.ev[e] + n0);
      csr_edge_ids[slot] = static_cast<int32_t>(e0 + e);
      slot = s0 + cursor[g.ev[e]]++;
      neighbors[slot] = static_cast<int32_t>(g.eu[e] + n0);
      csr_edge_ids[slot] = static_cast<int32_t>(e0 + e);
    }
  }
}

}  // extern "C"
