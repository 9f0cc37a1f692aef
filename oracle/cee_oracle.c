/* Test infrastructure: CPU oracle for the edge-elimination screen (see cee_oracle.h).
 * Plain C11 + the GCC __int128 extension, which the reference uses for the same checks.
 * Reference citations are paths inside the reference project. */
#include "cee_oracle.h"

#include <stdlib.h>
#include <string.h>

#define CEO_MAX_CANDIDATES 10 /* src/cpu/jv_elimination.cpp:28 */

/* ---- exact distance: src/common/distance.cpp:9-27 (restoring isqrt), :29-68 ---- */

uint64_t ceo_isqrt(uint64_t value) {
  uint64_t remainder = value, root = 0, bit = (uint64_t)1 << 62;
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
  return root;
}

int64_t ceo_distance(int64_t x1, int64_t y1, int64_t x2, int64_t y2, int32_t type) {
  const __int128 dx = (__int128)x1 - x2;
  const __int128 dy = (__int128)y1 - y2;
  const __int128 squared = dx * dx + dy * dy;
  if (squared < 0 || squared > (__int128)UINT64_MAX) return -1;
  const uint64_t s = (uint64_t)squared;
  const uint64_t root = ceo_isqrt(s);
  uint64_t rounded = root;
  if (type == CEO_EUC_2D) {
    if (s - root * root > root) ++rounded; /* s > r^2 + r  <=>  sqrt(s) >= r + 1/2 */
  } else {
    if (root * root != s) ++rounded;
  }
  if (rounded > (uint64_t)INT64_MAX) return -1;
  return (int64_t)rounded;
}

void ceo_distance_pairs(const int64_t* x, const int64_t* y, int32_t type, int64_t count, const int32_t* pi,
                        const int32_t* pj, int64_t* out) {
  for (int64_t k = 0; k < count; ++k) out[k] = ceo_distance(x[pi[k]], y[pi[k]], x[pj[k]], y[pj[k]], type);
}

static int64_t dist_nodes(const ceo_graph* g, int32_t a, int32_t b) {
  return ceo_distance(g->x[a], g->y[a], g->x[b], g->y[b], g->dist_type);
}

/* ---- CSR: src/common/graph.cpp:230-282 ---- */

typedef struct {
  int32_t neighbor, edge_id;
  int64_t weight;
} csr_slot;

static int cmp_slot(const void* lhs, const void* rhs) {
  const csr_slot* a = lhs;
  const csr_slot* b = rhs;
  if (a->neighbor != b->neighbor) return a->neighbor < b->neighbor ? -1 : 1;
  if (a->edge_id != b->edge_id) return a->edge_id < b->edge_id ? -1 : 1;
  if (a->weight != b->weight) return a->weight < b->weight ? -1 : 1;
  return 0;
}

int ceo_rebuild_csr(int32_t n, int64_t m, const int32_t* eu, const int32_t* ev, const int64_t* w,
                    const uint8_t* active, int32_t* row_offsets, int32_t* neighbors,
                    int32_t* csr_edge_ids, int64_t* csr_weights) {
  int canonical_sorted = 1;
  for (int64_t e = 0; e < m && canonical_sorted; ++e) {
    if (eu[e] >= ev[e]) canonical_sorted = 0;
    if (e > 0 && (eu[e - 1] > eu[e] || (eu[e - 1] == eu[e] && ev[e - 1] > ev[e]))) {
      canonical_sorted = 0;
    }
  }
  memset(row_offsets, 0, sizeof(int32_t) * ((size_t)n + 1));
  for (int64_t e = 0; e < m; ++e) {
    if (!active[e]) continue;
    ++row_offsets[eu[e] + 1];
    ++row_offsets[ev[e] + 1];
  }
  for (int32_t i = 1; i <= n; ++i) row_offsets[i] += row_offsets[i - 1];
  int32_t* cursor = malloc(sizeof(int32_t) * ((size_t)n + 1));
  if (cursor == NULL) return -1;
  memcpy(cursor, row_offsets, sizeof(int32_t) * ((size_t)n + 1));
  for (int64_t e = 0; e < m; ++e) {
    if (!active[e]) continue;
    int32_t s = cursor[eu[e]]++;
    neighbors[s] = ev[e];
    csr_edge_ids[s] = (int32_t)e;
    csr_weights[s] = w[e];
    s = cursor[ev[e]]++;
    neighbors[s] = eu[e];
    csr_edge_ids[s] = (int32_t)e;
    csr_weights[s] = w[e];
  }
  free(cursor);
  if (canonical_sorted) return 0;
  for (int32_t v = 0; v < n; ++v) {
    const int32_t begin = row_offsets[v], end = row_offsets[v + 1];
    if (end - begin < 2) continue;
    csr_slot* row = malloc(sizeof(csr_slot) * (size_t)(end - begin));
    if (row == NULL) return -1;
    for (int32_t i = begin; i < end; ++i) {
      row[i - begin].neighbor = neighbors[i];
      row[i - begin].edge_id = csr_edge_ids[i];
      row[i - begin].weight = csr_weights[i];
    }
    qsort(row, (size_t)(end - begin), sizeof(csr_slot), cmp_slot);
    for (int32_t i = begin; i < end; ++i) {
      neighbors[i] = row[i - begin].neighbor;
      csr_edge_ids[i] = row[i - begin].edge_id;
      csr_weights[i] = row[i - begin].weight;
    }
    free(row);
  }
  return 0;
}

static int32_t degree(const ceo_graph* g, int32_t v) {
  return g->row_offsets[v + 1] - g->row_offsets[v];
}

/* GraphSnapshot::HasActiveEdge, src/common/graph.cpp:356-364 (binary search in row u). */
static int has_active_edge(const ceo_graph* g, int32_t u, int32_t v) {
  if (u < 0 || v < 0 || u >= g->n || v >= g->n) return 0;
  int32_t lo = g->row_offsets[u], hi = g->row_offsets[u + 1];
  while (lo < hi) {
    const int32_t mid = lo + (hi - lo) / 2;
    if (g->neighbors[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo < g->row_offsets[u + 1] && g->neighbors[lo] == v;
}

/* ---- JV: src/cpu/jv_elimination.cpp:45-84 (candidates), :86-117 (witness) ---- */

typedef struct {
  int64_t score;
  int32_t node;
} scored_node;

/* Keeps the CEO_MAX_CANDIDATES smallest (score, node) pairs in ascending order; the
 * reference re-sorts after each push and drops the tail, which selects the same set. */
static void insert_candidate(scored_node* list, int32_t* count, int64_t score, int32_t node) {
  int32_t pos = *count;
  if (pos == CEO_MAX_CANDIDATES) {
    const scored_node* last = &list[CEO_MAX_CANDIDATES - 1];
    if (!(score < last->score || (score == last->score && node < last->node))) return;
    pos = CEO_MAX_CANDIDATES - 1;
  } else {
    ++*count;
  }
  while (pos > 0 && (score < list[pos - 1].score ||
                     (score == list[pos - 1].score && node < list[pos - 1].node))) {
    list[pos] = list[pos - 1];
    --pos;
  }
  list[pos].score = score;
  list[pos].node = node;
}

static int32_t potential_candidates(const ceo_graph* g, int32_t a, int32_t b, int32_t* out,
                                    int64_t* evals) {
  scored_node list[CEO_MAX_CANDIDATES];
  int32_t count = 0;
  for (int side = 0; side < 2; ++side) {
    const int32_t from = side == 0 ? a : b;
    const int32_t other = side == 0 ? b : a;
    for (int32_t off = g->row_offsets[from]; off < g->row_offsets[from + 1]; ++off) {
      const int32_t c = g->neighbors[off];
      if (c == a || c == b) continue;
      /* second row: nodes already visited through N(a) are not scored again */
      if (side == 1 && has_active_edge(g, a, c)) continue;
      const __int128 score = (__int128)g->csr_weights[off] + dist_nodes(g, c, other);
      ++*evals;
      if (score > (__int128)INT64_MAX) continue;
      insert_candidate(list, &count, (int64_t)score, c);
    }
  }
  for (int32_t i = 0; i < count; ++i) out[i] = list[i].node;
  return count;
}

static int is_jv_witness(const ceo_graph* g, int32_t edge_id, int32_t witness, int64_t* evals) {
  const int32_t u = g->edge_u[edge_id], v = g->edge_v[edge_id];
  if (witness < 0 || witness >= g->n || witness == u || witness == v) return 0;
  const int64_t cab = g->edge_w[edge_id];
  const int64_t cac = dist_nodes(g, u, witness);
  const int64_t cbc = dist_nodes(g, v, witness);
  *evals += 2;
  for (int32_t off = g->row_offsets[witness]; off < g->row_offsets[witness + 1]; ++off) {
    const int32_t d = g->neighbors[off];
    if (d == u || d == v) continue;
    const __int128 left = (__int128)cab + g->csr_weights[off];
    const __int128 first = (__int128)cac + dist_nodes(g, d, v);
    const __int128 second = (__int128)dist_nodes(g, u, d) + cbc;
    *evals += 2;
    if (left <= first || left <= second) return 0; /* d is compatible with (a,b) */
  }
  return 1;
}

/* FindJvCandidatesCpu, src/cpu/jv_elimination.cpp:209-224. */
int64_t ceo_jv_screen_range(const ceo_graph* g, int64_t first, int64_t last, int32_t* witness,
                            int64_t* dist_evals) {
  int64_t found = 0;
  for (int64_t e = first; e < last; ++e) {
    int64_t evals = 0;
    witness[e] = -1;
    const int32_t u = g->edge_u[e], v = g->edge_v[e];
    if (g->active[e] && degree(g, u) > 2 && degree(g, v) > 2) {
      int32_t cands[CEO_MAX_CANDIDATES];
      const int32_t count = potential_candidates(g, u, v, cands, &evals);
      for (int32_t i = 0; i < count; ++i) {
        if (is_jv_witness(g, (int32_t)e, cands[i], &evals)) {
          witness[e] = cands[i];
          ++found;
          break;
        }
      }
    }
    if (dist_evals != NULL) dist_evals[e] = evals;
  }
  return found;
}

int64_t ceo_jv_screen(const ceo_graph* g, int32_t* witness, int64_t* dist_evals) {
  return ceo_jv_screen_range(g, 0, g->m, witness, dist_evals);
}

/* VerifyJvCandidate, src/cpu/jv_elimination.cpp:226-248. */
int ceo_jv_verify(const ceo_graph* g, int32_t edge_id, int32_t witness) {
  if (edge_id < 0 || edge_id >= g->m) return 0;
  const int32_t u = g->edge_u[edge_id], v = g->edge_v[edge_id];
  if (!g->active[edge_id] || degree(g, u) <= 2 || degree(g, v) <= 2) return 0;
  int64_t evals = 0;
  return is_jv_witness(g, edge_id, witness, &evals);
}

/* ---- ContentHash: src/common/graph.cpp:323-346 (FNV-1a over field bytes) ---- */

static void fnv_bytes(uint64_t* hash, const void* data, size_t size) {
  const unsigned char* bytes = data;
  for (size_t i = 0; i < size; ++i) {
    *hash ^= bytes[i];
    *hash *= 1099511628211ULL;
  }
}

uint64_t ceo_content_hash(const ceo_graph* g) {
  uint64_t hash = 14695981039346656037ULL;
  const uint8_t type = (uint8_t)g->dist_type, integer = 1;
  fnv_bytes(&hash, &g->n, sizeof(int32_t));
  fnv_bytes(&hash, &type, 1);
  fnv_bytes(&hash, &integer, 1);
  for (int32_t i = 0; i < g->n; ++i) {
    fnv_bytes(&hash, &g->x[i], 8);
    fnv_bytes(&hash, &g->y[i], 8);
  }
  for (int64_t e = 0; e < g->m; ++e) {
    const uint8_t act = g->active[e] ? 1 : 0;
    fnv_bytes(&hash, &g->edge_u[e], 4);
    fnv_bytes(&hash, &g->edge_v[e], 4);
    fnv_bytes(&hash, &g->edge_w[e], 8);
    fnv_bytes(&hash, &act, 1);
  }
  return hash;
}

/* ---- commit gate: src/cpu/elimination_commit.cpp:13-76 ---- */

typedef struct {
  int32_t u, v, witness, edge_id;
} commit_key;

static int cmp_commit(const void* lhs, const void* rhs) {
  const commit_key* a = lhs;
  const commit_key* b = rhs;
  if (a->u != b->u) return a->u < b->u ? -1 : 1;
  if (a->v != b->v) return a->v < b->v ? -1 : 1;
  /* method is JV for every candidate here */
  if (a->witness != b->witness) return a->witness < b->witness ? -1 : 1;
  if (a->edge_id != b->edge_id) return a->edge_id < b->edge_id ? -1 : 1;
  return 0;
}

int64_t ceo_jv_commit(const ceo_graph* g, const int32_t* cand_edge, const int32_t* cand_witness,
                      int64_t count, int32_t* committed_edges, int32_t* committed_witness,
                      uint8_t* active_out) {
  commit_key* keys = malloc(sizeof(commit_key) * (size_t)(count > 0 ? count : 1));
  int32_t* deg = malloc(sizeof(int32_t) * (size_t)(g->n > 0 ? g->n : 1));
  if (keys == NULL || deg == NULL) {
    free(keys);
    free(deg);
    return -1;
  }
  for (int64_t i = 0; i < count; ++i) {
    keys[i].u = g->edge_u[cand_edge[i]];
    keys[i].v = g->edge_v[cand_edge[i]];
    keys[i].witness = cand_witness[i];
    keys[i].edge_id = cand_edge[i];
  }
  qsort(keys, (size_t)count, sizeof(commit_key), cmp_commit);
  int64_t unique = 0;
  for (int64_t i = 0; i < count; ++i) {
    if (unique == 0 || keys[unique - 1].edge_id != keys[i].edge_id) keys[unique++] = keys[i];
  }
  for (int32_t v = 0; v < g->n; ++v) deg[v] = degree(g, v);
  memcpy(active_out, g->active, (size_t)g->m);
  int64_t committed = 0;
  for (int64_t i = 0; i < unique; ++i) {
    if (deg[keys[i].u] <= 2 || deg[keys[i].v] <= 2) continue;
    --deg[keys[i].u];
    --deg[keys[i].v];
    if (committed_edges != NULL) committed_edges[committed] = keys[i].edge_id;
    if (committed_witness != NULL) committed_witness[committed] = keys[i].witness;
    active_out[keys[i].edge_id] = 0;
    ++committed;
  }
  free(keys);
  free(deg);
  return committed;
}

/* RunJvElimination, src/cpu/jv_elimination.cpp:250-322 (CPU backend; every CPU
 * candidate verifies by construction, so the verify step is the identity). */
int32_t ceo_jv_eliminate(int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y,
                         int64_t m, const int32_t* edge_u, const int32_t* edge_v,
                         const int64_t* edge_w, uint8_t* active, uint32_t max_rounds,
                         int64_t* epoch_edges_before, int64_t* epoch_committed,
                         uint64_t* final_hash) {
  const size_t slots = (size_t)(2 * m > 0 ? 2 * m : 1);
  int32_t* ro = malloc(sizeof(int32_t) * ((size_t)n + 1));
  int32_t* nb = malloc(sizeof(int32_t) * slots);
  int32_t* ids = malloc(sizeof(int32_t) * slots);
  int64_t* ws = malloc(sizeof(int64_t) * slots);
  int32_t* witness = malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  int32_t* cand_e = malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  int32_t* cand_w = malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  uint8_t* next = malloc((size_t)(m > 0 ? m : 1));
  int32_t epochs = -1;
  if (ro && nb && ids && ws && witness && cand_e && cand_w && next) {
    ceo_graph g = {n, dist_type, x, y, m, edge_u, edge_v, edge_w, active, ro, nb, ids, ws};
    epochs = 0;
    for (uint32_t epoch = 0; epoch < max_rounds; ++epoch) {
      ceo_rebuild_csr(n, m, edge_u, edge_v, edge_w, active, ro, nb, ids, ws);
      int64_t before = 0;
      for (int64_t e = 0; e < m; ++e) before += active[e] ? 1 : 0;
      ceo_jv_screen(&g, witness, NULL);
      int64_t count = 0;
      for (int64_t e = 0; e < m; ++e) {
        if (witness[e] >= 0) {
          cand_e[count] = (int32_t)e;
          cand_w[count] = witness[e];
          ++count;
        }
      }
      const int64_t committed = ceo_jv_commit(&g, cand_e, cand_w, count, NULL, NULL, next);
      memcpy(active, next, (size_t)m);
      if (epoch_edges_before != NULL) epoch_edges_before[epochs] = before;
      if (epoch_committed != NULL) epoch_committed[epochs] = committed;
      ++epochs;
      if (committed == 0) break;
    }
    ceo_rebuild_csr(n, m, edge_u, edge_v, edge_w, active, ro, nb, ids, ws);
    if (final_hash != NULL) *final_hash = ceo_content_hash(&g);
  }
  free(ro);
  free(nb);
  free(ids);
  free(ws);
  free(witness);
  free(cand_e);
  free(cand_w);
  free(next);
  return epochs;
}

/* ---- k-opt templates: src/cpu/kopt_search.cpp:1143-1193 with
 *      EnumerateInsideMatchings (src/cpu/path_system.cpp:46-70, 377-387) and
 *      IsAlternatingHamiltonianCycle (src/cpu/path_system.cpp:404-420) ---- */

#define CEO_UNMATCHED 0xffu

typedef struct {
  uint8_t count;
  uint8_t mate[14];
} matching;

static int alternating_cycle(const matching* outside, const matching* inside, uint32_t k) {
  uint8_t visited[14] = {0};
  uint32_t current = 0, steps = 0;
  for (uint32_t p = 0; p < 2 * k; ++p) {
    if (inside->mate[p] >= 2 * k || inside->mate[p] == p || inside->mate[inside->mate[p]] != p) return 0;
    if (outside->mate[p] >= 2 * k || outside->mate[p] == p || outside->mate[outside->mate[p]] != p) return 0;
  }
  while (!visited[current]) {
    visited[current] = 1;
    current = (steps % 2 == 0) ? inside->mate[current] : outside->mate[current];
    ++steps;
  }
  return steps == 2 * k && current == 0;
}

typedef struct {
  const matching* components;
  uint32_t k;
  uint8_t* out;
  int32_t count;
} template_sink;

static void enumerate_inside(matching* m, template_sink* sink) {
  uint32_t first = m->count;
  for (uint32_t p = 0; p < m->count; ++p) {
    if (m->mate[p] == CEO_UNMATCHED) {
      first = p;
      break;
    }
  }
  if (first == m->count) {
    /* a proper template closes one alternating cycle and re-adds no deleted edge */
    if (!alternating_cycle(sink->components, m, sink->k)) return;
    for (uint32_t e = 0; e < sink->k; ++e) {
      if (m->mate[2 * e] == 2 * e + 1) return;
    }
    if (sink->out != NULL) memcpy(sink->out + 14 * sink->count, m->mate, 14);
    ++sink->count;
    return;
  }
  for (uint32_t second = first + 1; second < m->count; ++second) {
    if (m->mate[second] != CEO_UNMATCHED) continue;
    m->mate[first] = (uint8_t)second;
    m->mate[second] = (uint8_t)first;
    enumerate_inside(m, sink);
    m->mate[first] = CEO_UNMATCHED;
    m->mate[second] = CEO_UNMATCHED;
  }
}

static void fnv_byte(uint64_t* hash, uint8_t value) {
  *hash ^= value;
  *hash *= 1099511628211ULL;
}

static void fnv_u32_le(uint64_t* hash, uint32_t value) {
  for (uint32_t shift = 0; shift < 32; shift += 8) fnv_byte(hash, (uint8_t)((value >> shift) & 0xffu));
}

int32_t ceo_kopt_templates(uint32_t k, uint8_t* mates, uint64_t* generator_hash) {
  if (k < 3 || k > 5) return -1;
  matching components, inside;
  components.count = inside.count = (uint8_t)(2 * k);
  memset(components.mate, CEO_UNMATCHED, 14);
  memset(inside.mate, CEO_UNMATCHED, 14);
  /* component matching: 1-2, 3-4, ..., (2k-1)-0 */
  for (uint32_t e = 0; e + 1 < k; ++e) {
    components.mate[2 * e + 1] = (uint8_t)(2 * e + 2);
    components.mate[2 * e + 2] = (uint8_t)(2 * e + 1);
  }
  components.mate[2 * k - 1] = 0;
  components.mate[0] = (uint8_t)(2 * k - 1);
  template_sink sink = {&components, k, mates, 0};
  enumerate_inside(&inside, &sink);
  if (generator_hash != NULL) {
    uint64_t hash = 14695981039346656037ULL;
    const char* domain = "CUDAEE_KOPT_RECONNECT_TEMPLATES_V1";
    for (const char* p = domain; *p != '\0'; ++p) fnv_byte(&hash, (uint8_t)*p);
    fnv_u32_le(&hash, k);
    fnv_u32_le(&hash, (uint32_t)sink.count);
    if (mates != NULL) {
      for (int32_t t = 0; t < sink.count; ++t) {
        for (uint32_t p = 0; p < 2 * k; ++p) fnv_byte(&hash, mates[14 * t + p]);
      }
    }
    *generator_hash = hash;
  }
  return sink.count;
}

/* ---- k-opt cell cost: src/cpu/kopt_search.cpp:962-1042, the edge-list oracle of
 *      tests/unit/test_kopt.cpp:48-74 ---- */

void ceo_kopt_costs(int32_t dist_type, const int64_t* x, const int64_t* y, uint32_t k,
                    const ceo_kopt_task* tasks, int64_t rows, const uint8_t* mates,
                    int32_t template_count, int64_t* costs) {
  for (int64_t r = 0; r < rows; ++r) {
    const int32_t* port = tasks[r].port_nodes;
    int32_t del_u[5], del_v[5];
    for (uint32_t e = 0; e < k; ++e) {
      const int32_t a = port[2 * e], b = port[2 * e + 1];
      del_u[e] = a < b ? a : b;
      del_v[e] = a < b ? b : a;
    }
    for (int32_t t = 0; t < template_count; ++t) {
      const uint8_t* mate = mates + 14 * t;
      int32_t add_u[5], add_v[5];
      uint32_t added = 0;
      __int128 total = 0;
      int invalid = 0;
      for (uint32_t p = 0; p < 2 * k && !invalid; ++p) {
        const uint32_t q = mate[p];
        if (p >= q) continue;
        const int32_t a = port[p], b = port[q];
        const int32_t u = a < b ? a : b, v = a < b ? b : a;
        if (u == v) invalid = 1;
        for (uint32_t e = 0; e < k && !invalid; ++e) {
          if (u == del_u[e] && v == del_v[e]) invalid = 1;
        }
        for (uint32_t e = 0; e < added && !invalid; ++e) {
          if (u == add_u[e] && v == add_v[e]) invalid = 1;
        }
        if (invalid) break;
        const int64_t dist = ceo_distance(x[u], y[u], x[v], y[v], dist_type);
        if (dist < 0) {
          invalid = 1;
          break;
        }
        add_u[added] = u;
        add_v[added] = v;
        ++added;
        total += dist;
      }
      costs[r * template_count + t] =
          (invalid || added != k || total > (__int128)INT64_MAX) ? CEO_INVALID_COST : (int64_t)total;
    }
  }
}

/* ---- HT c,d: src/cpu/hamilton_tutte.cpp:79-101 (admissibility), :168-216 (tasks) ---- */

typedef struct {
  __int128 score;
  int32_t node;
} ranked_node;

static int cmp_ranked(const void* lhs, const void* rhs) {
  const ranked_node* a = lhs;
  const ranked_node* b = rhs;
  if (a->score != b->score) return a->score < b->score ? -1 : 1;
  if (a->node != b->node) return a->node < b->node ? -1 : 1;
  return 0;
}

int64_t ceo_cd_tasks(const ceo_graph* g, int32_t u, int32_t v, uint32_t max_neighborhood,
                     uint32_t max_candidate_degree, int32_t* c, int32_t* d, uint8_t* active) {
  ranked_node* ranked = malloc(sizeof(ranked_node) * (size_t)(g->n > 0 ? g->n : 1));
  if (ranked == NULL) return -1;
  int64_t count = 0;
  for (int32_t node = 0; node < g->n; ++node) {
    if (node == u || node == v ||
        (max_candidate_degree != 0 && (uint32_t)degree(g, node) > max_candidate_degree)) {
      continue;
    }
    /* doubled midpoint coordinates keep the ranking in exact integers */
    const __int128 dx = (__int128)2 * g->x[node] - g->x[u] - g->x[v];
    const __int128 dy = (__int128)2 * g->y[node] - g->y[u] - g->y[v];
    ranked[count].score = dx * dx + dy * dy;
    ranked[count].node = node;
    ++count;
  }
  qsort(ranked, (size_t)count, sizeof(ranked_node), cmp_ranked);
  if (max_neighborhood != 0 && count > (int64_t)max_neighborhood) count = max_neighborhood;
  int64_t tasks = 0;
  for (int64_t i = 0; i < count; ++i) {
    for (int64_t j = i + 1; j < count; ++j) {
      const int32_t a = ranked[i].node, b = ranked[j].node;
      c[tasks] = a < b ? a : b;
      d[tasks] = a < b ? b : a;
      active[tasks] = (uint8_t)has_active_edge(g, c[tasks], d[tasks]);
      ++tasks;
    }
  }
  free(ranked);
  return tasks;
}

/* EdgesSurviveTwoOpt (:79-87): at least one 2-opt orientation is not a strict gain. */
static int survives_two_opt(const ceo_graph* g, int32_t tu, int32_t tv, int32_t ou, int32_t ov) {
  const __int128 original = (__int128)dist_nodes(g, tu, tv) + dist_nodes(g, ou, ov);
  const __int128 first = (__int128)dist_nodes(g, tu, ov) + dist_nodes(g, tv, ou);
  const __int128 second = (__int128)dist_nodes(g, tu, ou) + dist_nodes(g, tv, ov);
  return first >= original || second >= original;
}

/* ScreenCdTasksCpu (:218-228) over CandidateIsAdmissible (:89-101); the active bit is
 * recomputed from the snapshot as the reference does. */
void ceo_cd_screen(const ceo_graph* g, int32_t u, int32_t v, const int32_t* c, const int32_t* d,
                   const uint8_t* active, int64_t count, int32_t mode, uint8_t* flags) {
  (void)active;
  const int32_t tu = u < v ? u : v, tv = u < v ? v : u;
  for (int64_t i = 0; i < count; ++i) {
    const int32_t ci = c[i], di = d[i];
    if ((mode != 0 && mode != 1) || ci < 0 || di < 0 || ci >= g->n || di >= g->n || ci == di ||
        ci == tu || ci == tv || di == tu || di == tv) {
      flags[i] = 0;
      continue;
    }
    const int act = has_active_edge(g, ci, di);
    const int32_t ou = ci < di ? ci : di, ov = ci < di ? di : ci;
    const int incompatible = !survives_two_opt(g, tu, tv, ou, ov);
    flags[i] = (uint8_t)(mode == 0 ? (act && incompatible) : (!act || incompatible));
  }
}

/* ---- FinalizeCdCandidates: src/cpu/hamilton_tutte.cpp:283-327 ---- */

/* AppendHtHamiltonRepliesUnchecked (:230-269): pairs of neighbours (first < second in CSR order)
 * of `center` whose edges to the center both survive 2-opt against the target, whose node pair is
 * not the target, and for which the target plus the two center edges cost no more than the pair's
 * edge plus the center's two target edges. Writes the first `capacity` of them to `out` as
 * (center, first, second) triples (NULL: none) and returns how many there are. */
int64_t ceo_ht_replies(const ceo_graph* g, int32_t tu, int32_t tv, int32_t center, int32_t* out, int64_t capacity) {
  const int32_t begin = g->row_offsets[center], end = g->row_offsets[center + 1];
  const int32_t deg = end - begin;
  if (deg < 2) return 0;
  int64_t* cost = malloc(sizeof(int64_t) * (size_t)deg);
  int* survives = malloc(sizeof(int) * (size_t)deg);
  int64_t count = 0;
  if (cost != NULL && survives != NULL) {
    for (int32_t i = 0; i < deg; ++i) {
      const int32_t node = g->neighbors[begin + i];
      cost[i] = dist_nodes(g, center, node);
      const int32_t ou = center < node ? center : node, ov = center < node ? node : center;
      survives[i] = survives_two_opt(g, tu, tv, ou, ov);
    }
    const __int128 target_cost = dist_nodes(g, tu, tv);
    const __int128 center_target = (__int128)dist_nodes(g, tu, center) + dist_nodes(g, tv, center);
    for (int32_t a = 0; a < deg; ++a) {
      for (int32_t b = a + 1; b < deg; ++b) {
        const int32_t na = g->neighbors[begin + a], nb = g->neighbors[begin + b];
        const int32_t lo = na < nb ? na : nb, hi = na < nb ? nb : na;
        if ((lo == tu && hi == tv) || !survives[a] || !survives[b]) continue;
        const __int128 original = target_cost + cost[a] + cost[b];
        const __int128 replacement = (__int128)dist_nodes(g, na, nb) + center_target;
        if (original <= replacement) {
          if (out != NULL && count < capacity) {
            out[3 * count] = center;
            out[3 * count + 1] = na;
            out[3 * count + 2] = nb;
          }
          ++count;
        }
      }
    }
  }
  free(cost);
  free(survives);
  return count;
}

int64_t ceo_ht_reply_count(const ceo_graph* g, int32_t tu, int32_t tv, int32_t center) {
  return ceo_ht_replies(g, tu, tv, center, NULL, 0);
}

/* AppendHtEndRepliesUnchecked (:271-282): the edges at `endpoint` other than the one to
 * `internal_neighbor`, each as (lower id, higher id), in CSR order; writes the first `capacity`
 * pairs to `out` (NULL: none) and returns their number, or -1 when `internal_neighbor` is not a
 * neighbour of `endpoint`. */
int64_t ceo_ht_end_replies(const ceo_graph* g, int32_t endpoint, int32_t internal_neighbor, int32_t* out,
                           int64_t capacity) {
  const int32_t begin = g->row_offsets[endpoint], end = g->row_offsets[endpoint + 1];
  int found = 0;
  int64_t count = 0;
  for (int32_t s = begin; s < end; ++s) {
    const int32_t nb = g->neighbors[s];
    if (nb == internal_neighbor) {
      found = 1;
      continue;
    }
    if (out != NULL && count < capacity) {
      out[2 * count] = endpoint < nb ? endpoint : nb;
      out[2 * count + 1] = endpoint < nb ? nb : endpoint;
    }
    ++count;
  }
  return found ? count : -1;
}

typedef struct {
  uint64_t product;
  int32_t c, d;
} cd_candidate;

static int cmp_cd_candidate(const void* lhs, const void* rhs) {
  const cd_candidate* a = lhs;
  const cd_candidate* b = rhs;
  if (a->product != b->product) return a->product < b->product ? -1 : 1;
  if (a->c != b->c) return a->c < b->c ? -1 : 1;
  if (a->d != b->d) return a->d < b->d ? -1 : 1;
  return 0;
}

/* The flagged tasks ranked by (reply product, c, d), saturating the product at 2^64 - 1, first
 * max_cd kept (0 = all). Writes (c, d, product) triples; returns the count or -1. */
int64_t ceo_cd_finalize(const ceo_graph* g, int32_t u, int32_t v, const int32_t* c, const int32_t* d,
                        const uint8_t* flags, int64_t count, uint32_t max_cd, int32_t* out_c, int32_t* out_d,
                        uint64_t* out_product) {
  const int32_t tu = u < v ? u : v, tv = u < v ? v : u;
  cd_candidate* list = malloc(sizeof(cd_candidate) * (size_t)(count > 0 ? count : 1));
  if (list == NULL) return -1;
  int64_t kept = 0;
  for (int64_t i = 0; i < count; ++i) {
    if (flags[i] == 0) continue;
    const uint64_t rc = (uint64_t)ceo_ht_reply_count(g, tu, tv, c[i]);
    const uint64_t rd = (uint64_t)ceo_ht_reply_count(g, tu, tv, d[i]);
    uint64_t product = 0;
    if (rc != 0 && rd > UINT64_MAX / rc) {
      product = UINT64_MAX;
    } else {
      product = rc * rd;
    }
    list[kept].product = product;
    list[kept].c = c[i];
    list[kept].d = d[i];
    ++kept;
  }
  qsort(list, (size_t)kept, sizeof(cd_candidate), cmp_cd_candidate);
  if (max_cd != 0 && kept > (int64_t)max_cd) kept = max_cd;
  for (int64_t i = 0; i < kept; ++i) {
    out_c[i] = list[i].c;
    out_d[i] = list[i].d;
    out_product[i] = list[i].product;
  }
  free(list);
  return kept;
}

/* ---- SelectHtTargetEdgeIds: src/cpu/ht_scan.cpp:316-345 ---- */

/* Per thread, so that several host threads may check instances at once. */
static _Thread_local const ceo_graph* g_target_graph;
static _Thread_local int32_t g_target_order;

static int cmp_target(const void* lhs, const void* rhs) {
  const int32_t a = *(const int32_t*)lhs, b = *(const int32_t*)rhs;
  const ceo_graph* g = g_target_graph;
  if (g_target_order == 1 && g->edge_w[a] != g->edge_w[b]) return g->edge_w[a] > g->edge_w[b] ? -1 : 1;
  if (g->edge_u[a] != g->edge_u[b]) return g->edge_u[a] < g->edge_u[b] ? -1 : 1;
  if (g->edge_v[a] != g->edge_v[b]) return g->edge_v[a] < g->edge_v[b] ? -1 : 1;
  return a < b ? -1 : (a > b ? 1 : 0);
}

int64_t ceo_ht_targets(const ceo_graph* g, int32_t order, int32_t* out) {
  int64_t count = 0;
  for (int64_t e = 0; e < g->m; ++e) {
    if (g->active[e] && degree(g, g->edge_u[e]) > 2 && degree(g, g->edge_v[e]) > 2) {
      out[count++] = (int32_t)e;
    }
  }
  g_target_graph = g;
  g_target_order = order;
  qsort(out, (size_t)count, sizeof(int32_t), cmp_target);
  return count;
}

/* ---- The batched step of one instance range, in the batched screen's output layout ----
 *
 * For instances [first, last) of a disjoint union (instance i owns nodes
 * [node_begin[i], node_begin[i+1]) and edges [edge_begin[i], edge_begin[i+1])), writes what the
 * reference's CPU code computes for the step, with global node and edge ids:
 *   witness[e]                  FindJvCandidatesCpu (src/cpu/jv_elimination.cpp:209-224)
 *   target_ids[i][t], count[i]  SelectHtTargetEdgeIds (src/cpu/ht_scan.cpp:316-345), first `targets`
 *   nbhd[i][t][NB]              the ranked neighbourhood of BuildCdScreenTasks
 *                               (src/cpu/hamilton_tutte.cpp:168-216), -1 padded
 *   flags[i][t][words]          ScreenCdTasksCpu (:218-228) of its pairs i < j, bit p = task p
 *   cand_*[i][t][max_cd], cand_count[i][t]  FinalizeCdCandidates (:283-327), when max_cd > 0
 * Returns 0, or -1 when memory runs out. */
int ceo_batch_expect(const ceo_graph* g, const int64_t* node_begin, const int64_t* edge_begin, int64_t first,
                     int64_t last, uint32_t targets, uint32_t max_neighborhood, uint32_t max_candidate_degree,
                     int32_t mode, uint32_t flag_words, uint32_t max_cd, int32_t* witness, int32_t* target_ids,
                     int32_t* target_count, int32_t* nbhd, uint32_t* flags, int32_t* cand_c, int32_t* cand_d,
                     int64_t* cand_product, int32_t* cand_count) {
  int64_t max_nodes = 1, max_edges = 1;
  for (int64_t i = first; i < last; ++i) {
    if (node_begin[i + 1] - node_begin[i] > max_nodes) max_nodes = node_begin[i + 1] - node_begin[i];
    if (edge_begin[i + 1] - edge_begin[i] > max_edges) max_edges = edge_begin[i + 1] - edge_begin[i];
  }
  const int64_t pair_cap = (int64_t)max_neighborhood * (max_neighborhood > 0 ? max_neighborhood - 1 : 0) / 2 + 1;
  int32_t* order = malloc(sizeof(int32_t) * (size_t)max_edges);
  ranked_node* ranked = malloc(sizeof(ranked_node) * (size_t)max_nodes);
  int32_t* tc = malloc(sizeof(int32_t) * (size_t)pair_cap);
  int32_t* td = malloc(sizeof(int32_t) * (size_t)pair_cap);
  uint8_t* ta = malloc((size_t)pair_cap);
  uint8_t* tf = malloc((size_t)pair_cap);
  int32_t* oc = malloc(sizeof(int32_t) * (size_t)pair_cap);
  int32_t* od = malloc(sizeof(int32_t) * (size_t)pair_cap);
  uint64_t* op = malloc(sizeof(uint64_t) * (size_t)pair_cap);
  int rc = 0;
  if (!order || !ranked || !tc || !td || !ta || !tf || !oc || !od || !op) {
    rc = -1;
    goto done;
  }
  for (int64_t i = first; i < last; ++i) {
    const int64_t n0 = node_begin[i], n1 = node_begin[i + 1], e0 = edge_begin[i], e1 = edge_begin[i + 1];
    ceo_jv_screen_range(g, e0, e1, witness, NULL);
    /* targets: the instance's eligible edges in SelectHtTargetEdgeIds order */
    int64_t count = 0;
    for (int64_t e = e0; e < e1; ++e) {
      if (g->active[e] && degree(g, g->edge_u[e]) > 2 && degree(g, g->edge_v[e]) > 2) order[count++] = (int32_t)e;
    }
    g_target_graph = g;
    g_target_order = 1;
    qsort(order, (size_t)count, sizeof(int32_t), cmp_target);
    if (count > (int64_t)targets) count = targets;
    target_count[i] = (int32_t)count;
    for (uint32_t t = 0; t < targets; ++t) {
      const size_t slot = (size_t)i * targets + t;
      int32_t* hood = nbhd + slot * max_neighborhood;
      uint32_t* words = flags + slot * flag_words;
      for (uint32_t k = 0; k < max_neighborhood; ++k) hood[k] = -1;
      for (uint32_t k = 0; k < flag_words; ++k) words[k] = 0;
      if (max_cd > 0) {
        cand_count[slot] = 0;
        for (uint32_t k = 0; k < max_cd; ++k) {
          cand_c[slot * max_cd + k] = -1;
          cand_d[slot * max_cd + k] = -1;
          cand_product[slot * max_cd + k] = -1;
        }
      }
      if ((int64_t)t >= count) {
        target_ids[slot] = -1;
        continue;
      }
      const int32_t e = order[t];
      target_ids[slot] = e;
      const int32_t u = g->edge_u[e], v = g->edge_v[e];
      /* the ranked neighbourhood, as ceo_cd_tasks ranks it, over this instance's nodes */
      /* the first max_neighborhood by (score, node): a sorted list with insertion, which keeps
       * exactly the prefix that sorting every eligible node would give */
      int64_t size = 0;
      for (int64_t node = n0; node < n1; ++node) {
        if (node == u || node == v ||
            (max_candidate_degree != 0 && (uint32_t)degree(g, (int32_t)node) > max_candidate_degree)) {
          continue;
        }
        const __int128 dx = (__int128)2 * g->x[node] - g->x[u] - g->x[v];
        const __int128 dy = (__int128)2 * g->y[node] - g->y[u] - g->y[v];
        const ranked_node entry = {dx * dx + dy * dy, (int32_t)node};
        int64_t pos = size;
        if (size == (int64_t)max_neighborhood) {
          if (max_neighborhood == 0 || cmp_ranked(&entry, &ranked[size - 1]) >= 0) continue;
          pos = size - 1;
        } else {
          ++size;
        }
        while (pos > 0 && cmp_ranked(&entry, &ranked[pos - 1]) < 0) {
          ranked[pos] = ranked[pos - 1];
          --pos;
        }
        ranked[pos] = entry;
      }
      int64_t tasks = 0;
      for (int64_t a = 0; a < size; ++a) {
        hood[a] = ranked[a].node;
        for (int64_t b = a + 1; b < size; ++b) {
          const int32_t p = ranked[a].node, q = ranked[b].node;
          tc[tasks] = p < q ? p : q;
          td[tasks] = p < q ? q : p;
          ta[tasks] = (uint8_t)has_active_edge(g, tc[tasks], td[tasks]);
          ++tasks;
        }
      }
      ceo_cd_screen(g, u, v, tc, td, ta, tasks, mode, tf);
      for (int64_t p = 0; p < tasks; ++p) {
        if (tf[p]) words[p >> 5] |= 1u << (p & 31);
      }
      if (max_cd > 0) {
        const int64_t kept = ceo_cd_finalize(g, u, v, tc, td, tf, tasks, max_cd, oc, od, op);
        if (kept < 0) {
          rc = -1;
          goto done;
        }
        cand_count[slot] = (int32_t)kept;
        for (int64_t k = 0; k < kept; ++k) {
          cand_c[slot * max_cd + k] = oc[k];
          cand_d[slot * max_cd + k] = od[k];
          cand_product[slot * max_cd + k] = op[k] > (uint64_t)INT64_MAX ? INT64_MAX : (int64_t)op[k];
        }
      }
    }
  }
done:
  free(order);
  free(ranked);
  free(tc);
  free(td);
  free(ta);
  free(tf);
  free(oc);
  free(od);
  free(op);
  return rc;
}
