/* Test infrastructure: the CPU oracle for the edge-elimination screen.
 *
 * A plain-C restatement of the reference's CPU algorithm for the three screens on the
 * hot path (JV candidates, k-opt template cost matrix, HT c,d root screen) plus the
 * snapshot pieces they read (exact distance, CSR rebuild, content hash, commit gate,
 * target order). Each function cites the reference file:line it restates. It is pinned
 * against the reference's own known-answer tests and against the reference library
 * compiled from its sources (oracle/_ref) by tests/test_oracle_pins.py.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this code,
 * and only as the checker or as the timed CPU baseline; the product never calls it.
 */
#ifndef CEE_ORACLE_H
#define CEE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { CEO_EUC_2D = 0, CEO_CEIL_2D = 1 };
#define CEO_INVALID_COST INT64_MAX

/* A snapshot: coordinates, the stable edge list and the active-only CSR over it. */
typedef struct {
  int32_t n;
  int32_t dist_type;
  const int64_t* x;
  const int64_t* y;
  int64_t m;
  const int32_t* edge_u;
  const int32_t* edge_v;
  const int64_t* edge_w;
  const uint8_t* active;
  const int32_t* row_offsets; /* n + 1 */
  const int32_t* neighbors;   /* row_offsets[n] */
  const int32_t* csr_edge_ids;
  const int64_t* csr_weights;
} ceo_graph;

/* k-opt task row, byte-compatible with the reference's KOptCostTask (48 B). */
typedef struct {
  int32_t port_nodes[10];
  int64_t deleted_cost;
} ceo_kopt_task;

uint64_t ceo_isqrt(uint64_t value);
/* Exact TSPLIB distance; returns -1 when the squared distance overflows uint64. */
int64_t ceo_distance(int64_t x1, int64_t y1, int64_t x2, int64_t y2, int32_t type);
/* ceo_distance of points (pi[k], pj[k]) of (x, y), k < count. */
void ceo_distance_pairs(const int64_t* x, const int64_t* y, int32_t type, int64_t count, const int32_t* pi,
                        const int32_t* pj, int64_t* out);

/* Active-only CSR, rows ascending by neighbour (sort fallback for unsorted edge lists). */
int ceo_rebuild_csr(int32_t n, int64_t m, const int32_t* edge_u, const int32_t* edge_v,
                    const int64_t* edge_w, const uint8_t* active, int32_t* row_offsets,
                    int32_t* neighbors, int32_t* csr_edge_ids, int64_t* csr_weights);

/* JV screen: witness[e] = first witness or -1; returns the candidate count. When
 * dist_evals is non-null it receives, per edge, the number of exact distance
 * evaluations the sequential CPU algorithm performs (the algorithmic op count). */
int64_t ceo_jv_screen(const ceo_graph* g, int32_t* witness, int64_t* dist_evals);
/* Same, restricted to edges [first, last). */
int64_t ceo_jv_screen_range(const ceo_graph* g, int64_t first, int64_t last, int32_t* witness,
                            int64_t* dist_evals);
int ceo_jv_verify(const ceo_graph* g, int32_t edge_id, int32_t witness);

uint64_t ceo_content_hash(const ceo_graph* g);

/* Deterministic commit gate; candidates given as (edge_id, witness) pairs, all JV.
 * Writes committed edge ids (in commit order) and clears their active byte in
 * active_out (a copy of g->active). Returns the committed count. */
int64_t ceo_jv_commit(const ceo_graph* g, const int32_t* cand_edge, const int32_t* cand_witness,
                      int64_t count, int32_t* committed_edges, int32_t* committed_witness,
                      uint8_t* active_out);

/* Full JV loop to a fixed point (max_rounds epochs). active is updated in place.
 * epoch_edges_before[e] = active edges screened in epoch e. Returns the epoch count. */
int32_t ceo_jv_eliminate(int32_t n, int32_t dist_type, const int64_t* x, const int64_t* y,
                         int64_t m, const int32_t* edge_u, const int32_t* edge_v,
                         const int64_t* edge_w, uint8_t* active, uint32_t max_rounds,
                         int64_t* epoch_edges_before, int64_t* epoch_committed,
                         uint64_t* final_hash);

/* Proper k-opt reconnect templates: mates[t * 14 + p]; returns the template count. */
int32_t ceo_kopt_templates(uint32_t k, uint8_t* mates, uint64_t* generator_hash);
void ceo_kopt_costs(int32_t dist_type, const int64_t* x, const int64_t* y, uint32_t k,
                    const ceo_kopt_task* tasks, int64_t rows, const uint8_t* mates,
                    int32_t template_count, int64_t* costs);

/* HT c,d root screen for target (u,v). */
int64_t ceo_cd_tasks(const ceo_graph* g, int32_t u, int32_t v, uint32_t max_neighborhood,
                     uint32_t max_candidate_degree, int32_t* c, int32_t* d, uint8_t* active);
void ceo_cd_screen(const ceo_graph* g, int32_t u, int32_t v, const int32_t* c, const int32_t* d,
                   const uint8_t* active, int64_t count, int32_t mode, uint8_t* flags);
/* FinalizeCdCandidates (hamilton_tutte.cpp:283-327) and its Hamilton reply count (:230-269). */
int64_t ceo_ht_reply_count(const ceo_graph* g, int32_t tu, int32_t tv, int32_t center);
/* The Hamilton replies of `center` (AppendHtHamiltonRepliesUnchecked, hamilton_tutte.cpp:230-269)
 * as (center, first, second) triples in CSR pair order, and the end replies of a path end
 * (AppendHtEndRepliesUnchecked, :271-282) as (lower, higher) pairs in CSR order (-1: the internal
 * neighbour is not adjacent). Up to `capacity` records go to `out`; the return value is the count. */
int64_t ceo_ht_replies(const ceo_graph* g, int32_t tu, int32_t tv, int32_t center, int32_t* out, int64_t capacity);
int64_t ceo_ht_end_replies(const ceo_graph* g, int32_t endpoint, int32_t internal_neighbor, int32_t* out,
                           int64_t capacity);
int64_t ceo_cd_finalize(const ceo_graph* g, int32_t u, int32_t v, const int32_t* c, const int32_t* d,
                        const uint8_t* flags, int64_t count, uint32_t max_cd, int32_t* out_c, int32_t* out_d,
                        uint64_t* out_product);
/* HT scan target order (weight descending when order == 1, else canonical). */
int64_t ceo_ht_targets(const ceo_graph* g, int32_t order, int32_t* out);
/* The batched step (JV witnesses, HT targets, c,d neighbourhoods and flag words, optional
 * finalised candidates) of instances [first, last) of a disjoint union, in the batched
 * screen's output layout with global ids. */
int ceo_batch_expect(const ceo_graph* g, const int64_t* node_begin, const int64_t* edge_begin, int64_t first,
                     int64_t last, uint32_t targets, uint32_t max_neighborhood, uint32_t max_candidate_degree,
                     int32_t mode, uint32_t flag_words, uint32_t max_cd, int32_t* witness, int32_t* target_ids,
                     int32_t* target_count, int32_t* nbhd, uint32_t* flags, int32_t* cand_c, int32_t* cand_d,
                     int64_t* cand_product, int32_t* cand_count);

#ifdef __cplusplus
}
#endif
#endif
