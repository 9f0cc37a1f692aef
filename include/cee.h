/* cee.h -- C ABI of the B200 edge-elimination screen (libcee.so).
 *
 * Plain pointers and sizes only; no C++ or torch types cross this boundary. Each entry point
 * names the reference interface it replaces (paths inside the reference project). The C++
 * shim in cudaedgeelimination_b200/shim/cudaee_seam.cpp maps the reference's CUDA-backend
 * symbols onto these calls so that the reference's CPU code drives the B200 kernels.
 *
 * Conventions
 *   - Every int-returning function returns CEE_OK (0) or a negative CEE_ERR_* code (the serving
 *     loop's admission calls may also return CEE_BUSY, 1); the text
 *     of the last error is available from cee_last_error(ctx) (ctx may be NULL for errors
 *     raised before a context exists).
 *   - A cee_ctx belongs to one host thread and one device, owns a CUDA stream and all device
 *     buffers it allocates; calls on one ctx are serialised on its stream. Caller buffers are
 *     borrowed for the duration of the call only (error returns included), except a serving
 *     job's buffers, which stay borrowed until cee_serve_poll returns the job.
 *   - Host-buffer entry points copy inputs to the device, run, copy results back and
 *     synchronise before returning. Pinned host buffers are copied directly; pageable ones
 *     go through the CUDA driver's staging.
 *   - There is no CPU fallback: without a usable device the calls fail with CEE_ERR_NODEVICE.
 *   - Exact-arithmetic range: coordinates are stored as int32 offsets from the snapshot's
 *     bounding-box corner, so every snapshot must have max-min < 2^30 on both axes (every
 *     distance then fits int32 and every squared distance fits 2^61); edge weights must lie in
 *     [0, 2^31). Inputs outside this range fail with CEE_ERR_RANGE before any launch.
 */
#ifndef CEE_H
#define CEE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CEE_ABI_VERSION 1

enum cee_status {
  CEE_OK = 0,
  CEE_BUSY = 1,          /* serving loop: no slot or no HBM budget left now; poll, then retry */
  CEE_ERR_INVALID = -1,  /* malformed input (reference: std::invalid_argument / runtime_error) */
  CEE_ERR_RANGE = -2,    /* outside the exact-arithmetic range (reference: std::overflow_error) */
  CEE_ERR_CUDA = -3,     /* CUDA runtime or launch failure */
  CEE_ERR_NOMEM = -4,    /* device or pinned host allocation failed */
  CEE_ERR_NODEVICE = -5, /* no usable CUDA device */
  CEE_ERR_TIMEOUT = -6,  /* a bounded device-side wait ran out */
  CEE_ERR_STATE = -7     /* call out of order (e.g. launch before prepare) */
};

enum cee_distance_type { CEE_EUC_2D = 0, CEE_CEIL_2D = 1 };

/* HtCdMode, include/cuda_edge_elimination/hamilton_tutte.hpp:21-24 */
enum cee_cd_mode { CEE_CD_ACTIVE_INCOMPATIBLE = 0, CEE_CD_MISSING_OR_INCOMPATIBLE = 1 };

/* kInvalidKOptTemplateCost, include/cuda_edge_elimination/local_search.hpp:52 */
#define CEE_INVALID_KOPT_COST INT64_MAX

typedef struct cee_ctx cee_ctx;

/* ---- library / device ------------------------------------------------------------- */

int cee_abi_version(void);
/* Number of visible CUDA devices (0 when none; never fails for "no device"). */
int cee_device_count(int* count);
/* Picks the visible device with the most free memory, as the reference's SelectDevice does
 * when no device is forced (src/cuda/jv_cuda.cu:290-346). */
int cee_select_device(int* device);
/* Creates a context on `device` (-1: cee_select_device). */
int cee_create(int device, cee_ctx** out);
void cee_destroy(cee_ctx* ctx);
const char* cee_last_error(const cee_ctx* ctx);
int cee_ctx_device(const cee_ctx* ctx);
/* The cudaStream_t every launch of this context goes to. */
void* cee_ctx_stream(cee_ctx* ctx);
/* Streaming multiprocessors of the context's device (keys of autotuning caches). */
int cee_ctx_sm_count(const cee_ctx* ctx);
int cee_ctx_synchronize(cee_ctx* ctx);
/* Device bytes currently held by the context's caches and workspaces. */
uint64_t cee_ctx_resident_bytes(const cee_ctx* ctx);
/* Tuning options (defaults are the autotuned choices for B200; see cee_ctx_set_option). */
enum cee_option {
  CEE_OPT_JV_KERNEL = 1,    /* 0 = one thread per edge, 1 = one warp per edge (default) */
  CEE_OPT_JV_WAVES = 2,     /* grid of the thread-per-edge screen, in waves of resident blocks */
  CEE_OPT_KOPT_ROWS_K3 = 3, /* rows per k-opt tile for k = 3 / 4 / 5 (0 = default, even) */
  CEE_OPT_KOPT_ROWS_K4 = 4,
  CEE_OPT_KOPT_ROWS_K5 = 5,
  CEE_OPT_KOPT_KERNEL = 6   /* k-opt matrix kernel: 1 = one thread per row with the proper templates
                               compiled in, where it applies (default); 0 = the tiled kernel always */
};
/* Sets a launch-shape option of this context; results never depend on it. */
int cee_ctx_set_option(cee_ctx* ctx, int32_t option, int64_t value);
/* Frees cached device state: bit 1 = JV, bit 2 = k-opt, bit 4 = c,d, bit 8 = batch,
 * bit 16 = serving loop (stops it; its jobs are dropped), bit 32 = JV epoch loop workspace,
 * bit 64 = HT replies (ClearHtReplyCudaCache, hamilton_tutte.hpp:544-545).
 * Replaces ClearJvCudaCache (include/cuda_edge_elimination/elimination.hpp:338) and
 * ClearKOptCostCudaCache (include/cuda_edge_elimination/local_search.hpp:242). */
int cee_ctx_clear(cee_ctx* ctx, unsigned what);

/* ---- snapshot view ------------------------------------------------------------------ */

/* Host view of a GraphSnapshot (include/cuda_edge_elimination/graph.hpp:13-37): integer
 * coordinates, the stable edge list (edge ids are positions in it) and the active-only CSR
 * over it with rows ascending by neighbour (GraphSnapshot::RebuildCsr,
 * src/common/graph.cpp:230-282). */
typedef struct {
  int32_t n;
  int32_t dist_type;          /* cee_distance_type */
  const int64_t* x;           /* [n] */
  const int64_t* y;           /* [n] */
  int64_t m;
  const int32_t* edge_u;      /* [m] */
  const int32_t* edge_v;      /* [m] */
  const int64_t* edge_w;      /* [m] */
  const uint8_t* active;      /* [m] 0/1 */
  int64_t adjacency;          /* row_offsets[n] = 2 x active edges */
  const int32_t* row_offsets; /* [n + 1] */
  const int32_t* neighbors;   /* [adjacency] */
  const int32_t* csr_edge_ids;/* [adjacency] */
} cee_graph_view;

/* ---- exact distance ------------------------------------------------------------------ */

/* Span classes of a point set: the larger of its x and y spans (max - min) selects the device
 * routine for the exact distance (FP32 root, FP64 root or int64 residual; each followed by an
 * exact integer fix-up, so all three return the same integer). */
enum cee_span_class { CEE_SPAN_SMALL = 0 /* < 2^21 */, CEE_SPAN_NARROW = 1 /* < 2^26 */, CEE_SPAN_WIDE = 2 /* < 2^30 */ };

/* The reference's exact TSPLIB distance (src/common/distance.cpp:29-52: integer square root,
 * EUC_2D rounds to nearest, CEIL_2D rounds up) of `count` point pairs (pair_i[k], pair_j[k]) of
 * the point set (x, y), evaluated on the device by the routine every screen uses for that point
 * set, out[k] = the distance. *span_class (may be null) receives the cee_span_class used. A
 * checking aid for the distance routines. */
int cee_exact_distances(cee_ctx* ctx, int32_t n, const int64_t* x, const int64_t* y, int32_t dist_type,
                        int64_t count, const int32_t* pair_i, const int32_t* pair_j, int32_t* out,
                        int32_t* span_class);

/* The largest relative error of the device's one-instruction FP32 square-root estimate (the
 * estimate the CEE_SPAN_SMALL routine rounds and then corrects with an exact integer residual)
 * over every float in [1, 2^44), i.e. every FP32 sum of squares that class produces. The routine
 * is exact whenever this is below 2^-21.6; *max_relative_error receives it. A checking aid. */
int cee_sqrt_estimate_error(cee_ctx* ctx, double* max_relative_error);

/* ---- JV fast-elimination screen ------------------------------------------------------ */

/* JvCudaCacheUsage (include/cuda_edge_elimination/elimination.hpp:41-49) plus byte counts. */
typedef struct {
  int32_t static_hit;     /* coordinates, distance type and every edge (u, v, w) unchanged */
  int32_t workspace_hit;  /* no device buffer had to grow */
  uint64_t resident_bytes;
  double h2d_ms;          /* CUDA-event times on the context stream */
  double kernel_ms;
  double d2h_ms;
  int64_t h2d_bytes;
  int64_t d2h_bytes;
  int64_t edges_screened; /* active edges of the snapshot */
} cee_jv_stats;

/* Replaces FindJvCandidatesCuda (include/cuda_edge_elimination/elimination.hpp:335-337,
 * src/cuda/jv_cuda.cu:488-566). witness_out[e] = the first JV witness of edge e in the
 * reference's candidate order (src/cpu/jv_elimination.cpp:45-117, 209-224) or -1; the
 * candidate list is the edges with witness >= 0 in ascending edge id. Static data are
 * cached per context with the reference's exact element-wise key (src/cuda/jv_cuda.cu:360-430);
 * active bits and the CSR are uploaded on every call. */
int cee_jv_screen(cee_ctx* ctx, const cee_graph_view* graph, int32_t* witness_out,
                  cee_jv_stats* stats);
/* cee_jv_screen with hints (no counterpart in the reference). CEE_JV_STATIC_UNCHANGED: the caller
 * vouches that x, y, edge_u, edge_v and edge_w hold the values of this context's previous JV call,
 * as a binding that keeps its own copy and compares it element-wise (the reference's resident-cache
 * key) knows; the cached static data are then reused without comparing them again. The node and
 * edge counts and the distance type are still compared, and the hint does nothing once the cache
 * was cleared. Other flag bits: CEE_ERR_INVALID. */
#define CEE_JV_STATIC_UNCHANGED 1u
int cee_jv_screen_ex(cee_ctx* ctx, const cee_graph_view* graph, int32_t* witness_out,
                     cee_jv_stats* stats, uint32_t flags);
/* The three phases of cee_jv_screen, for callers that keep the snapshot resident and time
 * the kernel alone: prepare uploads (and waits for the copies), launch enqueues the screen on
 * the context stream (no synchronisation), fetch copies the witnesses back and checks the
 * device error word. */
int cee_jv_prepare(cee_ctx* ctx, const cee_graph_view* graph, cee_jv_stats* stats);
int cee_jv_launch(cee_ctx* ctx);
int cee_jv_fetch(cee_ctx* ctx, int32_t* witness_out);

/* A snapshot already resident in the caller's device memory, in this library's device layout:
 * coordinates as int32 (x, y) pairs in [0, 2^30) (offsets from a common corner), the stable
 * edge list as int32 (u, v) pairs plus int32 weights in [0, 2^31) and 0/1 active bytes, and
 * the active-only CSR (rows ascending by neighbour). All pointers are device pointers;
 * xy and edge_uv must be 8-byte aligned. */
typedef struct {
  int32_t n;
  int32_t dist_type;
  int64_t m;
  int64_t adjacency;
  const int32_t* xy;           /* [2n] */
  const int32_t* edge_uv;      /* [2m] */
  const int32_t* edge_w;       /* [m] */
  const uint8_t* active;       /* [m] */
  const int32_t* row_offsets;  /* [n + 1] */
  const int32_t* neighbors;    /* [adjacency] */
  const int32_t* csr_edge_ids; /* [adjacency] */
} cee_device_graph;

/* JV screen that allocates nothing. No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc -- hosts whose own pool or arena owns all device memory and
 * forbids library allocations, and paths that must not allocate while they run (latency-
 * critical loops that reserved their memory up front, processes under a hard device-memory
 * quota). The caller passes its snapshot and the witness output (int32 [m], same meaning as
 * cee_jv_screen's witness_out) in device memory and a cudaStream_t (NULL = legacy default
 * stream); the call runs on the calling thread's current device and returns after the
 * stream has finished the screen. It calls no cudaMalloc, cudaFree or other allocating
 * routine: its working memory (the per-slot edge weights and a status word) lives in
 * file-scope device arrays of fixed size that every GPU loading the library holds until the
 * process exits (16 MiB + 256 B). Limit: adjacency <= 4,194,304 CSR slots; larger snapshots
 * fail with CEE_ERR_RANGE before any launch. The first call on a device looks up the arrays'
 * device addresses (once per device), so make it before any stream capture. All calls share
 * the arrays: each call rewrites what it reads, but calls that overlap on the GPU race and must
 * be serialised by the caller. The snapshot is validated on the device first (CEE_ERR_INVALID
 * on failure); errors are reported through cee_last_error(NULL). */
int cee_jv_screen_noalloc(const cee_device_graph* graph, int32_t* witness_out, void* stream);

/* ---- JV elimination to a fixed point, device resident ------------------------------------ */

typedef struct {
  int32_t epochs;          /* epochs run (the last one commits nothing unless max_rounds stopped it) */
  int64_t committed;       /* edges eliminated in total */
  double total_ms;         /* wall time of the call */
  uint64_t resident_bytes; /* device workspace of the epoch loop */
} cee_jv_elim_stats;

/* RunJvElimination's epoch loop (src/cpu/jv_elimination.cpp:250-322) without the host in the
 * loop: screen, commit gate (CommitVerifiedCandidates, src/cpu/elimination_commit.cpp:13-76) and CSR
 * rebuild (GraphSnapshot::RebuildCsr, src/common/graph.cpp:230-282) all on the device, until an
 * epoch commits nothing or max_rounds epochs ran. Edges must be unique canonical pairs (u < v), as
 * the reference's edge files are. Outputs per edge: active_out (final flag), epoch_out (epoch that
 * eliminated it or -1), witness_out (its witness or -1); per epoch (capacity max_rounds): active
 * edges before the epoch and edges committed. The reference's CPU re-verification and proof log
 * stay with the caller (the outputs give every record: epoch, edge, witness). */
int cee_jv_eliminate(cee_ctx* ctx, const cee_graph_view* graph, uint32_t max_rounds, uint8_t* active_out,
                     int32_t* witness_out, int32_t* epoch_out, int64_t* epoch_edges_before,
                     int64_t* epoch_committed, cee_jv_elim_stats* stats);

/* Per-epoch figures of the context's last cee_jv_eliminate call, for the proof log's metrics lines
 * (EpochMetrics, include/cuda_edge_elimination/elimination.hpp:21-39): proposed[e] = candidates the
 * epoch's screen found, screen_ms[e] = device time of its screen and commit gate (CUDA events).
 * capacity >= the call's epoch count; CEE_ERR_STATE before any call. */
int cee_jv_eliminate_metrics(const cee_ctx* ctx, int64_t* proposed, double* screen_ms, int32_t capacity);

/* ---- JV proof log --------------------------------------------------------------------------- */

/* ProofRecord (include/cuda_edge_elimination/types.hpp:40-50) of a JV elimination. */
typedef struct {
  uint32_t epoch;
  int32_t edge_id;
  int32_t u;
  int32_t v;
  int32_t witness;
  int32_t reserved;
  uint64_t snapshot_hash; /* content hash of the snapshot the epoch screened */
} cee_jv_proof_record;

/* EpochMetrics' serialised fields (the proof's "metrics" lines). */
typedef struct {
  uint32_t epoch;
  uint32_t reserved;
  int64_t edges_before;
  int64_t proposed;
  int64_t verified;
  int64_t rejected;
  int64_t committed;
  double propose_ms;
  double verify_ms;
} cee_jv_epoch_metrics;

/* GraphSnapshot::ContentHash (src/common/graph.cpp:323-346) of an integer-coordinate snapshot:
 * 64-bit FNV-1a over its dimension (int32), distance type (uint8), integer-coordinate flag (1), every
 * point's (x, y) (int64 each) and every edge's (u, v, weight, active) (int32, int32, int64, bool), in
 * the snapshot's edge order. Host computation; needs no context or device. */
int cee_content_hash(const cee_graph_view* graph, uint64_t* hash);

/* The proof records of a device elimination, from cee_jv_eliminate's per-edge epoch_out and
 * witness_out (graph = the snapshot the elimination started from): the records RunJvElimination
 * appends (src/cpu/jv_elimination.cpp:304-312), epoch by epoch, each epoch in commit order
 * (src/cpu/elimination_commit.cpp:33-41: (u, v), then edge id), each carrying the content hash of the
 * snapshot its epoch screened. hashes[0..epochs] (may be null) receives the hash before every epoch
 * and, last, the final hash (hashes[0] is the proof's initial_hash, hashes[epochs] its final_hash);
 * `epochs` = cee_jv_elim_stats.epochs. The epochs' hashes are computed on parallel host threads.
 * *count = the number of records (at most capacity are written). CEE_ERR_INVALID when an eliminated
 * edge was not active, its epoch is outside [0, epochs) or its witness is not a node. */
int cee_jv_proof(const cee_graph_view* graph, uint32_t epochs, const int32_t* edge_epoch, const int32_t* witness,
                 cee_jv_proof_record* records, int64_t capacity, int64_t* count, uint64_t* hashes);

/* Writes the snapshot's active edges in GraphSnapshot::WriteActiveEdges' format (src/common/graph.cpp:284-298,
 * the Concorde .edg file): "n count", then "u v weight" per active edge in edge order. active = the
 * flags to write (e.g. cee_jv_eliminate's active_out), or null for graph->active. */
int cee_write_active_edges(const char* path, const cee_graph_view* graph, const uint8_t* active);

/* Writes a CUDAEE_PROOF_V1 file in WriteProof's format (src/cpu/jv_elimination.cpp:324-368): backend,
 * initial_hash, the records, one metrics line per epoch, final_hash, END. The reference's ReadProof
 * and ReplayProof accept it. */
int cee_jv_write_proof(const char* path, const char* backend, uint64_t initial_hash, uint64_t final_hash,
                       const cee_jv_proof_record* records, int64_t count, const cee_jv_epoch_metrics* metrics,
                       int32_t epochs);

/* ---- k-opt leaf cost matrix ----------------------------------------------------------- */

/* KOptCostTask, include/cuda_edge_elimination/local_search.hpp:54-57 (48 bytes). */
typedef struct {
  int32_t port_nodes[10];
  int64_t deleted_cost;
} cee_kopt_task;

/* KOptCudaCacheUsage (include/cuda_edge_elimination/local_search.hpp:59-64) plus timings. */
typedef struct {
  int32_t snapshot_hit;
  int32_t template_hit;
  int32_t workspace_hit;
  uint64_t resident_bytes;
  double h2d_ms;
  double kernel_ms;
  double d2h_ms;
  int64_t h2d_bytes;
  int64_t d2h_bytes;
} cee_kopt_stats;

/* The proper k-opt reconnect templates (BuildKOptReconnectTable,
 * src/cpu/kopt_search.cpp:1143-1193): writes mates[t * 14 + p] for t < count (14 bytes per
 * template, unused entries 0xff) and the generator hash pinned in
 * configs/kopt_reconnect_hashes_v1.txt. Returns the template count (4 / 25 / 208) or < 0. */
int cee_kopt_templates(uint32_t k, uint8_t* mates, uint64_t* generator_hash);

/* Replaces EvaluateKOptTemplateCostsCuda (include/cuda_edge_elimination/local_search.hpp:
 * 237-240, src/cuda/kopt_cost.cu:415-470). costs_out[row * template_count + t] is the exact
 * added cost of template t on the row, or CEE_INVALID_KOPT_COST. Templates are the caller's
 * (mates as above); the cache hits follow the reference (coordinates + type; k + hash +
 * template bytes; workspace capacities). */
int cee_kopt_costs(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x,
                   const int64_t* y, uint32_t k, const uint8_t* mates, int32_t template_count,
                   uint64_t template_hash, const cee_kopt_task* tasks, int64_t rows,
                   int64_t* costs_out, cee_kopt_stats* stats);

/* Several k buckets (each with the library's own proper templates) in one launch: segment s
 * has k = ks[s], rows[s] rows at tasks[s] and writes costs_out[s]. At most 8 segments. */
int cee_kopt_costs_multi(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x,
                         const int64_t* y, int32_t segments, const uint32_t* ks,
                         const cee_kopt_task* const* tasks, const int64_t* rows,
                         int64_t* const* costs_out, cee_kopt_stats* stats);
/* Fused leaf consume: for every row the set of templates whose added cost is below the row's
 * deleted_cost — the templates the reference's leaf consumer tries, in order
 * (src/cpu/kopt_search.cpp:694-715) — as a bit mask of ceil(T/32) uint32 words per row (bit t of word
 * t / 32 = template t, the library's proper templates) and the first such template (-1 if none).
 * costs_out may be NULL (or hold NULL segments): the full matrix is then not written, and only the
 * masks cross PCIe. */
int cee_kopt_improving_multi(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x,
                             const int64_t* y, int32_t segments, const uint32_t* ks,
                             const cee_kopt_task* const* tasks, const int64_t* rows,
                             uint32_t* const* masks_out, int32_t* const* first_out,
                             int64_t* const* costs_out, cee_kopt_stats* stats);
/* Phases of cee_kopt_costs_multi (prepare = upload and wait for it, launch = enqueue, fetch = copy back). */
int cee_kopt_prepare_multi(cee_ctx* ctx, int32_t n, int32_t dist_type, const int64_t* x,
                           const int64_t* y, int32_t segments, const uint32_t* ks,
                           const cee_kopt_task* const* tasks, const int64_t* rows,
                           cee_kopt_stats* stats);
int cee_kopt_launch(cee_ctx* ctx);
int cee_kopt_fetch(cee_ctx* ctx, int64_t* const* costs_out);
/* No counterpart in the reference: the launch shape of the k-opt matrix kernels of this context
 * (the same choices as CEE_OPT_KOPT_KERNEL and CEE_OPT_KOPT_ROWS_K3..K5; results never depend on
 * it). */
typedef struct {
  int32_t kernel;           /* 1 = one thread per row with the proper templates (where it applies), 0 = tiled */
  int32_t rows_per_tile[3]; /* tiled kernel: rows per tile for k = 3, 4, 5 (0 = default) */
  float ms;                 /* cee_kopt_autotune: the chosen shape's launch time */
} cee_kopt_tuning;
int cee_kopt_set_tuning(cee_ctx* ctx, const cee_kopt_tuning* tuning);
int cee_kopt_get_tuning(const cee_ctx* ctx, cee_kopt_tuning* tuning);
/* Times every candidate shape (the row kernel; the tiled kernel with half, default and double
 * tiles) on the prepared k-opt launch, `reps` launches each (CUDA events), keeps the fastest and
 * writes it to *chosen. */
int cee_kopt_autotune(cee_ctx* ctx, int32_t reps, cee_kopt_tuning* chosen);

/* ---- HT c,d root screen --------------------------------------------------------------- */

/* HtCdScreenTask, include/cuda_edge_elimination/hamilton_tutte.hpp:42-46 (12 bytes). */
typedef struct {
  int32_t c;
  int32_t d;
  uint8_t active;
  uint8_t reserved[3];
} cee_cd_task;

/* Replaces ScreenHtCdCandidatesCuda (include/cuda_edge_elimination/hamilton_tutte.hpp:528-531,
 * src/cuda/ht_cd.cu:384-442): flags_out[i] in {0,1} for target (u,v), u < v. Tasks are
 * validated as the reference does (c < d, no target endpoint, active bit equal to the CSR). */
int cee_cd_screen(cee_ctx* ctx, const cee_graph_view* graph, int32_t u, int32_t v,
                  const cee_cd_task* tasks, int64_t count, int32_t mode, uint8_t* flags_out);

/* ---- HT Hamilton and end replies -------------------------------------------------------- */

/* HtNeighborPair (include/cuda_edge_elimination/hamilton_tutte.hpp:26-32) and HtEndReplyTask
 * (:76-81); an end reply is a NodeEdge (local_search.hpp:17-22) with u < v. */
typedef struct {
  int32_t center;
  int32_t first;
  int32_t second;
} cee_ht_pair;
typedef struct {
  int32_t endpoint;
  int32_t internal_neighbor;
} cee_ht_end_task;
typedef struct {
  int32_t u;
  int32_t v;
} cee_node_edge;

/* HtReplyCudaCacheUsage (hamilton_tutte.hpp:515-519). */
typedef struct {
  int32_t graph_hit;     /* coordinates and CSR equal the previous reply call's: not uploaded */
  int32_t workspace_hit; /* no device buffer had to grow */
  uint64_t resident_bytes;
} cee_ht_reply_stats;

/* Replaces detail::EvaluateHtHamiltonRepliesCuda (include/cuda_edge_elimination/hamilton_tutte.hpp:
 * 533-537, src/cuda/ht_replies.cu:585-663): for target (u, v), u < v, an active edge, and each of
 * `count` centers (in [0, n), not u or v), the Hamilton replies of AppendHtHamiltonRepliesUnchecked
 * (src/cpu/hamilton_tutte.cpp:230-269) in its order. offsets_out[count + 1]: center i's replies are
 * [offsets_out[i], offsets_out[i + 1]) of the list that cee_ht_replies_fetch copies out (kept on the
 * device until the next reply call). The snapshot is validated as the reference does
 * (src/cuda/ht_replies.cu:521-566: CSR rows strictly ascending, symmetric, the active edges only,
 * at least 4 nodes): CEE_ERR_INVALID otherwise. stats may be null. */
int cee_ht_replies(cee_ctx* ctx, const cee_graph_view* graph, int32_t u, int32_t v, const int32_t* centers,
                   int64_t count, uint64_t* offsets_out, cee_ht_reply_stats* stats);
/* Replaces detail::EvaluateHtEndRepliesCuda (hamilton_tutte.hpp:539-542, src/cuda/ht_replies.cu:
 * 667-751): for each task, the edges at its endpoint other than the one to its internal neighbour
 * (AppendHtEndRepliesUnchecked, src/cpu/hamilton_tutte.cpp:271-282), as (lower, higher) node pairs in
 * CSR order; every task's edge must be active (CEE_ERR_INVALID otherwise). Offsets and fetch as above. */
int cee_ht_end_replies(cee_ctx* ctx, const cee_graph_view* graph, const cee_ht_end_task* tasks, int64_t count,
                       uint64_t* offsets_out, cee_ht_reply_stats* stats);
/* Copies the last reply call's list: offsets_out[count] records of cee_ht_pair (cee_ht_replies) or
 * cee_node_edge (cee_ht_end_replies). */
int cee_ht_replies_fetch(cee_ctx* ctx, void* replies_out);

/* ---- batched screen (many instances, one persistent graph-captured launch) ---------------- */

/* Many snapshots packed into one: instance i owns nodes [node_begin[i], node_begin[i+1]) and
 * edges [edge_begin[i], edge_begin[i+1]) of `graph`, which uses global node and edge ids; every
 * edge joins two nodes of its own instance and each instance's edges are sorted by (u, v) (the
 * order GraphSnapshot::Load produces, src/common/graph.cpp:223-226). */
typedef struct {
  int32_t instances;
  const int64_t* node_begin; /* [instances + 1] */
  const int64_t* edge_begin; /* [instances + 1] */
  cee_graph_view graph;
} cee_batch_view;

/* What the batch computes per instance: the JV screen of every active edge, and the HT c,d root
 * screen of the first `targets` edges of SelectHtTargetEdgeIds(kWeightDescending)
 * (src/cpu/ht_scan.cpp:316-345) with HtShallowOptions' neighbourhood / degree cap / mode
 * (include/cuda_edge_elimination/hamilton_tutte.hpp:95-108; defaults 64, 25, 50, active-incompatible). */
typedef struct {
  int32_t targets;              /* 1..64 */
  int32_t max_neighborhood;     /* 2..32 */
  int32_t max_candidate_degree; /* 0 = no cap */
  int32_t cd_mode;              /* cee_cd_mode */
  int32_t max_cd_candidates;    /* 0: flags only; 1..32: also FinalizeCdCandidates' ranked list
                                   (hamilton_tutte.cpp:283-327, reference default 5), read with
                                   cee_batch_fetch_candidates; needs instances of <= 65536 nodes */
} cee_batch_options;

/* Launch shape of the batch kernel (chosen by cee_batch_autotune; results never depend on it). */
typedef struct {
  int32_t jv_tile;         /* edges per JV work item */
  int32_t blocks_per_sm;   /* resident 256-thread blocks per SM (<= occupancy) */
  int32_t chunks;          /* instance chunks of the end-to-end call (copy/compute overlap) */
} cee_batch_tuning;

typedef struct {
  int64_t nodes, edges, adjacency, targets;
  int64_t pairs;            /* c,d pairs screened (sum over targets of s (s - 1) / 2) */
  int64_t flag_words;       /* per target */
  uint64_t resident_bytes;
  int64_t h2d_bytes, d2h_bytes;
  double h2d_ms, kernel_ms, d2h_ms, total_ms;
} cee_batch_stats;

/* Uploads the batch, plans the work items and captures the launch as a CUDA graph. */
int cee_batch_prepare(cee_ctx* ctx, const cee_batch_view* batch, const cee_batch_options* options,
                      cee_batch_stats* stats);
/* One graph launch of the persistent kernel over the prepared batch (no synchronisation). */
int cee_batch_launch(cee_ctx* ctx);
/* The same work as one synchronous launch per instance (the unbatched comparison path). */
int cee_batch_launch_plain(cee_ctx* ctx);
/* Copies the results back: witness[m] (as cee_jv_screen), target_ids[I * T] (global edge ids,
 * -1 padding) and target_count[I], nbhd[I * T * max_neighborhood] (global node ids, -1 padding;
 * the c,d task list of a target is every pair i < j of its neighbourhood as (min, max), in the
 * order of BuildCdScreenTasks, src/cpu/hamilton_tutte.cpp:204-214) and flags[I * T * flag_words]
 * (bit p of the target's words = ScreenCdTasksCpu flag of task p). Any pointer may be NULL. */
int cee_batch_fetch(cee_ctx* ctx, int32_t* witness, int32_t* target_ids, int32_t* target_count,
                    int32_t* nbhd, uint32_t* flags);
/* End to end from host buffers: uploads, screens and downloads chunk by chunk, overlapping the
 * copies of one chunk with the screen of another (pinned buffers overlap; pageable ones too,
 * at the driver's staging speed). The edge list must be canonical (u < v) and sorted by (u, v),
 * CEE_ERR_INVALID otherwise; edge_u itself is not copied (host threads turn it into per-node edge
 * starts). Output pointers as in cee_batch_fetch. */
int cee_batch_screen(cee_ctx* ctx, const cee_batch_view* batch, const cee_batch_options* options,
                     int32_t* witness, int32_t* target_ids, int32_t* target_count, int32_t* nbhd,
                     uint32_t* flags, cee_batch_stats* stats);
/* The finalised c,d candidates of the last launch (max_cd_candidates > 0): per (instance, target)
 * slot, `count` entries of (c, d, reply product) ranked by (product, c, d), global node ids;
 * arrays of instances x targets x max_cd_candidates (products saturate at 2^32 - 2; a product that
 * reaches it fails the launch with CEE_ERR_RANGE). */
int cee_batch_fetch_candidates(cee_ctx* ctx, int32_t* c, int32_t* d, int64_t* product, int32_t* count);
int cee_batch_set_tuning(cee_ctx* ctx, const cee_batch_tuning* tuning);
int cee_batch_get_tuning(const cee_ctx* ctx, cee_batch_tuning* tuning);
/* Times every candidate launch shape on the prepared batch (`reps` graph launches each, CUDA
 * events) and keeps the fastest; writes it to *chosen. */
int cee_batch_autotune(cee_ctx* ctx, int32_t reps, cee_batch_tuning* chosen);

/* ---- serving loop (device-resident snapshots, continuous batching) ----------------------- */
/* No counterpart in the reference: a request loop for callers that screen many snapshots as
 * they arrive. One persistent kernel runs every admitted job; a job's result is the same as
 * cee_jv_screen's (witness per edge) or cee_kopt_costs_multi's (the library's proper templates)
 * on the same snapshot, whatever else runs beside it. */
typedef struct {
  uint64_t hbm_budget_bytes; /* device arena for snapshots, k-opt rows and results */
  int32_t slots;             /* jobs in flight at most (1..256) */
  int32_t blocks_per_sm;     /* persistent kernel blocks per SM (0 = occupancy limit) */
  int32_t idle_ms;           /* the kernel leaves after about this long without work */
} cee_serve_config;

typedef struct {
  int32_t job;
  int32_t status;
  uint64_t tag;
} cee_serve_event;

int cee_serve_start(cee_ctx* ctx, const cee_serve_config* config);
/* Uploads a snapshot into the arena (validated on the host; ids as for cee_jv_screen).
 * CEE_BUSY when the arena has no room now. */
int cee_serve_add_snapshot(cee_ctx* ctx, const cee_graph_view* graph, int32_t* snapshot);
/* The snapshot's memory returns to the arena once its last job has completed. */
int cee_serve_release_snapshot(cee_ctx* ctx, int32_t snapshot);
/* Screens every edge of the snapshot; witness_out (m entries) is written before the job's
 * completion event is returned by cee_serve_poll. A witness_out that lies in one page-locked host
 * allocation (cudaHostAlloc, a pinned torch tensor), 4-byte aligned, is written by the kernel in
 * place as the job runs (no arena room, no copy); other buffers get a copy when the job ends.
 * CEE_BUSY: no slot or arena room now. */
int cee_serve_submit_jv(cee_ctx* ctx, int32_t snapshot, int32_t* witness_out, uint64_t tag,
                        int32_t* job);
/* k-opt leaf costs of 1..3 segments (k = ks[s], rows[s] rows at tasks[s], output costs_out[s],
 * rows x template_count(k) cells) on the snapshot's coordinates. The task rows go up by a copy
 * queued at submission: pageable rows are staged before the call returns, pinned ones are read
 * while the job runs, so keep them unchanged until cee_serve_poll returns the job. The rows are
 * not read on the host: a port node outside [0, n) is found by the device's bounds checks, and
 * the job then completes with status CEE_ERR_INVALID (other jobs are unaffected).
 * CEE_BUSY: no slot or arena room now. */
int cee_serve_submit_kopt(cee_ctx* ctx, int32_t snapshot, int32_t segments, const uint32_t* ks,
                          const cee_kopt_task* const* tasks, const int64_t* rows,
                          int64_t* const* costs_out, uint64_t tag, int32_t* job);
/* The same job producing cee_kopt_improving_multi's outputs: per segment the improving-template
 * masks (rows x ceil(template_count / 32) words, bit t = template t's cost is below the row's
 * deleted cost) and the first improving template per row (-1: none); costs_out may be null (no
 * cost matrix). */
int cee_serve_submit_kopt_improving(cee_ctx* ctx, int32_t snapshot, int32_t segments, const uint32_t* ks,
                                    const cee_kopt_task* const* tasks, const int64_t* rows,
                                    uint32_t* const* masks_out, int32_t* const* first_out,
                                    int64_t* const* costs_out, uint64_t tag, int32_t* job);
/* Returns up to `capacity` completed jobs (their host outputs are written) and relaunches the
 * kernel if it went idle while jobs wait. A job's downloads are issued by the loop's own host
 * thread as soon as the job ends, whether or not the caller is polling. */
int cee_serve_poll(cee_ctx* ctx, cee_serve_event* events, int32_t capacity, int32_t* count);
/* Jobs admitted and not yet returned by cee_serve_poll, and arena bytes in use. */
int cee_serve_pending(const cee_ctx* ctx, int32_t* jobs, uint64_t* arena_used);
/* Totals since cee_serve_start. */
typedef struct {
  uint64_t jobs;           /* jobs posted to the kernel */
  uint64_t rows_bytes;     /* k-opt rows copied to the device */
  uint64_t download_bytes; /* results copied back to the host */
  uint64_t direct_bytes;   /* results the kernel wrote straight into page-locked host memory */
} cee_serve_stats;
int cee_serve_get_stats(const cee_ctx* ctx, cee_serve_stats* stats);
/* Stops the kernel and frees the arena. Outstanding jobs are dropped; a dropped job's downloads
 * (results complete or not) may still write its output buffers until this call returns. */
int cee_serve_stop(cee_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* CEE_H */
