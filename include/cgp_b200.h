/*
 * cgp_b200 -- C ABI of the B200 multi-query traversal library.
 *
 * Many BFS, SSSP, k-hop BFS and WCC queries run over one CSR graph at once;
 * every vertex carries a query bitmask (64 queries per 64-bit word, up to 16
 * words = 1024 queries per traversal group), so one pass over an adjacency
 * list serves every query active at that vertex.
 *
 * All entry points return a cgp_status (0 = OK).  On failure the message is
 * kept per thread and can be read with cgp_last_error().  No C++ exception
 * crosses this boundary.  Pointers are plain host or device addresses; no
 * framework types appear in any signature.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project root).
 */
#ifndef CGP_B200_H
#define CGP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------- constants --- */

typedef int32_t cgp_status;
#define CGP_OK 0
#define CGP_ERR_INVALID_ARG 1 /* std::invalid_argument in the reference      */
#define CGP_ERR_OOM 2         /* device or host allocation failed            */
#define CGP_ERR_CUDA 3        /* std::runtime_error from throw_if_cuda_error */
#define CGP_ERR_TIMEOUT 4     /* a bounded wait gave up                      */
#define CGP_ERR_CANCELLED 5   /* request cancelled before completion         */
#define CGP_ERR_NOT_FOUND 6   /* unknown ticket                              */
#define CGP_ERR_BUSY 7        /* resource in use (e.g. server queue full)    */
#define CGP_ERR_DEVICE 8      /* a kernel reported an internal error flag    */

/* query kinds: algorithms::algo_kind_t (puercgp/include/puercgp/algorithms/hybrid.hxx:27-33) */
#define CGP_KIND_BFS 0
#define CGP_KIND_SSSP 1
#define CGP_KIND_WCC 2
#define CGP_KIND_KHOP 3 /* BFS bounded to depth k (new)                         */

/* traversal_mode_t (puercgp/include/puercgp/core/types.hxx:12) */
#define CGP_MODE_PUSH 0
#define CGP_MODE_PULL 1
#define CGP_MODE_HYBRID 2

/* edge weights */
#define CGP_WEIGHT_NONE 0 /* every weight is 1 (csr_graph.hxx:37-39)        */
#define CGP_WEIGHT_U32 1
#define CGP_WEIGHT_F32 2

/* output layouts */
#define CGP_LAYOUT_VERTEX_MAJOR 0 /* out[v*nq + q]: puercgp values (frontier_engine.hxx:90-95) */
#define CGP_LAYOUT_QUERY_MAJOR 1  /* out[q*V + v]: cgp distances (cgp_bfs.hxx:561), replenish final buffer */

/* depth bookkeeping for BFS bits */
#define CGP_DEPTH_AUTO 0
#define CGP_DEPTH_PLANES 1 /* bit-sliced depth planes, one output pass at the end */
#define CGP_DEPTH_DIRECT 2 /* depth written at discovery time                    */

/* graph flags */
#define CGP_GRAPH_DEVICE_POINTERS 1 /* inputs are device pointers (copied)      */
#define CGP_GRAPH_SYMMETRIC 2       /* caller asserts the CSR is symmetric      */
#define CGP_GRAPH_OFFSETS64 4       /* keep 64-bit row offsets on the device    */

/* unreached markers */
#define CGP_BFS_UNREACHED INT32_MAX /* cpu_bfs INT_MAX (mtx_loader.hxx:270)      */
#define CGP_U32_UNREACHED UINT32_MAX
/* f32 SSSP uses +inf (mtx_loader.hxx:293) */

/* ----------------------------------------------------------------- types --- */

typedef struct cgp_graph cgp_graph;
typedef struct cgp_enactor cgp_enactor;
typedef struct cgp_server cgp_server;

/* query_descriptor_t (puercgp/include/puercgp/core/query_descriptor.hxx:19-24);
 * `k` is the hop bound of CGP_KIND_KHOP.  WCC ignores `source`. */
typedef struct {
  int32_t source;
  int32_t kind;
  int32_t k;
  int32_t reserved;
} cgp_query;

/* run_options (puercgp/include/puercgp/core/types.hxx:26-46) plus the B200
 * execution knobs.  Fill with cgp_options_init() first. */
typedef struct {
  int32_t traversal_mode;     /* CGP_MODE_*, default HYBRID                      */
  int32_t push_strategy;      /* accepted for compatibility; mapping is tuned    */
  int32_t pull_strategy;      /* accepted for compatibility                      */
  int32_t max_iterations;     /* 0 = run to convergence                          */
  double pull_frontier_ratio; /* pull when frontier vertices >= ratio * V        */
  double pull_edge_ratio;     /* pull when frontier edges >= ratio * E           */
  int32_t profile_iterations; /* record per-level profiles                       */
  int32_t use_cuda_graph;     /* replay captured level chunks (default 1)        */
  int32_t levels_per_sync;    /* levels enqueued between host checks; 0 = auto   */
  int32_t mask_words;         /* 64-bit words per vertex mask; 0 = auto          */
  int32_t depth_mode;         /* CGP_DEPTH_*                                     */
  int32_t heavy_degree;       /* degree above which a vertex is split across CTAs; 0 = auto */
  int32_t max_queries;        /* run_options::max_queries; 0 = unlimited         */
  int32_t discard_results;    /* run_options::discard_results                    */
  int32_t profile_kernels;    /* time kernel classes with CUDA events (slower; no graphs) */
  int32_t dense_unroll;       /* edges per step of the dense SSSP kernel: 1 or 2; 0 = 1 */
  double sssp_pull_edge_ratio; /* SSSP levels gather (pull) when frontier edges >= ratio * E;
                                  <= 0: always scatter (push)                              */
  int32_t light_chunks;       /* SSSP gathers take light vertices in CTA chunks (wider groups
                                 in 256-slot slices): 0 = on, -1 = one warp per vertex     */
  int32_t level_loop;         /* CGP_LOOP_*: how a traversal to convergence is driven     */
  int32_t sssp_chunk_direction; /* SSSP gather/scatter decided per 32-slot chunk from the
                                   chunk's own frontier (1), or for the whole group (-1);
                                   0 = auto: per chunk in the serving loop, whole group in
                                   batch runs                                              */
  int32_t bfs_pull_form;      /* light-vertex BFS pull: 0 = a lane per vertex, vertex order;
                                 1 = CTA chunks on pull levels that read most in-edges
                                 (measured slower on R-MAT: kept as an option); 2 = a lane
                                 per vertex, vertices in decreasing in-degree order          */
  int32_t serve_admission;    /* serving loop: 0 = any free slot, preferring the chunk of the
                                 latest admissions; 1 = whole 32-slot cohorts: requests enter
                                 only chunks whose slots are all free; 2 = group cohorts:
                                 requests enter only an empty group, all pending at once     */
  int32_t serve_groups;       /* serving loop: traversal groups the slots are split into, each
                                 with its own masks and stream, their levels overlapping on
                                 the device (1..8); 0 = 1                                    */
  double sssp_pull_pair_ratio; /* a group's SSSP level also needs the next frontier's
                                  estimated (edge, slot) pairs (last level's improvements x
                                  the next frontier's mean out-degree) to reach ratio x E x
                                  the group's SSSP 32-slot chunks to gather: a scatter costs
                                  per pair, a gather per (in-edge, chunk); default 0.5;
                                  <= 0: edges alone decide                               */
  void* stream;               /* cudaStream_t; NULL = the library's own stream   */
} cgp_options;

/* level_loop values.  CHUNKS: CUDA graphs of levels_per_sync levels, the host
 * reads the control block once per chunk (one chunk in flight).  DEVICE: one
 * CUDA graph whose WHILE conditional node runs a level per iteration until
 * the device-side done flag is set: the host waits once per traversal (it
 * replaces the reference's per-level host synchronisation,
 * frontier_engine.hxx:3044-3071).  AUTO is CHUNKS: kernels inside a graph
 * with conditional nodes are invisible to kernel profilers, so the device
 * loop is asked for explicitly. */
#define CGP_LOOP_AUTO 0
#define CGP_LOOP_CHUNKS 1
#define CGP_LOOP_DEVICE 2

/* Per-level record: iteration_profile_t (puercgp/include/puercgp/core/result.hxx:21-46). */
typedef struct {
  int32_t iteration;
  int32_t mode;              /* 0 push, 1 pull                                    */
  uint64_t frontier_size;    /* unique frontier vertices entering the level       */
  uint64_t frontier_edges;   /* sum of their out-degrees                          */
  uint64_t next_size;        /* unique vertices of the next frontier              */
  uint64_t query_convergence_mask; /* bit q set: slot q wrote the next frontier (first 64 slots) */
  uint64_t new_pairs;        /* (query, vertex) pairs first reached (BFS bits)       */
  uint64_t pull_vertices;    /* vertices a pull level scanned                        */
  uint64_t pull_edges;       /* in-edges read before early exit                      */
  uint64_t sssp_pairs;       /* (edge, active query) relaxations attempted           */
  uint64_t sssp_active;      /* active SSSP bits summed over frontier vertices       */
  uint64_t improved;         /* SSSP (query, vertex) improvements                    */
  uint64_t sssp_pull_vertices; /* vertices an SSSP gather level scanned                 */
  uint64_t sssp_pull_edges;  /* in-edges an SSSP gather level scanned                    */
  int32_t sssp_mode;         /* SSSP direction of the level: 0 push (scatter), 1 pull (gather) */
  float kernel_ms;           /* the level's kernel time when profile_kernels is set, else 0 */
} cgp_level_profile;

/* run_result_t scalars (result.hxx:49-66). */
typedef struct {
  int32_t iterations;
  int32_t push_levels;
  int32_t pull_levels;
  int32_t groups;            /* traversal groups the batch was split into         */
  float gpu_time_ms;         /* CUDA-event time of the whole batch incl. init     */
  float wall_time_ms;
  uint64_t frontier_vertices; /* sum over levels of unique frontier sizes         */
  uint64_t frontier_edges;    /* sum over levels of frontier out-degree sums      */
  uint64_t device_status;     /* internal error flags (0 = clean)                 */
  int32_t mask_words;
  int32_t depth_mode;
  uint64_t kernel_launches;   /* kernels this library launched for the call        */
  uint64_t new_pairs;         /* totals of the cgp_level_profile counters          */
  uint64_t pull_vertices;
  uint64_t pull_edges;
  uint64_t sssp_pairs;
  uint64_t sssp_active;
  uint64_t improved;
  uint64_t sssp_pull_vertices;
  uint64_t sssp_pull_edges;
} cgp_stats;

/* Per-kernel-class CUDA-event times of the last cgp_batch_run on this thread
 * that had profile_kernels set. */
typedef struct {
  double ms[12];       /* clear, bfs_push, bfs_pull, sssp_push, level_end, init, output, wcc,
                          sssp_dense, sssp_heavy, sssp_pull */
  int64_t launches[12];
} cgp_kernel_profile;

/* Host CSR (generators and loaders); int64 row offsets. */
typedef struct {
  int64_t num_vertices;
  int64_t num_edges;
  int64_t* row_offsets;
  int32_t* col_indices;
  void* weights;       /* uint32 or float per edge, or NULL */
  int32_t weight_kind; /* CGP_WEIGHT_*                      */
  int32_t reserved;
} cgp_host_csr;

/* -------------------------------------------------------------- errors --- */

/* Copies the calling thread's last error message (NUL-terminated). */
cgp_status cgp_last_error(char* buf, size_t len);
const char* cgp_status_name(cgp_status s);
cgp_status cgp_options_init(cgp_options* opts);
/* Library version string and the device architecture it was built for. */
const char* cgp_version(void);
/* Selects the CUDA device used by this thread's subsequent calls (the
 * device of an execution_context, puercgp/include/puercgp/backend/graph_adapter.hxx:43-97).
 * The library keeps its own runtime state, so a framework's device choice
 * does not carry over. */
cgp_status cgp_set_device(int32_t device);

/* --------------------------------------------------------------- graph --- */

/* Uploads a CSR graph to the current device.  Replaces csr_graph_storage
 * (puercgp/include/puercgp/backend/csr_graph.hxx:42-75) and the device half of
 * load_matrix_market (puercgp/examples/mtx_loader.hxx:178-186).
 * offset_bytes is 4 or 8.  weights may be NULL (unit weights). */
cgp_status cgp_graph_create(const void* row_offsets, int32_t offset_bytes,
                            const int32_t* col_indices, const void* weights,
                            int32_t weight_kind, int64_t num_vertices,
                            int64_t num_edges, int32_t flags, cgp_graph** out);
cgp_status cgp_graph_destroy(cgp_graph* g);
/* get_number_of_vertices/edges (csr_graph.hxx:21-27). */
cgp_status cgp_graph_info(const cgp_graph* g, int64_t* num_vertices,
                          int64_t* num_edges, int32_t* weight_kind,
                          int32_t* symmetric);

/* ----------------------------------------------------------- batch run --- */

/* Runs a batch of queries to convergence and writes one 4-byte value per
 * (query, vertex): int32 depth (BFS, k-hop; CGP_BFS_UNREACHED), uint32 or
 * f32 distance (SSSP; uint32 for unweighted or u32-weighted graphs), uint32
 * label (WCC: minimum vertex id of the weak component).
 * Replaces puercgp::run<Policy> (puercgp/include/puercgp/run.hxx:11-23),
 * run_heterogeneous (puercgp/include/puercgp/engine/hybrid_engine.hxx:1144-1150),
 * gunrock::cgp_bfs::run (cgp/include/gunrock/algorithms/cgp_bfs.hxx:1050-1056)
 * and gunrock::cgp_sssp::run (cgp/include/gunrock/algorithms/cgp_sssp.hxx:973-979).
 * Unlike the reference there is no 64-query limit: batches larger than one
 * group (64 * mask_words queries) run group after group.
 * out: host or device buffer of nq*V 4-byte values in out_layout.
 * out_on_device: 1 if `out` is a device pointer.  stats may be NULL. */
cgp_status cgp_batch_run(cgp_graph* g, const cgp_query* queries, int32_t nq,
                         const cgp_options* opts, void* out, int32_t out_layout,
                         int32_t out_on_device, cgp_stats* stats);

/* Autotuner: times short runs of `sample` (a representative batch) and
 * writes the fastest mask width (mask_words: queries per traversal group),
 * heavy_degree and pull_edge_ratio into *opts, starting from *opts.  The
 * choice is cached on the graph per (traversal mode, batch size, BFS / SSSP
 * / k-hop counts); `reps` runs per candidate (0 = 3).  Replaces the
 * reference's fixed 64-bit masks, degree buckets and pull ratios
 * (puercgp/include/puercgp/core/types.hxx:24,30-31,
 * puercgp/include/puercgp/engine/frontier_engine.hxx:945-946). */
cgp_status cgp_autotune(cgp_graph* g, const cgp_query* sample, int32_t n,
                        cgp_options* opts, int32_t reps);

/* Fault-injection hook for tests (no counterpart in the reference): the
 * after-th next device allocation the library makes (0 = the very next one)
 * fails as if cudaMalloc had run out of memory, after which the hook disarms
 * itself; after < 0 disarms it.  The failing call returns CGP_ERR_OOM and
 * leaves the graph and its cached state usable. */
cgp_status cgp_debug_fail_allocations(int64_t after);

/* Per-level profiles of the last cgp_batch_run on this thread (group 0). */
cgp_status cgp_last_profiles(cgp_level_profile* out, int32_t cap, int32_t* count);
cgp_status cgp_last_kernel_profile(cgp_kernel_profile* out);

/* ----------------------------------------------- operator-level surface --- */

/* The Gunrock problem/enactor shape over one traversal group (<= 1024
 * queries): problem_t::init/reset (cgp/include/gunrock/framework/problem.hxx:48-49),
 * enactor_t::prepare_frontier / loop / is_converged / enact
 * (cgp/include/gunrock/framework/enactor.hxx:243-330). */
cgp_status cgp_enactor_create(cgp_graph* g, const cgp_query* queries, int32_t nq,
                              const cgp_options* opts, cgp_enactor** out);
cgp_status cgp_enactor_destroy(cgp_enactor* e);
/* problem_t::reset + enactor_t::prepare_frontier: clears state, seeds sources. */
cgp_status cgp_enactor_prepare_frontier(cgp_enactor* e);
/* One fused advance+filter level over the query-bitmask frontier
 * (operators::advance::execute_runtime, advance.hxx:244-270, followed by
 * operators::filter::execute_runtime, filter.hxx:187-203, in one pass).
 * direction: CGP_MODE_PUSH / CGP_MODE_PULL / CGP_MODE_HYBRID (decided on the
 * device from the options' ratios).  Returns the next unique frontier size. */
cgp_status cgp_advance_filter_level(cgp_enactor* e, int32_t direction,
                                    int64_t* next_frontier_size);
cgp_status cgp_enactor_is_converged(cgp_enactor* e, int32_t* converged);
/* enactor_t::enact: levels until convergence (device-driven, no per-level sync). */
cgp_status cgp_enactor_enact(cgp_enactor* e, cgp_stats* stats);
/* Copies the current frontier: unique vertex ids and their query masks
 * (mask_words words each).  cap is the capacity in vertices. */
cgp_status cgp_enactor_frontier(cgp_enactor* e, int32_t* vertices,
                                uint64_t* masks, int64_t cap, int64_t* count,
                                int32_t* mask_words);
/* Writes the values of every query of the enactor (layout as cgp_batch_run). */
cgp_status cgp_enactor_read_values(cgp_enactor* e, void* out, int32_t out_layout,
                                   int32_t out_on_device);

/* ------------------------------------------------- allocation-free BFS --- */

/* Size of the fixed device array that cgp_bfs_batch_noalloc works in (held by
 * every GPU that loads the library until the process exits), and its query
 * limit. */
#define CGP_NOALLOC_SCRATCH_BYTES (24u << 20)
#define CGP_NOALLOC_MAX_QUERIES 256

/* Batched BFS that allocates no memory.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc where they need a traversal (a
 * framework that reserved the device memory pool up front, latency paths
 * where cudaMalloc/cudaFree would synchronise the device, hosts that only
 * lend their own buffers).  The caller passes a device CSR (row_offsets of
 * offset_bytes 4 or 8, num_vertices + 1 entries; col_indices, num_edges
 * entries), host `sources` (nq <= 256) and a device output of
 * num_vertices * nq int32 depths, vertex-major out[v*nq + q], INT32_MAX for
 * unreached.  Working state lives in one static device array of
 * CGP_NOALLOC_SCRATCH_BYTES: about 17 KiB plus 36, 60 or 108 bytes per
 * vertex for up to 64, 128 or 256 queries; larger graphs are rejected with
 * CGP_ERR_INVALID_ARG.  symmetric != 0 (the CSR holds both directions)
 * allows pull levels; otherwise every level pushes.  The work is enqueued on
 * `stream` (cudaStream_t, NULL = default stream) of the current device and
 * the call is synchronous: it waits on `stream` between levels and returns
 * when the traversal is done.  Every call looks up the array's device
 * address on the current device.  Calls share the array: calls that overlap
 * on the same device race and must be serialised by the caller. */
cgp_status cgp_bfs_batch_noalloc(const void* row_offsets, int32_t offset_bytes,
                                 const int32_t* col_indices, int64_t num_vertices,
                                 int64_t num_edges, const int32_t* sources, int32_t nq,
                                 int32_t symmetric, int32_t* out, void* stream);

/* --------------------------------------------------------------- serving --- */

/* Continuous-batching server: replaces replenish_frontier_engine
 * (puercgp/include/puercgp/engine/replenish_engine.hxx:42-554) and
 * run_replenish_pipeline (replenish_engine.hxx:559-573).  Requests are
 * admitted into free bitmask slots at level boundaries while others are in
 * flight; state stays resident on the device; finished slots retire at level
 * boundaries and are reused.  `slots` <= 1024.  max_state_bytes bounds the
 * device memory the slot state may take (0 = 80% of free memory); the slot
 * count is reduced to fit. */
cgp_status cgp_server_create(cgp_graph* g, int32_t slots, const cgp_options* opts,
                             int64_t max_state_bytes, cgp_server** out);
cgp_status cgp_server_destroy(cgp_server* s);
/* Queues a request.  out (nullable) receives V 4-byte values on completion;
 * host memory unless out_on_device.  Returns a ticket. */
cgp_status cgp_server_submit(cgp_server* s, const cgp_query* q, void* out,
                             int32_t out_on_device, uint64_t* ticket);

typedef struct {
  int32_t state;             /* 0 queued, 1 running, 2 done, 3 cancelled, 4 failed */
  int32_t slot;
  int32_t admit_level;
  int32_t completion_level;  /* query_result_t::completion_level (result.hxx:13-19) */
  double submit_time_ms;     /* on the server's clock                               */
  double admit_time_ms;
  double finish_time_ms;     /* latency = finish - submit                           */
} cgp_request_info;

cgp_status cgp_server_poll(cgp_server* s, uint64_t ticket, cgp_request_info* info);
/* Blocks until the ticket finishes or timeout_ms passes (CGP_ERR_TIMEOUT). */
cgp_status cgp_server_wait(cgp_server* s, uint64_t ticket, int32_t timeout_ms,
                           cgp_request_info* info);
cgp_status cgp_server_cancel(cgp_server* s, uint64_t ticket);
/* Blocks until every submitted request has finished (or timeout). */
cgp_status cgp_server_drain(cgp_server* s, int32_t timeout_ms);

typedef struct {
  int32_t slots;
  int32_t active_slots;
  int64_t queued;
  int64_t completed;
  int64_t levels;            /* levels run since creation                           */
  double busy_ms;            /* host time spent running levels                       */
  int64_t state_bytes;
  double admit_ms;           /* host time spent admitting requests                   */
  double retire_ms;          /* host time spent retiring slots and copying results   */
  int64_t retire_passes;     /* snapshot-and-reset passes over the vertices          */
  double kernel_ms[12];      /* per kernel class when created with profile_kernels   */
  int64_t sssp_chunk_levels;   /* sum over levels of 32-slot chunks holding SSSP slots */
  int64_t gather_chunk_levels; /* ... of those chunks, the ones whose SSSP slots gathered */
} cgp_server_stats;
cgp_status cgp_server_get_stats(cgp_server* s, cgp_server_stats* st);

/* ---------------------------------------------------- host-side inputs --- */

/* Seeded synthetic graphs (symmetric, deduplicated, no self loops). */
cgp_status cgp_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b,
                        double c, uint64_t seed, int32_t permute, cgp_host_csr* out);
cgp_status cgp_gen_grid(int32_t rows, int32_t cols, double delete_frac,
                        double shortcut_frac, uint64_t seed, cgp_host_csr* out);
cgp_status cgp_gen_chung_lu(int64_t num_vertices, double exponent,
                            double mean_degree, uint64_t seed, cgp_host_csr* out);
cgp_status cgp_gen_weights(cgp_host_csr* g, int32_t kind, double p0, double p1,
                           int32_t lognormal, uint64_t seed);
cgp_status cgp_csr_from_edges(int64_t num_vertices, int64_t num_pairs,
                              const int32_t* src, const int32_t* dst,
                              int32_t symmetrize, cgp_host_csr* out);
/* Seeded sources among vertices with out-degree >= min_degree and, when
 * `allowed` is non-NULL, allowed[v] != 0. */
cgp_status cgp_pick_sources(const cgp_host_csr* g, int32_t count,
                            int32_t min_degree, const uint8_t* allowed,
                            uint64_t seed, int32_t* sources);
/* Matrix Market (mtx_loader.hxx:99-187) and binary CSR directories
 * (csr_vlist.bin / csr_elist.bin / csr_weightlist.bin, mtx_loader.hxx:189-260). */
cgp_status cgp_load_matrix_market(const char* path, cgp_host_csr* out);
cgp_status cgp_load_binary_csr(const char* dir, cgp_host_csr* out);
/* Galois binary graph, version 1 (load_gr, cgp/examples/algorithms/bfs/cgp_bfs.cu:215-260):
 * the topology as the reference reads it (unit weights); read_edge_data != 0
 * keeps 4-byte edge data as uint32 weights. */
cgp_status cgp_load_galois_gr(const char* path, int32_t read_edge_data, cgp_host_csr* out);
void cgp_host_csr_free(cgp_host_csr* g);

#ifdef __cplusplus
}
#endif

#endif /* CGP_B200_H */
